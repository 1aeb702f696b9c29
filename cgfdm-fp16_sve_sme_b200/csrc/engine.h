// Device-side simulation state of one handle and its time loop.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <memory>
#include <string>
#include <vector>

#include "../../include/cgfdm_b200.h"

namespace cgfdm {

// Per-thread last error text (cgfdm_last_error).
void set_error(const std::string &msg);
const char *last_error();

class Engine {
 public:
  virtual ~Engine() = default;
  virtual int set_model(const float *cjm, const float *rdz) = 0;
  virtual int set_point_source(int sx, int sy, int sz, float rickerfc) = 0;
  virtual int set_fault_source(const int64_t *idx, const float *rate, int64_t npts, int nt, float dt,
                               bool scaled) = 0;
  virtual int set_stations(const int32_t *xyz, int nsta) = 0;
  virtual int run(int nsteps, void *stream) = 0;
  virtual int stage(int irk, int fb1, int fb2, int fb3, void *stream) = 0;
  virtual int synchronize() = 0;
  virtual int steps_done() const = 0;
  virtual int get_stations(float *wave) = 0;
  virtual int get_station_rows(float *wave, int it0, int it1) = 0;
  virtual int get_pgv(float *pgv) = 0;
  virtual int get_wavefield(float *w) = 0;
  virtual int get_free_surface(float *v3) = 0;
  virtual int get_slice(int field, int axis, int at, double scale, float *out) = 0;
  // Packs an interior slice of field `field` of the step state (times scale)
  // into device memory on the stream of the handle's work, without waiting.
  virtual int enqueue_slice(int field, int axis, int at, double scale, float *dev_out) = 0;
  virtual cudaStream_t work_stream() const = 0;
  virtual int set_state(int irk, const float *W, const float *t, const float *m,
                        const float *aux) = 0;
  virtual int get_state(float *W, float *t, float *m, float *aux) = 0;
  virtual int64_t aux_floats() const = 0;
  virtual int set_timing(bool on) = 0;
  virtual int get_timing(float *ms3) = 0;
  virtual int get_kernel_stats(double *out8) = 0;
  virtual int get_tuning(int32_t *form_chunk) = 0;
  virtual int set_tile_rows(int rows) = 0;
  virtual int set_chunk(int planes) = 0;
  virtual int set_graph(bool on) = 0;
  virtual int inject_fault(int kind) = 0;
  virtual int64_t checkpoint_bytes() const = 0;
  virtual int checkpoint_save(void *buf, int64_t bytes) = 0;
  virtual int checkpoint_load(const void *buf, int64_t bytes) = 0;
  virtual const cgfdm_desc &desc() const = 0;
};

// Several handles of one precision and device advanced together with
// batched streaming launches (see BatchT in engine.cu).
class BatchBase {
 public:
  virtual ~BatchBase() = default;
  virtual int run(int nsteps, void *stream) = 0;
  virtual int set_graph(bool on) = 0;
  virtual int synchronize() = 0;
};

// Creates the engine for desc->precision; returns a status code.
int make_engine(const cgfdm_desc &desc, std::unique_ptr<Engine> &out);
int make_batch(Engine *const *members, int n, std::unique_ptr<BatchBase> &out);
int64_t engine_device_bytes(const cgfdm_desc &desc);

// PML profiles of init_pml_para.cpp:99-234 for a single rank with the free
// surface on top: alpha, beta, d along x, y, z (padded lengths).
std::vector<float> pml_profiles(int nx, int ny, int nz, int npml, float DH);

// Moment of the smoothed point source at stage 0 of step it
// (singleSource.cpp:29-56) and its 7^3 Gaussian weights
// (singleSource.cpp:101-107), both evaluated on the host.
float ricker_moment(float rickerfc, int it, float DT);
void gauss_weights343(float *amp);

}  // namespace cgfdm
