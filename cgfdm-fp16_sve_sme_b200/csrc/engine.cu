// Device state and time loop of one simulation (the body of propagate(),
// propagate.cpp:24-228, on one GPU).
//
// Buffers (each 9 fields of storage type S in the HBM Layout of
// device_common.cuh):
//   A  wavefield at the start of a step; receives the step's result
//   X, Y  RK stage ping-pong buffers
//   T  RK4 accumulator
// Stage mapping: irk0 A->X, irk1 X->Y, irk2 Y->X, irk3 X->A, with the RK
// "m" state read from A (it is the step-start wavefield for stages 0-2, the
// reference's m_W copy, wave_rk.cpp:29).  PML auxiliaries use the same
// four-buffer scheme per slab.
//
// Kernel choice per stage: the TMA-staged streaming kernel updates the
// planes below the three free-surface layers and the exact-order kernel the
// top three layers (KERNEL_STREAM / AUTO); KERNEL_EXACT runs the exact-order
// kernel everywhere (bit-identical to the reference's FP32 CPU build).
#include <cuda_runtime.h>

#include <unistd.h>

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <tuple>
#include <type_traits>
#include <vector>

#include "engine.h"
#include "json.h"
#include "kernels.h"

namespace cgfdm {

namespace {
thread_local std::string g_err;
}
void set_error(const std::string &msg) { g_err = msg; }
const char *last_error() { return g_err.c_str(); }

#define CUDA_TRY(x)                                                                     \
  do {                                                                                  \
    cudaError_t e_ = (x);                                                               \
    if (e_ != cudaSuccess) {                                                            \
      set_error(std::string(#x) + ": " + cudaGetErrorString(e_));                       \
      return e_ == cudaErrorMemoryAllocation ? CGFDM_ERR_NOMEM : CGFDM_ERR_CUDA;        \
    }                                                                                   \
  } while (0)

namespace {

const int kFB[8][3] = {{-1, -1, -1}, {1, 1, -1}, {1, 1, 1},  {-1, -1, 1},
                       {-1, 1, -1},  {1, -1, -1}, {1, -1, 1}, {-1, 1, 1}};

// Autotuner results: streaming-kernel tile height per (precision, nx, ny, nz,
// nPML), shared by every handle of the process.
std::mutex g_tune_mu;
// autotuned (tile form, work-item depth) per (precision, nx, ny, nz, nPML,
// fixed depth or -1, batch member)
struct Tuned {
  int form, chunk;
  bool fast_top;  // free-surface layers on the tiled kernel (else the exact-order kernel)
};
std::map<std::tuple<int, int, int, int, int, int, int>, Tuned> g_tuned;

// Tuning choices kept across processes (optional).  When the environment
// variable CGFDM_TUNE_CACHE names a file, a tuner that has no choice for its
// key in this process looks it up there before timing anything, and every
// choice it times is written back.  The file is a JSON object whose members
// map a key naming the GPU (name and SM count), the precision, the grid, the
// PML width, a fixed work-item depth (or -1) and batch membership to
// [tile form, work-item depth, tiled free-surface kernel 0/1].  A malformed
// file or entry is ignored (the tuner times as if it were absent); writers
// replace the file whole through a rename, so concurrent processes can lose
// each other's new entries but never leave a partial file.  The load and
// the store are called with g_tune_mu held.
std::string tune_cache_path() {
  const char *p = std::getenv("CGFDM_TUNE_CACHE");
  return p && *p ? std::string(p) : std::string();
}
std::string tune_cache_key(int device, const std::tuple<int, int, int, int, int, int, int> &k) {
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) return std::string();
  char buf[512];
  std::snprintf(buf, sizeof buf, "%s|sm%d|precision%d|%dx%dx%d|npml%d|chunk%d|batch%d", prop.name,
                prop.multiProcessorCount, std::get<0>(k), std::get<1>(k), std::get<2>(k),
                std::get<3>(k), std::get<4>(k), std::get<5>(k), std::get<6>(k));
  for (char *c = buf; *c; ++c)
    if (*c == '"' || *c == '\\' || (unsigned char)*c < 0x20) *c = '_';
  return buf;
}
bool tune_cache_load(const std::string &path, const std::string &key, int elem_bytes, Tuned &t) {
  Json doc;
  std::string err;
  if (key.empty() || !Json::parse_file(path, doc, err) || doc.kind != Json::Object) return false;
  for (const auto &m : doc.members) {
    if (m.first != key) continue;
    const Json &v = m.second;
    if (v.kind != Json::Array || v.items.size() != 3) return false;
    for (const Json &x : v.items)
      if (x.kind != Json::Number) return false;
    const int form = v.items[0].as_int(), chunk = v.items[1].as_int(), top = v.items[2].as_int();
    const bool form_ok = form == 16 || form == 8 || (form == kTilePair && elem_bytes == 2);
    if (!form_ok || chunk < 0 || (top != 0 && top != 1)) return false;
    t = {form, chunk, top == 1};
    return true;
  }
  return false;
}
void tune_cache_store(const std::string &path, const std::string &key, const Tuned &t) {
  if (key.empty()) return;
  std::vector<std::pair<std::string, std::string>> entries;  // key, serialised value
  Json doc;
  std::string err;
  if (Json::parse_file(path, doc, err) && doc.kind == Json::Object) {
    for (const auto &m : doc.members) {
      const Json &v = m.second;
      if (m.first == key || v.kind != Json::Array || v.items.size() != 3) continue;
      char val[64];
      std::snprintf(val, sizeof val, "[%d, %d, %d]", v.items[0].as_int(), v.items[1].as_int(),
                    v.items[2].as_int());
      std::string k = m.first;
      for (char &c : k)
        if (c == '"' || c == '\\' || (unsigned char)c < 0x20) c = '_';
      entries.emplace_back(k, val);
    }
  }
  char val[64];
  std::snprintf(val, sizeof val, "[%d, %d, %d]", t.form, t.chunk, t.fast_top ? 1 : 0);
  entries.emplace_back(key, val);
  const std::string tmp = path + ".tmp." + std::to_string((long long)getpid());
  FILE *f = std::fopen(tmp.c_str(), "w");
  if (!f) return;
  std::fprintf(f, "{\n");
  for (size_t e = 0; e < entries.size(); ++e)
    std::fprintf(f, "  \"%s\": %s%s\n", entries[e].first.c_str(), entries[e].second.c_str(),
                 e + 1 < entries.size() ? "," : "");
  std::fprintf(f, "}\n");
  const bool ok = std::fclose(f) == 0;
  if (!ok || std::rename(tmp.c_str(), path.c_str()) != 0) std::remove(tmp.c_str());
}

struct Dims {
  int nx, ny, nz, npml;
  Layout L;
  long long num, nsurf;
  long long slab_pts[5];
  int slab_n[5][3], slab_off[5][3];
};

Dims make_dims(const cgfdm_desc &d) {
  Dims m{};
  m.nx = d.nx; m.ny = d.ny; m.nz = d.nz; m.npml = d.npml;
  m.L = make_layout(d.nx, d.ny, d.nz,
                    d.precision == CGFDM_FP16 || d.precision == CGFDM_BF16 ? 2
                    : d.precision == CGFDM_FP64                            ? 8
                                                                           : 4);
  m.num = (long long)m.L.nx_ * m.L.ny_ * m.L.nz_;
  m.nsurf = (long long)m.L.nx_ * m.L.ny_;
  for (int s = 0; s < 5; ++s) {
    int ax = s % 3, flag = s >= 3;
    int n[3] = {d.nx, d.ny, d.nz};
    int off[3] = {HALO, HALO, HALO};
    int full = n[ax];
    n[ax] = d.npml;
    off[ax] = HALO + flag * (full - d.npml);
    for (int q = 0; q < 3; ++q) { m.slab_n[s][q] = n[q]; m.slab_off[s][q] = off[q]; }
    m.slab_pts[s] = d.npml > 0 ? (long long)n[0] * n[1] * n[2] : 0;
  }
  return m;
}

template <typename S> class BatchT;

template <typename S> class EngineT : public Engine {
  using R = typename Arith<S>::R;
  friend class BatchT<S>;

 public:
  explicit EngineT(const cgfdm_desc &d) : d_(d), g_(make_dims(d)) {}
  ~EngineT() override { release(); }

  int init() {
    CUDA_TRY(cudaSetDevice(d_.device));
    CUDA_TRY(cudaStreamCreateWithFlags(&own_stream_, cudaStreamNonBlocking));
    const size_t wbytes = sizeof(S) * 9 * g_.L.fs;
    for (S **p : {&A_, &X_, &Y_, &T_}) {
      CUDA_TRY(cudaMalloc(p, wbytes));
      CUDA_TRY(cudaMemsetAsync(*p, 0, wbytes, own_stream_));
    }
    CUDA_TRY(cudaMalloc(&cjm_, sizeof(S) * 13 * g_.L.fs));
    CUDA_TRY(cudaMemsetAsync(cjm_, 0, sizeof(S) * 13 * g_.L.fs, own_stream_));
    CUDA_TRY(cudaMalloc(&rdz_, sizeof(R) * 18 * g_.nsurf));
    CUDA_TRY(cudaMemsetAsync(rdz_, 0, sizeof(R) * 18 * g_.nsurf, own_stream_));
    std::vector<float> prof = pml_profiles(g_.nx, g_.ny, g_.nz, g_.npml, d_.dh);
    std::vector<R> profR(prof.begin(), prof.end());
    CUDA_TRY(cudaMalloc(&pml_, sizeof(R) * profR.size()));
    CUDA_TRY(h2d(pml_, profR.data(), sizeof(R) * profR.size()));
    aux_total_ = 0;
    for (int s = 0; s < 5; ++s) aux_total_ += g_.slab_pts[s] * 9;
    if (aux_total_ > 0) {
      CUDA_TRY(cudaMalloc(&aux_, sizeof(R) * 4 * aux_total_));
      CUDA_TRY(cudaMemsetAsync(aux_, 0, sizeof(R) * 4 * aux_total_, own_stream_));
    }
    CUDA_TRY(cudaMalloc(&pgv_, sizeof(float) * 2 * (size_t)g_.nx * g_.ny));
    CUDA_TRY(cudaMemsetAsync(pgv_, 0, sizeof(float) * 2 * (size_t)g_.nx * g_.ny, own_stream_));
    CUDA_TRY(cudaMalloc(&amp343_, sizeof(float) * 343));
    float amp[343];
    gauss_weights343(amp);
    CUDA_TRY(h2d(amp343_, amp, sizeof amp));
    // [0] device error flag of the streaming kernel, [1] its work-queue counter
    CUDA_TRY(cudaMalloc(&err_flag_, 2 * sizeof(int)));
    CUDA_TRY(cudaMemsetAsync(err_flag_, 0, 2 * sizeof(int), own_stream_));
    // the device copy of the step counter it_ (read by the per-step kernels)
    CUDA_TRY(cudaMalloc(&step_, 2 * sizeof(int)));  // the step, the end-of-step block counter
    CUDA_TRY(cudaMemsetAsync(step_, 0, 2 * sizeof(int), own_stream_));
    for (int q = 0; q < 2; ++q) CUDA_TRY(cudaEventCreate(&ev_[q]));
    // opposite PML slabs that overlap (nPML above half the grid, a point in
    // both x1 and x2) are left to the exact-order kernel, which applies every
    // slab of a point; the streaming kernel applies one slab per axis
    const bool overlap = g_.npml > 0 && (2 * g_.npml > g_.nx || 2 * g_.npml > g_.ny);
    // it also addresses a slab's auxiliaries with 32-bit offsets (9 x points < 2^32)
    bool slabs_fit = true;
    for (int s = 0; s < 5; ++s) slabs_fit = slabs_fit && 9 * g_.slab_pts[s] < (1LL << 32);
    use_stream_ = stage_stream_supported<S>() && d_.kernel != CGFDM_KERNEL_EXACT &&
                  g_.nz > 3 && !overlap && slabs_fit;
    if (d_.kernel == CGFDM_KERNEL_STREAM && !stage_stream_supported<S>() ) {
      set_error("the streaming kernel does not support this precision");
      return CGFDM_ERR_ARG;
    }
    if (use_stream_) {
      S *bufs[3] = {A_, X_, Y_};
      for (int b = 0; b < 3; ++b) {
        int rc = encode_stream_maps<S>(bufs[b], cjm_, A_, T_, g_.L, tmap_[b]);
        if (rc) return rc;
      }
    }
    CUDA_TRY(cudaStreamSynchronize(own_stream_));
    return CGFDM_OK;
  }

  int set_model(const float *cjm, const float *rdz) override {
    CUDA_TRY(cudaSetDevice(d_.device));
    int rc = synchronize();  // no stage of this handle may be reading the coefficients
    if (rc) return rc;
    CUDA_TRY(upload_through_accumulator(cjm, cjm_, 13));
    std::vector<R> r(rdz, rdz + 18 * g_.nsurf);
    CUDA_TRY(h2d(rdz_, r.data(), sizeof(R) * r.size()));
    host_cjm_J_.assign(cjm + 9 * g_.num, cjm + 10 * g_.num);
    host_cjm_mu_.assign(cjm + 10 * g_.num, cjm + 11 * g_.num);
    model_set_ = true;
    return CGFDM_OK;
  }

  int set_point_source(int sx, int sy, int sz, float rickerfc) override {
    const Layout &L = g_.L;
    if (sx < HALO || sx >= L.nx_ - HALO || sy < HALO || sy >= L.ny_ - HALO || sz < HALO ||
        sz >= L.nz_ - HALO) {
      point_on_ = false;  // singleSource.cpp:157-164: a source outside the rank is skipped
      drop_graphs();
      return CGFDM_OK;
    }
    if (sx - 3 < 0 || sy - 3 < 0 || sz - 3 < 0 || sx + 3 >= L.nx_ || sy + 3 >= L.ny_ ||
        sz + 3 >= L.nz_) {
      set_error("point source 7^3 smoothing window leaves the padded grid");
      return CGFDM_ERR_SOURCE;
    }
    CUDA_TRY(cudaSetDevice(d_.device));
    // moment of every step (singleSource.cpp:29-56), evaluated on the host
    std::vector<float> tab(d_.nt > 0 ? d_.nt : 1);
    for (int it = 0; it < d_.nt; ++it) tab[it] = ricker_moment(rickerfc, it, d_.dt);
    if (moment_tab_) cudaFree(moment_tab_);
    moment_tab_ = nullptr;
    CUDA_TRY(cudaMalloc(&moment_tab_, sizeof(float) * tab.size()));
    CUDA_TRY(h2d(moment_tab_, tab.data(), sizeof(float) * tab.size()));
    point_on_ = true;
    psrc_[0] = sx; psrc_[1] = sy; psrc_[2] = sz;
    rickerfc_ = rickerfc;
    drop_graphs();
    return CGFDM_OK;
  }

  int set_fault_source(const int64_t *idx, const float *rate, int64_t npts, int nt, float dt,
                       bool scaled) override {
    CUDA_TRY(cudaSetDevice(d_.device));
    free_fault();
    drop_graphs();
    if (npts <= 0) { fault_on_ = false; return CGFDM_OK; }
    const Layout &L = g_.L;
    std::vector<long long> lidx(npts);
    for (int64_t p = 0; p < npts; ++p) {
      if (idx[p] < 0 || idx[p] >= g_.num) {
        set_error("finite-fault cell index out of range");
        return CGFDM_ERR_SOURCE;
      }
      const long long r = idx[p];
      const int i = (int)(r % L.nx_), j = (int)((r / L.nx_) % L.ny_),
                k = (int)(r / ((long long)L.nx_ * L.ny_));
      lidx[p] = L.at(i, j, k);
    }
    std::vector<float> rr(rate, rate + (size_t)npts * nt * 6);
    if (!scaled) {
      if (!model_set_) {
        set_error("set the model before an unscaled fault source");
        return CGFDM_ERR_STATE;
      }
      // calculate_MomentRate (addMoment.cpp:25-48)
      const float DH = d_.dh;
      for (int t = 0; t < nt; ++t)
        for (int64_t p = 0; p < npts; ++p) {
          float jacb = host_cjm_J_[idx[p]], mu = host_cjm_mu_[idx[p]];
          float V = jacb * DH * DH * DH;
          V = (float)(1.0 / V);
          V = (float)(V * SCALE_OF<S>::cv);
          float *m = &rr[((size_t)t * npts + p) * 6];
          for (int q = 0; q < 6; ++q) m[q] *= mu * V;
        }
    }
    CUDA_TRY(cudaMalloc(&fidx_, sizeof(long long) * npts));
    CUDA_TRY(h2d(fidx_, lidx.data(), sizeof(long long) * npts));
    CUDA_TRY(cudaMalloc(&frate_, sizeof(float) * rr.size()));
    CUDA_TRY(h2d(frate_, rr.data(), sizeof(float) * rr.size()));
    // interpolation index and weight of every step (addMoment.cpp:238-264);
    // the source stops for good at the first step with srcIt + 1 >= nt
    const int nts = d_.nt > 0 ? d_.nt : 1;
    std::vector<int> sit(nts, -1);
    std::vector<float> stw(nts, 0.0f);
    for (int it = 0; it < d_.nt; ++it) {
      const float tmpT = (it + 0.0f) * d_.dt;
      const int srcIt = (int)(tmpT / dt);
      if (srcIt + 1 >= nt) break;
      const float t1 = float(srcIt) * dt;
      sit[it] = srcIt;
      stw[it] = (tmpT - t1) / dt;
    }
    CUDA_TRY(cudaMalloc(&fit_tab_, sizeof(int) * nts));
    CUDA_TRY(h2d(fit_tab_, sit.data(), sizeof(int) * nts));
    CUDA_TRY(cudaMalloc(&ftw_tab_, sizeof(float) * nts));
    CUDA_TRY(h2d(ftw_tab_, stw.data(), sizeof(float) * nts));
    fnpts_ = npts;
    fault_on_ = true;
    drop_graphs();
    return CGFDM_OK;
  }

  int set_stations(const int32_t *xyz, int nsta) override {
    CUDA_TRY(cudaSetDevice(d_.device));
    drop_graphs();
    if (sta_xyz_) { cudaFree(sta_xyz_); sta_xyz_ = nullptr; }
    if (sta_wave_) { cudaFree(sta_wave_); sta_wave_ = nullptr; }
    nsta_ = 0;
    if (nsta <= 0) return CGFDM_OK;
    const Layout &L = g_.L;
    for (int s = 0; s < nsta; ++s) {
      const int *q = xyz + 3 * s;
      if (q[0] < HALO || q[0] >= L.nx_ - HALO || q[1] < HALO || q[1] >= L.ny_ - HALO ||
          q[2] < HALO || q[2] >= L.nz_ - HALO) {
        set_error("station outside the interior grid");
        return CGFDM_ERR_ARG;
      }
    }
    CUDA_TRY(cudaMalloc(&sta_xyz_, sizeof(int) * 3 * nsta));
    CUDA_TRY(h2d(sta_xyz_, xyz, sizeof(int) * 3 * nsta));
    const size_t wb = sizeof(float) * (size_t)nsta * d_.nt * 9;
    CUDA_TRY(cudaMalloc(&sta_wave_, wb));
    CUDA_TRY(cudaMemsetAsync(sta_wave_, 0, wb, own_stream_));
    CUDA_TRY(cudaStreamSynchronize(own_stream_));
    nsta_ = nsta;
    return CGFDM_OK;
  }

  int run(int nsteps, void *stream) override {
    CUDA_TRY(cudaSetDevice(d_.device));
    cudaStream_t st = stream ? (cudaStream_t)stream : own_stream_;
    if (it_ + nsteps > d_.nt) {
      set_error("run past the configured number of steps nt");
      return CGFDM_ERR_ARG;
    }
    // work queued earlier on another stream (a batch, another caller) first
    if (last_stream_ && last_stream_ != st) CUDA_TRY(cudaStreamSynchronize(last_stream_));
    last_stream_ = st;
    if (use_stream_ && tile_rows_ == 0) {
      int rc = tune(st);
      if (rc) return rc;
    }
    stage_used_ = 0;
    launches_ = 0;
    stream_bytes_ = 0.0;
    if (timing_) CUDA_TRY(cudaEventRecord(ev_[0], st));
    for (int s = 0; s < nsteps; ++s) {
      const int p = it_ % 8;
      if (use_graph_ && !timing_) {
        // one step is replayed as a CUDA graph per phase it % 8 (the phase
        // fixes the MacCormack signs); the first step of a phase runs
        // eagerly (kernel attributes get set), the second is captured
        if (!gexec_[p] && gseen_[p]) {
          int rc = capture_step(st, gexec_[p]);
          if (rc) return rc;
        }
        if (gexec_[p]) {
          CUDA_TRY(cudaGraphLaunch(gexec_[p], st));
          launches_ += glaunches_[p];
          ++it_;
          continue;
        }
        gseen_[p] = true;
      }
      const int before = launches_;
      int rc = eager_step(st);
      if (rc) return rc;
      glaunches_[p] = launches_ - before;
    }
    if (timing_) CUDA_TRY(cudaEventRecord(ev_[1], st));
    return CGFDM_OK;
  }

  // The pieces of one step: sources into W once before stage 0
  // (propagate.cpp:145-151), then four stages, then stations / PGV and the
  // step counter.  The batch runner calls them member by member.
  int step_sources(cudaStream_t st) {
    if (point_on_) {
      const float DH3 = d_.dh * d_.dh * d_.dh;
      const double CsDT = SCALE_OF<S>::cs * (double)d_.dt;
      CUDA_TRY(launch_point_source<S>(A_, X_, Y_, cjm_, g_.L, psrc_[0], psrc_[1], psrc_[2],
                                      amp343_, moment_tab_, step_, DH3, CsDT, st));
      ++launches_;
    }
    if (fault_on_ && fnpts_ > 0) {
      CUDA_TRY(launch_fault_source<S>(A_, g_.L.fs, fidx_, frate_, fnpts_, fit_tab_, ftw_tab_,
                                      step_, d_.dt, st));
      ++launches_;
    }
    return CGFDM_OK;
  }

  int step_end(cudaStream_t st) {
    const float c1 = (float)(1.0 / SCALE_OF<S>::cv), c2 = (float)(1.0 / SCALE_OF<S>::cs);
    // stations and PGV of the step, and the device step counter's advance
    CUDA_TRY(launch_station_pgv<S>(A_, g_.L, sta_xyz_, nsta_, d_.nt, step_, sta_wave_, pgv_, c1,
                                   c2, 1.0 / SCALE_OF<S>::cv, st));
    launches_ += 1;
    ++it_;
    return CGFDM_OK;
  }

  void step_fb(int irk, int fb[3]) const {
    const int sg = (irk % 2) ? -1 : 1;  // the signs flip after every stage
    for (int q = 0; q < 3; ++q) fb[q] = sg * kFB[it_ % 8][q];
  }

  int eager_step(cudaStream_t st) {
    int rc = step_sources(st);
    for (int irk = 0; irk < 4 && !rc; ++irk) {
      int fb[3];
      step_fb(irk, fb);
      rc = launch_stage(irk, fb, st);
    }
    return rc ? rc : step_end(st);
  }

  int capture_step(cudaStream_t st, cudaGraphExec_t &out) {
    const int it0 = it_, l0 = launches_;
    CUDA_TRY(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    int rc = eager_step(st);
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamEndCapture(st, &g);
    it_ = it0;  // nothing ran: the graph replays the step
    launches_ = l0;
    if (rc) {
      if (g) cudaGraphDestroy(g);
      return rc;
    }
    CUDA_TRY(e);
    e = cudaGraphInstantiate(&out, g, 0);
    cudaGraphDestroy(g);
    CUDA_TRY(e);
    return CGFDM_OK;
  }

  int stage(int irk, int fb1, int fb2, int fb3, void *stream) override {
    CUDA_TRY(cudaSetDevice(d_.device));
    cudaStream_t st = stream ? (cudaStream_t)stream : own_stream_;
    int fb[3] = {fb1, fb2, fb3};
    if (last_stream_ && last_stream_ != st) CUDA_TRY(cudaStreamSynchronize(last_stream_));
    last_stream_ = st;
    return launch_stage(irk, fb, st);
  }

  int synchronize() override {
    CUDA_TRY(cudaSetDevice(d_.device));
    CUDA_TRY(cudaStreamSynchronize(own_stream_));
    if (last_stream_) CUDA_TRY(cudaStreamSynchronize(last_stream_));
    int flag = 0;
    CUDA_TRY(cudaMemcpy(&flag, err_flag_, sizeof(int), cudaMemcpyDeviceToHost));
    if (flag) {
      // reported once; the stage outputs of the failed launch are not valid
      CUDA_TRY(cudaMemset(err_flag_, 0, sizeof(int)));
      set_error("a bounded device-side wait of the streaming kernel expired");
      return CGFDM_ERR_TIMEOUT;
    }
    return CGFDM_OK;
  }

  int inject_fault(int kind) override {
    if (kind != 0 && kind != 1) {
      set_error("unknown fault kind");
      return CGFDM_ERR_ARG;
    }
    drop_next_load_ = kind == 1;
    drop_graphs();
    return CGFDM_OK;
  }

  int steps_done() const override { return it_; }

  int get_stations(float *wave) override {
    int rc = synchronize();
    if (rc) return rc;
    if (nsta_ > 0)
      CUDA_TRY(cudaMemcpy(wave, sta_wave_, sizeof(float) * (size_t)nsta_ * d_.nt * 9,
                          cudaMemcpyDeviceToHost));
    return CGFDM_OK;
  }

  int get_station_rows(float *wave, int it0, int it1) override {
    // rows [it0, it1) of every station into the same places of a host
    // [nsta][nt][9] array (one strided copy)
    int rc = synchronize();
    if (rc) return rc;
    if (nsta_ <= 0 || it1 <= it0) return CGFDM_OK;
    if (it0 < 0 || it1 > d_.nt) {
      set_error("station rows out of range");
      return CGFDM_ERR_ARG;
    }
    const size_t pitch = sizeof(float) * 9 * (size_t)d_.nt;
    CUDA_TRY(cudaMemcpy2D(wave + (size_t)it0 * 9, pitch, sta_wave_ + (size_t)it0 * 9, pitch,
                          sizeof(float) * 9 * (size_t)(it1 - it0), nsta_,
                          cudaMemcpyDeviceToHost));
    return CGFDM_OK;
  }

  int get_pgv(float *pgv) override {
    int rc = synchronize();
    if (rc) return rc;
    CUDA_TRY(cudaMemcpy(pgv, pgv_, sizeof(float) * 2 * (size_t)g_.nx * g_.ny, cudaMemcpyDeviceToHost));
    return CGFDM_OK;
  }

  int get_wavefield(float *w) override { return download_repacked(A_, w, 9); }

  // Checkpoint at a step boundary, raw device contents: a header, the three
  // stage buffers A, X, Y (A is the step state; X and Y keep point-source
  // values in their halo cells), the step-start PML auxiliaries, the PGV map,
  // the seismograms and the step counter.  T and the other auxiliary buffers
  // are rewritten by the next stage 0 before they are read.
  struct CkptHeader {
    char magic[8];
    int32_t precision, nx, ny, nz, npml, nt, nsta, it;
    int64_t wave_bytes, aux_bytes, pgv_bytes, sta_bytes;
  };
  int64_t checkpoint_bytes() const override {
    return (int64_t)sizeof(CkptHeader) + 3 * wave_bytes() + aux_bytes() + pgv_bytes() +
           sta_bytes();
  }
  int checkpoint_save(void *buf, int64_t bytes) override {
    if (bytes < checkpoint_bytes()) {
      set_error("checkpoint buffer too small");
      return CGFDM_ERR_ARG;
    }
    int rc = synchronize();
    if (rc) return rc;
    CkptHeader h = header();
    unsigned char *p = (unsigned char *)buf;
    std::memcpy(p, &h, sizeof h);
    p += sizeof h;
    for (S *w : {A_, X_, Y_}) {
      CUDA_TRY(cudaMemcpy(p, w, wave_bytes(), cudaMemcpyDeviceToHost));
      p += wave_bytes();
    }
    if (aux_bytes()) CUDA_TRY(cudaMemcpy(p, auxbuf(0), aux_bytes(), cudaMemcpyDeviceToHost));
    p += aux_bytes();
    CUDA_TRY(cudaMemcpy(p, pgv_, pgv_bytes(), cudaMemcpyDeviceToHost));
    p += pgv_bytes();
    if (sta_bytes()) CUDA_TRY(cudaMemcpy(p, sta_wave_, sta_bytes(), cudaMemcpyDeviceToHost));
    return CGFDM_OK;
  }
  int checkpoint_load(const void *buf, int64_t bytes) override {
    CUDA_TRY(cudaSetDevice(d_.device));
    CkptHeader h;
    if (bytes < (int64_t)sizeof h) {
      set_error("checkpoint buffer too small");
      return CGFDM_ERR_ARG;
    }
    std::memcpy(&h, buf, sizeof h);
    const CkptHeader mine = header();
    if (std::memcmp(h.magic, mine.magic, 8) || h.precision != mine.precision || h.nx != mine.nx ||
        h.ny != mine.ny || h.nz != mine.nz || h.npml != mine.npml || h.nt != mine.nt ||
        h.nsta != mine.nsta || h.wave_bytes != mine.wave_bytes || h.aux_bytes != mine.aux_bytes ||
        h.it < 0 || h.it > d_.nt || bytes < checkpoint_bytes()) {
      set_error("checkpoint does not match this handle (grid, precision, nt or stations)");
      return CGFDM_ERR_STATE;
    }
    int rc = synchronize();
    if (rc) return rc;
    const unsigned char *p = (const unsigned char *)buf + sizeof h;
    for (S *w : {A_, X_, Y_}) {
      CUDA_TRY(h2d(w, p, wave_bytes()));
      p += wave_bytes();
    }
    if (aux_bytes()) CUDA_TRY(h2d(auxbuf(0), p, aux_bytes()));
    p += aux_bytes();
    CUDA_TRY(h2d(pgv_, p, pgv_bytes()));
    p += pgv_bytes();
    if (sta_bytes()) CUDA_TRY(h2d(sta_wave_, p, sta_bytes()));
    it_ = h.it;
    CUDA_TRY(h2d(step_, &h.it, sizeof(int)));
    drop_graphs();
    return CGFDM_OK;
  }

  int get_free_surface(float *v3) override {
    const size_t n = (size_t)g_.nx * g_.ny;
    for (int v = 0; v < 3; ++v) {
      int rc = get_slice(v, 2, g_.L.nz_ - HALO - 1, 1.0 / SCALE_OF<S>::cv, v3 + v * n);
      if (rc) return rc;
    }
    return CGFDM_OK;
  }

  int enqueue_slice(int field, int axis, int at, double scale, float *dev_out) override {
    CUDA_TRY(launch_slice_pack<S>(A_ + field * g_.L.fs, g_.L, axis, at, scale, dev_out,
                                  work_stream()));
    return CGFDM_OK;
  }

  cudaStream_t work_stream() const override { return last_stream_ ? last_stream_ : own_stream_; }

  int get_slice(int field, int axis, int at, double scale, float *out) override {
    int rc = synchronize();
    if (rc) return rc;
    const size_t n = axis == 0 ? (size_t)g_.ny * g_.nz : axis == 1 ? (size_t)g_.nx * g_.nz
                                                                    : (size_t)g_.nx * g_.ny;
    float *tmp = nullptr;
    CUDA_TRY(cudaMalloc(&tmp, sizeof(float) * n));
    cudaError_t e = launch_slice_pack<S>(A_ + field * g_.L.fs, g_.L, axis, at, scale, tmp, own_stream_);
    if (e == cudaSuccess) e = cudaMemcpyAsync(out, tmp, sizeof(float) * n, cudaMemcpyDeviceToHost, own_stream_);
    if (e == cudaSuccess) e = cudaStreamSynchronize(own_stream_);
    cudaFree(tmp);
    CUDA_TRY(e);
    return CGFDM_OK;
  }

  int set_state(int irk, const float *W, const float *t, const float *m,
                const float *aux) override {
    // Places W in the input buffer of stage irk, m in the step-start buffer A
    // (for irk 0 the stage input is A itself) and t in the accumulator.
    CUDA_TRY(cudaSetDevice(d_.device));
    if (irk < 0 || irk > 3) { set_error("irk must be 0..3"); return CGFDM_ERR_ARG; }
    static const int in_of[4] = {0, 1, 2, 1};
    S *bufs[3] = {A_, X_, Y_};
    if (m && irk != 0) CUDA_TRY(upload_repacked(m, A_, 9));
    if (W) CUDA_TRY(upload_repacked(W, bufs[in_of[irk]], 9));
    if (t) CUDA_TRY(upload_repacked(t, T_, 9));
    if (aux && aux_total_ > 0) {
      // host layout: per slab {Aux, t, m}, each [pos][9]; device: [9][pos]
      std::vector<R> a(aux_total_), tt(aux_total_), mm(aux_total_);
      long long off = 0, dst = 0;
      for (int s = 0; s < 5; ++s) {
        const long long np = g_.slab_pts[s], n = np * 9;
        for (long long p = 0; p < np; ++p)
          for (int v = 0; v < 9; ++v) {
            const long long hq = p * 9 + v, dq = dst + v * np + p;
            a[dq] = aux[off + hq];
            tt[dq] = aux[off + n + hq];
            mm[dq] = aux[off + 2 * n + hq];
          }
        off += 3 * n;
        dst += n;
      }
      if (irk != 0) CUDA_TRY(h2d(auxbuf(0), mm.data(), sizeof(R) * aux_total_));
      CUDA_TRY(h2d(auxbuf(in_of[irk]), a.data(), sizeof(R) * aux_total_));
      CUDA_TRY(h2d(auxbuf(3), tt.data(), sizeof(R) * aux_total_));
    }
    return CGFDM_OK;
  }

  int get_state(float *W, float *t, float *m, float *aux) override {
    int rc = synchronize();
    if (rc) return rc;
    if (W && last_out_) { rc = download_repacked(last_out_, W, 9); if (rc) return rc; }
    if (t) { rc = download_repacked(T_, t, 9); if (rc) return rc; }
    if (m) { rc = download_repacked(A_, m, 9); if (rc) return rc; }
    if (aux && aux_total_ > 0 && last_aux_out_) {
      std::vector<R> o(aux_total_), tt(aux_total_), mm(aux_total_);
      CUDA_TRY(cudaMemcpy(o.data(), last_aux_out_, sizeof(R) * aux_total_, cudaMemcpyDeviceToHost));
      CUDA_TRY(cudaMemcpy(tt.data(), auxbuf(3), sizeof(R) * aux_total_, cudaMemcpyDeviceToHost));
      CUDA_TRY(cudaMemcpy(mm.data(), auxbuf(0), sizeof(R) * aux_total_, cudaMemcpyDeviceToHost));
      long long off = 0, src = 0;
      for (int s = 0; s < 5; ++s) {
        const long long np = g_.slab_pts[s], n = np * 9;
        for (long long p = 0; p < np; ++p)
          for (int v = 0; v < 9; ++v) {
            const long long hq = p * 9 + v, dq = src + v * np + p;
            aux[off + hq] = (float)o[dq];
            aux[off + n + hq] = (float)tt[dq];
            aux[off + 2 * n + hq] = (float)mm[dq];
          }
        off += 3 * n;
        src += n;
      }
    }
    return CGFDM_OK;
  }

  int64_t aux_floats() const override { return aux_total_; }

  int set_timing(bool on) override { timing_ = on; return CGFDM_OK; }

  int set_tile_rows(int rows) override {
    if (rows != 0 && rows != 8 && rows != 16 && !(rows == kTilePair && sizeof(S) == 2)) {
      set_error("tile form must be 0 (autotune), 8 or 16 (32-column tiles of that height), or "
                "64 (paired-point 64 x 8 tiles, FP16 / BF16 storage only)");
      return CGFDM_ERR_ARG;
    }
    tile_rows_ = rows;
    drop_graphs();
    return CGFDM_OK;
  }

  int set_chunk(int planes) override {
    if (planes < 0) {
      set_error("chunk must be 0 (automatic) or a positive number of planes");
      return CGFDM_ERR_ARG;
    }
    chunk_ = planes;
    chunk_fixed_ = planes > 0;
    drop_graphs();
    return CGFDM_OK;
  }

  int set_graph(bool on) override {
    use_graph_ = on;
    drop_graphs();
    return CGFDM_OK;
  }

  int get_timing(float *ms3) override {
    // [0] the last run() end to end, [1] sum over its stage-kernel launches,
    // [2] the number of those launches
    int rc = synchronize();
    if (rc) return rc;
    ms3[0] = ms3[1] = ms3[2] = 0.0f;
    if (!timing_) return CGFDM_OK;
    CUDA_TRY(cudaEventElapsedTime(&ms3[0], ev_[0], ev_[1]));
    double sum = 0;
    for (int q = 0; q < stage_used_; ++q) {
      float ms = 0;
      CUDA_TRY(cudaEventElapsedTime(&ms, stage_ev_[4 * q], stage_ev_[4 * q + 3]));
      sum += ms;
    }
    ms3[1] = (float)sum;
    ms3[2] = (float)stage_used_;
    return CGFDM_OK;
  }

  int get_kernel_stats(double *out) override {
    int rc = synchronize();
    if (rc) return rc;
    for (int q = 0; q < 8; ++q) out[q] = 0.0;
    out[3] = launches_;
    out[7] = use_stream_ ? (tile_rows_ ? tile_rows_ : 16) : 0;
    if (!timing_) return CGFDM_OK;
    double part[3] = {0, 0, 0};
    for (int q = 0; q < stage_used_; ++q)
      for (int p = 0; p < 3; ++p) {
        float ms = 0;
        CUDA_TRY(cudaEventElapsedTime(&ms, stage_ev_[4 * q + p], stage_ev_[4 * q + p + 1]));
        part[p] += ms;
      }
    out[0] = part[0];
    out[1] = use_stream_ ? stage_used_ : 0;
    out[2] = stream_bytes_;
    out[4] = part[1];
    out[5] = part[2];
    out[6] = stage_used_;
    out[7] = use_stream_ ? (tile_rows_ ? tile_rows_ : 16) : 0;
    return CGFDM_OK;
  }

  int get_tuning(int32_t *form_chunk) override {
    form_chunk[0] = use_stream_ ? (tile_rows_ ? tile_rows_ : 16) : 0;
    form_chunk[1] = use_stream_ ? chunk_ : 0;
    form_chunk[2] = use_stream_ && fast_top_ ? 1 : 0;
    return CGFDM_OK;
  }

  const cgfdm_desc &desc() const override { return d_; }

 private:
  R *auxbuf(int b) const { return aux_ + (size_t)b * aux_total_; }
  int64_t wave_bytes() const { return (int64_t)sizeof(S) * 9 * g_.L.fs; }
  int64_t aux_bytes() const { return (int64_t)sizeof(R) * aux_total_; }
  int64_t pgv_bytes() const { return (int64_t)sizeof(float) * 2 * g_.nx * g_.ny; }
  int64_t sta_bytes() const { return (int64_t)sizeof(float) * nsta_ * d_.nt * 9; }
  CkptHeader header() const {
    CkptHeader h{};
    std::memcpy(h.magic, "CGFDMCK1", 8);
    h.precision = d_.precision; h.nx = d_.nx; h.ny = d_.ny; h.nz = d_.nz; h.npml = d_.npml;
    h.nt = d_.nt; h.nsta = nsta_; h.it = it_;
    h.wave_bytes = wave_bytes(); h.aux_bytes = aux_bytes(); h.pgv_bytes = pgv_bytes();
    h.sta_bytes = sta_bytes();
    return h;
  }

  // Host-to-device copy ordered on the handle's stream and complete on
  // return (a plain cudaMemcpy from pageable memory may return before its
  // DMA lands, and the handle's kernels run on a non-blocking stream).
  cudaError_t h2d(void *dst, const void *src, size_t bytes) {
    cudaError_t e = cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, own_stream_);
    return e == cudaSuccess ? cudaStreamSynchronize(own_stream_) : e;
  }

  // Everything stage irk reads and writes (k range left to the caller).
  StageArgs<S> stage_args(int irk, const int fb[3]) const {
    static const int in_of[4] = {0, 1, 2, 1}, out_of[4] = {1, 2, 1, 0};
    S *const bufs[3] = {A_, X_, Y_};
    StageArgs<S> a{};
    a.win = bufs[in_of[irk]];
    a.wout = bufs[out_of[irk]];
    a.wm = A_;
    a.t = T_;
    a.cjm = cjm_;
    a.rdz = rdz_;
    a.pml = pml_;
    a.L = g_.L;
    a.npml = g_.npml;
    a.rDH = (float)(1.0 / d_.dh);
    a.DT = d_.dt;
    a.fb1 = fb[0]; a.fb2 = fb[1]; a.fb3 = fb[2];
    a.irk = irk;
    a.chunk = chunk_;
    a.nslab = g_.npml > 0 ? 5 : 0;
    size_t off = 0;
    for (int s = 0; s < a.nslab; ++s) {
      SlabDev<R> &sl = a.slab[s];
      sl.n0 = g_.slab_n[s][0]; sl.n1 = g_.slab_n[s][1]; sl.n2 = g_.slab_n[s][2];
      sl.off0 = g_.slab_off[s][0]; sl.off1 = g_.slab_off[s][1]; sl.off2 = g_.slab_off[s][2];
      sl.np = g_.slab_pts[s];
      sl.axis = s % 3;
      sl.ain = auxbuf(in_of[irk]) + off;
      sl.aout = auxbuf(out_of[irk]) + off;
      sl.am = auxbuf(0) + off;
      sl.at = auxbuf(3) + off;
      off += g_.slab_pts[s] * 9;
    }
    return a;
  }

  // Picks the streaming kernel's tile form (32 x 16, 32 x 8, and for 16-bit
  // storage the paired-point 64 x 8 form) and work-item depth in z (automatic,
  // 64 or 32 planes; the depth set by cgfdm_set_chunk is kept) for this grid
  // and precision: times the streaming part of stages 0 and 1 at the current
  // step boundary with each candidate and keeps the fastest.  Stage 0 reads
  // only the step state A and step-start auxiliaries and writes X, T and the
  // stage-1 auxiliary inputs; stage 1 reads those and writes Y and T; the
  // real step rewrites all of them before reading them, so the timing leaves
  // the run unchanged.  Results are cached per (precision, grid).
  // batch_form: a batch member, which always runs the 32 x 16 form inside
  // its batch; only the depth is chosen and the member's own form is kept.
  int tune(cudaStream_t st, bool batch_form = false) {
    const auto key = std::make_tuple((int)d_.precision, d_.nx, d_.ny, d_.nz, d_.npml,
                                     chunk_fixed_ ? chunk_ : -1, batch_form ? 1 : 0);
    const std::string cache = tune_cache_path();
    {
      std::lock_guard<std::mutex> lk(g_tune_mu);
      auto f = g_tuned.find(key);
      if (f == g_tuned.end() && !cache.empty()) {
        Tuned t;
        if (tune_cache_load(cache, tune_cache_key(d_.device, key), (int)sizeof(S), t))
          f = g_tuned.emplace(key, t).first;
      }
      if (f != g_tuned.end()) {
        if (!batch_form) {
          tile_rows_ = f->second.form;
          fast_top_ = f->second.fast_top;
        }
        chunk_ = f->second.chunk;
        return CGFDM_OK;
      }
    }
    const int fb0[3] = {kFB[it_ % 8][0], kFB[it_ % 8][1], kFB[it_ % 8][2]};
    const int fb1[3] = {-fb0[0], -fb0[1], -fb0[2]};
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    CUDA_TRY(cudaEventCreate(&e0));
    CUDA_TRY(cudaEventCreate(&e1));
    std::vector<int> forms = {16, 8};
    if (sizeof(S) == 2) forms.push_back(kTilePair);
    if (batch_form) forms = {16};
    std::vector<int> chunks = {0, 64, 32};
    if (chunk_fixed_) chunks = {chunk_};
    int best_form = 16, best_chunk = chunks[0];
    float best_ms = 1e30f;
    cudaError_t err = cudaSuccess;
    for (int rows : forms)
      for (int ch : chunks) {
        StageArgs<S> b0 = stage_args(0, fb0), b1 = stage_args(1, fb1);
        b0.kbeg = b1.kbeg = HALO;
        b0.kend = b1.kend = g_.L.nz_ - HALO - 3;
        b0.chunk = b1.chunk = ch;
        auto pair = [&]() {
          cudaError_t e = launch_stage_stream<S>(b0, tmap_[0], err_flag_, err_flag_ + 1, st,
                                                 nullptr, nullptr, rows);
          if (e == cudaSuccess)
            e = launch_stage_stream<S>(b1, tmap_[1], err_flag_, err_flag_ + 1, st, nullptr,
                                       nullptr, rows);
          return e;
        };
        err = pair();
        if (err == cudaSuccess) err = cudaEventRecord(e0, st);
        for (int r = 0; r < 2 && err == cudaSuccess; ++r) err = pair();
        if (err == cudaSuccess) err = cudaEventRecord(e1, st);
        if (err == cudaSuccess) err = cudaEventSynchronize(e1);
        float ms = 0;
        if (err == cudaSuccess) err = cudaEventElapsedTime(&ms, e0, e1);
        if (err != cudaSuccess) break;
        if (ms < best_ms) {
          best_ms = ms;
          best_form = rows;
          best_chunk = ch;
        }
      }
    // the free-surface layers: the tiled kernel (with the exact-order kernel
    // on the PML-slab columns) against the exact-order kernel alone, on the
    // surface of stage 0 (it writes X and T there, which stage 0 rewrites)
    // (a batch member keeps its own choice, so that it computes the same
    // bits alone and in the batch)
    float surf_ms[2] = {0, 0};
    for (int v = 0; v < 2 && err == cudaSuccess && !batch_form; ++v) {
      fast_top_ = v == 0;
      const StageArgs<S> s0 = stage_args(0, fb0);
      const int l0 = launches_;
      err = launch_surface(s0, st);
      if (err == cudaSuccess) err = cudaEventRecord(e0, st);
      for (int r = 0; r < 2 && err == cudaSuccess; ++r) err = launch_surface(s0, st);
      if (err == cudaSuccess) err = cudaEventRecord(e1, st);
      if (err == cudaSuccess) err = cudaEventSynchronize(e1);
      if (err == cudaSuccess) err = cudaEventElapsedTime(&surf_ms[v], e0, e1);
      launches_ = l0;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    CUDA_TRY(err);
    if (!batch_form) {
      fast_top_ = surf_ms[0] <= surf_ms[1];
      tile_rows_ = best_form;
    }
    chunk_ = best_chunk;
    std::lock_guard<std::mutex> lk(g_tune_mu);
    g_tuned[key] = {best_form, best_chunk, fast_top_};
    if (!cache.empty()) tune_cache_store(cache, tune_cache_key(d_.device, key), g_tuned[key]);
    return CGFDM_OK;
  }

  int launch_stage(int irk, const int fb[3], cudaStream_t st) {
    static const int in_of[4] = {0, 1, 2, 1}, out_of[4] = {1, 2, 1, 0};
    StageArgs<S> a = stage_args(irk, fb);
    last_out_ = a.wout;
    last_aux_out_ = aux_total_ > 0 ? auxbuf(out_of[irk]) : nullptr;
    // events per timed stage: [0] start, [1] after the streaming kernel,
    // [2] before the exact-order kernel, [3] end (after the exact-order kernel)
    cudaEvent_t *ev = nullptr;
    if (timing_) {
      while ((int)stage_ev_.size() < 4 * (stage_used_ + 1)) {
        cudaEvent_t e;
        CUDA_TRY(cudaEventCreate(&e));
        stage_ev_.push_back(e);
      }
      ev = &stage_ev_[4 * stage_used_];
      CUDA_TRY(cudaEventRecord(ev[0], st));
    }
    const int ksurf = g_.L.nz_ - HALO - 3;  // first of the three free-surface layers
    if (use_stream_) {
      StageArgs<S> b = a;
      b.kbeg = HALO;
      b.kend = ksurf;
      b.drop_one_load = drop_next_load_ ? 1 : 0;
      drop_next_load_ = false;
      CUDA_TRY(launch_stage_stream<S>(b, tmap_[in_of[irk]], err_flag_, err_flag_ + 1, st,
                                      ev ? ev[1] : nullptr, &launches_,
                                      tile_rows_ ? tile_rows_ : 16));
      if (ev) CUDA_TRY(cudaEventRecord(ev[2], st));
      // fields read and written per point by this stage: W in, 12 coefficients,
      // W out, plus m (stages 1, 2) and t (written in 0, updated in 1-2, read in 3)
      static const int nfield[4] = {39, 57, 57, 39};
      stream_bytes_ += (double)nfield[irk] * sizeof(S) * (double)(g_.nx) * g_.ny * (ksurf - HALO);
      CUDA_TRY(launch_surface(a, st));
    } else {
      if (ev) {
        CUDA_TRY(cudaEventRecord(ev[1], st));
        CUDA_TRY(cudaEventRecord(ev[2], st));
      }
      a.kbeg = HALO;
      a.kend = g_.L.nz_ - HALO;
      CUDA_TRY(launch_stage_exact<S>(a, st));
      ++launches_;
    }
    if (ev) {
      CUDA_TRY(cudaEventRecord(ev[3], st));
      ++stage_used_;
    }
    return CGFDM_OK;
  }

  // The three free-surface layers of a fast-path stage: the tiled kernel on
  // the columns outside the PML slabs, the exact-order kernel on the slab
  // columns (FP64 runs the exact-order kernel only).
  cudaError_t launch_surface(const StageArgs<S> &a0, cudaStream_t st) {
    StageArgs<S> a = a0;
    a.kbeg = g_.L.nz_ - HALO - 3;
    a.kend = g_.L.nz_ - HALO;
    if constexpr (std::is_same<S, double>::value) {
      ++launches_;
      return launch_stage_exact<S>(a, st);
    } else {
      if (!fast_top_) {
        ++launches_;
        return launch_stage_exact<S>(a, st);
      }
      launches_ += g_.npml > 0 ? 2 : 1;
      return launch_stage_top<S>(a, st);
    }
  }

  // The free-surface layers of stage irk (the streaming part of the stage
  // runs in a batch launch).
  int launch_top(int irk, const int fb[3], cudaStream_t st) {
    static const int out_of[4] = {1, 2, 1, 0};
    StageArgs<S> a = stage_args(irk, fb);
    last_out_ = a.wout;
    last_aux_out_ = aux_total_ > 0 ? auxbuf(out_of[irk]) : nullptr;
    CUDA_TRY(launch_surface(a, st));
    return CGFDM_OK;
  }

  cudaError_t upload_repacked(const float *src, S *dst, int nfield) {
    float *tmp = nullptr;
    const size_t n = (size_t)nfield * g_.num;
    cudaError_t e = cudaMalloc(&tmp, sizeof(float) * n);
    if (e != cudaSuccess) return e;
    e = cudaMemcpyAsync(tmp, src, sizeof(float) * n, cudaMemcpyHostToDevice, own_stream_);
    if (e == cudaSuccess) e = launch_repack_in<S>(tmp, dst, g_.L, nfield, own_stream_);
    if (e == cudaSuccess) e = cudaStreamSynchronize(own_stream_);
    cudaFree(tmp);
    return e;
  }

  // The coefficient upload stages the host fields through the RK accumulator
  // T, a few fields at a time, instead of allocating a staging buffer as
  // large as the model: outside a stage T is free (every stage 0 rewrites it
  // before anything reads it).  T is cleared afterwards.
  cudaError_t upload_through_accumulator(const float *src, S *dst, int nfield) {
    const size_t tbytes = sizeof(S) * 9 * (size_t)g_.L.fs;
    const int per = (int)std::min<size_t>((size_t)nfield, tbytes / (sizeof(float) * (size_t)g_.num));
    if (per < 1) return upload_repacked(src, dst, nfield);
    float *stage = (float *)T_;
    cudaError_t e = cudaSuccess;
    for (int f0 = 0; f0 < nfield && e == cudaSuccess; f0 += per) {
      const int nf = std::min(per, nfield - f0);
      e = cudaMemcpyAsync(stage, src + (size_t)f0 * g_.num, sizeof(float) * nf * (size_t)g_.num,
                          cudaMemcpyHostToDevice, own_stream_);
      if (e == cudaSuccess)
        e = launch_repack_in<S>(stage, dst + (size_t)f0 * g_.L.fs, g_.L, nf, own_stream_);
    }
    if (e == cudaSuccess) e = cudaMemsetAsync(T_, 0, tbytes, own_stream_);
    if (e == cudaSuccess) e = cudaStreamSynchronize(own_stream_);
    return e;
  }

  int download_repacked(const S *src, float *dst, int nfield) {
    int rc = synchronize();
    if (rc) return rc;
    float *tmp = nullptr;
    const size_t n = (size_t)nfield * g_.num;
    CUDA_TRY(cudaMalloc(&tmp, sizeof(float) * n));
    cudaError_t e = launch_repack_out<S>(src, tmp, g_.L, nfield, own_stream_);
    if (e == cudaSuccess) e = cudaMemcpyAsync(dst, tmp, sizeof(float) * n, cudaMemcpyDeviceToHost, own_stream_);
    if (e == cudaSuccess) e = cudaStreamSynchronize(own_stream_);
    cudaFree(tmp);
    CUDA_TRY(e);
    return CGFDM_OK;
  }

  void free_fault() {
    for (void *p : {(void *)fidx_, (void *)frate_, (void *)fit_tab_, (void *)ftw_tab_})
      if (p) cudaFree(p);
    fidx_ = nullptr;
    frate_ = nullptr;
    fit_tab_ = nullptr;
    ftw_tab_ = nullptr;
  }

  void drop_graphs() {
    for (int p = 0; p < 8; ++p) {
      if (gexec_[p]) cudaGraphExecDestroy(gexec_[p]);
      gexec_[p] = nullptr;
      gseen_[p] = false;
    }
  }

  void release() {
    cudaSetDevice(d_.device);
    if (own_stream_) cudaStreamSynchronize(own_stream_);
    if (last_stream_) cudaStreamSynchronize(last_stream_);
    for (void *p : {(void *)A_, (void *)X_, (void *)Y_, (void *)T_, (void *)cjm_, (void *)rdz_,
                    (void *)pml_, (void *)aux_, (void *)pgv_, (void *)amp343_, (void *)sta_xyz_,
                    (void *)sta_wave_, (void *)err_flag_, (void *)step_, (void *)moment_tab_})
      if (p) cudaFree(p);
    free_fault();
    drop_graphs();
    for (auto &e : ev_)
      if (e) cudaEventDestroy(e);
    for (auto &e : stage_ev_) cudaEventDestroy(e);
    if (own_stream_) cudaStreamDestroy(own_stream_);
  }

  cgfdm_desc d_;
  Dims g_;
  cudaStream_t own_stream_ = nullptr, last_stream_ = nullptr;
  S *A_ = nullptr, *X_ = nullptr, *Y_ = nullptr, *T_ = nullptr, *cjm_ = nullptr;
  R *rdz_ = nullptr, *pml_ = nullptr, *aux_ = nullptr;
  long long aux_total_ = 0;
  float *pgv_ = nullptr, *amp343_ = nullptr, *sta_wave_ = nullptr;
  int *sta_xyz_ = nullptr, *err_flag_ = nullptr;
  int nsta_ = 0;
  bool point_on_ = false, fault_on_ = false, model_set_ = false, timing_ = false,
       use_stream_ = false;
  int psrc_[3] = {0, 0, 0};
  float rickerfc_ = 0;
  long long *fidx_ = nullptr;
  float *frate_ = nullptr;
  long long fnpts_ = 0;
  int it_ = 0;
  S *last_out_ = nullptr;
  R *last_aux_out_ = nullptr;
  std::vector<float> host_cjm_J_, host_cjm_mu_;
  alignas(64) unsigned char tmap_[3][kStreamMapsBytes] = {};
  cudaEvent_t ev_[2] = {};
  std::vector<cudaEvent_t> stage_ev_;
  int stage_used_ = 0;
  int launches_ = 0;          // kernels launched by the last run()
  int tile_rows_ = 0;         // streaming-kernel tile height; 0 = autotune at the first run()
  int chunk_ = 0;             // planes per streaming work item in z; 0 = automatic
  bool chunk_fixed_ = false;  // set by set_chunk: the autotuner keeps chunk_
  bool fast_top_ = true;      // free-surface layers: tiled kernel + exact on slab columns
  bool drop_next_load_ = false;  // fault injection for failure-detection tests
  int *step_ = nullptr;       // device copy of it_, then the end-of-step kernel's block counter
  float *moment_tab_ = nullptr;            // point-source moment per step
  int *fit_tab_ = nullptr;                 // fault interpolation index per step (-1: ended)
  float *ftw_tab_ = nullptr;               // fault interpolation weight per step
  bool use_graph_ = false;
  cudaGraphExec_t gexec_[8] = {};          // one step per phase it % 8
  bool gseen_[8] = {};
  int glaunches_[8] = {};                  // kernels in a step of that phase
  double stream_bytes_ = 0;   // algorithmic bytes of its streaming-kernel launches
};

}  // namespace

int64_t engine_device_bytes(const cgfdm_desc &d) {
  Dims g = make_dims(d);
  int64_t s = d.precision == CGFDM_FP32 ? 4 : d.precision == CGFDM_FP64 ? 8 : 2;
  int64_t r = d.precision == CGFDM_FP64 ? 8 : 4;
  int64_t aux = 0;
  for (int q = 0; q < 5; ++q) aux += g.slab_pts[q] * 9;
  return s * (4 * 9 + 13) * g.L.fs + r * (18 * g.nsurf + 4 * aux) + 8 * (int64_t)d.nx * d.ny;
}

namespace {

// Several handles of one precision advanced together: per step, each
// member's sources; per stage, the streaming part of all members in
// persistent launches whose work queue spans them (members grouped by their
// MacCormack signs, which depend on each member's own step), then each
// member's free-surface layers; then stations / PGV.  A step can be
// replayed as a CUDA graph (per phase of the batch's step count mod 8, since
// every member's signs repeat with period 8).
template <typename S> class BatchT : public BatchBase {
 public:
  explicit BatchT(std::vector<EngineT<S> *> m) : m_(std::move(m)) {}
  ~BatchT() override {
    cudaSetDevice(dev_);
    if (own_) cudaStreamSynchronize(own_);
    if (last_) cudaStreamSynchronize(last_);
    for (auto *m : m_)  // the batch's stream goes away with it; its work is done
      if (m->last_stream_ == own_) m->last_stream_ = nullptr;
    drop_graphs();
    if (err_) cudaFree(err_);
    if (own_) cudaStreamDestroy(own_);
  }

  int init() {
    dev_ = m_[0]->d_.device;
    CUDA_TRY(cudaSetDevice(dev_));
    CUDA_TRY(cudaStreamCreateWithFlags(&own_, cudaStreamNonBlocking));
    CUDA_TRY(cudaMalloc(&err_, 2 * sizeof(int)));
    CUDA_TRY(cudaMemsetAsync(err_, 0, 2 * sizeof(int), own_));
    CUDA_TRY(cudaStreamSynchronize(own_));
    return CGFDM_OK;
  }

  int set_graph(bool on) override {
    use_graph_ = on;
    drop_graphs();
    return CGFDM_OK;
  }

  int run(int nsteps, void *stream) override {
    CUDA_TRY(cudaSetDevice(dev_));
    cudaStream_t st = stream ? (cudaStream_t)stream : own_;
    for (auto *m : m_)
      if (m->it_ + nsteps > m->d_.nt) {
        set_error("batch run past a member's configured number of steps nt");
        return CGFDM_ERR_ARG;
      }
    last_ = st;
    for (auto *m : m_) {
      // members' own work (uploads, earlier runs) comes first on this stream
      if (m->last_stream_ && m->last_stream_ != st) CUDA_TRY(cudaStreamSynchronize(m->last_stream_));
      CUDA_TRY(cudaStreamSynchronize(m->own_stream_));
      m->last_stream_ = st;
    }
    if (!tuned_) {
      // every member's work-item depth for the batch's 32 x 16 form
      for (auto *m : m_)
        if (m->use_stream_ && !m->chunk_fixed_) {
          int rc = m->tune(st, true);
          if (rc) return rc;
        }
      tuned_ = true;
    }
    for (int s = 0; s < nsteps; ++s) {
      const int p = count_ % 8;
      if (use_graph_) {
        if (!gexec_[p] && gseen_[p]) {
          int rc = capture_step(st, gexec_[p]);
          if (rc) return rc;
        }
        if (gexec_[p]) {
          CUDA_TRY(cudaGraphLaunch(gexec_[p], st));
          for (auto *m : m_) ++m->it_;
          ++count_;
          continue;
        }
        gseen_[p] = true;
      }
      int rc = eager_step(st);
      if (rc) return rc;
      ++count_;
    }
    return CGFDM_OK;
  }

  int synchronize() override {
    CUDA_TRY(cudaSetDevice(dev_));
    if (last_) CUDA_TRY(cudaStreamSynchronize(last_));
    int flag = 0;
    CUDA_TRY(cudaMemcpy(&flag, err_, sizeof(int), cudaMemcpyDeviceToHost));
    if (flag) {
      set_error("a bounded device-side wait of the streaming kernel expired");
      return CGFDM_ERR_TIMEOUT;
    }
    return CGFDM_OK;
  }

 private:
  int eager_step(cudaStream_t st) {
    static const int in_of[4] = {0, 1, 2, 1};
    for (auto *m : m_) {
      int rc = m->step_sources(st);
      if (rc) return rc;
    }
    std::vector<StageArgs<S>> args;
    std::vector<const void *> maps;
    for (int irk = 0; irk < 4; ++irk) {
      for (int code = 0; code < 8; ++code) {
        args.clear();
        maps.clear();
        for (auto *m : m_) {
          int fb[3];
          m->step_fb(irk, fb);
          if (!m->use_stream_ || (fb[0] > 0) * 4 + (fb[1] > 0) * 2 + (fb[2] > 0) != code) continue;
          StageArgs<S> a = m->stage_args(irk, fb);
          a.kbeg = HALO;
          a.kend = m->g_.L.nz_ - HALO - 3;
          args.push_back(a);
          maps.push_back(m->tmap_[in_of[irk]]);
        }
        if (!args.empty())
          CUDA_TRY(launch_stage_stream_batch<S>(args.data(), maps.data(), (int)args.size(), err_,
                                                err_ + 1, st));
      }
      for (auto *m : m_) {
        int fb[3];
        m->step_fb(irk, fb);
        int rc = m->use_stream_ ? m->launch_top(irk, fb, st) : m->launch_stage(irk, fb, st);
        if (rc) return rc;
      }
    }
    for (auto *m : m_) {
      int rc = m->step_end(st);
      if (rc) return rc;
    }
    return CGFDM_OK;
  }

  int capture_step(cudaStream_t st, cudaGraphExec_t &out) {
    std::vector<int> it0, l0;
    for (auto *m : m_) {
      it0.push_back(m->it_);
      l0.push_back(m->launches_);
    }
    CUDA_TRY(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    int rc = eager_step(st);
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamEndCapture(st, &g);
    for (size_t q = 0; q < m_.size(); ++q) {  // nothing ran: the graph replays the step
      m_[q]->it_ = it0[q];
      m_[q]->launches_ = l0[q];
    }
    if (rc) {
      if (g) cudaGraphDestroy(g);
      return rc;
    }
    CUDA_TRY(e);
    e = cudaGraphInstantiate(&out, g, 0);
    cudaGraphDestroy(g);
    CUDA_TRY(e);
    return CGFDM_OK;
  }

  void drop_graphs() {
    for (int p = 0; p < 8; ++p) {
      if (gexec_[p]) cudaGraphExecDestroy(gexec_[p]);
      gexec_[p] = nullptr;
      gseen_[p] = false;
    }
  }

  std::vector<EngineT<S> *> m_;
  int dev_ = 0;
  cudaStream_t own_ = nullptr, last_ = nullptr;
  int *err_ = nullptr;  // [0] error flag, [1] work counter of the batched launches
  bool use_graph_ = false;
  cudaGraphExec_t gexec_[8] = {};
  bool gseen_[8] = {};
  long long count_ = 0;  // steps run by this batch
  bool tuned_ = false;   // members' work-item depths chosen (first run)
};

template <typename S>
int make_batch_t(Engine *const *members, int n, std::unique_ptr<BatchBase> &out) {
  std::vector<EngineT<S> *> m;
  for (int q = 0; q < n; ++q) {
    auto *e = dynamic_cast<EngineT<S> *>(members[q]);
    if (!e) {
      set_error("batch members must share one precision");
      return CGFDM_ERR_ARG;
    }
    for (auto *o : m)
      if (o == e) {
        set_error("a handle appears twice in the batch");
        return CGFDM_ERR_ARG;
      }
    if (!m.empty() && e->desc().device != m[0]->desc().device) {
      set_error("batch members must share one device");
      return CGFDM_ERR_ARG;
    }
    m.push_back(e);
  }
  auto *b = new BatchT<S>(std::move(m));
  out.reset(b);
  return b->init();
}

}  // namespace

int make_batch(Engine *const *members, int n, std::unique_ptr<BatchBase> &out) {
  if (!members || n <= 0) {
    set_error("empty batch");
    return CGFDM_ERR_ARG;
  }
  switch (members[0]->desc().precision) {
    case CGFDM_FP32: return make_batch_t<float>(members, n, out);
    case CGFDM_FP16: return make_batch_t<__half>(members, n, out);
    case CGFDM_BF16: return make_batch_t<__nv_bfloat16>(members, n, out);
    default: return make_batch_t<double>(members, n, out);
  }
}

int make_engine(const cgfdm_desc &d, std::unique_ptr<Engine> &out) {
  if (d.nx <= 0 || d.ny <= 0 || d.nz <= 0 || d.nt < 0 || !(d.dh > 0) || !(d.dt > 0)) {
    set_error("invalid grid descriptor");
    return CGFDM_ERR_ARG;
  }
  if (d.nz < 4) {
    set_error("nz must be at least 4 (three free-surface layers plus one interior layer)");
    return CGFDM_ERR_ARG;
  }
  if (d.npml < 0 || d.npml > d.nx || d.npml > d.ny || d.npml > d.nz) {
    set_error("the PML layer (nPML) is bigger than the grid");  // pml_deriv.cpp:53-59
    return CGFDM_ERR_PML;
  }
  if (d.npml == 1) {
    set_error("nPML must be 0 or at least 2 (the profile length is DH*(nPML-1))");
    return CGFDM_ERR_PML;
  }
  int dev_count = 0;
  if (cudaGetDeviceCount(&dev_count) != cudaSuccess || dev_count <= d.device || d.device < 0) {
    set_error("no CUDA device available for the CGFDM kernels");
    return CGFDM_ERR_NO_KERNEL;
  }
  int rc = CGFDM_OK;
  switch (d.precision) {
    case CGFDM_FP32: { auto *e = new EngineT<float>(d); out.reset(e); rc = e->init(); } break;
    case CGFDM_FP16: { auto *e = new EngineT<__half>(d); out.reset(e); rc = e->init(); } break;
    case CGFDM_BF16: { auto *e = new EngineT<__nv_bfloat16>(d); out.reset(e); rc = e->init(); } break;
    case CGFDM_FP64: { auto *e = new EngineT<double>(d); out.reset(e); rc = e->init(); } break;
    default:
      set_error("unknown precision");
      return CGFDM_ERR_ARG;
  }
  if (rc) out.reset();
  return rc;
}

}  // namespace cgfdm
