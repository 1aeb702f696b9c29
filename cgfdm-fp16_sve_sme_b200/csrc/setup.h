// Host-side setup of a CGFDM run: everything the reference computes on the
// CPU before propagate() (run.cpp:56-131, propagate.cpp:65-128), redone in
// C++ with the reference's precision and operation order so that the
// coefficient arrays handed to the GPU equal the reference's bit for bit.
#pragma once
#include <cstdint>
#include <string>
#include <vector>

#include "../../include/cgfdm_b200.h"

namespace cgfdm {

// The params.json keys the hot path and its setup read (getParams.cpp:55-242).
struct Params {
  double TMAX = 0, DT = 0, DH = 0;
  int NX = 0, NY = 0, NZ = 0, PX = 1, PY = 1, PZ = 1;
  int centerX = 0, centerY = 0;
  double centerLatitude = 0, centerLongitude = 0;
  int sourceX = 0, sourceY = 0, sourceZ = 0;
  int IT_SKIP = 0;
  int sliceX = 0, sliceY = 0, sliceZ = 0, sliceFreeSurf = 0;
  int nPML = 0;
  int gauss_hill = 0, useTerrain = 0, useMedium = 0, useMultiSource = 0, useSingleSource = 0;
  float rickerfc = 0;
  int ShenModel = 0, Crust_1Medel = 0, LayeredModel = 0;
  std::string LayeredFileName, OUT, sourceFile, sourceDir;
  float Depth = 0;  // km
  // real terrain from SRTM90 tiles (terrain.cpp:217-940)
  int SRTM90 = 0, lonStart = 0, latStart = 0, blockX = 0, blockY = 0;
  std::string TerrainDir;
  // Extensions of this implementation (absent from the reference):
  float mediumPerturbation = 0;  // +-fraction of a seeded uniform Vs/Vp perturbation
  int mediumSeed = 0;
};

struct Setup {
  Params p;
  cgfdm_desc desc{};
  int nx_ = 0, ny_ = 0, nz_ = 0;
  long long num = 0, nsurf = 0;
  std::vector<float> terrain;  // nsurf
  std::vector<float> coord;    // num x 3
  std::vector<float> medium;   // num x 3 (Vs, Vp, rho)
  std::vector<float> cjm;      // 13 x num
  std::vector<float> rdz;      // 2 x nsurf x 9
  std::vector<float> pml;      // profiles
  bool point_src = false;
  int point_xyz[3] = {0, 0, 0};
  std::vector<int64_t> src_index;
  std::vector<float> moment_rate;  // [nt][npts][6], scaled
  int src_nt = 0;
  float src_dt = 0;
  std::vector<int32_t> sta_xyz;     // padded
  std::vector<int32_t> sta_global;  // interior-global, as written to the station file
};

// Reads params.json of run_dir (case-insensitive keys).
int load_params(const std::string &run_dir, Params &p);

// Builds the whole setup; precision selects the storage scaling constants
// (Cv, Cs, Crho of macro.h:65-73 for FP16/BF16).
int build_setup(const std::string &run_dir, int precision, Setup &s);

// Reference output files (station.cpp:382-405, PGV.cpp:103-111,
// data_io.cpp:323-526).
int write_station_file(const Setup &s, const std::string &out_dir, const float *wave);
int write_pgv_file(const Setup &s, const std::string &out_dir, const float *pgv);
int write_slice_file(const std::string &name, char axis, const float *data, size_t n);
int write_model_slices(const Setup &s, const std::string &out_dir);

}  // namespace cgfdm
