// Host setup of a CGFDM run (see setup.h).  Compiled with -ffp-contract=off;
// float/double mixing follows the reference's declarations line by line.
#include "setup.h"

#include <sys/stat.h>

#include <chrono>
#include <cmath>
#include <cstdlib>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <map>

#include "engine.h"
#include "json.h"

namespace cgfdm {

namespace {

constexpr int H = 3;
constexpr float kPI = 3.141592657f;                  // macro.h:60
constexpr double kDEG2RAD = (double)kPI / 180.0;     // macro.h:63
constexpr float kAm1 = -0.30874f, kA0 = -0.6326f, kA1 = 1.2330f, kA2 = -0.3334f, kA3 = 0.04168f;

std::string join(const std::string &dir, const std::string &f) {
  if (f.empty()) return dir;
  if (f[0] == '/' || dir.empty()) return f;
  return dir + "/" + f;
}

int fail(int code, const std::string &msg) {
  set_error(msg);
  return code;
}

struct Scale {
  double Cv, Cs, Crho;
};
Scale scale_of(int precision) {
  if (precision == CGFDM_FP16 || precision == CGFDM_BF16) return {5.0e3, 1.0e-6, 1e6};
  return {1.0, 1.0, 1.0};
}

// A float as it reads back from the storage format of `precision`
// (round-to-nearest-even, as the reference's FLOAT = __fp16 assignments).
float storage_round(float v, int precision) {
  if (precision == CGFDM_FP16) return (float)(_Float16)v;
  if (precision == CGFDM_BF16) {
    uint32_t u;
    std::memcpy(&u, &v, 4);
    if ((u & 0x7f800000u) != 0x7f800000u) u += 0x7fffu + ((u >> 16) & 1u);
    u &= 0xffff0000u;
    std::memcpy(&v, &u, 4);
  }
  return v;
}

inline long long IDX(const Setup &s, int i, int j, int k) {
  return i + (long long)j * s.nx_ + (long long)k * s.nx_ * s.ny_;
}


// ---------------------------------------------------------------------------
// Real terrain from SRTM90 DEM tiles (terrain.cpp:217-940).
//
// The reference reads blockX x blockY tiles of 6000 x 6000 heights (5 degrees
// each, srtm_<lat>N<lon>E.bin, x fastest), clears invalid elevations,
// replaces the points of steep local gradient by their four-neighbour mean
// and smooths with an 11 x 11 Gaussian inside the model's window, then
// interpolates the DEM onto the grid (plus a 5-point margin) and smooths
// again.  Grid points are mapped to longitude / latitude by PROJ's
// azimuthal equidistant projection about (centerLongitude,
// centerLatitude).  PROJ is not available to this library: the same
// projection is evaluated on a sphere (radius kEarthRadius) with the inverse
// formulas of Snyder (1987), eqs. 20-14 and 20-15.  Everything after the
// projection keeps the reference's arithmetic and order.
constexpr int kDemPointsPerBlock = 6000;  // terrain.cpp:15-16
constexpr int kDemDegreesPerBlock = 5;    // terrain.cpp:12-13
constexpr int kDemExpand = 10;            // callibrateTotalTerrain expandPoint
constexpr double kEarthRadius = 6371008.8;
constexpr double kRAD2DEG = 180.0 / (double)kPI;  // macro.h:62

struct Aeqd {
  double lam0, phi0, sin0, cos0;
  Aeqd(double lon_0, double lat_0) {
    // the centre passes through PROJ's "+lon_0=%lf +lat_0=%lf" string
    char buf[64];
    std::snprintf(buf, sizeof buf, "%lf %lf", lon_0, lat_0);
    double lo = 0, la = 0;
    std::sscanf(buf, "%lf %lf", &lo, &la);
    const double d2r = M_PI / 180.0;
    lam0 = lo * d2r;
    phi0 = la * d2r;
    sin0 = std::sin(phi0);
    cos0 = std::cos(phi0);
  }
  // x, y in metres -> longitude, latitude in radians
  void inverse(double x, double y, double &lam, double &phi) const {
    const double rho = std::sqrt(x * x + y * y);
    if (rho == 0.0) {
      lam = lam0;
      phi = phi0;
      return;
    }
    const double c = rho / kEarthRadius, sc = std::sin(c), cc = std::cos(c);
    phi = std::asin(cc * sin0 + y * sc * cos0 / rho);
    lam = lam0 + std::atan2(x * sc, rho * cos0 * cc - y * sin0 * sc);
  }
};

// GAUSS_FUN (macro.h:39) weights of the 11-point smoothing, nGauss = 5
void dem_gauss(double Dg[11]) {
  const int nGauss = 5;
  const double ra = nGauss * 0.5;
  for (int n = 0; n < 2 * nGauss + 1; ++n) {
    const double t = (n - nGauss) - 0.0;
    Dg[n] = std::exp(-((t / ra) * (t / ra))) / (ra * 1.772453850905516);
  }
}

int build_srtm_terrain(const std::string &dir, Setup &s) {
  const Params &p = s.p;
  if (p.blockX <= 0 || p.blockY <= 0)
    return fail(CGFDM_ERR_PARAMS, "SRTM90 needs blockX >= 1 and blockY >= 1");
  const int totalX = (kDemPointsPerBlock - 1) * p.blockX + 1;
  const int totalY = (kDemPointsPerBlock - 1) * p.blockY + 1;
  const size_t ntot = (size_t)totalX * totalY;
  std::vector<float> T(ntot, 0.0f);
  // readSRTM90 (terrain.cpp:217-307): each tile's last row and column are
  // dropped (shared with the next tile); the DEM's own last ones stay zero
  {
    std::vector<float> tile((size_t)kDemPointsPerBlock * kDemPointsPerBlock);
    const std::string tdir = p.TerrainDir.empty() ? dir : (p.TerrainDir[0] == '/' ? p.TerrainDir
                                                                                 : join(dir, p.TerrainDir));
    for (int bj = 0; bj < p.blockY; ++bj)
      for (int bi = 0; bi < p.blockX; ++bi) {
        const int lat = p.latStart + kDemDegreesPerBlock * bj, lon = p.lonStart + kDemDegreesPerBlock * bi;
        const std::string fn = tdir + "/srtm_" + std::to_string(lat) + "N" + std::to_string(lon) + "E.bin";
        std::ifstream f(fn, std::ios::binary);
        if (!f) return fail(CGFDM_ERR_IO, "missing DEM tile " + fn);
        f.read((char *)tile.data(), sizeof(float) * tile.size());
        if ((size_t)f.gcount() != sizeof(float) * tile.size())
          return fail(CGFDM_ERR_IO, "DEM tile " + fn + " is shorter than 6000 x 6000 floats");
        const int i0 = bi * (kDemPointsPerBlock - 1), j0 = bj * (kDemPointsPerBlock - 1);
        #pragma omp parallel for schedule(static)
        for (int jj = 0; jj < kDemPointsPerBlock - 1; ++jj)
          for (int ii = 0; ii < kDemPointsPerBlock - 1; ++ii)
            T[(size_t)(i0 + ii) + (size_t)(j0 + jj) * totalX] = tile[ii + (size_t)jj * kDemPointsPerBlock];
      }
  }
  // resetTotalTerrain (terrain.cpp:309-325, ERROR_ELEVATION)
  #pragma omp parallel for schedule(static)
  for (long long q = 0; q < (long long)ntot; ++q)
    if (T[q] < -32768 + 1.0 || T[q] > 32768 - 1.0) T[q] = 0.0f;

  const float DH = (float)p.DH;
  const Aeqd proj(p.centerLongitude, p.centerLatitude);
  const double lonStart = p.lonStart, latStart = p.latStart;
  const double deltaLon = double(kDemDegreesPerBlock * p.blockX) / double(totalX);
  const double deltaLat = double(kDemDegreesPerBlock * p.blockY) / double(totalY);
  double Dg[11];
  dem_gauss(Dg);

  // callibrateTotalTerrain (terrain.cpp:328-483): the window of DEM points
  // around the grid's corners (calculateCutLonLatLoc, terrain.cpp:169-213)
  {
    const int I0 = 0, I1 = s.nx_, J0 = 0, J1 = s.ny_;  // frontN = 0 on a single rank
    const double left = (I0 - H) * DH - p.centerX * DH, right = (I1 - H) * DH - p.centerX * DH;
    const double down = (J0 - H) * DH - p.centerY * DH, up = (J1 - H) * DH - p.centerY * DH;
    const double cx[4] = {left, left, right, right}, cy[4] = {down, up, down, up};
    float maxLon = -1000.0, maxLat = -1000.0, minLon = 1000.0, minLat = 1000.0;
    for (int c = 0; c < 4; ++c) {
      double lam, phi;
      proj.inverse(cx[c], cy[c], lam, phi);
      const double Lon = lam * kRAD2DEG, Lat = phi * kRAD2DEG;
      if (maxLon <= Lon) maxLon = Lon;
      if (maxLat <= Lat) maxLat = Lat;
      if (minLon >= Lon) minLon = Lon;
      if (minLat >= Lat) minLat = Lat;
    }
    const int Is = int((minLon - lonStart) / deltaLon) - kDemExpand;
    const int Js = int((minLat - latStart) / deltaLat) - kDemExpand;
    const int Ie = int((maxLon - lonStart) / deltaLon) + kDemExpand;
    const int Je = int((maxLat - latStart) / deltaLat) + kDemExpand;
    if (Is - 6 < 0 || Js - 6 < 0 || Ie + 6 > totalX || Je + 6 > totalY)
      return fail(CGFDM_ERR_PARAMS, "the model area reaches the edge of the DEM tiles");
    std::vector<float> N(T);
    #pragma omp parallel for schedule(static)
    for (int j = Js; j < Je; ++j)
      for (int i = Is; i < Ie; ++i) {
        const size_t q = (size_t)i + (size_t)j * totalX;
        const float a = T[q + 1], b = T[q - 1];
        const float gx = a - b;
        const float c = T[q + totalX], d = T[q - totalX];
        const float gy = c - d;
        const float grad = std::sqrt(gx * gx + gy * gy);
        if (grad > 100.0) N[q] = (a + b + c + d) * 0.25;
      }
    T.swap(N);
    N = T;
    #pragma omp parallel for schedule(static)
    for (int j = Js; j < Je; ++j)
      for (int i = Is; i < Ie; ++i) {
        double sum = 0.0;
        for (int jj = j - 5; jj < j + 6; ++jj)
          for (int ii = i - 5; ii < i + 6; ++ii) {
            const double amp = Dg[ii + 5 - i] * Dg[jj + 5 - j] / 0.996768;
            sum += amp * T[(size_t)ii + (size_t)jj * totalX];
          }
        N[(size_t)i + (size_t)j * totalX] = sum;
      }
    T.swap(N);
  }

  // terrainInterp (terrain.cpp:653-836) over the grid and a 5-point margin
  const int nG = 5, enx = s.nx_ + 2 * nG, eny = s.ny_ + 2 * nG;
  std::vector<float> ex((size_t)enx * eny);
  int bad = 0;
  #pragma omp parallel for schedule(static) reduction(+ : bad)
  for (int j = 0; j < eny; ++j)
    for (int i = 0; i < enx; ++i) {
      const int I = i - nG, J = j - nG;  // frontN = 0
      const double x = (I - H) * DH - p.centerX * DH, y = (J - H) * DH - p.centerY * DH;
      double lam, phi;
      proj.inverse(x, y, lam, phi);
      const double x_ = lam * kRAD2DEG, y_ = phi * kRAD2DEG;
      const int II = int((x_ - lonStart) / deltaLon), JJ = int((y_ - latStart) / deltaLat);
      if (II < 0 || JJ < 0 || II + 1 >= totalX || JJ + 1 >= totalY) {
        ++bad;
        continue;
      }
      const double x1 = II * deltaLon + lonStart, y1 = JJ * deltaLat + latStart;
      const double xs[2] = {x1, x1 + deltaLon}, ys[2] = {y1, y1 + deltaLat};
      // the reference's corner order (terrain.cpp:764-778): z[1] and z[3] are both (I+1, J+1)
      const double z[4] = {T[II + (size_t)JJ * totalX], T[II + 1 + (size_t)(JJ + 1) * totalX],
                           T[II + 1 + (size_t)JJ * totalX], T[II + 1 + (size_t)(JJ + 1) * totalX]};
      // interp2d (terrain.cpp:615-650)
      double Lx[2], Ly[2];
      for (int a = 0; a < 2; ++a) {
        Lx[a] = 1;
        for (int b = 0; b < 2; ++b)
          if (a != b) Lx[a] = Lx[a] * (x_ - xs[b]) / (xs[a] - xs[b]);
      }
      for (int a = 0; a < 2; ++a) {
        Ly[a] = 1;
        for (int b = 0; b < 2; ++b)
          if (a != b) Ly[a] = Ly[a] * (y_ - ys[b]) / (ys[a] - ys[b]);
      }
      double Li = 0.0;
      for (int b = 0; b < 2; ++b)
        for (int a = 0; a < 2; ++a) Li = Li + Lx[a] * Ly[b] * z[a * 2 + b];
      ex[i + (size_t)j * enx] = Li;
    }
  if (bad) return fail(CGFDM_ERR_PARAMS, "grid points fall outside the DEM tiles");
  #pragma omp parallel for schedule(static)
  for (int j = nG; j < eny - nG; ++j)
    for (int i = nG; i < enx - nG; ++i) {
      double sum = 0;
      for (int jj = j - nG; jj < j + nG + 1; ++jj)
        for (int ii = i - nG; ii < i + nG + 1; ++ii) {
          const double amp = Dg[ii + nG - i] * Dg[jj + nG - j] / 0.996768;
          sum += amp * ex[ii + (size_t)jj * enx];
        }
      s.terrain[(i - nG) + (long long)(j - nG) * s.nx_] = sum;
    }
  return CGFDM_OK;
}

// constructCoord (coord.cpp:106-402): flat, Gaussian hill, the SRTM90 DEM
// (preprocessTerrain, terrain.cpp:839-940) or a terrain injected as
// terrain_input.bin, then the stretch of terrain.cpp:917-937.
int build_coord(const std::string &dir, Setup &s) {
  const Params &p = s.p;
  const float DH = (float)p.DH;
  s.coord.assign(3 * s.num, 0.0f);
  s.terrain.assign(s.nsurf, 0.0f);
  const int NZ = p.NZ;
  #pragma omp parallel for schedule(static)
  for (int k = 0; k < s.nz_; ++k)
    for (int j = 0; j < s.ny_; ++j)
      for (int i = 0; i < s.nx_; ++i) {
        long long q = IDX(s, i, j, k) * 3;
        int I = i, J = j, K = k;  // frontN = 0 on a single rank
        if (K == NZ + H - 1) s.terrain[i + (long long)j * s.nx_] = (K - H + 1) * DH - NZ * DH;
        s.coord[q + 0] = (I - H) * DH - p.centerX * DH;
        s.coord[q + 1] = (J - H) * DH - p.centerY * DH;
        s.coord[q + 2] = (K - H + 1) * DH - NZ * DH;
      }
  const float cal_depth = p.Depth * 1000;
  if (p.gauss_hill) {
    // construct_gauss_hill_surface (coord.cpp:146-186) + construct_terrain_coord (256-307)
    float h = 0.2 * cal_depth;
    float a = 0.1 * cal_depth, b = 0.1 * cal_depth;
    for (int j = 0; j < s.ny_; ++j)
      for (int i = 0; i < s.nx_; ++i) {
        float x = (i - H) * DH - p.centerX * DH;
        float y = (j - H) * DH - p.centerY * DH;
        float height = h * std::exp(-0.5f * (x * x / (a * a) + y * y / (b * b)));
        s.terrain[i + (long long)j * s.nx_] = height;
      }
    #pragma omp parallel for schedule(static)
    for (int k = 0; k < s.nz_; ++k)
      for (int j = 0; j < s.ny_; ++j)
        for (int i = 0; i < s.nx_; ++i) {
          long long q = IDX(s, i, j, k);
          int K = k - H;
          float height = s.terrain[i + (long long)j * s.nx_];
          float DZ = double(height + std::abs(cal_depth)) / double(NZ - 1);
          s.coord[q * 3 + 2] = -std::abs(cal_depth) + DZ * K;
        }
  }
  if (p.useTerrain) {
    if (p.SRTM90 == 1) {
      int rc = build_srtm_terrain(dir, s);
      if (rc) return rc;
    } else {
      const int NXP = p.NX + 2 * H, NYP = p.NY + 2 * H;
      std::ifstream f(join(dir, "terrain_input.bin"), std::ios::binary);
      if (!f) return fail(CGFDM_ERR_IO, "useTerrain is set but terrain_input.bin is missing");
      std::vector<float> g((size_t)NXP * NYP);
      f.read((char *)g.data(), sizeof(float) * g.size());
      if ((size_t)f.gcount() != sizeof(float) * g.size())
        return fail(CGFDM_ERR_IO, "terrain_input.bin is shorter than (NX+6)*(NY+6) floats");
      for (int j = 0; j < s.ny_; ++j)
        for (int i = 0; i < s.nx_; ++i) s.terrain[i + (long long)j * s.nx_] = g[i + (size_t)j * NXP];
    }
    double Depth = p.Depth * 1e3;
    #pragma omp parallel for schedule(static)
    for (int k = 0; k < s.nz_; ++k)
      for (int j = 0; j < s.ny_; ++j)
        for (int i = 0; i < s.nx_; ++i) {
          long long q = IDX(s, i, j, k) * 3;
          int K = k - H;
          double DZ = double(s.terrain[i + (long long)j * s.nx_] + std::abs(Depth)) / double(NZ - 1);
          s.coord[q + 2] = -std::abs(Depth) + DZ * K;
        }
  }
  return CGFDM_OK;
}

uint64_t splitmix(uint64_t &x) {
  uint64_t z = (x += 0x9E3779B97F4A7C15ull);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

// constructMedium (medium.cpp:256-326): homogeneous, then the layered model
// (generate_1D_medium, medium.cpp:84-216, LayeredStructureTerrain).
int build_medium(const std::string &dir, Setup &s) {
  const Params &p = s.p;
  s.medium.assign(3 * s.num, 0.0f);
  #pragma omp parallel for schedule(static)
  for (long long q = 0; q < s.num; ++q) {
    s.medium[3 * q + 0] = 3464.0f;
    s.medium[3 * q + 1] = 6000.0f;
    s.medium[3 * q + 2] = 2670.0f;
  }
  if (!p.useMedium) return CGFDM_OK;
  if (p.ShenModel || p.Crust_1Medel)
    if (!p.LayeredModel)
      return fail(CGFDM_ERR_PARAMS, "the Shen / CRUST1.0 crust models are not supported");
  if (p.LayeredModel) {
    std::ifstream f(join(dir, p.LayeredFileName), std::ios::binary);
    if (!f) return fail(CGFDM_ERR_IO, "cannot open layered model " + p.LayeredFileName);
    int layers = 0;
    f.read((char *)&layers, 4);
    if (!f || layers < 0 || layers > 100000) return fail(CGFDM_ERR_IO, "bad layered model header");
    std::vector<float> hd(layers), vs(layers), vp(layers), rho(layers);
    for (int F = 0; F < layers; ++F) {
      float row[4];
      f.read((char *)row, sizeof row);
      if (!f) return fail(CGFDM_ERR_IO, "layered model file is truncated");
      hd[F] = row[0] * 1000.0f;
      if (F != 0) hd[F] += 0.0f;
      vs[F] = row[1] * 1000.f;
      vp[F] = row[2] * 1000.f;
      rho[F] = row[3] * 1000.f;
    }
    const float tolerance = 1.0f;
    #pragma omp parallel for schedule(static)
    for (int k = 0; k < s.nz_; ++k)
      for (int j = 0; j < s.ny_; ++j)
        for (int i = 0; i < s.nx_; ++i) {
          long long q = IDX(s, i, j, k);
          double terrain = s.terrain[i + (long long)j * s.nx_];
          float coordz = s.coord[q * 3 + 2];
          for (int F = 1; F < layers; ++F) {
            float h0 = -hd[0] + terrain;
            float h1 = -hd[F - 1] + terrain;
            float h2 = -hd[F] + terrain;
            // the three tests run in sequence; the last true one wins
            auto set = [&](int L) {
              s.medium[3 * q] = vs[L];
              s.medium[3 * q + 1] = vp[L];
              s.medium[3 * q + 2] = rho[L];
            };
            if (coordz > (h0 - tolerance)) set(0);
            if ((h1 - tolerance) > coordz && coordz > (h2 - tolerance)) set(F - 1);
            if ((h2 - tolerance) > coordz) set(F);
          }
        }
  }
  if (p.mediumPerturbation != 0.0f) {
    // Extension: seeded uniform +-fraction perturbation of Vs and Vp per cell.
    const uint64_t seed = 0x5EEDull ^ (uint64_t)(uint32_t)p.mediumSeed;
    #pragma omp parallel for schedule(static)
    for (long long q = 0; q < s.num; ++q) {
      uint64_t st = seed + (uint64_t)q * 0xD1B54A32D192ED03ull;
      double u = (splitmix(st) >> 11) * (1.0 / 9007199254740992.0);
      float f = (float)(1.0 + p.mediumPerturbation * (2.0 * u - 1.0));
      s.medium[3 * q] *= f;
      s.medium[3 * q + 1] *= f;
    }
  }
  return CGFDM_OK;
}

double distance_point2plane(const double P[3], const double A[3], const double B[3],
                            const double C[3]) {
  double AB[3] = {B[0] - A[0], B[1] - A[1], B[2] - A[2]};
  double AC[3] = {C[0] - A[0], C[1] - A[1], C[2] - A[2]};
  double n[3] = {AB[1] * AC[2] - AB[2] * AC[1], AB[2] * AC[0] - AB[0] * AC[2],
                 AB[0] * AC[1] - AB[1] * AC[0]};
  double PA[3] = {P[0] - A[0], P[1] - A[1], P[2] - A[2]};
  double nd = std::sqrt(n[0] * n[0] + n[1] * n[1] + n[2] * n[2]);
  n[0] = n[0] / nd;
  n[1] = n[1] / nd;
  n[2] = n[2] / nd;
  return std::abs(PA[0] * n[0] + PA[1] * n[1] + PA[2] * n[2]);
}

// calc_CFL (calc_CFL.cpp:265-363): smallest cell height against Vp max.
int check_cfl(const Setup &s) {
  double hmin = 1.0e20;
  #pragma omp parallel for schedule(dynamic, 1) reduction(min : hmin)
  for (int k = H; k < s.nz_ - H; ++k)
    for (int j = H; j < s.ny_ - H; ++j)
      for (int i = H; i < s.nx_ - H; ++i) {
        const float *c = &s.coord[IDX(s, i, j, k) * 3];
        double P[3] = {c[0], c[1], c[2]}, A[3], B[3], C[3];
        for (int ii = -1; ii <= 1; ii += 2)
          for (int jj = -1; jj <= 1; jj += 2)
            for (int kk = -1; kk <= 1; kk += 2) {
              const float *a = &s.coord[IDX(s, i - ii, j, k) * 3];
              const float *b = &s.coord[IDX(s, i, j - jj, k) * 3];
              const float *cc = &s.coord[IDX(s, i, j, k - kk) * 3];
              for (int q = 0; q < 3; ++q) { A[q] = a[q]; B[q] = b[q]; C[q] = cc[q]; }
              double d = distance_point2plane(P, A, B, C);
              hmin = hmin < d ? hmin : d;
            }
      }
  float H_min = (float)hmin;
  float vpmax = -1.0e20f;
  #pragma omp parallel for reduction(max : vpmax)
  for (long long q = 0; q < s.num; ++q)
    if (s.medium[3 * q + 1] > vpmax) vpmax = s.medium[3 * q + 1];
  float dtmax = 1.34 * H_min / vpmax;
  if (s.p.DT > dtmax) {
    char buf[160];
    std::snprintf(buf, sizeof buf, "DT = %g exceeds the CFL limit %g (1.34 Hmin / Vpmax)", s.p.DT,
                  (double)dtmax);
    return fail(CGFDM_ERR_CFL, buf);
  }
  return CGFDM_OK;
}

// constructCJM (CJM.cpp:170-236): medium conversion, metrics and Jacobian
// with the MacCormack operators (contravariant.cpp:72-171), free-surface
// matrices and the mirror above the surface (contravariant.cpp:209-412).
void build_cjm(Setup &s, const Scale &sc) {
  const long long num = s.num;
  std::vector<float> med = s.medium;  // converted copy
  const double c = 1.0 * sc.Cs / sc.Cv;
  #pragma omp parallel for schedule(static)
  for (long long q = 0; q < num; ++q) {
    float Vs = med[3 * q], Vp = med[3 * q + 1];
    float rho = med[3 * q + 2] * c;
    med[3 * q + 0] = rho * (Vs * Vs);
    med[3 * q + 1] = rho * (Vp * Vp - 2.0f * Vs * Vs);
    med[3 * q + 2] = 1.0f / rho / sc.Crho;
  }
  std::vector<float> con(9 * num, 0.0f), Jac(num, 0.0f);
  const float DH = (float)s.p.DH;
  const float rDH = 1.0 / DH;
  const long long st[3] = {1, s.nx_, (long long)s.nx_ * s.ny_};
  const float *C = s.coord.data();
  auto LC = [&](long long idx, int var, int fb, int ax) -> float {
    long long o = fb * st[ax];
    return fb *
           (kAm1 * C[(idx - o) * 3 + var] + kA0 * C[idx * 3 + var] + kA1 * C[(idx + o) * 3 + var] +
            kA2 * C[(idx + 2 * o) * 3 + var] + kA3 * C[(idx + 3 * o) * 3 + var]) *
           rDH;
  };
  #pragma omp parallel for schedule(dynamic, 1)
  for (int k = H; k < s.nz_ - H; ++k)
    for (int j = H; j < s.ny_ - H; ++j)
      for (int i = H; i < s.nx_ - H; ++i) {
        long long idx = IDX(s, i, j, k);
        float x_xi = 0.5f * (LC(idx, 0, 1, 0) + LC(idx, 0, -1, 0));
        float x_et = 0.5f * (LC(idx, 0, 1, 1) + LC(idx, 0, -1, 1));
        float x_zt = 0.5f * (LC(idx, 0, 1, 2) + LC(idx, 0, -1, 2));
        float y_xi = 0.5f * (LC(idx, 1, 1, 0) + LC(idx, 1, -1, 0));
        float y_et = 0.5f * (LC(idx, 1, 1, 1) + LC(idx, 1, -1, 1));
        float y_zt = 0.5f * (LC(idx, 1, 1, 2) + LC(idx, 1, -1, 2));
        float z_xi = 0.5f * (LC(idx, 2, 1, 0) + LC(idx, 2, -1, 0));
        float z_et = 0.5f * (LC(idx, 2, 1, 1) + LC(idx, 2, -1, 1));
        float z_zt = 0.5f * (LC(idx, 2, 1, 2) + LC(idx, 2, -1, 2));
        float J = x_xi * y_et * z_zt + x_et * y_zt * z_xi + x_zt * y_xi * z_et -
                  x_zt * y_et * z_xi - x_et * y_xi * z_zt - x_xi * z_et * y_zt;
        Jac[idx] = J;
        float Ji = 1.0f / J;
        float *m = &con[9 * idx];
        m[0] = (y_et * z_zt - y_zt * z_et) * Ji;
        m[1] = (x_zt * z_et - x_et * z_zt) * Ji;
        m[2] = (x_et * y_zt - x_zt * y_et) * Ji;
        m[3] = (y_zt * z_xi - y_xi * z_zt) * Ji;
        m[4] = (x_xi * z_zt - x_zt * z_xi) * Ji;
        m[5] = (x_zt * y_xi - x_xi * y_zt) * Ji;
        m[6] = (y_xi * z_et - y_et * z_xi) * Ji;
        m[7] = (x_et * z_xi - x_xi * z_et) * Ji;
        m[8] = (x_xi * y_et - x_et * y_xi) * Ji;
      }
  // free surface (FREE_SURFACE build): k = _nz - 1 and the mirrored layers above
  s.rdz.assign(18 * s.nsurf, 0.0f);
  const int ktop = s.nz_ - H - 1;
  float *DXo = s.rdz.data(), *DYo = s.rdz.data() + 9 * s.nsurf;
  #pragma omp parallel for schedule(static)
  for (int k = ktop; k < s.nz_; ++k)
    for (int j = H; j < s.ny_ - H; ++j)
      for (int i = H; i < s.nx_ - H; ++i) {
        long long idx = IDX(s, i, j, k);
        if (k == ktop) {
          const float *m = &con[9 * idx];
          float xi_x = m[0], xi_y = m[1], xi_z = m[2], et_x = m[3], et_y = m[4], et_z = m[5],
                zt_x = m[6], zt_y = m[7], zt_z = m[8];
          long long sidx = i + (long long)j * s.nx_;
          float mu = med[3 * idx], lambda = med[3 * idx + 1];
          float chi = 2.0f * lambda + mu;
          float lam_mu = lambda + mu;
          float DZ[9], DX[9], DY[9], rDZ[9];
          DZ[0] = chi * zt_x * zt_x + mu * (zt_y * zt_y + zt_z * zt_z);
          DZ[1] = lam_mu * zt_x * zt_y;
          DZ[2] = lam_mu * zt_x * zt_z;
          DZ[3] = DZ[1];
          DZ[4] = chi * zt_y * zt_y + mu * (zt_x * zt_x + zt_z * zt_z);
          DZ[5] = lam_mu * zt_y * zt_z;
          DZ[6] = DZ[2];
          DZ[7] = DZ[5];
          DZ[8] = chi * zt_z * zt_z + mu * (zt_x * zt_x + zt_y * zt_y);
          float det = DZ[0] * DZ[4] * DZ[8] + DZ[1] * DZ[5] * DZ[6] + DZ[2] * DZ[7] * DZ[3] -
                      DZ[2] * DZ[4] * DZ[6] - DZ[1] * DZ[3] * DZ[8] - DZ[0] * DZ[7] * DZ[5];
          DX[0] = chi * zt_x * xi_x + mu * (zt_y * xi_y + zt_z * xi_z);
          DX[1] = lambda * zt_x * xi_y + mu * zt_y * xi_x;
          DX[2] = lambda * zt_x * xi_z + mu * zt_z * xi_x;
          DX[3] = lambda * zt_y * xi_x + mu * zt_x * xi_y;
          DX[4] = chi * zt_y * xi_y + mu * (zt_x * xi_x + zt_z * xi_z);
          DX[5] = lambda * zt_y * xi_z + mu * zt_z * xi_y;
          DX[6] = lambda * zt_z * xi_x + mu * zt_x * xi_z;
          DX[7] = lambda * zt_z * xi_y + mu * zt_y * xi_z;
          DX[8] = chi * zt_z * xi_z + mu * (zt_x * xi_x + zt_y * xi_y);
          DY[0] = chi * zt_x * et_x + mu * (zt_y * et_y + zt_z * et_z);
          DY[1] = lambda * zt_x * et_y + mu * zt_y * et_x;
          DY[2] = lambda * zt_x * et_z + mu * zt_z * et_x;
          DY[3] = lambda * zt_y * et_x + mu * zt_x * et_y;
          DY[4] = chi * zt_y * et_y + mu * (zt_x * et_x + zt_z * et_z);
          DY[5] = lambda * zt_y * et_z + mu * zt_z * et_y;
          DY[6] = lambda * zt_z * et_x + mu * zt_x * et_z;
          DY[7] = lambda * zt_z * et_y + mu * zt_y * et_z;
          DY[8] = chi * zt_z * et_z + mu * (zt_x * et_x + zt_y * et_y);
          rDZ[0] = (DZ[4] * DZ[8] - DZ[5] * DZ[7]) / det;
          rDZ[1] = (-DZ[3] * DZ[8] + DZ[5] * DZ[6]) / det;
          rDZ[2] = (DZ[3] * DZ[7] - DZ[4] * DZ[6]) / det;
          rDZ[3] = (-DZ[1] * DZ[8] + DZ[2] * DZ[7]) / det;
          rDZ[4] = (DZ[0] * DZ[8] - DZ[2] * DZ[6]) / det;
          rDZ[5] = (-DZ[0] * DZ[7] + DZ[1] * DZ[6]) / det;
          rDZ[6] = (DZ[1] * DZ[5] - DZ[2] * DZ[4]) / det;
          rDZ[7] = (-DZ[0] * DZ[5] + DZ[2] * DZ[3]) / det;
          rDZ[8] = (DZ[0] * DZ[4] - DZ[1] * DZ[3]) / det;
          for (int r = 0; r < 3; ++r)
            for (int cc = 0; cc < 3; ++cc) {
              DXo[sidx * 9 + 3 * r + cc] =
                  -(rDZ[3 * r] * DX[cc] + rDZ[3 * r + 1] * DX[3 + cc] + rDZ[3 * r + 2] * DX[6 + cc]);
              DYo[sidx * 9 + 3 * r + cc] =
                  -(rDZ[3 * r] * DY[cc] + rDZ[3 * r + 1] * DY[3 + cc] + rDZ[3 * r + 2] * DY[6 + cc]);
            }
        } else {
          long long pos = IDX(s, i, j, 2 * ktop - k);
          Jac[idx] = Jac[pos];
          for (int q = 0; q < 9; ++q) con[9 * idx + q] = con[9 * pos + q];
        }
      }
  s.cjm.assign(13 * num, 0.0f);  // set_CJM (CJM.cpp:106-134)
  #pragma omp parallel for schedule(static)
  for (long long q = 0; q < num; ++q) {
    for (int v = 0; v < 9; ++v) s.cjm[q + num * v] = con[9 * q + v];
    s.cjm[q + num * 9] = Jac[q];
    s.cjm[q + num * 10] = med[3 * q];
    s.cjm[q + num * 11] = med[3 * q + 1];
    s.cjm[q + num * 12] = med[3 * q + 2];
  }
}

// init_MultiSource (multiSource.cpp:824-923) without a map projection: the
// file's lon/lat fields are read as metres from the grid centre.
int build_fault(const std::string &dir, Setup &s, const Scale &sc) {
  const Params &p = s.p;
  const std::string fn = join(join(dir, p.sourceDir), p.sourceFile);
  std::ifstream f(fn, std::ios::binary);
  if (!f) return fail(CGFDM_ERR_SOURCE, "cannot open source file " + fn);
  int npts = 0, nt = 0;
  float dt = 0;
  f.read((char *)&npts, 4);
  f.read((char *)&nt, 4);
  f.read((char *)&dt, 4);
  if (!f || npts < 0 || nt < 0) return fail(CGFDM_ERR_SOURCE, "bad source file header");
  const long long rec = 6 * 4 + 2LL * 4 * nt;
  std::vector<float> x(npts), y(npts), z(npts);
  for (int q = 0; q < npts; ++q) {
    f.seekg(12 + rec * q);
    float v[3];
    f.read((char *)v, sizeof v);
    if (!f) return fail(CGFDM_ERR_SOURCE, "source file is truncated");
    x[q] = v[0]; y[q] = v[1]; z[q] = v[2];
  }
  // srcCoord2Index (multiSource.cpp:174-323, NO_SOURCE_SMOOTH)
  const float DH = (float)p.DH;
  const float Depth = p.Depth * 1000;
  float maxz = -Depth;
  for (int q = 0; q < npts; ++q)
    if (maxz < z[q]) maxz = z[q];
  for (int q = 0; q < npts; ++q) z[q] = z[q] - maxz;
  std::map<long long, long long> point_index;
  const int nxl = s.nx_ - H, nyl = s.ny_ - H, nzl = s.nz_ - H;
  for (int q = 0; q < npts; ++q) {
    int sx = int(x[q] / DH + 0.5) + p.centerX + H;
    int sy = int(y[q] / DH + 0.5) + p.centerY + H;
    if (sx >= H && sx < nxl && sy >= H && sy < nyl) {
      for (int k = H; k < nzl; ++k) {
        long long i1 = IDX(s, sx, sy, k - 1), i2 = IDX(s, sx, sy, k + 1), i0 = IDX(s, sx, sy, k);
        double dz1 = (s.coord[i0 * 3 + 2] - s.coord[i1 * 3 + 2]) * 0.5;
        double dz2 = (s.coord[i2 * 3 + 2] - s.coord[i0 * 3 + 2]) * 0.5;
        if (s.coord[i0 * 3 + 2] - dz1 <= z[q] && z[q] < dz2 + s.coord[i0 * 3 + 2])
          point_index[q] = i0;
      }
    }
  }
  // readSourceParams + solveMomentRate (multiSource.cpp:362-561): the
  // records are read in order, then every (point, sample) is solved
  // independently, in parallel
  const long long pn = (long long)point_index.size();
  std::vector<float> mr((size_t)pn * nt * 6, 0.0f);
  std::vector<float> asd_all((size_t)pn * 3), rake_all((size_t)pn * nt), rate_all((size_t)pn * nt);
  {
    long long row = 0;
    for (auto &kv : point_index) {
      f.seekg(12 + rec * kv.first + 3 * 4);
      f.read((char *)&asd_all[row * 3], 3 * sizeof(float));
      f.read((char *)&rake_all[(size_t)row * nt], 4LL * nt);
      f.read((char *)&rate_all[(size_t)row * nt], 4LL * nt);
      if (!f) return fail(CGFDM_ERR_SOURCE, "source file is truncated");
      ++row;
    }
  }
  #pragma omp parallel for schedule(static)
  for (long long row = 0; row < pn; ++row) {
    const float *asd = &asd_all[row * 3];
    const float *rake = &rake_all[(size_t)row * nt], *rate = &rate_all[(size_t)row * nt];
    float s_ = asd[1] * kDEG2RAD, d = asd[2] * kDEG2RAD, a = asd[0];
    for (int t = 0; t < nt; ++t) {
      float r = rake[t] * kDEG2RAD, rt = rate[t];
      float M11 = -(std::sin(d) * std::cos(r) * std::sin(2.0 * s_) +
                    std::sin(2.0 * d) * std::sin(r) * std::sin(s_) * std::sin(s_));
      float M22 = std::sin(d) * std::cos(r) * std::sin(2.0 * s_) -
                  std::sin(2.0 * d) * std::sin(r) * std::cos(s_) * std::cos(s_);
      float M33 = -(M11 + M22);
      float M12 = std::sin(d) * std::cos(r) * std::cos(2.0 * s_) +
                  0.5 * std::sin(2.0 * d) * std::sin(r) * std::sin(2.0 * s_);
      float M13 = -(std::cos(d) * std::cos(r) * std::cos(s_) +
                    std::cos(2.0 * d) * std::sin(r) * std::sin(s_));
      float M23 = -(std::cos(d) * std::cos(r) * std::sin(s_) -
                    std::cos(2.0 * d) * std::sin(r) * std::cos(s_));
      float *m = &mr[((size_t)row * nt + t) * 6];
      m[0] = M22 * a * rt;
      m[1] = M11 * a * rt;
      m[2] = M33 * a * rt;
      m[3] = M12 * a * rt;
      m[4] = -M23 * a * rt;
      m[5] = -M13 * a * rt;
    }
  }
  // dealDuplicateIndex (multiSource.cpp:566-624): the last row of a cell
  // accumulates the earlier rows of that cell in order.
  std::map<long long, long long> index_point;
  long long r = 0;
  for (auto &kv : point_index) index_point[kv.second] = r++;
  r = 0;
  for (auto &kv : point_index) {
    long long ii = index_point[kv.second];
    if (ii > r)
      for (int t = 0; t < nt; ++t)
        for (int q = 0; q < 6; ++q) mr[((size_t)ii * nt + t) * 6 + q] += mr[((size_t)r * nt + t) * 6 + q];
    ++r;
  }
  // changeStorageOrder (multiSource.cpp:750-796) + calculate_MomentRate
  const long long np = (long long)index_point.size();
  s.src_index.assign(np, 0);
  s.moment_rate.assign((size_t)np * nt * 6, 0.0f);
  long long J = 0;
  for (auto &kv : index_point) {
    s.src_index[J] = kv.first;
    for (int t = 0; t < nt; ++t)
      for (int q = 0; q < 6; ++q)
        s.moment_rate[((size_t)J + (size_t)t * np) * 6 + q] = mr[((size_t)kv.second * nt + t) * 6 + q];
    ++J;
  }
  #pragma omp parallel for schedule(static)
  for (int t = 0; t < nt; ++t)
    for (long long i = 0; i < np; ++i) {
      long long idx = s.src_index[i];
      // J and mu as the reference reads them back from its CJM storage
      float jacb = storage_round(s.cjm[idx + s.num * 9], s.desc.precision);
      float mu = storage_round(s.cjm[idx + s.num * 10], s.desc.precision);
      float V = jacb * DH * DH * DH;
      V = 1.0 / V;
      V = V * sc.Cv;
      float *m = &s.moment_rate[((size_t)i + (size_t)t * np) * 6];
      for (int q = 0; q < 6; ++q) m[q] *= mu * V;
    }
  s.src_nt = nt;
  s.src_dt = dt;
  return CGFDM_OK;
}

// readStationIndex / initStationIndex (station.cpp:83-296).
int build_stations(const std::string &dir, Setup &s) {
  Json j;
  std::string err;
  if (!Json::parse_file(join(dir, "station.json"), j, err)) return CGFDM_OK;  // no stations
  const Json *obj = j.get("station(point)");
  if (!obj) return CGFDM_OK;
  const std::vector<Json> *items = nullptr;
  std::vector<Json> tmp;
  if (obj->kind == Json::Object) {
    for (auto &m : obj->members) tmp.push_back(m.second);
    items = &tmp;
  } else if (obj->kind == Json::Array) {
    items = &obj->items;
  } else {
    return CGFDM_OK;
  }
  for (auto &st : *items)
    if (st.items.size() != 3) return CGFDM_OK;  // station.cpp:155-159: no stations at all
  for (auto &st : *items) {
    int X = st.items[0].as_int(), Y = st.items[1].as_int(), Z = st.items[2].as_int();
    int tx = X + H, ty = Y + H, tz = Z + H;
    if (tx >= H && tx < s.nx_ - H && ty >= H && ty < s.ny_ - H && tz >= H && tz < s.nz_ - H) {
      s.sta_xyz.insert(s.sta_xyz.end(), {tx, ty, tz});
      s.sta_global.insert(s.sta_global.end(), {X, Y, Z});
    }
  }
  return CGFDM_OK;
}

}  // namespace

int load_params(const std::string &dir, Params &p) {
  Json j;
  std::string err;
  if (!Json::parse_file(join(dir, "params.json"), j, err))
    return fail(CGFDM_ERR_PARAMS, "params.json: " + err);
  if (j.kind != Json::Object) return fail(CGFDM_ERR_PARAMS, "params.json is not an object");
  auto D = [&](const char *k, double &v) { if (const Json *x = j.get(k)) v = x->as_double(); };
  auto F = [&](const char *k, float &v) { if (const Json *x = j.get(k)) v = (float)x->as_double(); };
  auto I = [&](const char *k, int &v) { if (const Json *x = j.get(k)) v = x->as_int(); };
  auto S = [&](const char *k, std::string &v) { if (const Json *x = j.get(k)) v = x->str; };
  D("TMAX", p.TMAX); D("DT", p.DT); D("DH", p.DH);
  I("NX", p.NX); I("NY", p.NY); I("NZ", p.NZ);
  I("PX", p.PX); I("PY", p.PY); I("PZ", p.PZ);
  I("centerX", p.centerX); I("centerY", p.centerY);
  D("centerLongitude", p.centerLongitude); D("centerLatitude", p.centerLatitude);
  I("IT_SKIP", p.IT_SKIP);
  I("sliceX", p.sliceX); I("sliceY", p.sliceY); I("sliceZ", p.sliceZ);
  I("sliceFreeSurf", p.sliceFreeSurf);
  I("nPML", p.nPML);
  I("gauss_hill", p.gauss_hill); I("useTerrain", p.useTerrain); I("useMedium", p.useMedium);
  I("useMultiSource", p.useMultiSource);
  I("LayeredModel", p.LayeredModel); S("LayeredFileName", p.LayeredFileName);
  I("useSingleSource(ricker)", p.useSingleSource);
  F("rickerfc", p.rickerfc);
  I("ShenModel", p.ShenModel); I("Crust_1Medel", p.Crust_1Medel);
  S("OUT", p.OUT);
  F("Depth(km)", p.Depth);
  I("sourceX", p.sourceX); I("sourceY", p.sourceY); I("sourceZ", p.sourceZ);
  S("sourceFile", p.sourceFile); S("sourceDir", p.sourceDir);
  F("mediumPerturbation", p.mediumPerturbation); I("mediumSeed", p.mediumSeed);
  I("SRTM90", p.SRTM90); S("TerrainDir", p.TerrainDir);
  I("lonStart", p.lonStart); I("latStart", p.latStart);
  I("blockX", p.blockX); I("blockY", p.blockY);
  if (!p.useTerrain) p.Depth = p.DH * p.NZ * 1e-3;  // getParams.cpp:244-247
  return CGFDM_OK;
}

int build_setup(const std::string &dir, int precision, Setup &s) {
  int rc = load_params(dir, s.p);
  if (rc) return rc;
  const Params &p = s.p;
  if (p.NX <= 0 || p.NY <= 0 || p.NZ <= 0 || !(p.DH > 0) || !(p.DT > 0))
    return fail(CGFDM_ERR_PARAMS, "params.json needs positive NX, NY, NZ, DH and DT");
  if (!(p.useMultiSource || p.useSingleSource))
    return fail(CGFDM_ERR_NO_SOURCE, "no source configured (modelChecking.cpp:28-37)");
  if (p.nPML > p.NX || p.nPML > p.NY || p.nPML > p.NZ)
    return fail(CGFDM_ERR_PML, "the PML layer (nPML) is bigger than the grid");
  s.nx_ = p.NX + 2 * H;
  s.ny_ = p.NY + 2 * H;
  s.nz_ = p.NZ + 2 * H;
  s.num = (long long)s.nx_ * s.ny_ * s.nz_;
  s.nsurf = (long long)s.nx_ * s.ny_;
  cgfdm_desc &d = s.desc;
  d.nx = p.NX; d.ny = p.NY; d.nz = p.NZ; d.npml = p.nPML;
  d.dh = (float)p.DH;
  d.dt = (float)p.DT;
  d.nt = (int)(p.TMAX / d.dt);  // propagate.cpp:35-36
  d.precision = precision;
  d.kernel = CGFDM_KERNEL_AUTO;
  d.device = 0;
  const Scale sc = scale_of(precision);
  // CGFDM_VERBOSE=1 prints the duration of each setup phase to stderr
  const bool verbose = std::getenv("CGFDM_VERBOSE") != nullptr;
  auto t0 = std::chrono::steady_clock::now();
  auto phase = [&](const char *name) {
    if (!verbose) return;
    auto t1 = std::chrono::steady_clock::now();
    std::fprintf(stderr, "[cgfdm setup] %-8s %.2f s\n", name,
                 std::chrono::duration<double>(t1 - t0).count());
    t0 = t1;
  };
  if ((rc = build_coord(dir, s))) return rc;
  phase("coord");
  if ((rc = build_medium(dir, s))) return rc;
  phase("medium");
  if ((rc = check_cfl(s))) return rc;
  phase("cfl");
  build_cjm(s, sc);
  phase("cjm");
  s.pml = pml_profiles(p.NX, p.NY, p.NZ, p.nPML, (float)p.DH);
  if (p.useSingleSource) {
    int sx = p.sourceX + H, sy = p.sourceY + H, sz = p.sourceZ + H;  // locateSource
    if (sx >= H && sx < s.nx_ - H && sy >= H && sy < s.ny_ - H && sz >= H && sz < s.nz_ - H) {
      s.point_src = true;
      s.point_xyz[0] = sx; s.point_xyz[1] = sy; s.point_xyz[2] = sz;
    }
  }
  if (p.useMultiSource && (rc = build_fault(dir, s, sc))) return rc;
  if ((rc = build_stations(dir, s))) return rc;
  return CGFDM_OK;
}

int write_station_file(const Setup &s, const std::string &out, const float *wave) {
  const int nsta = (int)s.sta_global.size() / 3;
  if (nsta == 0) return CGFDM_OK;
  FILE *f = std::fopen(join(out, "station_mpi_0_0_0.bin").c_str(), "wb");
  if (!f) return fail(CGFDM_ERR_IO, "cannot write the station file");
  std::fwrite(s.sta_global.data(), sizeof(int32_t), s.sta_global.size(), f);
  std::fwrite(wave, sizeof(float), (size_t)nsta * s.desc.nt * 9, f);
  std::fclose(f);
  return CGFDM_OK;
}

int write_pgv_file(const Setup &s, const std::string &out, const float *pgv) {
  FILE *f = std::fopen(join(out, "PGV_Z_mpi_0_0_0.bin").c_str(), "wb");
  if (!f) return fail(CGFDM_ERR_IO, "cannot write the PGV file");
  std::fwrite(pgv, sizeof(float), 2 * (size_t)s.p.NX * s.p.NY, f);
  std::fclose(f);
  return CGFDM_OK;
}

int write_slice_file(const std::string &name, char axis, const float *data, size_t n) {
  std::string fn = name + "_" + axis + "_mpi_0_0_0.bin";
  FILE *f = std::fopen(fn.c_str(), "wb");
  if (!f) return fail(CGFDM_ERR_IO, "cannot write " + fn);
  std::fwrite(data, sizeof(float), n, f);
  std::fclose(f);
  return CGFDM_OK;
}

int write_model_slices(const Setup &s, const std::string &out) {
  // data2D_Model_out (data_io.cpp:497-526): coordX/Y/Z and Vs/Vp/rho slices
  const Params &p = s.p;
  const int at[3] = {p.sliceX + H, p.sliceY + H, p.sliceZ + H};
  const int lim[3] = {s.nx_ - H, s.ny_ - H, s.nz_ - H};
  const char *names[6] = {"coordX", "coordY", "coordZ", "Vs", "Vp", "rho"};
  for (int ax = 0; ax < 3; ++ax) {
    if (at[ax] < H || at[ax] >= lim[ax]) continue;
    const int n0 = ax == 0 ? p.NY : p.NX, n1 = ax == 2 ? p.NY : p.NZ;
    std::vector<float> buf((size_t)n0 * n1);
    for (int v = 0; v < 6; ++v) {
      const std::vector<float> &src = v < 3 ? s.coord : s.medium;
      const int var = v % 3;
      for (int b = 0; b < n1; ++b)
        for (int a = 0; a < n0; ++a) {
          int i, j, k;
          if (ax == 0) { i = at[0]; j = a + H; k = b + H; }
          else if (ax == 1) { i = a + H; j = at[1]; k = b + H; }
          else { i = a + H; j = b + H; k = at[2]; }
          buf[a + (size_t)b * n0] = src[IDX(s, i, j, k) * 3 + var];
        }
      int rc = write_slice_file(join(out, names[v]), "XYZ"[ax], buf.data(), buf.size());
      if (rc) return rc;
    }
  }
  return CGFDM_OK;
}

}  // namespace cgfdm
