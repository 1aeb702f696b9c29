// Host-side arithmetic that the reference performs on the CPU before or
// around the time loop, in the reference's precision and operation order
// (compiled with -ffp-contract=off).
#include <cmath>
#include <vector>

#include "engine.h"

namespace cgfdm {

namespace {
constexpr float kPI = 3.141592657f;  // macro.h:60
constexpr int H = 3;
}  // namespace

std::vector<float> pml_profiles(int nx, int ny, int nz, int npml, float DH) {
  // init_pml_para.cpp:99-234: profiles 13-19, Cp = 6000 (line 117),
  // R from the layer count (line 120), d/beta and 1/beta (lines 211-226).
  const int n_[3] = {nx + 2 * H, ny + 2 * H, nz + 2 * H};
  std::vector<float> out(3 * (size_t)(n_[0] + n_[1] + n_[2]), 0.0f);
  const float Cp = 6000.0f, pml_fc = 0.5f;
  const float L = DH * (npml - 1);
  const float R = std::pow(10.0, -(std::log10((double)npml) - 1.0) / std::log10(2.0) - 3.0);
  const float d0 = -(2.0f + 1.0f) * Cp / (2.0f * L) * std::log(R);
  const float a0 = kPI * pml_fc, b0 = 3.0f;
  size_t base = 0;
  for (int ax = 0; ax < 3; ++ax) {
    const int np = n_[ax], ni = np - H;
    float *alpha = out.data() + base, *beta = alpha + np, *dd = beta + np;
    for (int i = 0; i < np; ++i) {
      float a = 0.0f, b = 1.0f, d = 0.0f;
      if (npml > 0 && i >= H && i < ni) {
        float l = -1.0f;
        if (i < H + npml) l = (H + npml - 1 - i) * DH;
        if (ax != 2 && i >= ni - npml) l = (i - (ni - npml)) * DH;
        a = l < 0.0f ? 0.0f : a0 * (1.0f - std::pow(l / L, 1.0f));
        b = l < 0.0f ? 1.0f : 1.0f + (b0 - 1.0f) * std::pow(l / L, 2.0f);
        d = l < 0.0f ? 0.0f : d0 * std::pow(l / L, 2.0f);
      }
      alpha[i] = a;
      dd[i] = d / b;
      beta[i] = 1.0f / b;
    }
    base += 3 * (size_t)np;
  }
  return out;
}

float ricker_moment(float rickerfc, int it, float DT) {
  // sourceFunction with irk = 0 (singleSource.cpp:29-56)
  float t = (it + 0.0f) * DT;
  float tdelay = 1.2f / rickerfc;
  float f0 = 2;
  float r = kPI * rickerfc * (t - tdelay);
  float rr = r * r;
  float s = r * (2.0f * rr - 3.0) * std::exp(-rr) * f0 * kPI * rickerfc;
  float M0 = 1e16f;
  s *= M0;
  return s;
}

void gauss_weights343(float *amp) {
  // singleSource.cpp:101-107 with nGauss = 3, GAUSS_FUN (macro.h:39)
  const int nG = 3;
  const float ra = nG * 0.5f;
  auto gauss = [&](int t) -> float {
    double x = (t - 0.0) / ra;
    return (float)(std::exp(-(x * x)) / (ra * 1.772453850905516));
  };
  for (int dk = -nG; dk <= nG; ++dk)
    for (int dj = -nG; dj <= nG; ++dj)
      for (int di = -nG; di <= nG; ++di) {
        float a = gauss(di) * gauss(dj) * gauss(dk);
        a = (float)(a / 0.998125703461425);
        amp[(di + nG) + 7 * (dj + nG) + 49 * (dk + nG)] = a;
      }
}

}  // namespace cgfdm
