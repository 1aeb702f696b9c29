// Small per-step kernels around the fused stage: source injection, station
// and PGV sampling, slice packing, storage conversion.  Compiled with
// --fmad=false: each follows the reference's arithmetic exactly.
#include "kernels.h"

namespace cgfdm {
namespace {

template <typename S>
__global__ void point_source_kernel(S *w0, S *w1, S *w2, const S *cjm, long long num, int nx_, int ny_,
                                    int nz_, int sx, int sy, int sz, const float *amp343, float s,
                                    float DH3, double CsDT) {
  const int t = threadIdx.x;
  if (t >= 343) return;
  const int di = t % 7, dj = (t / 7) % 7, dk = t / 49;
  const int i = sx - 3 + di, j = sy - 3 + dj, k = sz - 3 + dk;
  const long long sxy = (long long)nx_ * ny_;
  const long long c = i + (long long)j * nx_ + k * sxy;
  const long long src = sx + (long long)sy * nx_ + sz * sxy;
  const float jacb = ldv(cjm + src + num * 9);
  // singleSource.cpp:112-123
  float value = -1.0f * s * amp343[t] / (jacb * DH3);
  value = (float)((double)value * CsDT);
  const bool halo = i < HALO || i >= nx_ - HALO || j < HALO || j >= ny_ - HALO || k < HALO ||
                    k >= nz_ - HALO;
  using R = typename Arith<S>::R;
  for (int v = 3; v < 6; ++v) {
    const long long q = c + v * num;
    stv(w0 + q, (R)ldv(w0 + q) + (R)value);
    if (halo) {
      stv(w1 + q, (R)ldv(w1 + q) + (R)value);
      stv(w2 + q, (R)ldv(w2 + q) + (R)value);
    }
  }
}

template <typename S>
__global__ void fault_source_kernel(S *w, long long num, const long long *idx, const float *rate,
                                    long long npts, int srcIt, float tw, float DT) {
  const long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (p >= npts) return;
  const float *m0 = rate + ((long long)srcIt * npts + p) * 6;
  const float *m1 = rate + ((long long)(srcIt + 1) * npts + p) * 6;
  const long long c = idx[p];
  for (int q = 0; q < 6; ++q) {
    const float slice = (m1[q] - m0[q]) * tw + m0[q];  // interp_momentRate
    const long long a = c + (3 + q) * num;
    stv(w + a, (typename Arith<S>::R)ldv(w + a) - slice * DT);  // addSource1
  }
}

template <typename S>
__global__ void station_pgv_kernel(const S *w, long long num, int nx_, int ny_, int nz_, const int *xyz,
                                   int nsta, int NT, int it, float *wave, float *pgv, float c1,
                                   float c2, double cv_inv) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int nx = nx_ - 2 * HALO, ny = ny_ - 2 * HALO;
  const long long sxy = (long long)nx_ * ny_;
  if (t < nsta) {
    const long long c = xyz[3 * t] + (long long)xyz[3 * t + 1] * nx_ + xyz[3 * t + 2] * sxy;
    const long long pos = it + (long long)t * NT;
    for (int v = 0; v < 9; ++v) wave[pos * 9 + v] = (float)ldv(w + c + v * num) * (v < 3 ? c1 : c2);
  }
  if (t < nx * ny) {
    const int i0 = t % nx, j0 = t / nx;
    const int k = nz_ - HALO - 1;
    const long long c = (i0 + HALO) + (long long)(j0 + HALO) * nx_ + k * sxy;
    const float vx = (float)((double)(float)ldv(w + c) * cv_inv);
    const float vy = (float)((double)(float)ldv(w + c + num) * cv_inv);
    const float vz = (float)((double)(float)ldv(w + c + 2 * num) * cv_inv);
    const float vh = sqrtf(vx * vx + vy * vy);
    const float vv = sqrtf(vx * vx + vy * vy + vz * vz);
    if (pgv[2 * t] < vh) pgv[2 * t] = vh;
    if (pgv[2 * t + 1] < vv) pgv[2 * t + 1] = vv;
  }
}

template <typename S>
__global__ void slice_pack_kernel(const S *f, int nx_, int ny_, int nz_, int axis, int at, double c,
                                  float *out) {
  const int nx = nx_ - 2 * HALO, ny = ny_ - 2 * HALO, nz = nz_ - 2 * HALO;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  int i, j, k, n0;
  if (axis == 0) { n0 = ny; if (t >= ny * nz) return; i = at; j = t % ny + HALO; k = t / ny + HALO; }
  else if (axis == 1) { n0 = nx; if (t >= nx * nz) return; i = t % nx + HALO; j = at; k = t / nx + HALO; }
  else { n0 = nx; if (t >= nx * ny) return; i = t % nx + HALO; j = t / nx + HALO; k = at; }
  (void)n0;
  const long long q = i + (long long)j * nx_ + (long long)k * nx_ * ny_;
  out[t] = (float)((double)(float)ldv(f + q) * c);
}

template <typename S> __global__ void convert_in_kernel(const float *src, S *dst, long long n) {
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n;
       q += (long long)gridDim.x * blockDim.x)
    stv(dst + q, src[q]);
}
template <typename S> __global__ void convert_out_kernel(const S *src, float *dst, long long n) {
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n;
       q += (long long)gridDim.x * blockDim.x)
    dst[q] = (float)ldv(src + q);
}

}  // namespace

template <typename S>
cudaError_t launch_point_source(S *w0, S *w1, S *w2, const S *cjm, long long num, int nx_, int ny_,
                                int nz_, int sx, int sy, int sz, const float *amp343, float s,
                                float DH3, double CsDT, cudaStream_t st) {
  point_source_kernel<S><<<1, 352, 0, st>>>(w0, w1, w2, cjm, num, nx_, ny_, nz_, sx, sy, sz, amp343,
                                            s, DH3, CsDT);
  return cudaGetLastError();
}

template <typename S>
cudaError_t launch_fault_source(S *w, long long num, const long long *idx, const float *rate,
                                long long npts, int srcIt, float tw, float DT, cudaStream_t st) {
  if (npts <= 0) return cudaSuccess;
  fault_source_kernel<S><<<(unsigned)((npts + 255) / 256), 256, 0, st>>>(w, num, idx, rate, npts,
                                                                        srcIt, tw, DT);
  return cudaGetLastError();
}

template <typename S>
cudaError_t launch_station_pgv(const S *w, long long num, int nx_, int ny_, int nz_, const int *xyz,
                               int nsta, int NT, int it, float *wave, float *pgv, float c1, float c2,
                               double cv_inv, cudaStream_t st) {
  const int n = (nx_ - 2 * HALO) * (ny_ - 2 * HALO);
  const int total = n > nsta ? n : nsta;
  station_pgv_kernel<S><<<(total + 255) / 256, 256, 0, st>>>(w, num, nx_, ny_, nz_, xyz, nsta, NT, it,
                                                             wave, pgv, c1, c2, cv_inv);
  return cudaGetLastError();
}

template <typename S>
cudaError_t launch_free_surface_pack(const S *w, long long num, int nx_, int ny_, int nz_,
                                     double cv_inv, float *out, cudaStream_t st) {
  const int n = (nx_ - 2 * HALO) * (ny_ - 2 * HALO);
  for (int v = 0; v < 3; ++v) {
    slice_pack_kernel<S><<<(n + 255) / 256, 256, 0, st>>>(w + v * num, nx_, ny_, nz_, 2,
                                                          nz_ - HALO - 1, cv_inv, out + v * n);
  }
  return cudaGetLastError();
}

template <typename S>
cudaError_t launch_slice_pack(const S *field, int nx_, int ny_, int nz_, int axis, int at, double c,
                              float *out, cudaStream_t st) {
  const int nx = nx_ - 2 * HALO, ny = ny_ - 2 * HALO, nz = nz_ - 2 * HALO;
  const int n = axis == 0 ? ny * nz : axis == 1 ? nx * nz : nx * ny;
  slice_pack_kernel<S><<<(n + 255) / 256, 256, 0, st>>>(field, nx_, ny_, nz_, axis, at, c, out);
  return cudaGetLastError();
}

template <typename S> cudaError_t launch_convert_in(const float *src, S *dst, long long n, cudaStream_t st) {
  convert_in_kernel<S><<<1184, 256, 0, st>>>(src, dst, n);
  return cudaGetLastError();
}
template <typename S> cudaError_t launch_convert_out(const S *src, float *dst, long long n, cudaStream_t st) {
  convert_out_kernel<S><<<1184, 256, 0, st>>>(src, dst, n);
  return cudaGetLastError();
}

#define CGFDM_INST(S)                                                                              \
  template cudaError_t launch_point_source<S>(S *, S *, S *, const S *, long long, int, int, int, int, \
                                              int, int, const float *, float, float, double,       \
                                              cudaStream_t);                                       \
  template cudaError_t launch_fault_source<S>(S *, long long, const long long *, const float *,    \
                                              long long, int, float, float, cudaStream_t);         \
  template cudaError_t launch_station_pgv<S>(const S *, long long, int, int, int, const int *, int, \
                                             int, int, float *, float *, float, float, double,     \
                                             cudaStream_t);                                        \
  template cudaError_t launch_free_surface_pack<S>(const S *, long long, int, int, int, double,    \
                                                   float *, cudaStream_t);                         \
  template cudaError_t launch_slice_pack<S>(const S *, int, int, int, int, int, double, float *,   \
                                            cudaStream_t);                                         \
  template cudaError_t launch_convert_in<S>(const float *, S *, long long, cudaStream_t);         \
  template cudaError_t launch_convert_out<S>(const S *, float *, long long, cudaStream_t);

CGFDM_INST(float)
CGFDM_INST(__half)
CGFDM_INST(__nv_bfloat16)
CGFDM_INST(double)

}  // namespace cgfdm
