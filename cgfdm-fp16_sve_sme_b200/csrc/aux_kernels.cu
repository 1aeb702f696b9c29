// Small per-step kernels around the fused stage: source injection, station
// and PGV sampling, slice packing, layout conversion.  Compiled with
// --fmad=false: each follows the reference's arithmetic exactly.
#include "kernels.h"

namespace cgfdm {
namespace {

template <typename S>
__global__ void point_source_kernel(S *w0, S *w1, S *w2, const S *cjm, Layout L, int sx, int sy,
                                    int sz, const float *amp343, const float *moment,
                                    const int *step, float DH3, double CsDT) {
  using R = typename Arith<S>::R;
  const int t = threadIdx.x;
  if (t >= 343) return;
  const float s = moment[*step];
  const int i = sx - 3 + t % 7, j = sy - 3 + (t / 7) % 7, k = sz - 3 + t / 49;
  const long long c = L.at(i, j, k);
  const float jacb = ldv(cjm + L.at(sx, sy, sz) + L.fs * 9);
  // singleSource.cpp:112-123
  float value = -1.0f * s * amp343[t] / (jacb * DH3);
  value = (float)((double)value * CsDT);
  const bool halo = i < HALO || i >= L.nx_ - HALO || j < HALO || j >= L.ny_ - HALO || k < HALO ||
                    k >= L.nz_ - HALO;
  for (int v = 3; v < 6; ++v) {
    const long long q = c + v * L.fs;
    stv(w0 + q, (R)ldv(w0 + q) + (R)value);
    if (halo) {
      stv(w1 + q, (R)ldv(w1 + q) + (R)value);
      stv(w2 + q, (R)ldv(w2 + q) + (R)value);
    }
  }
}

template <typename S>
__global__ void fault_source_kernel(S *w, long long fs, const long long *idx, const float *rate,
                                    long long npts, const int *src_it, const float *src_tw,
                                    const int *step, float DT) {
  const long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const int srcIt = src_it[*step];
  if (p >= npts || srcIt < 0) return;  // srcIt < 0: the source has ended
  const float tw = src_tw[*step];
  const float *m0 = rate + ((long long)srcIt * npts + p) * 6;
  const float *m1 = rate + ((long long)(srcIt + 1) * npts + p) * 6;
  const long long c = idx[p];
  for (int q = 0; q < 6; ++q) {
    const float slice = (m1[q] - m0[q]) * tw + m0[q];  // interp_momentRate
    const long long a = c + (3 + q) * fs;
    stv(w + a, (typename Arith<S>::R)ldv(w + a) - slice * DT);  // addSource1
  }
}

// Stations and PGV of step *step, then the step counter advances: every
// block reads *step first, and the last block to finish (counted in
// step[1]) increments it, so the step ends with one launch.
template <typename S>
__global__ void station_pgv_kernel(const S *w, Layout L, const int *xyz, int nsta, int NT,
                                   int *step, float *wave, float *pgv, float c1, float c2,
                                   double cv_inv) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int it = *(volatile int *)step;
  const int nx = L.nx_ - 2 * HALO, ny = L.ny_ - 2 * HALO;
  if (t < nsta) {
    const long long c = L.at(xyz[3 * t], xyz[3 * t + 1], xyz[3 * t + 2]);
    const long long pos = it + (long long)t * NT;
    for (int v = 0; v < 9; ++v)
      wave[pos * 9 + v] = (float)ldv(w + c + v * L.fs) * (v < 3 ? c1 : c2);
  }
  if (t < nx * ny) {
    const long long c = L.at(t % nx + HALO, t / nx + HALO, L.nz_ - HALO - 1);
    const float vx = (float)((double)(float)ldv(w + c) * cv_inv);
    const float vy = (float)((double)(float)ldv(w + c + L.fs) * cv_inv);
    const float vz = (float)((double)(float)ldv(w + c + 2 * L.fs) * cv_inv);
    const float vh = sqrtf(vx * vx + vy * vy);
    const float vv = sqrtf(vx * vx + vy * vy + vz * vz);
    if (pgv[2 * t] < vh) pgv[2 * t] = vh;
    if (pgv[2 * t + 1] < vv) pgv[2 * t + 1] = vv;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    if (atomicAdd(step + 1, 1) == (int)gridDim.x - 1) {
      step[1] = 0;
      step[0] = it + 1;
      __threadfence();
    }
  }
}

template <typename S>
__global__ void slice_pack_kernel(const S *f, Layout L, int axis, int at, double c, float *out) {
  const int nx = L.nx_ - 2 * HALO, ny = L.ny_ - 2 * HALO, nz = L.nz_ - 2 * HALO;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  int i, j, k;
  if (axis == 0) {
    if (t >= ny * nz) return;
    i = at; j = t % ny + HALO; k = t / ny + HALO;
  } else if (axis == 1) {
    if (t >= nx * nz) return;
    i = t % nx + HALO; j = at; k = t / nx + HALO;
  } else {
    if (t >= nx * ny) return;
    i = t % nx + HALO; j = t / nx + HALO; k = at;
  }
  out[t] = (float)((double)(float)ldv(f + L.at(i, j, k)) * c);
}

template <typename S>
__global__ void repack_in_kernel(const float *src, S *dst, Layout L, int nfield) {
  const long long num = (long long)L.nx_ * L.ny_ * L.nz_;
  const long long total = num * nfield;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < total;
       q += (long long)gridDim.x * blockDim.x) {
    const long long f = q / num, r = q % num;
    const int i = (int)(r % L.nx_), j = (int)((r / L.nx_) % L.ny_), k = (int)(r / ((long long)L.nx_ * L.ny_));
    stv(dst + f * L.fs + L.at(i, j, k), src[q]);
  }
}

template <typename S>
__global__ void repack_out_kernel(const S *src, float *dst, Layout L, int nfield) {
  const long long num = (long long)L.nx_ * L.ny_ * L.nz_;
  const long long total = num * nfield;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < total;
       q += (long long)gridDim.x * blockDim.x) {
    const long long f = q / num, r = q % num;
    const int i = (int)(r % L.nx_), j = (int)((r / L.nx_) % L.ny_), k = (int)(r / ((long long)L.nx_ * L.ny_));
    dst[q] = (float)ldv(src + f * L.fs + L.at(i, j, k));
  }
}

}  // namespace

template <typename S>
cudaError_t launch_point_source(S *w0, S *w1, S *w2, const S *cjm, Layout L, int sx, int sy,
                                int sz, const float *amp343, const float *moment, const int *step,
                                float DH3, double CsDT, cudaStream_t st) {
  point_source_kernel<S><<<1, 352, 0, st>>>(w0, w1, w2, cjm, L, sx, sy, sz, amp343, moment, step,
                                            DH3, CsDT);
  return cudaGetLastError();
}

template <typename S>
cudaError_t launch_fault_source(S *w, long long fs, const long long *idx, const float *rate,
                                long long npts, const int *src_it, const float *src_tw,
                                const int *step, float DT, cudaStream_t st) {
  if (npts <= 0) return cudaSuccess;
  fault_source_kernel<S><<<(unsigned)((npts + 255) / 256), 256, 0, st>>>(w, fs, idx, rate, npts,
                                                                        src_it, src_tw, step, DT);
  return cudaGetLastError();
}

template <typename S>
cudaError_t launch_station_pgv(const S *w, Layout L, const int *xyz, int nsta, int NT,
                               int *step, float *wave, float *pgv, float c1, float c2,
                               double cv_inv, cudaStream_t st) {
  const int n = (L.nx_ - 2 * HALO) * (L.ny_ - 2 * HALO);
  const int total = n > nsta ? n : nsta;
  station_pgv_kernel<S><<<(total + 255) / 256, 256, 0, st>>>(w, L, xyz, nsta, NT, step, wave, pgv,
                                                             c1, c2, cv_inv);
  return cudaGetLastError();
}

template <typename S>
cudaError_t launch_slice_pack(const S *field, Layout L, int axis, int at, double c, float *out,
                              cudaStream_t st) {
  const int nx = L.nx_ - 2 * HALO, ny = L.ny_ - 2 * HALO, nz = L.nz_ - 2 * HALO;
  const int n = axis == 0 ? ny * nz : axis == 1 ? nx * nz : nx * ny;
  slice_pack_kernel<S><<<(n + 255) / 256, 256, 0, st>>>(field, L, axis, at, c, out);
  return cudaGetLastError();
}

template <typename S>
cudaError_t launch_repack_in(const float *src, S *dst, Layout L, int nfield, cudaStream_t st) {
  repack_in_kernel<S><<<2368, 256, 0, st>>>(src, dst, L, nfield);
  return cudaGetLastError();
}
template <typename S>
cudaError_t launch_repack_out(const S *src, float *dst, Layout L, int nfield, cudaStream_t st) {
  repack_out_kernel<S><<<2368, 256, 0, st>>>(src, dst, L, nfield);
  return cudaGetLastError();
}

#define CGFDM_INST(S)                                                                              \
  template cudaError_t launch_point_source<S>(S *, S *, S *, const S *, Layout, int, int, int,     \
                                              const float *, const float *, const int *, float,    \
                                              double, cudaStream_t);                               \
  template cudaError_t launch_fault_source<S>(S *, long long, const long long *, const float *,    \
                                              long long, const int *, const float *, const int *,  \
                                              float, cudaStream_t);                                \
  template cudaError_t launch_station_pgv<S>(const S *, Layout, const int *, int, int, int *,      \
                                             float *, float *, float, float, double,               \
                                             cudaStream_t);                                        \
  template cudaError_t launch_slice_pack<S>(const S *, Layout, int, int, double, float *,         \
                                            cudaStream_t);                                         \
  template cudaError_t launch_repack_in<S>(const float *, S *, Layout, int, cudaStream_t);        \
  template cudaError_t launch_repack_out<S>(const S *, float *, Layout, int, cudaStream_t);

CGFDM_INST(float)
CGFDM_INST(__half)
CGFDM_INST(__nv_bfloat16)
CGFDM_INST(double)

}  // namespace cgfdm
