// Free-surface layers of the fast path: the three top interior layers of a
// stage (freeSurface.cpp:104-256 with the RK combination of wave_rk.cpp:13-99)
// for the columns outside every PML slab, tiled through shared memory.
//
// The exact-order kernel (stage_exact.cu) computes each point's traction-image
// rows -- the J-weighted tractions J (xi . T) of its seven neighbours along
// each direction -- and its velocity stencils straight from global memory,
// so a row is rebuilt by every point whose stencil reaches it.  Here a 32 x 8
// column tile first builds, once each, the rows along x (with a 3-column
// halo), along y (3-row halo) and along z (the five planes below the
// surface), and the velocities of the three layers with their x/y halo, in
// shared memory; each thread then forms its column's three output points from
// them.  FP32 arithmetic with FMA contraction (this file is compiled without
// --fmad=false), so results agree with the reference to rounding; the
// exact-order kernel keeps the bit-exact path and the PML-slab columns.
#include <atomic>

#include "device_common.cuh"
#include "kernels.h"

namespace cgfdm {
namespace {

constexpr int TTX = 32, TTY = 8;  // tile of columns
constexpr int HX = TTX + 6, HY = TTY + 6;

// J-weighted traction rows of direction dir at q (freeSurface.cpp:128-153).
template <typename S>
__device__ __forceinline__ void jt3(const S *W, const S *cjm, long long fs, long long q, int dir,
                                    float r[3]) {
  const float m0 = ldv(cjm + q + fs * (3 * dir)), m1 = ldv(cjm + q + fs * (3 * dir + 1)),
              m2 = ldv(cjm + q + fs * (3 * dir + 2)), J = ldv(cjm + q + fs * 9);
  const float txx = ldv(W + q + fs * 3), tyy = ldv(W + q + fs * 4), tzz = ldv(W + q + fs * 5);
  const float txy = ldv(W + q + fs * 6), txz = ldv(W + q + fs * 7), tyz = ldv(W + q + fs * 8);
  r[0] = (m0 * txx + m1 * txy + m2 * txz) * J;
  r[1] = (m0 * txy + m1 * tyy + m2 * tyz) * J;
  r[2] = (m0 * txz + m1 * tyz + m2 * tzz) * J;
}

// One-sided 5-point MacCormack sum over taps t[3 - FB] .. t[3 + 3 FB] of a
// 7-entry row with stride `st`, times FB (the caller applies 1/DH)
template <int FB>
__device__ __forceinline__ float lsum(const float *t, int st) {
  return (float)FB * (kAm1 * t[(3 - FB) * st] + kA0 * t[3 * st] + kA1 * t[(3 + FB) * st] +
                      kA2 * t[(3 + 2 * FB) * st] + kA3 * t[(3 + 3 * FB) * st]);
}

__device__ __forceinline__ void elastic_v(const float m[3], const float dv[3], float mu, float lam,
                                          float out[6]) {
  const float div = m[0] * dv[0] + m[1] * dv[1] + m[2] * dv[2];
  out[0] = div * lam + 2.0f * mu * (m[0] * dv[0]);
  out[1] = div * lam + 2.0f * mu * (m[1] * dv[1]);
  out[2] = div * lam + 2.0f * mu * (m[2] * dv[2]);
  out[3] = (m[1] * dv[0] + m[0] * dv[1]) * mu;
  out[4] = (m[2] * dv[0] + m[0] * dv[2]) * mu;
  out[5] = (m[2] * dv[1] + m[1] * dv[2]) * mu;
}

// (the traction row at the surface plane itself is zero: the z rows are
// needed on the five planes below it)
struct TopSmem {
  float jx[3][3][TTY][HX];  // [layer][component][row][column with x halo]
  float jy[3][3][HY][TTX];  // [layer][component][row with y halo][column]
  float jz[5][3][TTY][TTX];  // [plane ktop-5+p][component][row][column]
  float v[3][3][HY][HX];    // [layer][velocity][row][column], x and y halo
};

template <typename S, int FB1, int FB2, int FB3>
__global__ void __launch_bounds__(TTX *TTY) stage_top_kernel(const __grid_constant__ StageArgs<S> a,
                                                             int i0, int i1, int j0, int j1) {
  extern __shared__ float4 top_smem[];
  TopSmem &sm = *reinterpret_cast<TopSmem *>(top_smem);
  const Layout L = a.L;
  const long long fs = L.fs;
  const int ktop = L.nz_ - HALO - 1;
  const int ix = i0 + TTX * blockIdx.x, jy = j0 + TTY * blockIdx.y;
  const int tid = threadIdx.x + TTX * threadIdx.y;
  const S *W = a.win, *cjm = a.cjm;
  // (1) the shared rows; entries outside the padded grid stay unused
  for (int e = tid; e < 3 * TTY * HX; e += TTX * TTY) {
    const int l = e / (TTY * HX), r = (e / HX) % TTY, c = e % HX;
    const int gi = ix - 3 + c, gj = jy + r;
    if (gi < 0 || gi >= L.nx_ || gj >= L.ny_) continue;
    float t[3];
    jt3(W, cjm, fs, L.at(gi, gj, ktop - 2 + l), 0, t);
    sm.jx[l][0][r][c] = t[0]; sm.jx[l][1][r][c] = t[1]; sm.jx[l][2][r][c] = t[2];
  }
  for (int e = tid; e < 3 * HY * TTX; e += TTX * TTY) {
    const int l = e / (HY * TTX), r = (e / TTX) % HY, c = e % TTX;
    const int gi = ix + c, gj = jy - 3 + r;
    if (gi >= L.nx_ || gj < 0 || gj >= L.ny_) continue;
    float t[3];
    jt3(W, cjm, fs, L.at(gi, gj, ktop - 2 + l), 1, t);
    sm.jy[l][0][r][c] = t[0]; sm.jy[l][1][r][c] = t[1]; sm.jy[l][2][r][c] = t[2];
  }
  for (int e = tid; e < 5 * TTY * TTX; e += TTX * TTY) {
    const int p = e / (TTY * TTX), r = (e / TTX) % TTY, c = e % TTX;
    const int gi = ix + c, gj = jy + r;
    if (gi >= L.nx_ || gj >= L.ny_) continue;
    float t[3];
    jt3(W, cjm, fs, L.at(gi, gj, ktop - 5 + p), 2, t);
    sm.jz[p][0][r][c] = t[0]; sm.jz[p][1][r][c] = t[1]; sm.jz[p][2][r][c] = t[2];
  }
  for (int e = tid; e < 3 * HY * HX; e += TTX * TTY) {
    const int l = e / (HY * HX), r = (e / HX) % HY, c = e % HX;
    const int gi = ix - 3 + c, gj = jy - 3 + r;
    if (gi < 0 || gi >= L.nx_ || gj < 0 || gj >= L.ny_) continue;
    const long long q = L.at(gi, gj, ktop - 2 + l);
    sm.v[l][0][r][c] = ldv(W + q);
    sm.v[l][1][r][c] = ldv(W + q + fs);
    sm.v[l][2][r][c] = ldv(W + q + 2 * fs);
  }
  __syncthreads();

  // (2) the column's three points
  const int tx = threadIdx.x, ty = threadIdx.y;
  const int i = ix + tx, j = jy + ty;
  if (i >= i1 || j >= j1) return;
  const float rDH = a.rDH, DT = a.DT;
  const float *px = a.pml, *py = a.pml + 3 * L.nx_;
  const float bx = px[L.nx_ + i], by = py[L.ny_ + j];
  const long long s2 = i + (long long)j * L.nx_;
  const float *DX = a.rdz + s2 * 9, *DY = a.rdz + (long long)L.nx_ * L.ny_ * 9 + s2 * 9;
#pragma unroll
  for (int l = 0; l < 3; ++l) {
    const int k = ktop - 2 + l;
    const long long c = L.at(i, j, k);
    float m[3][3];
#pragma unroll
    for (int d = 0; d < 3; ++d)
#pragma unroll
      for (int q = 0; q < 3; ++q) m[d][q] = ldv(cjm + c + fs * (3 * d + q));
    const float J = ldv(cjm + c + fs * 9), mu = ldv(cjm + c + fs * 10), lam = ldv(cjm + c + fs * 11);
    const float bu = ldv(cjm + c + fs * 12) * (float)CRHO_OF<S>::v;
    float h[9];
    // velocity rows: image rows above the surface are the negated rows below
    const int ks = 5 - l;  // the surface's index in the point's 7-entry z row
#pragma unroll
    for (int q = 0; q < 3; ++q) {
      float zr[7];
#pragma unroll
      for (int e = 0; e < 7; ++e) {
        if (e < ks)
          zr[e] = sm.jz[l + e][q][ty][tx];
        else if (e == ks)
          zr[e] = 0.0f;
        else
          zr[e] = -sm.jz[l + 2 * ks - e][q][ty][tx];
      }
      const float lx = lsum<FB1>(&sm.jx[l][q][ty][tx], 1);
      const float ly = lsum<FB2>(&sm.jy[l][q][ty][tx], TTX);
      const float lz = lsum<FB3>(zr, 1);
      h[q] = bu / J * ((lx * bx + ly * by + lz) * rDH) * DT;
    }
    // stress rows from the velocity derivatives
    float vxi[3], vet[3], vzt[3];
#pragma unroll
    for (int v = 0; v < 3; ++v) {
      vxi[v] = lsum<FB1>(&sm.v[l][v][ty + 3][tx], 1) * rDH * bx;
      vet[v] = lsum<FB2>(&sm.v[l][v][ty][tx + 3], HX) * rDH * by;
    }
    if (l == 2) {
#pragma unroll
      for (int q = 0; q < 3; ++q)
        vzt[q] = (DX[3 * q] * vxi[0] + DX[3 * q + 1] * vxi[1] + DX[3 * q + 2] * vxi[2]) +
                 (DY[3 * q] * vet[0] + DY[3 * q + 1] * vet[1] + DY[3 * q + 2] * vet[2]);
    } else if (l == 1) {  // 2-point operator (axis.h:92)
#pragma unroll
      for (int v = 0; v < 3; ++v)
        vzt[v] = (float)FB3 * (sm.v[1 + FB3][v][ty + 3][tx + 3] - sm.v[1][v][ty + 3][tx + 3]) * rDH;
    } else {  // 3-point operator (axis.h:93)
#pragma unroll
      for (int v = 0; v < 3; ++v) {
        const float w0 = sm.v[0][v][ty + 3][tx + 3];
        float w1, w2;
        if (FB3 > 0) {
          w1 = sm.v[1][v][ty + 3][tx + 3];
          w2 = sm.v[2][v][ty + 3][tx + 3];
        } else {
          w1 = ldv(W + v * fs + c - L.plane);
          w2 = ldv(W + v * fs + c - 2 * L.plane);
        }
        vzt[v] = (float)FB3 * (kCf1 * w0 + kCf2 * w1 + kCf3 * w2) * rDH;
      }
    }
    float t1[6], t2[6], t3[6];
    elastic_v(m[0], vxi, mu, lam, t1);
    elastic_v(m[1], vet, mu, lam, t2);
    elastic_v(m[2], vzt, mu, lam, t3);
#pragma unroll
    for (int v = 0; v < 6; ++v) h[3 + v] = (t1[v] + t2[v] + t3[v]) * DT;
    // wave_rk.cpp:13-99
#pragma unroll
    for (int v = 0; v < 9; ++v) {
      const long long q = c + v * fs;
      switch (a.irk) {
        case 0: {
          const float mv = ldv(W + q);
          stv(a.t + q, mv + kB1 * h[v]);
          stv(a.wout + q, mv + kA2rk * h[v]);
        } break;
        case 1:
          stv(a.t + q, ldv(a.t + q) + kB2 * h[v]);
          stv(a.wout + q, ldv(a.wm + q) + kA3rk * h[v]);
          break;
        case 2:
          stv(a.t + q, ldv(a.t + q) + kB3 * h[v]);
          stv(a.wout + q, ldv(a.wm + q) + h[v]);
          break;
        default:
          stv(a.wout + q, ldv(a.t + q) + kB4 * h[v]);
      }
    }
  }
}

// Sets a kernel's dynamic shared-memory limit once per device (the bit set
// is per kernel; the attribute call is idempotent, so racing threads agree).
template <typename K>
cudaError_t top_smem_attr(K kern, std::atomic<unsigned long long> &done) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  const unsigned long long bit = dev < 64 ? 1ull << dev : 0ull;
  if (bit && (done.load(std::memory_order_acquire) & bit)) return cudaSuccess;
  e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(TopSmem));
  if (e == cudaSuccess && bit) done.fetch_or(bit, std::memory_order_acq_rel);
  return e;
}

template <typename S, int FB1, int FB2, int FB3>
cudaError_t launch_top_kernel(const StageArgs<S> &a, int i0, int i1, int j0, int j1,
                              cudaStream_t st) {
  static std::atomic<unsigned long long> done{0};
  auto kern = stage_top_kernel<S, FB1, FB2, FB3>;
  cudaError_t e = top_smem_attr(kern, done);
  if (e != cudaSuccess) return e;
  dim3 grid((i1 - i0 + TTX - 1) / TTX, (j1 - j0 + TTY - 1) / TTY), block(TTX, TTY);
  kern<<<grid, block, sizeof(TopSmem), st>>>(a, i0, i1, j0, j1);
  return cudaGetLastError();
}

template <typename S, int FB1, int FB2>
cudaError_t launch_top_fb3(const StageArgs<S> &a, int i0, int i1, int j0, int j1, cudaStream_t st) {
  return a.fb3 > 0 ? launch_top_kernel<S, FB1, FB2, 1>(a, i0, i1, j0, j1, st)
                   : launch_top_kernel<S, FB1, FB2, -1>(a, i0, i1, j0, j1, st);
}

}  // namespace

template <typename S> cudaError_t launch_stage_top(const StageArgs<S> &a, cudaStream_t st) {
  const Layout &L = a.L;
  const int np = a.nslab ? a.npml : 0;
  const int i0 = HALO + np, i1 = L.nx_ - HALO - np, j0 = HALO + np, j1 = L.ny_ - HALO - np;
  StageArgs<S> e = a;
  e.kbeg = L.nz_ - HALO - 3;
  e.kend = L.nz_ - HALO;
  if (i1 > i0 && j1 > j0) {
    cudaError_t err;
    if (a.fb1 > 0)
      err = a.fb2 > 0 ? launch_top_fb3<S, 1, 1>(a, i0, i1, j0, j1, st)
                      : launch_top_fb3<S, 1, -1>(a, i0, i1, j0, j1, st);
    else
      err = a.fb2 > 0 ? launch_top_fb3<S, -1, 1>(a, i0, i1, j0, j1, st)
                      : launch_top_fb3<S, -1, -1>(a, i0, i1, j0, j1, st);
    if (err != cudaSuccess) return err;
    if (np == 0) return cudaSuccess;
    // the exact-order kernel for the PML-slab columns only
    e.skip_i0 = i0; e.skip_i1 = i1; e.skip_j0 = j0; e.skip_j1 = j1;
  }
  return launch_stage_exact<S>(e, st);
}

template cudaError_t launch_stage_top<float>(const StageArgs<float> &, cudaStream_t);
template cudaError_t launch_stage_top<__half>(const StageArgs<__half> &, cudaStream_t);
template cudaError_t launch_stage_top<__nv_bfloat16>(const StageArgs<__nv_bfloat16> &, cudaStream_t);

}  // namespace cgfdm
