// Exact-order fused RK stage kernel.
//
// One thread per interior grid point performs, for its point, everything one
// RK stage of the reference does there (propagate.cpp:157-167):
//   the curvilinear MacCormack derivative x PML beta (wave_deriv.cpp:116-201)
//   or, on the top three layers, the traction-image free surface
//   (freeSurface.cpp:104-256); the ADE-CFS PML auxiliary update and the
//   -beta*Aux*DT correction of every slab that contains the point, in the
//   slab order x1 y1 z1 x2 y2 (pml_deriv.cpp:90-544,591-599); the surface
//   correction of the x/y slab auxiliaries (pml_freeSurface.cpp:65-117,
//   179-233); and the RK4 combination of wavefield and auxiliaries
//   (wave_rk.cpp:13-99, pml_rk.cpp:15-69).
// Every expression keeps the reference's operation order and this file is
// compiled with --fmad=false, so in FP32 the result is bit-identical to the
// reference's scalar CPU build.  In FP16/BF16 storage the intermediate
// roundings of the reference's FLOAT h_W buffer are reproduced with rnd<S>.
// The derivative input is read straight from global memory; this kernel is
// the correctness baseline, the streaming kernel is the fast path.
#include "device_common.cuh"
#include "kernels.h"

namespace cgfdm {
namespace {

template <typename S, typename R>
__device__ __forceinline__ R Lop(const S *w, long long c, long long o, int fb, R rDH) {
  // FB * (a_-1 W[-FB] + a0 W0 + a1 W[+FB] + a2 W[+2FB] + a3 W[+3FB]) * rDH
  long long q = fb * o;
  return (R)fb *
         ((R)kAm1 * (R)ldv(w + c - q) + (R)kA0 * (R)ldv(w + c) + (R)kA1 * (R)ldv(w + c + q) +
          (R)kA2 * (R)ldv(w + c + 2 * q) + (R)kA3 * (R)ldv(w + c + 3 * q)) *
         rDH;
}

// Elastic combination for one direction (wave_deriv.cpp:163-191).
template <typename R>
__device__ __forceinline__ void elastic(const R m[3], const R dv[3], const R dt[6], R mu, R lam,
                                        R b, R out[9]) {
  out[0] = (m[0] * dt[0] + m[1] * dt[3] + m[2] * dt[4]) * b;
  out[1] = (m[0] * dt[3] + m[1] * dt[1] + m[2] * dt[5]) * b;
  out[2] = (m[0] * dt[4] + m[1] * dt[5] + m[2] * dt[2]) * b;
  R div = m[0] * dv[0] + m[1] * dv[1] + m[2] * dv[2];
  out[3] = div * lam + (R)2.0f * mu * (m[0] * dv[0]);
  out[4] = div * lam + (R)2.0f * mu * (m[1] * dv[1]);
  out[5] = div * lam + (R)2.0f * mu * (m[2] * dv[2]);
  out[6] = (m[1] * dv[0] + m[0] * dv[1]) * mu;
  out[7] = (m[2] * dv[0] + m[0] * dv[2]) * mu;
  out[8] = (m[2] * dv[1] + m[1] * dv[2]) * mu;
}

template <typename S, typename R>
__device__ __forceinline__ void metric(const S *cjm, long long num, long long c, int dir, R m[3]) {
  m[0] = ldv(cjm + c + num * (3 * dir + 0));
  m[1] = ldv(cjm + c + num * (3 * dir + 1));
  m[2] = ldv(cjm + c + num * (3 * dir + 2));
}

// J-weighted traction rows at q (freeSurface.cpp:128-153).
template <typename S, typename R>
__device__ __forceinline__ void jt_rows(const S *W, const S *cjm, long long num, long long q, int dir,
                                        R r[3]) {
  R m0 = ldv(cjm + q + num * (3 * dir)), m1 = ldv(cjm + q + num * (3 * dir + 1)),
    m2 = ldv(cjm + q + num * (3 * dir + 2)), J = ldv(cjm + q + num * 9);
  r[0] = (m0 * (R)ldv(W + q + num * 3) + m1 * (R)ldv(W + q + num * 6) + m2 * (R)ldv(W + q + num * 7)) * J;
  r[1] = (m0 * (R)ldv(W + q + num * 6) + m1 * (R)ldv(W + q + num * 4) + m2 * (R)ldv(W + q + num * 8)) * J;
  r[2] = (m0 * (R)ldv(W + q + num * 7) + m1 * (R)ldv(W + q + num * 8) + m2 * (R)ldv(W + q + num * 5)) * J;
}

// The sign FB is dispatched to a template so that every index into the row
// array is a compile-time constant (the array stays in registers); the
// expression and its operation order are the same for both signs.
template <int FB, typename R> __device__ __forceinline__ R LJT_fb(const R *jt, R rDH) {
  return (R)FB *
         ((R)kAm1 * jt[3 - FB] + (R)kA0 * jt[3] + (R)kA1 * jt[3 + FB] + (R)kA2 * jt[3 + 2 * FB] +
          (R)kA3 * jt[3 + 3 * FB]) *
         rDH;
}
template <typename R> __device__ __forceinline__ R LJT(const R *jt, int fb, R rDH) {
  return fb > 0 ? LJT_fb<1>(jt, rDH) : LJT_fb<-1>(jt, rDH);
}

template <typename S>
__global__ void __launch_bounds__(256) stage_exact_kernel(StageArgs<S> a) {
  using R = typename Arith<S>::R;
  const int i = blockIdx.x * blockDim.x + threadIdx.x + HALO;
  const int j = blockIdx.y * blockDim.y + threadIdx.y + HALO;
  const int k = blockIdx.z * blockDim.z + threadIdx.z + a.kbeg;
  const int nx_ = a.L.nx_, ny_ = a.L.ny_, nz_ = a.L.nz_;
  if (i >= nx_ - HALO || j >= ny_ - HALO || k >= a.kend) return;
  if (i >= a.skip_i0 && i < a.skip_i1 && j >= a.skip_j0 && j < a.skip_j1) return;
  const long long num = a.L.fs;  // field stride
  const long long sx = 1, sy = a.L.px, sz = a.L.plane;
  const long long c = a.L.at(i, j, k);
  const int ktop = nz_ - HALO - 1;  // top interior layer (_nz - 1)
  const R rDH = a.rDH, DT = a.DT;
  const S *W = a.win;
  const S *cjm = a.cjm;
  const R *px = a.pml, *py = a.pml + 3 * nx_, *pz = a.pml + 3 * nx_ + 3 * ny_;
  const R mu = ldv(cjm + c + num * 10), lam = ldv(cjm + c + num * 11);
  const R b = ldv(cjm + c + num * 12);  // buoyancy already includes 1/Crho; *Crho below
  const int fbv[3] = {a.fb1, a.fb2, a.fb3};
  const long long stv3[3] = {sx, sy, sz};
  R h[9];

  if (k < ktop - 2) {
    // wave_deriv.cpp:116-201
    const R beta[3] = {px[nx_ + i], py[ny_ + j], pz[nz_ + k]};
    const R bu = b * (R)CRHO_OF<S>::v;
    R term[3][9];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      R m[3], dv[3], dt[6];
      metric(cjm, num, c, d, m);
#pragma unroll
      for (int v = 0; v < 3; ++v) dv[v] = Lop(W + v * num, c, stv3[d], fbv[d], rDH) * beta[d];
#pragma unroll
      for (int v = 0; v < 6; ++v) dt[v] = Lop(W + (3 + v) * num, c, stv3[d], fbv[d], rDH) * beta[d];
      elastic(m, dv, dt, mu, lam, bu, term[d]);
    }
#pragma unroll
    for (int v = 0; v < 9; ++v) h[v] = rnd<S>((term[0][v] + term[1][v] + term[2][v]) * DT);
  } else {
    // free_surface_deriv (freeSurface.cpp:104-256)
    const R bx = px[nx_ + i], by = py[ny_ + j];
    const R bu = b * (R)CRHO_OF<S>::v;
    const int ks = ktop - k + HALO;
    R jx[3][7], jy[3][7], jz[3][7], r[3];
#pragma unroll
    for (int l = 0; l < 7; ++l) {
      jt_rows(W, cjm, num, c + (l - HALO) * sx, 0, r);
      jx[0][l] = r[0]; jx[1][l] = r[1]; jx[2][l] = r[2];
      jt_rows(W, cjm, num, c + (l - HALO) * sy, 1, r);
      jy[0][l] = r[0]; jy[1][l] = r[1]; jy[2][l] = r[2];
    }
    // rows below the surface; zero at it; above it the antisymmetric image
    // -row(2 ks - l), recomputed at the mirrored point (the same bits)
#pragma unroll
    for (int l = 0; l < 7; ++l) {
      if (l < ks) {
        jt_rows(W, cjm, num, c + (l - HALO) * sz, 2, r);
        jz[0][l] = r[0]; jz[1][l] = r[1]; jz[2][l] = r[2];
      } else if (l == ks) {
        jz[0][l] = jz[1][l] = jz[2][l] = (R)0.0f;
      } else {
        jt_rows(W, cjm, num, c + (2 * ks - l - HALO) * sz, 2, r);
        jz[0][l] = -r[0]; jz[1][l] = -r[1]; jz[2][l] = -r[2];
      }
    }
    const R Jinv = (R)1.0f / (R)ldv(cjm + c + num * 9);
#pragma unroll
    for (int q = 0; q < 3; ++q)
      h[q] = rnd<S>(bu * Jinv *
                    (LJT(jx[q], a.fb1, rDH) * bx + LJT(jy[q], a.fb2, rDH) * by +
                     LJT(jz[q], a.fb3, rDH)) *
                    DT);
    R vxi[3], vet[3], vzt[3];
#pragma unroll
    for (int v = 0; v < 3; ++v) {
      vxi[v] = Lop(W + v * num, c, sx, a.fb1, rDH) * bx;
      vet[v] = Lop(W + v * num, c, sy, a.fb2, rDH) * by;
    }
    if (k == ktop) {
      const long long s2 = i + (long long)j * nx_;
      const R *DX = a.rdz + s2 * 9;
      const R *DY = a.rdz + (long long)nx_ * ny_ * 9 + s2 * 9;
#pragma unroll
      for (int q = 0; q < 3; ++q)
        vzt[q] = (DX[3 * q] * vxi[0] + DX[3 * q + 1] * vxi[1] + DX[3 * q + 2] * vxi[2]) +
                 (DY[3 * q] * vet[0] + DY[3 * q + 1] * vet[1] + DY[3 * q + 2] * vet[2]);
    } else if (k == ktop - 1) {
      const long long o = a.fb3 * sz;
#pragma unroll
      for (int v = 0; v < 3; ++v)
        vzt[v] = (R)a.fb3 * ((R)ldv(W + v * num + c + o) - (R)ldv(W + v * num + c)) * rDH;
    } else {
      const long long o = a.fb3 * sz;
#pragma unroll
      for (int v = 0; v < 3; ++v)
        vzt[v] = (R)a.fb3 *
                 ((R)kCf1 * (R)ldv(W + v * num + c) + (R)kCf2 * (R)ldv(W + v * num + c + o) +
                  (R)kCf3 * (R)ldv(W + v * num + c + 2 * o)) *
                 rDH;
    }
    R m[3][3], t1[9], t2[9], t3[9];
    const R z6[6] = {0, 0, 0, 0, 0, 0};
    metric(cjm, num, c, 0, m[0]);
    metric(cjm, num, c, 1, m[1]);
    metric(cjm, num, c, 2, m[2]);
    elastic(m[0], vxi, z6, mu, lam, bu, t1);
    elastic(m[1], vet, z6, mu, lam, bu, t2);
    elastic(m[2], vzt, z6, mu, lam, bu, t3);
#pragma unroll
    for (int v = 3; v < 9; ++v) h[v] = rnd<S>((t1[v] + t2[v] + t3[v]) * DT);
  }

  // PML slabs in the reference's order x1 y1 z1 x2 y2.
  for (int s = 0; s < a.nslab; ++s) {
    const SlabDev<R> &sl = a.slab[s];
    const int i0 = i - sl.off0, j0 = j - sl.off1, k0 = k - sl.off2;
    if (i0 < 0 || i0 >= sl.n0 || j0 < 0 || j0 >= sl.n1 || k0 < 0 || k0 >= sl.n2) continue;
    const int ax = sl.axis;
    const long long sa = ax == 0 ? sx : ax == 1 ? sy : sz;  // the slab's stride and sign
    const int fa = ax == 0 ? a.fb1 : ax == 1 ? a.fb2 : a.fb3;
    const int l = ax == 0 ? i : ax == 1 ? j : k;
    const R *prof = ax == 0 ? px : ax == 1 ? py : pz;
    const int nax = ax == 0 ? nx_ : ax == 1 ? ny_ : nz_;
    const R alpha = prof[l], bt = prof[nax + l], dl = prof[2 * nax + l];
    const R ad = dl + alpha;
    const long long pos = i0 + (long long)j0 * sl.n0 + (long long)k0 * sl.n0 * sl.n1;
    const long long np = sl.np;
    const R *ain = sl.ain + pos;  // value v at ain[v * np]
    R m[3], dv[3], dt[6], term[9], ha[9];
    metric(cjm, num, c, ax, m);
#pragma unroll
    for (int v = 0; v < 3; ++v) dv[v] = Lop(W + v * num, c, sa, fa, rDH) * dl;
#pragma unroll
    for (int v = 0; v < 6; ++v) dt[v] = Lop(W + (3 + v) * num, c, sa, fa, rDH) * dl;
    elastic(m, dv, dt, mu, lam, b * (R)CRHO_OF<S>::v, term);
#pragma unroll
    for (int v = 0; v < 9; ++v) {
      const R av = ain[v * np];
      ha[v] = (term[v] - ad * av) * DT;
      h[v] = rnd<S>(h[v] + -bt * av * DT);
    }
    if (k == ktop && ax != 2) {
      // pml_freeSurface.cpp: surface-gradient correction of the stress aux
      const long long s2 = i + (long long)j * nx_;
      const R *M = a.rdz + (ax == 0 ? 0 : (long long)nx_ * ny_ * 9) + s2 * 9;
      R vd[3], vz[3], zt[3], t[9];
      const R z6[6] = {0, 0, 0, 0, 0, 0};
#pragma unroll
      for (int v = 0; v < 3; ++v) vd[v] = Lop(W + v * num, c, sa, fa, rDH) * dl;
#pragma unroll
      for (int q = 0; q < 3; ++q) vz[q] = M[3 * q] * vd[0] + M[3 * q + 1] * vd[1] + M[3 * q + 2] * vd[2];
      metric(cjm, num, c, 2, zt);
      elastic(zt, vz, z6, mu, lam, (R)0.0f, t);
#pragma unroll
      for (int v = 3; v < 9; ++v) ha[v] = ha[v] + t[v] * DT;
    }
    // pml_rk.cpp:15-69
    R *aout = sl.aout + pos;
    R *at = sl.at + pos;
    const R *am = sl.am + pos;
#pragma unroll
    for (int v = 0; v < 9; ++v) {
      const R hv = ha[v];
      const long long q = v * np;
      switch (a.irk) {
        case 0: {
          const R mv = ain[q];
          at[q] = mv + (R)kB1 * hv;
          aout[q] = mv + (R)kA2rk * hv;
        } break;
        case 1:
          at[q] = at[q] + (R)kB2 * hv;
          aout[q] = am[q] + (R)kA3rk * hv;
          break;
        case 2:
          at[q] = at[q] + (R)kB3 * hv;
          aout[q] = am[q] + hv;
          break;
        default:
          aout[q] = at[q] + (R)kB4 * hv;
      }
    }
  }

  // wave_rk.cpp:13-99
#pragma unroll
  for (int v = 0; v < 9; ++v) {
    const long long q = c + v * num;
    const R hv = h[v];
    switch (a.irk) {
      case 0: {
        const R mv = ldv(W + q);
        stv(a.t + q, mv + (R)kB1 * hv);
        stv(a.wout + q, mv + (R)kA2rk * hv);
      } break;
      case 1: {
        const R tv = ldv(a.t + q), mv = ldv(a.wm + q);
        stv(a.t + q, tv + (R)kB2 * hv);
        stv(a.wout + q, mv + (R)kA3rk * hv);
      } break;
      case 2: {
        const R tv = ldv(a.t + q), mv = ldv(a.wm + q);
        stv(a.t + q, tv + (R)kB3 * hv);
        stv(a.wout + q, mv + hv);
      } break;
      default: {
        const R tv = ldv(a.t + q);
        stv(a.wout + q, tv + (R)kB4 * hv);
      }
    }
  }
}

}  // namespace

template <typename S> cudaError_t launch_stage_exact(const StageArgs<S> &a, cudaStream_t st) {
  // one plane per block: the three free-surface layers of the streaming path
  // leave no thread idle, and a block's 8 rows share their y-neighbour rows
  dim3 block(32, 8, 1);
  if (a.kend <= a.kbeg) return cudaSuccess;
  dim3 grid((a.L.nx_ - 2 * HALO + 31) / 32, (a.L.ny_ - 2 * HALO + 7) / 8, a.kend - a.kbeg);
  stage_exact_kernel<S><<<grid, block, 0, st>>>(a);
  return cudaGetLastError();
}

template cudaError_t launch_stage_exact<float>(const StageArgs<float> &, cudaStream_t);
template cudaError_t launch_stage_exact<__half>(const StageArgs<__half> &, cudaStream_t);
template cudaError_t launch_stage_exact<__nv_bfloat16>(const StageArgs<__nv_bfloat16> &, cudaStream_t);
template cudaError_t launch_stage_exact<double>(const StageArgs<double> &, cudaStream_t);

}  // namespace cgfdm
