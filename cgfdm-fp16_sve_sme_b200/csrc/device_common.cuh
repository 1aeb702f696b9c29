// Shared device-side definitions of the CGFDM hot path.
//
// Storage types S: float (FP32), __half (scaled FP16), __nv_bfloat16 (scaled
// BF16), double (FP64 accuracy oracle).  Arithmetic runs in R = float for the
// first three and double for FP64.
#pragma once
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cstdint>

namespace cgfdm {

constexpr int HALO = 3;
constexpr int NFIELD = 9;  // Vx Vy Vz Txx Tyy Tzz Txy Txz Tyz

// MacCormack one-sided 5-point coefficients (macro.h:123-128), the 2- and
// 3-point one-sided surface operators (macro.h:149-151) and RK4 weights
// (macro.h:138-147), as the reference's float literals.
constexpr float kAm1 = -0.30874f, kA0 = -0.6326f, kA1 = 1.2330f, kA2 = -0.3334f,
                kA3 = 0.04168f;
constexpr float kCf1 = -1.16666667f, kCf2 = 1.33333333f, kCf3 = -0.16666667f;
constexpr float kB1 = 0.16666667f, kB2 = 0.33333333f, kB3 = 0.33333333f, kB4 = 0.16666667f,
                kA2rk = 0.5f, kA3rk = 0.5f;

template <typename S> struct Arith { using R = float; };
template <> struct Arith<double> { using R = double; };

__device__ __forceinline__ float ldv(const float *p) { return *p; }
__device__ __forceinline__ float ldv(const __half *p) { return __half2float(*p); }
__device__ __forceinline__ float ldv(const __nv_bfloat16 *p) { return __bfloat162float(*p); }
__device__ __forceinline__ double ldv(const double *p) { return *p; }

__device__ __forceinline__ void stv(float *p, float v) { *p = v; }
__device__ __forceinline__ void stv(__half *p, float v) { *p = __float2half_rn(v); }
__device__ __forceinline__ void stv(__nv_bfloat16 *p, float v) { *p = __float2bfloat16_rn(v); }
__device__ __forceinline__ void stv(double *p, double v) { *p = v; }

// Value as it reads back after a store to S (round to the storage format).
template <typename S, typename R> __device__ __forceinline__ R rnd(R v) {
  S t;
  stv(&t, v);
  return ldv(&t);
}

// One PML slab on the device: slab-local box, offset into the padded grid,
// the derivative axis, and its four auxiliary buffers ([npos][9] values of
// type A, AoS as pml_deriv.cpp:199-207; float except in the FP64 run).
template <typename A> struct SlabDev {
  int n0, n1, n2;        // extent along x, y, z
  int off0, off1, off2;  // padded index of the slab origin
  int axis;              // 0 = x, 1 = y, 2 = z
  const A *ain;          // stage-input auxiliaries
  A *aout;               // stage-output auxiliaries
  const A *am;           // step-start auxiliaries
  A *at;                 // RK accumulator of the auxiliaries
};

// Everything one RK stage reads and writes.
template <typename S> struct StageArgs {
  const S *win;          // stage input wavefield, 9 x num
  S *wout;               // stage output wavefield
  const S *wm;           // step-start wavefield (the RK "m" state)
  S *t;                  // RK accumulator, 9 x num
  const S *cjm;          // 13 x num
  const typename Arith<S>::R *rdz;  // 2 x nsurf x 9 (_rDZ_DX then _rDZ_DY)
  const typename Arith<S>::R *pml;  // alpha, beta, d for x (nx_), y (ny_), z (nz_)
  SlabDev<typename Arith<S>::R> slab[5];  // x1 y1 z1 x2 y2
  int nslab;
  int nx_, ny_, nz_;     // padded extents
  long long num;
  int npml;
  float rDH, DT;
  int fb1, fb2, fb3, irk;
};

}  // namespace cgfdm
