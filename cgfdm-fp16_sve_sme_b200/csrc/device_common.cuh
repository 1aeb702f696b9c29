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

// HBM layout of every 3-D field (wavefield components, coefficients): the
// reference's padded grid (_nx_ x _ny_ x _nz_, halo 3, x fastest) with the
// rows shifted by xoff elements and padded to a pitch that is a multiple of
// 32 elements, so that the first interior column (i = 3) and every 32-column
// tile origin i = 3 + 32 t start on a 128-byte boundary (whole L2 lines for
// the tile loads and stores) and the halo box origin 16 bytes before it is a
// legal TMA start.  The pad columns are zero.
struct Layout {
  int nx_, ny_, nz_;  // padded extents
  int px;             // row pitch in elements
  int xoff;           // row shift in elements
  long long plane;    // px * ny_
  long long fs;       // field stride (elements), a multiple of 32
  __host__ __device__ __forceinline__ long long at(int i, int j, int k) const {
    return (long long)(i + xoff) + (long long)j * px + (long long)k * plane;
  }
};

__host__ __device__ inline Layout make_layout(int nx, int ny, int nz, int elem_bytes) {
  Layout L;
  L.nx_ = nx + 2 * HALO;
  L.ny_ = ny + 2 * HALO;
  L.nz_ = nz + 2 * HALO;
  L.xoff = (128 / elem_bytes) - HALO;  // 29 (4-byte), 61 (2-byte), 13 (8-byte)
  L.px = ((L.nx_ + L.xoff) + 31) / 32 * 32;
  L.plane = (long long)L.px * L.ny_;
  L.fs = (L.plane * L.nz_ + 31) / 32 * 32;
  return L;
}

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
// the derivative axis, and its four auxiliary buffers of type A (float except
// in the FP64 run).  On the device the 9 auxiliary fields of a slab are
// stored field-major, [9][np] (value v of slab point pos at v * np + pos,
// pos x-fastest), so that a warp's consecutive points read and write
// consecutive addresses; the host interface keeps the reference's [pos][9]
// (pml_deriv.cpp:199-207) and converts.
template <typename A> struct SlabDev {
  int n0, n1, n2;        // extent along x, y, z
  int off0, off1, off2;  // padded index of the slab origin
  int axis;              // 0 = x, 1 = y, 2 = z
  long long np;          // n0 * n1 * n2
  const A *ain;          // stage-input auxiliaries
  A *aout;               // stage-output auxiliaries
  const A *am;           // step-start auxiliaries
  A *at;                 // RK accumulator of the auxiliaries
};

// Everything one RK stage reads and writes.
template <typename S> struct StageArgs {
  const S *win;          // stage input wavefield, 9 fields
  S *wout;               // stage output wavefield
  const S *wm;           // step-start wavefield (the RK "m" state)
  S *t;                  // RK accumulator
  const S *cjm;          // 13 coefficient fields
  const typename Arith<S>::R *rdz;  // 2 x (_nx_*_ny_) x 9 (_rDZ_DX then _rDZ_DY)
  const typename Arith<S>::R *pml;  // alpha, beta, d for x (nx_), y (ny_), z (nz_)
  SlabDev<typename Arith<S>::R> slab[5];  // x1 y1 z1 x2 y2
  int nslab;
  Layout L;
  int kbeg, kend;        // padded z range of the points this launch updates
  int npml;
  float rDH, DT;
  int fb1, fb2, fb3, irk;
  // planes per upper z chunk of the streaming kernel's work items (0: about
  // 40 items per CTA slot, chunks of at least 16 planes)
  int chunk;
  // exact-order kernel only: points whose column lies in [skip_i0, skip_i1) x
  // [skip_j0, skip_j1) are left to another kernel (empty box: none)
  int skip_i0, skip_i1, skip_j0, skip_j1;
  // failure-detection tests only: the streaming kernel leaves one input-plane
  // load of its first work item unissued, so that the bounded wait on it
  // expires (no memory is touched); 0 in every normal launch
  int drop_one_load;
};

}  // namespace cgfdm
