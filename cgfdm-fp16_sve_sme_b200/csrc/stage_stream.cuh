// TMA-staged z-streaming fused RK stage (the fast path).  Included by one
// translation unit per storage type (stage_stream_f32.cu, _f16.cu, _bf16.cu),
// each instantiating its own kernels.
//
// Persistent CTAs (one 512-thread CTA per SM) pull work items from an atomic
// queue; an item is a 32 x 16 column tile and a chunk of z planes, ordered so
// that concurrently running items are neighbours at the same depth (their
// halo rows meet in L2).  Within an item the CTA sweeps z against the
// MacCormack z direction (upward when FB3 = -1, downward when FB3 = +1), so
// the one-sided z stencil of output plane k only needs plane k + dir beyond
// it: a 5-plane register window per thread holds the z stencil, and shared
// memory holds three rings fed by 4-D TMA tile loads (cp.async.bulk.tensor,
// no multicast), each slot guarded by an mbarrier:
//   W ring (3): the 9 wavefield components of one input plane with the x/y
//               halo of the one-sided stencils (x origin 16-byte aligned);
//   C ring (2): the 9 metrics and (mu, lambda, buoyancy) of one output plane;
//   M ring (2): the RK step state m and accumulator t of one output plane
//               (stages that read them);
// (4/3/3 slots in the 16-bit PML variant, see Geo).
// With 16-bit storage the interior variant converts each W plane to FP32 once
// in shared memory (two plane buffers), so its stencils read FP32 like the
// FP32 kernel instead of converting every tap.
// Every operand of the stage therefore arrives asynchronously ahead of use;
// only the PML auxiliaries (a minority of points) are read with plain loads,
// by a second instantiation (PMLK) that runs the tiles and bottom chunks
// touching a PML slab.
// Derivative, elastic combination, PML ADE update and the RK4 combination of
// wavefield and auxiliaries are fused: each field is read and written once
// per stage, stores are whole 128-byte lines per warp row.
//
// Arithmetic: FP32 with FMA contraction, two fields per packed FP32x2
// instruction in the stencil sums, increments and RK update; the stencil
// sums use the bare MacCormack weights, and each direction's elastic
// combination is formed once and scaled by the sign FB, 1/DH and the PML beta
// (main update) or d (auxiliary update), equal to the reference up to
// rounding.  The three free-surface layers are left to the exact-order kernel.
//
// Every mbarrier wait is bounded (2^31 clock cycles); on expiry the CTA sets
// the error flag, drains the copies it issued (again bounded) and returns.
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cstdint>
#include <cstring>
#include <memory>
#include <string>
#include <type_traits>

#include "engine.h"
#include "kernels.h"

namespace cgfdm {
namespace {

constexpr int TX = 32;
constexpr long long kWaitCycles = 1LL << 31;

// Tile and shared-memory geometry for storage type S and tile height TYv
// (16: one 512-thread CTA per SM; 8: 256-thread CTAs, two per SM when their
// shared memory fits, so one CTA's per-plane barrier overlaps the other's work).
template <typename S, int TYv, bool PMLK = false> struct Geo {
  static constexpr int TY = TYv, NTHR = TX * TYv;
  static constexpr int BY = TYv + 4;  // y box: 1 or 3 rows before the tile, 3 or 1 after
  static constexpr int MINB = TYv == 8 ? 2 : 1;
  static constexpr int ES = (int)sizeof(S);
  static constexpr int HB = 16 / ES;                             // elements per 16 bytes
  static constexpr int BX = ((HB + TX + 3) + HB - 1) / HB * HB;  // x box, aligned origin
  static constexpr int W_BYTES = ((9 * BY * BX * ES) + 127) / 128 * 128;
  static constexpr int C_BYTES = 12 * NTHR * ES;                 // 9 metrics + mu, lambda, b
  static constexpr int M_BYTES = 18 * NTHR * ES;                 // m (9) and t (9)
  // 16-bit storage, interior variant: each W plane is converted to FP32 once,
  // into one of two plane buffers (by plane parity) that the x and y stencils
  // read.  The PML variant (latency-bound) reads the 16-bit planes directly
  // and keeps deeper rings instead.
  static constexpr bool CONV = ES != 4 && !PMLK;
  static constexpr int NW = ES == 4 || CONV ? 3 : 4;
  static constexpr int NC = ES == 4 || CONV ? 2 : 3;
  static constexpr int NM = NC;
  static constexpr int F_BYTES = CONV ? ((9 * BY * BX * 4) + 127) / 128 * 128 : 0;
  static constexpr int OFF_C = NW * W_BYTES;
  static constexpr int OFF_M = OFF_C + NC * C_BYTES;
  static constexpr int OFF_F = OFF_M + NM * M_BYTES;
  static constexpr int OFF_BAR = OFF_F + 2 * F_BYTES;
  static constexpr int SMEM = OFF_BAR + 8 * (NW + NC + NM) + 128;
  static_assert(SMEM <= 232448, "shared memory budget");
  static_assert(MINB == 1 || MINB * (SMEM + 1024) <= 233472, "two CTAs per SM");
};

// Four 16-bit values at p (8-byte aligned) as four floats.
__device__ __forceinline__ float4 cvt4(const __half *p) {
  const uint2 r = *(const uint2 *)p;
  const float2 a = __half22float2(*(const __half2 *)&r.x), b = __half22float2(*(const __half2 *)&r.y);
  return make_float4(a.x, a.y, b.x, b.y);
}
__device__ __forceinline__ float4 cvt4(const __nv_bfloat16 *p) {
  const uint2 r = *(const uint2 *)p;
  const float2 a = __bfloat1622float2(*(const __nv_bfloat162 *)&r.x),
               b = __bfloat1622float2(*(const __nv_bfloat162 *)&r.y);
  return make_float4(a.x, a.y, b.x, b.y);
}
__device__ __forceinline__ float4 cvt4(const float *p) { return *(const float4 *)p; }

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint32_t bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(bar), "r"(parity), "r"(1000000u)
      : "memory");
  return ok != 0;
}
__device__ __forceinline__ bool mbar_wait_bounded(uint32_t bar, uint32_t parity) {
  const long long t0 = clock64();
  while (!mbar_try_wait(bar, parity))
    if (clock64() - t0 > kWaitCycles) return false;
  return true;
}
__device__ __forceinline__ void tma_load_4d(uint32_t dst, const CUtensorMap *map, int x, int y,
                                            int z, int f, uint32_t bar) {
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3, %4, %5}], [%6];" ::"r"(dst),
      "l"(map), "r"(x), "r"(y), "r"(z), "r"(f), "r"(bar)
      : "memory");
}

// Elastic combination of one direction from its raw derivatives
// (wave_deriv.cpp:163-191 without the PML factor): m = metric row,
// L = d(Vx,Vy,Vz,Txx,Tyy,Tzz,Txy,Txz,Tyz).  Velocity rows include b.
__device__ __forceinline__ void elastic9(const float m[3], const float L[9], float mu, float lam,
                                         float b, float E[9]) {
  E[0] = (m[0] * L[3] + m[1] * L[6] + m[2] * L[7]) * b;
  E[1] = (m[0] * L[6] + m[1] * L[4] + m[2] * L[8]) * b;
  E[2] = (m[0] * L[7] + m[1] * L[8] + m[2] * L[5]) * b;
  const float mvx = m[0] * L[0], mvy = m[1] * L[1], mvz = m[2] * L[2];
  const float div = (mvx + mvy + mvz) * lam;
  const float tmu = 2.0f * mu;
  E[3] = div + tmu * mvx;
  E[4] = div + tmu * mvy;
  E[5] = div + tmu * mvz;
  E[6] = (m[1] * L[0] + m[0] * L[1]) * mu;
  E[7] = (m[2] * L[0] + m[0] * L[2]) * mu;
  E[8] = (m[2] * L[1] + m[1] * L[2]) * mu;
}

// The interior variant's form of the three directions' elastic combinations
// and their sum into the stage increment (wave_deriv.cpp:163-201,
// reassociated; equal up to rounding): mu, lambda and the buoyancy are the
// point's own, so each direction adds its metric row scaled by the
// direction factor g times the derivatives, and mu, lambda and b multiply
// the sums once (the PML variant keeps the per-direction combination E,
// which its auxiliary update needs).
struct ElasticSum {
  float v0, v1, v2;  // velocity rows, before b
  float nx, ny, nz;  // normal terms m_x dVx, m_y dVy, m_z dVz
  float s6, s7, s8;  // shear terms, before mu
  template <bool FIRST>
  __device__ __forceinline__ void add(const float m[3], float g, const float L[9]) {
    const float a0 = g * m[0], a1 = g * m[1], a2 = g * m[2];
    v0 = fmaf(a2, L[7], fmaf(a1, L[6], FIRST ? a0 * L[3] : fmaf(a0, L[3], v0)));
    v1 = fmaf(a2, L[8], fmaf(a1, L[4], FIRST ? a0 * L[6] : fmaf(a0, L[6], v1)));
    v2 = fmaf(a2, L[5], fmaf(a1, L[8], FIRST ? a0 * L[7] : fmaf(a0, L[7], v2)));
    nx = FIRST ? a0 * L[0] : fmaf(a0, L[0], nx);
    ny = FIRST ? a1 * L[1] : fmaf(a1, L[1], ny);
    nz = FIRST ? a2 * L[2] : fmaf(a2, L[2], nz);
    s6 = fmaf(a0, L[1], FIRST ? a1 * L[0] : fmaf(a1, L[0], s6));
    s7 = fmaf(a0, L[2], FIRST ? a2 * L[0] : fmaf(a2, L[0], s7));
    s8 = fmaf(a1, L[2], FIRST ? a2 * L[1] : fmaf(a2, L[1], s8));
  }
  __device__ __forceinline__ void finish(float mu, float lam, float b, float h[9]) const {
    h[0] = v0 * b;
    h[1] = v1 * b;
    h[2] = v2 * b;
    const float div = (nx + ny + nz) * lam, tmu = 2.0f * mu;
    h[3] = fmaf(tmu, nx, div);
    h[4] = fmaf(tmu, ny, div);
    h[5] = fmaf(tmu, nz, div);
    h[6] = s6 * mu;
    h[7] = s7 * mu;
    h[8] = s8 * mu;
  }
};

// Packed FP32x2 arithmetic (FFMA2 / FMUL2 on sm_100): one instruction applies
// the same operation to two fields of a point, each lane rounding exactly as
// the scalar operation would.
__device__ __forceinline__ float2 pk(float a, float b) { return make_float2(a, b); }
__device__ __forceinline__ float2 pk(float a) { return make_float2(a, a); }

// One-sided 5-point sum with the MacCormack weights as they stand
// (macro.h:126-136), taps in the order (-FB, 0, +FB, +2FB, +3FB); the sign FB
// and 1/DH multiply the direction's elastic combination afterwards (it is
// linear in the derivatives).
__device__ __forceinline__ float2 stencil2(float2 t0, float2 t1, float2 t2, float2 t3, float2 t4) {
  float2 s = __fmul2_rn(pk(kAm1), t0);
  s = __ffma2_rn(pk(kA0), t1, s);
  s = __ffma2_rn(pk(kA1), t2, s);
  s = __ffma2_rn(pk(kA2), t3, s);
  return __ffma2_rn(pk(kA3), t4, s);
}
__device__ __forceinline__ float stencil1(float t0, float t1, float t2, float t3, float t4) {
  return fmaf(kA3, t4, fmaf(kA2, t3, fmaf(kA1, t2, fmaf(kA0, t1, kAm1 * t0))));
}

__device__ __forceinline__ unsigned slab_pos(const SlabDev<float> &sl, int i, int j, int k) {
  return (unsigned)((i - sl.off0) + (j - sl.off1) * sl.n0 + (k - sl.off2) * sl.n0 * sl.n1);
}

// PML auxiliary update of one slab point (pml_deriv.cpp:199-237,
// pml_rk.cpp:15-69) given the direction's elastic combination E; adds
// -beta * Aux * DT into h (the point's slab corrections).  The auxiliaries are field-major on the device
// (value v at v * np + pos), so the lanes of a warp, consecutive points of
// the slab, touch consecutive addresses.
//
// A point's inputs are the auxiliary input (part 1), what the stage adds the
// increment to (part 2: m in stages 1-2, t in stage 3) and t (part 4, stages
// 1-2).  pml_load<RK> loads the parts in a mask for all nine fields, so that
// the loads can be issued at the top of a plane iteration and their latency
// overlaps the stencil work; pml_apply<RK> is told which parts are already
// in registers (a compile-time or a per-thread mask), loads the others
// (three fields at a time, each group's loads before its stores) and updates.
template <int RK> constexpr int pml_parts() { return RK == 0 ? 1 : RK == 3 ? 3 : 7; }
struct PmlIn {
  float a[9], b[9], t[9];
};
template <int RK>
__device__ __forceinline__ void pml_load_fields(const SlabDev<float> &sl, unsigned pos, int v0,
                                                int nv, int mask, PmlIn &in) {
  constexpr int P = pml_parts<RK>();
  const unsigned np = (unsigned)sl.np;
#pragma unroll
  for (int v = v0; v < v0 + nv; ++v) {
    const unsigned q = v * np + pos;
    if ((P & 1) && (mask & 1)) in.a[v] = sl.ain[q];
    if ((P & 2) && (mask & 2)) in.b[v] = RK == 3 ? sl.at[q] : sl.am[q];
    if ((P & 4) && (mask & 4)) in.t[v] = sl.at[q];
  }
}
template <int RK>
__device__ __forceinline__ void pml_load(const SlabDev<float> &sl, unsigned pos, int mask, PmlIn &in) {
  pml_load_fields<RK>(sl, pos, 0, 9, mask, in);
}
// L1 prefetch of the parts in a mask (no registers held), for the parts the
// stage needs but does not keep in registers across the stencils.
template <int RK>
__device__ __forceinline__ void pml_prefetch(const SlabDev<float> &sl, unsigned pos, int mask) {
  constexpr int P = pml_parts<RK>();
  const unsigned np = (unsigned)sl.np;
#pragma unroll
  for (int v = 0; v < 9; ++v) {
    const unsigned q = v * np + pos;
    if ((P & 2) && (mask & 2))
      asm volatile("prefetch.global.L1 [%0];" ::"l"(RK == 3 ? sl.at + q : sl.am + q));
    if ((P & 4) && (mask & 4)) asm volatile("prefetch.global.L1 [%0];" ::"l"(sl.at + q));
  }
}
template <int RK>
__device__ __forceinline__ void pml_apply(const SlabDev<float> &sl, unsigned pos, const float E[9],
                                          float dl, float ad, float bt, float DT, float cB,
                                          float cA, float h[9], int held, PmlIn &in) {
  const unsigned np = (unsigned)sl.np;
  float *__restrict__ aout = sl.aout;
  float *__restrict__ at = sl.at;
#pragma unroll
  for (int g = 0; g < 9; g += 3) {
    pml_load_fields<RK>(sl, pos, g, 3, 7 & ~held, in);
#pragma unroll
    for (int v = g; v < g + 3; ++v) {
      const unsigned q = v * np + pos;
      const float a = in.a[v];
      const float ha = (dl * E[v] - ad * a) * DT;
      h[v] -= bt * a * DT;
      if (RK == 0) {
        at[q] = a + kB1 * ha;
        aout[q] = a + kA2rk * ha;
      } else if (RK == 1) {
        at[q] = in.t[v] + cB * ha;
        aout[q] = in.b[v] + cA * ha;
      } else {
        aout[q] = in.b[v] + kB4 * ha;
      }
    }
  }
}
// The parts of a slab point loaded at the top of its plane iteration: all of
// them in stages 0 and 3; the auxiliary input alone in stages 1-2, where
// holding all three parts (27 registers) across the stencils spills.  The
// loads are for the point's first slab in application order (x, then y,
// then the bottom z slab); a corner point loads its later slabs in place.
template <int RK> constexpr int hoist_parts() { return RK == 1 ? 1 : pml_parts<RK>(); }

struct Maps {
  CUtensorMap w;   // stage input wavefield, box BX x BY x 1 x 9
  CUtensorMap c9;  // coefficients, box 32 x TY x 1 x 9 (metrics)
  CUtensorMap c3;  // coefficients, box 32 x TY x 1 x 3 (mu, lambda, b at field 10)
  CUtensorMap m;   // step-start wavefield, box 32 x TY x 1 x 9
  CUtensorMap t;   // RK accumulator, box 32 x TY x 1 x 9
};
struct MapSet {
  Maps ty16, ty8;  // the same buffers, boxes for tile heights 16 and 8
  Maps pair;       // 16-bit storage: 64 x 8 tiles of the paired-point kernel
};

// Work items of one launch.  The z range [kbeg, kend) is cut at kz, the top
// of the bottom PML slab: nzc chunks of chunk_p planes below it and nic
// chunks of chunk_i planes above it.  Tiles are 32 x 16 columns on an
// ntx x nty grid; tiles [bx_lo, bx_hi) x [by_lo, by_hi) touch no x or y PML
// slab.  The interior launch covers interior tiles x upper chunks; the PML
// launch covers every tile of the lower chunks and the edge tiles (all
// others) of the upper chunks.  Tiles vary fastest, so the items running at
// one time are neighbours at the same depth.
struct Work {
  int ntx, nty, bx_lo, bx_hi, by_lo, by_hi;
  int kz, nzc, chunk_p, nic, chunk_i;
  int nitems;
  int *counter;
};

template <bool PMLK>
__device__ __forceinline__ void item_of(const Work &w, int item, int &bxi, int &byi, int &kb,
                                        int &ke, int kbeg, int kend) {
  int chk;
  if (!PMLK) {
    const int nxi = w.bx_hi - w.bx_lo, ti = nxi * (w.by_hi - w.by_lo);
    const int t = item % ti;
    chk = w.nzc + item / ti;
    bxi = w.bx_lo + t % nxi;
    byi = w.by_lo + t / nxi;
  } else {
    const int tall = w.ntx * w.nty;
    if (item < w.nzc * tall) {
      chk = item / tall;
      bxi = (item % tall) % w.ntx;
      byi = (item % tall) / w.ntx;
    } else {
      const int nside = w.bx_lo + (w.ntx - w.bx_hi);
      const int nedge = tall - (w.bx_hi - w.bx_lo) * (w.by_hi - w.by_lo);
      const int q = item - w.nzc * tall;
      chk = w.nzc + q / nedge;
      int e = q % nedge;
      if (e < w.by_lo * w.ntx) {
        byi = e / w.ntx;
        bxi = e % w.ntx;
      } else {
        e -= w.by_lo * w.ntx;
        if (e < (w.by_hi - w.by_lo) * nside) {
          byi = w.by_lo + e / nside;
          const int r = e % nside;
          bxi = r < w.bx_lo ? r : w.bx_hi + (r - w.bx_lo);
        } else {
          e -= (w.by_hi - w.by_lo) * nside;
          byi = w.by_hi + e / w.ntx;
          bxi = e % w.ntx;
        }
      }
    }
  }
  if (chk < w.nzc) {
    kb = kbeg + chk * w.chunk_p;
    ke = min(kb + w.chunk_p, w.kz);
  } else {
    kb = w.kz + (chk - w.nzc) * w.chunk_i;
    ke = min(kb + w.chunk_i, kend);
  }
}

// Where the work items of a launch come from: one scenario (SingleSrc) or
// up to kBatchMax scenarios of one batch (BatchSrc), each with its own stage
// arguments, tensor maps and item geometry; the items of a batch are numbered
// scenario after scenario.
template <typename S> struct SingleSrc {
  const Maps &m;
  const StageArgs<S> &a;
  const Work &w;
  __device__ int *counter() const { return w.counter; }
  __device__ int nitems() const { return w.nitems; }
  __device__ int entry_of(int item, int &local) const {
    local = item;
    return 0;
  }
  __device__ const StageArgs<S> &args(int) const { return a; }
  __device__ const Maps &maps(int) const { return m; }
  __device__ const Work &work(int) const { return w; }
};

constexpr int kBatchMax = 16;
template <typename S> struct BatchParams {
  Maps maps[kBatchMax];
  StageArgs<S> args[kBatchMax];
  Work work[kBatchMax];
  int item_end[kBatchMax];  // items of scenarios 0..e together
  int n;
  int *counter;
};

template <typename S> struct BatchSrc {
  const BatchParams<S> &p;
  __device__ int *counter() const { return p.counter; }
  __device__ int nitems() const { return p.item_end[p.n - 1]; }
  __device__ int entry_of(int item, int &local) const {
    int e = 0;
    while (e + 1 < p.n && item >= p.item_end[e]) ++e;
    local = item - (e ? p.item_end[e - 1] : 0);
    return e;
  }
  __device__ const StageArgs<S> &args(int e) const { return p.args[e]; }
  __device__ const Maps &maps(int e) const { return p.maps[e]; }
  __device__ const Work &work(int e) const { return p.work[e]; }
};

template <typename S, int TYv, int FB1, int FB2, int FB3, bool PMLK, int RK, typename Src>
__device__ __forceinline__ void stream_body(const Src &src, int *err) {
  using G = Geo<S, TYv, PMLK>;
  constexpr int TY = G::TY, NTHR = G::NTHR, BY = G::BY;
  constexpr int NW = G::NW, NC = G::NC, NM = G::NM, BX = G::BX;
  constexpr int DIR = -FB3;  // sweep direction in z
  extern __shared__ unsigned char smem_raw[];
  // 128-byte aligned base, derived by pointer arithmetic on the shared array
  // (not through an integer) so that every access through it compiles to a
  // shared-memory load with a 32-bit address
  unsigned char *smem = smem_raw + ((128u - (smem_u32(smem_raw) & 127u)) & 127u);
  uint64_t *bw = (uint64_t *)(smem + G::OFF_BAR);
  uint64_t *bc = bw + NW;
  uint64_t *bm = bc + NC;
  __shared__ int s_item, s_bad;

  const int tid = threadIdx.x;
  const int c = tid % TX, r = tid / TX;
  const int cidx = r * TX + c;

  if (tid == 0) {
    s_bad = 0;
    for (int s = 0; s < NW + NC + NM; ++s) mbar_init(smem_u32(&bw[s]), 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();

  // ring fill counters, continued across work items
  unsigned fw0 = 0, fc0 = 0, fm0 = 0;

  for (;;) {
    if (tid == 0) s_item = atomicAdd(src.counter(), 1);
    __syncthreads();
    const int item = s_item;
    if (item >= src.nitems() || s_bad) break;
    int local;
    const int e = src.entry_of(item, local);
    const StageArgs<S> &a = src.args(e);
    const Maps &maps = src.maps(e);
    const Work &wk = src.work(e);
    const Layout L = a.L;
    // stages 1 and 2 (RK = 1) differ only in the weights of the t and output updates
    constexpr bool need_m = RK == 1, need_t = RK >= 1;
    const float cB = a.irk == 2 ? kB3 : kB2, cA = a.irk == 2 ? 1.0f : kA3rk;
    const uint32_t m_bytes = (need_m ? 9 : 0) * NTHR * G::ES + (need_t ? 9 : 0) * NTHR * G::ES;
    const float rDH = a.rDH, DT = a.DT;
    // the MacCormack sign and 1/DH of each direction, applied to its elastic
    // combination (the stencil sums use the bare weights)
    const float gx = FB1 * rDH, gy = FB2 * rDH, gz = FB3 * rDH;
    const float *px = a.pml, *py = a.pml + 3 * L.nx_, *pz = a.pml + 3 * L.nx_ + 3 * L.ny_;
    const long long fs = L.fs;
    int bxi, byi, kb, ke;
    item_of<PMLK>(wk, local, bxi, byi, kb, ke, a.kbeg, a.kend);
    const int nout = ke - kb, nplanes = nout + 4;
    const int q0 = DIR > 0 ? kb - 3 : ke + 2;  // input planes q_n = q0 + n*DIR
    const int i = HALO + bxi * TX + c, j = HALO + byi * TY + r;
    const bool valid = i < L.nx_ - HALO && j < L.ny_ - HALO;
    const int tx0 = HALO + L.xoff + bxi * TX;  // HBM x of the tile's first column
    const int wx0 = tx0 - G::HB;
    const int wy0 = HALO + byi * TY - (FB2 > 0 ? 1 : 3);
    const int ty0 = HALO + byi * TY;
    const int xs = c + G::HB, ys = r + (FB2 > 0 ? 1 : 3);

    auto issue_w = [&](int n) {
      if (a.drop_one_load && local == 0 && n == NW - 1) return;  // test hook, see StageArgs
      const unsigned f = fw0 + n, s = f % NW;
      const uint32_t bar = smem_u32(&bw[s]);
      mbar_expect_tx(bar, 9 * BY * BX * G::ES);
      tma_load_4d(smem_u32(smem + s * G::W_BYTES), &maps.w, wx0, wy0, q0 + n * DIR, 0, bar);
    };
    auto issue_c = [&](int o) {  // output o is plane kb + o (DIR > 0) or ke-1-o
      const unsigned f = fc0 + o, s = f % NC;
      const int k = DIR > 0 ? kb + o : ke - 1 - o;
      const uint32_t bar = smem_u32(&bc[s]);
      unsigned char *dst = smem + G::OFF_C + s * G::C_BYTES;
      mbar_expect_tx(bar, G::C_BYTES);
      tma_load_4d(smem_u32(dst), &maps.c9, tx0, ty0, k, 0, bar);
      tma_load_4d(smem_u32(dst + 9 * NTHR * G::ES), &maps.c3, tx0, ty0, k, 10, bar);
    };
    auto issue_m = [&](int o) {
      const unsigned f = fm0 + o, s = f % NM;
      const int k = DIR > 0 ? kb + o : ke - 1 - o;
      const uint32_t bar = smem_u32(&bm[s]);
      unsigned char *dst = smem + G::OFF_M + s * G::M_BYTES;
      mbar_expect_tx(bar, m_bytes);
      if (need_m) tma_load_4d(smem_u32(dst), &maps.m, tx0, ty0, k, 0, bar);
      if (need_t) tma_load_4d(smem_u32(dst + 9 * NTHR * G::ES), &maps.t, tx0, ty0, k, 0, bar);
    };
    if (tid == 0) {
      for (int n = 0; n < NW - 1 && n < nplanes; ++n) issue_w(n);
      for (int o = 0; o < NC && o < nout; ++o) issue_c(o);
      if (need_t)
        for (int o = 0; o < NM && o < nout; ++o) issue_m(o);
    }

    // per-column PML beta times DT, with the direction's sign and 1/DH
    const int ic = valid ? i : HALO, jc = valid ? j : HALO;
    const float bxd = px[L.nx_ + ic] * DT * gx, byd = py[L.ny_ + jc] * DT * gy;
    // PML variant: the x (x1/x2) and y (y1/y2) slab of this column
    int sx = -1, sy = -1;
    if (PMLK && valid && a.nslab) {
      const int np = a.npml;
      sx = i < HALO + np ? 0 : i >= L.nx_ - HALO - np ? 3 : -1;
      sy = j < HALO + np ? 1 : j >= L.ny_ - HALO - np ? 4 : -1;
    }
    // PML profile d (times the direction's sign and 1/DH, as it multiplies
    // the elastic combination), alpha + d and beta of this column
    float dlx = 0.f, btx = 0.f, adx = 0.f, dly = 0.f, bty = 0.f, ady = 0.f;
    if (PMLK && sx >= 0) {
      const float d = __ldg(px + 2 * L.nx_ + i);
      btx = __ldg(px + L.nx_ + i);
      adx = __ldg(px + i) + d;
      dlx = d * gx;
    }
    if (PMLK && sy >= 0) {
      const float d = __ldg(py + 2 * L.ny_ + j);
      bty = __ldg(py + L.ny_ + j);
      ady = __ldg(py + j) + d;
      dly = d * gy;
    }

    // z window in registers: physical slot n mod 5 holds input plane q_n; the
    // plane loop is unrolled five times so that every slot index is a
    // compile-time constant and the window rotates without register moves.
    float win[9][5];
#pragma unroll
    for (int v = 0; v < 9; ++v)
#pragma unroll
      for (int m = 0; m < 5; ++m) win[v][m] = 0.0f;
    // z-profile beta of the next output plane, loaded one iteration ahead
    // (its latency then overlaps the barrier and ring waits)
    float bz_next = 0.0f;

    // one input plane with window rotation R = n mod 5; false on a failed wait
    auto iter = [&](auto Rc, const int n) -> bool {
      constexpr int R = decltype(Rc)::value;
      constexpr int P0 = R, P1 = (R + 4) % 5, P2 = (R + 3) % 5, P3 = (R + 2) % 5, P4 = (R + 1) % 5;
      const int o = n - 4;  // output index of this iteration (o < 0: window warm-up)
      const float bz_cur = bz_next;
      if (o + 1 >= 0 && n + 1 < nplanes) bz_next = __ldg(pz + L.nz_ + q0 + n * DIR);
      constexpr int HP = hoist_parts<RK>();
      // the inputs of this plane's point in its first slab (x, y or the
      // bottom z slab), issued before the waits
      PmlIn pin;
      const int kk = q0 + n * DIR - DIR;
      int sh = -1;  // the slab whose parts HP are in pin
      if (PMLK && o >= 0 && valid && a.nslab) {
        sh = sx >= 0 ? sx : sy >= 0 ? sy : kk < HALO + a.npml ? 2 : -1;
        if (sh >= 0) {
          const unsigned pos = slab_pos(a.slab[sh], i, j, kk);
          pml_load<RK>(a.slab[sh], pos, HP, pin);
          if (HP != pml_parts<RK>()) pml_prefetch<RK>(a.slab[sh], pos, pml_parts<RK>() & ~HP);
        }
      }
      bool ok = mbar_wait_bounded(smem_u32(&bw[(fw0 + n) % NW]), ((fw0 + n) / NW) & 1);
      if (o >= 0) {
        ok = ok && mbar_wait_bounded(smem_u32(&bc[(fc0 + o) % NC]), ((fc0 + o) / NC) & 1);
        if (need_t) ok = ok && mbar_wait_bounded(smem_u32(&bm[(fm0 + o) % NM]), ((fm0 + o) / NM) & 1);
      }
      // Every thread waits on the ring barriers itself, so no block barrier is
      // needed before the plane is read; a thread whose wait expired skips the
      // plane, and all threads leave after the barrier below.
      if (!ok) {
        s_bad = 1;
        atomicExch(err, 1);
      }
      const S *tq = (const S *)(smem + ((fw0 + n) % NW) * G::W_BYTES);
      if (ok) {
      if constexpr (G::CONV) {  // plane n to FP32 for the stencils of the next iteration
        constexpr int NE = 9 * BY * BX;
        static_assert(NE % 4 == 0, "conversion in groups of four");
        float *fd = (float *)(smem + G::OFF_F + (n & 1) * G::F_BYTES);
#pragma unroll
        for (int g = 0; g < (NE + 4 * NTHR - 1) / (4 * NTHR); ++g) {
          const int e = 4 * (tid + g * NTHR);
          if (e < NE) *(float4 *)(fd + e) = cvt4(tq + e);
        }
      }
#pragma unroll
      for (int v = 0; v < 9; ++v) win[v][P0] = ldv(tq + (v * BY + ys) * BX + xs);
      if (o >= 0 && valid) {
        const int k = q0 + n * DIR - DIR;
        // plane k: its FP32 copy, or the W slot itself
        using XT = std::conditional_t<G::CONV, float, S>;
        const XT *xy;
        if constexpr (G::CONV)
          xy = (const float *)(smem + G::OFF_F + ((n - 1) & 1) * G::F_BYTES);
        else
          xy = (const S *)(smem + ((fw0 + n + NW - 1) % NW) * G::W_BYTES);
        const S *cf = (const S *)(smem + G::OFF_C + ((fc0 + o) % NC) * G::C_BYTES);
        float mx[3], my[3], mz[3];
#pragma unroll
        for (int q = 0; q < 3; ++q) {
          mx[q] = ldv(cf + q * NTHR + cidx);
          my[q] = ldv(cf + (3 + q) * NTHR + cidx);
          mz[q] = ldv(cf + (6 + q) * NTHR + cidx);
        }
        const float mu = ldv(cf + 9 * NTHR + cidx), lam = ldv(cf + 10 * NTHR + cidx);
        const float bu = ldv(cf + 11 * NTHR + cidx) * (float)CRHO_OF<S>::v;
        const float bzd = bz_cur * DT * gz;
        float h[9], Lr[9], E[9];
        ElasticSum es;
        // PML variant: the slab corrections -beta * Aux * DT of this point,
        // added to the increment after the elastic sums
        float pc[9];
        if constexpr (PMLK) {
#pragma unroll
          for (int v = 0; v < 9; ++v) pc[v] = 0.0f;
        }
        // Fields are taken in pairs (0,1) (2,3) (4,5) (6,7) and 8 for the
        // stencil sums, the increment and the RK combination.  The centre
        // tap of the x and y stencils, plane k at this point, is window slot
        // P1 (loaded from the same shared-memory plane one iteration ago).
        // x direction
#pragma unroll
        for (int v = 0; v < 8; v += 2) {
          const XT *r0 = xy + (v * BY + ys) * BX + xs, *r1 = r0 + BY * BX;
          const float2 s = stencil2(pk(ldv(r0 - FB1), ldv(r1 - FB1)), pk(win[v][P1], win[v + 1][P1]),
                                    pk(ldv(r0 + FB1), ldv(r1 + FB1)),
                                    pk(ldv(r0 + 2 * FB1), ldv(r1 + 2 * FB1)),
                                    pk(ldv(r0 + 3 * FB1), ldv(r1 + 3 * FB1)));
          Lr[v] = s.x;
          Lr[v + 1] = s.y;
        }
        {
          const XT *r0 = xy + (8 * BY + ys) * BX + xs;
          Lr[8] = stencil1(ldv(r0 - FB1), win[8][P1], ldv(r0 + FB1), ldv(r0 + 2 * FB1), ldv(r0 + 3 * FB1));
        }
        es.add<true>(mx, bxd, Lr);
        if constexpr (PMLK) {
          if (sx >= 0) {  // profile values d, alpha + d, beta at this x
            elastic9(mx, Lr, mu, lam, bu, E);
            pml_apply<RK>(a.slab[sx], slab_pos(a.slab[sx], i, j, k), E, dlx, adx, btx, DT, cB, cA, pc, HP, pin);
          }
        }
        // y direction
#pragma unroll
        for (int v = 0; v < 8; v += 2) {
          const XT *c0 = xy + (v * BY + ys) * BX + xs, *c1 = c0 + BY * BX;
          const float2 s = stencil2(pk(ldv(c0 - FB2 * BX), ldv(c1 - FB2 * BX)), pk(win[v][P1], win[v + 1][P1]),
                                    pk(ldv(c0 + FB2 * BX), ldv(c1 + FB2 * BX)),
                                    pk(ldv(c0 + 2 * FB2 * BX), ldv(c1 + 2 * FB2 * BX)),
                                    pk(ldv(c0 + 3 * FB2 * BX), ldv(c1 + 3 * FB2 * BX)));
          Lr[v] = s.x;
          Lr[v + 1] = s.y;
        }
        {
          const XT *c0 = xy + (8 * BY + ys) * BX + xs;
          Lr[8] = stencil1(ldv(c0 - FB2 * BX), win[8][P1], ldv(c0 + FB2 * BX), ldv(c0 + 2 * FB2 * BX),
                           ldv(c0 + 3 * FB2 * BX));
        }
        es.add<false>(my, byd, Lr);
        if constexpr (PMLK) {
          if (sy >= 0) {
            elastic9(my, Lr, mu, lam, bu, E);
            pml_apply<RK>(a.slab[sy], slab_pos(a.slab[sy], i, j, k), E, dly, ady, bty, DT, cB, cA, pc,
                          sh == sy ? HP : 0, pin);
          }
        }
        // z direction: W[k - m*DIR] for m = -1..3 sits in slots P0 (q = k + DIR) .. P4
#pragma unroll
        for (int v = 0; v < 8; v += 2) {
          const float2 s = stencil2(pk(win[v][P0], win[v + 1][P0]), pk(win[v][P1], win[v + 1][P1]),
                                    pk(win[v][P2], win[v + 1][P2]), pk(win[v][P3], win[v + 1][P3]),
                                    pk(win[v][P4], win[v + 1][P4]));
          Lr[v] = s.x;
          Lr[v + 1] = s.y;
        }
        Lr[8] = stencil1(win[8][P0], win[8][P1], win[8][P2], win[8][P3], win[8][P4]);
        es.add<false>(mz, bzd, Lr);
        const bool zslab = PMLK && a.nslab && k < HALO + a.npml;
        if constexpr (PMLK) {
          if (zslab) {
            elastic9(mz, Lr, mu, lam, bu, E);
            const float d = __ldg(pz + 2 * L.nz_ + k), btz = __ldg(pz + L.nz_ + k), adz = __ldg(pz + k) + d;
            pml_apply<RK>(a.slab[2], slab_pos(a.slab[2], i, j, k), E, d * gz, adz, btz, DT, cB, cA, pc,
                          sh == 2 ? HP : 0, pin);
          }
        }
        es.finish(mu, lam, bu, h);
        if constexpr (PMLK) {
          if (sx >= 0 || sy >= 0 || zslab) {
#pragma unroll
            for (int v = 0; v < 9; ++v) h[v] += pc[v];
          }
        }
        // RK4 combination (wave_rk.cpp:13-99), two fields at a time:
        // stage 0: t = m + B1 h, out = m + A2 h (the stage input at k is the step state m);
        // stages 1-2: t += B h, out = m + A h; stage 3: out = t + B4 h
        const S *ms = (const S *)(smem + G::OFF_M + ((fm0 + o) % NM) * G::M_BYTES);
        const S *ts = ms + 9 * NTHR;
        const long long ctr = L.at(i, j, k);
        const float cT = RK == 0 ? kB1 : RK == 1 ? cB : 0.0f;
        const float cO = RK == 0 ? kA2rk : RK == 1 ? cA : kB4;
#pragma unroll
        for (int v = 0; v < 9; v += 2) {
          const bool two = v < 8;
          const float2 hv = pk(h[v], two ? h[v + 1] : 0.0f);
          const long long q = ctr + v * fs;
          float2 base_t, base_o;  // what t and the output add the increment to
          if (RK == 0) {
            base_t = base_o = pk(win[v][P1], two ? win[v + 1][P1] : 0.0f);
          } else if (RK == 1) {
            base_t = pk(ldv(ts + v * NTHR + cidx), two ? ldv(ts + (v + 1) * NTHR + cidx) : 0.0f);
            base_o = pk(ldv(ms + v * NTHR + cidx), two ? ldv(ms + (v + 1) * NTHR + cidx) : 0.0f);
          } else {
            base_o = pk(ldv(ts + v * NTHR + cidx), two ? ldv(ts + (v + 1) * NTHR + cidx) : 0.0f);
          }
          const float2 wo = __ffma2_rn(pk(cO), hv, base_o);
          stv(a.wout + q, wo.x);
          if (two) stv(a.wout + q + fs, wo.y);
          if (RK <= 1) {
            const float2 wt = __ffma2_rn(pk(cT), hv, base_t);
            stv(a.t + q, wt.x);
            if (two) stv(a.t + q + fs, wt.y);
          }
        }
      }
      }  // ok
      __syncthreads();  // every thread is done with W plane n-1, C and M slot of o
      if (s_bad) return false;
      if (tid == 0) {
        if (n + NW - 1 < nplanes) issue_w(n + NW - 1);
        if (o >= 0 && o + NC < nout) issue_c(o + NC);
        if (o >= 0 && need_t && o + NM < nout) issue_m(o + NM);
      }
      return true;
    };
    int n = 0;
    if (PMLK) {
      // one loop body (the PML variant's code is large; unrolled it no longer
      // fits the instruction cache): the window moves down one slot per plane
#pragma unroll 1
      for (; n < nplanes; ++n) {
        if (!iter(std::integral_constant<int, 0>{}, n)) break;
#pragma unroll
        for (int v = 0; v < 9; ++v) {
          win[v][1] = win[v][2];
          win[v][2] = win[v][3];
          win[v][3] = win[v][4];
          win[v][4] = win[v][0];
        }
      }
    } else
    while (n < nplanes) {
      if (!iter(std::integral_constant<int, 0>{}, n)) break;
      if (++n >= nplanes) break;
      if (!iter(std::integral_constant<int, 1>{}, n)) break;
      if (++n >= nplanes) break;
      if (!iter(std::integral_constant<int, 2>{}, n)) break;
      if (++n >= nplanes) break;
      if (!iter(std::integral_constant<int, 3>{}, n)) break;
      if (++n >= nplanes) break;
      if (!iter(std::integral_constant<int, 4>{}, n)) break;
      ++n;
    }
    if (n < nplanes) {
      // error exit: drain what was issued and not yet waited for (bounded)
      if (tid == 0) {
        for (int m = n + 1; m < nplanes && m < n + NW - 1; ++m)
          mbar_wait_bounded(smem_u32(&bw[(fw0 + m) % NW]), ((fw0 + m) / NW) & 1);
        const int o = n - 4 > 0 ? n - 4 : 0;
        for (int m = o; m < nout && m < o + NC; ++m)
          mbar_wait_bounded(smem_u32(&bc[(fc0 + m) % NC]), ((fc0 + m) / NC) & 1);
        if (need_t)
          for (int m = o; m < nout && m < o + NM; ++m)
            mbar_wait_bounded(smem_u32(&bm[(fm0 + m) % NM]), ((fm0 + m) / NM) & 1);
      }
      break;
    }
    fw0 += nplanes;
    fc0 += nout;
    if (need_t) fm0 += nout;
  }
}

template <typename S, int TYv, int FB1, int FB2, int FB3, bool PMLK, int RK>
__global__ void __launch_bounds__(TX * TYv, Geo<S, TYv>::MINB)
    stage_stream_kernel(const __grid_constant__ Maps maps, const __grid_constant__ StageArgs<S> a,
                        const __grid_constant__ Work wk, int *err) {
  stream_body<S, TYv, FB1, FB2, FB3, PMLK, RK>(SingleSrc<S>{maps, a, wk}, err);
}

template <typename S, int FB1, int FB2, int FB3, bool PMLK, int RK>
__global__ void __launch_bounds__(TX * 16, 1)
    stage_stream_batch_kernel(const __grid_constant__ BatchParams<S> p, int *err) {
  stream_body<S, 16, FB1, FB2, FB3, PMLK, RK>(BatchSrc<S>{p}, err);
}

// ---------------------------------------------------------------------------
// 16-bit storage, interior items: the paired-point kernel.
//
// A 64 x 8 column tile per item and 256 threads, each owning two x-adjacent
// points (columns i and i + 1, i - HALO even), so that every shared-memory
// read, conversion and global store of the tile moves one 32-bit pair of
// 16-bit values and the arithmetic of the two points is one packed FP32x2
// instruction.  Per point and stage this issues about half the instructions
// of the one-point 16-bit kernel, whose interior launches are bound by
// instruction issue rather than by HBM.  The per-point arithmetic (operands,
// operation order, rounding) is that of the one-point kernel's interior
// variant, so both give the same bits.  Rings: W 4 slots (9 fields x 12 rows
// x 80 columns: the tile, a 16-byte aligned 8-column halo on each side and
// the y halo), coefficients 3 slots, m / t 3 slots; one CTA per SM.  (An FP32
// copy of each plane, converted once cooperatively, measured slower: the
// extra barrier-bound work per plane and the shallower W ring cost more
// than the conversions it saves.)
template <typename S> struct PairGeo {
  static constexpr int TY = 8, TXP = 64, NTHR = 256, PLANE = TY * TXP;
  static constexpr int BY = TY + 4, BX = 8 + TXP + 8;
  static constexpr int W_BYTES = ((9 * BY * BX * 2) + 127) / 128 * 128;
  static constexpr int C_BYTES = 12 * PLANE * 2;
  static constexpr int M_BYTES = 18 * PLANE * 2;
  static constexpr int NW = 4, NC = 3, NM = 3;
  static constexpr int OFF_C = NW * W_BYTES;
  static constexpr int OFF_M = OFF_C + NC * C_BYTES;
  static constexpr int OFF_BAR = OFF_M + NM * M_BYTES;
  static constexpr int SMEM = OFF_BAR + 8 * (NW + NC + NM) + 128;
  static_assert(sizeof(S) == 2, "the paired-point kernel is for 16-bit storage");
  static_assert(SMEM <= 232448, "shared memory budget");
};

// Two adjacent 16-bit values (4-byte aligned) as a float2, and back.
__device__ __forceinline__ float2 ld2(const __half *p) { return __half22float2(*(const __half2 *)p); }
__device__ __forceinline__ float2 ld2(const __nv_bfloat16 *p) {
  return __bfloat1622float2(*(const __nv_bfloat162 *)p);
}
__device__ __forceinline__ void st2(__half *p, float2 v) { *(__half2 *)p = __float22half2_rn(v); }
__device__ __forceinline__ void st2(__nv_bfloat16 *p, float2 v) {
  *(__nv_bfloat162 *)p = __float22bfloat162_rn(v);
}
__device__ __forceinline__ float2 f2mul(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 f2fma(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float2 f2add(float2 a, float2 b) { return __fadd2_rn(a, b); }

// ElasticSum for two points at once (lane x: point i, lane y: point i + 1),
// the same operations in the same order.
struct ElasticSum2 {
  float2 v0, v1, v2, nx, ny, nz, s6, s7, s8;
  template <bool FIRST>
  __device__ __forceinline__ void add(const float2 m[3], float2 g, const float2 L[9]) {
    const float2 a0 = f2mul(g, m[0]), a1 = f2mul(g, m[1]), a2 = f2mul(g, m[2]);
    v0 = f2fma(a2, L[7], f2fma(a1, L[6], FIRST ? f2mul(a0, L[3]) : f2fma(a0, L[3], v0)));
    v1 = f2fma(a2, L[8], f2fma(a1, L[4], FIRST ? f2mul(a0, L[6]) : f2fma(a0, L[6], v1)));
    v2 = f2fma(a2, L[5], f2fma(a1, L[8], FIRST ? f2mul(a0, L[7]) : f2fma(a0, L[7], v2)));
    nx = FIRST ? f2mul(a0, L[0]) : f2fma(a0, L[0], nx);
    ny = FIRST ? f2mul(a1, L[1]) : f2fma(a1, L[1], ny);
    nz = FIRST ? f2mul(a2, L[2]) : f2fma(a2, L[2], nz);
    s6 = f2fma(a0, L[1], FIRST ? f2mul(a1, L[0]) : f2fma(a1, L[0], s6));
    s7 = f2fma(a0, L[2], FIRST ? f2mul(a2, L[0]) : f2fma(a2, L[0], s7));
    s8 = f2fma(a1, L[2], FIRST ? f2mul(a2, L[1]) : f2fma(a2, L[1], s8));
  }
  __device__ __forceinline__ void finish(float2 mu, float2 lam, float2 b, float2 h[9]) const {
    h[0] = f2mul(v0, b);
    h[1] = f2mul(v1, b);
    h[2] = f2mul(v2, b);
    const float2 div = f2mul(f2add(f2add(nx, ny), nz), lam), tmu = f2mul(pk(2.0f), mu);
    h[3] = f2fma(tmu, nx, div);
    h[4] = f2fma(tmu, ny, div);
    h[5] = f2fma(tmu, nz, div);
    h[6] = f2mul(s6, mu);
    h[7] = f2mul(s7, mu);
    h[8] = f2mul(s8, mu);
  }
};

// Interior items of a paired launch: 64 x 8 tiles (two 32-column tiles of
// the Work grid, starting at bx_lo; bx_hi - bx_lo is even) x the upper z
// chunks, tiles fastest.
__device__ __forceinline__ void item_of_pair(const Work &w, int item, int &pxi, int &byi, int &kb,
                                             int &ke, int kend) {
  const int npx = (w.bx_hi - w.bx_lo) / 2, ti = npx * (w.by_hi - w.by_lo);
  const int t = item % ti, chk = item / ti;
  pxi = t % npx;
  byi = w.by_lo + t / npx;
  kb = w.kz + chk * w.chunk_i;
  ke = min(kb + w.chunk_i, kend);
}

template <typename S, int FB1, int FB2, int FB3, int RK>
__global__ void __launch_bounds__(256, 1)
    stage_pair_kernel(const __grid_constant__ Maps maps, const __grid_constant__ StageArgs<S> a,
                      const __grid_constant__ Work wk, int *err) {
  using G = PairGeo<S>;
  constexpr int TY = G::TY, PLANE = G::PLANE, BY = G::BY, BX = G::BX, NTHR = G::NTHR;
  constexpr int NW = G::NW, NC = G::NC, NM = G::NM;
  constexpr int DIR = -FB3;  // sweep direction in z
  extern __shared__ unsigned char smem_raw[];
  unsigned char *smem = smem_raw + ((128u - (smem_u32(smem_raw) & 127u)) & 127u);
  uint64_t *bw = (uint64_t *)(smem + G::OFF_BAR);
  uint64_t *bc = bw + NW;
  uint64_t *bm = bc + NC;
  __shared__ int s_item, s_bad;

  const int tid = threadIdx.x;
  const int c = tid % 32, r = tid / 32;
  const int cidx = r * G::TXP + 2 * c;  // the pair's first element in a C / M plane

  if (tid == 0) {
    s_bad = 0;
    for (int q = 0; q < NW + NC + NM; ++q) mbar_init(smem_u32(&bw[q]), 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();

  unsigned fw0 = 0, fc0 = 0, fm0 = 0;  // ring fill counters, continued across items
  const Layout L = a.L;
  constexpr bool need_m = RK == 1, need_t = RK >= 1;
  const float cB = a.irk == 2 ? kB3 : kB2, cA = a.irk == 2 ? 1.0f : kA3rk;
  const uint32_t m_bytes = ((need_m ? 9 : 0) + (need_t ? 9 : 0)) * PLANE * 2;
  const float rDH = a.rDH, DT = a.DT;
  const float gx = FB1 * rDH, gy = FB2 * rDH, gz = FB3 * rDH;
  const float *px = a.pml, *py = a.pml + 3 * L.nx_, *pz = a.pml + 3 * L.nx_ + 3 * L.ny_;
  const long long fs = L.fs;

  for (;;) {
    if (tid == 0) s_item = atomicAdd(wk.counter, 1);
    __syncthreads();
    const int item = s_item;
    if (item >= wk.nitems || s_bad) break;
    int pxi, byi, kb, ke;
    item_of_pair(wk, item, pxi, byi, kb, ke, a.kend);
    const int nout = ke - kb, nplanes = nout + 4;
    const int q0 = DIR > 0 ? kb - 3 : ke + 2;  // input planes q_n = q0 + n*DIR
    const int x0 = HALO + 32 * (wk.bx_lo + 2 * pxi);  // padded index of the tile's column 0
    const int i = x0 + 2 * c, j = HALO + byi * TY + r;
    const int tx0 = L.xoff + x0;  // HBM x of the tile's first column
    const int wx0 = tx0 - 8;
    const int wy0 = HALO + byi * TY - (FB2 > 0 ? 1 : 3);
    const int ty0 = HALO + byi * TY;
    const int xs = 2 * c + 8, ys = r + (FB2 > 0 ? 1 : 3);

    auto issue_w = [&](int n) {
      if (a.drop_one_load && item == 0 && n == NW - 1) return;  // test hook, see StageArgs
      const unsigned f = fw0 + n, q = f % NW;
      const uint32_t bar = smem_u32(&bw[q]);
      mbar_expect_tx(bar, 9 * BY * BX * 2);
      tma_load_4d(smem_u32(smem + q * G::W_BYTES), &maps.w, wx0, wy0, q0 + n * DIR, 0, bar);
    };
    auto issue_c = [&](int o) {  // output o is plane kb + o (DIR > 0) or ke-1-o
      const unsigned f = fc0 + o, q = f % NC;
      const int k = DIR > 0 ? kb + o : ke - 1 - o;
      const uint32_t bar = smem_u32(&bc[q]);
      unsigned char *dst = smem + G::OFF_C + q * G::C_BYTES;
      mbar_expect_tx(bar, G::C_BYTES);
      tma_load_4d(smem_u32(dst), &maps.c9, tx0, ty0, k, 0, bar);
      tma_load_4d(smem_u32(dst + 9 * PLANE * 2), &maps.c3, tx0, ty0, k, 10, bar);
    };
    auto issue_m = [&](int o) {
      const unsigned f = fm0 + o, q = f % NM;
      const int k = DIR > 0 ? kb + o : ke - 1 - o;
      const uint32_t bar = smem_u32(&bm[q]);
      unsigned char *dst = smem + G::OFF_M + q * G::M_BYTES;
      mbar_expect_tx(bar, m_bytes);
      if (need_m) tma_load_4d(smem_u32(dst), &maps.m, tx0, ty0, k, 0, bar);
      if (need_t) tma_load_4d(smem_u32(dst + 9 * PLANE * 2), &maps.t, tx0, ty0, k, 0, bar);
    };
    if (tid == 0) {
      for (int n = 0; n < NW - 1 && n < nplanes; ++n) issue_w(n);
      for (int o = 0; o < NC && o < nout; ++o) issue_c(o);
      if (need_t)
        for (int o = 0; o < NM && o < nout; ++o) issue_m(o);
    }

    // per-column PML beta times DT, with the direction's sign and 1/DH
    const float2 bxd = make_float2(px[L.nx_ + i] * DT * gx, px[L.nx_ + i + 1] * DT * gx);
    const float2 byd = pk(py[L.ny_ + j] * DT * gy);

    float2 win[9][5];
#pragma unroll
    for (int v = 0; v < 9; ++v)
#pragma unroll
      for (int m = 0; m < 5; ++m) win[v][m] = pk(0.0f);
    // z-profile beta of the next output plane, loaded one iteration ahead
    // (its latency then overlaps the barrier and ring waits)
    float bz_next = 0.0f;

    auto iter = [&](auto Rc, const int n) -> bool {
      constexpr int R = decltype(Rc)::value;
      constexpr int P0 = R, P1 = (R + 4) % 5, P2 = (R + 3) % 5, P3 = (R + 2) % 5, P4 = (R + 1) % 5;
      const int o = n - 4;
      const float bz_cur = bz_next;
      if (o + 1 >= 0 && n + 1 < nplanes) bz_next = __ldg(pz + L.nz_ + q0 + n * DIR);
      bool ok = mbar_wait_bounded(smem_u32(&bw[(fw0 + n) % NW]), ((fw0 + n) / NW) & 1);
      if (o >= 0) {
        ok = ok && mbar_wait_bounded(smem_u32(&bc[(fc0 + o) % NC]), ((fc0 + o) / NC) & 1);
        if (need_t) ok = ok && mbar_wait_bounded(smem_u32(&bm[(fm0 + o) % NM]), ((fm0 + o) / NM) & 1);
      }
      // Every thread waits on the ring barriers itself, so no block barrier is
      // needed before the plane is read; a thread whose wait expired skips the
      // plane, and all threads leave after the barrier below.
      if (!ok) {
        s_bad = 1;
        atomicExch(err, 1);
      }
      const S *tq = (const S *)(smem + ((fw0 + n) % NW) * G::W_BYTES);
#pragma unroll
      for (int v = 0; v < 9; ++v) win[v][P0] = ok ? ld2(tq + (v * BY + ys) * BX + xs) : pk(0.0f);
      if (o >= 0 && ok) {
        const int k = q0 + n * DIR - DIR;
        const S *xy = (const S *)(smem + ((fw0 + n + NW - 1) % NW) * G::W_BYTES);  // plane k
        const S *cf = (const S *)(smem + G::OFF_C + ((fc0 + o) % NC) * G::C_BYTES);
        float2 mx[3], my[3], mz[3];
#pragma unroll
        for (int q = 0; q < 3; ++q) {
          mx[q] = ld2(cf + q * PLANE + cidx);
          my[q] = ld2(cf + (3 + q) * PLANE + cidx);
          mz[q] = ld2(cf + (6 + q) * PLANE + cidx);
        }
        const float2 mu = ld2(cf + 9 * PLANE + cidx), lam = ld2(cf + 10 * PLANE + cidx);
        const float2 bu = f2mul(ld2(cf + 11 * PLANE + cidx), pk((float)CRHO_OF<S>::v));
        const float2 bzd = pk(bz_cur * DT * gz);
        float2 h[9], Lr[9];
        ElasticSum2 es;
        // x direction: taps of the pair from the plane's row; the centre
        // pair (plane k at i, i + 1) is window slot P1
#pragma unroll
        for (int v = 0; v < 9; ++v) {
          const S *row = xy + (v * BY + ys) * BX + xs;
          const float2 cen = win[v][P1];
          if (FB1 > 0) {
            const float xm1 = ldv(row - 1), x4 = ldv(row + 4);
            const float2 w23 = ld2(row + 2);
            Lr[v] = stencil2(make_float2(xm1, cen.x), cen, make_float2(cen.y, w23.x), w23,
                             make_float2(w23.y, x4));
          } else {
            const float xm3 = ldv(row - 3), x2 = ldv(row + 2);
            const float2 w21 = ld2(row - 2);
            Lr[v] = stencil2(make_float2(cen.y, x2), cen, make_float2(w21.y, cen.x), w21,
                             make_float2(xm3, w21.x));
          }
        }
        es.add<true>(mx, bxd, Lr);
        // y direction
#pragma unroll
        for (int v = 0; v < 9; ++v) {
          const S *c0 = xy + (v * BY + ys) * BX + xs;
          Lr[v] = stencil2(ld2(c0 - FB2 * BX), win[v][P1], ld2(c0 + FB2 * BX),
                           ld2(c0 + 2 * FB2 * BX), ld2(c0 + 3 * FB2 * BX));
        }
        es.add<false>(my, byd, Lr);
        // z direction: W[k - m*DIR] for m = -1..3 sits in slots P0 (q = k + DIR) .. P4
#pragma unroll
        for (int v = 0; v < 9; ++v)
          Lr[v] = stencil2(win[v][P0], win[v][P1], win[v][P2], win[v][P3], win[v][P4]);
        es.add<false>(mz, bzd, Lr);
        es.finish(mu, lam, bu, h);
        // RK4 combination (wave_rk.cpp:13-99), as the one-point kernel
        const S *ms = (const S *)(smem + G::OFF_M + ((fm0 + o) % NM) * G::M_BYTES);
        const S *ts = ms + 9 * PLANE;
        const long long ctr = L.at(i, j, k);
        const float cT = RK == 0 ? kB1 : RK == 1 ? cB : 0.0f;
        const float cO = RK == 0 ? kA2rk : RK == 1 ? cA : kB4;
#pragma unroll
        for (int v = 0; v < 9; ++v) {
          const long long q = ctr + v * fs;
          float2 base_t, base_o;
          if (RK == 0) {
            base_t = base_o = win[v][P1];
          } else if (RK == 1) {
            base_t = ld2(ts + v * PLANE + cidx);
            base_o = ld2(ms + v * PLANE + cidx);
          } else {
            base_t = pk(0.0f);
            base_o = ld2(ts + v * PLANE + cidx);
          }
          st2(a.wout + q, f2fma(pk(cO), h[v], base_o));
          if (RK <= 1) st2(a.t + q, f2fma(pk(cT), h[v], base_t));
        }
      }
      __syncthreads();  // every thread is done with W plane n-1, C and M slot of o
      if (s_bad) return false;
      if (tid == 0) {
        if (n + NW - 1 < nplanes) issue_w(n + NW - 1);
        if (o >= 0 && o + NC < nout) issue_c(o + NC);
        if (o >= 0 && need_t && o + NM < nout) issue_m(o + NM);
      }
      return true;
    };
    int n = 0;
    while (n < nplanes) {
      if (!iter(std::integral_constant<int, 0>{}, n)) break;
      if (++n >= nplanes) break;
      if (!iter(std::integral_constant<int, 1>{}, n)) break;
      if (++n >= nplanes) break;
      if (!iter(std::integral_constant<int, 2>{}, n)) break;
      if (++n >= nplanes) break;
      if (!iter(std::integral_constant<int, 3>{}, n)) break;
      if (++n >= nplanes) break;
      if (!iter(std::integral_constant<int, 4>{}, n)) break;
      ++n;
    }
    if (n < nplanes) {
      // error exit: drain what was issued and not yet waited for (bounded)
      if (tid == 0) {
        for (int m = n + 1; m < nplanes && m < n + NW - 1; ++m)
          mbar_wait_bounded(smem_u32(&bw[(fw0 + m) % NW]), ((fw0 + m) / NW) & 1);
        const int o = n - 4 > 0 ? n - 4 : 0;
        for (int m = o; m < nout && m < o + NC; ++m)
          mbar_wait_bounded(smem_u32(&bc[(fc0 + m) % NC]), ((fc0 + m) / NC) & 1);
        if (need_t)
          for (int m = o; m < nout && m < o + NM; ++m)
            mbar_wait_bounded(smem_u32(&bm[(fm0 + m) % NM]), ((fm0 + m) / NM) & 1);
      }
      break;
    }
    fw0 += nplanes;
    fc0 += nout;
    if (need_t) fm0 += nout;
  }
}

// Sets a kernel's dynamic shared-memory limit once per device.  `done` is
// the kernel variant's own bit set of devices that have it; the attribute
// call is idempotent, so two host threads that race here both make it and
// both set the bit.
template <typename K>
cudaError_t ensure_smem_attr(K kern, int smem, std::atomic<unsigned long long> &done) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  const unsigned long long bit = dev < 64 ? 1ull << dev : 0ull;
  if (bit && (done.load(std::memory_order_acquire) & bit)) return cudaSuccess;
  e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
  if (e == cudaSuccess && bit) done.fetch_or(bit, std::memory_order_acq_rel);
  return e;
}

template <typename S, int TYv, int FB1, int FB2, int FB3, bool PMLK, int RK>
cudaError_t launch_variant(const StageArgs<S> &a, const Maps &maps, const Work &wk, int *err,
                           int nsm, cudaStream_t st) {
  using G = Geo<S, TYv, PMLK>;
  static std::atomic<unsigned long long> attr_done{0};
  auto kern = stage_stream_kernel<S, TYv, FB1, FB2, FB3, PMLK, RK>;
  const int smem = G::SMEM;
  cudaError_t e = ensure_smem_attr(kern, smem, attr_done);
  if (e != cudaSuccess) return e;
  e = cudaMemsetAsync(wk.counter, 0, sizeof(int), st);
  if (e != cudaSuccess) return e;
  kern<<<std::min(wk.nitems, nsm * G::MINB), G::NTHR, smem, st>>>(maps, a, wk, err);
  return cudaGetLastError();
}

// SM count of the current device, cached per device (atomics: handles may be
// driven from several host threads).
int sm_count() {
  static std::atomic<int> cache[64];
  int dev = 0;
  cudaGetDevice(&dev);
  int nsm = dev >= 0 && dev < 64 ? cache[dev].load(std::memory_order_relaxed) : 0;
  if (nsm <= 0) {
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    if (nsm <= 0) nsm = 148;
    if (dev >= 0 && dev < 64) cache[dev].store(nsm, std::memory_order_relaxed);
  }
  return nsm;
}

// Item geometry of one stage of one scenario (see Work) and the item counts
// of its interior and PML launches.
struct WorkPlan {
  Work wk;
  int n_in, n_pml;
};
template <typename S, int TYv>
WorkPlan plan_work(const StageArgs<S> &a, int nsm, int *counter) {
  constexpr int TY = TYv;
  constexpr int slots = Geo<S, TYv>::MINB;  // CTAs resident per SM
  const int nx = a.L.nx_ - 2 * HALO, ny = a.L.ny_ - 2 * HALO;
  const int np = a.nslab ? a.npml : 0;
  Work wk;
  wk.counter = counter;
  wk.ntx = (nx + TX - 1) / TX;
  wk.nty = (ny + TY - 1) / TY;
  if (np > 0) {
    wk.bx_lo = (np + TX - 1) / TX;
    wk.bx_hi = (nx - np) / TX;
    wk.by_lo = (np + TY - 1) / TY;
    wk.by_hi = (ny - np) / TY;
    if (wk.bx_hi <= wk.bx_lo || wk.by_hi <= wk.by_lo) wk.bx_lo = wk.bx_hi = wk.by_lo = wk.by_hi = 0;
  } else {
    wk.bx_lo = 0; wk.bx_hi = wk.ntx; wk.by_lo = 0; wk.by_hi = wk.nty;
  }
  const int tiles = wk.ntx * wk.nty;
  const int tiles_in = (wk.bx_hi - wk.bx_lo) * (wk.by_hi - wk.by_lo);
  // bottom PML planes [kbeg, kz), at most 32 planes per chunk
  wk.kz = std::min(a.kbeg + np, a.kend);
  const int pl_p = wk.kz - a.kbeg, pl_i = a.kend - wk.kz;
  wk.nzc = pl_p > 0 ? (pl_p + 31) / 32 : 0;
  wk.chunk_p = wk.nzc ? (pl_p + wk.nzc - 1) / wk.nzc : 1;
  // upper planes: a.chunk planes per item, or about 40 items per CTA slot
  // with chunks of at least 16 planes
  int nic = pl_i > 0 ? (40 * nsm * slots + tiles - 1) / tiles : 0;
  if (pl_i > 0) nic = std::max(1, std::min(nic, pl_i / 16));
  if (pl_i > 0 && a.chunk > 0) nic = (pl_i + a.chunk - 1) / a.chunk;
  wk.chunk_i = nic ? (pl_i + nic - 1) / nic : 1;
  wk.nic = nic ? (pl_i + wk.chunk_i - 1) / wk.chunk_i : 0;
  wk.nitems = 0;
  return {wk, tiles_in * wk.nic, wk.nzc * tiles + (tiles - tiles_in) * wk.nic};
}

// Splits the stage into the interior launch (tiles and chunks that touch no
// PML slab) and the PML launch (the rest), see Work.
template <typename S, int TYv, int FB1, int FB2, int FB3, int RK>
cudaError_t launch_one(const StageArgs<S> &a, const Maps &maps, int *err, int *counter,
                       cudaStream_t st, int *nlaunch) {
  const int nsm = sm_count();
  const WorkPlan wp = plan_work<S, TYv>(a, nsm, counter);
  cudaError_t e = cudaSuccess;
  Work wi = wp.wk;
  wi.nitems = wp.n_in;
  if (wi.nitems > 0) {
    e = launch_variant<S, TYv, FB1, FB2, FB3, false, RK>(a, maps, wi, err, nsm, st);
    if (e != cudaSuccess) return e;
    if (nlaunch) ++*nlaunch;
  }
  Work wq = wp.wk;
  wq.nitems = wp.n_pml;
  if (wq.nitems > 0) {
    e = launch_variant<S, TYv, FB1, FB2, FB3, true, RK>(a, maps, wq, err, nsm, st);
    if (e != cudaSuccess) return e;
    if (nlaunch) ++*nlaunch;
  }
  return cudaSuccess;
}

// One stage with the paired-point kernel for the interior (64 x 8 tiles:
// pairs of 32 x 8 tiles of the Work grid that touch no PML slab and lie
// inside the grid) and the one-point 32 x 8 PML variant for every other
// tile and chunk (an odd interior tile column and partial edge tiles
// included).  16-bit storage only.
template <typename S, int FB1, int FB2, int FB3, int RK>
cudaError_t launch_one_pair(const StageArgs<S> &a, const Maps &m8, const Maps &mp, int *err,
                            int *counter, cudaStream_t st, int *nlaunch) {
  if constexpr (sizeof(S) != 2) {
    return cudaErrorInvalidValue;
  } else {
    const int nsm = sm_count();
    WorkPlan wp = plan_work<S, 8>(a, nsm, counter);
    Work w = wp.wk;
    const int nx = a.L.nx_ - 2 * HALO, ny = a.L.ny_ - 2 * HALO;
    // full tiles only, an even number of them in x
    int bx_hi = std::min(w.bx_hi, nx / TX), by_hi = std::min(w.by_hi, ny / 8);
    if (bx_hi - w.bx_lo < 2 || by_hi <= w.by_lo) {
      bx_hi = w.bx_lo;
      by_hi = w.by_lo;
    }
    bx_hi = w.bx_lo + (bx_hi - w.bx_lo) / 2 * 2;
    w.bx_hi = bx_hi;
    w.by_hi = by_hi;
    const int tiles = w.ntx * w.nty, tiles_in = (w.bx_hi - w.bx_lo) * (w.by_hi - w.by_lo);
    cudaError_t e = cudaSuccess;
    Work wi = w;
    wi.nitems = tiles_in / 2 * w.nic;
    if (wi.nitems > 0) {
      using G = PairGeo<S>;
      static std::atomic<unsigned long long> attr_done{0};
      auto kern = stage_pair_kernel<S, FB1, FB2, FB3, RK>;
      e = ensure_smem_attr(kern, G::SMEM, attr_done);
      if (e != cudaSuccess) return e;
      e = cudaMemsetAsync(wi.counter, 0, sizeof(int), st);
      if (e != cudaSuccess) return e;
      kern<<<std::min(wi.nitems, nsm), G::NTHR, G::SMEM, st>>>(mp, a, wi, err);
      e = cudaGetLastError();
      if (e != cudaSuccess) return e;
      if (nlaunch) ++*nlaunch;
    }
    Work wq = w;
    wq.nitems = w.nzc * tiles + (tiles - tiles_in) * w.nic;
    if (wq.nitems > 0) {
      e = launch_variant<S, 8, FB1, FB2, FB3, true, RK>(a, m8, wq, err, nsm, st);
      if (e != cudaSuccess) return e;
      if (nlaunch) ++*nlaunch;
    }
    return cudaSuccess;
  }
}

template <typename S, int FB1, int FB2, int FB3, bool PMLK, int RK>
cudaError_t launch_batch_variant(const BatchParams<S> &p, int items, int *err, int nsm,
                                 cudaStream_t st) {
  using G = Geo<S, 16, PMLK>;
  static_assert(sizeof(BatchParams<S>) <= 32000, "kernel parameter space");
  static std::atomic<unsigned long long> attr_done{0};
  auto kern = stage_stream_batch_kernel<S, FB1, FB2, FB3, PMLK, RK>;
  const int smem = G::SMEM;
  cudaError_t e = ensure_smem_attr(kern, smem, attr_done);
  if (e != cudaSuccess) return e;
  e = cudaMemsetAsync(p.counter, 0, sizeof(int), st);
  if (e != cudaSuccess) return e;
  kern<<<std::min(items, nsm), G::NTHR, smem, st>>>(p, err);
  return cudaGetLastError();
}

// One stage of n scenarios that share the MacCormack signs: kBatchMax
// scenarios per launch pair (interior items of all of them, then PML items).
template <typename S, int FB1, int FB2, int FB3, int RK>
cudaError_t launch_batch(const StageArgs<S> *args, const void *const *maps, int n, int *err,
                         int *counter, cudaStream_t st, int *nlaunch) {
  const int nsm = sm_count();
  // the launch parameters (about 19 KB) are assembled in per-thread storage
  static thread_local BatchParams<S> params;
  BatchParams<S> *bp = &params;
  for (int b0 = 0; b0 < n; b0 += kBatchMax) {
    const int nb = std::min(kBatchMax, n - b0);
    for (int pass = 0; pass < 2; ++pass) {
      std::memset((void *)bp, 0, sizeof(BatchParams<S>));
      int total = 0, m = 0;
      for (int q = 0; q < nb; ++q) {
        const StageArgs<S> &a = args[b0 + q];
        if (a.kend <= a.kbeg) continue;
        const WorkPlan wp = plan_work<S, 16>(a, nsm, counter);
        const int cnt = pass == 0 ? wp.n_in : wp.n_pml;
        if (cnt <= 0) continue;
        bp->maps[m] = ((const MapSet *)maps[b0 + q])->ty16;
        bp->args[m] = a;
        bp->work[m] = wp.wk;
        bp->work[m].nitems = cnt;
        total += cnt;
        bp->item_end[m] = total;
        ++m;
      }
      if (!m) continue;
      bp->n = m;
      bp->counter = counter;
      cudaError_t e = pass == 0
                          ? launch_batch_variant<S, FB1, FB2, FB3, false, RK>(*bp, total, err, nsm, st)
                          : launch_batch_variant<S, FB1, FB2, FB3, true, RK>(*bp, total, err, nsm, st);
      if (e != cudaSuccess) return e;
      if (nlaunch) ++*nlaunch;
    }
  }
  return cudaSuccess;
}

typedef CUresult (*EncodeTiledFn)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *,
                                  const cuuint64_t *, const cuuint64_t *, const cuuint32_t *,
                                  const cuuint32_t *, CUtensorMapInterleave, CUtensorMapSwizzle,
                                  CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
EncodeTiledFn encode_fn() {
  // resolved once (a function-local static is initialised thread-safely)
  static const EncodeTiledFn fn = []() -> EncodeTiledFn {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) ==
            cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      return (EncodeTiledFn)p;
    return nullptr;
  }();
  return fn;
}
template <typename S> CUtensorMapDataType dtype_of();
template <> CUtensorMapDataType dtype_of<float>() { return CU_TENSOR_MAP_DATA_TYPE_FLOAT32; }
template <> CUtensorMapDataType dtype_of<__half>() { return CU_TENSOR_MAP_DATA_TYPE_FLOAT16; }
template <> CUtensorMapDataType dtype_of<__nv_bfloat16>() { return CU_TENSOR_MAP_DATA_TYPE_BFLOAT16; }

// 4-D map (x, y, z, field) over nfield fields of the HBM layout with the
// given box.
template <typename S>
int encode_map(const S *base, const Layout &L, int nfield, int bx, int by, int bf, CUtensorMap *m) {
  EncodeTiledFn fn = encode_fn();
  if (!fn) {
    set_error("cuTensorMapEncodeTiled is unavailable in this driver");
    return CGFDM_ERR_NO_KERNEL;
  }
  const cuuint64_t es = sizeof(S);
  cuuint64_t dims[4] = {(cuuint64_t)L.px, (cuuint64_t)L.ny_, (cuuint64_t)L.nz_, (cuuint64_t)nfield};
  cuuint64_t strides[3] = {(cuuint64_t)L.px * es, (cuuint64_t)L.plane * es, (cuuint64_t)L.fs * es};
  cuuint32_t box[4] = {(cuuint32_t)bx, (cuuint32_t)by, 1, (cuuint32_t)bf};
  cuuint32_t estr[4] = {1, 1, 1, 1};
  CUresult r = fn(m, dtype_of<S>(), 4, (void *)base, dims, strides, box, estr,
                  CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                  CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) {
    set_error("cuTensorMapEncodeTiled failed with code " + std::to_string((int)r));
    return CGFDM_ERR_CUDA;
  }
  return CGFDM_OK;
}

}  // namespace

template <typename S> bool stage_stream_supported() { return true; }
// FP64 has none (stage_stream_f32.cu defines these specialisations)
template <> bool stage_stream_supported<double>();
template <>
int encode_stream_maps<double>(const double *, const double *, const double *, const double *,
                               const Layout &, void *);
template <>
cudaError_t launch_stage_stream_batch<double>(const StageArgs<double> *, const void *const *, int,
                                              int *, int *, cudaStream_t, int *);
template <>
cudaError_t launch_stage_stream<double>(const StageArgs<double> &, const void *, int *, int *,
                                        cudaStream_t, cudaEvent_t, int *, int);

template <typename S>
int encode_stream_maps(const S *wave, const S *cjm, const S *wm, const S *t, const Layout &L,
                       void *out) {
  static_assert(sizeof(MapSet) <= kStreamMapsBytes, "tensor-map buffer too small");
  MapSet ms;
  int rc = CGFDM_OK;
  for (int ty : {16, 8}) {
    Maps &m = ty == 16 ? ms.ty16 : ms.ty8;
    if (!rc) rc = encode_map<S>(wave, L, 9, Geo<S, 16>::BX, ty + 4, 9, &m.w);
    if (!rc) rc = encode_map<S>(cjm, L, 13, TX, ty, 9, &m.c9);
    if (!rc) rc = encode_map<S>(cjm, L, 13, TX, ty, 3, &m.c3);
    if (!rc) rc = encode_map<S>(wm, L, 9, TX, ty, 9, &m.m);
    if (!rc) rc = encode_map<S>(t, L, 9, TX, ty, 9, &m.t);
  }
  if constexpr (sizeof(S) == 2) {  // the paired-point kernel's 64 x 8 tiles
    using G = PairGeo<S>;
    Maps &m = ms.pair;
    if (!rc) rc = encode_map<S>(wave, L, 9, G::BX, G::BY, 9, &m.w);
    if (!rc) rc = encode_map<S>(cjm, L, 13, G::TXP, G::TY, 9, &m.c9);
    if (!rc) rc = encode_map<S>(cjm, L, 13, G::TXP, G::TY, 3, &m.c3);
    if (!rc) rc = encode_map<S>(wm, L, 9, G::TXP, G::TY, 9, &m.m);
    if (!rc) rc = encode_map<S>(t, L, 9, G::TXP, G::TY, 9, &m.t);
  }
  if (!rc) std::memcpy(out, &ms, sizeof ms);
  return rc;
}

// The stage class RK of stage irk: 0, 1 (stages 1 and 2) or 3.
inline int rk_class(int irk) { return irk == 0 ? 0 : irk == 3 ? 3 : 1; }

template <typename S, int TYv, int RK>
cudaError_t launch_fb_rk(const StageArgs<S> &a, const Maps &m, int *err, int *counter,
                         cudaStream_t st, int *nlaunch) {
  const int code = (a.fb1 > 0) * 4 + (a.fb2 > 0) * 2 + (a.fb3 > 0);
  switch (code) {
    case 0: return launch_one<S, TYv, -1, -1, -1, RK>(a, m, err, counter, st, nlaunch);
    case 1: return launch_one<S, TYv, -1, -1, 1, RK>(a, m, err, counter, st, nlaunch);
    case 2: return launch_one<S, TYv, -1, 1, -1, RK>(a, m, err, counter, st, nlaunch);
    case 3: return launch_one<S, TYv, -1, 1, 1, RK>(a, m, err, counter, st, nlaunch);
    case 4: return launch_one<S, TYv, 1, -1, -1, RK>(a, m, err, counter, st, nlaunch);
    case 5: return launch_one<S, TYv, 1, -1, 1, RK>(a, m, err, counter, st, nlaunch);
    case 6: return launch_one<S, TYv, 1, 1, -1, RK>(a, m, err, counter, st, nlaunch);
    default: return launch_one<S, TYv, 1, 1, 1, RK>(a, m, err, counter, st, nlaunch);
  }
}
template <typename S, int RK>
cudaError_t launch_fb_rk_pair(const StageArgs<S> &a, const MapSet &ms, int *err, int *counter,
                              cudaStream_t st, int *nlaunch) {
  const Maps &m8 = ms.ty8, &mp = ms.pair;
  switch ((a.fb1 > 0) * 4 + (a.fb2 > 0) * 2 + (a.fb3 > 0)) {
    case 0: return launch_one_pair<S, -1, -1, -1, RK>(a, m8, mp, err, counter, st, nlaunch);
    case 1: return launch_one_pair<S, -1, -1, 1, RK>(a, m8, mp, err, counter, st, nlaunch);
    case 2: return launch_one_pair<S, -1, 1, -1, RK>(a, m8, mp, err, counter, st, nlaunch);
    case 3: return launch_one_pair<S, -1, 1, 1, RK>(a, m8, mp, err, counter, st, nlaunch);
    case 4: return launch_one_pair<S, 1, -1, -1, RK>(a, m8, mp, err, counter, st, nlaunch);
    case 5: return launch_one_pair<S, 1, -1, 1, RK>(a, m8, mp, err, counter, st, nlaunch);
    case 6: return launch_one_pair<S, 1, 1, -1, RK>(a, m8, mp, err, counter, st, nlaunch);
    default: return launch_one_pair<S, 1, 1, 1, RK>(a, m8, mp, err, counter, st, nlaunch);
  }
}
template <typename S>
cudaError_t launch_pair(const StageArgs<S> &a, const MapSet &ms, int *err, int *counter,
                        cudaStream_t st, int *nlaunch) {
  switch (rk_class(a.irk)) {
    case 0: return launch_fb_rk_pair<S, 0>(a, ms, err, counter, st, nlaunch);
    case 1: return launch_fb_rk_pair<S, 1>(a, ms, err, counter, st, nlaunch);
    default: return launch_fb_rk_pair<S, 3>(a, ms, err, counter, st, nlaunch);
  }
}

template <typename S, int TYv>
cudaError_t launch_fb(const StageArgs<S> &a, const Maps &m, int *err, int *counter,
                      cudaStream_t st, int *nlaunch) {
  switch (rk_class(a.irk)) {
    case 0: return launch_fb_rk<S, TYv, 0>(a, m, err, counter, st, nlaunch);
    case 1: return launch_fb_rk<S, TYv, 1>(a, m, err, counter, st, nlaunch);
    default: return launch_fb_rk<S, TYv, 3>(a, m, err, counter, st, nlaunch);
  }
}

template <typename S, int RK>
cudaError_t launch_batch_rk(const StageArgs<S> *args, const void *const *maps, int n, int *err,
                            int *counter, cudaStream_t st, int *nlaunch) {
  const StageArgs<S> &a = args[0];
  switch ((a.fb1 > 0) * 4 + (a.fb2 > 0) * 2 + (a.fb3 > 0)) {
    case 0: return launch_batch<S, -1, -1, -1, RK>(args, maps, n, err, counter, st, nlaunch);
    case 1: return launch_batch<S, -1, -1, 1, RK>(args, maps, n, err, counter, st, nlaunch);
    case 2: return launch_batch<S, -1, 1, -1, RK>(args, maps, n, err, counter, st, nlaunch);
    case 3: return launch_batch<S, -1, 1, 1, RK>(args, maps, n, err, counter, st, nlaunch);
    case 4: return launch_batch<S, 1, -1, -1, RK>(args, maps, n, err, counter, st, nlaunch);
    case 5: return launch_batch<S, 1, -1, 1, RK>(args, maps, n, err, counter, st, nlaunch);
    case 6: return launch_batch<S, 1, 1, -1, RK>(args, maps, n, err, counter, st, nlaunch);
    default: return launch_batch<S, 1, 1, 1, RK>(args, maps, n, err, counter, st, nlaunch);
  }
}

template <typename S>
cudaError_t launch_stage_stream(const StageArgs<S> &a, const void *maps_in, int *err, int *counter,
                                cudaStream_t st, cudaEvent_t after_main, int *nlaunch,
                                int tile_rows) {
  if (a.kend <= a.kbeg) return cudaSuccess;
  const MapSet &ms = *(const MapSet *)maps_in;
  // tile height 16 runs the batched kernel as a batch of one, so that a
  // scenario gives the same bits alone and inside a batch
  cudaError_t e;
  if (tile_rows == kTilePair) {
    if constexpr (sizeof(S) == 2)
      e = launch_pair<S>(a, ms, err, counter, st, nlaunch);
    else
      e = cudaErrorInvalidValue;
  } else {
    e = tile_rows == 8 ? launch_fb<S, 8>(a, ms.ty8, err, counter, st, nlaunch)
                       : launch_stage_stream_batch<S>(&a, &maps_in, 1, err, counter, st, nlaunch);
  }
  if (e != cudaSuccess) return e;
  if (after_main) e = cudaEventRecord(after_main, st);
  return e;
}
template <typename S>
cudaError_t launch_stage_stream_batch(const StageArgs<S> *args, const void *const *maps, int n,
                                      int *err, int *counter, cudaStream_t st, int *nlaunch) {
  if (n <= 0) return cudaSuccess;
  for (int q = 1; q < n; ++q)
    if (args[q].fb1 != args[0].fb1 || args[q].fb2 != args[0].fb2 || args[q].fb3 != args[0].fb3 ||
        args[q].irk != args[0].irk)
      return cudaErrorInvalidValue;
  switch (rk_class(args[0].irk)) {
    case 0: return launch_batch_rk<S, 0>(args, maps, n, err, counter, st, nlaunch);
    case 1: return launch_batch_rk<S, 1>(args, maps, n, err, counter, st, nlaunch);
    default: return launch_batch_rk<S, 3>(args, maps, n, err, counter, st, nlaunch);
  }
}

}  // namespace cgfdm
