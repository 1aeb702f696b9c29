// Host-visible launchers of the device kernels.
#pragma once
#include <cuda_runtime.h>

#include "device_common.cuh"

namespace cgfdm {

// Storage scaling of the reduced-precision forms (macro.h:65-73): velocities
// are stored times Cv, stresses times Cs, buoyancy divided by Crho.  FP32 and
// FP64 are unscaled.
template <typename S> struct CRHO_OF { static constexpr double v = 1.0; };
template <> struct CRHO_OF<__half> { static constexpr double v = 1e6; };
template <> struct CRHO_OF<__nv_bfloat16> { static constexpr double v = 1e6; };
template <typename S> struct SCALE_OF { static constexpr double cv = 1.0, cs = 1.0; };
template <> struct SCALE_OF<__half> { static constexpr double cv = 5.0e3, cs = 1.0e-6; };
template <> struct SCALE_OF<__nv_bfloat16> { static constexpr double cv = 5.0e3, cs = 1.0e-6; };

// Exact-order fused stage over the points kbeg <= k < kend (all i, j).
template <typename S> cudaError_t launch_stage_exact(const StageArgs<S> &a, cudaStream_t st);

// The three free-surface layers of the fast path: a shared-memory tiled
// kernel for the columns outside every PML slab and the exact-order kernel
// for the slab columns (FP32, FP16, BF16 storage).
template <typename S> cudaError_t launch_stage_top(const StageArgs<S> &a, cudaStream_t st);

// TMA-staged z-streaming fused stage over kbeg <= k < kend, which must lie
// below the three free-surface layers.  `maps` holds the tensor maps of the
// stage input wavefield and of the coefficients (encode_stream_maps).
constexpr int kStreamMapsBytes = 2048;
// Tile form code of the paired-point kernel (16-bit storage): 64 x 8 tiles,
// two x-adjacent points per thread.
constexpr int kTilePair = 64;
// `after_main` (optional) is recorded right after the streaming kernel,
// before the exact-order kernel; `nlaunch` (optional) is increased by the
// number of kernels launched; `tile_rows` selects the tile form: 16 (32 x 16
// tiles, one CTA per SM), 8 (32 x 8, two CTAs per SM) or kTilePair (16-bit
// storage: the paired-point kernel on 64 x 8 interior tiles, the 32 x 8 PML
// variant elsewhere).
template <typename S>
cudaError_t launch_stage_stream(const StageArgs<S> &a, const void *maps, int *err_flag,
                                int *work_counter, cudaStream_t st,
                                cudaEvent_t after_main = nullptr, int *nlaunch = nullptr,
                                int tile_rows = 16);
// One stage (same irk and MacCormack signs for all) of n scenarios in
// persistent launches whose work queue spans all of them (16 scenarios per
// launch pair); maps[q] is scenario q's encode_stream_maps buffer.  Tile
// height 16.
template <typename S>
cudaError_t launch_stage_stream_batch(const StageArgs<S> *args, const void *const *maps, int n,
                                      int *err_flag, int *work_counter, cudaStream_t st,
                                      int *nlaunch = nullptr);
template <typename S> bool stage_stream_supported();
// Encodes the tensor maps the streaming kernel loads its tiles through (the
// 9 wavefield components of the stage input `wave`, the 13 coefficient
// fields of `cjm`, the step state `wm` and the RK accumulator `t`) into `out`
// (kStreamMapsBytes, 64-byte aligned host memory).
template <typename S>
int encode_stream_maps(const S *wave, const S *cjm, const S *wm, const S *t, const Layout &L,
                       void *out);

// Per-step values come from device memory so that a step can be replayed as
// a CUDA graph: `step` points at the device step counter, advanced by the
// station / PGV launch at the end of every step.

// Smoothed point source (singleSource.cpp:78-127) with the source moment
// moment[*step]: adds value(cell) to Txx, Tyy, Tzz of w0 and, for cells in
// the halo, of w1 and w2 too (halo cells hold constant values that every
// stage buffer must share).
template <typename S>
cudaError_t launch_point_source(S *w0, S *w1, S *w2, const S *cjm, Layout L, int sx, int sy,
                                int sz, const float *amp343, const float *moment, const int *step,
                                float DH3, double CsDT, cudaStream_t st);

// Finite-fault injection (addMoment.cpp:98-219, NO_SOURCE_SMOOTH) at the
// interpolation index src_it[*step] (negative: the source has ended) and
// weight src_tw[*step]; idx are offsets in the HBM layout.
template <typename S>
cudaError_t launch_fault_source(S *w, long long fs, const long long *idx, const float *rate,
                                long long npts, const int *src_it, const float *src_tw,
                                const int *step, float DT, cudaStream_t st);

// Station sampling (station.cpp:310-347) and PGV (PGV.cpp:49-101) of step
// step[0], which the same launch then advances by one (step[1] is the
// launch's block counter, zero between launches).
template <typename S>
cudaError_t launch_station_pgv(const S *w, Layout L, const int *xyz, int nsta, int NT,
                               int *step, float *wave, float *pgv, float c1, float c2,
                               double cv_inv, cudaStream_t st);

// One field's interior slice at padded index `at` along axis 0/1/2, times
// c (data_io.cpp:86-231).
template <typename S>
cudaError_t launch_slice_pack(const S *field, Layout L, int axis, int at, double c, float *out,
                              cudaStream_t st);

// Reference layout (float, nfield x num) <-> HBM layout (S, nfield x fs).
template <typename S>
cudaError_t launch_repack_in(const float *src, S *dst, Layout L, int nfield, cudaStream_t st);
template <typename S>
cudaError_t launch_repack_out(const S *src, float *dst, Layout L, int nfield, cudaStream_t st);

}  // namespace cgfdm
