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

template <typename S> cudaError_t launch_stage_exact(const StageArgs<S> &a, cudaStream_t st);

// Streaming fused stage kernel (FP32/FP16/BF16 storage).
template <typename S> cudaError_t launch_stage_stream(const StageArgs<S> &a, cudaStream_t st);
template <typename S> bool stage_stream_supported(const StageArgs<S> &a);

// Smoothed point source (singleSource.cpp:78-127): adds value(cell) to
// Txx, Tyy, Tzz of w0 and, for cells in the halo, of w1 and w2 too (halo
// cells hold constant values that every stage buffer must share).
template <typename S>
cudaError_t launch_point_source(S *w0, S *w1, S *w2, const S *cjm, long long num, int nx_, int ny_,
                                int nz_, int sx, int sy, int sz, const float *amp343, float s,
                                float DH3, double CsDT, cudaStream_t st);

// Finite-fault injection (addMoment.cpp:98-219, NO_SOURCE_SMOOTH).
template <typename S>
cudaError_t launch_fault_source(S *w, long long num, const long long *idx, const float *rate,
                                long long npts, int srcIt, float tw, float DT, cudaStream_t st);

// Station sampling (station.cpp:310-347) and PGV (PGV.cpp:49-101).
template <typename S>
cudaError_t launch_station_pgv(const S *w, long long num, int nx_, int ny_, int nz_, const int *xyz,
                               int nsta, int NT, int it, float *wave, float *pgv, float c1, float c2,
                               double cv_inv, cudaStream_t st);

// Top-layer velocity snapshot [3][ny][nx] (data_io.cpp:186-231 on the free
// surface slice).
template <typename S>
cudaError_t launch_free_surface_pack(const S *w, long long num, int nx_, int ny_, int nz_,
                                     double cv_inv, float *out, cudaStream_t st);
// Generic slice pack of one field: axis 0/1/2 at padded index `at`.
template <typename S>
cudaError_t launch_slice_pack(const S *field, int nx_, int ny_, int nz_, int axis, int at,
                              double c, float *out, cudaStream_t st);

// float <-> storage conversions on the device.
template <typename S> cudaError_t launch_convert_in(const float *src, S *dst, long long n, cudaStream_t st);
template <typename S> cudaError_t launch_convert_out(const S *src, float *dst, long long n, cudaStream_t st);

}  // namespace cgfdm
