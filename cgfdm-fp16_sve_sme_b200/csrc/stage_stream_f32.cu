// Streaming stage kernels for FP32 storage.
#include "stage_stream.cuh"

namespace cgfdm {

// FP64 has no streaming kernel (the exact-order kernel runs it)
template <> bool stage_stream_supported<double>() { return false; }

template <>
int encode_stream_maps<double>(const double *, const double *, const double *, const double *,
                               const Layout &, void *) {
  set_error("no streaming kernel for FP64");
  return CGFDM_ERR_ARG;
}

template <>
cudaError_t launch_stage_stream_batch<double>(const StageArgs<double> *, const void *const *, int,
                                              int *, int *, cudaStream_t, int *) {
  return cudaErrorNotSupported;
}

template <>
cudaError_t launch_stage_stream<double>(const StageArgs<double> &, const void *, int *, int *,
                                        cudaStream_t, cudaEvent_t, int *, int) {
  return cudaErrorNotSupported;
}

template cudaError_t launch_stage_stream_batch<float>(const StageArgs<float> *,
                                                      const void *const *, int, int *, int *,
                                                      cudaStream_t, int *);
template bool stage_stream_supported<float>();
template int encode_stream_maps<float>(const float *, const float *, const float *, const float *,
                                       const Layout &, void *);
template cudaError_t launch_stage_stream<float>(const StageArgs<float> &, const void *, int *,
                                                int *, cudaStream_t, cudaEvent_t, int *, int);

}  // namespace cgfdm
