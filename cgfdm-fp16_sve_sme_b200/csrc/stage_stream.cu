// Streaming fused stage kernel: placeholder until the TMA-staged kernel
// lands; reports itself unsupported so the exact kernel runs.
#include "kernels.h"

namespace cgfdm {

template <typename S> bool stage_stream_supported(const StageArgs<S> &) { return false; }

template <typename S> cudaError_t launch_stage_stream(const StageArgs<S> &, cudaStream_t) {
  return cudaErrorNotSupported;
}

template bool stage_stream_supported<float>(const StageArgs<float> &);
template bool stage_stream_supported<__half>(const StageArgs<__half> &);
template bool stage_stream_supported<__nv_bfloat16>(const StageArgs<__nv_bfloat16> &);
template bool stage_stream_supported<double>(const StageArgs<double> &);
template cudaError_t launch_stage_stream<float>(const StageArgs<float> &, cudaStream_t);
template cudaError_t launch_stage_stream<__half>(const StageArgs<__half> &, cudaStream_t);
template cudaError_t launch_stage_stream<__nv_bfloat16>(const StageArgs<__nv_bfloat16> &, cudaStream_t);
template cudaError_t launch_stage_stream<double>(const StageArgs<double> &, cudaStream_t);

}  // namespace cgfdm
