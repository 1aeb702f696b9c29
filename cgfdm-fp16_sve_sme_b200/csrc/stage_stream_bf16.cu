// Streaming stage kernels for BF16 storage.
#include "stage_stream.cuh"

namespace cgfdm {

template cudaError_t launch_stage_stream_batch<__nv_bfloat16>(const StageArgs<__nv_bfloat16> *,
                                                              const void *const *, int, int *,
                                                              int *, cudaStream_t, int *);
template bool stage_stream_supported<__nv_bfloat16>();
template int encode_stream_maps<__nv_bfloat16>(const __nv_bfloat16 *, const __nv_bfloat16 *,
                                               const __nv_bfloat16 *, const __nv_bfloat16 *,
                                               const Layout &, void *);
template cudaError_t launch_stage_stream<__nv_bfloat16>(const StageArgs<__nv_bfloat16> &,
                                                        const void *, int *, int *, cudaStream_t, cudaEvent_t, int *, int);

}  // namespace cgfdm
