// Streaming stage kernels for FP16 storage.
#include "stage_stream.cuh"

namespace cgfdm {

template cudaError_t launch_stage_stream_batch<__half>(const StageArgs<__half> *,
                                                       const void *const *, int, int *, int *,
                                                       cudaStream_t, int *);
template bool stage_stream_supported<__half>();
template int encode_stream_maps<__half>(const __half *, const __half *, const __half *,
                                        const __half *, const Layout &, void *);
template cudaError_t launch_stage_stream<__half>(const StageArgs<__half> &, const void *, int *,
                                                 int *, cudaStream_t, cudaEvent_t, int *, int);

}  // namespace cgfdm
