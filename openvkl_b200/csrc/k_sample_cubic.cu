// cubic filter instantiation of the sampling kernels (sample_kernels.cuh).
#include "sample_kernels.cuh"

namespace vklcuda {
template void dispatchFilter<kFilterCubic>(const DevGrid &, uint32_t, uint64_t, const float *, uint32_t,
                                  float *, bool, cudaStream_t);
}  // namespace vklcuda
