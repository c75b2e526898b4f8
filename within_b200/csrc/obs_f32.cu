// FP32 observation-pass kernels (the operator apply of the mixed-precision inner solves).
#define WB_OBS_DEFINE
#include "obs_launch.cuh"

namespace wb {
template cudaError_t obs_dispatch<float, OBS_GRAM>(const ObsParams&, int, int, int, int, size_t, cudaStream_t, const float*,
                                                   const float*, const float*, float*, float*);
}  // namespace wb
