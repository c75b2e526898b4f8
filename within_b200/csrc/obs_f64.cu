// FP64 observation-pass kernels (every mode; LSMR runs in FP64 only).
#define WB_OBS_DEFINE
#include "obs_launch.cuh"

namespace wb {
template cudaError_t obs_dispatch<double, OBS_GRAM>(const ObsParams&, int, int, int, int, size_t, cudaStream_t, const double*,
                                                    const double*, const double*, double*, double*);
template cudaError_t obs_dispatch<double, OBS_RHS>(const ObsParams&, int, int, int, int, size_t, cudaStream_t, const double*,
                                                   const double*, const double*, double*, double*);
template cudaError_t obs_dispatch<double, OBS_RESID>(const ObsParams&, int, int, int, int, size_t, cudaStream_t, const double*,
                                                     const double*, const double*, double*, double*);
template cudaError_t obs_dispatch<double, OBS_DX>(const ObsParams&, int, int, int, int, size_t, cudaStream_t, const double*,
                                                  const double*, const double*, double*, double*);
template cudaError_t obs_dispatch<double, OBS_LSMR>(const ObsParams&, int, int, int, int, size_t, cudaStream_t, const double*,
                                                    const double*, const double*, double*, double*);
}  // namespace wb
