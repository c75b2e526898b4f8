// Launch of the observation pass (obs_pass_kernel), compiled in its own translation
// units (obs_f64.cu, obs_f32.cu) so that its many instantiations build in parallel
// with the rest of the library.
#pragma once

#include <cuda_runtime.h>

#include <type_traits>

#include "kernels.cuh"

namespace wb {

// Picks the exact kernel for P.Q <= 4 with the trailing np private slots (Q = 4: np <= 1),
// else the generic one, for G lanes per row of rv 4-wide RHS vectors each (rv = 2: wide
// lanes, FP32 operator apply, exact kernels only), and launches `grid` blocks of
// obs_block<T, rv>() threads on `stream`.
template <typename T, int MODE>
cudaError_t obs_dispatch(const ObsParams& P, int np, int G, int rv, int grid, size_t smem, cudaStream_t stream,
                         const T* w, const T* x, const T* yin, T* out, T* eout);

#ifdef WB_OBS_DEFINE
template <typename T, int MODE>
cudaError_t obs_dispatch(const ObsParams& P, int np, int G, int rv, int grid, size_t smem, cudaStream_t stream,
                         const T* w, const T* x, const T* yin, T* out, T* eout) {
    cudaError_t err = cudaSuccess;
    int bt = obs_block<T>();
    auto go = [&](auto kern) {
        if (smem > 48 * 1024) {
            err = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
            if (err != cudaSuccess) return;
        }
        kern<<<grid, bt, smem, stream>>>(P, w, x, yin, out, eout);
        err = cudaGetLastError();
    };
    if constexpr (std::is_same<T, float>::value && MODE == OBS_GRAM) {
        if (rv == 2) {
            bt = obs_block<T, 2>();
            auto wide = [&](auto gtag) {
                constexpr int GV = decltype(gtag)::value;
                switch (P.Q * 8 + (np < 2 ? np : 2)) {
                    case 1 * 8 + 0: go(obs_pass_kernel<T, GV, MODE, 1, 0, 2>); break;
                    case 2 * 8 + 0: go(obs_pass_kernel<T, GV, MODE, 2, 0, 2>); break;
                    case 2 * 8 + 1: go(obs_pass_kernel<T, GV, MODE, 2, 1, 2>); break;
                    case 3 * 8 + 0: go(obs_pass_kernel<T, GV, MODE, 3, 0, 2>); break;
                    case 3 * 8 + 1: go(obs_pass_kernel<T, GV, MODE, 3, 1, 2>); break;
                    case 3 * 8 + 2: go(obs_pass_kernel<T, GV, MODE, 3, 2, 2>); break;
                    case 4 * 8 + 0: go(obs_pass_kernel<T, GV, MODE, 4, 0, 2>); break;
                    case 4 * 8 + 1: go(obs_pass_kernel<T, GV, MODE, 4, 1, 2>); break;
                    default: err = cudaErrorInvalidValue; break;  // no generic wide kernel
                }
            };
            switch (G) {
                case 1: wide(std::integral_constant<int, 1>{}); break;
                case 2: wide(std::integral_constant<int, 2>{}); break;
                case 4: wide(std::integral_constant<int, 4>{}); break;
                default: err = cudaErrorInvalidValue; break;
            }
            return err;
        }
    }
    if (rv != 1) return cudaErrorInvalidValue;
    auto by_q = [&](auto gtag) {
        constexpr int GV = decltype(gtag)::value;
        switch (P.Q * 8 + (np < 2 ? np : 2)) {
            case 1 * 8 + 0: go(obs_pass_kernel<T, GV, MODE, 1, 0>); break;
            case 2 * 8 + 0: go(obs_pass_kernel<T, GV, MODE, 2, 0>); break;
            case 2 * 8 + 1: go(obs_pass_kernel<T, GV, MODE, 2, 1>); break;
            case 3 * 8 + 0: go(obs_pass_kernel<T, GV, MODE, 3, 0>); break;
            case 3 * 8 + 1: go(obs_pass_kernel<T, GV, MODE, 3, 1>); break;
            case 3 * 8 + 2: go(obs_pass_kernel<T, GV, MODE, 3, 2>); break;
            case 4 * 8 + 0: go(obs_pass_kernel<T, GV, MODE, 4, 0>); break;
            case 4 * 8 + 1: go(obs_pass_kernel<T, GV, MODE, 4, 1>); break;
            default: go(obs_pass_kernel<T, GV, MODE, kMaxQ, 0>); break;  // reads every slot's sink
        }
    };
    switch (G) {
        case 1: by_q(std::integral_constant<int, 1>{}); break;
        case 2: by_q(std::integral_constant<int, 2>{}); break;
        case 4: by_q(std::integral_constant<int, 4>{}); break;
        default: by_q(std::integral_constant<int, 8>{}); break;
    }
    return err;
}
#endif

}  // namespace wb
