// Learned coarse space: the message-passing network over the level graph (forward on
// BF16 tensor cores with FP32 accumulation, backward on FP32 CUDA cores), its loss
// against Ritz-vector targets, and the coarse correction z += Z E^+ Z' r that CG adds to
// the additive Schwarz output.  There is no counterpart in the reference: the
// correction augments its additive Schwarz apply (schwarz-precond/src/schwarz/additive/
// executor.rs:59-147) inside its CG (schwarz-precond/src/solve/cg.rs:45-133), which stays
// valid because Schwarz + Z E^+ Z' is symmetric positive semi-definite.
//
// Network (per level l of every factor; d = diag(G), G = D'WD):
//   X = [one-hot(min(factor,3)), log1p(d)/8, log1p(count)/8, 10 probe signs]   (m x 16)
//   Ahat h = D^-1/2 (G - diag G) D^-1/2 h   (0 on unobserved levels)
//   S_l = [Ahat H_l, H_l];  H_{l+1} = tanh(bf16(S_l) bf16(W_l) + b_l),  l = 0, 1, 2
//   Zt = bf16(H_3) bf16(W_o)   (m x 32, scaled space);  Z = D^-1/2 Zt
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>

#include "kernels.cuh"

namespace wb {

constexpr int kCnIn = 16, kCnHidden = 64, kCnOut = 32, kCnProbe = 10, kCnLayers = 3;
// parameter vector: per layer W_l (2 F_l x 64, row-major) then b_l (64); then W_o (64 x 32)
constexpr int64_t kCnParams = (2 * kCnIn * kCnHidden + kCnHidden) + 2 * (2 * kCnHidden * kCnHidden + kCnHidden) +
                              kCnHidden * kCnOut;

// splitmix64 finalizer (Steele, Lea & Flood 2014)
__host__ __device__ __forceinline__ uint64_t splitmix_fin(uint64_t z) {
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

struct CnOffsets {
    int32_t Q;
    int64_t off[kMaxQ + 1];  // level offsets of the factors, off[Q] = m
};

// Features of every level (m x 16, row-major).
__global__ void cn_features_kernel(int64_t m, CnOffsets fo, const double* __restrict__ d,
                                   const double* __restrict__ cnt, uint64_t seed, float* __restrict__ X) {
    const int64_t l = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (l >= m) return;
    int q = 0;
    while (q + 1 < fo.Q && l >= fo.off[q + 1]) ++q;
    float* x = X + (size_t)l * kCnIn;
    for (int c = 0; c < 4; ++c) x[c] = (c == (q < 3 ? q : 3)) ? 1.f : 0.f;
    x[4] = (float)(log1p(d[l]) / 8.0);
    x[5] = (float)(log1p(cnt[l]) / 8.0);
    const uint64_t base = 0x9E3779B97F4A7C15ull * (seed + 1);
    for (int c = 0; c < kCnProbe; ++c)
        x[6 + c] = (splitmix_fin((uint64_t)l * 64u + (uint64_t)c + base) & 1u) ? 1.f : -1.f;
}

// T (m x kt) = isq * H[:, c0:c0+kt]  (the scaled input of one message-passing pass; kt <= 32)
__global__ void cn_scale_cols_kernel(int64_t m, int F, int c0, int kt, const float* __restrict__ H,
                                     const double* __restrict__ isq, float* __restrict__ T) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m * kt) return;
    const int64_t row = i / kt;
    const int j = (int)(i % kt);
    T[i] = (float)(isq[row] * (double)H[(size_t)row * F + c0 + j]);
}

// P[:, c0:c0+kt] (+)= isq * GT - H[:, c0:c0+kt] on observed levels, 0 on the others:
// Ahat of one column block.  accumulate: add to P instead of storing (backward pass).
__global__ void cn_combine_kernel(int64_t m, int F, int c0, int kt, const float* __restrict__ GT,
                                  const double* __restrict__ isq, const float* __restrict__ H, float* __restrict__ P,
                                  int PF, int pc0, int accumulate) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m * kt) return;
    const int64_t row = i / kt;
    const int j = (int)(i % kt);
    const double s = isq[row];
    const float v = s > 0.0 ? (float)(s * (double)GT[i] - (double)H[(size_t)row * F + c0 + j]) : 0.f;
    float* p = P + (size_t)row * PF + pc0 + j;
    *p = accumulate ? *p + v : v;
}

__device__ __forceinline__ uint32_t pack_bf16x2(float lo, float hi) {
    const __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<const uint32_t*>(&v);
}

// out (m x N) = act(bf16([A0 | A1]) bf16(W) + bias): A0 is m x K0, A1 is m x K1 (row-major
// FP32, either may be absent with K = 0), W is (K0+K1) x N row-major BF16, bias N FP32
// (or null).  One warp per 16 rows, mma.sync m16n8k16 (BF16 in, FP32 accumulate), the
// weights staged in shared memory.  ACT 1: tanh.  N in {32, 64}; K0, K1 multiples of 16.
template <int N, int ACT>
__global__ void __launch_bounds__(128) cn_dense_fwd_kernel(int64_t m, const float* __restrict__ A0, int K0,
                                                           const float* __restrict__ A1, int K1,
                                                           const __nv_bfloat16* __restrict__ W,
                                                           const float* __restrict__ bias, float* __restrict__ out) {
    constexpr int NT = N / 8;
    extern __shared__ __align__(16) unsigned char cn_smem[];
    __nv_bfloat16* Ws = reinterpret_cast<__nv_bfloat16*>(cn_smem);
    const int K = K0 + K1;
    for (int i = threadIdx.x; i < K * N; i += blockDim.x) Ws[i] = W[i];
    __syncthreads();
    const int lane = threadIdx.x & 31, gid = lane >> 2, tig = lane & 3;
    const int64_t row0 = ((int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5)) * 16;
    if (row0 >= m) return;
    const int64_t ra = row0 + gid, rb = row0 + gid + 8;
    auto ld2 = [&](int64_t r, int k) -> float2 {
        if (r >= m) return make_float2(0.f, 0.f);
        if (k < K0) return *reinterpret_cast<const float2*>(A0 + (size_t)r * K0 + k);
        return *reinterpret_cast<const float2*>(A1 + (size_t)r * K1 + (k - K0));
    };
    float acc[NT][4];
#pragma unroll
    for (int t = 0; t < NT; ++t) acc[t][0] = acc[t][1] = acc[t][2] = acc[t][3] = 0.f;
    for (int k0 = 0; k0 < K; k0 += 16) {
        const float2 a00 = ld2(ra, k0 + tig * 2), a10 = ld2(rb, k0 + tig * 2);
        const float2 a01 = ld2(ra, k0 + tig * 2 + 8), a11 = ld2(rb, k0 + tig * 2 + 8);
        const uint32_t a0 = pack_bf16x2(a00.x, a00.y), a1 = pack_bf16x2(a10.x, a10.y);
        const uint32_t a2 = pack_bf16x2(a01.x, a01.y), a3 = pack_bf16x2(a11.x, a11.y);
#pragma unroll
        for (int t = 0; t < NT; ++t) {
            const int n = t * 8 + gid;
            const int kb = k0 + tig * 2;
            __nv_bfloat162 b01, b23;
            b01.x = Ws[(size_t)kb * N + n];
            b01.y = Ws[(size_t)(kb + 1) * N + n];
            b23.x = Ws[(size_t)(kb + 8) * N + n];
            b23.y = Ws[(size_t)(kb + 9) * N + n];
            const uint32_t b0 = *reinterpret_cast<const uint32_t*>(&b01);
            const uint32_t b1 = *reinterpret_cast<const uint32_t*>(&b23);
            asm volatile(
                "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
                "{%0,%1,%2,%3};\n"
                : "+f"(acc[t][0]), "+f"(acc[t][1]), "+f"(acc[t][2]), "+f"(acc[t][3])
                : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
        }
    }
#pragma unroll
    for (int t = 0; t < NT; ++t) {
        const int c = t * 8 + tig * 2;
        float v[4] = {acc[t][0], acc[t][1], acc[t][2], acc[t][3]};
        if (bias) {
            v[0] += bias[c]; v[1] += bias[c + 1]; v[2] += bias[c]; v[3] += bias[c + 1];
        }
        if (ACT == 1)
            for (int e = 0; e < 4; ++e) v[e] = tanhf(v[e]);
        if (ra < m) *reinterpret_cast<float2*>(out + (size_t)ra * N + c) = make_float2(v[0], v[1]);
        if (rb < m) *reinterpret_cast<float2*>(out + (size_t)rb * N + c) = make_float2(v[2], v[3]);
    }
}

// Block partials of C (K x N) = sum_rows a[row][k] b[row][n], a = [A0 | A1] (FP32, rounded
// to BF16 when round_a, as the forward pass saw it), b (m x N).  K <= 128, N <= 64,
// K*N <= 32 * blockDim.x; rows staged 32 at a time in shared memory; partial[blk][K*N].
template <typename TACC>
__global__ void __launch_bounds__(256) cn_tn_partial_kernel(int64_t m, const float* __restrict__ A0, int K0,
                                                            const float* __restrict__ A1, int K1, int round_a,
                                                            const float* __restrict__ B, int N,
                                                            TACC* __restrict__ partial) {
    constexpr int R = 32;
    __shared__ float As[R][128];
    __shared__ float Bs[R][64];
    const int K = K0 + K1;
    const int KN = K * N;
    TACC acc[32];
#pragma unroll
    for (int i = 0; i < 32; ++i) acc[i] = TACC(0);
    const int64_t rows_per_blk = (m + gridDim.x - 1) / gridDim.x;
    const int64_t r0 = (int64_t)blockIdx.x * rows_per_blk, r1 = min(m, r0 + rows_per_blk);
    for (int64_t t0 = r0; t0 < r1; t0 += R) {
        const int nr = (int)min((int64_t)R, r1 - t0);
        __syncthreads();
        for (int i = threadIdx.x; i < R * K; i += blockDim.x) {
            const int r = i / K, k = i % K;
            float a = 0.f;
            if (r < nr) {
                const int64_t row = t0 + r;
                a = k < K0 ? A0[(size_t)row * K0 + k] : A1[(size_t)row * K1 + (k - K0)];
                if (round_a) a = __bfloat162float(__float2bfloat16_rn(a));
            }
            As[r][k] = a;
        }
        for (int i = threadIdx.x; i < R * N; i += blockDim.x) {
            const int r = i / N, n = i % N;
            Bs[r][n] = r < nr ? B[(size_t)(t0 + r) * N + n] : 0.f;
        }
        __syncthreads();
#pragma unroll
        for (int i = 0; i < 32; ++i) {
            const int o = threadIdx.x + i * blockDim.x;
            if (o < KN) {
                const int k = o / N, n = o % N;
                TACC s = acc[i];
                for (int r = 0; r < nr; ++r) s += (TACC)As[r][k] * (TACC)Bs[r][n];
                acc[i] = s;
            }
        }
    }
#pragma unroll
    for (int i = 0; i < 32; ++i) {
        const int o = threadIdx.x + i * blockDim.x;
        if (o < KN) partial[(size_t)blockIdx.x * KN + o] = acc[i];
    }
}

// out[o] = sum_b partial[b][o] (fixed order: deterministic)
template <typename TACC, typename TOUT>
__global__ void cn_reduce_partials_kernel(const TACC* __restrict__ partial, int nb, int64_t len, TOUT* __restrict__ out) {
    const int64_t o = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (o >= len) return;
    TACC s = TACC(0);
    for (int b = 0; b < nb; ++b) s += partial[(size_t)b * len + o];
    out[o] = (TOUT)s;
}

// dpre = dH * (1 - Hn^2)
__global__ void cn_dtanh_kernel(int64_t n, const float* __restrict__ dH, const float* __restrict__ Hn,
                                float* __restrict__ dpre) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) dpre[i] = dH[i] * (1.f - Hn[i] * Hn[i]);
}

// out (m x K) = D (m x N) W' with W (K x N) BF16: out[row][k] = sum_n D[row][n] W[k][n]
__global__ void __launch_bounds__(256) cn_matmul_nt_kernel(int64_t m, const float* __restrict__ D, int N,
                                                           const __nv_bfloat16* __restrict__ W, int K,
                                                           float* __restrict__ out) {
    extern __shared__ __align__(16) unsigned char cn_smem[];
    float* Ws = reinterpret_cast<float*>(cn_smem);
    for (int i = threadIdx.x; i < K * N; i += blockDim.x) Ws[i] = __bfloat162float(W[i]);
    __syncthreads();
    const int64_t total = m * K;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t row = i / K;
        const int k = (int)(i % K);
        const float* d = D + (size_t)row * N;
        const float* w = Ws + (size_t)k * N;
        float s = 0.f;
        for (int n = 0; n < N; ++n) s += d[n] * w[n];
        out[i] = s;
    }
}

// dst[row][j] = src[row][c0 + j], j < kt (a column block of a row-major matrix)
__global__ void cn_copy_cols_kernel(int64_t m, int F, int c0, int kt, const float* __restrict__ src,
                                    float* __restrict__ dst, int DF, int dc0) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m * kt) return;
    const int64_t row = i / kt;
    const int j = (int)(i % kt);
    dst[(size_t)row * DF + dc0 + j] = src[(size_t)row * F + c0 + j];
}

// dZ (m x 32) = V C1 + Z C2: V (m x t), C1 (t x 32), Z (m x 32), C2 (32 x 32), all FP64
// coefficients from the host (C1 = -2/t B'A^-1, C2 = 2/t A^-1 B B'A^-1).
__global__ void cn_dz_kernel(int64_t m, const float* __restrict__ V, int t, const double* __restrict__ C1,
                             const float* __restrict__ Z, const double* __restrict__ C2, float* __restrict__ dZ) {
    __shared__ double c1[32 * 32], c2[32 * 32];
    for (int i = threadIdx.x; i < t * 32; i += blockDim.x) c1[i] = C1[i];
    for (int i = threadIdx.x; i < 32 * 32; i += blockDim.x) c2[i] = C2[i];
    __syncthreads();
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m * 32) return;
    const int64_t row = i / 32;
    const int j = (int)(i % 32);
    double s = 0.0;
    for (int a = 0; a < t; ++a) s += (double)V[(size_t)row * t + a] * c1[a * 32 + j];
    for (int a = 0; a < 32; ++a) s += (double)Z[(size_t)row * 32 + a] * c2[a * 32 + j];
    dZ[i] = (float)s;
}

// Z = isq * Zt (the coarse basis in dof coordinates), as FP64 and FP32 copies.
__global__ void cn_unscale_kernel(int64_t m, const float* __restrict__ Zt, const double* __restrict__ isq,
                                  double* __restrict__ Z64, float* __restrict__ Z32) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m * kCnOut) return;
    const double v = isq[i / kCnOut] * (double)Zt[i];
    Z64[i] = v;
    if (Z32) Z32[i] = (float)v;
}

// Adam on the FP32 masters (Kingma & Ba 2015), with the BF16 copies the forward pass reads.
__global__ void cn_adam_kernel(int64_t n, float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m1,
                               float* __restrict__ m2, float lr, float b1, float b2, float eps, float c1, float c2,
                               __nv_bfloat16* __restrict__ pb) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float gi = g[i];
    const float a = b1 * m1[i] + (1.f - b1) * gi;
    const float b = b2 * m2[i] + (1.f - b2) * gi * gi;
    m1[i] = a;
    m2[i] = b;
    const float v = p[i] - lr * (a / c1) / (sqrtf(b / c2) + eps);
    p[i] = v;
    pb[i] = __float2bfloat16_rn(v);
}

__global__ void cn_to_bf16_kernel(int64_t n, const float* __restrict__ p, __nv_bfloat16* __restrict__ pb) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) pb[i] = __float2bfloat16_rn(p[i]);
}

// ---------------------------------------------------------------------------
// Coarse correction inside CG, balancing form (Mandel 1993, BNN):
//   z = P' M^-1 P r + Q r,  Q = Z E^+ Z',  P = I - G Q,  E = Z' G Z
// With GZ = G Z kept on the device: u1 = E^+ Z' r;  y = M^-1 (r - GZ u1);
// u2 = E^+ (GZ)' y;  z = y + Z (u1 - u2).  Symmetric, and on span(Z) the preconditioned
// operator is the identity while its other eigenvalues stay within the Schwarz bounds.
// ---------------------------------------------------------------------------

constexpr int kCoarseTileRows = 64;

// Block partials of C (32 x kp) = A' B, A: m x 32 (Z or GZ), B: m x kp interleaved, in
// FP64; tiles of 64 rows staged in shared memory, each thread owning 32*kp/256 outputs.
template <typename T>
__global__ void __launch_bounds__(256) coarse_tn_kernel(int64_t m, const T* __restrict__ A, const T* __restrict__ B,
                                                        int kp, double* __restrict__ part) {
    constexpr int R = kCoarseTileRows;
    __shared__ T As[R][32];
    __shared__ T Bs[R][32];
    double acc[4] = {0.0, 0.0, 0.0, 0.0};
    const int nout = 32 * kp;
    const int64_t ntiles = (m + R - 1) / R;
    for (int64_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const int64_t r0 = tile * R;
        const int nr = (int)min((int64_t)R, m - r0);
        __syncthreads();
        for (int i = threadIdx.x; i < R * 32; i += blockDim.x) {
            const int r = i >> 5, j = i & 31;
            As[r][j] = r < nr ? A[(size_t)(r0 + r) * 32 + j] : T(0);
        }
        for (int i = threadIdx.x; i < R * kp; i += blockDim.x) {
            const int r = i / kp, c = i % kp;
            Bs[r][c] = r < nr ? B[(size_t)(r0 + r) * kp + c] : T(0);
        }
        __syncthreads();
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int o = threadIdx.x + q * 256;
            if (o < nout) {
                const int j = o / kp, c = o % kp;
                double s = 0.0;
#pragma unroll 8
                for (int r = 0; r < R; ++r) s += (double)As[r][j] * (double)Bs[r][c];
                acc[q] += s;
            }
        }
    }
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const int o = threadIdx.x + q * 256;
        if (o < nout) part[(size_t)blockIdx.x * nout + o] = acc[q];
    }
}

// One block of 1024 threads: c = the sum of the partials (each output summed by
// 1024/(32 kp) threads over strided subsets, eight loads in flight, then combined in a
// fixed order: deterministic); u = E^+ c (32 x kp).
constexpr int kCoarseSolveThreads = 1024;
__global__ void __launch_bounds__(kCoarseSolveThreads) coarse_solve_kernel(const double* __restrict__ part, int nb,
                                                                           const double* __restrict__ Einv, int kp,
                                                                           double* __restrict__ u) {
    __shared__ double c[32 * 32];
    __shared__ double sub[kCoarseSolveThreads];
    const int nout = 32 * kp;
    const int J = blockDim.x / nout;  // threads per output (>= 1)
    {
        const int i = threadIdx.x % nout, j = threadIdx.x / nout;
        double a[8] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
        if (j < J) {
            int b = j;
            for (; b + 7 * J < nb; b += 8 * J) {
#pragma unroll
                for (int q = 0; q < 8; ++q) a[q] += part[(size_t)(b + q * J) * nout + i];
            }
            for (; b < nb; b += J) a[0] += part[(size_t)b * nout + i];
        }
        sub[threadIdx.x] = ((a[0] + a[1]) + (a[2] + a[3])) + ((a[4] + a[5]) + (a[6] + a[7]));
    }
    __syncthreads();
    for (int i = threadIdx.x; i < nout; i += blockDim.x) {
        double s = 0.0;
        for (int j = 0; j < J; ++j) s += sub[j * nout + i];
        c[i] = s;
    }
    __syncthreads();
    for (int i = threadIdx.x; i < 32 * kp; i += blockDim.x) {
        const int j = i / kp, col = i % kp;
        double s = 0.0;
        for (int a = 0; a < 32; ++a) s += Einv[j * 32 + a] * c[a * kp + col];
        u[i] = s;
    }
}

// out = x + alpha * A (ua - ub), A: m x 32, ua/ub: 32 x kp (ub may be null); one thread
// per (row, 4 RHS), the row of A shared through L1 by the row's kp/4 threads.
template <typename T>
__global__ void __launch_bounds__(256) coarse_axpy_kernel(int64_t m, const T* __restrict__ A,
                                                          const double* __restrict__ ua,
                                                          const double* __restrict__ ub, double alpha, int kp,
                                                          const T* __restrict__ x, T* __restrict__ out) {
    __shared__ float us[32 * 32];
    for (int i = threadIdx.x; i < 32 * kp; i += blockDim.x) us[i] = (float)(alpha * (ua[i] - (ub ? ub[i] : 0.0)));
    __shared__ double ud[32 * 32];
    for (int i = threadIdx.x; i < 32 * kp; i += blockDim.x) ud[i] = alpha * (ua[i] - (ub ? ub[i] : 0.0));
    __syncthreads();
    const int g = kp / 4;
    const int64_t total = m * g;
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t row = t / g;
        const int c4 = (int)(t % g) * 4;
        const T* ar = A + (size_t)row * 32;
        V4<T> s(T(0));
#pragma unroll 8
        for (int j = 0; j < 32; ++j) {
            const T a = ar[j];
            if (sizeof(T) == 4) {
                const float* uj = us + j * kp + c4;
                s.a += a * (T)uj[0]; s.b += a * (T)uj[1]; s.c += a * (T)uj[2]; s.d += a * (T)uj[3];
            } else {
                const double* uj = ud + j * kp + c4;
                s.a += a * (T)uj[0]; s.b += a * (T)uj[1]; s.c += a * (T)uj[2]; s.d += a * (T)uj[3];
            }
        }
        st4(out + (size_t)row * kp + c4, ld4(x + (size_t)row * kp + c4) + s);
    }
}

}  // namespace wb
