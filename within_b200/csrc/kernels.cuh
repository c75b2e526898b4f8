// sm_100a kernels of the solve phase.  All vectors with k right-hand sides are
// stored RHS-interleaved: element (row, c) at row*k + c, so one row of a
// gather or scatter is k contiguous values (128 bytes for k = 16 in FP64).
// A "group" of G = pow2ceil(k) <= 32 lanes works on one row; lane c owns RHS c.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace wb {

constexpr int kMaxQ = 16;
constexpr int kBlock = 256;

// ---------------------------------------------------------------------------
// small device helpers
// ---------------------------------------------------------------------------

template <int G>
__device__ __forceinline__ unsigned group_mask() {
    if constexpr (G == 32) {
        return 0xffffffffu;
    } else {
        const unsigned lane = threadIdx.x & 31u;
        return ((1u << G) - 1u) << (lane & ~(unsigned)(G - 1));
    }
}

template <typename T>
__device__ __forceinline__ void atomic_add(T* p, T v) { atomicAdd(p, v); }

// ---------------------------------------------------------------------------
// Observation pass: y = D'W(D x) and its relatives, one read of the codes.
// ---------------------------------------------------------------------------

enum ObsMode { OBS_GRAM = 0, OBS_RHS = 1, OBS_RESID = 2, OBS_DX = 3 };

// Work unit of the observation pass: a run of observations (sorted by the primary
// factor) covering primary levels [lvl_begin, lvl_end).  A split chunk holds a piece
// of one long level and adds its partial sum atomically.
struct ObsChunk {
    uint32_t obs_begin, obs_end, lvl_begin, lvl_end;
    uint32_t split;
};

struct ObsParams {
    int64_t n;
    int32_t Q, k, primary;
    int32_t smem_elems;
    const uint32_t* codes;  // Q x n, primary-sorted order
    int64_t off[kMaxQ];
    // Per non-primary factor, a block-local shared-memory region of smem_len[q] values at
    // smem_base[q] (-1: none).  full[q]: the region holds every level (level*k + c);
    // otherwise it holds the factor's hottest levels: hot_slot[q][level] >= 0 gives the
    // slot, hot_level[q][slot] the level.  Other levels go to global atomics.
    int32_t smem_base[kMaxQ];
    int32_t smem_len[kMaxQ];
    int32_t full[kMaxQ];
    const int32_t* hot_slot[kMaxQ];
    const uint32_t* hot_level[kMaxQ];
    const ObsChunk* chunks;
    int64_t nchunks;
};

template <typename T>
__device__ __forceinline__ void obs_flush(const ObsParams& P, T* sm, T* out, int q, uint32_t lvl, T a, int k, int c) {
    if (a == T(0)) return;
    if (P.smem_base[q] >= 0) {
        if (P.full[q]) {
            atomic_add(sm + P.smem_base[q] + (size_t)lvl * k + c, a);
            return;
        }
        const int32_t h = __ldg(P.hot_slot[q] + lvl);
        if (h >= 0) {
            atomic_add(sm + P.smem_base[q] + (size_t)h * k + c, a);
            return;
        }
    }
    atomic_add(out + (size_t)(P.off[q] + lvl) * k + c, a);
}

// QT >= Q is the compile-time bound of the factor loops (4 or 16).
// Each group walks a chunk of observations sorted by the primary factor: the primary
// factor's sums close with a plain store when its level changes; every other factor
// keeps a running sum while its level repeats (a worker's firm rarely changes) and
// flushes it to shared memory (small factor or hot level) or a global atomic.
template <typename T, int G, int MODE, int QT>
__global__ void __launch_bounds__(kBlock) obs_pass_kernel(ObsParams P, const T* __restrict__ w,
                                                          const T* __restrict__ x, const T* __restrict__ yin,
                                                          T* __restrict__ out, T* __restrict__ eout) {
    extern __shared__ unsigned char smem_raw[];
    T* sm = reinterpret_cast<T*>(smem_raw);
    constexpr bool kScatter = MODE != OBS_DX;
    if (kScatter) {
        for (int i = threadIdx.x; i < P.smem_elems; i += blockDim.x) sm[i] = T(0);
        __syncthreads();
    }
    const int lane_g = threadIdx.x & (G - 1);
    const int c = lane_g;
    const bool cval = c < P.k;
    const int k = P.k;
    const unsigned mask = group_mask<G>();
    const int64_t groups_per_block = blockDim.x / G;
    const int64_t gid = (int64_t)blockIdx.x * groups_per_block + threadIdx.x / G;
    const int64_t ngroups = (int64_t)gridDim.x * groups_per_block;
    const int Q = P.Q, pq = P.primary;
    const int64_t n = P.n;

    for (int64_t ch = gid; ch < P.nchunks; ch += ngroups) {
        const ObsChunk C = P.chunks[ch];
        uint32_t lvl = C.lvl_begin;
        T acc = T(0);
        uint32_t run_l[QT];
        T run_a[QT];
#pragma unroll
        for (int q = 0; q < QT; ++q) { run_l[q] = 0xffffffffu; run_a[q] = T(0); }
        for (uint32_t base = C.obs_begin; base < C.obs_end; base += G) {
            const uint32_t cnt = min((uint32_t)G, C.obs_end - base);
            // cooperative loads: lane j holds the codes and weight of observation base+j
            uint32_t my_codes[QT];
            const uint32_t j = base + (lane_g < (int)cnt ? lane_g : 0);
#pragma unroll
            for (int q = 0; q < QT; ++q)
                my_codes[q] = q < Q ? __ldg(P.codes + (size_t)q * n + j) : 0u;
            T my_w = (MODE == OBS_DX || w == nullptr) ? T(1) : __ldg(w + j);
            for (uint32_t jj = 0; jj < cnt; ++jj) {
                const uint32_t i = base + jj;
                uint32_t lq[QT];
#pragma unroll
                for (int q = 0; q < QT; ++q) lq[q] = __shfl_sync(mask, my_codes[q], jj, G);
                const T wi = __shfl_sync(mask, my_w, jj, G);
                T t = T(0);
                if (cval) {
                    T s = T(0);
                    if (MODE != OBS_RHS) {
#pragma unroll
                        for (int q = 0; q < QT; ++q)
                            if (q < Q) s += __ldg(x + (size_t)(P.off[q] + lq[q]) * k + c);
                    }
                    if (MODE == OBS_GRAM) {
                        t = wi * s;
                    } else if (MODE == OBS_RHS) {
                        t = wi * yin[(size_t)i * k + c];
                    } else if (MODE == OBS_RESID) {
                        const T e = yin[(size_t)i * k + c] - s;
                        eout[(size_t)i * k + c] = e;
                        t = wi * e;
                    } else {
                        eout[(size_t)i * k + c] = s;
                    }
                }
                if (kScatter) {
                    const uint32_t p = lq[pq];
                    while (lvl < p) {  // primary level complete: plain store (zero for empty levels)
                        if (cval) out[(size_t)(P.off[pq] + lvl) * k + c] = acc;
                        acc = T(0);
                        ++lvl;
                    }
                    acc += t;
#pragma unroll
                    for (int q = 0; q < QT; ++q) {
                        if (q >= Q || q == pq) continue;
                        if (lq[q] == run_l[q]) {
                            run_a[q] += t;
                        } else {
                            if (run_l[q] != 0xffffffffu && cval) obs_flush(P, sm, out, q, run_l[q], run_a[q], k, c);
                            run_l[q] = lq[q];
                            run_a[q] = t;
                        }
                    }
                }
            }
        }
        if (kScatter && cval) {
#pragma unroll
            for (int q = 0; q < QT; ++q)
                if (q < Q && q != pq && run_l[q] != 0xffffffffu) obs_flush(P, sm, out, q, run_l[q], run_a[q], k, c);
            if (C.split) {
                atomic_add(out + (size_t)(P.off[pq] + C.lvl_begin) * k + c, acc);
            } else {
                while (lvl < C.lvl_end) {
                    out[(size_t)(P.off[pq] + lvl) * k + c] = acc;
                    acc = T(0);
                    ++lvl;
                }
            }
        }
    }
    if (kScatter && P.smem_elems > 0) {
        __syncthreads();
        // the block's partial sums of each shared-memory region, one atomic per nonzero entry
        for (int q = 0; q < Q; ++q) {
            if (P.smem_base[q] < 0) continue;
            for (int idx = threadIdx.x; idx < P.smem_len[q]; idx += blockDim.x) {
                const T v = sm[P.smem_base[q] + idx];
                if (v == T(0)) continue;
                const int slot = idx / k, cc = idx % k;
                const uint32_t lev = P.full[q] ? (uint32_t)slot : P.hot_level[q][slot];
                atomic_add(out + (size_t)(P.off[q] + lev) * k + cc, v);
            }
        }
    }
}

// Column-major (RHS-major) original order <-> interleaved primary-sorted order.
// perm[i] = original index of sorted observation i (nullptr = identity).
template <typename T>
__global__ void gather_interleave_kernel(const double* __restrict__ ycol, int64_t n, int k,
                                         const uint32_t* __restrict__ perm, T* __restrict__ yi) {
    __shared__ double tile[32][33];
    const int64_t i0 = (int64_t)blockIdx.x * 32;
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;  // 32 x 8
    for (int c0 = 0; c0 < k; c0 += 32) {
        for (int cc = ty; cc < 32; cc += 8) {
            const int c = c0 + cc;
            const int64_t i = i0 + tx;
            double v = 0.0;
            if (c < k && i < n) v = ycol[(size_t)c * n + (perm ? perm[i] : i)];
            tile[cc][tx] = v;
        }
        __syncthreads();
        const int cw = min(32, k - c0);
        for (int e = threadIdx.x; e < 32 * cw; e += blockDim.x) {
            const int r = e / cw, cc = e % cw;
            const int64_t i = i0 + r;
            if (i < n) yi[(size_t)i * k + c0 + cc] = (T)tile[cc][r];
        }
        __syncthreads();
    }
}

template <typename T>
__global__ void scatter_deinterleave_kernel(const T* __restrict__ ei, int64_t n, int k,
                                            const uint32_t* __restrict__ perm, double* __restrict__ ecol) {
    __shared__ double tile[32][33];
    const int64_t i0 = (int64_t)blockIdx.x * 32;
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
    for (int c0 = 0; c0 < k; c0 += 32) {
        const int cw = min(32, k - c0);
        for (int e = threadIdx.x; e < 32 * cw; e += blockDim.x) {
            const int r = e / cw, cc = e % cw;
            const int64_t i = i0 + r;
            tile[cc][r] = (i < n) ? (double)ei[(size_t)i * k + c0 + cc] : 0.0;
        }
        __syncthreads();
        for (int cc = ty; cc < 32; cc += 8) {
            const int c = c0 + cc;
            const int64_t i = i0 + tx;
            if (c < k && i < n) ecol[(size_t)c * n + (perm ? perm[i] : i)] = tile[cc][tx];
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// Row-wise vector kernels over (rows x k) interleaved vectors; dots in FP64.
// ---------------------------------------------------------------------------

// Each block reduces its share into part[blockIdx.x * k + c] (fixed order: deterministic).
template <int G>
__device__ __forceinline__ void block_reduce_store(double v, int k, double* part) {
    __shared__ double red[kBlock];
    red[threadIdx.x] = v;
    __syncthreads();
    for (int s = blockDim.x / 2; s >= G; s >>= 1) {
        if (threadIdx.x < s) red[threadIdx.x] += red[threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x < G && threadIdx.x < k) part[(size_t)blockIdx.x * k + threadIdx.x] = red[threadIdx.x];
}

template <typename TA, typename TB, int G>
__global__ void __launch_bounds__(kBlock) dot_kernel(const TA* __restrict__ a, const TB* __restrict__ b,
                                                     int64_t rows, int k, double* __restrict__ part) {
    const int c = threadIdx.x & (G - 1);
    double s = 0.0;
    if (c < k) {
        const int64_t rpb = blockDim.x / G;
        for (int64_t r = (int64_t)blockIdx.x * rpb + threadIdx.x / G; r < rows; r += (int64_t)gridDim.x * rpb)
            s += (double)a[(size_t)r * k + c] * (double)b[(size_t)r * k + c];
    }
    block_reduce_store<G>(s, k, part);
}

// CG step 4 (cg.rs:87-94): x += alpha p, r -= alpha ap, partial ||r||^2.
template <typename T, int G>
__global__ void __launch_bounds__(kBlock) cg_xr_kernel(T* __restrict__ x, T* __restrict__ r,
                                                       const T* __restrict__ p, const T* __restrict__ ap,
                                                       const double* __restrict__ alpha, int64_t rows, int k,
                                                       double* __restrict__ part) {
    const int c = threadIdx.x & (G - 1);
    double s = 0.0;
    if (c < k) {
        const T al = (T)alpha[c];
        const int64_t rpb = blockDim.x / G;
        for (int64_t row = (int64_t)blockIdx.x * rpb + threadIdx.x / G; row < rows; row += (int64_t)gridDim.x * rpb) {
            const size_t e = (size_t)row * k + c;
            x[e] += al * p[e];
            const T rv = r[e] - al * ap[e];
            r[e] = rv;
            s += (double)rv * (double)rv;
        }
    }
    block_reduce_store<G>(s, k, part);
}

// p = z + beta p (cg.rs:120-124); columns with active == 0 are left alone.
template <typename T, int G>
__global__ void __launch_bounds__(kBlock) cg_p_kernel(T* __restrict__ p, const T* __restrict__ z,
                                                      const double* __restrict__ beta,
                                                      const int32_t* __restrict__ active, int64_t rows, int k) {
    const int c = threadIdx.x & (G - 1);
    if (c >= k || !active[c]) return;
    const T be = (T)beta[c];
    const int64_t rpb = blockDim.x / G;
    for (int64_t row = (int64_t)blockIdx.x * rpb + threadIdx.x / G; row < rows; row += (int64_t)gridDim.x * rpb) {
        const size_t e = (size_t)row * k + c;
        p[e] = z[e] + be * p[e];
    }
}

// ---------------------------------------------------------------------------
// Schwarz local solves over the flattened slots of all subdomains of a stage.
// ---------------------------------------------------------------------------

// Work unit of a row-wise CSR pass: rows [row_begin, row_end) restricted to the
// entries [nz_begin, nz_end); rows cut by the range are partial and add atomically.
struct CsrChunk {
    uint32_t row_begin, row_end;
    int64_t nz_begin, nz_end;
};

enum CsrEpi { EPI_ACC = 0, EPI_ACC_SCALED = 1, EPI_PIVOT = 2 };

// out[row_slot] (+)= [scale] * sum_e val[e] * v[col[e]]  per RHS.
//   EPI_ACC:        v[row] += acc
//   EPI_ACC_SCALED: v[row] += rscale[row] * acc     (back substitution, rscale = 1/D_elim)
//   EPI_PIVOT:      v[row]  = v[row] * rscale[row] + acc   (backward AC sweep, rscale = 1/d)
template <typename T, int G, int EPI>
__global__ void __launch_bounds__(kBlock) csr_rows_kernel(const CsrChunk* __restrict__ chunks, int64_t nchunks,
                                                          const uint32_t* __restrict__ row_slot,
                                                          const int64_t* __restrict__ ptr,
                                                          const uint32_t* __restrict__ col,
                                                          const T* __restrict__ val,
                                                          const T* __restrict__ rscale, T* __restrict__ v, int k) {
    const int c = threadIdx.x & (G - 1);
    const bool cval = c < k;
    const int64_t gpb = blockDim.x / G;
    const int64_t ng = (int64_t)gridDim.x * gpb;
    for (int64_t ch = (int64_t)blockIdx.x * gpb + threadIdx.x / G; ch < nchunks; ch += ng) {
        const CsrChunk C = chunks[ch];
        for (uint32_t row = C.row_begin; row < C.row_end; ++row) {
            const int64_t rb = ptr[row], re = ptr[row + 1];
            const int64_t e0 = max(rb, C.nz_begin), e1 = min(re, C.nz_end);
            T acc = T(0);
            if (cval)
                for (int64_t e = e0; e < e1; ++e) acc += __ldg(val + e) * v[(size_t)__ldg(col + e) * k + c];
            if (!cval) continue;
            const uint32_t s = row_slot[row];
            T* dst = v + (size_t)s * k + c;
            const bool partial = (e0 != rb) || (e1 != re);
            if (EPI == EPI_ACC) {
                if (partial) atomic_add(dst, acc); else *dst += acc;
            } else if (EPI == EPI_ACC_SCALED) {
                const T sc = rscale[row];
                if (partial) atomic_add(dst, sc * acc); else *dst += sc * acc;
            } else {
                *dst = *dst * rscale[row] + acc;  // rows of the backward sweep are never split
            }
        }
    }
}

// Segmented sums over a list of slots (slot_list == nullptr: slots [0, nslots)) into
// msum[sub_of[slot] * k + c]; one atomic per (run of equal subdomain, RHS).
template <typename T, int G>
__global__ void __launch_bounds__(kBlock) slot_sum_kernel(const uint32_t* __restrict__ slot_list, int64_t nslots,
                                                          const uint32_t* __restrict__ sub_of,
                                                          const T* __restrict__ v, int k, double* __restrict__ msum,
                                                          int64_t chunk) {
    const int c = threadIdx.x & (G - 1);
    if (c >= k) return;
    const int64_t gpb = blockDim.x / G;
    const int64_t ng = (int64_t)gridDim.x * gpb;
    for (int64_t g = (int64_t)blockIdx.x * gpb + threadIdx.x / G; g * chunk < nslots; g += ng) {
        const int64_t a0 = g * chunk, a1 = min(nslots, a0 + chunk);
        uint32_t cur = UINT32_MAX;
        double acc = 0.0;
        for (int64_t a = a0; a < a1; ++a) {
            const uint32_t s = slot_list ? slot_list[a] : (uint32_t)a;
            const uint32_t sb = sub_of[s];
            if (sb != cur) {
                if (cur != UINT32_MAX) atomicAdd(msum + (size_t)cur * k + c, acc);
                cur = sb;
                acc = 0.0;
            }
            acc += (double)v[(size_t)s * k + c];
        }
        if (cur != UINT32_MAX) atomicAdd(msum + (size_t)cur * k + c, acc);
    }
}

// Restrict: v[l] = spou[l] * r[gidx[l]] (sign of the r-block folded into spou),
// followed by the subdomain sums of the first subtract_mean (local_solver.rs:360-367).
template <typename T, int G>
__global__ void __launch_bounds__(kBlock) restrict_kernel(int64_t nslots, const uint32_t* __restrict__ gidx,
                                                          const T* __restrict__ spou, const T* __restrict__ r,
                                                          T* __restrict__ v, int k) {
    const int c = threadIdx.x & (G - 1);
    if (c >= k) return;
    const int64_t rpb = blockDim.x / G;
    for (int64_t l = (int64_t)blockIdx.x * rpb + threadIdx.x / G; l < nslots; l += (int64_t)gridDim.x * rpb)
        v[(size_t)l * k + c] = spou[l] * r[(size_t)gidx[l] * k + c];
}

// v[l] = (v[l] - msum[s]/n_s) * scale[l]   (scale = 1/D_elim on eliminated slots, 1 on kept).
template <typename T, int G>
__global__ void __launch_bounds__(kBlock) center_scale_kernel(const uint32_t* __restrict__ slot_list, int64_t nslots,
                                                              const uint32_t* __restrict__ sub_of,
                                                              const int32_t* __restrict__ sub_n,
                                                              const double* __restrict__ msum,
                                                              const T* __restrict__ scale, T* __restrict__ v, int k) {
    const int c = threadIdx.x & (G - 1);
    if (c >= k) return;
    const int64_t rpb = blockDim.x / G;
    for (int64_t a = (int64_t)blockIdx.x * rpb + threadIdx.x / G; a < nslots; a += (int64_t)gridDim.x * rpb) {
        const uint32_t l = slot_list ? slot_list[a] : (uint32_t)a;
        const uint32_t s = sub_of[l];
        const double mean = msum[(size_t)s * k + c] / (double)sub_n[s];
        T x = (T)((double)v[(size_t)l * k + c] - mean);
        if (scale) x *= scale[l];
        v[(size_t)l * k + c] = x;
    }
}

// Anchored dense Cholesky solves (AnchoredDenseCholesky::solve_in_place,
// local_solver.rs:252-299): one warp per (dense subdomain, RHS).  For m <= 32 lane i
// keeps row i in a register; larger minors are swept in place in v.
template <typename T>
__global__ void dense_solve_kernel(int32_t ndense, const int64_t* __restrict__ keep0,
                                   const int32_t* __restrict__ nkeep, const int64_t* __restrict__ loff,
                                   const T* __restrict__ L, T* __restrict__ v, int k) {
    const int warp = (int)(((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    const int lane = threadIdx.x & 31;
    if (warp >= ndense * k) return;  // uniform per warp
    const int d = warp / k, c = warp % k;
    const int n = nkeep[d];
    const int64_t s0 = keep0[d];
    if (n == 0) return;
    if (n == 1) {
        if (lane == 0) v[(size_t)s0 * k + c] = T(0);
        return;
    }
    const int m = n - 1;
    const T* Ld = L + loff[d];
    if (m <= 32) {
        T xi = (lane < m) ? v[(size_t)(s0 + lane) * k + c] : T(0);
        for (int j = 0; j < m; ++j) {  // forward L y = b
            T xj = __shfl_sync(0xffffffffu, xi, j);
            xj = xj / Ld[(size_t)j * m + j];
            if (lane == j) xi = xj;
            if (lane > j && lane < m) xi -= Ld[(size_t)lane * m + j] * xj;
        }
        for (int j = m - 1; j >= 0; --j) {  // backward L^T x = y
            T xj = __shfl_sync(0xffffffffu, xi, j);
            xj = xj / Ld[(size_t)j * m + j];
            if (lane == j) xi = xj;
            if (lane < j) xi -= Ld[(size_t)j * m + lane] * xj;
        }
        if (lane < m) v[(size_t)(s0 + lane) * k + c] = xi;
    } else {
        T* x = v + (size_t)s0 * k + c;  // element i at x[i*k]
        for (int j = 0; j < m; ++j) {
            const T xj = x[(size_t)j * k] / Ld[(size_t)j * m + j];
            __syncwarp();
            if (lane == 0) x[(size_t)j * k] = xj;
            for (int i = j + 1 + lane; i < m; i += 32) x[(size_t)i * k] -= Ld[(size_t)i * m + j] * xj;
            __syncwarp();
        }
        for (int j = m - 1; j >= 0; --j) {
            const T xj = x[(size_t)j * k] / Ld[(size_t)j * m + j];
            __syncwarp();
            if (lane == 0) x[(size_t)j * k] = xj;
            for (int i = lane; i < j; i += 32) x[(size_t)i * k] -= Ld[(size_t)j * m + i] * xj;
            __syncwarp();
        }
    }
    if (lane == 0) v[(size_t)(s0 + m) * k + c] = T(0);
}

// Dense core of an AC factor: v[core] = Z v[core] (anchored inverse), RHS [c0, c0+kc).
// Block b of core g computes rows [row0, row0 + rows_per_block); the core input is
// staged in shared memory (c-major, conflict-free) before any output is produced, and
// outputs go to `tmp` because other blocks of the same core still read the input.
template <typename T, int KC>
__global__ void core_gemv_kernel(const int32_t* __restrict__ core_of_block, const int32_t* __restrict__ row0_of_block,
                                 const int32_t* __restrict__ core_n, const int64_t* __restrict__ core_slot_off,
                                 const uint32_t* __restrict__ core_slot, const int64_t* __restrict__ core_z_off,
                                 const T* __restrict__ Z, const T* __restrict__ v, T* __restrict__ tmp,
                                 int k, int c0, int kc, int rows_per_block) {
    extern __shared__ unsigned char smem_raw[];
    T* yc = reinterpret_cast<T*>(smem_raw);
    const int g = core_of_block[blockIdx.x];
    const int r = core_n[g];
    const uint32_t* slots = core_slot + core_slot_off[g];
    for (int e = threadIdx.x; e < r * kc; e += blockDim.x) {
        const int c = e / r, a = e % r;
        yc[e] = v[(size_t)slots[a] * k + c0 + c];
    }
    __syncthreads();
    const T* Zg = Z + core_z_off[g];
    const int row0 = row0_of_block[blockIdx.x];
    const int row1 = min(r, row0 + rows_per_block);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    for (int row = row0 + warp; row < row1; row += nw) {
        const T* zr = Zg + (size_t)row * r;
        T acc[KC];
#pragma unroll
        for (int c = 0; c < KC; ++c) acc[c] = T(0);
        for (int b = lane; b < r; b += 32) {
            const T zv = __ldg(zr + b);
#pragma unroll
            for (int c = 0; c < KC; ++c)
                if (c < kc) acc[c] += zv * yc[c * r + b];
        }
#pragma unroll
        for (int c = 0; c < KC; ++c) {
            if (c >= kc) break;
            T a = acc[c];
            for (int o = 16; o > 0; o >>= 1) a += __shfl_xor_sync(0xffffffffu, a, o);
            if (lane == 0) tmp[(size_t)(core_slot_off[g] + row) * k + c0 + c] = a;
        }
    }
}

template <typename T>
__global__ void core_writeback_kernel(int64_t total, const uint32_t* __restrict__ core_slot,
                                      const T* __restrict__ tmp, T* __restrict__ v, int k) {
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total * k; e += (int64_t)gridDim.x * blockDim.x) {
        const int64_t a = e / k;
        const int c = (int)(e % k);
        v[(size_t)core_slot[a] * k + c] = tmp[e];
    }
}

// Additive prolongation as a gather over global dofs (no atomics):
// z[j] = sum_{slots l of j} spou[l] * (v[l] - msum[s(l)]/n_s), optionally with the
// partial dot r.z for CG.  Dofs in no subdomain get z = 0.
template <typename T, int G>
__global__ void __launch_bounds__(kBlock) prolong_gather_kernel(int64_t m, const int64_t* __restrict__ gptr,
                                                                const uint32_t* __restrict__ gslot,
                                                                const uint32_t* __restrict__ sub_of,
                                                                const int32_t* __restrict__ sub_n,
                                                                const T* __restrict__ spou,
                                                                const double* __restrict__ msum,
                                                                const T* __restrict__ v, T* __restrict__ z,
                                                                const T* __restrict__ rdot, int k,
                                                                double* __restrict__ part) {
    const int c = threadIdx.x & (G - 1);
    double s = 0.0;
    if (c < k) {
        const int64_t rpb = blockDim.x / G;
        for (int64_t j = (int64_t)blockIdx.x * rpb + threadIdx.x / G; j < m; j += (int64_t)gridDim.x * rpb) {
            double acc = 0.0;
            for (int64_t e = gptr[j]; e < gptr[j + 1]; ++e) {
                const uint32_t l = gslot[e];
                const uint32_t sb = sub_of[l];
                const double mean = msum[(size_t)sb * k + c] / (double)sub_n[sb];
                acc += (double)spou[l] * ((double)v[(size_t)l * k + c] - mean);
            }
            const T zv = (T)acc;
            z[(size_t)j * k + c] = zv;
            if (rdot) s += (double)rdot[(size_t)j * k + c] * (double)zv;
        }
    }
    if (part) block_reduce_store<G>(s, k, part);
}

// Multiplicative stage: z[gidx[l]] += c_l and r_work -= G[:, gidx[l]] * c_l with
// c_l = spou[l] * (v[l] - mean) (multiplicative.rs:128-168, residual_update.rs:36-53).
template <typename T, int G>
__global__ void __launch_bounds__(kBlock) mult_update_kernel(int64_t nslots, const uint32_t* __restrict__ gidx,
                                                             const uint32_t* __restrict__ sub_of,
                                                             const int32_t* __restrict__ sub_n,
                                                             const T* __restrict__ spou,
                                                             const double* __restrict__ msum,
                                                             const T* __restrict__ v, T* __restrict__ z,
                                                             const int64_t* __restrict__ gram_ptr,
                                                             const uint32_t* __restrict__ gram_col,
                                                             const T* __restrict__ gram_val,
                                                             T* __restrict__ rwork, int k) {
    const int c = threadIdx.x & (G - 1);
    if (c >= k) return;
    const int64_t rpb = blockDim.x / G;
    for (int64_t l = (int64_t)blockIdx.x * rpb + threadIdx.x / G; l < nslots; l += (int64_t)gridDim.x * rpb) {
        const uint32_t sb = sub_of[l];
        const double mean = msum[(size_t)sb * k + c] / (double)sub_n[sb];
        const T cl = (T)((double)spou[l] * ((double)v[(size_t)l * k + c] - mean));
        const uint32_t g = gidx[l];
        z[(size_t)g * k + c] += cl;  // dofs are unique within one stage
        if (cl == T(0)) continue;
        for (int64_t e = gram_ptr[g]; e < gram_ptr[g + 1]; ++e)
            atomic_add(rwork + (size_t)gram_col[e] * k + c, -cl * gram_val[e]);
    }
}

}  // namespace wb
