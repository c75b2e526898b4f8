// Cross-tabulation of one factor pair on the device (the heavy part of
// gramian/cross_tab.rs:514-664 in the reference): for every observation the key
// (compact q level, compact r level), a stable LSD radix sort of the keys carrying the
// observation indices, and a segmented sum of the weights over equal keys in observation
// order.  The sums are therefore the same floating-point sums, in the same order, as the
// host's sequential build, and the (row, column) structure comes out row-major with
// ascending columns: the host assembles the CSR from them bit-identically.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <vector>

#include "setup.hpp"

namespace wb {
namespace {

constexpr int kSortTile = 4096;      // keys per block of the radix passes
constexpr int kSortThreads = 256;    // 16 rounds of 256 keys per tile
constexpr int kScanThreads = 1024;

__global__ void ct_keys_kernel(int64_t n, const uint32_t* __restrict__ cq, const uint32_t* __restrict__ cr,
                               const uint32_t* __restrict__ qmap, const uint32_t* __restrict__ rmap, uint64_t nr,
                               uint64_t* __restrict__ keys, uint32_t* __restrict__ idx) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    keys[i] = (uint64_t)qmap[cq[i]] * nr + (uint64_t)rmap[cr[i]];
    idx[i] = (uint32_t)i;
}

// Digit counts of each tile: hist[digit * nblocks + block].
__global__ void __launch_bounds__(kSortThreads) radix_hist_kernel(const uint64_t* __restrict__ keys, int64_t n,
                                                                  int shift, uint32_t* __restrict__ hist, int nblocks) {
    __shared__ uint32_t h[256];
    h[threadIdx.x] = 0;
    __syncthreads();
    const int64_t t0 = (int64_t)blockIdx.x * kSortTile, t1 = min(n, t0 + kSortTile);
    for (int64_t i = t0 + threadIdx.x; i < t1; i += blockDim.x) atomicAdd(&h[(keys[i] >> shift) & 255u], 1u);
    __syncthreads();
    hist[(size_t)threadIdx.x * nblocks + blockIdx.x] = h[threadIdx.x];
}

// Stable scatter of one tile: keys go in index order, 256 per round; within a round a
// key's position is its digit's running base, plus the keys of that digit in earlier
// warps of the round, plus its rank among equal digits of its own warp.
__global__ void __launch_bounds__(kSortThreads) radix_scatter_kernel(const uint64_t* __restrict__ kin,
                                                                     const uint32_t* __restrict__ iin, int64_t n,
                                                                     int shift, const uint32_t* __restrict__ offs,
                                                                     int nblocks, uint64_t* __restrict__ kout,
                                                                     uint32_t* __restrict__ iout) {
    constexpr int W = kSortThreads / 32;
    __shared__ uint32_t base[256];
    __shared__ uint32_t wcnt[W][256];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    base[threadIdx.x] = offs[(size_t)threadIdx.x * nblocks + blockIdx.x];
    const int64_t t0 = (int64_t)blockIdx.x * kSortTile, t1 = min(n, t0 + kSortTile);
    for (int64_t r0 = t0; r0 < t1; r0 += kSortThreads) {
        for (int w = 0; w < W; ++w) wcnt[w][threadIdx.x] = 0;
        const int64_t i = r0 + threadIdx.x;
        const bool valid = i < t1;
        uint64_t key = 0;
        uint32_t id = 0;
        unsigned digit = 256;  // invalid lanes match only each other
        if (valid) {
            key = kin[i];
            id = iin[i];
            digit = (unsigned)((key >> shift) & 255u);
        }
        __syncthreads();
        const unsigned peers = __match_any_sync(0xffffffffu, digit);
        const unsigned rank = __popc(peers & ((1u << lane) - 1u));
        if (valid && rank == 0) wcnt[warp][digit] = __popc(peers);
        __syncthreads();
        if (valid) {
            uint32_t pos = base[digit] + rank;
            for (int w = 0; w < warp; ++w) pos += wcnt[w][digit];
            kout[pos] = key;
            iout[pos] = id;
        }
        __syncthreads();
        uint32_t add = 0;
        for (int w = 0; w < W; ++w) add += wcnt[w][threadIdx.x];
        base[threadIdx.x] += add;
        __syncthreads();
    }
}

// Exclusive scan of a[0..len) in place, one block of 1024 threads (len < 2^32 in total).
__global__ void __launch_bounds__(kScanThreads) scan_block_kernel(uint32_t* __restrict__ a, int64_t len) {
    __shared__ uint32_t part[kScanThreads];
    const int64_t per = (len + kScanThreads - 1) / kScanThreads;
    const int64_t b0 = threadIdx.x * per, b1 = min(len, b0 + per);
    uint32_t s = 0;
    for (int64_t i = b0; i < b1; ++i) s += a[i];
    part[threadIdx.x] = s;
    __syncthreads();
    for (int off = 1; off < kScanThreads; off <<= 1) {  // inclusive Hillis-Steele over the partials
        const uint32_t v = threadIdx.x >= off ? part[threadIdx.x - off] : 0u;
        __syncthreads();
        part[threadIdx.x] += v;
        __syncthreads();
    }
    uint32_t run = threadIdx.x ? part[threadIdx.x - 1] : 0u;
    for (int64_t i = b0; i < b1; ++i) {
        const uint32_t v = a[i];
        a[i] = run;
        run += v;
    }
}

// Per tile of 4096: exclusive scan of the tile in place, its total into tot[block].
__global__ void __launch_bounds__(kSortThreads) scan_tile_kernel(uint32_t* __restrict__ a, int64_t n,
                                                                 uint32_t* __restrict__ tot) {
    __shared__ uint32_t part[kSortThreads];
    const int64_t t0 = (int64_t)blockIdx.x * kSortTile, t1 = min(n, t0 + kSortTile);
    constexpr int per = kSortTile / kSortThreads;
    const int64_t b0 = t0 + (int64_t)threadIdx.x * per, b1 = min(t1, b0 + per);
    uint32_t s = 0;
    for (int64_t i = b0; i < b1; ++i) s += a[i];
    part[threadIdx.x] = s;
    __syncthreads();
    for (int off = 1; off < kSortThreads; off <<= 1) {
        const uint32_t v = threadIdx.x >= off ? part[threadIdx.x - off] : 0u;
        __syncthreads();
        part[threadIdx.x] += v;
        __syncthreads();
    }
    uint32_t run = threadIdx.x ? part[threadIdx.x - 1] : 0u;
    for (int64_t i = b0; i < b1; ++i) {
        const uint32_t v = a[i];
        a[i] = run;
        run += v;
    }
    if (threadIdx.x == kSortThreads - 1) tot[blockIdx.x] = part[threadIdx.x];
}

__global__ void scan_add_kernel(uint32_t* __restrict__ a, int64_t n, const uint32_t* __restrict__ tot) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) a[i] += tot[i / kSortTile];
}

__global__ void seg_head_kernel(const uint64_t* __restrict__ keys, int64_t n, uint32_t* __restrict__ flag) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) flag[i] = (i == 0 || keys[i] != keys[i - 1]) ? 1u : 0u;
}

// start[s] = first position of segment s (pos = exclusive scan of the head flags).
__global__ void seg_start_kernel(const uint64_t* __restrict__ keys, int64_t n, const uint32_t* __restrict__ pos,
                                 uint32_t* __restrict__ start) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n && (i == 0 || keys[i] != keys[i - 1])) start[pos[i]] = (uint32_t)i;
}

// ws[e] = w[idx[e]]: the weights in sorted order, contiguous.
__global__ void gather_weights_kernel(int64_t n, const uint32_t* __restrict__ idx, const double* __restrict__ w,
                                      double* __restrict__ ws) {
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e < n) ws[e] = w[idx[e]];
}

// One thread per segment: the key and the sum of its weights in sorted (= observation)
// order; ws null = unit weights.
__global__ void seg_sum_kernel(const uint64_t* __restrict__ keys, const double* __restrict__ ws,
                               const uint32_t* __restrict__ start, int64_t nseg, int64_t n,
                               uint64_t* __restrict__ skey, double* __restrict__ ssum) {
    const int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= nseg) return;
    const int64_t a = start[s], b = s + 1 < nseg ? (int64_t)start[s + 1] : n;
    double sum = 0.0;
    int64_t e = a;
    if (ws) {  // sixteen loads in flight, the additions still one after another in order
        for (; e + 16 <= b; e += 16) {
            double v[16];
#pragma unroll
            for (int u = 0; u < 16; ++u) v[u] = ws[e + u];
#pragma unroll
            for (int u = 0; u < 16; ++u) sum += v[u];
        }
        for (; e < b; ++e) sum += ws[e];
    } else {
        sum = (double)(b - a);  // unit weights: an exact count
    }
    skey[s] = keys[a];
    ssum[s] = sum;
}

int blocks_for(int64_t n, int t) { return (int)std::max<int64_t>(1, (n + t - 1) / t); }

// Exclusive scan of a[0..n) in place (tiles, then the tile totals, then the offsets).
bool scan_u32(uint32_t* a, int64_t n, uint32_t* tot, cudaStream_t st) {
    const int nb = blocks_for(n, kSortTile);
    scan_tile_kernel<<<nb, kSortThreads, 0, st>>>(a, n, tot);
    scan_block_kernel<<<1, kScanThreads, 0, st>>>(tot, nb);
    scan_add_kernel<<<blocks_for(n, 256), 256, 0, st>>>(a, n, tot);
    return cudaGetLastError() == cudaSuccess;
}

// Stream-ordered device buffer (cudaMallocAsync / cudaFreeAsync): no device-wide
// synchronisation with the other setup threads' work.
template <typename T>
struct Buf {
    T* p = nullptr;
    cudaStream_t st = nullptr;
    ~Buf() {
        if (p) cudaFreeAsync(p, st);
    }
    bool alloc(size_t n, cudaStream_t s) {
        st = s;
        return cudaMallocAsync((void**)&p, std::max<size_t>(n, 1) * sizeof(T), s) == cudaSuccess;
    }
};

}  // namespace

bool device_pair_sums(int device, int64_t n, const uint32_t* cq, const uint32_t* cr, const double* w,
                      const std::vector<uint32_t>& qmap, const std::vector<uint32_t>& rmap, uint32_t nq, uint32_t nr,
                      std::vector<uint64_t>& seg_key, std::vector<double>& seg_sum) {
    if (n <= 0 || n >= ((int64_t)1 << 32) || device < 0) return false;
    if (cudaSetDevice(device) != cudaSuccess) return false;
    cudaStream_t st = nullptr;
    if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess) return false;
    bool ok = true;
    {
        Buf<uint32_t> dcq, dcr, dqm, drm, i0, i1, hist, flag, start, tot;
        Buf<uint64_t> k0, k1, skey;
        Buf<double> dw, dws, ssum;
        const int nb = blocks_for(n, kSortTile);
        ok = dcq.alloc(n, st) && dcr.alloc(n, st) && dqm.alloc(qmap.size(), st) && drm.alloc(rmap.size(), st) &&
             i0.alloc(n, st) && i1.alloc(n, st) && k0.alloc(n, st) && k1.alloc(n, st) &&
             hist.alloc((size_t)256 * nb, st) && flag.alloc(n, st) && start.alloc(n, st) &&
             tot.alloc(blocks_for(std::max<int64_t>(n, (int64_t)256 * nb), kSortTile) + 1, st) &&
             (!w || (dw.alloc(n, st) && dws.alloc(n, st)));
        ok = ok && cudaMemcpyAsync(dcq.p, cq, sizeof(uint32_t) * n, cudaMemcpyHostToDevice, st) == cudaSuccess &&
             cudaMemcpyAsync(dcr.p, cr, sizeof(uint32_t) * n, cudaMemcpyHostToDevice, st) == cudaSuccess &&
             cudaMemcpyAsync(dqm.p, qmap.data(), sizeof(uint32_t) * qmap.size(), cudaMemcpyHostToDevice, st) ==
                 cudaSuccess &&
             cudaMemcpyAsync(drm.p, rmap.data(), sizeof(uint32_t) * rmap.size(), cudaMemcpyHostToDevice, st) ==
                 cudaSuccess &&
             (!w || cudaMemcpyAsync(dw.p, w, sizeof(double) * n, cudaMemcpyHostToDevice, st) == cudaSuccess);
        if (ok) {
            ct_keys_kernel<<<blocks_for(n, 256), 256, 0, st>>>(n, dcq.p, dcr.p, dqm.p, drm.p, nr, k0.p, i0.p);
            // radix passes over the key bits (8 per pass), ping-ponging the buffers
            const uint64_t kmax = (uint64_t)nq * nr;
            int bits = 1;
            while (bits < 64 && (kmax >> bits) != 0) ++bits;
            uint64_t *kin = k0.p, *kout = k1.p;
            uint32_t *iin = i0.p, *iout = i1.p;
            for (int shift = 0; shift < bits && ok; shift += 8) {
                radix_hist_kernel<<<nb, kSortThreads, 0, st>>>(kin, n, shift, hist.p, nb);
                ok = scan_u32(hist.p, (int64_t)256 * nb, tot.p, st);
                radix_scatter_kernel<<<nb, kSortThreads, 0, st>>>(kin, iin, n, shift, hist.p, nb, kout, iout);
                ok = cudaGetLastError() == cudaSuccess;
                std::swap(kin, kout);
                std::swap(iin, iout);
            }
            seg_head_kernel<<<blocks_for(n, 256), 256, 0, st>>>(kin, n, flag.p);
            uint32_t last_flag = 0;
            ok = ok && cudaMemcpyAsync(&last_flag, flag.p + (n - 1), sizeof(uint32_t), cudaMemcpyDeviceToHost, st) ==
                           cudaSuccess;
            ok = ok && scan_u32(flag.p, n, tot.p, st);
            uint32_t last_pos = 0;
            ok = ok && cudaMemcpyAsync(&last_pos, flag.p + (n - 1), sizeof(uint32_t), cudaMemcpyDeviceToHost, st) ==
                           cudaSuccess;
            ok = ok && cudaStreamSynchronize(st) == cudaSuccess;
            const int64_t nseg = ok ? (int64_t)last_pos + last_flag : 0;
            ok = ok && nseg > 0 && skey.alloc(nseg, st) && ssum.alloc(nseg, st);
            if (ok) {
                seg_start_kernel<<<blocks_for(n, 256), 256, 0, st>>>(kin, n, flag.p, start.p);
                if (w) gather_weights_kernel<<<blocks_for(n, 256), 256, 0, st>>>(n, iin, dw.p, dws.p);
                seg_sum_kernel<<<blocks_for(nseg, 256), 256, 0, st>>>(kin, w ? dws.p : nullptr, start.p, nseg, n,
                                                                      skey.p, ssum.p);
                seg_key.resize((size_t)nseg);
                seg_sum.resize((size_t)nseg);
                ok = cudaGetLastError() == cudaSuccess &&
                     cudaMemcpyAsync(seg_key.data(), skey.p, sizeof(uint64_t) * nseg, cudaMemcpyDeviceToHost, st) ==
                         cudaSuccess &&
                     cudaMemcpyAsync(seg_sum.data(), ssum.p, sizeof(double) * nseg, cudaMemcpyDeviceToHost, st) ==
                         cudaSuccess &&
                     cudaStreamSynchronize(st) == cudaSuccess;
            }
        }
    }
    cudaStreamSynchronize(st);  // the buffers' stream-ordered frees
    cudaStreamDestroy(st);
    if (!ok) cudaGetLastError();  // clear a non-sticky error; the host path takes over
    return ok;
}

}  // namespace wb
