// Device-side containers and the flattened layout of a Schwarz stage.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <memory>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <utility>
#include <vector>

#include "kernels.cuh"

namespace wb {

struct CudaError : std::runtime_error {
    using std::runtime_error::runtime_error;
};

#define WB_CUDA(call)                                                                           \
    do {                                                                                        \
        cudaError_t e_ = (call);                                                                \
        if (e_ != cudaSuccess)                                                                  \
            throw ::wb::CudaError(std::string(#call) + ": " + cudaGetErrorString(e_) + " at " + \
                                  __FILE__ + ":" + std::to_string(__LINE__));                   \
    } while (0)

// Allocator whose construct() without arguments default-initializes: resize() of a
// vector of plain numbers then leaves the new elements unwritten, so that a large array
// filled in parallel afterwards is not first zeroed page by page on one thread.
template <typename T>
struct DefaultInitAllocator : std::allocator<T> {
    DefaultInitAllocator() = default;
    template <typename U>
    DefaultInitAllocator(const DefaultInitAllocator<U>&) noexcept {}
    template <typename U>
    struct rebind {
        using other = DefaultInitAllocator<U>;
    };
    template <typename U>
    void construct(U* p) noexcept(std::is_nothrow_default_constructible<U>::value) {
        ::new (static_cast<void*>(p)) U;
    }
    template <typename U, typename... A>
    void construct(U* p, A&&... a) {
        ::new (static_cast<void*>(p)) U(std::forward<A>(a)...);
    }
};
// Host array of a stage layout that is written in full after it is sized.
template <typename T>
using HostVec = std::vector<T, DefaultInitAllocator<T>>;

// Owning device array.
template <typename T>
struct DArr {
    T* p = nullptr;
    size_t n = 0;
    DArr() = default;
    DArr(const DArr&) = delete;
    DArr& operator=(const DArr&) = delete;
    DArr(DArr&& o) noexcept : p(o.p), n(o.n) { o.p = nullptr; o.n = 0; }
    DArr& operator=(DArr&& o) noexcept {
        if (this != &o) { release(); p = o.p; n = o.n; o.p = nullptr; o.n = 0; }
        return *this;
    }
    ~DArr() { release(); }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        n = 0;
    }
    void alloc(size_t count) {
        if (count <= n && p) return;
        release();
        if (count == 0) return;
        WB_CUDA(cudaMalloc(&p, count * sizeof(T)));
        n = count;
    }
    template <typename V>
    void upload(const V& h) {
        static_assert(std::is_same<typename V::value_type, T>::value, "upload: element type");
        release();
        if (h.empty()) return;
        alloc(h.size());
        WB_CUDA(cudaMemcpy(p, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice));
    }
    template <typename V>
    void upload_cast(const V& h) {
        if constexpr (std::is_same<typename V::value_type, T>::value) {
            upload(h);
        } else {
            std::vector<T> t(h.begin(), h.end());
            upload(t);
        }
    }
};

// Row-wise CSR over local slots with its balanced work chunks.
template <typename T>
struct CsrDev {
    int64_t nrows = 0;
    DArr<uint32_t> row_slot;
    DArr<int64_t> ptr;
    DArr<uint32_t> col;
    DArr<T> val;
    DArr<T> rscale;
    DArr<CsrChunk> chunks;
    int64_t nchunks = 0;
};

// Host form of a row-wise CSR over slots.
struct CsrHost {
    HostVec<uint32_t> row_slot;
    std::vector<int64_t> ptr{0};
    HostVec<uint32_t> col;
    HostVec<double> val;
    std::vector<double> rscale;
    std::vector<CsrChunk> chunks;
    int64_t nrows() const { return (int64_t)row_slot.size(); }
};

// One Schwarz stage: the local solves of a set of subdomains over their concatenated
// slots (slots of subdomain s: q-block then r-block), in the fused form of kernels.cuh.
struct StageHost {
    int32_t nsub = 0;
    int64_t nslots = 0;
    HostVec<uint32_t> gidx, sub_of, keep_slots;
    HostVec<double> spou, rho;                  // per slot, per keep entry
    std::vector<double> invd;                   // per slot (0 = kept)
    std::vector<int32_t> sub_nloc, sub_nkeep;
    std::vector<double> sub_I;                  // sum of invd over eliminated slots
    CsrHost keep;                               // rows: keep list; cols: global dofs
    std::vector<int64_t> bs_ptr{0};             // back substitution rows over all slots
    HostVec<uint32_t> bs_col;                   // keep slot
    HostVec<double> bs_val;                     // C_ek
    // dense reduced solves
    std::vector<int64_t> dn_keep0, dn_loff;
    std::vector<int32_t> dn_n;
    std::vector<double> dn_L;
    // approximate Cholesky level sweeps: rows of level l are chunks [lp[l], lp[l+1])
    CsrHost fwd, bwd;
    std::vector<int64_t> fwd_lp, bwd_lp;
    // dense cores
    std::vector<int32_t> core_of_block, row0_of_block, core_n;
    std::vector<int64_t> core_slot_off, core_z_off;
    std::vector<uint32_t> core_slot;
    std::vector<double> core_z;
    // additive prolongation gather: dof j <- slots gslot[gptr[j]..gptr[j+1]), with the
    // per-slot data and back-substitution rows stored in the same (gather) order, so the
    // prolongation reads them without going through the slot index; each row starts at a
    // multiple of 4 entries (16-byte loads of 4 columns and values) and holds gbs_cnt
    // entries, padded to a multiple of 4 with the row's first column and value 0
    std::vector<int64_t> gptr;
    HostVec<uint32_t> gslot, gsub;
    HostVec<double> gspou, ginvd;
    std::vector<int64_t> gbs_ptr;
    std::vector<uint32_t> gbs_cnt;
    HostVec<uint32_t> gbs_col;
    HostVec<double> gbs_val;
};

template <typename T>
struct StageDev {
    int32_t nsub = 0;
    int64_t nslots = 0, nkeep = 0;
    DArr<uint32_t> gidx, sub_of, keep_slots;
    DArr<T> spou, invd, rho;
    DArr<int32_t> sub_nloc, sub_nkeep;
    DArr<double> sub_I;
    CsrDev<T> keep, fwd, bwd;
    DArr<int64_t> bs_ptr;
    DArr<uint32_t> bs_col;
    DArr<T> bs_val;
    std::vector<int64_t> fwd_lp, bwd_lp;  // host copies (launch ranges)
    DArr<int64_t> fwd_lp_d, bwd_lp_d;     // device copies (fused sweeps)
    int32_t ndense = 0;
    DArr<int64_t> dn_keep0, dn_loff;
    DArr<int32_t> dn_n;
    DArr<T> dn_L;
    int32_t ncore_blocks = 0, core_rmax = 0;
    int64_t core_total = 0;
    DArr<int32_t> core_of_block, row0_of_block, core_n;
    DArr<int64_t> core_slot_off, core_z_off;
    DArr<uint32_t> core_slot;
    DArr<T> core_z;
    DArr<int64_t> gptr;
    DArr<uint32_t> gslot, gsub;
    DArr<T> gspou, ginvd;
    DArr<int64_t> gbs_ptr;
    DArr<uint32_t> gbs_cnt;
    DArr<uint32_t> gbs_col;
    DArr<T> gbs_val;
};

constexpr int kCoreRowsPerBlock = 2;  // output rows per block of core_gemv_kernel (4 warps each)

}  // namespace wb
