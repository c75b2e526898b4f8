// sm_100a kernels of the solve phase.
//
// Vectors with k right-hand sides are RHS-interleaved with the RHS count padded to
// kp, a multiple of 4: element (row, c) at row*kp + c.  A lane owns 4 consecutive RHS
// (one 16-byte float4, or two double2), and a group of G = kp/4 lanes (1, 2, 4 or 8)
// owns a row, so a row of a gather or scatter is one coalesced 16*G-byte (FP32) or
// 32*G-byte (FP64) access.  Padded RHS are zero and stay inactive in the Krylov loops.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <type_traits>

namespace wb {

constexpr int kMaxQ = 16;
constexpr int kBlock = 256;

// ---------------------------------------------------------------------------
// 4-wide RHS vectors
// ---------------------------------------------------------------------------

template <typename T>
struct V4 {
    T a, b, c, d;
    __device__ __forceinline__ V4() {}
    __device__ __forceinline__ V4(T s) : a(s), b(s), c(s), d(s) {}
    __device__ __forceinline__ V4(T a_, T b_, T c_, T d_) : a(a_), b(b_), c(c_), d(d_) {}
    __device__ __forceinline__ V4& operator+=(const V4& o) { a += o.a; b += o.b; c += o.c; d += o.d; return *this; }
    __device__ __forceinline__ V4& operator-=(const V4& o) { a -= o.a; b -= o.b; c -= o.c; d -= o.d; return *this; }
    __device__ __forceinline__ V4& operator*=(T s) { a *= s; b *= s; c *= s; d *= s; return *this; }
    __device__ __forceinline__ bool any() const { return a != T(0) || b != T(0) || c != T(0) || d != T(0); }
};
template <typename T>
__device__ __forceinline__ V4<T> operator*(T s, const V4<T>& v) { return V4<T>(s * v.a, s * v.b, s * v.c, s * v.d); }
template <typename T>
__device__ __forceinline__ V4<T> operator+(V4<T> x, const V4<T>& y) { x += y; return x; }
template <typename T>
__device__ __forceinline__ V4<T> operator-(V4<T> x, const V4<T>& y) { x -= y; return x; }

__device__ __forceinline__ V4<float> ld4(const float* p) {
    const float4 v = *reinterpret_cast<const float4*>(p);
    return V4<float>(v.x, v.y, v.z, v.w);
}
__device__ __forceinline__ V4<double> ld4(const double* p) {
    const double2 u = reinterpret_cast<const double2*>(p)[0], v = reinterpret_cast<const double2*>(p)[1];
    return V4<double>(u.x, u.y, v.x, v.y);
}
__device__ __forceinline__ V4<float> ldg4(const float* p) {
    const float4 v = __ldg(reinterpret_cast<const float4*>(p));
    return V4<float>(v.x, v.y, v.z, v.w);
}
__device__ __forceinline__ V4<double> ldg4(const double* p) {
    const double2 u = __ldg(reinterpret_cast<const double2*>(p)), v = __ldg(reinterpret_cast<const double2*>(p) + 1);
    return V4<double>(u.x, u.y, v.x, v.y);
}
__device__ __forceinline__ void st4(float* p, const V4<float>& v) {
    *reinterpret_cast<float4*>(p) = make_float4(v.a, v.b, v.c, v.d);
}
__device__ __forceinline__ void st4(double* p, const V4<double>& v) {
    reinterpret_cast<double2*>(p)[0] = make_double2(v.a, v.b);
    reinterpret_cast<double2*>(p)[1] = make_double2(v.c, v.d);
}
// global reductions (result unused): one 16-byte vector reduction for FP32, one per
// value for FP64; p is 16-byte aligned
__device__ __forceinline__ void atomic_add4(float* p, const V4<float>& v) {
    asm volatile("red.global.add.v4.f32 [%0], {%1,%2,%3,%4};" ::"l"(p), "f"(v.a), "f"(v.b), "f"(v.c), "f"(v.d)
                 : "memory");
}
__device__ __forceinline__ void atomic_add4(double* p, const V4<double>& v) {
    atomicAdd(p, v.a); atomicAdd(p + 1, v.b); atomicAdd(p + 2, v.c); atomicAdd(p + 3, v.d);
}
// shared-memory reductions without a returned value (red.shared: no retry loop, no
// scoreboard wait on the result)
__device__ __forceinline__ void red_shared(float* p, float v) {
    const unsigned a = (unsigned)__cvta_generic_to_shared(p);
    asm volatile("red.shared.add.f32 [%0], %1;" ::"r"(a), "f"(v) : "memory");
}
__device__ __forceinline__ void red_shared(double* p, double v) {
    const unsigned a = (unsigned)__cvta_generic_to_shared(p);
    asm volatile("red.shared.add.f64 [%0], %1;" ::"r"(a), "d"(v) : "memory");
}
template <typename T>
__device__ __forceinline__ void red_shared4(T* p, const V4<T>& v) {
    red_shared(p, v.a); red_shared(p + 1, v.b); red_shared(p + 2, v.c); red_shared(p + 3, v.d);
}
template <typename T> __device__ __forceinline__ T quiet_nan();
template <> __device__ __forceinline__ float quiet_nan<float>() { return __int_as_float(0x7fc00000); }
template <> __device__ __forceinline__ double quiet_nan<double>() { return __longlong_as_double(0x7ff8000000000000LL); }
template <typename T>
__device__ __forceinline__ V4<double> to_d(const V4<T>& v) { return V4<double>(v.a, v.b, v.c, v.d); }
template <typename T>
__device__ __forceinline__ V4<T> from_d(const V4<double>& v) { return V4<T>((T)v.a, (T)v.b, (T)v.c, (T)v.d); }

// RV consecutive 4-wide RHS vectors of one lane (4 RV right-hand sides), for the
// observation pass's wide lanes; VecR<T, 1> is V4<T> itself.
template <typename T, int RV>
struct VR {
    V4<T> v[RV];
    __device__ __forceinline__ VR() {}
    __device__ __forceinline__ VR(T s) {
#pragma unroll
        for (int j = 0; j < RV; ++j) v[j] = V4<T>(s);
    }
    __device__ __forceinline__ VR& operator+=(const VR& o) {
#pragma unroll
        for (int j = 0; j < RV; ++j) v[j] += o.v[j];
        return *this;
    }
    __device__ __forceinline__ VR& operator-=(const VR& o) {
#pragma unroll
        for (int j = 0; j < RV; ++j) v[j] -= o.v[j];
        return *this;
    }
};
template <typename T, int RV>
__device__ __forceinline__ VR<T, RV> operator*(T s, const VR<T, RV>& a) {
    VR<T, RV> r;
#pragma unroll
    for (int j = 0; j < RV; ++j) r.v[j] = s * a.v[j];
    return r;
}
template <typename T, int RV>
__device__ __forceinline__ VR<T, RV> operator+(VR<T, RV> x, const VR<T, RV>& y) { x += y; return x; }
template <typename T, int RV>
__device__ __forceinline__ VR<T, RV> operator-(VR<T, RV> x, const VR<T, RV>& y) { x -= y; return x; }
template <typename T, int RV>
using VecR = typename std::conditional<RV == 1, V4<T>, VR<T, RV>>::type;
template <int RV, typename T>
__device__ __forceinline__ VecR<T, RV> ldv(const T* p) {
    if constexpr (RV == 1) {
        return ld4(p);
    } else {
        VR<T, RV> r;
#pragma unroll
        for (int j = 0; j < RV; ++j) r.v[j] = ld4(p + 4 * j);
        return r;
    }
}
template <int RV, typename T>
__device__ __forceinline__ VecR<T, RV> ldgv(const T* p) {
    if constexpr (RV == 1) {
        return ldg4(p);
    } else {
        VR<T, RV> r;
#pragma unroll
        for (int j = 0; j < RV; ++j) r.v[j] = ldg4(p + 4 * j);
        return r;
    }
}
template <typename T, int RV>
__device__ __forceinline__ void st4(T* p, const VR<T, RV>& a) {
#pragma unroll
    for (int j = 0; j < RV; ++j) st4(p + 4 * j, a.v[j]);
}
template <typename T, int RV>
__device__ __forceinline__ void atomic_add4(T* p, const VR<T, RV>& a) {
#pragma unroll
    for (int j = 0; j < RV; ++j) atomic_add4(p + 4 * j, a.v[j]);
}
template <typename T, int RV>
__device__ __forceinline__ void red_shared4(T* p, const VR<T, RV>& a) {
#pragma unroll
    for (int j = 0; j < RV; ++j) red_shared4(p + 4 * j, a.v[j]);
}

// ---------------------------------------------------------------------------
// Observation pass: y = D'W(D x) and its relatives, one read of the codes.
// ---------------------------------------------------------------------------

enum ObsMode { OBS_GRAM = 0, OBS_RHS = 1, OBS_RESID = 2, OBS_DX = 3, OBS_LSMR = 4 };

// Work unit: observations [obs_begin, obs_end) (sorted by the primary factor) covering
// primary levels [lvl_begin, lvl_end); a split chunk is a piece of one long level.
struct ObsChunk {
    uint32_t obs_begin, obs_end, lvl_begin, lvl_end;
    uint32_t split;
};

// Where a non-primary factor's weighted sums go.
enum ObsSink : int32_t {
    SINK_GLOBAL = 0,   // run sums flushed by global atomics
    SINK_BLOCK = 1,    // run sums flushed into a block-shared table of every level
    SINK_HOT = 2,      // run sums of the factor's hottest levels into a block-shared table, others global
    SINK_PRIVATE = 3,  // every observation updates a table of every level owned by its lane group
};

// A packed factor's device codes carry, above the level's kObsLevelBits bits, its hot
// slot + 1 (0: not hot), so the observation pass needs no lookup to find a hot level.
constexpr int kObsLevelBits = 24;
constexpr uint32_t kObsLevelMask = (1u << kObsLevelBits) - 1u;
constexpr int kObsMaxHot = 255;

// Factor slots are in device order: slot 0 is the primary factor, the one the
// observations are sorted by.
struct ObsParams {
    int64_t n, ns;          // observations; stride of one factor's codes (n rounded up to 4)
    int32_t Q, kp;
    int32_t smem_elems;     // dynamic shared memory, elements
    int32_t priv_stride;    // elements between consecutive lane groups' private tables
    const uint32_t* codes;  // Q x ns, primary-sorted
    int64_t off[kMaxQ];     // first dof of each slot's level block
    int32_t sink[kMaxQ];
    int32_t packed[kMaxQ];  // codes carry a hot slot (see kObsLevelBits)
    // SINK_PRIVATE: offset of the factor's table inside a group's private area;
    // SINK_BLOCK / SINK_HOT: offset of the block-shared table (after all private areas).
    int32_t smem_base[kMaxQ];
    int32_t smem_len[kMaxQ];           // levels x kp (SINK_HOT: hot levels x kp)
    int32_t hot_cap[kMaxQ];            // SINK_HOT: hot slots held in the table (the rest go global)
    const uint32_t* hot_level[kMaxQ];  // hot slot -> level
    const ObsChunk* chunks;
    int64_t nchunks;
    // OBS_LSMR: per-RHS scale of the old u, and per-warp partial sums of u^2
    // ((block * warps + warp) * kp + rhs)
    const double* lsmr_scale;
    double* lsmr_part;
    // SINK_HOT tables in global memory instead of shared memory when non-null: block b's
    // copy starts at hot_glob + b * hot_glob_stride elements, factor q's table at
    // hot_goff[q] within it (hot_cap[q] x kp); the block zeroes its copy first and adds it
    // into `out` at the end
    void* hot_glob;
    int64_t hot_glob_stride;
    int32_t hot_goff[kMaxQ];
};

template <typename T> struct W4;
template <> struct W4<float> { using type = float4; };
template <> struct W4<double> { struct type { double2 lo, hi; }; };
template <typename T>
__device__ __forceinline__ typename W4<T>::type load_w4v(const T* __restrict__ w, uint32_t i);
template <>
__device__ __forceinline__ float4 load_w4v<float>(const float* __restrict__ w, uint32_t i) {
    return __ldg(reinterpret_cast<const float4*>(w + i));
}
template <>
__device__ __forceinline__ W4<double>::type load_w4v<double>(const double* __restrict__ w, uint32_t i) {
    return W4<double>::type{__ldg(reinterpret_cast<const double2*>(w + i)), __ldg(reinterpret_cast<const double2*>(w + i) + 1)};
}
__device__ __forceinline__ float wcomp(const float4& v, int b) { return b == 0 ? v.x : b == 1 ? v.y : b == 2 ? v.z : v.w; }
__device__ __forceinline__ double wcomp(const W4<double>::type& v, int b) {
    return b == 0 ? v.lo.x : b == 1 ? v.lo.y : b == 2 ? v.hi.x : v.hi.y;
}
__device__ __forceinline__ uint32_t ucomp(const uint4& v, int b) { return b == 0 ? v.x : b == 1 ? v.y : b == 2 ? v.z : v.w; }

// One pass over the observations computing, with one read of the codes,
//   GRAM:  out = D'W D x          RHS:  out = D'W yin
//   RESID: eout = yin - D x, out = D'W eout          DX: eout = D x
//   LSMR:  eout = W D x + scale yin (w = the square roots of the weights; the LSMR
//          bidiagonalization's u = A v + scale u with A = W^(1/2) D), out = D'W eout
//          (A'u), and per-warp partial sums of eout^2 (||u||^2)
// QT == Q, and the last NP factor slots are SINK_PRIVATE (both compile-time); QT = kMaxQ
// is the generic kernel (any Q up to 16, sinks read at run time, no reuse of gathered
// rows).  kp = 4 G.
// Each lane group (G lanes, 4 RHS each) walks whole chunks of primary-sorted
// observations: the primary factor's sums close with a plain store when its level
// changes; a gathered coefficient row is reused while its factor's level repeats; a
// non-primary factor keeps a running sum while its level repeats and flushes it to its
// sink, except SINK_PRIVATE factors (few levels, changing every observation), whose
// group-private table is updated without atomics.  Observations go in aligned batches
// of 4 (one 16-byte load of 4 codes per factor, and of 4 weights) with the next
// batch's loads in flight; a chunk's unaligned head and tail (and
// every observation of the generic kernel) go one at a time.  Addresses come from
// per-factor base pointers with the row stride a compile-time constant.  The block adds
// its shared tables into `out` at the end.
// Wide lanes (RV = 2, the FP32 operator apply only): a lane owns 8 RHS and a group of
// G = kp/8 lanes a row, so the per-observation control (level tests, code and weight
// loads, addresses) is shared by twice the RHS; the group-private tables are as large
// as with 4 RHS per lane, so the block has half the threads (same tables per block).
// Threads per block of the observation pass: 256, or 128 for FP64, whose group-private
// tables are twice as large (the tables of a block are its lane groups' copies), and for
// wide lanes.
template <typename T, int RV = 1>
constexpr int obs_block() { return (sizeof(T) == 8 || RV > 1) ? 128 : 256; }

template <typename T, int G, int MODE, int QT, int NP, int RV = 1>
__global__ void __launch_bounds__(obs_block<T, RV>(), 2) obs_pass_kernel(ObsParams P, const T* __restrict__ w,
                                                             const T* __restrict__ x, const T* __restrict__ yin,
                                                             T* __restrict__ out, T* __restrict__ eout) {
    static_assert(RV == 1 || MODE == OBS_GRAM, "wide lanes: operator apply only");
    using Vec = VecR<T, RV>;
    constexpr int KP = 4 * G * RV;
    constexpr bool kScatter = MODE != OBS_DX;
    constexpr bool kGather = MODE != OBS_RHS;
    constexpr bool kGeneric = QT == kMaxQ;
    constexpr bool kBatch = !kGeneric;                                    // 4-observation batches
    constexpr bool kPrefetch = kBatch;  // next batch's codes and weights in flight
    constexpr int NS = kGeneric ? 1 : QT;                                 // per-slot register arrays
    constexpr uint32_t kNone = 0xffffffffu;
    static_assert(kGeneric || NP < QT, "the primary slot is never private");
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T* sm = reinterpret_cast<T*>(smem_raw);
    T* const hotg = (kScatter && P.hot_glob) ? reinterpret_cast<T*>(P.hot_glob) + (size_t)blockIdx.x * P.hot_glob_stride
                                             : nullptr;
    if (kScatter) {
        for (int i = threadIdx.x; i < P.smem_elems; i += blockDim.x) sm[i] = T(0);
        if (hotg)
            for (int i = threadIdx.x; i < (int)P.hot_glob_stride; i += blockDim.x) hotg[i] = T(0);
        __syncthreads();
    }
    const int c4 = (threadIdx.x & (G - 1)) * 4 * RV;
    const int gl = threadIdx.x / G;
    const int64_t gpb = blockDim.x / G;
    const int64_t ngroups = (int64_t)gridDim.x * gpb;
    const int Q = kGeneric ? P.Q : QT;
    const int64_t ns = P.ns;
    const bool weighted = MODE != OBS_DX && w != nullptr;
    T* const priv = sm + (size_t)gl * P.priv_stride + c4;
    T* const out0 = out + (size_t)P.off[0] * KP + c4;  // primary block, this lane's RHS
    // slot q is private: compile-time for the exact kernels
    auto is_priv = [&](int q) -> bool {
        if constexpr (kGeneric) return q > 0 && P.sink[q] == SINK_PRIVATE;
        else return q >= QT - NP;
    };
    auto lev = [&](int q, uint32_t c) { return P.packed[q] ? (c & kObsLevelMask) : c; };
    auto xrow = [&](int q, uint32_t c) -> const T* {
        return x + ((size_t)P.off[q] + (q == 0 || is_priv(q) ? c : lev(q, c))) * KP + c4;
    };
    // run sum of non-private slot q at device code c into its sink
    auto flush = [&](int q, uint32_t c, const Vec& a) {
        const int32_t sink = P.sink[q];
        const uint32_t lv = lev(q, c), hot = P.packed[q] ? (c >> kObsLevelBits) : 0u;
        if (sink == SINK_BLOCK) red_shared4(sm + P.smem_base[q] + c4 + (size_t)lv * KP, a);
        else if (sink == SINK_HOT && hot && (int32_t)hot <= P.hot_cap[q]) {
            if (hotg) atomic_add4(hotg + P.hot_goff[q] + c4 + (size_t)(hot - 1) * KP, a);
            else red_shared4(sm + P.smem_base[q] + c4 + (size_t)(hot - 1) * KP, a);
        } else atomic_add4(out + ((size_t)P.off[q] + lv) * KP + c4, a);
    };

    V4<double> lsc(0.0), usq(0.0);  // OBS_LSMR: this lane's scales and sum of u^2
    if constexpr (MODE == OBS_LSMR) lsc = V4<double>(P.lsmr_scale[c4], P.lsmr_scale[c4 + 1], P.lsmr_scale[c4 + 2], P.lsmr_scale[c4 + 3]);
    for (int64_t ch = (int64_t)blockIdx.x * gpb + gl; ch < P.nchunks; ch += ngroups) {
        const ObsChunk C = P.chunks[ch];
        uint32_t lvl = C.lvl_begin;
        Vec acc(T(0));
        uint32_t run_l[QT], cl[NS];
        Vec run_a[QT], cv[NS];
#pragma unroll
        for (int q = 0; q < QT; ++q) {
            run_l[q] = kNone;
            run_a[q] = Vec(T(0));
        }
#pragma unroll
        for (int q = 0; q < NS; ++q) {
            cl[q] = kNone;
            cv[q] = Vec(T(0));
        }
        // one observation: codes c[0..Q), weight wi
        // one observation in two phases: its row sum (loads) and its scatter; a batch
        // runs the first phase for all its observations before the second, so their
        // loads are in flight together (the scatter's reductions order memory)
        auto gather = [&](uint32_t i, const uint32_t (&c)[QT]) -> Vec {
            Vec s(T(0));
            if constexpr (kGather) {
#pragma unroll
                for (int q = 0; q < QT; ++q) {
                    if (q >= Q) continue;
                    if (kGeneric || is_priv(q)) {
                        s += ldgv<RV>(xrow(q, c[q]));  // generic kernel, or a level that changes every time
                    } else {
                        if (c[q] != cl[q]) cv[q] = ldgv<RV>(xrow(q, c[q]));
                        cl[q] = c[q];
                        s += cv[q];
                    }
                }
            }
            if constexpr (MODE == OBS_RHS || MODE == OBS_RESID) {
                const Vec yv = ldv<RV>(yin + (size_t)i * KP + c4);
                s = (MODE == OBS_RHS) ? yv : yv - s;
            }
            return s;
        };
        auto scatter = [&](uint32_t i, const uint32_t (&c)[QT], T wi, const Vec& s0) {
            Vec s = s0;
            if constexpr (MODE == OBS_LSMR) {  // u = w (D x) + scale u_old
                const Vec uo = ldv<RV>(yin + (size_t)i * KP + c4);
                s = wi * s0;
                if (lsc.a != 0.0) s.a += (T)lsc.a * uo.a;
                if (lsc.b != 0.0) s.b += (T)lsc.b * uo.b;
                if (lsc.c != 0.0) s.c += (T)lsc.c * uo.c;
                if (lsc.d != 0.0) s.d += (T)lsc.d * uo.d;
                usq.a += (double)s.a * s.a; usq.b += (double)s.b * s.b;
                usq.c += (double)s.c * s.c; usq.d += (double)s.d * s.d;
            }
            if constexpr (MODE == OBS_DX || MODE == OBS_RESID || MODE == OBS_LSMR) st4(eout + (size_t)i * KP + c4, s);
            if constexpr (kScatter) {
                const Vec t = wi * s;
                const uint32_t p = c[0];
                if (p != lvl) {  // primary level complete: plain store
                    st4(out0 + (size_t)lvl * KP, acc);
                    for (uint32_t l = lvl + 1; l < p; ++l) st4(out0 + (size_t)l * KP, Vec(T(0)));  // empty levels
                    acc = Vec(T(0));
                    lvl = p;
                }
                acc += t;
#pragma unroll
                for (int q = 1; q < QT; ++q) {
                    if (q >= Q) continue;
                    if (is_priv(q)) {
                        T* pt = priv + P.smem_base[q] + (size_t)c[q] * KP;
                        st4(pt, ldv<RV>(pt) + t);
                    } else if (c[q] != run_l[q]) {
                        if (run_l[q] != kNone) flush(q, run_l[q], run_a[q]);
                        run_l[q] = c[q];
                        run_a[q] = t;
                    } else {
                        run_a[q] += t;
                    }
                }
            }
        };
        auto body = [&](uint32_t i, const uint32_t (&c)[QT], T wi) { scatter(i, c, wi, gather(i, c)); };
        auto single = [&](uint32_t i) {
            uint32_t c[QT];
#pragma unroll
            for (int q = 0; q < QT; ++q) c[q] = q < Q ? __ldg(P.codes + (size_t)q * ns + i) : 0u;
            body(i, c, weighted ? __ldg(w + i) : T(1));
        };
        uint32_t i = C.obs_begin;
        if constexpr (kBatch) {
            for (; i < C.obs_end && (i & 3u); ++i) single(i);
            if (i + 4 <= C.obs_end) {
                uint4 cb[QT];
                typename W4<T>::type wb{};
#pragma unroll
                for (int q = 0; q < QT; ++q) cb[q] = __ldg(reinterpret_cast<const uint4*>(P.codes + (size_t)q * ns + i));
                if (weighted) wb = load_w4v(w, i);
                for (; i + 4 <= C.obs_end; i += 4) {
                    uint4 nb[kPrefetch ? QT : 1];
                    typename W4<T>::type nw = wb;
                    const bool more = i + 8 <= C.obs_end;
                    if constexpr (kPrefetch) {  // next batch in flight while this one is processed
#pragma unroll
                        for (int q = 0; q < QT; ++q)
                            nb[q] = more ? __ldg(reinterpret_cast<const uint4*>(P.codes + (size_t)q * ns + i + 4)) : cb[q];
                        if (weighted && more) nw = load_w4v(w, i + 4);
                    }
                    uint32_t c[4][QT];
                    Vec s[4];
#pragma unroll
                    for (int b = 0; b < 4; ++b) {
#pragma unroll
                        for (int q = 0; q < QT; ++q) c[b][q] = ucomp(cb[q], b);
                        s[b] = gather(i + b, c[b]);
                    }
#pragma unroll
                    for (int b = 0; b < 4; ++b) scatter(i + b, c[b], weighted ? (T)wcomp(wb, b) : T(1), s[b]);
                    if constexpr (kPrefetch) {
#pragma unroll
                        for (int q = 0; q < QT; ++q) cb[q] = nb[q];
                        wb = nw;
                    } else if (more) {
#pragma unroll
                        for (int q = 0; q < QT; ++q)
                            cb[q] = __ldg(reinterpret_cast<const uint4*>(P.codes + (size_t)q * ns + i + 4));
                        if (weighted) wb = load_w4v(w, i + 4);
                    }
                }
            }
        }
        for (; i < C.obs_end; ++i) single(i);
        if constexpr (kScatter) {
#pragma unroll
            for (int q = 1; q < QT; ++q)
                if (q < Q && !is_priv(q) && run_l[q] != kNone) flush(q, run_l[q], run_a[q]);
            if (C.split) {
                atomic_add4(out0 + (size_t)C.lvl_begin * KP, acc);
            } else {
                for (; lvl < C.lvl_end; ++lvl) {
                    st4(out0 + (size_t)lvl * KP, acc);
                    acc = Vec(T(0));
                }
            }
        }
    }
    if constexpr (MODE == OBS_LSMR) {  // sum the warp's lane groups; lanes < G store
#pragma unroll
        for (int o = G; o < 32; o <<= 1) {
            usq.a += __shfl_xor_sync(0xffffffffu, usq.a, o);
            usq.b += __shfl_xor_sync(0xffffffffu, usq.b, o);
            usq.c += __shfl_xor_sync(0xffffffffu, usq.c, o);
            usq.d += __shfl_xor_sync(0xffffffffu, usq.d, o);
        }
        if ((threadIdx.x & 31) < G) {
            double* pw = P.lsmr_part + ((size_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5)) * KP + c4;
            pw[0] = usq.a; pw[1] = usq.b; pw[2] = usq.c; pw[3] = usq.d;
        }
    }
    if (kScatter && (P.smem_elems > 0 || hotg)) {
        __syncthreads();
        // the block's tables into `out`: one atomic per nonzero entry (the global hot
        // tables read from L2, where the reductions went)
        for (int q = 1; q < Q; ++q) {
            const int32_t sink = P.sink[q];
            if (sink == SINK_GLOBAL) continue;
            for (int e = threadIdx.x; e < P.smem_len[q]; e += blockDim.x) {
                T v = T(0);
                uint32_t lv;
                if (sink == SINK_PRIVATE) {
                    for (int g = 0; g < (int)gpb; ++g) v += sm[(size_t)g * P.priv_stride + P.smem_base[q] + e];
                    lv = (uint32_t)(e / KP);
                } else {
                    v = (sink == SINK_HOT && hotg) ? __ldcg(hotg + P.hot_goff[q] + e) : sm[P.smem_base[q] + e];
                    lv = (sink == SINK_BLOCK) ? (uint32_t)(e / KP) : P.hot_level[q][e / KP];
                }
                if (v != T(0)) atomicAdd(out + (size_t)(P.off[q] + lv) * KP + e % KP, v);
            }
        }
    }
}

// ---------------------------------------------------------------------------
// Hybrid operator apply, primary-major part.  G x splits into the blocks between the
// primary factor P and the small factors S (their cross-tabulations hold one entry per
// observation, so they stay implicit: one pass over the observations), and every block
// that involves another factor O (small cross-tabulations, applied as CSR rows of the
// assembled Gramian: csr_rows_kernel).  This kernel computes, per primary level p,
//   y_P[p] = (sum_i w_i) x_P[p] + sum_i w_i sum_j x_Sj[s_j,i] + sum_e C_PO[p,e] x_O[o_e]
// over its observations i and its C_PO entries, stored once (pieces of split levels add
// atomically), and adds w_i x_P[p] into group-private tables of the S factors, summed
// into y_S at the end (the S rows' other terms, D_S x_S, C_SO x_O and C_SS' x_S', come
// from the CSR rows).  Each lane group (G lanes x 4 RHS) walks whole level-aligned chunks
// of primary-sorted observations in aligned batches of 4 (16-byte loads of 4 codes and
// 4 weights), with a level change the only per-observation test; no code of the primary
// or of an O factor is read.
// ---------------------------------------------------------------------------
constexpr int kPrimMaxS = 2;

struct PrimParams {
    int64_t ns;                    // stride of one factor's codes
    int32_t nsmall;                // S factors (1 or 2)
    int32_t smem_elems;            // dynamic shared memory, elements
    int32_t priv_stride;           // elements between consecutive lane groups' private tables
    int64_t off_p;                 // first dof of the primary factor
    const uint32_t* codes_s[kPrimMaxS];  // the S factors' device codes (primary-sorted)
    int64_t off_s[kPrimMaxS];      // first dof of each S factor
    int32_t nlev_s[kPrimMaxS];
    int32_t priv_base[kPrimMaxS];  // offset of the factor's table inside a group's area
    int32_t xs_base[kPrimMaxS];    // offset of the factor's staged x rows (after the private areas)
    const ObsChunk* chunks;
    int64_t nchunks;
    const uint32_t* lvl_ptr;       // first observation of each primary level (+ n)
    const int64_t* pptr;           // C_PO rows of the primary levels
    const uint32_t* pcol;          // global dof of each entry
};

template <typename T, int G, int NS>
__global__ void __launch_bounds__(obs_block<T>(), 2) prim_rows_kernel(PrimParams P, const T* __restrict__ w,
                                                              const T* __restrict__ pval, const T* __restrict__ x,
                                                              T* __restrict__ out) {
    constexpr int KP = 4 * G;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T* sm = reinterpret_cast<T*>(smem_raw);
    const int gpb0 = blockDim.x / G;
    for (int i = threadIdx.x; i < P.smem_elems; i += blockDim.x) sm[i] = T(0);
    __syncthreads();
#pragma unroll
    for (int j = 0; j < NS; ++j)  // stage the S factors' rows of x
        for (int e = threadIdx.x; e < P.nlev_s[j] * KP; e += blockDim.x)
            sm[P.xs_base[j] + e] = x[(size_t)P.off_s[j] * KP + e];
    __syncthreads();
    const int c4 = (threadIdx.x & (G - 1)) * 4;
    const int gl = threadIdx.x / G;
    const int64_t ngroups = (int64_t)gridDim.x * gpb0;
    const bool weighted = w != nullptr;
    T* const priv = sm + (size_t)gl * P.priv_stride + c4;
    T* const out0 = out + (size_t)P.off_p * KP + c4;
    const T* const x0 = x + (size_t)P.off_p * KP + c4;
    // The next chunk's descriptor, first primary row, first kPrimPre C_PO gathers and
    // first batch of codes and weights are loaded while the current chunk runs (a chunk
    // is often one primary level of a few dozen observations: its loads would otherwise
    // stand exposed at its start and end).
    constexpr int kPrimPre = 4;
    struct Pre {
        ObsChunk C;
        uint32_t nb;
        bool first;
        V4<T> xp, g[kPrimPre];
        T v[kPrimPre];
        int64_t e1;
        uint4 cb[NS];
        typename W4<T>::type wb;
    };
    auto prefetch = [&](int64_t c, Pre& q) {
        q.C = P.chunks[c];
        const uint32_t p = q.C.lvl_begin;
        q.first = __ldg(P.lvl_ptr + p) >= q.C.obs_begin;
        q.nb = __ldg(P.lvl_ptr + p + 1);
        q.xp = ldg4(x0 + (size_t)p * KP);
        const int64_t e0 = __ldg(P.pptr + p);
        q.e1 = __ldg(P.pptr + p + 1);
#pragma unroll
        for (int k = 0; k < kPrimPre; ++k) {
            const bool ok = q.first && e0 + k < q.e1;
            const uint32_t col = ok ? __ldg(P.pcol + e0 + k) : (uint32_t)P.off_p;
            q.v[k] = ok ? __ldg(pval + e0 + k) : T(0);
            q.g[k] = ldg4(x + (size_t)col * KP + c4);
        }
        const uint32_t i0 = q.C.obs_begin;
        const bool full = (i0 & 3u) == 0 && i0 + 4 <= q.C.obs_end;
#pragma unroll
        for (int j = 0; j < NS; ++j)
            q.cb[j] = full ? __ldg(reinterpret_cast<const uint4*>(P.codes_s[j] + i0)) : make_uint4(0, 0, 0, 0);
        q.wb = typename W4<T>::type{};
        if (weighted && full) q.wb = load_w4v(w, i0);
    };
    int64_t ch = (int64_t)blockIdx.x * gpb0 + gl;
    Pre nx;
    if (ch < P.nchunks) prefetch(ch, nx);
    for (; ch < P.nchunks; ch += ngroups) {
        const Pre cu = nx;
        if (ch + ngroups < P.nchunks) prefetch(ch + ngroups, nx);
        const ObsChunk C = cu.C;
        uint32_t p = C.lvl_begin;
        uint32_t nb = cu.nb;
        bool first = cu.first, lead = true;  // lead: the chunk's first level (prefetched C_PO)
        V4<T> xp = cu.xp, acc(T(0));
        T ws = T(0);
        // level p complete (or the chunk's piece of it): its sums into y_P
        auto finish = [&]() {
            acc += ws * xp;
            if (first) {
                int64_t e = __ldg(P.pptr + p);
                const int64_t e1 = lead ? cu.e1 : __ldg(P.pptr + p + 1);
                if (lead) {
#pragma unroll
                    for (int k = 0; k < kPrimPre; ++k) acc += cu.v[k] * cu.g[k];
                    e += kPrimPre;
                }
                for (; e < e1; ++e) acc += __ldg(pval + e) * ldg4(x + (size_t)__ldg(P.pcol + e) * KP + c4);
            }
            if (C.split) atomic_add4(out0 + (size_t)p * KP, acc);
            else st4(out0 + (size_t)p * KP, acc);
        };
        // observation i with S codes s[] and weight wi; advances the level first
        auto body = [&](uint32_t i, const uint32_t (&s)[NS], T wi) {
            if (i == nb) {
                finish();
                lead = false;
                for (++p; __ldg(P.lvl_ptr + p + 1) == i; ++p) st4(out0 + (size_t)p * KP, V4<T>(T(0)));  // empty levels
                nb = __ldg(P.lvl_ptr + p + 1);
                first = true;
                xp = ldg4(x0 + (size_t)p * KP);
                acc = V4<T>(T(0));
                ws = T(0);
            }
            V4<T> xs = ld4(sm + P.xs_base[0] + (size_t)s[0] * KP + c4);
            if (NS > 1) xs += ld4(sm + P.xs_base[NS - 1] + (size_t)s[NS - 1] * KP + c4);
            ws += wi;
            acc += wi * xs;
            const V4<T> t = wi * xp;
#pragma unroll
            for (int j = 0; j < NS; ++j) {
                T* pt = priv + P.priv_base[j] + (size_t)s[j] * KP;
                st4(pt, ld4(pt) + t);
            }
        };
        auto single = [&](uint32_t i) {
            uint32_t s[NS];
#pragma unroll
            for (int j = 0; j < NS; ++j) s[j] = __ldg(P.codes_s[j] + i);
            body(i, s, weighted ? __ldg(w + i) : T(1));
        };
        uint32_t i = C.obs_begin;
        for (; i < C.obs_end && (i & 3u); ++i) single(i);
        if (i + 4 <= C.obs_end) {
            uint4 cb[NS];
            typename W4<T>::type wb = cu.wb;
#pragma unroll
            for (int j = 0; j < NS; ++j) cb[j] = cu.cb[j];
            if (i != C.obs_begin) {  // unaligned start: the first batch was not prefetched
#pragma unroll
                for (int j = 0; j < NS; ++j) cb[j] = __ldg(reinterpret_cast<const uint4*>(P.codes_s[j] + i));
                if (weighted) wb = load_w4v(w, i);
            }
            for (; i + 4 <= C.obs_end; i += 4) {
                uint4 nbk[NS];
                typename W4<T>::type nw = wb;
                const bool more = i + 8 <= C.obs_end;
#pragma unroll
                for (int j = 0; j < NS; ++j)
                    nbk[j] = more ? __ldg(reinterpret_cast<const uint4*>(P.codes_s[j] + i + 4)) : cb[j];
                if (weighted && more) nw = load_w4v(w, i + 4);
#pragma unroll
                for (int b = 0; b < 4; ++b) {
                    uint32_t s[NS];
#pragma unroll
                    for (int j = 0; j < NS; ++j) s[j] = ucomp(cb[j], b);
                    body(i + b, s, weighted ? (T)wcomp(wb, b) : T(1));
                }
#pragma unroll
                for (int j = 0; j < NS; ++j) cb[j] = nbk[j];
                wb = nw;
            }
        }
        for (; i < C.obs_end; ++i) single(i);
        finish();
        if (!C.split)
            for (++p; p < C.lvl_end; ++p) st4(out0 + (size_t)p * KP, V4<T>(T(0)));  // trailing empty levels
    }
    __syncthreads();
    // the lane groups' tables into y_S: one atomic per nonzero entry
#pragma unroll
    for (int j = 0; j < NS; ++j)
        for (int e = threadIdx.x; e < P.nlev_s[j] * KP; e += blockDim.x) {
            T v = T(0);
            for (int g = 0; g < gpb0; ++g) v += sm[(size_t)g * P.priv_stride + P.priv_base[j] + e];
            if (v != T(0)) atomicAdd(out + (size_t)P.off_s[j] * KP + e, v);
        }
}

// ---------------------------------------------------------------------------
// Primary-major pass of the hybrid apply on the FP64 tensor cores (16 RHS).  A warp
// takes 8 pieces of primary levels at a time (a level of at most 64 observations, or a
// 64-observation piece of a longer one), one per lane group.  Each group sums its
// piece's weights by small-factor level into row g of an 8 x wcols tile W in shared
// memory (the levels of up to two small factors side by side, each padded to 8), so that
//   Y_P = W X_S     (the piece's sum_i w_i x_S[s_i]; 8 x 16, K = wcols)
//   Y_S += W' X_P   (the small factors' sum_i w_i x_P[p_i]; wcols x 16, K = 8)
// are products on the tensor cores (mma.sync m8n8k4, FP64, exact for FP32 inputs too)
// instead of per-observation gathers and lane-group tables.  Y_S stays in the warp's
// accumulator fragments until the end.  The piece's C_PO entries and its diagonal
// (sum_i w_i) x_P[p] complete y_P[p] as in prim_rows_kernel.
// ---------------------------------------------------------------------------
constexpr int kMmaKP = 16;        // RHS columns (kp) of this kernel
constexpr int kMmaMaxCols = 48;   // small-factor levels, padded to 8 per factor
constexpr int kMmaPiece = 64;     // observations per piece at most

struct PrimMmaParams {
    int64_t off_p;
    int32_t nsmall;                     // 1 or 2
    const uint32_t* codes_s[kPrimMaxS];
    int64_t off_s[kPrimMaxS];
    int32_t nlev_s[kPrimMaxS];
    int32_t col_s[kPrimMaxS];           // first column of each factor in W
    int32_t wcols;                      // multiple of 8, <= kMmaMaxCols
    const uint4* pieces;                // (level, first obs, end obs, first piece | split << 1)
    int64_t npieces;
    const int64_t* pptr;                // C_PO rows of the primary levels
    const uint32_t* pcol;
};

// d = a b + c for an 8x4 by 4x8 FP64 product; per lane: a = A[lane/4][lane%4],
// b = B[lane%4][lane/4], c and d = C[lane/4][2 (lane%4) + {0, 1}]
__device__ __forceinline__ void dmma_8x8x4(double& d0, double& d1, double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
                 : "+d"(d0), "+d"(d1)
                 : "d"(a), "d"(b));
}

template <typename T>
__global__ void __launch_bounds__(256, 2) prim_mma_kernel(PrimMmaParams P, const T* __restrict__ w,
                                                          const T* __restrict__ pval, const T* __restrict__ x,
                                                          T* __restrict__ out) {
    constexpr int KP = kMmaKP;
    constexpr int MC = kMmaMaxCols;
    __shared__ __align__(16) double XS[MC * KP];          // the small factors' rows of x
    __shared__ __align__(16) double Wt[8][8 * MC];         // per warp: W, 8 x wcols (row stride MC)
    __shared__ __align__(16) double XP[8][8 * KP];         // per warp: the pieces' rows of x_P
    __shared__ __align__(16) double YP[8][8 * KP];         // per warp: W X_S
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int g = lane >> 2, c = lane & 3;
    const int wc = P.wcols;
    for (int e = threadIdx.x; e < MC * KP; e += blockDim.x) {
        const int col = e / KP, n = e % KP;
        double v = 0.0;
        for (int j = 0; j < P.nsmall; ++j)
            if (col >= P.col_s[j] && col < P.col_s[j] + P.nlev_s[j])
                v = (double)x[(size_t)(P.off_s[j] + (col - P.col_s[j])) * KP + n];
        XS[e] = v;
    }
    __syncthreads();
    double* W = Wt[warp];
    double* xpw = XP[warp];
    double* ypw = YP[warp];
    double cs[MC / 8][2][2];  // Y_S fragments: rows 8 mt + g, columns 8 nt + 2 c + {0, 1}
#pragma unroll
    for (int mt = 0; mt < MC / 8; ++mt)
#pragma unroll
        for (int nt = 0; nt < 2; ++nt) cs[mt][nt][0] = cs[mt][nt][1] = 0.0;
    const T* const x0 = x + (size_t)P.off_p * KP + 4 * c;
    T* const out0 = out + (size_t)P.off_p * KP + 4 * c;
    const int64_t ntasks = (P.npieces + 7) / 8;
    for (int64_t task = (int64_t)blockIdx.x * (blockDim.x >> 5) + warp; task < ntasks;
         task += (int64_t)gridDim.x * (blockDim.x >> 5)) {
        const int64_t pi = task * 8 + g;
        const bool has = pi < P.npieces;
        const uint4 pc = has ? __ldg(P.pieces + pi) : make_uint4(0u, 0u, 0u, 0u);
        const uint32_t p = pc.x;
        const V4<T> xp = has ? ldg4(x0 + (size_t)p * KP) : V4<T>(T(0));
        xpw[g * KP + 4 * c + 0] = (double)xp.a;
        xpw[g * KP + 4 * c + 1] = (double)xp.b;
        xpw[g * KP + 4 * c + 2] = (double)xp.c;
        xpw[g * KP + 4 * c + 3] = (double)xp.d;
        for (int j = c; j < wc; j += 4) W[g * MC + j] = 0.0;
        __syncwarp();
        // row g of W: the piece's weights by small-factor level; the group's four lanes
        // take every fourth observation (consecutive lanes, consecutive observations) and
        // add with shared-memory reductions (two of them meet only on a repeated level)
        double ws = 0.0;
        for (uint32_t i = pc.y + c; i < pc.z; i += 4) {
            const double wi = w ? (double)__ldg(w + i) : 1.0;
            ws += wi;
            for (int j = 0; j < P.nsmall; ++j) red_shared(W + g * MC + P.col_s[j] + __ldg(P.codes_s[j] + i), wi);
        }
        ws += __shfl_xor_sync(0xffffffffu, ws, 1);
        ws += __shfl_xor_sync(0xffffffffu, ws, 2);
        __syncwarp();
        // Y_P = W X_S (8 x 16): two 8-column tiles, K = wcols in steps of 4
#pragma unroll
        for (int nt = 0; nt < 2; ++nt) {
            double d0 = 0.0, d1 = 0.0;
            for (int kk = 0; kk < wc; kk += 4)
                dmma_8x8x4(d0, d1, W[g * MC + kk + c], XS[(kk + c) * KP + 8 * nt + g]);
            ypw[g * KP + 8 * nt + 2 * c] = d0;
            ypw[g * KP + 8 * nt + 2 * c + 1] = d1;
        }
        // Y_S += W' X_P (wcols x 16): rows in tiles of 8, K = the 8 pieces
#pragma unroll
        for (int mt = 0; mt < MC / 8; ++mt) {
            if (8 * mt >= wc) break;
#pragma unroll
            for (int nt = 0; nt < 2; ++nt)
#pragma unroll
                for (int kk = 0; kk < 8; kk += 4)
                    dmma_8x8x4(cs[mt][nt][0], cs[mt][nt][1], W[(kk + c) * MC + 8 * mt + g],
                               xpw[(kk + c) * KP + 8 * nt + g]);
        }
        __syncwarp();
        if (has) {
            V4<double> acc(ypw[g * KP + 4 * c], ypw[g * KP + 4 * c + 1], ypw[g * KP + 4 * c + 2],
                           ypw[g * KP + 4 * c + 3]);
            acc += ws * to_d(xp);
            if (pc.w & 1u)  // the level's first piece: its C_PO entries
                for (int64_t e = __ldg(P.pptr + p), e1 = __ldg(P.pptr + p + 1); e < e1; ++e)
                    acc += (double)__ldg(pval + e) * to_d(ldg4(x + (size_t)__ldg(P.pcol + e) * KP + 4 * c));
            if (pc.w & 2u) atomic_add4(out0 + (size_t)p * KP, from_d<T>(acc));
            else st4(out0 + (size_t)p * KP, from_d<T>(acc));
        }
        __syncwarp();  // W, XP and YP are rewritten by the next task
    }
    // the warp's Y_S into y_S
#pragma unroll
    for (int mt = 0; mt < MC / 8; ++mt) {
        const int col = 8 * mt + g;
        if (col >= wc) break;
        for (int j = 0; j < P.nsmall; ++j) {
            if (col < P.col_s[j] || col >= P.col_s[j] + P.nlev_s[j]) continue;
            T* d = out + (size_t)(P.off_s[j] + (col - P.col_s[j])) * KP;
#pragma unroll
            for (int nt = 0; nt < 2; ++nt) {
                if (cs[mt][nt][0] != 0.0) atomicAdd(d + 8 * nt + 2 * c, (T)cs[mt][nt][0]);
                if (cs[mt][nt][1] != 0.0) atomicAdd(d + 8 * nt + 2 * c + 1, (T)cs[mt][nt][1]);
            }
        }
    }
}

// Column-major (RHS-major) user order <-> interleaved primary-sorted order with kp
// columns (padding columns are zero).  perm[i] = user index of sorted row i (or identity).
// Each warp transposes tiles of 32 rows through its own shared-memory tile (32 x kp+1):
// column-major accesses are one row per lane (coalesced per column), row-major ones run
// over the tile's flat elements (consecutive lanes, consecutive addresses).
constexpr int kXposeWarps = 4;  // warps per block of the transpose kernels
inline size_t xpose_smem(int kp) { return (size_t)kXposeWarps * 32 * (kp + 1) * sizeof(double); }

template <typename T>
__global__ void __launch_bounds__(kXposeWarps * 32) gather_interleave_kernel(const double* __restrict__ ycol, int64_t n,
                                                                             int k, int kp,
                                                                             const uint32_t* __restrict__ perm,
                                                                             T* __restrict__ yi) {
    extern __shared__ double xtile[];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int ld = kp + 1;
    double* tile = xtile + (size_t)warp * 32 * ld;
    const int64_t nw = (int64_t)gridDim.x * kXposeWarps;
    for (int64_t i0 = ((int64_t)blockIdx.x * kXposeWarps + warp) * 32; i0 < n; i0 += nw * 32) {
        const int64_t i = i0 + lane;
        const bool ok = i < n;
        const size_t src = ok ? (perm ? (size_t)perm[i] : (size_t)i) : 0;
        for (int c = 0; c < kp; ++c) tile[lane * ld + c] = (ok && c < k) ? ycol[(size_t)c * n + src] : 0.0;
        __syncwarp();
        const int rows = (int)min((int64_t)32, n - i0);
        T* dst = yi + (size_t)i0 * kp;
        for (int f = lane; f < rows * kp; f += 32) dst[f] = (T)tile[(f / kp) * ld + f % kp];
        __syncwarp();
    }
}

template <typename T>
__global__ void __launch_bounds__(kXposeWarps * 32) scatter_deinterleave_kernel(const T* __restrict__ ei, int64_t n,
                                                                                int k, int kp,
                                                                                const uint32_t* __restrict__ perm,
                                                                                double* __restrict__ ecol) {
    extern __shared__ double xtile[];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int ld = kp + 1;
    double* tile = xtile + (size_t)warp * 32 * ld;
    const int64_t nw = (int64_t)gridDim.x * kXposeWarps;
    for (int64_t i0 = ((int64_t)blockIdx.x * kXposeWarps + warp) * 32; i0 < n; i0 += nw * 32) {
        const int rows = (int)min((int64_t)32, n - i0);
        const T* src = ei + (size_t)i0 * kp;
        for (int f = lane; f < rows * kp; f += 32) tile[(f / kp) * ld + f % kp] = (double)src[f];
        __syncwarp();
        const int64_t i = i0 + lane;
        if (i < n) {
            const size_t dst = perm ? (size_t)perm[i] : (size_t)i;
            for (int c = 0; c < k; ++c) ecol[(size_t)c * n + dst] = tile[lane * ld + c];
        }
        __syncwarp();
    }
}

// Row permutation of an interleaved n x kp FP64 array: out[i] = in[perm[i]] (gather) or
// out[perm[i]] = in[i] (scatter), in 16-byte pieces.  With a non-identity order the
// column-major <-> interleaved transposes run in user order (coalesced) and only this
// pass moves whole rows (one random 16*kp/2-byte access per row instead of kp random
// 8-byte ones).
static __global__ void permute_rows_kernel(const double* __restrict__ in, int64_t n, int kp,
                                    const uint32_t* __restrict__ perm, int scatter, double* __restrict__ out) {
    const int per_row = kp / 2;
    const int64_t total = n * per_row;
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t i = t / per_row;
        const int c = (int)(t % per_row);
        const int64_t p = perm[i];
        const int64_t src = scatter ? i : p, dst = scatter ? p : i;
        reinterpret_cast<double2*>(out + (size_t)dst * kp)[c] = reinterpret_cast<const double2*>(in + (size_t)src * kp)[c];
    }
}

// z = NaN everywhere when *failed is set (a multiplicative apply whose local solve did
// not complete).
template <typename T>
__global__ void nan_on_failure_kernel(T* __restrict__ z, int64_t n, const int32_t* __restrict__ failed) {
    if (*failed == 0) return;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        z[i] = quiet_nan<T>();
}

// Blocks for a transpose over `rows` rows (grid-stride beyond 16 blocks per SM).
inline unsigned xpose_blocks(int64_t rows, int n_sm) {
    const int64_t need = (rows + 32 * kXposeWarps - 1) / (32 * kXposeWarps);
    return (unsigned)(need < 1 ? 1 : (need < (int64_t)n_sm * 16 ? need : (int64_t)n_sm * 16));
}

// ---------------------------------------------------------------------------
// Row-wise vector kernels over (rows x kp) vectors; dots accumulate in FP64.
// ---------------------------------------------------------------------------

// Block partial sums: part[blockIdx.x * kp + c] (fixed order: deterministic).
template <int G>
__device__ __forceinline__ void block_reduce_store4(const V4<double>& v, int kp, double* part) {
    __shared__ double red[kBlock * 4];
    const int t = threadIdx.x;
    red[4 * t] = v.a; red[4 * t + 1] = v.b; red[4 * t + 2] = v.c; red[4 * t + 3] = v.d;
    __syncthreads();
    // thread t owns RHS (t % G)*4 .. +3; fold groups onto the first group
    for (int s = blockDim.x / 2; s >= G; s >>= 1) {
        if (t < s) {
#pragma unroll
            for (int j = 0; j < 4; ++j) red[4 * t + j] += red[4 * (t + s) + j];
        }
        __syncthreads();
    }
    if (t < G) {
#pragma unroll
        for (int j = 0; j < 4; ++j) part[(size_t)blockIdx.x * kp + 4 * t + j] = red[4 * t + j];
    }
}

template <typename TA, typename TB, int G>
__global__ void __launch_bounds__(kBlock) dot_kernel(const TA* __restrict__ a, const TB* __restrict__ b,
                                                     int64_t rows, int kp, double* __restrict__ part) {
    const int c4 = (threadIdx.x & (G - 1)) * 4;
    V4<double> s(0.0);
    const int64_t rpb = blockDim.x / G;
    for (int64_t r = (int64_t)blockIdx.x * rpb + threadIdx.x / G; r < rows; r += (int64_t)gridDim.x * rpb) {
        const V4<double> x = to_d(ld4(a + (size_t)r * kp + c4)), y = to_d(ld4(b + (size_t)r * kp + c4));
        s.a += x.a * y.a; s.b += x.b * y.b; s.c += x.c * y.c; s.d += x.d * y.d;
    }
    block_reduce_store4<G>(s, kp, part);
}

// CG step (cg.rs:87-94): x += alpha p, r -= alpha ap, partial ||r||^2.
template <typename T, int G>
__global__ void __launch_bounds__(kBlock) cg_xr_kernel(T* __restrict__ x, T* __restrict__ r,
                                                       const T* __restrict__ p, const T* __restrict__ ap,
                                                       const double* __restrict__ alpha, int64_t rows, int kp,
                                                       double* __restrict__ part) {
    const int c4 = (threadIdx.x & (G - 1)) * 4;
    const V4<T> al((T)alpha[c4], (T)alpha[c4 + 1], (T)alpha[c4 + 2], (T)alpha[c4 + 3]);
    V4<double> s(0.0);
    const int64_t rpb = blockDim.x / G;
    for (int64_t row = (int64_t)blockIdx.x * rpb + threadIdx.x / G; row < rows; row += (int64_t)gridDim.x * rpb) {
        const size_t e = (size_t)row * kp + c4;
        V4<T> xv = ld4(x + e), rv = ld4(r + e);
        const V4<T> pv = ld4(p + e), av = ld4(ap + e);
        xv.a += al.a * pv.a; xv.b += al.b * pv.b; xv.c += al.c * pv.c; xv.d += al.d * pv.d;
        rv.a -= al.a * av.a; rv.b -= al.b * av.b; rv.c -= al.c * av.c; rv.d -= al.d * av.d;
        st4(x + e, xv);
        st4(r + e, rv);
        s.a += (double)rv.a * rv.a; s.b += (double)rv.b * rv.b; s.c += (double)rv.c * rv.c; s.d += (double)rv.d * rv.d;
    }
    block_reduce_store4<G>(s, kp, part);
}

// p = z + beta p (cg.rs:120-124); inactive RHS keep p.
template <typename T, int G>
__global__ void __launch_bounds__(kBlock) cg_p_kernel(T* __restrict__ p, const T* __restrict__ z,
                                                      const double* __restrict__ beta,
                                                      const int32_t* __restrict__ active, int64_t rows, int kp) {
    const int c4 = (threadIdx.x & (G - 1)) * 4;
    const bool o0 = active[c4], o1 = active[c4 + 1], o2 = active[c4 + 2], o3 = active[c4 + 3];
    if (!(o0 || o1 || o2 || o3)) return;
    const V4<T> be((T)beta[c4], (T)beta[c4 + 1], (T)beta[c4 + 2], (T)beta[c4 + 3]);
    const int64_t rpb = blockDim.x / G;
    for (int64_t row = (int64_t)blockIdx.x * rpb + threadIdx.x / G; row < rows; row += (int64_t)gridDim.x * rpb) {
        const size_t e = (size_t)row * kp + c4;
        const V4<T> zv = ld4(z + e), pv = ld4(p + e);
        V4<T> o;
        o.a = o0 ? zv.a + be.a * pv.a : pv.a;
        o.b = o1 ? zv.b + be.b * pv.b : pv.b;
        o.c = o2 ? zv.c + be.c * pv.c : pv.c;
        o.d = o3 ? zv.d + be.d * pv.d : pv.d;
        st4(p + e, o);
    }
}

// ---------------------------------------------------------------------------
// Schwarz local solves over the flattened slots of a stage (block elimination,
// local_solver.rs:360-449).  With u_l = spou_l r[gidx_l] (the restriction, r-block
// sign folded into spou) and, per subdomain s of n_s slots:
//   m0 = sum_l u_l / n_s                                   (first subtract_mean)
//   red_k = u_k - m0 + sum_e C_ke invd_e (u_e - m0)        (keep rows, reduced rhs)
//   red -= mean over keep;  sol_keep = Solve(red)          (dense or AC)
//   sol_e = invd_e (u_e - m0) + invd_e sum_k C_ek sol_k     (back substitution)
//   m2 = (sum_k sol_k (1 + rho_k) + SB - m0 I) / n_s        (final subtract_mean)
//   z[gidx_l] += spou_l (sol_l - m2)
// with rho_k = sum_e C_ke invd_e, SB = sum_e u_e invd_e and I = sum_e invd_e.  Only kept
// slots are ever stored; eliminated slots are recomputed where they are needed.
// ---------------------------------------------------------------------------

// Work unit of a row-wise CSR pass: rows [row_begin, row_end) restricted to entries
// [nz_begin, nz_end); rows cut by the range are partial and add atomically.  whole: the
// chunk is exactly one complete row, so its range needs no row-pointer loads.
struct CsrChunk {
    uint32_t row_begin, row_end;
    int64_t nz_begin, nz_end;
    uint32_t whole;
};

enum CsrEpi { EPI_ACC = 0, EPI_PIVOT = 1 };

// dst[row_slot] (+)= sum_e val[e] * src[col[e]]   per RHS
//   EPI_ACC:   dst[row] += acc (partial rows atomically)
//   EPI_PIVOT: dst[row]  = dst[row] * rscale[row] + acc   (backward AC sweep; never split)
// One warp per chunk (a row, or a piece of a long row): its 32/G lane groups take the
// row's entries in turn, so a row costs one round of gathers instead of a chain of
// them (the sweeps of one AC level are latency-bound), then combine with shuffles.
// src and dst may be the same vector: a row's own slot is never among its columns'
// slots in one launch (an AC level is an independent set).
template <typename T, int G, int EPI>
__global__ void __launch_bounds__(kBlock) csr_rows_kernel(const CsrChunk* __restrict__ chunks, int64_t nchunks,
                                                          const uint32_t* __restrict__ row_slot,
                                                          const int64_t* __restrict__ ptr,
                                                          const uint32_t* __restrict__ col,
                                                          const T* __restrict__ val, const T* __restrict__ rscale,
                                                          const T* src, T* dst, int kp) {
    constexpr int NG = 32 / G;
    const int lane = threadIdx.x & 31;
    const int grp = lane / G;
    const int c4 = (lane & (G - 1)) * 4;
    const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t ch = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; ch < nchunks; ch += nw) {
        const CsrChunk C = chunks[ch];
        for (uint32_t row = C.row_begin; row < C.row_end; ++row) {
            const bool one = C.whole != 0;  // one complete row: its range is the chunk's
            const int64_t rb = one ? C.nz_begin : ptr[row], re = one ? C.nz_end : ptr[row + 1];
            const int64_t e0 = max(rb, C.nz_begin), e1 = min(re, C.nz_end);
            V4<T> acc(T(0));
            int64_t e = e0 + grp;
            for (; e + 3 * NG < e1; e += 4 * NG) {  // four independent gathers in flight
                const uint32_t j0 = __ldg(col + e), j1 = __ldg(col + e + NG);
                const uint32_t j2 = __ldg(col + e + 2 * NG), j3 = __ldg(col + e + 3 * NG);
                const T v0 = __ldg(val + e), v1 = __ldg(val + e + NG), v2 = __ldg(val + e + 2 * NG), v3 = __ldg(val + e + 3 * NG);
                const V4<T> s0 = ld4(src + (size_t)j0 * kp + c4), s1 = ld4(src + (size_t)j1 * kp + c4);
                const V4<T> s2 = ld4(src + (size_t)j2 * kp + c4), s3 = ld4(src + (size_t)j3 * kp + c4);
                acc += v0 * s0;
                acc += v1 * s1;
                acc += v2 * s2;
                acc += v3 * s3;
            }
            for (; e < e1; e += NG) acc += __ldg(val + e) * ld4(src + (size_t)__ldg(col + e) * kp + c4);
#pragma unroll
            for (int off = G; off < 32; off <<= 1) {
                acc.a += __shfl_xor_sync(0xffffffffu, acc.a, off);
                acc.b += __shfl_xor_sync(0xffffffffu, acc.b, off);
                acc.c += __shfl_xor_sync(0xffffffffu, acc.c, off);
                acc.d += __shfl_xor_sync(0xffffffffu, acc.d, off);
            }
            if (grp == 0) {
                T* d = dst + (size_t)row_slot[row] * kp + c4;
                if (EPI == EPI_ACC) {
                    if (e0 != rb || e1 != re) atomic_add4(d, acc);
                    else st4(d, ld4(d) + acc);
                } else {
                    st4(d, rscale[row] * ld4(d) + acc);
                }
            }
        }
    }
}

// L2-coherent loads and stores, for data that other blocks of the same launch write
// (an L1 line read before a grid barrier may be stale after it).
__device__ __forceinline__ V4<float> ldcg4(const float* p) {
    const float4 v = __ldcg(reinterpret_cast<const float4*>(p));
    return V4<float>(v.x, v.y, v.z, v.w);
}
__device__ __forceinline__ V4<double> ldcg4(const double* p) {
    const double2 u = __ldcg(reinterpret_cast<const double2*>(p)), v = __ldcg(reinterpret_cast<const double2*>(p) + 1);
    return V4<double>(u.x, u.y, v.x, v.y);
}
__device__ __forceinline__ void stcg4(float* p, const V4<float>& v) {
    __stcg(reinterpret_cast<float4*>(p), make_float4(v.a, v.b, v.c, v.d));
}
__device__ __forceinline__ void stcg4(double* p, const V4<double>& v) {
    __stcg(reinterpret_cast<double2*>(p), make_double2(v.a, v.b));
    __stcg(reinterpret_cast<double2*>(p) + 1, make_double2(v.c, v.d));
}

// Barrier over all blocks of a cooperative launch (every block is resident): each block
// adds one to *count and waits until it reaches `target`.  The wait is bounded; if it
// runs out, *err is set and the block goes on (the results are then invalid and the
// host reports the error).
constexpr unsigned kBarrierSpins = 1u << 22;
__device__ __forceinline__ void grid_barrier(unsigned* count, unsigned target, int* err, unsigned max_spins) {
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        atomicAdd(count, 1u);
        for (unsigned spins = 0;; ++spins) {
            unsigned c;
            asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(c) : "l"(count) : "memory");
            if (c >= target) break;
            if (spins >= max_spins) {
                atomicExch(err, 1);
                break;
            }
            __nanosleep(64);
        }
        __threadfence();
    }
    __syncthreads();
}

// One chunk of an AC level (csr_rows_kernel's work for one warp) on the vector v, read
// and written through L2: the warp's lane groups take the chunk's entries in turn, four
// gathers in flight each, and combine with shuffles; lane group 0 writes the row.
template <typename T, int G, int EPI>
__device__ __forceinline__ void level_chunk(const CsrChunk& C, const uint32_t* __restrict__ row_slot,
                                            const int64_t* __restrict__ ptr, const uint32_t* __restrict__ col,
                                            const T* __restrict__ val, const T* __restrict__ rscale, T* v, int kp,
                                            int grp, int c4) {
    constexpr int NG = 32 / G;
    for (uint32_t row = C.row_begin; row < C.row_end; ++row) {
        const bool one = C.whole != 0;  // one complete row: its range is the chunk's
        const int64_t rb = one ? C.nz_begin : ptr[row], re = one ? C.nz_end : ptr[row + 1];
        const int64_t e0 = max(rb, C.nz_begin), e1 = min(re, C.nz_end);
        V4<T> acc(T(0));
        int64_t e = e0 + grp;
        for (; e + 3 * NG < e1; e += 4 * NG) {
            const uint32_t j0 = __ldg(col + e), j1 = __ldg(col + e + NG);
            const uint32_t j2 = __ldg(col + e + 2 * NG), j3 = __ldg(col + e + 3 * NG);
            const T v0 = __ldg(val + e), v1 = __ldg(val + e + NG), v2 = __ldg(val + e + 2 * NG), v3 = __ldg(val + e + 3 * NG);
            const V4<T> s0 = ldcg4(v + (size_t)j0 * kp + c4), s1 = ldcg4(v + (size_t)j1 * kp + c4);
            const V4<T> s2 = ldcg4(v + (size_t)j2 * kp + c4), s3 = ldcg4(v + (size_t)j3 * kp + c4);
            acc += v0 * s0;
            acc += v1 * s1;
            acc += v2 * s2;
            acc += v3 * s3;
        }
        for (; e < e1; e += NG) acc += __ldg(val + e) * ldcg4(v + (size_t)__ldg(col + e) * kp + c4);
#pragma unroll
        for (int off = G; off < 32; off <<= 1) {
            acc.a += __shfl_xor_sync(0xffffffffu, acc.a, off);
            acc.b += __shfl_xor_sync(0xffffffffu, acc.b, off);
            acc.c += __shfl_xor_sync(0xffffffffu, acc.c, off);
            acc.d += __shfl_xor_sync(0xffffffffu, acc.d, off);
        }
        if (grp == 0) {
            T* d = v + (size_t)row_slot[row] * kp + c4;
            if (EPI == EPI_ACC) {
                if (e0 != rb || e1 != re) atomic_add4(d, acc);
                else stcg4(d, ldcg4(d) + acc);
            } else {
                stcg4(d, rscale[row] * ldcg4(d) + acc);
            }
        }
    }
}

// Levels lev0 .. lev0 + nlev - 1 of one AC sweep direction in one cooperative launch:
// level l's chunks are [lp[l], lp[l+1]); levels run in order (backward: from the last),
// separated by grid barriers.
template <typename T, int G, int EPI>
__global__ void __launch_bounds__(kBlock) csr_levels_kernel(const CsrChunk* __restrict__ chunks,
                                                            const int64_t* __restrict__ lp, int lev0, int nlev,
                                                            int backward, const uint32_t* __restrict__ row_slot,
                                                            const int64_t* __restrict__ ptr,
                                                            const uint32_t* __restrict__ col,
                                                            const T* __restrict__ val, const T* __restrict__ rscale,
                                                            T* v, int kp, unsigned* bar, int* err,
                                                            unsigned target_extra, unsigned max_spins) {
    const int lane = threadIdx.x & 31;
    const int grp = lane / G;
    const int c4 = (lane & (G - 1)) * 4;
    const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
    const int64_t wid = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    for (int li = 0; li < nlev; ++li) {
        const int l = lev0 + (backward ? nlev - 1 - li : li);
        for (int64_t ch = lp[l] + wid; ch < lp[l + 1]; ch += nw)
            level_chunk<T, G, EPI>(chunks[ch], row_slot, ptr, col, val, rscale, v, kp, grp, c4);
        if (li + 1 < nlev) grid_barrier(bar, (unsigned)(li + 1) * gridDim.x + target_extra, err, max_spins);
    }
}

// The small levels lev0 .. lev0 + nlev - 1 of a sweep direction (a few thousand rows or
// fewer each: the last levels of an AC factor) in one thread-block cluster, separated by
// the cluster's hardware barrier (release/acquire at cluster scope; v is read and written
// through L2) instead of a barrier across the whole grid.  Launched as exactly one
// cluster of gridDim.x blocks.
constexpr int kLevelClusterBlock = 1024;

template <typename T, int G, int EPI>
__global__ void __launch_bounds__(kLevelClusterBlock, 1)
    csr_levels_cluster_kernel(const CsrChunk* __restrict__ chunks, const int64_t* __restrict__ lp, int lev0,
                              int nlev, int backward, const uint32_t* __restrict__ row_slot,
                              const int64_t* __restrict__ ptr, const uint32_t* __restrict__ col,
                              const T* __restrict__ val, const T* __restrict__ rscale, T* v, int kp) {
    const int lane = threadIdx.x & 31;
    const int grp = lane / G;
    const int c4 = (lane & (G - 1)) * 4;
    const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
    const int64_t wid = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    for (int li = 0; li < nlev; ++li) {
        const int l = lev0 + (backward ? nlev - 1 - li : li);
        for (int64_t ch = lp[l] + wid; ch < lp[l + 1]; ch += nw)
            level_chunk<T, G, EPI>(chunks[ch], row_slot, ptr, col, val, rscale, v, kp, grp, c4);
        if (li + 1 < nlev) {
            asm volatile("barrier.cluster.arrive.release.aligned;" ::: "memory");
            asm volatile("barrier.cluster.wait.acquire.aligned;" ::: "memory");
        }
    }
}

// Segmented per-subdomain sums over a contiguous range, block-reduced: the block's
// first and last subdomain accumulate in shared memory (one global atomic per block),
// other runs (small subdomains inside the block) go straight to global atomics.
struct SegSum {
    double* sm;  // [2 bins][2 quantities][kp]
    uint32_t first, last;
    int kp;
    __device__ void flush(double* g0, double* g1, uint32_t sub, const V4<double>& a, const V4<double>& b, int c4) {
        const int bin = sub == first ? 0 : (sub == last ? 1 : -1);
        if (bin >= 0) {
            double* s = sm + (size_t)bin * 2 * kp + c4;
            atomic_add4(s, a);
            if (g1) atomic_add4(s + kp, b);
        } else {
            atomic_add4(g0 + (size_t)sub * kp + c4, a);
            if (g1) atomic_add4(g1 + (size_t)sub * kp + c4, b);
        }
    }
    __device__ void finish(double* g0, double* g1, bool skip_first = false) {
        __syncthreads();
        for (int i = threadIdx.x; i < 2 * kp; i += blockDim.x) {
            const int bin = i / kp, c = i % kp;
            if (bin == 1 && last == first) continue;
            if (bin == 0 && skip_first) continue;
            const uint32_t sub = bin == 0 ? first : last;
            atomicAdd(g0 + (size_t)sub * kp + c, sm[bin * 2 * kp + c]);
            if (g1) atomicAdd(g1 + (size_t)sub * kp + c, sm[bin * 2 * kp + kp + c]);
        }
    }
};

// Sum of a V4 over the lane groups of a warp (lanes with equal lane % G).
template <int G>
__device__ __forceinline__ V4<double> warp_sum_groups(V4<double> v) {
#pragma unroll
    for (int off = G; off < 32; off <<= 1) {
        v.a += __shfl_xor_sync(0xffffffffu, v.a, off);
        v.b += __shfl_xor_sync(0xffffffffu, v.b, off);
        v.c += __shfl_xor_sync(0xffffffffu, v.c, off);
        v.d += __shfl_xor_sync(0xffffffffu, v.d, off);
    }
    return v;
}

// Pass 1 (all slots): S0[s] += u_l, SB[s] += u_l invd_l.  Block b owns slots
// [b*spb, +spb), a lane group spb/(groups) consecutive slots, four loads at a time.
// Subdomains are long runs of slots, so nearly everything belongs to the block's first
// subdomain: that part is summed in registers, then over the block with shuffles (one
// set of global atomics per block); other runs go through SegSum.
template <typename T, int G>
__global__ void __launch_bounds__(kBlock) schwarz_sums_kernel(int64_t nslots, int spb,
                                                              const uint32_t* __restrict__ gidx,
                                                              const T* __restrict__ spou, const T* __restrict__ invd,
                                                              const uint32_t* __restrict__ sub_of,
                                                              const T* __restrict__ r, int kp,
                                                              double* __restrict__ S0, double* __restrict__ SB) {
    __shared__ double sm[2 * 2 * 32];
    __shared__ double wsum[2][kBlock / 32][32];
    const int c4 = (threadIdx.x & (G - 1)) * 4;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int64_t b0 = (int64_t)blockIdx.x * spb, b1 = min(nslots, b0 + spb);
    if (b0 >= nslots) return;  // uniform per block
    for (int i = threadIdx.x; i < 4 * kp; i += blockDim.x) sm[i] = 0.0;
    SegSum seg{sm, sub_of[b0], sub_of[b1 - 1], kp};
    __syncthreads();
    const int gpb = blockDim.x / G, g = threadIdx.x / G;
    const int64_t per = (spb + gpb - 1) / gpb;
    const int64_t a0 = b0 + g * per, a1 = min(b1, a0 + per);
    uint32_t cur = 0xffffffffu;
    V4<double> acc0(0.0), accb(0.0), f0(0.0), fb(0.0);
    auto close = [&]() {
        if (cur == seg.first) {
            f0 += acc0;
            fb += accb;
        } else if (cur != 0xffffffffu) {
            seg.flush(S0, SB, cur, acc0, accb, c4);
        }
    };
    for (int64_t l = a0; l < a1; l += 4) {
        const int nb = (int)min((int64_t)4, a1 - l);
        uint32_t sbv[4], gv[4];
        T spv[4], iv[4];
        V4<T> rv[4];
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            if (j < nb) {
                sbv[j] = sub_of[l + j];
                gv[j] = gidx[l + j];
                spv[j] = spou[l + j];
                iv[j] = invd[l + j];
            }
        }
#pragma unroll
        for (int j = 0; j < 4; ++j)
            if (j < nb) rv[j] = ld4(r + (size_t)gv[j] * kp + c4);
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            if (j >= nb) break;
            if (sbv[j] != cur) {
                close();
                cur = sbv[j];
                acc0 = V4<double>(0.0);
                accb = V4<double>(0.0);
            }
            const V4<double> u = (double)spv[j] * to_d(rv[j]);
            acc0 += u;
            accb += (double)iv[j] * u;
        }
    }
    close();
    f0 = warp_sum_groups<G>(f0);
    fb = warp_sum_groups<G>(fb);
    if (lane < G) {
        wsum[0][warp][c4] = f0.a; wsum[0][warp][c4 + 1] = f0.b; wsum[0][warp][c4 + 2] = f0.c; wsum[0][warp][c4 + 3] = f0.d;
        wsum[1][warp][c4] = fb.a; wsum[1][warp][c4 + 1] = fb.b; wsum[1][warp][c4 + 2] = fb.c; wsum[1][warp][c4 + 3] = fb.d;
    }
    __syncthreads();
    for (int i = threadIdx.x; i < 2 * kp; i += blockDim.x) {
        const int q = i / kp, c = i % kp;
        double s = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += wsum[q][w][c];
        atomicAdd((q ? SB : S0) + (size_t)seg.first * kp + c, s);
    }
    seg.finish(S0, SB, /*skip_first=*/true);
}

// Keep slots, in keep-list order: v[k] = u_k - m0 - m0 rho_k (the base of the reduced rhs).
template <typename T, int G>
__global__ void __launch_bounds__(kBlock) keep_init_kernel(int64_t nkeep, const uint32_t* __restrict__ keep_slots,
                                                           const uint32_t* __restrict__ gidx, const T* __restrict__ spou,
                                                           const T* __restrict__ rho, const uint32_t* __restrict__ sub_of,
                                                           const int32_t* __restrict__ sub_n,
                                                           const double* __restrict__ S0, const T* __restrict__ r,
                                                           T* __restrict__ v, int kp) {
    const int c4 = (threadIdx.x & (G - 1)) * 4;
    const int64_t rpb = blockDim.x / G;
    for (int64_t a = (int64_t)blockIdx.x * rpb + threadIdx.x / G; a < nkeep; a += (int64_t)gridDim.x * rpb) {
        const uint32_t l = keep_slots[a];
        const uint32_t s = sub_of[l];
        const double inv_n = 1.0 / (double)sub_n[s];
        const size_t o = (size_t)s * kp + c4;
        const V4<double> m0 = inv_n * V4<double>(S0[o], S0[o + 1], S0[o + 2], S0[o + 3]);
        const V4<double> u = (double)spou[l] * to_d(ld4(r + (size_t)gidx[l] * kp + c4));
        st4(v + (size_t)l * kp + c4, from_d<T>(u - m0 - (double)rho[a] * m0));
    }
}

// Keep-list segmented sums: M[s] += v[k] * (1 + rho_k if with_rho), block-reduced.
template <typename T, int G>
__global__ void __launch_bounds__(kBlock) keep_sum_kernel(int64_t nkeep, int spb, const uint32_t* __restrict__ keep_slots,
                                                          const T* __restrict__ rho, int with_rho,
                                                          const uint32_t* __restrict__ sub_of,
                                                          const T* __restrict__ v, int kp, double* __restrict__ M) {
    __shared__ double sm[2 * 2 * 32];
    const int c4 = (threadIdx.x & (G - 1)) * 4;
    const int64_t b0 = (int64_t)blockIdx.x * spb, b1 = min(nkeep, b0 + spb);
    if (b0 >= nkeep) return;  // uniform per block
    for (int i = threadIdx.x; i < 4 * kp; i += blockDim.x) sm[i] = 0.0;
    SegSum seg{sm, sub_of[keep_slots[b0]], sub_of[keep_slots[b1 - 1]], kp};
    __syncthreads();
    const int gpb = blockDim.x / G, g = threadIdx.x / G;
    const int64_t per = (spb + gpb - 1) / gpb;
    const int64_t a0 = b0 + g * per, a1 = min(b1, a0 + per);
    uint32_t cur = 0xffffffffu;
    V4<double> acc(0.0);
    for (int64_t a = a0; a < a1; ++a) {
        const uint32_t l = keep_slots[a];
        const uint32_t sb = sub_of[l];
        if (sb != cur) {
            if (cur != 0xffffffffu) seg.flush(M, nullptr, cur, acc, acc, c4);
            cur = sb;
            acc = V4<double>(0.0);
        }
        const double f = with_rho ? 1.0 + (double)rho[a] : 1.0;
        acc += f * to_d(ld4(v + (size_t)l * kp + c4));
    }
    if (cur != 0xffffffffu) seg.flush(M, nullptr, cur, acc, acc, c4);
    seg.finish(M, nullptr);
}

// v[k] -= M1[s] / n_keep[s] over the keep list.
template <typename T, int G>
__global__ void __launch_bounds__(kBlock) keep_center_kernel(int64_t nkeep, const uint32_t* __restrict__ keep_slots,
                                                             const uint32_t* __restrict__ sub_of,
                                                             const int32_t* __restrict__ sub_nkeep,
                                                             const double* __restrict__ M1, T* __restrict__ v, int kp) {
    const int c4 = (threadIdx.x & (G - 1)) * 4;
    const int64_t rpb = blockDim.x / G;
    for (int64_t a = (int64_t)blockIdx.x * rpb + threadIdx.x / G; a < nkeep; a += (int64_t)gridDim.x * rpb) {
        const uint32_t l = keep_slots[a];
        const uint32_t s = sub_of[l];
        const double inv = 1.0 / (double)sub_nkeep[s];
        const size_t o = (size_t)s * kp + c4;
        const V4<double> m(M1[o] * inv, M1[o + 1] * inv, M1[o + 2] * inv, M1[o + 3] * inv);
        T* p = v + (size_t)l * kp + c4;
        st4(p, from_d<T>(to_d(ld4(p)) - m));
    }
}

// Solution of slot l of a stage: kept slots read v; eliminated slots back-substitute
// from the kept solution (sol_e = invd_e (u_e - m0) + invd_e sum_k C_ek v_k).
template <typename T>
__device__ __forceinline__ V4<double> slot_solution(uint32_t l, const V4<double>& u, const V4<double>& m0, T invd,
                                                    const int64_t* __restrict__ bs_ptr,
                                                    const uint32_t* __restrict__ bs_col,
                                                    const T* __restrict__ bs_val, const T* __restrict__ v, int kp,
                                                    int c4) {
    if (invd == T(0)) return to_d(ld4(v + (size_t)l * kp + c4));
    V4<T> acc(T(0));
    const int64_t e0 = bs_ptr[l], e1 = bs_ptr[l + 1];
    int64_t e = e0;
    for (; e + 2 <= e1; e += 2) {
        const uint32_t j0 = __ldg(bs_col + e), j1 = __ldg(bs_col + e + 1);
        const T v0 = __ldg(bs_val + e), v1 = __ldg(bs_val + e + 1);
        const V4<T> s0 = ld4(v + (size_t)j0 * kp + c4), s1 = ld4(v + (size_t)j1 * kp + c4);
        acc += v0 * s0;
        acc += v1 * s1;
    }
    if (e < e1) acc += __ldg(bs_val + e) * ld4(v + (size_t)__ldg(bs_col + e) * kp + c4);
    const double id = (double)invd;
    return id * (u - m0) + id * to_d(acc);
}

struct SubMeans {
    const int32_t* sub_n;
    const double *S0, *SB, *M2, *I;
};
__device__ __forceinline__ void sub_means(const SubMeans& M, uint32_t s, int kp, int c4, V4<double>& m0, V4<double>& m2) {
    const double inv = 1.0 / (double)M.sub_n[s];
    const double I = M.I[s];
    const size_t o = (size_t)s * kp + c4;
    m0 = V4<double>(M.S0[o], M.S0[o + 1], M.S0[o + 2], M.S0[o + 3]);
    m0 *= inv;
    const V4<double> sb(M.SB[o], M.SB[o + 1], M.SB[o + 2], M.SB[o + 3]);
    const V4<double> k2(M.M2[o], M.M2[o + 1], M.M2[o + 2], M.M2[o + 3]);
    m2 = inv * (k2 + sb - I * m0);
}

// Per-subdomain means once per apply: mm[s][0] = m0 = S0/n, mm[s][1] = m2.
static __global__ void sub_means_kernel(int32_t nsub, int kp, SubMeans M, double* __restrict__ mm) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (int64_t)nsub * kp) return;
    const int64_t s = i / kp, c = i % kp;
    const double inv = 1.0 / (double)M.sub_n[s];
    const double m0 = M.S0[i] * inv;
    mm[(s * 2) * kp + c] = m0;
    mm[(s * 2 + 1) * kp + c] = inv * (M.M2[i] + M.SB[i] - M.I[s] * m0);
}

// Additive prolongation as a gather over global dofs (no atomics), with the back
// substitution of eliminated slots folded in: z[j] = sum_{slots l of j} spou_l (sol_l - m2),
// sol_e = invd_e (spou_e r_j - m0) + invd_e sum_k C_ek v_k on eliminated slots, v_l on
// kept ones.  The slot data and back-substitution rows are read in gather order, so a
// dof's loads depend only on gptr[j].  Dofs in no subdomain get z = 0.  Optionally the
// partial dot r.z for CG.
template <typename T, int G>
__global__ void __launch_bounds__(kBlock, 4) prolong_kernel(int64_t m, const int64_t* __restrict__ gptr,
                                                         const uint32_t* __restrict__ gslot,
                                                         const uint32_t* __restrict__ gsub,
                                                         const T* __restrict__ gspou, const T* __restrict__ ginvd,
                                                         const int64_t* __restrict__ gbs_ptr,
                                                         const uint32_t* __restrict__ gbs_cnt,
                                                         const uint32_t* __restrict__ gbs_col,
                                                         const T* __restrict__ gbs_val, const double* __restrict__ mm,
                                                         const T* __restrict__ v, const T* __restrict__ r,
                                                         T* __restrict__ z, int kp, double* __restrict__ part,
                                                         const int32_t* __restrict__ failed) {
    const int c4 = (threadIdx.x & (G - 1)) * 4;
    V4<double> dotp(0.0);
    // a local solve that did not complete (an AC sweep's barrier wait ran out): z is NaN
    // everywhere, as the reference's apply fills it (schwarz-precond additive/
    // preconditioner.rs:197-201)
    const bool nan_out = failed != nullptr && *failed != 0;
    const int64_t rpb = blockDim.x / G;
    for (int64_t j = (int64_t)blockIdx.x * rpb + threadIdx.x / G; j < m; j += (int64_t)gridDim.x * rpb) {
        const V4<double> rj = to_d(ld4(r + (size_t)j * kp + c4));
        V4<double> acc(0.0);
        const int64_t e0 = gptr[j], e1 = gptr[j + 1];
        for (int64_t e = e0; e < e1; ++e) {
            const uint32_t s = gsub[e];
            const double sp = (double)gspou[e];
            const T id = ginvd[e];
            V4<double> sol;
            if (id == T(0)) {
                sol = to_d(ld4(v + (size_t)gslot[e] * kp + c4));
            } else {
                V4<T> bs(T(0)), bs2(T(0));
                // the row starts at a multiple of 4 entries and is padded to one (repeats of
                // its first column with value 0): one 16-byte load of 4 columns and one of 4
                // values, then four independent gathers in flight
                const int64_t t0 = gbs_ptr[e], t1 = t0 + gbs_cnt[e];
                for (int64_t t = t0; t < t1; t += 4) {
                    const uint4 jj = __ldg(reinterpret_cast<const uint4*>(gbs_col + t));
                    const V4<T> vv = ldg4(gbs_val + t);
                    const V4<T> s0 = ld4(v + (size_t)jj.x * kp + c4), s1 = ld4(v + (size_t)jj.y * kp + c4);
                    const V4<T> s2 = ld4(v + (size_t)jj.z * kp + c4), s3 = ld4(v + (size_t)jj.w * kp + c4);
                    bs += vv.a * s0;
                    bs2 += vv.b * s1;
                    bs += vv.c * s2;
                    bs2 += vv.d * s3;
                }
                bs += bs2;
                const double idd = (double)id;
                const V4<double> m0 = ld4(mm + (size_t)(2 * s) * kp + c4);
                sol = idd * (sp * rj - m0) + idd * to_d(bs);
            }
            const V4<double> m2 = ld4(mm + (size_t)(2 * s + 1) * kp + c4);
            acc += sp * (sol - m2);
        }
        const V4<T> zt = nan_out ? V4<T>(quiet_nan<T>()) : from_d<T>(acc);
        st4(z + (size_t)j * kp + c4, zt);
        const V4<double> zd = to_d(zt);
        dotp.a += rj.a * zd.a; dotp.b += rj.b * zd.b; dotp.c += rj.c * zd.c; dotp.d += rj.d * zd.d;
    }
    if (part) block_reduce_store4<G>(dotp, kp, part);
}

// Multiplicative stage, part 1: c_l = spou_l (sol_l - m2); z[gidx_l] += c_l and
// cneg[gidx_l] = -c_l (dofs are unique within one factor-pair stage; cneg is zero
// elsewhere).  Part 2 is r_work += G cneg, the assembled Gramian's rows as a CSR SpMV
// (residual_update.rs:36-53 restricted to the touched columns, which cneg selects).
template <typename T, int G>
__global__ void __launch_bounds__(kBlock) mult_sol_kernel(int64_t nslots, const uint32_t* __restrict__ gidx,
                                                          const uint32_t* __restrict__ sub_of,
                                                          const T* __restrict__ spou, const T* __restrict__ invd,
                                                          const int64_t* __restrict__ bs_ptr,
                                                          const uint32_t* __restrict__ bs_col,
                                                          const T* __restrict__ bs_val, SubMeans M,
                                                          const T* __restrict__ v, const T* __restrict__ rw,
                                                          T* __restrict__ z, T* __restrict__ cneg, int kp) {
    const int c4 = (threadIdx.x & (G - 1)) * 4;
    const int64_t rpb = blockDim.x / G;
    for (int64_t l = (int64_t)blockIdx.x * rpb + threadIdx.x / G; l < nslots; l += (int64_t)gridDim.x * rpb) {
        const uint32_t g = gidx[l];
        const uint32_t s = sub_of[l];
        V4<double> m0, m2;
        sub_means(M, s, kp, c4, m0, m2);
        const double sp = (double)spou[l];
        const V4<double> u = sp * to_d(ld4(rw + (size_t)g * kp + c4));
        const V4<double> sol = slot_solution<T>((uint32_t)l, u, m0, invd[l], bs_ptr, bs_col, bs_val, v, kp, c4);
        const V4<T> cl = from_d<T>(sp * (sol - m2));
        st4(cneg + (size_t)g * kp + c4, V4<T>(-cl.a, -cl.b, -cl.c, -cl.d));
        T* zp = z + (size_t)g * kp + c4;
        st4(zp, ld4(zp) + cl);
    }
}

// Anchored dense Cholesky solves (AnchoredDenseCholesky::solve_in_place,
// local_solver.rs:252-299): one warp per (dense subdomain, RHS).  For m <= 32 lane i
// keeps row i in a register; larger minors are swept in place in v.
template <typename T>
__global__ void dense_solve_kernel(int32_t ndense, const int64_t* __restrict__ keep0,
                                   const int32_t* __restrict__ nkeep, const int64_t* __restrict__ loff,
                                   const T* __restrict__ L, T* __restrict__ v, int kp) {
    const int warp = (int)(((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    const int lane = threadIdx.x & 31;
    if (warp >= ndense * kp) return;  // uniform per warp
    const int d = warp / kp, c = warp % kp;
    const int n = nkeep[d];
    const int64_t s0 = keep0[d];
    if (n == 0) return;
    if (n == 1) {
        if (lane == 0) v[(size_t)s0 * kp + c] = T(0);
        return;
    }
    const int m = n - 1;
    const T* Ld = L + loff[d];
    if (m <= 32) {
        T xi = (lane < m) ? v[(size_t)(s0 + lane) * kp + c] : T(0);
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
        if (lane < m) v[(size_t)(s0 + lane) * kp + c] = xi;
    } else {
        T* x = v + (size_t)s0 * kp + c;  // element i at x[i*kp]
        for (int j = 0; j < m; ++j) {
            const T xj = x[(size_t)j * kp] / Ld[(size_t)j * m + j];
            __syncwarp();
            if (lane == 0) x[(size_t)j * kp] = xj;
            for (int i = j + 1 + lane; i < m; i += 32) x[(size_t)i * kp] -= Ld[(size_t)i * m + j] * xj;
            __syncwarp();
        }
        for (int j = m - 1; j >= 0; --j) {
            const T xj = x[(size_t)j * kp] / Ld[(size_t)j * m + j];
            __syncwarp();
            if (lane == 0) x[(size_t)j * kp] = xj;
            for (int i = lane; i < j; i += 32) x[(size_t)i * kp] -= Ld[(size_t)j * m + i] * xj;
            __syncwarp();
        }
    }
    if (lane == 0) v[(size_t)(s0 + m) * kp + c] = T(0);
}

// Dense core of an AC factor: v[core] = Z v[core] (anchored inverse).  First the core
// rows of v are copied to a contiguous buffer (core_stage_kernel), then each block
// computes kCoreRowsPerBlock output rows with four warps per row: a warp takes a
// quarter of the row's columns, its lane groups (4 RHS per lane) take the columns in
// turn with four loads in flight, and the partial sums combine with shuffles and
// shared memory before the row is written back into v.
template <typename T>
__global__ void core_stage_kernel(int64_t total, const uint32_t* __restrict__ core_slot, const T* __restrict__ v,
                                  T* __restrict__ cin, int kp) {
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total * kp; e += (int64_t)gridDim.x * blockDim.x)
        cin[e] = v[(size_t)core_slot[e / kp] * kp + e % kp];
}

template <typename T, int G>
__global__ void __launch_bounds__(kBlock) core_gemv_kernel(const int32_t* __restrict__ core_of_block,
                                                           const int32_t* __restrict__ row0_of_block,
                                                           const int32_t* __restrict__ core_n,
                                                           const int64_t* __restrict__ core_slot_off,
                                                           const uint32_t* __restrict__ core_slot,
                                                           const int64_t* __restrict__ core_z_off,
                                                           const T* __restrict__ Z, const T* __restrict__ cin,
                                                           T* __restrict__ v, int kp) {
    constexpr int NG = 32 / G;
    constexpr int kParts = 4;  // warps per row
    __shared__ T part[kBlock / 32][32];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int grp = lane / G, c4 = (lane & (G - 1)) * 4;
    const int g = core_of_block[blockIdx.x];
    const int r = core_n[g];
    const int64_t off = core_slot_off[g];
    const int row = row0_of_block[blockIdx.x] + warp / kParts;
    V4<T> acc(T(0)), acc2(T(0));
    if (row < r) {
        const T* zr = Z + core_z_off[g] + (size_t)row * r;
        const T* x = cin + (size_t)off * kp + c4;
        const int q = warp % kParts;
        const int b0 = (int)((int64_t)r * q / kParts), b1 = (int)((int64_t)r * (q + 1) / kParts);
        int b = b0 + grp;
        for (; b + 3 * NG < b1; b += 4 * NG) {
            const T z0 = __ldg(zr + b), z1 = __ldg(zr + b + NG), z2 = __ldg(zr + b + 2 * NG), z3 = __ldg(zr + b + 3 * NG);
            const V4<T> s0 = ldg4(x + (size_t)b * kp), s1 = ldg4(x + (size_t)(b + NG) * kp);
            const V4<T> s2 = ldg4(x + (size_t)(b + 2 * NG) * kp), s3 = ldg4(x + (size_t)(b + 3 * NG) * kp);
            acc += z0 * s0;
            acc2 += z1 * s1;
            acc += z2 * s2;
            acc2 += z3 * s3;
        }
        for (; b < b1; b += NG) acc += __ldg(zr + b) * ldg4(x + (size_t)b * kp);
    }
    acc += acc2;
#pragma unroll
    for (int o = G; o < 32; o <<= 1) {
        acc.a += __shfl_xor_sync(0xffffffffu, acc.a, o);
        acc.b += __shfl_xor_sync(0xffffffffu, acc.b, o);
        acc.c += __shfl_xor_sync(0xffffffffu, acc.c, o);
        acc.d += __shfl_xor_sync(0xffffffffu, acc.d, o);
    }
    if (lane < G) {
        part[warp][c4] = acc.a; part[warp][c4 + 1] = acc.b; part[warp][c4 + 2] = acc.c; part[warp][c4 + 3] = acc.d;
    }
    __syncthreads();
    const int rows_here = kBlock / 32 / kParts;
    for (int t = threadIdx.x; t < rows_here * kp; t += blockDim.x) {
        const int rr = t / kp, c = t % kp;
        const int orow = row0_of_block[blockIdx.x] + rr;
        if (orow >= r) continue;
        T s = T(0);
#pragma unroll
        for (int w = 0; w < kParts; ++w) s += part[rr * kParts + w][c];
        v[(size_t)core_slot[off + orow] * kp + c] = s;
    }
}

}  // namespace wb
