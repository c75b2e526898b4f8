// Solver of the B200-native solve phase: device layout, Schwarz/Krylov drivers and
// the C ABI declared in include/within_b200.h.  Reference citations are relative to
// the reference's crates/ directory.
#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <chrono>
#include <cfloat>
#include <cmath>
#include <cstring>
#include <functional>
#include <future>
#include <map>
#include <memory>
#include <mutex>
#include <thread>
#include <atomic>
#include <numeric>
#include <string>
#include <tuple>
#include <type_traits>
#include <unordered_map>
#include <vector>

#include "../../include/within_b200.h"
#include "device.cuh"
#include "obs_launch.cuh"
#include "kernels.cuh"
#include "coarse.cuh"
#include "setup.hpp"

namespace wb {

namespace {
thread_local std::string g_last_error;

int fail(int code, const std::string& msg) {
    g_last_error = msg;
    return code;
}

int pad4(int k) { return (k + 3) & ~3; }

double now_s() {
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

// Balanced chunks of a row-wise CSR: at most max_rows rows / max_nz entries each;
// rows longer than max_nz are cut into pieces when allow_split.
std::vector<CsrChunk> make_chunks(const std::vector<int64_t>& ptr, int64_t row_lo, int64_t row_hi,
                                  int64_t max_nz, int64_t max_rows, bool allow_split) {
    std::vector<CsrChunk> out;
    int64_t r = row_lo;
    while (r < row_hi) {
        const int64_t len = ptr[r + 1] - ptr[r];
        if (allow_split && len > max_nz) {
            for (int64_t a = ptr[r]; a < ptr[r + 1]; a += max_nz)
                out.push_back(CsrChunk{(uint32_t)r, (uint32_t)(r + 1), a, std::min(a + max_nz, ptr[r + 1]), 0u});
            ++r;
            continue;
        }
        int64_t r1 = r + 1;
        while (r1 < row_hi && r1 - r < max_rows && ptr[r1 + 1] - ptr[r] <= max_nz &&
               !(allow_split && ptr[r1 + 1] - ptr[r1] > max_nz))
            ++r1;
        out.push_back(CsrChunk{(uint32_t)r, (uint32_t)r1, ptr[r], ptr[r1], r1 == r + 1 ? 1u : 0u});
        r = r1;
    }
    return out;
}

// Flatten the subdomains `ids` into one stage (see StageHost and kernels.cuh).  The
// per-slot arrays, the keep rows and the back-substitution rows are sized first and then
// filled in parallel over ranges of slots and rows (every range writes its own part, with
// the same arithmetic as a sequential fill); the dense and AC factors follow in order.
StageHost build_stage(const std::vector<Subdomain>& subs, const std::vector<int32_t>& ids, int64_t ndofs,
                      bool with_gather) {
    StageHost st;
    st.nsub = (int32_t)ids.size();
    const int32_t ns = st.nsub;
    std::vector<int32_t> ac_subs;  // stage-local indices of the AC subdomains, in order
    int32_t max_lev = 0;
    // offsets per subdomain: slots, keep rows, keep entries, back-substitution entries
    std::vector<int64_t> so(ns + 1, 0), kro(ns + 1, 0), kno(ns + 1, 0), bno(ns + 1, 0);
    auto k2e_of = [&](const Subdomain& sd) -> const Csr& { return sd.elim_q ? sd.ct.ct : sd.ct.c; };
    auto e2k_of = [&](const Subdomain& sd) -> const Csr& { return sd.elim_q ? sd.ct.c : sd.ct.ct; };
    for (int32_t si = 0; si < ns; ++si) {
        const Subdomain& sd = subs[ids[si]];
        so[si + 1] = so[si] + sd.n_local();
        kro[si + 1] = kro[si] + (sd.elim_q ? sd.n_r() : sd.n_q());
        kno[si + 1] = kno[si] + k2e_of(sd).nnz();
        bno[si + 1] = bno[si] + e2k_of(sd).nnz();
    }
    const int64_t nslots = so[ns], nkeep = kro[ns];
    st.sub_nloc.resize(ns);
    st.sub_nkeep.resize(ns);
    st.sub_I.resize(ns);
    st.gidx.resize(nslots);
    st.sub_of.resize(nslots);
    st.spou.resize(nslots);
    st.invd.assign(nslots, 0.0);
    st.keep_slots.resize(nkeep);
    st.keep.row_slot.resize(nkeep);
    st.keep.rscale.assign(nkeep, 1.0);
    st.rho.resize(nkeep);
    st.keep.ptr.assign(nkeep + 1, 0);
    st.keep.col.resize(kno[ns]);
    st.keep.val.resize(kno[ns]);
    st.bs_ptr.assign(nslots + 1, 0);
    st.bs_col.resize(bno[ns]);
    st.bs_val.resize(bno[ns]);
    // tasks: (subdomain, kind 0 = slots / 1 = keep rows, begin, end)
    struct Task { int32_t si, kind; int64_t b, e; };
    std::vector<Task> tasks;
    constexpr int64_t kSlotsPerTask = 1 << 16, kEntriesPerTask = 1 << 18;
    for (int32_t si = 0; si < ns; ++si) {
        const Subdomain& sd = subs[ids[si]];
        const int64_t nl = sd.n_local();
        for (int64_t b0 = 0; b0 < nl; b0 += kSlotsPerTask) tasks.push_back({si, 0, b0, std::min(nl, b0 + kSlotsPerTask)});
        const Csr& k2e = k2e_of(sd);
        int64_t r0 = 0;
        for (int64_t r = 0; r < k2e.nrows; ++r)
            if ((int64_t)k2e.ptr[r + 1] - (int64_t)k2e.ptr[r0] >= kEntriesPerTask || r + 1 == k2e.nrows) {
                tasks.push_back({si, 1, r0, r + 1});
                r0 = r + 1;
            }
    }
    parallel_tasks(tasks.size(), [&](size_t t) {
        const Task& T = tasks[t];
        const Subdomain& sd = subs[ids[T.si]];
        const int32_t nq = sd.n_q();
        const int64_t o = so[T.si];
        const int64_t keep0 = o + (sd.elim_q ? nq : 0), elim0 = o + (sd.elim_q ? 0 : nq);
        const int64_t le0 = elim0 - o;  // first eliminated slot, local
        const int32_t n_elim = sd.elim_q ? nq : sd.n_r();
        auto spou_of = [&](int64_t a) {  // r-block sign flip (local_solver.rs:83-87, 362, 447)
            const double pw = sd.pou.empty() ? 1.0 : sd.pou[a];
            return a < nq ? pw : -pw;
        };
        if (T.kind == 0) {
            const Csr& e2k = e2k_of(sd);
            for (int64_t a = T.b; a < T.e; ++a) {
                const int64_t l = o + a;
                st.gidx[l] = sd.gidx[a];
                st.sub_of[l] = (uint32_t)T.si;
                st.spou[l] = spou_of(a);
                // back substitution rows over all slots of the subdomain (local_solver.rs:111-151)
                int64_t end = 0;
                if (a >= le0 && a < le0 + n_elim) {
                    const int64_t e = a - le0;
                    st.invd[l] = sd.inv_diag[e];
                    for (uint32_t x = e2k.ptr[e]; x < e2k.ptr[e + 1]; ++x) {
                        st.bs_col[bno[T.si] + x] = (uint32_t)(keep0 + e2k.idx[x]);
                        st.bs_val[bno[T.si] + x] = e2k.val[x];
                    }
                    end = e2k.ptr[e + 1];
                } else {
                    end = a < le0 ? 0 : e2k.nnz();
                }
                st.bs_ptr[l + 1] = bno[T.si] + end;
            }
        } else {
            // reduced rhs rows (local_solver.rs:374-381, 410-417), premultiplied by the restriction
            const Csr& k2e = k2e_of(sd);
            for (int64_t i = T.b; i < T.e; ++i) {
                const int64_t row = kro[T.si] + i;
                st.keep_slots[row] = (uint32_t)(keep0 + i);
                st.keep.row_slot[row] = (uint32_t)(keep0 + i);
                double rho = 0.0;
                for (uint32_t e = k2e.ptr[i]; e < k2e.ptr[i + 1]; ++e) {
                    const int64_t a = le0 + k2e.idx[e];
                    const double ci = k2e.val[e] * sd.inv_diag[k2e.idx[e]];
                    rho += ci;
                    st.keep.col[kno[T.si] + e] = sd.gidx[a];
                    st.keep.val[kno[T.si] + e] = ci * spou_of(a);
                }
                st.rho[row] = rho;
                st.keep.ptr[row + 1] = kno[T.si] + k2e.ptr[i + 1];
            }
        }
    });
    for (int32_t si = 0; si < ns; ++si) {
        const Subdomain& sd = subs[ids[si]];
        const int32_t nq = sd.n_q(), nr = sd.n_r(), nl = nq + nr;
        const int64_t o = so[si];
        const int64_t keep0 = o + (sd.elim_q ? nq : 0);
        const int32_t n_keep = sd.elim_q ? nr : nq, n_elim = sd.elim_q ? nq : nr;
        st.sub_nloc[si] = nl;
        st.sub_nkeep[si] = n_keep;
        double I = 0.0;
        for (int32_t e = 0; e < n_elim; ++e) I += sd.inv_diag[e];
        st.sub_I[si] = I;
        if (sd.kind == 0) {
            st.dn_keep0.push_back(keep0);
            st.dn_n.push_back(sd.n_red);
            st.dn_loff.push_back((int64_t)st.dn_L.size());
            st.dn_L.insert(st.dn_L.end(), sd.L.begin(), sd.L.end());
        } else {
            const AcFactor& f = sd.ac;
            ac_subs.push_back(si);
            max_lev = std::max(max_lev, f.nlev);
            if (f.ncore > 0) {
                const int32_t g = (int32_t)st.core_n.size();
                st.core_n.push_back(f.ncore);
                st.core_slot_off.push_back((int64_t)st.core_slot.size());
                st.core_z_off.push_back((int64_t)st.core_z.size());
                for (int32_t a = 0; a < f.ncore; ++a) st.core_slot.push_back((uint32_t)(keep0 + f.core_vertex[a]));
                st.core_z.insert(st.core_z.end(), f.core_z.begin(), f.core_z.end());
                for (int32_t r0 = 0; r0 < f.ncore; r0 += kCoreRowsPerBlock) {
                    st.core_of_block.push_back(g);
                    st.row0_of_block.push_back(r0);
                }
            }
        }
    }
    st.nslots = nslots;
    // AC rows per (AC subdomain, level), built in parallel: bwd rows are the level's
    // columns in order (pivot slot, 1/pivot, entries in column order); fwd rows are the
    // level's targets in ascending slot order, each with its sources in ascending order
    // (within one level every (target, source) pair occurs once).
    struct LevelRows {
        std::vector<uint32_t> slot;
        std::vector<double> scale;
        std::vector<int64_t> len;
        std::vector<uint32_t> col;
        std::vector<double> val;
    };
    const size_t nac = ac_subs.size();
    std::vector<std::vector<LevelRows>> fwd_sl(nac), bwd_sl(nac);
    std::vector<std::pair<int32_t, int32_t>> ac_tasks;
    for (size_t i = 0; i < nac; ++i) {
        const int32_t nlev = subs[ids[ac_subs[i]]].ac.nlev;
        fwd_sl[i].resize(nlev);
        bwd_sl[i].resize(nlev);
        for (int32_t lv = 0; lv < nlev; ++lv) ac_tasks.push_back({(int32_t)i, lv});
    }
    parallel_tasks(ac_tasks.size(), [&](size_t t) {
        const int32_t i = ac_tasks[t].first, lv = ac_tasks[t].second;
        const int32_t si = ac_subs[i];
        const Subdomain& sd = subs[ids[si]];
        const AcFactor& f = sd.ac;
        const int64_t keep0 = so[si] + (sd.elim_q ? sd.n_q() : 0);
        LevelRows& B = bwd_sl[i][lv];
        LevelRows& F = fwd_sl[i][lv];
        std::vector<std::tuple<uint32_t, uint32_t, double>> trip;  // (target, source, coef)
        for (int32_t c = f.level_ptr[lv]; c < f.level_ptr[lv + 1]; ++c) {
            const uint32_t v = (uint32_t)(keep0 + f.col_vertex[c]);
            for (int32_t e = f.col_ptr[c]; e < f.col_ptr[c + 1]; ++e) {
                const uint32_t u = (uint32_t)(keep0 + f.col_idx[e]);
                B.col.push_back(u);
                B.val.push_back(f.col_coef[e]);
                trip.emplace_back(u, v, f.col_coef[e]);
            }
            const double dd = f.col_diag[c];
            B.slot.push_back(v);
            B.scale.push_back(dd > 0.0 ? 1.0 / dd : 0.0);
            B.len.push_back(f.col_ptr[c + 1] - f.col_ptr[c]);
        }
        std::sort(trip.begin(), trip.end(), [](const auto& x, const auto& y) {
            return std::get<0>(x) != std::get<0>(y) ? std::get<0>(x) < std::get<0>(y) : std::get<1>(x) < std::get<1>(y);
        });
        for (size_t a = 0; a < trip.size();) {
            const uint32_t u = std::get<0>(trip[a]);
            const size_t a0 = a;
            while (a < trip.size() && std::get<0>(trip[a]) == u) {
                F.col.push_back(std::get<1>(trip[a]));
                F.val.push_back(std::get<2>(trip[a]));
                ++a;
            }
            F.slot.push_back(u);
            F.scale.push_back(1.0);
            F.len.push_back((int64_t)(a - a0));
        }
    });
    // level-major AC rows: fwd (targets, may split) and bwd (columns, never split)
    st.fwd_lp.push_back(0);
    st.bwd_lp.push_back(0);
    auto append = [](CsrHost& c, const LevelRows& R) {
        c.row_slot.insert(c.row_slot.end(), R.slot.begin(), R.slot.end());
        c.rscale.insert(c.rscale.end(), R.scale.begin(), R.scale.end());
        c.col.insert(c.col.end(), R.col.begin(), R.col.end());
        c.val.insert(c.val.end(), R.val.begin(), R.val.end());
        for (int64_t l : R.len) c.ptr.push_back(c.ptr.back() + l);
    };
    for (int32_t lv = 0; lv < max_lev; ++lv) {
        const int64_t r0 = st.fwd.nrows();
        for (size_t i = 0; i < nac; ++i)
            if (lv < (int32_t)fwd_sl[i].size()) append(st.fwd, fwd_sl[i][lv]);
        auto fc = make_chunks(st.fwd.ptr, r0, st.fwd.nrows(), 64, 1, true);  // long rows in pieces (atomics)
        st.fwd.chunks.insert(st.fwd.chunks.end(), fc.begin(), fc.end());
        st.fwd_lp.push_back((int64_t)st.fwd.chunks.size());
        const int64_t b0 = st.bwd.nrows();
        for (size_t i = 0; i < nac; ++i)
            if (lv < (int32_t)bwd_sl[i].size()) append(st.bwd, bwd_sl[i][lv]);
        auto bc = make_chunks(st.bwd.ptr, b0, st.bwd.nrows(), 256, 1, false);
        st.bwd.chunks.insert(st.bwd.chunks.end(), bc.begin(), bc.end());
        st.bwd_lp.push_back((int64_t)st.bwd.chunks.size());
    }
    // one warp per chunk (csr_rows_kernel): single rows, long rows in pieces of 256
    st.keep.chunks = make_chunks(st.keep.ptr, 0, st.keep.nrows(), 256, 1, true);
    if (with_gather) {
        st.gptr.assign((size_t)ndofs + 1, 0);
        for (uint32_t g : st.gidx) st.gptr[g + 1]++;
        for (int64_t j = 0; j < ndofs; ++j) st.gptr[j + 1] += st.gptr[j];
        st.gslot.resize(st.gidx.size());
        std::vector<int64_t> cur(st.gptr.begin(), st.gptr.end() - 1);
        for (size_t l = 0; l < st.gidx.size(); ++l) st.gslot[cur[st.gidx[l]]++] = (uint32_t)l;
        const size_t ng = st.gslot.size();
        st.gsub.resize(ng);
        st.gspou.resize(ng);
        st.ginvd.resize(ng);
        st.gbs_ptr.assign(ng + 1, 0);
        st.gbs_cnt.resize(ng);
        for (size_t e = 0; e < ng; ++e) {
            const uint32_t l = st.gslot[e];
            const int64_t len = st.bs_ptr[l + 1] - st.bs_ptr[l];
            st.gbs_cnt[e] = (uint32_t)len;
            st.gbs_ptr[e + 1] = st.gbs_ptr[e] + ((len + 3) & ~int64_t(3));  // rows start at multiples of 4
        }
        st.gbs_col.resize((size_t)st.gbs_ptr[ng]);  // every entry, padding included, written below
        st.gbs_val.resize((size_t)st.gbs_ptr[ng]);
        constexpr size_t kPer = 1 << 16;
        parallel_tasks((ng + kPer - 1) / kPer, [&](size_t t) {
            for (size_t e = t * kPer; e < std::min(ng, (t + 1) * kPer); ++e) {
                const uint32_t l = st.gslot[e];
                st.gsub[e] = st.sub_of[l];
                st.gspou[e] = st.spou[l];
                st.ginvd[e] = st.invd[l];
                std::copy(st.bs_col.begin() + st.bs_ptr[l], st.bs_col.begin() + st.bs_ptr[l + 1],
                          st.gbs_col.begin() + st.gbs_ptr[e]);
                std::copy(st.bs_val.begin() + st.bs_ptr[l], st.bs_val.begin() + st.bs_ptr[l + 1],
                          st.gbs_val.begin() + st.gbs_ptr[e]);
                for (int64_t q = st.gbs_ptr[e] + st.gbs_cnt[e]; q < st.gbs_ptr[e + 1]; ++q) {  // padding
                    st.gbs_col[q] = st.gbs_col[st.gbs_ptr[e]];
                    st.gbs_val[q] = 0.0;
                }
            }
        });
    }
    return st;
}

template <typename T>
void upload_csr(CsrDev<T>& d, const CsrHost& h) {
    d.nrows = h.nrows();
    d.row_slot.upload(h.row_slot);
    d.ptr.upload(h.ptr);
    d.col.upload(h.col);
    d.val.upload_cast(h.val);
    d.rscale.upload_cast(h.rscale);
    d.chunks.upload(h.chunks);
    d.nchunks = (int64_t)h.chunks.size();
}

template <typename T>
void upload_stage(StageDev<T>& d, const StageHost& h) {
    d.nsub = h.nsub;
    d.nslots = h.nslots;
    d.nkeep = (int64_t)h.keep_slots.size();
    d.gidx.upload(h.gidx);
    d.sub_of.upload(h.sub_of);
    d.keep_slots.upload(h.keep_slots);
    d.spou.upload_cast(h.spou);
    d.invd.upload_cast(h.invd);
    d.rho.upload_cast(h.rho);
    d.sub_nloc.upload(h.sub_nloc);
    d.sub_nkeep.upload(h.sub_nkeep);
    d.sub_I.upload(h.sub_I);
    upload_csr(d.keep, h.keep);
    upload_csr(d.fwd, h.fwd);
    upload_csr(d.bwd, h.bwd);
    if (h.gptr.empty()) {  // slot-order back substitution (multiplicative stages)
        d.bs_ptr.upload(h.bs_ptr);
        d.bs_col.upload(h.bs_col);
        d.bs_val.upload_cast(h.bs_val);
    }
    d.fwd_lp = h.fwd_lp;
    d.bwd_lp = h.bwd_lp;
    d.fwd_lp_d.upload(h.fwd_lp);
    d.bwd_lp_d.upload(h.bwd_lp);
    d.ndense = (int32_t)h.dn_n.size();
    d.dn_keep0.upload(h.dn_keep0);
    d.dn_loff.upload(h.dn_loff);
    d.dn_n.upload(h.dn_n);
    d.dn_L.upload_cast(h.dn_L);
    d.ncore_blocks = (int32_t)h.core_of_block.size();
    d.core_rmax = h.core_n.empty() ? 0 : *std::max_element(h.core_n.begin(), h.core_n.end());
    d.core_total = (int64_t)h.core_slot.size();
    d.core_of_block.upload(h.core_of_block);
    d.row0_of_block.upload(h.row0_of_block);
    d.core_n.upload(h.core_n);
    d.core_slot_off.upload(h.core_slot_off);
    d.core_z_off.upload(h.core_z_off);
    d.core_slot.upload(h.core_slot);
    d.core_z.upload_cast(h.core_z);
    d.gptr.upload(h.gptr);
    d.gslot.upload(h.gslot);
    d.gsub.upload(h.gsub);
    d.gspou.upload_cast(h.gspou);
    d.ginvd.upload_cast(h.ginvd);
    d.gbs_ptr.upload(h.gbs_ptr);
    d.gbs_cnt.upload(h.gbs_cnt);
    d.gbs_col.upload(h.gbs_col);
    d.gbs_val.upload_cast(h.gbs_val);
}

}  // namespace

// ---------------------------------------------------------------------------
// Solver
// ---------------------------------------------------------------------------



struct Workspace {
    int kp = 0;
    int64_t gen = 0;                         // bumped whenever the buffers move
    DArr<double> yi, e;                      // n x kp interleaved (primary-sorted)
    DArr<double> b, x, r, gx;                // m x kp FP64: rhs, solution, refinement residual, G x
    DArr<double> cx, cr, dz, dp, dap;        // FP64 inner CG vectors
    DArr<float> frhs, fx, fr, fz, fp, fap;   // FP32 inner CG vectors (mixed precision)
    DArr<double> vloc, cbuf;                 // slots x kp; cbuf: m x kp, a multiplicative stage's -correction
    DArr<float> floc, fcbuf;                 // the same in FP32
    DArr<double> core_tmp;
    DArr<float> fcore_tmp;
    DArr<double> rwork;                      // multiplicative residual
    DArr<float> frwork;
    DArr<double> msum;                       // 6 x nsub x kp: S0, SB, M1, M2, means (m0, m2)
    DArr<double> part;                       // block partial sums
    DArr<double> red;                        // reduced partial sums (kp)
    // per-RHS Krylov state
    DArr<double> st_bnorm, st_rz, st_rz0, st_alpha, st_beta, st_rnorm, st_tol;
    DArr<int32_t> st_active, st_conv, st_iters, st_part;
    DArr<int32_t> n_active;
    DArr<unsigned> sweep_bar;                // grid-barrier counters of the fused AC sweeps
    DArr<int32_t> sweep_err;                 // set when a barrier wait ran out
};

// The active-RHS count into the host's pinned status word, written by a kernel rather than
// copied: a copy would wait in the copy engine's queue behind bulk transfers of other
// calls (host-buffer solves overlap their uploads and downloads with other solves).
__global__ void publish_active_kernel(const int32_t* __restrict__ n_active, volatile int32_t* host) {
    *host = *n_active;
    __threadfence_system();
}

// Small device-to-host reads of the solve loop (flags, per-RHS counters, partial sums)
// go the same way: a kernel stores them into pinned host staging memory.
__global__ void d2h_words_kernel(const uint32_t* __restrict__ src, volatile uint32_t* dst, size_t nwords) {
    for (size_t i = threadIdx.x; i < nwords; i += blockDim.x) dst[i] = src[i];
    __threadfence_system();
}

// Small host-to-device writes (per-RHS masks and tolerances, at most 32 each) travel as
// kernel arguments, for the same reason.
struct SmallI32 { int32_t v[32]; };
struct SmallF64 { double v[32]; };
__global__ void set_small_kernel(SmallI32 a, int32_t* __restrict__ da, SmallF64 b, double* __restrict__ db, int n) {
    const int t = threadIdx.x;
    if (t < n) {
        if (da) da[t] = a.v[t];
        if (db) db[t] = b.v[t];
    }
}

// Resident blocks per SM of `kern` at kBlock threads without dynamic shared memory,
// queried once per kernel (the instantiations of one template differ in registers, so
// the count is kept per kernel, not per signature).
inline int resident_per_sm(const void* kern) {
    static std::mutex mu;
    static std::unordered_map<const void*, int> cache;
    std::lock_guard<std::mutex> lk(mu);
    const auto it = cache.find(kern);
    if (it != cache.end()) return it->second;
    int n = 0;
    WB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, kern, kBlock, 0));
    n = std::max(n, 1);
    cache.emplace(kern, n);
    return n;
}

// Device arrays of the hybrid operator apply (prim_rows_kernel + CSR rows; see
// build_hybrid): the C_PO entries of every primary level, and the Gramian rows of the
// other factors' dofs.  Built for one set of small factors (smask: bits of design
// factors).
struct HybridDev {
    uint32_t smask = 0;
    DArr<uint32_t> lvl_ptr;  // primary level -> first observation in device order (+ n)
    DArr<int64_t> pptr;      // C_PO rows of the primary levels
    DArr<uint32_t> pcol;
    DArr<double> pval64;
    DArr<float> pval32;
    DArr<uint32_t> rows;     // dofs of the other rows
    DArr<int64_t> optr;
    DArr<uint32_t> ocol;
    DArr<double> oval64;
    DArr<float> oval32;
    DArr<CsrChunk> ochunks;
    int64_t nochunks = 0, nnz = 0;
    // the primary levels in pieces of at most kMmaPiece observations (prim_mma_kernel):
    // (level, first observation, end, first piece | split << 1)
    DArr<uint4> pieces;
    int64_t npieces = 0;
    bool any_split = false;
};

// Device buffers of one host-buffer solve (its inputs, outputs and copy stream).
struct HostCall {
    DArr<double> y, x, dem;
    cudaStream_t stream = nullptr;
    bool busy = false;
    ~HostCall() {
        if (stream) cudaStreamDestroy(stream);
    }
};

struct SolverImpl {
    std::mutex mu;
    Design d;
    PrecondConfig pc;
    int32_t reduction_strategy = 0;  // as configured (AdditiveSchwarz reduction)
    within_params params{};
    std::vector<Subdomain> subs;
    int primary = 0;
    bool perm_identity = true;
    cudaStream_t stream = nullptr;
    int n_sm = 148;
    bool coop = false;  // cooperative launches available (fused AC sweeps)
    // device design
    DArr<uint32_t> codes, perm;
    DArr<double> w64;
    DArr<float> w32;
    DArr<ObsChunk> chunks;
    ObsParams obs{};
    bool has_split = false;
    // observation-pass block shapes the autotuner picks from: chunk tables of 16, 32 and
    // 64 observations per work unit, and 1 or 2 resident blocks per SM; choice per
    // (kp class, element size), -1 = not tuned (32 observations, 2 blocks per SM)
    DArr<ObsChunk> chunk_tab[3];
    int64_t nchunk_tab[3] = {0, 0, 0};
    bool split_tab[3] = {false, false, false};
    int32_t obs_choice[4][2] = {{-1, -1}, {-1, -1}, {-1, -1}, {-1, -1}};
    DArr<unsigned char> obs_hot;  // per-block global hot tables of the observation pass
    float obs_tune_ms[4][2][24] = {};  // the autotuner's time per candidate (0: not timed)
    // hybrid operator apply: per (kp class, precision) -1 not decided, 0 off, 1 on (the
    // autotuner's choice), its timed apply (ms; 0 not timed), and its arrays
    int32_t hyb_on[4][2] = {{-1, -1}, {-1, -1}, {-1, -1}, {-1, -1}};
    float hyb_ms[4][2] = {};
    std::unique_ptr<HybridDev> hyb;
    std::vector<int64_t> lvl_ptr_h;  // primary level -> first observation (device order)
    // hottest levels of every non-primary factor, for the observation pass
    std::vector<DArr<uint32_t>> hot_level;
    std::vector<int32_t> hot_count;
    std::vector<int> dev_factor;  // device factor slot -> design factor (slot 0 = primary)
    // Schwarz stages
    std::vector<StageDev<double>> stages64;
    std::vector<StageDev<float>> stages32;
    int32_t max_nsub = 0;
    int64_t max_slots = 0, max_core_total = 0;
    // explicit Gramian (multiplicative)
    DArr<int64_t> g_ptr;
    DArr<uint32_t> g_idx;
    DArr<double> g_val64;
    DArr<float> g_val32;
    // The Krylov operator is the explicit G above (OperatorRepr::Explicit, or a
    // multiplicative preconditioner, whose residual updates need G anyway): its rows in
    // chunks for csr_rows_kernel (one warp per row, long rows in pieces).
    bool explicit_op = false;
    DArr<uint32_t> g_rows;
    DArr<CsrChunk> g_chunks;
    int64_t g_nchunks = 0;
    Workspace ws;
    // device side of the host-buffer entry points: one slot per call in flight (calls from
    // several host threads upload and download concurrently; their solves take turns)
    std::mutex calls_mu;
    std::vector<std::unique_ptr<HostCall>> calls;
    std::shared_ptr<void> gmres;  // GmresBufs, created on first GMRES solve
    std::shared_ptr<void> lsmr;   // LsmrBufs, created on first LSMR solve
    std::shared_ptr<void> cn;     // CnState of the coarse-space network, kept while training
    bool precond_only = false;    // built from a serialized preconditioner: no design
    bool inject_sweep_timeout = false;  // test hook: AC sweep barriers that cannot be met
    int64_t sweep_cluster_chunks = 512;  // AC levels of at most this many chunks go to one cluster (0: none)
    std::vector<uint8_t> pc_bytes;  // serialized preconditioner, made on first request
    int32_t* h_active = nullptr;  // pinned
    uint32_t* h_stage = nullptr;  // pinned staging of small reads (read_small)
    size_t h_stage_words = 0;
    double setup_time = 0.0;
    int64_t gpu_launches = 0;
    // Optional event timing of selected launches (0: FP64 operator, 1: FP32 operator,
    // 2: Schwarz apply FP64, 3: Schwarz apply FP32).
    bool profiling = false;
    std::vector<cudaEvent_t> ev_pool;
    std::vector<std::pair<int, std::pair<cudaEvent_t, cudaEvent_t>>> ev_pending;
    int64_t prof_count[4] = {0, 0, 0, 0};
    double prof_ms[4] = {0, 0, 0, 0};
    // One CG iteration captured as a CUDA graph, reused while its buffers stay the same.
    cudaGraphExec_t cg_exec = nullptr;
    std::array<uintptr_t, 9> cg_key{};
    int64_t cg_launches = 0;  // kernels in one captured iteration
    // Coarse space (learned by the message-passing network, or given): CG adds
    // Z E^+ Z' r to the Schwarz output.  Z is n_dofs x 32 row-major (unused columns zero).
    int32_t coarse_k = 0;
    DArr<double> coarse_z64, coarse_gz64, coarse_einv, coarse_part, coarse_u, coarse_tmp64;
    DArr<float> coarse_z32, coarse_gz32, coarse_tmp32;
    // training targets of the network on this design (n_dofs x t, scaled space)
    DArr<float> cn_targets;
    int32_t cn_t = 0;

    ~SolverImpl() {
        for (auto& p : ev_pending) { cudaEventDestroy(p.second.first); cudaEventDestroy(p.second.second); }
        for (cudaEvent_t e : ev_pool) cudaEventDestroy(e);
        if (cg_exec) cudaGraphExecDestroy(cg_exec);
        if (h_active) cudaFreeHost(h_active);
        if (h_stage) cudaFreeHost(h_stage);
        if (stream) cudaStreamDestroy(stream);
    }
    bool mixed() const { return params.precision == WITHIN_PRECISION_MIXED; }
    // blocks for a grid-stride pass over `rows` rows with G lanes per row
    int nblk(int64_t rows, int G, int cap_per_sm = 8) const {
        const int64_t need = (rows * G + kBlock - 1) / kBlock;
        return (int)std::max<int64_t>(1, std::min<int64_t>(need, (int64_t)n_sm * cap_per_sm));
    }
    // blocks for a grid-stride pass that needs `need` blocks, at most one resident wave
    // of `kern` (a second, partial wave would leave SMs idle at the end)
    int fit(int64_t need, const void* kern) const {
        return (int)std::max<int64_t>(1, std::min<int64_t>(need, (int64_t)n_sm * resident_per_sm(kern)));
    }
    cudaEvent_t take_event() {
        if (ev_pool.empty()) {
            cudaEvent_t e;
            WB_CUDA(cudaEventCreate(&e));
            return e;
        }
        cudaEvent_t e = ev_pool.back();
        ev_pool.pop_back();
        return e;
    }
    void prof_begin(cudaEvent_t& a) {
        if (!profiling) return;
        a = take_event();
        WB_CUDA(cudaEventRecord(a, stream));
    }
    void prof_end(int which, cudaEvent_t a) {
        if (!profiling) return;
        cudaEvent_t b = take_event();
        WB_CUDA(cudaEventRecord(b, stream));
        ev_pending.push_back({which, {a, b}});
    }
    // after a stream synchronisation: fold finished intervals into the totals
    void prof_harvest() {
        for (auto& p : ev_pending) {
            float ms = 0.f;
            WB_CUDA(cudaEventElapsedTime(&ms, p.second.first, p.second.second));
            prof_ms[p.first] += ms;
            prof_count[p.first] += 1;
            ev_pool.push_back(p.second.first);
            ev_pool.push_back(p.second.second);
        }
        ev_pending.clear();
    }
};

namespace {

#define WB_DISPATCH_G(G, ...)                                      \
    switch (G) {                                                   \
        case 1: { constexpr int GV = 1; __VA_ARGS__; } break;      \
        case 2: { constexpr int GV = 2; __VA_ARGS__; } break;      \
        case 4: { constexpr int GV = 4; __VA_ARGS__; } break;      \
        default: { constexpr int GV = 8; __VA_ARGS__; } break;     \
    }

// Lanes per row for kp RHS (kp a multiple of 4, <= 32): kp/4 rounded up to 1, 2, 4 or 8.
// For kp in {12, 20, 24, 28} the extra lanes would own columns past kp, so those widths
// are padded: kp is rounded to 16 or 32 by pad_kp below.
// dst <- bytes (a multiple of 4) of device memory at src, after the work already on the
// solver's stream (which this synchronizes).
void read_small(SolverImpl& S, void* dst, const void* src, size_t bytes) {
    const size_t words = bytes / 4;
    if (words > S.h_stage_words) {
        if (S.h_stage) WB_CUDA(cudaFreeHost(S.h_stage));
        S.h_stage = nullptr;
        S.h_stage_words = 0;
        WB_CUDA(cudaMallocHost(&S.h_stage, std::max<size_t>(words, 1 << 16) * 4));
        S.h_stage_words = std::max<size_t>(words, 1 << 16);
    }
    if (words > 0) {
        d2h_words_kernel<<<1, 256, 0, S.stream>>>(static_cast<const uint32_t*>(src), S.h_stage, words);
        WB_CUDA(cudaGetLastError());
    }
    WB_CUDA(cudaStreamSynchronize(S.stream));
    std::memcpy(dst, S.h_stage, words * 4);
}

// da[0..n) <- a, db[0..n) <- b (either may be null; n <= 32), in order on the stream.
void write_small(SolverImpl& S, int32_t* da, const int32_t* a, double* db, const double* b, int n) {
    SmallI32 ai{};
    SmallF64 bi{};
    for (int i = 0; i < n; ++i) {
        if (a) ai.v[i] = a[i];
        if (b) bi.v[i] = b[i];
    }
    set_small_kernel<<<1, 32, 0, S.stream>>>(ai, a ? da : nullptr, bi, b ? db : nullptr, n);
    WB_CUDA(cudaGetLastError());
}

void publish_active(SolverImpl& S, const int32_t* n_active) {
    publish_active_kernel<<<1, 1, 0, S.stream>>>(n_active, S.h_active);
    WB_CUDA(cudaGetLastError());
}

int group_for(int kp) { return kp / 4; }
int pad_kp(int k) {
    const int kp = pad4(k);
    if (kp <= 8) return kp;
    if (kp <= 16) return 16;
    return 32;
}

// Observation chunks over primary-sorted observations (level-aligned; long levels split).
std::vector<ObsChunk> make_obs_chunks(const std::vector<int64_t>& lvl_ptr, int64_t nlev, bool& has_split,
                                      int64_t kObsPerChunk = 32) {
    std::vector<ObsChunk> out;
    has_split = false;
    int64_t l = 0;
    while (l < nlev) {
        const int64_t len = lvl_ptr[l + 1] - lvl_ptr[l];
        if (len > 2 * kObsPerChunk) {
            for (int64_t a = lvl_ptr[l]; a < lvl_ptr[l + 1]; a += kObsPerChunk)
                out.push_back(ObsChunk{(uint32_t)a, (uint32_t)std::min(a + kObsPerChunk, lvl_ptr[l + 1]),
                                       (uint32_t)l, (uint32_t)(l + 1), 1u});
            has_split = true;
            ++l;
            continue;
        }
        int64_t l1 = l + 1;
        while (l1 < nlev && lvl_ptr[l1 + 1] - lvl_ptr[l] <= kObsPerChunk &&
               lvl_ptr[l1 + 1] - lvl_ptr[l1] <= 2 * kObsPerChunk)
            ++l1;
        out.push_back(ObsChunk{(uint32_t)lvl_ptr[l], (uint32_t)lvl_ptr[l1], (uint32_t)l, (uint32_t)l1, 0u});
        l = l1;
    }
    return out;
}

void upload_design(SolverImpl& S) {
    const Design& d = S.d;
    // primary = factor with the most levels; observations sorted by its level (stable)
    S.primary = 0;
    for (int q = 1; q < d.Q; ++q)
        if (d.nlev[q] > d.nlev[S.primary]) S.primary = q;
    const uint32_t* cp = d.codes.data() + (size_t)S.primary * d.n;
    const int64_t np = d.nlev[S.primary];
    std::vector<int64_t> lvl_ptr((size_t)np + 1, 0);
    for (int64_t i = 0; i < d.n; ++i) lvl_ptr[cp[i] + 1]++;
    for (int64_t l = 0; l < np; ++l) lvl_ptr[l + 1] += lvl_ptr[l];
    // device factor order: the primary factor first, then the others by level count,
    // largest first (the observation pass's private-table factors are a suffix)
    S.dev_factor.clear();
    S.dev_factor.push_back(S.primary);
    for (int q = 0; q < d.Q; ++q)
        if (q != S.primary) S.dev_factor.push_back(q);
    std::stable_sort(S.dev_factor.begin() + 1, S.dev_factor.end(),
                     [&](int a, int b) { return d.nlev[a] > d.nlev[b]; });
    std::vector<uint32_t> perm((size_t)d.n);
    {
        std::vector<int64_t> cur(lvl_ptr.begin(), lvl_ptr.end() - 1);
        for (int64_t i = 0; i < d.n; ++i) perm[cur[cp[i]]++] = (uint32_t)i;
    }
    // Within a primary level the observation pass keeps a running sum of the slot-1
    // factor while its level repeats.  When the rows come in an order where that factor
    // alternates (short runs: a worker's years shuffled between its firms), the
    // observations of each primary level are also sorted by it (G does not depend on the
    // order): a stable counting sort by the slot-1 level, then by the primary level.
    if (d.Q >= 2) {
        const uint32_t* c1 = d.codes.data() + (size_t)S.dev_factor[1] * d.n;
        int64_t runs = 0;
        for (int64_t i = 0; i < d.n; ++i)
            if (i == 0 || cp[perm[i]] != cp[perm[i - 1]] || c1[perm[i]] != c1[perm[i - 1]]) ++runs;
        if (runs > d.n * 3 / 10) {
            const int64_t L1 = d.nlev[S.dev_factor[1]];
            std::vector<int64_t> c1ptr((size_t)L1 + 1, 0);
            for (int64_t i = 0; i < d.n; ++i) c1ptr[c1[i] + 1]++;
            for (int64_t l = 0; l < L1; ++l) c1ptr[l + 1] += c1ptr[l];
            std::vector<uint32_t> by1((size_t)d.n);
            for (int64_t i = 0; i < d.n; ++i) by1[c1ptr[c1[i]]++] = (uint32_t)i;
            std::vector<int64_t> cur(lvl_ptr.begin(), lvl_ptr.end() - 1);
            for (int64_t a = 0; a < d.n; ++a) perm[cur[cp[by1[a]]]++] = by1[a];
        }
    }
    S.perm_identity = true;
    for (int64_t i = 0; i < d.n; ++i)
        if (perm[i] != (uint32_t)i) { S.perm_identity = false; break; }
    // hot levels: the 255 most frequent levels (hit >= 64 times) of each non-primary
    // factor with more than 256 levels and fewer than 2^24; their codes on the device
    // carry the hot slot + 1 in bits 24-31 (kObsLevelBits) next to the level
    S.hot_level.clear();
    S.hot_level.resize(d.Q);
    S.hot_count.assign(d.Q, 0);
    std::vector<std::vector<uint32_t>> hot_tag((size_t)d.Q);  // level -> tag (slot + 1) << 24, or 0
    ObsParams& P = S.obs;
    for (int sl = 1; sl < d.Q; ++sl) {
        P.packed[sl] = 0;
        P.hot_level[sl] = nullptr;
        const int q = S.dev_factor[sl];
        const int64_t L = d.nlev[q];
        if (L <= 256 || L >= ((int64_t)1 << kObsLevelBits)) continue;
        std::vector<int64_t> cnt((size_t)L, 0);
        const uint32_t* c = d.codes.data() + (size_t)q * d.n;
        for (int64_t i = 0; i < d.n; ++i) cnt[c[i]]++;
        std::vector<uint32_t> order((size_t)L);
        std::iota(order.begin(), order.end(), 0u);
        const int64_t h = std::min<int64_t>(kObsMaxHot, L);
        std::partial_sort(order.begin(), order.begin() + h, order.end(),
                          [&](uint32_t a, uint32_t b) { return cnt[a] != cnt[b] ? cnt[a] > cnt[b] : a < b; });
        std::vector<uint32_t> lev;
        hot_tag[sl].assign((size_t)L, 0u);
        for (int64_t a = 0; a < h; ++a) {
            if (cnt[order[a]] < 64) break;
            hot_tag[sl][order[a]] = (uint32_t)(lev.size() + 1) << kObsLevelBits;
            lev.push_back(order[a]);
        }
        P.packed[sl] = 1;
        S.hot_count[sl] = (int32_t)lev.size();
        S.hot_level[sl].upload(lev);
        P.hot_level[sl] = S.hot_level[sl].p;
    }
    // codes and weights padded to a multiple of 4 observations (16-byte batch loads)
    const int64_t ns = (d.n + 3) / 4 * 4;
    {
        std::vector<uint32_t> codes((size_t)ns * d.Q, 0u);
        for (int s = 0; s < d.Q; ++s) {
            const uint32_t* src = d.codes.data() + (size_t)S.dev_factor[s] * d.n;
            uint32_t* dst = codes.data() + (size_t)s * ns;
            if (P.packed[s]) {
                const std::vector<uint32_t>& tag = hot_tag[s];
                for (int64_t i = 0; i < d.n; ++i) dst[i] = src[perm[i]] | tag[src[perm[i]]];
            } else {
                for (int64_t i = 0; i < d.n; ++i) dst[i] = src[perm[i]];
            }
        }
        S.codes.upload(codes);
    }
    if (!S.perm_identity) S.perm.upload(perm);
    if (!d.w.empty()) {
        std::vector<double> w((size_t)ns, 0.0);
        for (int64_t i = 0; i < d.n; ++i) w[i] = d.w[perm[i]];
        S.w64.upload(w);
        if (S.mixed()) S.w32.upload_cast(w);
    }
    auto ch = make_obs_chunks(lvl_ptr, np, S.has_split);
    S.chunks.upload(ch);
    S.lvl_ptr_h = lvl_ptr;
    for (int ci = 0; ci < 3; ++ci) {
        const int64_t per = (int64_t)16 << ci;
        auto t = make_obs_chunks(lvl_ptr, np, S.split_tab[ci], per);
        S.nchunk_tab[ci] = (int64_t)t.size();
        S.chunk_tab[ci].upload(t);
    }
    P.n = d.n;
    P.ns = ns;
    P.Q = d.Q;
    P.packed[0] = 0;
    P.codes = S.codes.p;
    for (int s = 0; s < d.Q; ++s) P.off[s] = d.off[S.dev_factor[s]];
    P.chunks = S.chunks.p;
    P.nchunks = (int64_t)ch.size();
}

// Shared-memory plan of the observation pass for kp interleaved RHS of `elem` bytes:
// the smallest non-primary factors get a table private to every lane group while those
// fit (kObsPrivBytes per block); then factors of <= 256 levels get a block-shared table
// and the others their hottest levels, within kObsSmemBytes per block (two blocks/SM).
constexpr int64_t kObsPrivBytes = 96 * 1024, kObsSmemBytes = 110 * 1024;

// `hot_global`: the hot tables go to per-block copies in S.obs_hot (sized by
// obs_hot_bytes) instead of shared memory, all of each factor's hot levels.
int obs_params_for(SolverImpl& S, int kp, size_t elem, ObsParams& P, bool hot_global = false) {
    P = S.obs;
    P.kp = kp;
    P.hot_glob = nullptr;
    P.hot_glob_stride = 0;
    const int G = group_for(kp);
    const int64_t gpb = (elem == 8 ? obs_block<double>() : obs_block<float>()) / G;
    const int Q = S.d.Q;
    for (int sl = 0; sl < kMaxQ; ++sl) {
        P.sink[sl] = SINK_GLOBAL;
        P.smem_base[sl] = -1;
        P.smem_len[sl] = 0;
    }
    // private tables for a suffix of the slots (the smallest factors); a group's area
    // stride is padded so that the 16-byte accesses of neighbouring groups at the same
    // level fall in different banks
    const int64_t target = elem == 4 ? (16 * G) % 128 : 16;
    auto padded = [&](int64_t r) {
        int64_t st = r;
        while ((st * (int64_t)elem) % 128 != target) ++st;
        return st;
    };
    int64_t raw = 0;
    int np = 0;
    for (int sl = Q - 1; sl >= 1; --sl) {
        const int64_t len = S.d.nlev[S.dev_factor[sl]] * kp;
        if (gpb * padded(raw + len) * (int64_t)elem > kObsPrivBytes) break;
        P.sink[sl] = SINK_PRIVATE;
        P.smem_base[sl] = (int32_t)raw;
        P.smem_len[sl] = (int32_t)len;
        raw += len;
        ++np;
    }
    P.priv_stride = raw > 0 ? (int32_t)padded(raw) : 0;
    int64_t used = gpb * P.priv_stride;
    const int64_t budget = kObsSmemBytes / (int64_t)elem;
    for (int sl = Q - 1; sl >= 1; --sl) {  // smallest first
        if (P.sink[sl] == SINK_PRIVATE) continue;
        const int64_t nl = S.d.nlev[S.dev_factor[sl]];
        if (nl <= 256 && used + nl * kp <= budget) {
            P.sink[sl] = SINK_BLOCK;
            P.smem_base[sl] = (int32_t)used;
            P.smem_len[sl] = (int32_t)(nl * kp);
            used += nl * kp;
        }
    }
    int64_t goff = 0;
    for (int sl = 1; sl < Q; ++sl) {  // hot levels, the hottest first, as many as fit
        P.hot_cap[sl] = 0;
        P.hot_goff[sl] = 0;
        if (P.sink[sl] != SINK_GLOBAL || S.hot_count[sl] == 0) continue;
        if (hot_global) {
            P.sink[sl] = SINK_HOT;
            P.hot_cap[sl] = S.hot_count[sl];
            P.hot_goff[sl] = (int32_t)goff;
            P.smem_len[sl] = (int32_t)(S.hot_count[sl] * kp);
            goff += (int64_t)S.hot_count[sl] * kp;
            continue;
        }
        const int64_t cap = std::min<int64_t>(S.hot_count[sl], (budget - used) / kp);
        if (cap < 16) continue;
        P.sink[sl] = SINK_HOT;
        P.hot_cap[sl] = (int32_t)cap;
        P.smem_base[sl] = (int32_t)used;
        P.smem_len[sl] = (int32_t)(cap * kp);
        used += cap * kp;
    }
    P.smem_elems = (int32_t)used;
    if (goff > 0) {
        // 16-byte aligned per-block copies; the pass runs at most 2 blocks per SM
        P.hot_glob_stride = (goff + 1) / 2 * 2;
        const size_t need = (size_t)S.n_sm * 2 * (size_t)P.hot_glob_stride * elem;
        P.hot_glob = S.obs_hot.n >= need ? (void*)S.obs_hot.p : nullptr;
    }
    return np;
}

// Grows S.obs_hot to `bytes`; a captured CG iteration holds the old address, so it is
// dropped (recaptured on its next use).  Outside any stream capture.
void grow_obs_hot(SolverImpl& S, size_t bytes) {
    if (bytes <= S.obs_hot.n) return;
    if (S.cg_exec) {
        WB_CUDA(cudaGraphExecDestroy(S.cg_exec));
        S.cg_exec = nullptr;
    }
    S.obs_hot.alloc(bytes);
}

// Bytes of S.obs_hot that the global hot tables need for kp RHS of `elem` bytes (0: the
// design has no hot levels outside shared memory's other tables).
size_t obs_hot_bytes(SolverImpl& S, int kp, size_t elem) {
    ObsParams P;
    obs_params_for(S, kp, elem, P, true);
    return (size_t)S.n_sm * 2 * (size_t)P.hot_glob_stride * elem;
}

int kp_class(int kp) { return kp <= 4 ? 0 : kp <= 8 ? 1 : kp <= 16 ? 2 : 3; }

// Returns the number of per-warp partial rows written (OBS_LSMR; grid x warps per block).
// Shapes of the observation pass: choice c < kObsShapes runs 16 << (c / 2) observations
// per chunk and 1 + c % 2 blocks per SM with the hot tables in shared memory; choice
// kObsShapes + c the same shape with them in per-block global copies (S.obs_hot); choice
// 2 kObsShapes + c the shape of c with wide lanes (8 RHS per lane; FP32, kp >= 8).
constexpr int kObsShapes = 6;
inline bool obs_wide_ok(int kp, size_t elem) { return elem == 4 && kp >= 8; }
// Wide lanes exist for the exact kernels only (Q <= 3, or Q = 4 with at most one private
// factor).
inline bool obs_wide_exact(int Q, int np) { return Q <= 3 || (Q == 4 && np <= 1); }
bool obs_wide_for(SolverImpl& S, int kp, size_t elem) {
    if (!obs_wide_ok(kp, elem)) return false;
    ObsParams P;
    return obs_wide_exact(S.d.Q, obs_params_for(S, kp, elem, P));
}

template <typename T, int MODE>
int launch_obs(SolverImpl& S, int kp, const T* w, const T* x, const T* yin, T* out, T* eout,
               const double* lsmr_scale = nullptr, double* lsmr_part = nullptr) {
    ObsParams P;
    // the autotuned block shape (obs_autotune), else 32 observations per chunk, 2 blocks/SM
    int choice = S.obs_choice[kp_class(kp)][sizeof(T) == 8 ? 1 : 0];
    int rv = (MODE == OBS_GRAM && choice >= 2 * kObsShapes && obs_wide_ok(kp, sizeof(T))) ? 2 : 1;
    if (choice >= 0) choice %= 2 * kObsShapes;
    int np = obs_params_for(S, kp, sizeof(T), P, choice >= kObsShapes);
    if (choice >= kObsShapes && !P.hot_glob) np = obs_params_for(S, kp, sizeof(T), P);  // no global copies
    if (!obs_wide_exact(S.d.Q, np)) rv = 1;
    choice = choice < 0 ? -1 : choice % kObsShapes;
    P.lsmr_scale = lsmr_scale;
    P.lsmr_part = lsmr_part;
    const int G = group_for(kp) / rv;
    bool split = S.has_split;
    int blocks_per_sm = 2;
    if (choice >= 0) {
        const int ci = choice / 2;
        P.chunks = S.chunk_tab[ci].p;
        P.nchunks = S.nchunk_tab[ci];
        split = S.split_tab[ci];
        blocks_per_sm = 1 + choice % 2;
    }
    if (MODE != OBS_DX && out) {
        // zero the outputs that are accumulated (every non-primary factor, split levels)
        const size_t m = (size_t)S.d.ndofs;
        if (split) {
            WB_CUDA(cudaMemsetAsync(out, 0, m * kp * sizeof(T), S.stream));
        } else {
            const size_t a = (size_t)S.d.off[S.primary] * kp, b = (size_t)(S.d.off[S.primary] + S.d.nlev[S.primary]) * kp;
            if (a > 0) WB_CUDA(cudaMemsetAsync(out, 0, a * sizeof(T), S.stream));
            if (m * kp > b) WB_CUDA(cudaMemsetAsync(out + b, 0, (m * kp - b) * sizeof(T), S.stream));
        }
    }
    const size_t smem = (size_t)P.smem_elems * sizeof(T);
    // two resident blocks per SM (registers and shared memory)
    const int bt = rv == 2 ? obs_block<T, 2>() : obs_block<T>();
    const int grid = (int)std::max<int64_t>(1, std::min<int64_t>((P.nchunks * G + bt - 1) / bt, (int64_t)S.n_sm * blocks_per_sm));
    const cudaError_t err = obs_dispatch<T, MODE>(P, np, G, rv, grid, smem, S.stream, w, x, yin, out, eout);
    WB_CUDA(err);
    S.gpu_launches++;
    return grid * (bt / 32);
}

// ---- hybrid operator apply ----
// G x = D'W D x splits by blocks of factor pairs.  The blocks between the primary factor
// P and the small factors S (those whose lane-group tables fit the observation pass's
// shared memory; their cross-tabulations have one entry per observation) stay implicit:
// prim_rows_kernel walks the observations.  Every other block is a cross-tabulation
// that the Schwarz setup already built (factor_pairs.rs:63-304, cross_tab.rs:514-664),
// much smaller than the observations, and is applied as CSR rows: the C_PO entries of
// each primary level inside prim_rows_kernel, and the rows of the other factors' dofs
// (their diagonal, C_OP, C_OO', C_OS, and for the S dofs D_S, C_SO, C_SS') by
// csr_rows_kernel.  Same sums as D'W D x up to the order of the additions.

// Design factors in the private tables of the pass for kp RHS of `elem` bytes, as a
// bit mask (0: none, or more than kPrimMaxS); np = their count.
uint32_t hybrid_smask(SolverImpl& S, int kp, size_t elem, int& np) {
    ObsParams P;
    np = obs_params_for(S, kp, elem, P);
    uint32_t m = 0;
    for (int sl = 1; sl < S.d.Q; ++sl)
        if (P.sink[sl] == SINK_PRIVATE) m |= 1u << S.dev_factor[sl];
    return (np >= 1 && np <= kPrimMaxS) ? m : 0u;
}

// The hybrid apply needs the factor-pair cross-tabulations of an additive Schwarz
// preconditioner (every pair of factors is a subdomain set) and the implicit operator.
bool hybrid_possible(const SolverImpl& S) {
    return !S.explicit_op && !S.precond_only && S.pc.kind == 1 && !S.subs.empty() && S.d.n > 0 && S.d.Q >= 2 &&
           S.d.n < ((int64_t)1 << 32);
}

void build_hybrid(SolverImpl& S, uint32_t smask) {
    const Design& d = S.d;
    const int P = S.primary;
    const int64_t nP = d.nlev[P], offP = d.off[P], m = d.ndofs;
    auto small = [&](int f) { return ((smask >> f) & 1u) != 0; };
    // each non-primary factor's diagonal comes from the first pair (in subdomain order)
    // that holds it: its levels are spread over that pair's components
    std::vector<int64_t> dsrc((size_t)d.Q, -1);
    for (const Subdomain& sd : S.subs)
        for (int f : {sd.q, sd.r})
            if (f != P && dsrc[f] < 0) dsrc[f] = (int64_t)sd.q * d.Q + sd.r;
    std::vector<int64_t> pcnt((size_t)nP + 1, 0), ocnt((size_t)m + 1, 0);
    std::vector<uint32_t> pcol, ocol;
    std::vector<double> pval, oval;
    // two passes: count the entries of every row, then place them
    for (int pass = 0; pass < 2; ++pass) {
        auto emit = [&](uint32_t row, uint32_t col, double v) {
            if ((int64_t)row >= offP && (int64_t)row < offP + nP) {
                const int64_t l = (int64_t)row - offP;
                if (pass == 0) { pcnt[l + 1]++; return; }
                const int64_t at = pcnt[l]++;
                pcol[at] = col;
                pval[at] = v;
            } else {
                if (pass == 0) { ocnt[row + 1]++; return; }
                const int64_t at = ocnt[row]++;
                ocol[at] = col;
                oval[at] = v;
            }
        };
        for (const Subdomain& sd : S.subs) {
            const int nq = sd.n_q();
            const bool implicit = (sd.q == P && small(sd.r)) || (sd.r == P && small(sd.q));
            if (!implicit) {
                const Csr& c = sd.ct.c;
                for (int32_t a = 0; a < c.nrows; ++a)
                    for (uint32_t e = c.ptr[a]; e < c.ptr[a + 1]; ++e) {
                        const uint32_t gq = sd.gidx[a], gr = sd.gidx[nq + c.idx[e]];
                        emit(gq, gr, c.val[e]);
                        emit(gr, gq, c.val[e]);
                    }
            }
            const int64_t pair = (int64_t)sd.q * d.Q + sd.r;
            if (sd.q != P && dsrc[sd.q] == pair)
                for (int32_t a = 0; a < nq; ++a) emit(sd.gidx[a], sd.gidx[a], sd.ct.dq[a]);
            if (sd.r != P && dsrc[sd.r] == pair)
                for (int32_t b = 0; b < sd.n_r(); ++b) emit(sd.gidx[nq + b], sd.gidx[nq + b], sd.ct.dr[b]);
        }
        if (pass == 0) {
            for (int64_t l = 0; l < nP; ++l) pcnt[l + 1] += pcnt[l];
            for (int64_t r = 0; r < m; ++r) ocnt[r + 1] += ocnt[r];
            pcol.resize((size_t)pcnt[nP]);
            pval.resize((size_t)pcnt[nP]);
            ocol.resize((size_t)ocnt[m]);
            oval.resize((size_t)ocnt[m]);
        } else {  // the cursors ended at the next row's start: shift back
            for (int64_t l = nP; l > 0; --l) pcnt[l] = pcnt[l - 1];
            pcnt[0] = 0;
            for (int64_t r = m; r > 0; --r) ocnt[r] = ocnt[r - 1];
            ocnt[0] = 0;
        }
    }
    // columns ascending within each row (fixed summation order)
    auto sort_rows = [&](const std::vector<int64_t>& ptr, std::vector<uint32_t>& col, std::vector<double>& val,
                         int64_t nrows) {
        const int64_t tasks = std::min<int64_t>(64, std::max<int64_t>(1, nrows / 4096));
        parallel_tasks((size_t)tasks, [&](size_t t) {
            std::vector<std::pair<uint32_t, double>> tmp;
            for (int64_t r = nrows * (int64_t)t / tasks; r < nrows * ((int64_t)t + 1) / tasks; ++r) {
                const int64_t a = ptr[r], b = ptr[r + 1];
                if (b - a < 2) continue;
                tmp.clear();
                for (int64_t e = a; e < b; ++e) tmp.emplace_back(col[e], val[e]);
                std::sort(tmp.begin(), tmp.end());
                for (int64_t e = a; e < b; ++e) col[e] = tmp[e - a].first, val[e] = tmp[e - a].second;
            }
        });
    };
    sort_rows(pcnt, pcol, pval, nP);
    sort_rows(ocnt, ocol, oval, m);
    // the non-empty other rows, compacted
    std::vector<uint32_t> rows;
    std::vector<int64_t> optr(1, 0);
    for (int64_t r = 0; r < m; ++r)
        if (ocnt[r + 1] > ocnt[r]) {
            rows.push_back((uint32_t)r);
            optr.push_back(ocnt[r + 1]);
        }
    auto H = std::make_unique<HybridDev>();
    H->smask = smask;
    std::vector<uint32_t> lp(S.lvl_ptr_h.begin(), S.lvl_ptr_h.end());
    H->lvl_ptr.upload(lp);
    H->pptr.upload(pcnt);
    H->pcol.upload(pcol);
    H->pval64.upload(pval);
    if (S.mixed()) H->pval32.upload_cast(pval);
    H->rows.upload(rows);
    H->optr.upload(optr);
    H->ocol.upload(ocol);
    H->oval64.upload(oval);
    if (S.mixed()) H->oval32.upload_cast(oval);
    const std::vector<CsrChunk> ch = make_chunks(optr, 0, (int64_t)rows.size(), 256, 1, true);
    H->ochunks.upload(ch);
    {
        std::vector<uint4> pcs;
        pcs.reserve((size_t)nP + 16);
        for (int64_t l = 0; l < nP; ++l) {
            const int64_t a = S.lvl_ptr_h[l], b = S.lvl_ptr_h[l + 1];
            const bool split = b - a > kMmaPiece;
            H->any_split = H->any_split || split;
            int64_t at = a;
            do {
                const int64_t e = std::min(b, at + kMmaPiece);
                pcs.push_back(make_uint4((uint32_t)l, (uint32_t)at, (uint32_t)e, (at == a ? 1u : 0u) | (split ? 2u : 0u)));
                at = e;
            } while (at < b);
        }
        H->pieces.upload(pcs);
        H->npieces = (int64_t)pcs.size();
    }
    H->nochunks = (int64_t)ch.size();
    H->nnz = (int64_t)pcol.size() + (int64_t)ocol.size();
    if (S.cg_exec) {  // a captured CG iteration may hold the old arrays
        WB_CUDA(cudaGraphExecDestroy(S.cg_exec));
        S.cg_exec = nullptr;
    }
    S.hyb = std::move(H);
}

template <typename T> const T* hyb_pval(const HybridDev& H);
template <> const double* hyb_pval<double>(const HybridDev& H) { return H.pval64.p; }
template <> const float* hyb_pval<float>(const HybridDev& H) { return H.pval32.p; }
template <typename T> const T* hyb_oval(const HybridDev& H);
template <> const double* hyb_oval<double>(const HybridDev& H) { return H.oval64.p; }
template <> const float* hyb_oval<float>(const HybridDev& H) { return H.oval32.p; }

// y = G x by the hybrid apply (S.hyb built for the pass's small factors at this kp and
// precision): zero the accumulated outputs, the primary-major pass, then the other rows.
// The small factors' columns in prim_mma_kernel's tile (each padded to 8); false when the
// tile does not apply (kp other than 16, or more than kMmaMaxCols columns).
bool mma_layout(SolverImpl& S, int kp, size_t elem, PrimMmaParams& M) {
    if (kp != kMmaKP) return false;
    ObsParams O;
    const int np = obs_params_for(S, kp, elem, O);
    if (np < 1 || np > kPrimMaxS) return false;
    M = PrimMmaParams{};
    M.off_p = S.d.off[S.primary];
    M.nsmall = np;
    int j = 0, col = 0;
    for (int sl = 1; sl < S.d.Q; ++sl) {
        if (O.sink[sl] != SINK_PRIVATE) continue;
        M.codes_s[j] = S.codes.p + (size_t)sl * O.ns;
        M.off_s[j] = O.off[sl];
        M.nlev_s[j] = (int32_t)S.d.nlev[S.dev_factor[sl]];
        M.col_s[j] = col;
        col += (M.nlev_s[j] + 7) / 8 * 8;
        ++j;
    }
    M.wcols = col;
    return col <= kMmaMaxCols;
}

template <typename T>
void launch_hybrid(SolverImpl& S, int kp, const T* w, const T* x, T* y, bool mma = false) {
    const HybridDev& H = *S.hyb;
    ObsParams O;
    const int np = obs_params_for(S, kp, sizeof(T), O);
    const int G = group_for(kp);
    PrimMmaParams M;
    if (mma && mma_layout(S, kp, sizeof(T), M)) {
        M.pieces = H.pieces.p;
        M.npieces = H.npieces;
        M.pptr = H.pptr.p;
        M.pcol = H.pcol.p;
        const size_t mrow = (size_t)S.d.ndofs;
        if (H.any_split) {
            WB_CUDA(cudaMemsetAsync(y, 0, mrow * kp * sizeof(T), S.stream));
        } else {
            const size_t a = (size_t)M.off_p * kp, b = (size_t)(M.off_p + S.d.nlev[S.primary]) * kp;
            if (a > 0) WB_CUDA(cudaMemsetAsync(y, 0, a * sizeof(T), S.stream));
            if (mrow * kp > b) WB_CUDA(cudaMemsetAsync(y + b, 0, (mrow * kp - b) * sizeof(T), S.stream));
        }
        const int64_t tasks = (H.npieces + 7) / 8;
        const int grid = (int)std::max<int64_t>(1, std::min<int64_t>((tasks + 7) / 8, (int64_t)S.n_sm * 2));
        prim_mma_kernel<T><<<grid, 256, 0, S.stream>>>(M, w, hyb_pval<T>(H), x, y);
        WB_CUDA(cudaGetLastError());
        if (H.nochunks > 0) {
            const int64_t need = (H.nochunks * 32 + kBlock - 1) / kBlock;
            auto kern = csr_rows_kernel<T, 4, EPI_ACC>;
            kern<<<S.fit(need, (const void*)kern), kBlock, 0, S.stream>>>(H.ochunks.p, H.nochunks, H.rows.p, H.optr.p,
                                                                          H.ocol.p, hyb_oval<T>(H), nullptr, x, y, kp);
            WB_CUDA(cudaGetLastError());
        }
        S.gpu_launches += 2;
        return;
    }
    const int ci = 1;  // 32 observations per chunk
    PrimParams P{};
    P.ns = O.ns;
    P.nsmall = np;
    P.priv_stride = O.priv_stride;
    P.off_p = S.d.off[S.primary];
    const int64_t gpb = obs_block<T>() / G;
    int64_t used = gpb * O.priv_stride;
    int j = 0;
    for (int sl = 1; sl < S.d.Q; ++sl) {
        if (O.sink[sl] != SINK_PRIVATE) continue;
        P.codes_s[j] = S.codes.p + (size_t)sl * O.ns;
        P.off_s[j] = O.off[sl];
        P.nlev_s[j] = (int32_t)S.d.nlev[S.dev_factor[sl]];
        P.priv_base[j] = O.smem_base[sl];
        used = (used + 3) / 4 * 4;
        P.xs_base[j] = (int32_t)used;
        used += (int64_t)P.nlev_s[j] * kp;
        ++j;
    }
    P.smem_elems = (int32_t)used;
    P.chunks = S.chunk_tab[ci].p;
    P.nchunks = S.nchunk_tab[ci];
    P.lvl_ptr = H.lvl_ptr.p;
    P.pptr = H.pptr.p;
    P.pcol = H.pcol.p;
    const bool split = S.split_tab[ci];
    const size_t mrow = (size_t)S.d.ndofs;
    if (split) {
        WB_CUDA(cudaMemsetAsync(y, 0, mrow * kp * sizeof(T), S.stream));
    } else {  // every row but the primary factor's is accumulated
        const size_t a = (size_t)P.off_p * kp, b = (size_t)(P.off_p + S.d.nlev[S.primary]) * kp;
        if (a > 0) WB_CUDA(cudaMemsetAsync(y, 0, a * sizeof(T), S.stream));
        if (mrow * kp > b) WB_CUDA(cudaMemsetAsync(y + b, 0, (mrow * kp - b) * sizeof(T), S.stream));
    }
    const size_t smem = (size_t)used * sizeof(T);
    const int bt = obs_block<T>();
    const int grid = (int)std::max<int64_t>(1, std::min<int64_t>((P.nchunks * G + bt - 1) / bt, (int64_t)S.n_sm * 2));
    auto go = [&](auto kern) {
        if (smem > 48 * 1024) WB_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        kern<<<grid, bt, smem, S.stream>>>(P, w, hyb_pval<T>(H), x, y);
    };
    WB_DISPATCH_G(G, {
        if (np == 1) go(prim_rows_kernel<T, GV, 1>);
        else go(prim_rows_kernel<T, GV, 2>);
    });
    WB_CUDA(cudaGetLastError());
    if (H.nochunks > 0) {
        const int64_t need = (H.nochunks * 32 + kBlock - 1) / kBlock;  // one warp per chunk
        WB_DISPATCH_G(G, {
            auto kern = csr_rows_kernel<T, GV, EPI_ACC>;
            kern<<<S.fit(need, (const void*)kern), kBlock, 0, S.stream>>>(H.ochunks.p, H.nochunks, H.rows.p, H.optr.p,
                                                                          H.ocol.p, hyb_oval<T>(H), nullptr, x, y, kp);
        });
        WB_CUDA(cudaGetLastError());
    }
    S.gpu_launches += 2;
}

// Autotuner of the observation pass's block shape (the dominant kernel): the first time a
// solver needs the pass for kp RHS in a precision, each candidate (16, 32 or 64
// observations per chunk; 1 or 2 resident blocks per SM) runs twice on the solver's own
// design, timed with events on its stream after a warm-up launch, and the fastest is
// kept.  The choice is cached for the process per shape class (log2 of the observation
// count, factor count, kp, element size), so that solvers of the same class (the
// problems of an uneven batch) reuse it without timing.  Runs outside any stream
// capture; x is read and y overwritten.
std::mutex g_obs_tune_mu;
std::map<std::array<int64_t, 4>, int32_t> g_obs_tune;
// same classes: hybrid apply off (0), on with prim_rows_kernel (1) or with prim_mma_kernel (2)
std::map<std::array<int64_t, 4>, int32_t> g_hyb_tune;

bool hybrid_in_use(const SolverImpl& S) {
    for (const auto& c : S.hyb_on)
        for (int32_t v : c)
            if (v >= 1) return true;
    return false;
}

// Whether the operator apply for kp RHS in T runs as the hybrid apply, and with which
// primary-major kernel: decided once per shape class by timing both forms (the tensor-core
// one where it applies) against the tuned observation pass (`best_ms`; < 0: take the
// class's cached decision).  x is read and y overwritten.
template <typename T>
void hybrid_decide(SolverImpl& S, int kp, const T* w, const T* x, T* y, float best_ms,
                   const std::array<int64_t, 4>& key) {
    int32_t& on = S.hyb_on[kp_class(kp)][sizeof(T) == 8 ? 1 : 0];
    if (on >= 0) return;
    on = 0;
    int np = 0;
    const uint32_t smask = hybrid_possible(S) ? hybrid_smask(S, kp, sizeof(T), np) : 0u;
    if (smask == 0) return;
    int32_t cached = -1;
    {
        std::lock_guard<std::mutex> lk(g_obs_tune_mu);
        const auto it = g_hyb_tune.find(key);
        if (it != g_hyb_tune.end()) cached = it->second;
    }
    if (best_ms < 0.f && cached == 0) return;
    if (S.hyb && S.hyb->smask != smask && hybrid_in_use(S)) return;  // one set of arrays per solver
    if (!S.hyb || S.hyb->smask != smask) build_hybrid(S, smask);
    if (best_ms < 0.f && cached >= 1) {
        on = cached;
        return;
    }
    PrimMmaParams M;
    const bool mma_ok = mma_layout(S, kp, sizeof(T), M);
    cudaEvent_t e0, e1;
    WB_CUDA(cudaEventCreate(&e0));
    WB_CUDA(cudaEventCreate(&e1));
    float ms_v[3] = {0.f, 0.f, 0.f};
    for (int sweep = 0; sweep < 2; ++sweep)
        for (int v = 1; v <= (mma_ok ? 2 : 1); ++v) {
            launch_hybrid<T>(S, kp, w, x, y, v == 2);
            WB_CUDA(cudaEventRecord(e0, S.stream));
            for (int rep = 0; rep < 2; ++rep) launch_hybrid<T>(S, kp, w, x, y, v == 2);
            WB_CUDA(cudaEventRecord(e1, S.stream));
            WB_CUDA(cudaEventSynchronize(e1));
            float ms = 0.f;
            WB_CUDA(cudaEventElapsedTime(&ms, e0, e1));
            ms *= 0.5f;
            if (sweep == 0 || ms < ms_v[v]) ms_v[v] = ms;
        }
    WB_CUDA(cudaEventDestroy(e0));
    WB_CUDA(cudaEventDestroy(e1));
    // the tensor-core form only when it is clearly faster (3%): the two are within timing
    // noise of each other on the panels measured
    const int vb = (mma_ok && ms_v[2] < 0.97f * ms_v[1]) ? 2 : 1;
    const float ms_best = ms_v[vb];
    S.hyb_ms[kp_class(kp)][sizeof(T) == 8 ? 1 : 0] = ms_best;
    on = (best_ms < 0.f || ms_best < best_ms) ? vb : 0;
    if (!on && !hybrid_in_use(S)) S.hyb.reset();
    std::lock_guard<std::mutex> lk(g_obs_tune_mu);
    g_hyb_tune.emplace(key, on);
}

template <typename T>
void obs_autotune(SolverImpl& S, int kp, const T* w, const T* x, T* y) {
    int32_t& choice = S.obs_choice[kp_class(kp)][sizeof(T) == 8 ? 1 : 0];
    if (choice >= 0 || S.d.n == 0) return;
    int64_t lg = 0;
    for (int64_t v = S.d.n; v > 1; v >>= 1) ++lg;
    const std::array<int64_t, 4> key{lg, (int64_t)S.d.Q, (int64_t)kp, (int64_t)sizeof(T)};
    {
        std::lock_guard<std::mutex> lk(g_obs_tune_mu);
        const auto it = g_obs_tune.find(key);
        if (it != g_obs_tune.end()) choice = it->second;
    }
    if (choice >= 0) {  // tuned by a solver of the same class: this one's global copies
        if (choice % (2 * kObsShapes) >= kObsShapes) grow_obs_hot(S, obs_hot_bytes(S, kp, sizeof(T)));
        hybrid_decide<T>(S, kp, w, x, y, -1.f, key);
        return;
    }
    cudaEvent_t e0, e1;
    WB_CUDA(cudaEventCreate(&e0));
    WB_CUDA(cudaEventCreate(&e1));
    float best = 0.f;
    int32_t best_c = 3;  // 32 observations per chunk, 2 blocks per SM
    // candidates with global hot tables when the design has hot levels (their copies are
    // allocated here, outside any stream capture)
    const size_t hot = obs_hot_bytes(S, kp, sizeof(T));
    grow_obs_hot(S, hot);
    std::vector<int32_t> cands;
    const bool wide = obs_wide_for(S, kp, sizeof(T));
    for (int32_t c = 0; c < (hot ? 2 * kObsShapes : kObsShapes); ++c) {
        cands.push_back(c);
        if (wide) cands.push_back(2 * kObsShapes + c);
    }
    const int32_t nc = (int32_t)cands.size();
    // two sweeps over the candidates, the second in reverse order; each keeps its best
    float* tms = S.obs_tune_ms[kp_class(kp)][sizeof(T) == 8 ? 1 : 0];
    for (int32_t c = 0; c < 4 * kObsShapes; ++c) tms[c] = 0.f;
    for (int32_t it = 0; it < 2 * nc; ++it) {
        const int32_t c = cands[it < nc ? it : 2 * nc - 1 - it];
        choice = c;
        launch_obs<T, OBS_GRAM>(S, kp, w, x, nullptr, y, nullptr);
        WB_CUDA(cudaEventRecord(e0, S.stream));
        for (int rep = 0; rep < 2; ++rep) launch_obs<T, OBS_GRAM>(S, kp, w, x, nullptr, y, nullptr);
        WB_CUDA(cudaEventRecord(e1, S.stream));
        WB_CUDA(cudaEventSynchronize(e1));
        float ms = 0.f;
        WB_CUDA(cudaEventElapsedTime(&ms, e0, e1));
        ms *= 0.5f;
        if (tms[c] == 0.f || ms < tms[c]) tms[c] = ms;
    }
    for (int32_t i = 0; i < nc; ++i)
        if (i == 0 || tms[cands[i]] < best) {
            best = tms[cands[i]];
            best_c = cands[i];
        }
    WB_CUDA(cudaEventDestroy(e0));
    WB_CUDA(cudaEventDestroy(e1));
    choice = best_c;
    {
        std::lock_guard<std::mutex> lk(g_obs_tune_mu);
        g_obs_tune.emplace(key, best_c);
    }
    hybrid_decide<T>(S, kp, w, x, y, best, key);
}

// Dot partials over rows (at most 2 blocks per SM: few partials to reduce).
template <typename TA, typename TB>
void launch_dot(SolverImpl& S, const TA* a, const TB* b, int64_t rows, int kp, double* part, int& nb) {
    const int G = group_for(kp);
    nb = S.nblk(rows, G, 2);
    WB_DISPATCH_G(G, dot_kernel<TA, TB, GV><<<nb, kBlock, 0, S.stream>>>(a, b, rows, kp, part));
    WB_CUDA(cudaGetLastError());
    S.gpu_launches++;
}

// red[c] = sum_b part[b*kp + c] (fixed order per c; deterministic).  Each thread sums a
// strided subset of the partials with eight independent accumulators, so that eight
// loads are in flight at a time, and combines them in a fixed order.
__device__ __forceinline__ void reduce_parts_body(const double* __restrict__ part, int nb, int kp,
                                                  double* __restrict__ red) {
    __shared__ double sm[kBlock];
    const int t = threadIdx.x;
    const int J = blockDim.x / kp;
    double s = 0.0;
    if (t < J * kp) {
        const int c = t % kp, j = t / kp;
        double a[8] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
        int b = j;
        for (; b + 7 * J < nb; b += 8 * J) {
#pragma unroll
            for (int u = 0; u < 8; ++u) a[u] += part[(size_t)(b + u * J) * kp + c];
        }
        for (; b < nb; b += J) a[0] += part[(size_t)b * kp + c];
        s = ((a[0] + a[1]) + (a[2] + a[3])) + ((a[4] + a[5]) + (a[6] + a[7]));
    }
    sm[t] = s;
    __syncthreads();
    if (t < kp) {
        double a = 0.0;
        for (int j = 0; j < J; ++j) a += sm[j * kp + t];
        red[t] = a;
    }
}

__global__ void reduce_parts_kernel(const double* __restrict__ part, int nb, int kp, double* __restrict__ red) {
    reduce_parts_body(part, nb, kp, red);
}

void launch_reduce(SolverImpl& S, const double* part, int nb, int kp, double* red) {
    reduce_parts_kernel<<<1, kBlock, 0, S.stream>>>(part, nb, kp, red);
    WB_CUDA(cudaGetLastError());
    S.gpu_launches++;
}

template <typename T> T* loc_buf(SolverImpl& S);
template <> double* loc_buf<double>(SolverImpl& S) { return S.ws.vloc.p; }
template <> float* loc_buf<float>(SolverImpl& S) { return S.ws.floc.p; }
template <typename T> T* cbuf(SolverImpl& S);
template <> double* cbuf<double>(SolverImpl& S) { return S.ws.cbuf.p; }
template <> float* cbuf<float>(SolverImpl& S) { return S.ws.fcbuf.p; }
template <typename T> T* core_buf(SolverImpl& S);
template <> double* core_buf<double>(SolverImpl& S) { return S.ws.core_tmp.p; }
template <> float* core_buf<float>(SolverImpl& S) { return S.ws.fcore_tmp.p; }
template <typename T> std::vector<StageDev<T>>& stages(SolverImpl& S);
template <> std::vector<StageDev<double>>& stages<double>(SolverImpl& S) { return S.stages64; }
template <> std::vector<StageDev<float>>& stages<float>(SolverImpl& S) { return S.stages32; }
template <typename T> const T* gram_val(SolverImpl& S);
template <> const double* gram_val<double>(SolverImpl& S) { return S.g_val64.p; }
template <> const float* gram_val<float>(SolverImpl& S) { return S.g_val32.p; }
template <typename T> T* rwork_buf(SolverImpl& S);
template <> double* rwork_buf<double>(SolverImpl& S) { return S.ws.rwork.p; }
template <> float* rwork_buf<float>(SolverImpl& S) { return S.ws.frwork.p; }

template <typename T, int EPI>
void launch_csr(SolverImpl& S, CsrDev<T>& c, int64_t ch0, int64_t ch1, const T* src, T* dst, int kp) {
    const int64_t nch = ch1 - ch0;
    if (nch <= 0) return;
    const int G = group_for(kp);
    const int64_t need = (nch * 32 + kBlock - 1) / kBlock;  // one warp per chunk
    WB_DISPATCH_G(G, {
        auto kern = csr_rows_kernel<T, GV, EPI>;
        kern<<<S.fit(need, (const void*)kern), kBlock, 0, S.stream>>>(c.chunks.p + ch0, nch, c.row_slot.p, c.ptr.p,
                                                                      c.col.p, c.val.p, c.rscale.p, src, dst, kp);
    });
    WB_CUDA(cudaGetLastError());
    S.gpu_launches++;
}

// y = G x for the Krylov methods and the refinement residual.  Implicit: one pass over
// the observations.  Explicit (solver.rs:103-121, 350-360: when the solver holds the
// assembled Gramian): y = 0, then the CSR rows of G, one warp per row, the pieces of
// long rows added atomically.
template <typename T>
void launch_gram_acc(SolverImpl& S, int kp, const T* x, T* y);
template <typename T>
void launch_gram(SolverImpl& S, int kp, const T* w, const T* x, T* y) {
    if (!S.explicit_op) {
        const int32_t hv = S.hyb_on[kp_class(kp)][sizeof(T) == 8 ? 1 : 0];
        if (hv >= 1 && S.hyb) {
            launch_hybrid<T>(S, kp, w, x, y, hv == 2);
            return;
        }
        launch_obs<T, OBS_GRAM>(S, kp, w, x, nullptr, y, nullptr);
        return;
    }
    WB_CUDA(cudaMemsetAsync(y, 0, sizeof(T) * (size_t)S.d.ndofs * kp, S.stream));
    launch_gram_acc<T>(S, kp, x, y);
}
// y += G x with the assembled Gramian
template <typename T>
void launch_gram_acc(SolverImpl& S, int kp, const T* x, T* y) {
    const int G = group_for(kp);
    const int64_t need = (S.g_nchunks * 32 + kBlock - 1) / kBlock;  // one warp per chunk
    WB_DISPATCH_G(G, {
        auto kern = csr_rows_kernel<T, GV, EPI_ACC>;
        kern<<<S.fit(need, (const void*)kern), kBlock, 0, S.stream>>>(S.g_chunks.p, S.g_nchunks, S.g_rows.p, S.g_ptr.p,
                                                                      S.g_idx.p, gram_val<T>(S), nullptr, x, y, kp);
    });
    WB_CUDA(cudaGetLastError());
    S.gpu_launches++;
}

// Spin limit of the barrier waits under the test hook (about a millisecond per wait).
constexpr unsigned kInjectedBarrierSpins = 1u << 12;

// Blocks of the thread-block cluster that runs the small last levels of an AC sweep
// (csr_levels_cluster_kernel), per kernel: 16 (non-portable size) or 8 when the device
// can hold such a cluster of 1024-thread blocks, else 0 (no cluster path).
inline int level_cluster_blocks(const void* kern) {
    static std::mutex mu;
    static std::unordered_map<const void*, int> cache;
    std::lock_guard<std::mutex> lk(mu);
    const auto it = cache.find(kern);
    if (it != cache.end()) return it->second;
    int best = 0;
    if (cudaFuncSetAttribute(kern, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) != cudaSuccess) cudaGetLastError();
    for (int cb : {16, 8}) {
        cudaLaunchConfig_t cfg = {};
        cudaLaunchAttribute at[1];
        at[0].id = cudaLaunchAttributeClusterDimension;
        at[0].val.clusterDim.x = (unsigned)cb;
        at[0].val.clusterDim.y = 1;
        at[0].val.clusterDim.z = 1;
        cfg.gridDim = dim3(cb);
        cfg.blockDim = dim3(kLevelClusterBlock);
        cfg.attrs = at;
        cfg.numAttrs = 1;
        int nc = 0;
        if (cudaOccupancyMaxActiveClusters(&nc, kern, &cfg) != cudaSuccess) {
            cudaGetLastError();
            nc = 0;
        }
        if (nc >= 1) {
            best = cb;
            break;
        }
    }
    cache.emplace(kern, best);
    return best;
}

// All levels of one AC sweep direction of a stage: the large levels as one cooperative
// launch (grid barriers between levels), the trailing run of small levels (the last
// rounds of the factor: a few hundred rows each) as one launch of a single thread-block
// cluster, whose hardware barrier separates them.  The forward direction runs the large
// levels first, the backward one the small levels first.  Without cooperative launches,
// one launch per level.
template <typename T, int EPI>
void launch_sweep(SolverImpl& S, CsrDev<T>& c, const std::vector<int64_t>& lp, const int64_t* lp_d, bool backward,
                  T* v, int kp, int which) {
    const int nlev = (int)lp.size() - 1;
    if (nlev <= 0) return;
    if (!S.coop || nlev == 1) {
        if (!backward)
            for (int l = 0; l < nlev; ++l) launch_csr<T, EPI>(S, c, lp[l], lp[l + 1], v, v, kp);
        else
            for (int l = nlev - 1; l >= 0; --l) launch_csr<T, EPI>(S, c, lp[l], lp[l + 1], v, v, kp);
        return;
    }
    const int G = group_for(kp);
    unsigned* bar = S.ws.sweep_bar.p + which;
    int* err = S.ws.sweep_err.p;
    const CsrChunk* ch = c.chunks.p;
    const uint32_t* rs = c.row_slot.p;
    const int64_t* pt = c.ptr.p;
    const uint32_t* cl = c.col.p;
    const T* vl = c.val.p;
    const T* sc = c.rscale.p;
    int bw = backward ? 1 : 0, k = kp;
    // the longest run [a, b) of consecutive small levels (at least two, so that a barrier
    // is saved); the levels before and after it run on the grid
    int a = 0, b = 0;
    const int64_t max_chunks = S.sweep_cluster_chunks;
    if (max_chunks > 0 && !S.inject_sweep_timeout) {
        for (int l = 0; l < nlev;) {
            if (lp[l + 1] - lp[l] > max_chunks) {
                ++l;
                continue;
            }
            int e = l;
            while (e < nlev && lp[e + 1] - lp[e] <= max_chunks) ++e;
            if (e - l > b - a) a = l, b = e;
            l = e;
        }
        if (b - a < 2) a = b = 0;
    }
    auto grid_part = [&](auto kern, int l0, int nl) {  // levels [l0, l0 + nl)
        if (nl <= 0) return;
        if (nl == 1) {
            launch_csr<T, EPI>(S, c, lp[l0], lp[l0 + 1], v, v, kp);
            return;
        }
        WB_CUDA(cudaMemsetAsync(bar, 0, sizeof(unsigned), S.stream));
        const int grid = resident_per_sm((const void*)kern) * S.n_sm;  // every block resident
        // a test can make every barrier wait for one block more than the grid has, with a
        // short limit: the waits run out, the error flag is set, the launch ends
        unsigned extra = S.inject_sweep_timeout ? 1u : 0u;
        unsigned spins = S.inject_sweep_timeout ? kInjectedBarrierSpins : kBarrierSpins;
        void* args[] = {(void*)&ch, (void*)&lp_d, (void*)&l0, (void*)&nl, (void*)&bw, (void*)&rs, (void*)&pt,
                        (void*)&cl, (void*)&vl, (void*)&sc, (void*)&v, (void*)&k, (void*)&bar, (void*)&err,
                        (void*)&extra, (void*)&spins};
        WB_CUDA(cudaLaunchCooperativeKernel((const void*)kern, dim3(grid), dim3(kBlock), args, 0, S.stream));
        S.gpu_launches++;
    };
    auto cluster_part = [&](auto kern) {  // levels [a, b)
        if (b == a) return;
        const int cb = level_cluster_blocks((const void*)kern);
        cudaLaunchConfig_t cfg = {};
        cudaLaunchAttribute at[1];
        at[0].id = cudaLaunchAttributeClusterDimension;
        at[0].val.clusterDim.x = (unsigned)cb;
        at[0].val.clusterDim.y = 1;
        at[0].val.clusterDim.z = 1;
        cfg.gridDim = dim3(cb);
        cfg.blockDim = dim3(kLevelClusterBlock);
        cfg.stream = S.stream;
        cfg.attrs = at;
        cfg.numAttrs = 1;
        WB_CUDA(cudaLaunchKernelEx(&cfg, kern, ch, lp_d, a, b - a, bw, rs, pt, cl, vl, sc, v, k));
        S.gpu_launches++;
    };
    WB_DISPATCH_G(G, {
        auto gk = csr_levels_kernel<T, GV, EPI>;
        auto ck = csr_levels_cluster_kernel<T, GV, EPI>;
        if (b > a && level_cluster_blocks((const void*)ck) == 0) a = b = 0;  // no cluster: all levels on the grid
        if (b == a) {
            grid_part(gk, 0, nlev);
        } else if (!backward) {
            grid_part(gk, 0, a);
            cluster_part(ck);
            grid_part(gk, b, nlev - b);
        } else {
            grid_part(gk, b, nlev - b);
            cluster_part(ck);
            grid_part(gk, 0, a);
        }
    });
}

// The host learns of a grid-barrier timeout here (after the work that set it is done):
// true when a local solve did not complete since the last check (the flag is cleared).
bool sweeps_failed(SolverImpl& S) {
    if (!S.coop || !S.ws.sweep_err.p) return false;
    int32_t e = 0;
    read_small(S, &e, S.ws.sweep_err.p, sizeof(int32_t));
    if (e) WB_CUDA(cudaMemset(S.ws.sweep_err.p, 0, sizeof(int32_t)));
    return e != 0;
}

// The local solves of one stage from the restriction input r up to the kept solution
// in v and the subdomain sums in msum (see kernels.cuh for the algebra).
template <typename T>
SubMeans stage_local_solve(SolverImpl& S, StageDev<T>& st, const T* r, T* v, int kp) {
    const int G = group_for(kp);
    double* msum = S.ws.msum.p;
    const size_t ms = (size_t)S.max_nsub * kp;
    double *S0 = msum, *SB = msum + ms, *M1 = msum + 2 * ms, *M2 = msum + 3 * ms;
    WB_CUDA(cudaMemsetAsync(msum, 0, sizeof(double) * 4 * ms, S.stream));
    constexpr int kSpb = 256;  // keep-list entries per block of the segmented sums (4 per lane group)
    {
        constexpr int kSlotsPerBlock = 1024;  // 16 slots per lane group
        const int grid = (int)std::max<int64_t>(1, (st.nslots + kSlotsPerBlock - 1) / kSlotsPerBlock);
        WB_DISPATCH_G(G, schwarz_sums_kernel<T, GV><<<grid, kBlock, 0, S.stream>>>(
                             st.nslots, kSlotsPerBlock, st.gidx.p, st.spou.p, st.invd.p, st.sub_of.p, r, kp, S0, SB));
    }
    if (st.nkeep > 0) {
        const int grid = S.nblk(st.nkeep, G);
        WB_DISPATCH_G(G, keep_init_kernel<T, GV><<<grid, kBlock, 0, S.stream>>>(
                             st.nkeep, st.keep_slots.p, st.gidx.p, st.spou.p, st.rho.p, st.sub_of.p, st.sub_nloc.p, S0, r,
                             v, kp));
        launch_csr<T, EPI_ACC>(S, st.keep, 0, st.keep.nchunks, r, v, kp);
        const int gs = (int)std::max<int64_t>(1, (st.nkeep + kSpb - 1) / kSpb);
        WB_DISPATCH_G(G, keep_sum_kernel<T, GV><<<gs, kBlock, 0, S.stream>>>(st.nkeep, kSpb, st.keep_slots.p, st.rho.p, 0,
                                                                              st.sub_of.p, v, kp, M1));
        WB_DISPATCH_G(G, keep_center_kernel<T, GV><<<grid, kBlock, 0, S.stream>>>(st.nkeep, st.keep_slots.p, st.sub_of.p,
                                                                                 st.sub_nkeep.p, M1, v, kp));
    }
    WB_CUDA(cudaGetLastError());
    S.gpu_launches += 4;
    // reduced solves: dense anchored Cholesky and approximate Cholesky sweeps
    if (st.ndense > 0) {
        const int64_t warps = (int64_t)st.ndense * kp;
        const int grid = (int)((warps * 32 + kBlock - 1) / kBlock);
        dense_solve_kernel<T><<<grid, kBlock, 0, S.stream>>>(st.ndense, st.dn_keep0.p, st.dn_n.p, st.dn_loff.p, st.dn_L.p,
                                                             v, kp);
        WB_CUDA(cudaGetLastError());
        S.gpu_launches++;
    }
    launch_sweep<T, EPI_ACC>(S, st.fwd, st.fwd_lp, st.fwd_lp_d.p, false, v, kp, 0);
    if (st.ncore_blocks > 0) {
        T* cin = core_buf<T>(S);  // the cores' input rows, contiguous
        core_stage_kernel<T><<<S.nblk(st.core_total * kp, 1), kBlock, 0, S.stream>>>(st.core_total, st.core_slot.p, v,
                                                                                     cin, kp);
        WB_DISPATCH_G(G, core_gemv_kernel<T, GV><<<st.ncore_blocks, kBlock, 0, S.stream>>>(
                             st.core_of_block.p, st.row0_of_block.p, st.core_n.p, st.core_slot_off.p, st.core_slot.p,
                             st.core_z_off.p, st.core_z.p, cin, v, kp));
        WB_CUDA(cudaGetLastError());
        S.gpu_launches += 2;
    }
    launch_sweep<T, EPI_PIVOT>(S, st.bwd, st.bwd_lp, st.bwd_lp_d.p, true, v, kp, 1);
    // sum over the kept solution with the back-substitution weights -> final means
    if (st.nkeep > 0) {
        const int gs = (int)std::max<int64_t>(1, (st.nkeep + kSpb - 1) / kSpb);
        WB_DISPATCH_G(G, keep_sum_kernel<T, GV><<<gs, kBlock, 0, S.stream>>>(st.nkeep, kSpb, st.keep_slots.p, st.rho.p, 1,
                                                                              st.sub_of.p, v, kp, M2));
        WB_CUDA(cudaGetLastError());
        S.gpu_launches++;
    }
    return SubMeans{st.sub_nloc.p, S0, SB, M2, st.sub_I.p};
}

// z = M^{-1} r.  With part non-null also the block partials of r.z (nb_part blocks).
template <typename T>
void apply_precond(SolverImpl& S, const T* r, T* z, int kp, double* part, int& nb_part) {
    const int64_t m = S.d.ndofs;
    const int G = group_for(kp);
    auto& sts = stages<T>(S);
    T* v = loc_buf<T>(S);
    nb_part = 0;
    if (S.pc.kind == 0 || sts.empty()) {
        if (S.pc.kind == 0) WB_CUDA(cudaMemcpyAsync(z, r, sizeof(T) * m * kp, cudaMemcpyDeviceToDevice, S.stream));
        else WB_CUDA(cudaMemsetAsync(z, 0, sizeof(T) * m * kp, S.stream));
        if (part) launch_dot<T, T>(S, r, z, m, kp, part, nb_part);
        return;
    }
    if (S.pc.kind == 1) {
        StageDev<T>& st = sts[0];
        const SubMeans M = stage_local_solve<T>(S, st, r, v, kp);
        double* mm = S.ws.msum.p + (size_t)4 * S.max_nsub * kp;  // [nsub][2][kp]
        const int64_t nm = (int64_t)st.nsub * kp;
        sub_means_kernel<<<(unsigned)((nm + kBlock - 1) / kBlock), kBlock, 0, S.stream>>>(st.nsub, kp, M, mm);
        // latency-bound gathers: as many resident blocks as registers allow, one wave
        WB_DISPATCH_G(G, {
            auto kern = prolong_kernel<T, GV>;
            nb_part = S.fit(((int64_t)m * G + kBlock - 1) / kBlock, (const void*)kern);
            kern<<<nb_part, kBlock, 0, S.stream>>>(m, st.gptr.p, st.gslot.p, st.gsub.p, st.gspou.p, st.ginvd.p,
                                                   st.gbs_ptr.p, st.gbs_cnt.p, st.gbs_col.p, st.gbs_val.p, mm, v, r, z,
                                                   kp, part, S.ws.sweep_err.p);
        });
        WB_CUDA(cudaGetLastError());
        S.gpu_launches += 2;
        if (!part) nb_part = 0;
        return;
    }
    // multiplicative: sequential stages (one per factor pair), residual updated after each
    T* rw = rwork_buf<T>(S);
    T* cb = cbuf<T>(S);  // -(this stage's correction) on global dofs
    WB_CUDA(cudaMemcpyAsync(rw, r, sizeof(T) * m * kp, cudaMemcpyDeviceToDevice, S.stream));
    WB_CUDA(cudaMemsetAsync(z, 0, sizeof(T) * m * kp, S.stream));
    for (auto& st : sts) {
        const SubMeans M = stage_local_solve<T>(S, st, rw, v, kp);
        const int grid = S.nblk(st.nslots, G);
        WB_CUDA(cudaMemsetAsync(cb, 0, sizeof(T) * m * kp, S.stream));
        WB_DISPATCH_G(G, mult_sol_kernel<T, GV><<<grid, kBlock, 0, S.stream>>>(
                             st.nslots, st.gidx.p, st.sub_of.p, st.spou.p, st.invd.p, st.bs_ptr.p, st.bs_col.p,
                             st.bs_val.p, M, v, rw, z, cb, kp));
        WB_CUDA(cudaGetLastError());
        S.gpu_launches++;
        launch_gram_acc<T>(S, kp, cb, rw);  // r_work -= G c
    }
    if (S.coop && S.ws.sweep_err.p) {  // a local solve that did not complete: z = NaN
        nan_on_failure_kernel<T><<<S.nblk(m * kp, 1), kBlock, 0, S.stream>>>(z, m * kp, S.ws.sweep_err.p);
        WB_CUDA(cudaGetLastError());
        S.gpu_launches++;
    }
    if (part) launch_dot<T, T>(S, r, z, m, kp, part, nb_part);
}

template <typename T> const T* coarse_basis(SolverImpl& S);
template <> const double* coarse_basis<double>(SolverImpl& S) { return S.coarse_z64.p; }
template <> const float* coarse_basis<float>(SolverImpl& S) { return S.coarse_z32.p; }
template <typename T> const T* coarse_gbasis(SolverImpl& S);
template <> const double* coarse_gbasis<double>(SolverImpl& S) { return S.coarse_gz64.p; }
template <> const float* coarse_gbasis<float>(SolverImpl& S) { return S.coarse_gz32.p; }
template <typename T> DArr<T>& coarse_tmp(SolverImpl& S);
template <> DArr<double>& coarse_tmp<double>(SolverImpl& S) { return S.coarse_tmp64; }
template <> DArr<float>& coarse_tmp<float>(SolverImpl& S) { return S.coarse_tmp32; }
int coarse_blocks(const SolverImpl& S) {
    const int64_t tiles = (S.d.ndofs + kCoarseTileRows - 1) / kCoarseTileRows;
    return (int)std::max<int64_t>(1, std::min<int64_t>(tiles, (int64_t)S.n_sm * 2));
}

// The CG preconditioner: z = M^{-1} r, or with a coarse space the balancing form
// z = P' M^-1 P r + Z E^+ Z' r (coarse.cuh), whose r.z partials come from a dot of their
// own (nb_part rows in part).
template <typename T>
void apply_precond_cg(SolverImpl& S, const T* r, T* z, int kp, double* part, int& nb_part) {
    if (S.coarse_k == 0) {
        apply_precond<T>(S, r, z, kp, part, nb_part);
        return;
    }
    const T* Z = coarse_basis<T>(S);
    const T* GZ = coarse_gbasis<T>(S);
    T* rp = coarse_tmp<T>(S).p;
    const int64_t m = S.d.ndofs;
    const int nbc = coarse_blocks(S);
    double* u1 = S.coarse_u.p;
    double* u2 = S.coarse_u.p + 32 * 32;
    const int ga = S.nblk(m * kp / 4, 1);
    coarse_tn_kernel<T><<<nbc, 256, 0, S.stream>>>(m, Z, r, kp, S.coarse_part.p);
    coarse_solve_kernel<<<1, kCoarseSolveThreads, 0, S.stream>>>(S.coarse_part.p, nbc, S.coarse_einv.p, kp, u1);
    coarse_axpy_kernel<T><<<ga, 256, 0, S.stream>>>(m, GZ, u1, nullptr, -1.0, kp, r, rp);  // P r
    WB_CUDA(cudaGetLastError());
    int nb = 0;
    apply_precond<T>(S, rp, z, kp, nullptr, nb);  // y = M^-1 P r
    coarse_tn_kernel<T><<<nbc, 256, 0, S.stream>>>(m, GZ, z, kp, S.coarse_part.p);
    coarse_solve_kernel<<<1, kCoarseSolveThreads, 0, S.stream>>>(S.coarse_part.p, nbc, S.coarse_einv.p, kp, u2);
    coarse_axpy_kernel<T><<<ga, 256, 0, S.stream>>>(m, Z, u1, u2, 1.0, kp, z, z);  // z = y + Z (u1 - u2)
    WB_CUDA(cudaGetLastError());
    S.gpu_launches += 6;
    nb_part = 0;
    if (part) launch_dot<T, T>(S, r, z, m, kp, part, nb_part);
}

// ---------------------------------------------------------------------------
// Krylov state kernels (one thread per RHS; inputs reduced by reduce_parts_kernel)
// ---------------------------------------------------------------------------

struct KState {
    double *bnorm, *rz, *rz0, *alpha, *beta, *rnorm, *tol;
    int32_t *active, *conv, *iters, *part_of;
    int32_t* n_active;
};

__device__ void count_active(KState s, int kp) {
    __syncwarp();
    if (threadIdx.x == 0) {
        int na = 0;
        for (int j = 0; j < kp; ++j) na += s.active[j];
        *s.n_active = na;
    }
}

// cg.rs:52-74: ||b||; zero RHS converge at iteration 0.  Columns outside part_of idle.
__global__ void cg_init_kernel(KState s, const double* red, int kp) {
    const int c = threadIdx.x;
    if (c < kp) {
        const double bn = sqrt(red[c]);
        s.bnorm[c] = bn;
        s.iters[c] = 0;
        s.alpha[c] = 0.0;
        s.beta[c] = 0.0;
        s.rnorm[c] = bn;
        if (!s.part_of[c]) {
            s.active[c] = 0;
        } else if (bn < 2.220446049250313e-16) {
            s.active[c] = 0;
            s.conv[c] = 1;
        } else {
            s.active[c] = 1;
            s.conv[c] = 0;
        }
    }
}
__global__ void cg_rz0_kernel(KState s, const double* red, int kp) {
    const int c = threadIdx.x;
    if (c < kp) {
        s.rz[c] = red[c];
        s.rz0[c] = red[c];
    }
    count_active(s, kp);
}
// cg.rs:76-86
// An RHS is active from the first iteration until it stops, so counting its alpha steps
// gives the iteration number without passing it in (the iteration is graph-captured).
__device__ void cg_alpha_step(KState s, const double* red, int kp) {
    const int c = threadIdx.x;
    if (c < kp) {
        s.alpha[c] = 0.0;
        if (s.active[c]) {
            const double pap = red[c];
            s.iters[c] += 1;
            if (!(pap > 0.0)) {  // pAp <= 0 (cg.rs:79-84), or not finite (a failed local solve)
                s.active[c] = 0;
                s.conv[c] = 0;
            } else {
                s.alpha[c] = s.rz[c] / pap;
            }
        }
    }
    count_active(s, kp);
}
// cg.rs:94-103
__device__ void cg_check_step(KState s, const double* red, int kp) {
    const int c = threadIdx.x;
    if (c < kp && s.active[c]) {
        const double rn = sqrt(red[c]);
        s.rnorm[c] = rn;
        if (rn / s.bnorm[c] <= s.tol[c]) { s.active[c] = 0; s.conv[c] = 1; }
    }
    count_active(s, kp);
}
// cg.rs:105-125 (EPS^2 stagnation guard)
__device__ void cg_beta_step(KState s, const double* red, int kp) {
    const int c = threadIdx.x;
    if (c < kp && s.active[c]) {
        const double rzn = red[c];
        const double eps = 2.220446049250313e-16;
        const double thr = eps * eps * fmax(fabs(s.rz0[c]), 2.2250738585072014e-308);
        if (fabs(rzn) < thr) {
            s.active[c] = 0;
            s.conv[c] = s.rnorm[c] / s.bnorm[c] <= s.tol[c];
        } else {
            s.beta[c] = rzn / s.rz[c];
            s.rz[c] = rzn;
        }
    }
    count_active(s, kp);
}
// The partial-sum reduction of reduce_parts_kernel followed, in the same launch, by one
// CG scalar step on the reduced values (threads < kp of warp 0; the reduction's thread t
// wrote red[t] itself).  Saves a launch per step.
enum CgStep { CG_STEP_ALPHA = 0, CG_STEP_CHECK = 1, CG_STEP_BETA = 2 };
template <int STEP>
__global__ void reduce_step_kernel(const double* __restrict__ part, int nb, int kp, double* __restrict__ red,
                                   KState ks) {
    reduce_parts_body(part, nb, kp, red);
    if (threadIdx.x >= 32) return;
    if (STEP == CG_STEP_ALPHA) cg_alpha_step(ks, red, kp);
    else if (STEP == CG_STEP_CHECK) cg_check_step(ks, red, kp);
    else cg_beta_step(ks, red, kp);
}

__global__ void cg_final_kernel(KState s, int kp, int maxiter) {
    const int c = threadIdx.x;
    if (c < kp && s.active[c]) { s.active[c] = 0; s.conv[c] = 0; s.iters[c] = maxiter; }
}

template <typename TA, typename TB>
__global__ void convert_kernel(const TA* __restrict__ a, TB* __restrict__ b, int64_t n) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        b[i] = (TB)a[i];
}
// x64 += d on the RHS with mask[c]
template <typename TD>
__global__ void masked_axpy_kernel(double* __restrict__ x, const TD* __restrict__ d, const int32_t* __restrict__ mask,
                                   int64_t rows, int kp) {
    const int64_t n = rows * kp;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        if (mask[i % kp]) x[i] += (double)d[i];
}
__global__ void sub_kernel(const double* __restrict__ a, const double* __restrict__ b, double* __restrict__ out, int64_t n) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        out[i] = a[i] - b[i];
}

KState kstate(Workspace& w) {
    return KState{w.st_bnorm.p, w.st_rz.p, w.st_rz0.p, w.st_alpha.p, w.st_beta.p, w.st_rnorm.p, w.st_tol.p,
                  w.st_active.p, w.st_conv.p, w.st_iters.p, w.st_part.p, w.n_active.p};
}

void ensure_ws(SolverImpl& S, int kp) {
    Workspace& w = S.ws;
    if (w.kp >= kp) return;
    const size_t n = (size_t)S.d.n, m = (size_t)S.d.ndofs;
    w.yi.alloc(n * kp);
    w.e.alloc(n * kp);
    for (DArr<double>* a : {&w.b, &w.x, &w.r, &w.gx, &w.cx, &w.cr, &w.dz, &w.dp, &w.dap}) a->alloc(m * kp);
    if (S.mixed()) {
        for (DArr<float>* a : {&w.frhs, &w.fx, &w.fr, &w.fz, &w.fp, &w.fap}) a->alloc(m * kp);
        w.floc.alloc(std::max<size_t>(1, S.max_slots * kp));
        w.fcore_tmp.alloc(std::max<size_t>(1, S.max_core_total * kp));
        if (S.pc.kind == 2) { w.frwork.alloc(m * kp); w.fcbuf.alloc(m * kp); }
    }
    w.vloc.alloc(std::max<size_t>(1, S.max_slots * kp));
    w.core_tmp.alloc(std::max<size_t>(1, S.max_core_total * kp));
    if (S.pc.kind == 2) { w.rwork.alloc(m * kp); w.cbuf.alloc(m * kp); }
    w.msum.alloc(std::max<size_t>(1, 6 * (size_t)std::max(S.max_nsub, 1) * kp));  // S0, SB, M1, M2, means
    w.part.alloc((size_t)S.n_sm * 8 * kp + 64);
    w.red.alloc(32);
    for (DArr<double>* a : {&w.st_bnorm, &w.st_rz, &w.st_rz0, &w.st_alpha, &w.st_beta, &w.st_rnorm, &w.st_tol}) a->alloc(32);
    for (DArr<int32_t>* a : {&w.st_active, &w.st_conv, &w.st_iters, &w.st_part}) a->alloc(32);
    w.n_active.alloc(1);
    if (!w.sweep_err.p) {
        w.sweep_bar.alloc(2);
        w.sweep_err.alloc(1);
        WB_CUDA(cudaMemset(w.sweep_err.p, 0, sizeof(int32_t)));
    }
    w.kp = kp;
    ++w.gen;
}

// Preconditioned CG on the RHS marked in st_part (device), solution into x (zeroed here),
// per-RHS relative tolerance st_tol (device).  Vectors of type T; inner products in FP64.
template <typename T>
void cg_device(SolverImpl& S, int kp, const T* b, T* x, T* r, T* z, T* p, T* ap, int maxiter) {
    Workspace& w = S.ws;
    const int64_t m = S.d.ndofs;
    const int G = group_for(kp);
    KState ks = kstate(w);
    double* part = w.part.p;
    double* red = w.red.p;
    int nb = 0;
    if (S.coarse_k) coarse_tmp<T>(S).alloc((size_t)m * kp);  // before any capture
    WB_CUDA(cudaMemsetAsync(x, 0, sizeof(T) * m * kp, S.stream));
    WB_CUDA(cudaMemcpyAsync(r, b, sizeof(T) * m * kp, cudaMemcpyDeviceToDevice, S.stream));
    launch_dot<T, T>(S, b, b, m, kp, part, nb);
    launch_reduce(S, part, nb, kp, red);
    cg_init_kernel<<<1, 32, 0, S.stream>>>(ks, red, kp);
    apply_precond_cg<T>(S, r, z, kp, part, nb);
    launch_reduce(S, part, nb, kp, red);
    cg_rz0_kernel<<<1, 32, 0, S.stream>>>(ks, red, kp);
    WB_CUDA(cudaMemcpyAsync(p, z, sizeof(T) * m * kp, cudaMemcpyDeviceToDevice, S.stream));
    S.gpu_launches += 2;
    const T* w_t = std::is_same<T, double>::value ? (const T*)S.w64.p : (const T*)S.w32.p;
    if (!S.explicit_op) obs_autotune<T>(S, kp, w_t, p, ap);  // before the iteration is captured
    const int kind = std::is_same<T, double>::value ? 0 : 1;
    // one iteration: q = G p, alpha, x/r update, convergence check, z = M r, beta, p update
    auto body = [&]() {
        cudaEvent_t e0 = nullptr;
        S.prof_begin(e0);
        launch_gram<T>(S, kp, w_t, p, ap);
        S.prof_end(kind, e0);
        launch_dot<T, T>(S, p, ap, m, kp, part, nb);
        reduce_step_kernel<CG_STEP_ALPHA><<<1, kBlock, 0, S.stream>>>(part, nb, kp, red, ks);
        const int grid = S.nblk(m, G, 2);
        WB_DISPATCH_G(G, cg_xr_kernel<T, GV><<<grid, kBlock, 0, S.stream>>>(x, r, p, ap, w.st_alpha.p, m, kp, part));
        reduce_step_kernel<CG_STEP_CHECK><<<1, kBlock, 0, S.stream>>>(part, grid, kp, red, ks);
        cudaEvent_t e1 = nullptr;
        S.prof_begin(e1);
        apply_precond_cg<T>(S, r, z, kp, part, nb);
        S.prof_end(kind + 2, e1);
        reduce_step_kernel<CG_STEP_BETA><<<1, kBlock, 0, S.stream>>>(part, nb, kp, red, ks);
        const int gridp = S.nblk(m, G);
        WB_DISPATCH_G(G, cg_p_kernel<T, GV><<<gridp, kBlock, 0, S.stream>>>(p, z, w.st_beta.p, w.st_active.p, m, kp));
        WB_CUDA(cudaGetLastError());
        S.gpu_launches += 5;
    };
    // Without event timing, the iteration is captured once as a CUDA graph and replayed
    // (one launch per iteration); the capture is kept while its buffers stay the same.
    const bool graph = !S.profiling;
    if (graph) {
        const std::array<uintptr_t, 9> key{(uintptr_t)b, (uintptr_t)x, (uintptr_t)r, (uintptr_t)z, (uintptr_t)p,
                                           (uintptr_t)ap, (uintptr_t)kp, (uintptr_t)w.gen, sizeof(T)};
        if (!S.cg_exec || key != S.cg_key) {
            if (S.cg_exec) {
                WB_CUDA(cudaGraphExecDestroy(S.cg_exec));
                S.cg_exec = nullptr;
            }
            const int64_t l0 = S.gpu_launches;
            // a capture that fails with the fused (cooperative) sweeps is retried without them
            for (int attempt = 0;; ++attempt) {
                S.gpu_launches = l0;
                cudaGraph_t g = nullptr;
                WB_CUDA(cudaStreamBeginCapture(S.stream, cudaStreamCaptureModeRelaxed));
                try {
                    body();
                } catch (const CudaError&) {
                    cudaStreamEndCapture(S.stream, &g);
                    if (g) cudaGraphDestroy(g);
                    cudaGetLastError();
                    if (attempt == 0 && S.coop) {
                        S.coop = false;
                        continue;
                    }
                    throw;
                }
                cudaError_t ie = cudaStreamEndCapture(S.stream, &g);
                if (ie == cudaSuccess) ie = cudaGraphInstantiate(&S.cg_exec, g, 0);
                if (g) cudaGraphDestroy(g);
                if (ie != cudaSuccess && attempt == 0 && S.coop) {
                    cudaGetLastError();
                    S.cg_exec = nullptr;
                    S.coop = false;
                    continue;
                }
                WB_CUDA(ie);
                break;
            }
            S.cg_key = key;
            S.cg_launches = S.gpu_launches - l0;
            S.gpu_launches = l0;
        }
    }
    cudaEvent_t ev;
    WB_CUDA(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
    auto enqueue_iter = [&]() {
        if (graph) {
            WB_CUDA(cudaGraphLaunch(S.cg_exec, S.stream));
            S.gpu_launches += S.cg_launches;
        } else {
            body();
        }
        publish_active(S, w.n_active.p);
        WB_CUDA(cudaEventRecord(ev, S.stream));
    };
    // The host check of iteration `it` overlaps the device work of iteration it+1; an
    // iteration enqueued after every RHS stopped changes nothing (alpha = 0, masked p).
    publish_active(S, w.n_active.p);
    WB_CUDA(cudaStreamSynchronize(S.stream));
    if (*S.h_active > 0 && maxiter > 0) {
        cudaEvent_t evb;
        WB_CUDA(cudaEventCreateWithFlags(&evb, cudaEventDisableTiming));
        enqueue_iter();
        int it = 1;
        while (it < maxiter) {
            std::swap(ev, evb);     // evb = event of iteration it
            enqueue_iter();         // records ev for iteration it+1
            WB_CUDA(cudaEventSynchronize(evb));
            ++it;
            if (*S.h_active == 0) break;
        }
        WB_CUDA(cudaEventDestroy(evb));
    }
    WB_CUDA(cudaEventDestroy(ev));
    cg_final_kernel<<<1, 32, 0, S.stream>>>(ks, kp, maxiter);
    WB_CUDA(cudaGetLastError());
    S.gpu_launches++;
}

// ---------------------------------------------------------------------------
// Right-preconditioned GMRES(restart) on the device (gmres.rs:201-530), batched over
// RHS: every RHS runs its own Arnoldi cycle; Hessenberg, Givens and the small solves
// stay on the device in FP64, one thread per RHS.
// ---------------------------------------------------------------------------

struct GState {
    int R;  // restart
    double *H, *g, *cs, *sn, *y, *scale, *hcur, *hmax, *abs_tol, *resid;
    int32_t *cyc, *done, *conv, *iters, *jc, *brk, *n_active;
};

__device__ void g_count(GState s, int kp) {
    __syncwarp();
    if (threadIdx.x == 0) {
        int na = 0;
        for (int j = 0; j < kp; ++j) na += s.cyc[j];
        *s.n_active = na;
    }
}
#define GH(s, c, i, j) (s).H[((size_t)(c) * ((s).R) + (j)) * ((s).R + 1) + (i)]

// ||b||, abs_tol; zero RHS converge at iteration 0 (gmres.rs:357-369).  RHS outside
// part_of do not take part.
__global__ void gm_init_kernel(GState s, const double* red, int kp, const double* tol, const int32_t* part_of) {
    const int c = threadIdx.x;
    if (c < kp) {
        const double bn = sqrt(red[c]);
        s.iters[c] = 0;
        s.brk[c] = 0;
        s.cyc[c] = 0;
        s.abs_tol[c] = tol[c] * bn;
        if (!part_of[c]) { s.done[c] = 1; s.conv[c] = 0; }
        else if (bn < 2.220446049250313e-16) { s.done[c] = 1; s.conv[c] = 1; }
        else { s.done[c] = 0; s.conv[c] = 0; }
    }
}
// Start of a cycle: beta = ||b - A x|| (gmres.rs:375-393, 428-437).
__global__ void gm_restart_kernel(GState s, const double* red, int kp, int maxiter) {
    const int c = threadIdx.x;
    if (c < kp) {
        s.cyc[c] = 0;
        s.jc[c] = 0;
        if (!s.done[c]) {
            const double beta = sqrt(red[c]);
            s.resid[c] = beta;
            if (s.brk[c]) {  // lucky breakdown: the true residual decides
                s.done[c] = 1;
                s.conv[c] = beta <= s.abs_tol[c];
            } else if (beta <= s.abs_tol[c]) {
                s.done[c] = 1;
                s.conv[c] = 1;
            } else if (s.iters[c] >= maxiter) {
                s.done[c] = 1;
                s.conv[c] = 0;
            } else {
                s.cyc[c] = 1;
                for (int i = 0; i <= s.R; ++i) s.g[(size_t)c * (s.R + 1) + i] = 0.0;
                for (int j = 0; j < s.R; ++j) {
                    s.cs[(size_t)c * s.R + j] = 0.0;
                    s.sn[(size_t)c * s.R + j] = 0.0;
                    for (int i = 0; i <= s.R; ++i) GH(s, c, i, j) = 0.0;
                }
                s.g[(size_t)c * (s.R + 1)] = beta;
                s.hmax[c] = 0.0;
                s.scale[c] = 1.0 / beta;
            }
        }
    }
    g_count(s, kp);
}
// MGS coefficient h_ij = w . v_i (gmres.rs:201-220).
__global__ void gm_mgs_coef_kernel(GState s, const double* red, int kp, int i, int j) {
    const int c = threadIdx.x;
    if (c < kp) {
        const double h = s.cyc[c] ? red[c] : 0.0;
        s.hcur[c] = h;
        if (s.cyc[c]) {
            GH(s, c, i, j) = h;
            s.hmax[c] = fmax(s.hmax[c], fabs(h));
        }
    }
}
template <typename T>
__global__ void gm_axpy_kernel(T* __restrict__ w, const T* __restrict__ v, const double* __restrict__ h,
                               int64_t rows, int kp) {
    const int64_t n = rows * kp;
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x)
        w[e] -= (T)h[e % kp] * v[e];
}
template <typename T>
__global__ void gm_scale_kernel(const T* __restrict__ w, T* __restrict__ v, const double* __restrict__ scale,
                                const int32_t* __restrict__ cyc, int64_t rows, int kp) {
    const int64_t n = rows * kp;
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
        const int c = (int)(e % kp);
        v[e] = cyc[c] ? (T)((double)w[e] * scale[c]) : T(0);
    }
}
// h_{j+1,j} = ||w||, Givens rotations, residual estimate, outcome (gmres.rs:256-313).
__global__ void gm_givens_kernel(GState s, const double* red, int kp, int j, int maxiter) {
    const int c = threadIdx.x;
    if (c < kp && s.cyc[c]) {
        const int R = s.R;
        double* cs = s.cs + (size_t)c * R;
        double* sn = s.sn + (size_t)c * R;
        double* g = s.g + (size_t)c * (R + 1);
        const double hn = sqrt(red[c]);
        GH(s, c, j + 1, j) = hn;
        s.hmax[c] = fmax(s.hmax[c], hn);
        for (int i = 0; i < j; ++i) {
            const double a = GH(s, c, i, j), b = GH(s, c, i + 1, j);
            const double t = cs[i] * a + sn[i] * b;
            GH(s, c, i + 1, j) = -sn[i] * a + cs[i] * b;
            GH(s, c, i, j) = t;
        }
        const double a = GH(s, c, j, j), b = GH(s, c, j + 1, j);
        const double r = hypot(a, b);
        double cc = 1.0, ss = 0.0;
        if (r != 0.0) { cc = a / r; ss = b / r; }
        cs[j] = cc;
        sn[j] = ss;
        GH(s, c, j, j) = cc * a + ss * b;
        GH(s, c, j + 1, j) = 0.0;
        const double t = cc * g[j] + ss * g[j + 1];
        g[j + 1] = -ss * g[j] + cc * g[j + 1];
        g[j] = t;
        s.jc[c] = j + 1;
        s.iters[c] += 1;
        const double res = fabs(g[j + 1]);
        s.resid[c] = res;
        s.scale[c] = 0.0;
        if (res <= s.abs_tol[c]) {
            s.cyc[c] = 0; s.done[c] = 1; s.conv[c] = 1;
        } else if (s.iters[c] >= maxiter) {
            s.cyc[c] = 0; s.done[c] = 1; s.conv[c] = 0;
        } else if (hn > 1e-14 * s.hmax[c]) {
            s.scale[c] = 1.0 / hn;
        } else {
            s.cyc[c] = 0; s.brk[c] = 1;  // lucky breakdown
        }
    }
    g_count(s, kp);
}
// y = R^{-1} g over the cycle's jc steps (solve_upper_triangular, gmres.rs:499-519).
__global__ void gm_trisolve_kernel(GState s, int kp) {
    const int c = threadIdx.x;
    if (c >= kp) return;
    const int jn = s.jc[c], R = s.R;
    double* y = s.y + (size_t)c * R;
    const double* g = s.g + (size_t)c * (R + 1);
    for (int i = 0; i < R; ++i) y[i] = 0.0;
    for (int i = jn - 1; i >= 0; --i) {
        double sum = g[i];
        for (int jj = i + 1; jj < jn; ++jj) sum -= GH(s, c, i, jj) * y[jj];
        const double d = GH(s, c, i, i);
        y[i] = fabs(d) < 1e-14 * (1.0 + fabs(sum)) ? 0.0 : sum / d;
    }
}
// x += sum_i y_i z_i (update_solution, gmres.rs:523-530).
template <typename T>
__global__ void gm_update_kernel(double* __restrict__ x, const T* __restrict__ Z, const double* __restrict__ y,
                                 int R, int jmax, int64_t rows, int kp) {
    const int64_t n = rows * kp;
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
        const int c = (int)(e % kp);
        double acc = 0.0;
        for (int i = 0; i < jmax; ++i) acc += y[(size_t)c * R + i] * (double)Z[(size_t)i * n + e];
        x[e] += acc;
    }
}
__global__ void gm_final_kernel(GState s, int kp) {
    const int c = threadIdx.x;
    if (c < kp && !s.done[c]) { s.done[c] = 1; s.conv[c] = 0; }
}
#undef GH

struct GmresBufs {
    int R = 0, kp = 0;
    int64_t m = 0;
    DArr<double> H, g, cs, sn, y, scale, hcur, hmax, abs_tol, resid;
    DArr<int32_t> cyc, done, conv, iters, jc, brk, n_active;
    DArr<double> r64, w64, V64, Z64;
    DArr<float> w32, V32, Z32;
};

// GMRES(R) for A d = rhs (FP64 rhs and solution x; Arnoldi vectors of type T).
template <typename T>
void gmres_device(SolverImpl& S, GmresBufs& B, int kp, const double* rhs, double* x, int maxiter) {
    const int64_t m = S.d.ndofs;
    const int R = std::max(1, S.params.gmres_restart);
    const size_t mk = (size_t)m * kp;
    if (B.R != R || B.kp < kp || B.m != m) {
        B.R = R; B.kp = kp; B.m = m;
        B.g.alloc((size_t)32 * (R + 1));
        B.H.alloc((size_t)32 * R * (R + 1));
        for (DArr<double>* a : {&B.cs, &B.sn, &B.y}) a->alloc((size_t)32 * R);
        for (DArr<double>* a : {&B.scale, &B.hcur, &B.hmax, &B.abs_tol, &B.resid}) a->alloc(32);
        for (DArr<int32_t>* a : {&B.cyc, &B.done, &B.conv, &B.iters, &B.jc, &B.brk, &B.n_active}) a->alloc(32);
        B.r64.alloc(mk);
        B.w64.alloc(mk);
        if (std::is_same<T, double>::value) { B.V64.alloc(mk * (R + 1)); B.Z64.alloc(mk * R); }
        else { B.w32.alloc(mk); B.V32.alloc(mk * (R + 1)); B.Z32.alloc(mk * R); }
    }
    GState s{R, B.H.p, B.g.p, B.cs.p, B.sn.p, B.y.p, B.scale.p, B.hcur.p, B.hmax.p, B.abs_tol.p, B.resid.p,
             B.cyc.p, B.done.p, B.conv.p, B.iters.p, B.jc.p, B.brk.p, B.n_active.p};
    T* V = std::is_same<T, double>::value ? (T*)B.V64.p : (T*)B.V32.p;
    T* Z = std::is_same<T, double>::value ? (T*)B.Z64.p : (T*)B.Z32.p;
    T* wv = std::is_same<T, double>::value ? (T*)B.w64.p : (T*)B.w32.p;
    const T* w_t = std::is_same<T, double>::value ? (const T*)S.w64.p : (const T*)S.w32.p;
    double* part = S.ws.part.p;
    double* red = S.ws.red.p;
    int nb = 0;
    const int gridv = S.nblk(m * kp, 1);
    WB_CUDA(cudaMemsetAsync(x, 0, sizeof(double) * mk, S.stream));
    launch_dot<double, double>(S, rhs, rhs, m, kp, part, nb);
    launch_reduce(S, part, nb, kp, red);
    gm_init_kernel<<<1, 32, 0, S.stream>>>(s, red, kp, S.ws.st_tol.p, S.ws.st_part.p);
    const int kind = std::is_same<T, double>::value ? 0 : 1;
    for (int cycle = 0; cycle < maxiter + 2; ++cycle) {
        // r = rhs - A x (FP64), beta, v_0 = r / beta
        launch_gram<double>(S, kp, S.w64.p, x, B.w64.p);
        sub_kernel<<<gridv, kBlock, 0, S.stream>>>(rhs, B.w64.p, B.r64.p, (int64_t)mk);
        launch_dot<double, double>(S, B.r64.p, B.r64.p, m, kp, part, nb);
        launch_reduce(S, part, nb, kp, red);
        gm_restart_kernel<<<1, 32, 0, S.stream>>>(s, red, kp, maxiter);
        publish_active(S, B.n_active.p);
        WB_CUDA(cudaStreamSynchronize(S.stream));
        S.gpu_launches += 2;
        if (*S.h_active == 0) break;
        if (std::is_same<T, double>::value) {
            gm_scale_kernel<double><<<gridv, kBlock, 0, S.stream>>>(B.r64.p, (double*)V, B.scale.p, B.cyc.p, m, kp);
        } else {
            convert_kernel<double, float><<<gridv, kBlock, 0, S.stream>>>(B.r64.p, B.w32.p, (int64_t)mk);
            gm_scale_kernel<float><<<gridv, kBlock, 0, S.stream>>>(B.w32.p, (float*)V, B.scale.p, B.cyc.p, m, kp);
        }
        int jmax = 0;
        for (int j = 0; j < R; ++j) {
            T* vj = V + (size_t)j * mk;
            T* zj = Z + (size_t)j * mk;
            int nbp = 0;
            cudaEvent_t e1 = nullptr;
            S.prof_begin(e1);
            apply_precond<T>(S, vj, zj, kp, nullptr, nbp);
            S.prof_end(kind + 2, e1);
            cudaEvent_t e0 = nullptr;
            S.prof_begin(e0);
            launch_gram<T>(S, kp, w_t, zj, wv);
            S.prof_end(kind, e0);
            for (int i = 0; i <= j; ++i) {
                const T* vi = V + (size_t)i * mk;
                launch_dot<T, T>(S, wv, vi, m, kp, part, nb);
                launch_reduce(S, part, nb, kp, red);
                gm_mgs_coef_kernel<<<1, 32, 0, S.stream>>>(s, red, kp, i, j);
                gm_axpy_kernel<T><<<gridv, kBlock, 0, S.stream>>>(wv, vi, B.hcur.p, m, kp);
            }
            launch_dot<T, T>(S, wv, wv, m, kp, part, nb);
            launch_reduce(S, part, nb, kp, red);
            gm_givens_kernel<<<1, 32, 0, S.stream>>>(s, red, kp, j, maxiter);
            gm_scale_kernel<T><<<gridv, kBlock, 0, S.stream>>>(wv, V + (size_t)(j + 1) * mk, B.scale.p, B.cyc.p, m, kp);
            WB_CUDA(cudaGetLastError());
            S.gpu_launches += 2 * (j + 1) + 2;
            jmax = j + 1;
            publish_active(S, B.n_active.p);
            WB_CUDA(cudaStreamSynchronize(S.stream));
            if (*S.h_active == 0) break;
        }
        gm_trisolve_kernel<<<1, 32, 0, S.stream>>>(s, kp);
        gm_update_kernel<T><<<gridv, kBlock, 0, S.stream>>>(x, Z, B.y.p, R, jmax, m, kp);
        WB_CUDA(cudaGetLastError());
        S.gpu_launches += 2;
    }
    gm_final_kernel<<<1, 32, 0, S.stream>>>(s, kp);
    WB_CUDA(cudaGetLastError());
}

// ---------------------------------------------------------------------------
// LSMR (schwarz-precond/src/solve/lsmr.rs, lsmr/bidiag.rs, lsmr/recurrence.rs):
// min ||b - A x|| with A = W^(1/2) D (within/src/operator.rs:111-190), b = W^(1/2) y,
// batched over the RHS columns.  Every column runs its own Golub-Kahan process and
// Givens recurrences; their scalars live on the device (one thread per column), the
// vectors are the interleaved n x kp / m x kp layout of the other solvers.  With a
// preconditioner M ~ A'A the Modified Golub-Kahan process applies M^-1 once per step.
// ---------------------------------------------------------------------------

struct LsmrBufs {
    int kp = 0, cap = 0;
    int64_t n = 0, m = 0;
    DArr<double> u, av, sw;                      // observation space (n x kp; sw: n)
    DArr<double> v, atu, pt, h, hb;              // dof space (m x kp)
    DArr<double> ring_v, ring_p;                 // cap x m x kp
    // per-column scalars (kp each)
    DArr<double> bnorm, beta, alpha, bpi, scale, pa, pb, inv_alpha;
    DArr<double> abar, phibar, cbar, sbar, zbar, a2, prho, prhob, coef, zeros;
    DArr<int32_t> active, conv, iters, part_of, brk, n_active;
};

struct LsmrState {
    double *bnorm, *beta, *alpha, *bpi, *scale, *pa, *pb, *inv_alpha;
    double *abar, *phibar, *cbar, *sbar, *zbar, *a2, *prho, *prhob, *coef;
    int32_t *active, *conv, *iters, *part_of, *brk, *n_active;
    double tol;
    int maxiter, precond;
};

LsmrState lsmr_state(LsmrBufs& B, double tol, int maxiter, int precond) {
    return LsmrState{B.bnorm.p, B.beta.p, B.alpha.p, B.bpi.p, B.scale.p, B.pa.p, B.pb.p, B.inv_alpha.p,
                     B.abar.p, B.phibar.p, B.cbar.p, B.sbar.p, B.zbar.p, B.a2.p, B.prho.p, B.prhob.p, B.coef.p,
                     B.active.p, B.conv.p, B.iters.p, B.part_of.p, B.brk.p, B.n_active.p, tol, maxiter, precond};
}

__device__ void lsmr_count(const LsmrState& s, int kp) {
    __syncwarp();
    if (threadIdx.x == 0) {
        int na = 0;
        for (int j = 0; j < kp; ++j) na += s.active[j];
        *s.n_active = na;
    }
}

// u = sw .* x + scale[c] u (u not read where scale is 0), with partial sums of u^2.
template <int G>
__global__ void __launch_bounds__(kBlock) lsmr_obs_axpy_kernel(double* __restrict__ u, const double* __restrict__ x,
                                                               const double* __restrict__ sw,
                                                               const double* __restrict__ scale, int64_t rows, int kp,
                                                               double* __restrict__ part) {
    const int c4 = (threadIdx.x & (G - 1)) * 4;
    const V4<double> sc(scale[c4], scale[c4 + 1], scale[c4 + 2], scale[c4 + 3]);
    V4<double> acc(0.0);
    const int64_t rpb = blockDim.x / G;
    for (int64_t r = (int64_t)blockIdx.x * rpb + threadIdx.x / G; r < rows; r += (int64_t)gridDim.x * rpb) {
        const size_t e = (size_t)r * kp + c4;
        const double wr = sw ? sw[r] : 1.0;
        V4<double> xv = ld4(x + e);
        const V4<double> uv = ld4(u + e);
        xv.a = wr * xv.a + (sc.a != 0.0 ? sc.a * uv.a : 0.0);
        xv.b = wr * xv.b + (sc.b != 0.0 ? sc.b * uv.b : 0.0);
        xv.c = wr * xv.c + (sc.c != 0.0 ? sc.c * uv.c : 0.0);
        xv.d = wr * xv.d + (sc.d != 0.0 ? sc.d * uv.d : 0.0);
        st4(u + e, xv);
        acc.a += xv.a * xv.a; acc.b += xv.b * xv.b; acc.c += xv.c * xv.c; acc.d += xv.d * xv.d;
    }
    block_reduce_store4<G>(acc, kp, part);
}

// y = sa * a[c] x + b[c] y per column (b == nullptr: 1; y not read where b[c] is 0),
// with partial sums of y^2 when part is given.
template <int G>
__global__ void __launch_bounds__(kBlock) lsmr_axpby_kernel(double* y, const double* x,
                                                            const double* __restrict__ a, double sa,
                                                            const double* __restrict__ b, int64_t rows, int kp,
                                                            double* __restrict__ part) {
    const int c4 = (threadIdx.x & (G - 1)) * 4;
    const V4<double> av(sa * a[c4], sa * a[c4 + 1], sa * a[c4 + 2], sa * a[c4 + 3]);
    const V4<double> bv = b ? V4<double>(b[c4], b[c4 + 1], b[c4 + 2], b[c4 + 3]) : V4<double>(1.0);
    V4<double> acc(0.0);
    const int64_t rpb = blockDim.x / G;
    for (int64_t r = (int64_t)blockIdx.x * rpb + threadIdx.x / G; r < rows; r += (int64_t)gridDim.x * rpb) {
        const size_t e = (size_t)r * kp + c4;
        const V4<double> xv = ld4(x + e), yv = ld4(y + e);
        V4<double> o;
        o.a = av.a * xv.a + (bv.a != 0.0 ? bv.a * yv.a : 0.0);
        o.b = av.b * xv.b + (bv.b != 0.0 ? bv.b * yv.b : 0.0);
        o.c = av.c * xv.c + (bv.c != 0.0 ? bv.c * yv.c : 0.0);
        o.d = av.d * xv.d + (bv.d != 0.0 ? bv.d * yv.d : 0.0);
        st4(y + e, o);
        acc.a += o.a * o.a; acc.b += o.b * o.b; acc.c += o.c * o.c; acc.d += o.d * o.d;
    }
    if (part) block_reduce_store4<G>(acc, kp, part);
}

// SolutionState::update (recurrence.rs:186-240): hb = h - t_hbar hb; x += t_x hb;
// h = v - t_h h, with coef = [t_x | t_hbar | t_h] per column (zeros freeze a column's x).
template <int G>
__global__ void __launch_bounds__(kBlock) lsmr_update_kernel(double* __restrict__ x, double* __restrict__ h,
                                                             double* __restrict__ hb, const double* __restrict__ v,
                                                             const double* __restrict__ coef, int64_t rows, int kp) {
    const int c4 = (threadIdx.x & (G - 1)) * 4;
    const V4<double> tx(coef[c4], coef[c4 + 1], coef[c4 + 2], coef[c4 + 3]);
    const V4<double> thb(coef[kp + c4], coef[kp + c4 + 1], coef[kp + c4 + 2], coef[kp + c4 + 3]);
    const V4<double> th(coef[2 * kp + c4], coef[2 * kp + c4 + 1], coef[2 * kp + c4 + 2], coef[2 * kp + c4 + 3]);
    const int64_t rpb = blockDim.x / G;
    for (int64_t r = (int64_t)blockIdx.x * rpb + threadIdx.x / G; r < rows; r += (int64_t)gridDim.x * rpb) {
        const size_t e = (size_t)r * kp + c4;
        const V4<double> ho = ld4(h + e), hbo = ld4(hb + e), vv = ld4(v + e);
        V4<double> xv = ld4(x + e), hn, hbn;
        hbn.a = ho.a - thb.a * hbo.a; hbn.b = ho.b - thb.b * hbo.b; hbn.c = ho.c - thb.c * hbo.c; hbn.d = ho.d - thb.d * hbo.d;
        xv.a += tx.a * hbn.a; xv.b += tx.b * hbn.b; xv.c += tx.c * hbn.c; xv.d += tx.d * hbn.d;
        hn.a = vv.a - th.a * ho.a; hn.b = vv.b - th.b * ho.b; hn.c = vv.c - th.c * ho.c; hn.d = vv.d - th.d * ho.d;
        st4(hb + e, hbn);
        st4(x + e, xv);
        st4(h + e, hn);
    }
}

__global__ void lsmr_sqrt_kernel(const double* __restrict__ w, double* __restrict__ sw, int64_t n) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        sw[i] = sqrt(w[i]);
}

// beta_1 = ||b|| (GolubKahan::init / ModifiedGolubKahan::init); zero right-hand sides
// are solved at iteration 0 (zero_rhs_result).  inv_alpha holds 1 / beta_1 for u.
__global__ void lsmr_init_kernel(LsmrState s, const double* __restrict__ red, int kp) {
    const int c = threadIdx.x;
    if (c < kp) {
        const double bn = sqrt(red[c]);
        s.bnorm[c] = bn;
        s.beta[c] = bn;
        s.inv_alpha[c] = bn > 0.0 ? 1.0 / bn : 0.0;
        const int on = s.part_of[c] && bn != 0.0;
        s.active[c] = on;
        s.conv[c] = s.part_of[c] && !on;
        s.iters[c] = 0;
        s.brk[c] = 0;
    }
    lsmr_count(s, kp);
}

// alpha_1 (Euclidean or M-norm of A'u_1), then the recurrence and convergence state
// (LsmrRecurrenceState::init, ConvergenceState::new, RotationStep::initial); A'b = 0
// stops at iteration 0.  inv_alpha = 1 / alpha_1 normalizes v_1.
__global__ void lsmr_alpha1_kernel(LsmrState s, const double* __restrict__ red, int kp) {
    const int c = threadIdx.x;
    if (c < kp) {
        const double q = red[c];
        const double al = s.precond ? (q > 0.0 ? sqrt(q) : 0.0) : sqrt(q);
        s.alpha[c] = al;
        s.inv_alpha[c] = al > 0.0 ? 1.0 / al : 0.0;
        if (s.active[c] && al == 0.0) {
            s.active[c] = 0;
            s.conv[c] = 1;
        }
        const double be = s.beta[c];
        s.abar[c] = al; s.phibar[c] = be; s.cbar[c] = 1.0; s.sbar[c] = 0.0; s.zbar[c] = al * be;
        s.a2[c] = al * al; s.prho[c] = 1.0; s.prhob[c] = 1.0; s.bpi[c] = 1.0;
        // the first step's u-update scale: -alpha (GK) or -alpha / beta_prev (MGK, u normalized)
        s.scale[c] = s.active[c] ? -al : 0.0;
    }
    lsmr_count(s, kp);
}

// beta_{k+1} = ||u||: the breakdown flag, and the coefficients of the next vector update.
// u is kept unnormalized in both processes (its 1/beta goes into the coefficients):
// GK: v = (1/beta) A'u - beta v;  MGK: p~ = (1/beta) A'u - (beta/alpha) p~.  The next
// step's u-update scale is -alpha_{k+1} / beta_{k+1} (bpi = 1/beta).
// Inactive or broken-down columns get zeros, which zero their v (and p~).
__global__ void lsmr_beta_kernel(LsmrState s, const double* __restrict__ red, int kp) {
    const int c = threadIdx.x;
    if (c < kp) {
        const double be = sqrt(red[c]);
        const int on = s.active[c];
        s.beta[c] = be;
        s.brk[c] = on && be == 0.0;
        const int go = on && be != 0.0;
        const double binv = be > 0.0 ? 1.0 / be : 0.0;
        if (!s.precond) {  // u stays unnormalized: A'u_{k+1} = A'u / beta
            s.pa[c] = go ? binv : 0.0;
            s.pb[c] = go ? -be : 0.0;
            s.bpi[c] = go ? binv : 0.0;
        } else {
            const double al = s.alpha[c];
            s.pa[c] = go ? binv : 0.0;
            s.pb[c] = (go && al > 0.0) ? -(be / al) : 0.0;
            s.bpi[c] = go ? binv : 0.0;
        }
    }
}

// One LSMR step's scalars after the new v: alpha_{k+1}, the ||A||_F^2 estimate, both
// Givens rotations, the solution-update coefficients and the stop tests
// (lsmr.rs:225-262, recurrence.rs:92-140, 186-240, 265-284).  red: GK ||v||^2, MGK <v, p~>.
__global__ void lsmr_step_kernel(LsmrState s, const double* __restrict__ red, int kp, int itn) {
    const int c = threadIdx.x;
    if (c < kp) {
        double* coef = s.coef;
        coef[c] = 0.0; coef[kp + c] = 0.0; coef[2 * kp + c] = 0.0;
        if (s.active[c]) {
            const double q = red[c];
            const double sb = s.beta[c];
            double sa = s.precond ? (q > 0.0 ? sqrt(q) : 0.0) : sqrt(q);
            if (s.brk[c]) sa = 0.0;
            s.inv_alpha[c] = sa > 0.0 ? 1.0 / sa : 0.0;
            s.a2[c] += sa * sa + sb * sb;
            // P-hat: eliminate beta_{k+1} against alpha_bar
            const double ab = s.abar[c];
            const double r1 = hypot(ab, sb);
            const double c1 = r1 > 0.0 ? ab / r1 : 1.0, s1 = r1 > 0.0 ? sb / r1 : 0.0;
            const double theta_new = s1 * sa;
            s.abar[c] = -c1 * sa;
            s.phibar[c] = s1 * s.phibar[c];
            // P-bar: eliminate theta_{k+1} against c_bar rho (theta_bar uses the old s_bar)
            const double theta_bar = s.sbar[c] * r1;
            const double a_ = s.cbar[c] * r1;
            const double r2 = hypot(a_, theta_new);
            const double c2 = r2 > 0.0 ? a_ / r2 : 1.0, s2 = r2 > 0.0 ? theta_new / r2 : 0.0;
            const double zeta = c2 * s.zbar[c];
            s.zbar[c] = -s2 * s.zbar[c];
            s.cbar[c] = c2;
            s.sbar[c] = s2;
            // solution-update coefficients
            const double dx = r1 * r2, dh = s.prho[c] * s.prhob[c];
            coef[c] = fabs(dx) > DBL_EPSILON ? zeta / dx : 0.0;
            coef[kp + c] = fabs(dh) > DBL_EPSILON ? theta_bar * r1 / dh : 0.0;
            coef[2 * kp + c] = fabs(r1) > DBL_EPSILON ? theta_new / r1 : 0.0;
            s.prho[c] = r1;
            s.prhob[c] = r2;
            // stop tests: ||r|| <= tol ||b||, or ||A'r|| / (||A|| ||r||) <= tol
            const double res = fabs(s.phibar[c]);
            bool stop = res <= s.tol * s.bnorm[c];
            if (!stop) {
                const double an = fmax(sqrt(s.a2[c]), DBL_MIN);
                stop = fabs(s.zbar[c]) / (an * fmax(res, DBL_MIN)) <= s.tol;
            }
            s.iters[c] = itn;
            s.alpha[c] = sa;
            if (stop || sa == 0.0) {
                s.conv[c] = 1;
                s.active[c] = 0;
            } else if (itn >= s.maxiter) {
                s.active[c] = 0;
            }
            s.scale[c] = s.active[c] ? -(sa * s.bpi[c]) : 0.0;
        } else {
            s.inv_alpha[c] = 0.0;
            s.scale[c] = 0.0;
        }
    }
    lsmr_count(s, kp);
}

// LSMR for the columns in part_of, into x (m x kp, FP64).  y_i: interleaved n x kp.
void lsmr_device(SolverImpl& S, LsmrBufs& B, int kp, const double* yi, double* x, const std::vector<int32_t>& part_of,
                 std::vector<int32_t>& conv, std::vector<int32_t>& iters) {
    const int64_t n = S.d.n, m = S.d.ndofs;
    const int precond = S.pc.kind != 0 ? 1 : 0;
    const int cap = (int)std::max<int64_t>(0, std::min<int64_t>(S.params.lsmr_local_size, std::min(n, m)));
    if (B.kp != kp || B.n != n || B.m != m || B.cap != cap) {
        B.kp = kp; B.n = n; B.m = m; B.cap = cap;
        B.u.alloc((size_t)n * kp); B.av.alloc((size_t)n * kp);
        for (DArr<double>* a : {&B.v, &B.atu, &B.pt, &B.h, &B.hb}) a->alloc((size_t)m * kp);
        if (cap) {
            B.ring_v.alloc((size_t)cap * m * kp);
            if (precond) B.ring_p.alloc((size_t)cap * m * kp);
        }
        for (DArr<double>* a : {&B.bnorm, &B.beta, &B.alpha, &B.bpi, &B.scale, &B.pa, &B.pb, &B.inv_alpha, &B.abar,
                                &B.phibar, &B.cbar, &B.sbar, &B.zbar, &B.a2, &B.prho, &B.prhob, &B.zeros})
            a->alloc(32);
        B.coef.alloc(96);
        for (DArr<int32_t>* a : {&B.active, &B.conv, &B.iters, &B.part_of, &B.brk, &B.n_active}) a->alloc(32);
        B.sw.release();
        if (S.w64.p) {
            B.sw.alloc((size_t)n);
            lsmr_sqrt_kernel<<<S.nblk(n, 1, 4), kBlock, 0, S.stream>>>(S.w64.p, B.sw.p, n);
            WB_CUDA(cudaGetLastError());
            S.gpu_launches++;
        }
        WB_CUDA(cudaMemsetAsync(B.zeros.p, 0, 32 * sizeof(double), S.stream));
    }
    LsmrState s = lsmr_state(B, S.params.tol, S.params.maxiter, precond);
    write_small(S, B.part_of.p, part_of.data(), nullptr, nullptr, kp);
    const int G = group_for(kp);
    const double* sw = B.sw.p;
    double* part = S.ws.part.p;
    double* red = S.ws.red.p;
    const int gn = S.nblk(n, G, 2), gm = S.nblk(m, G, 2);
    const size_t mk = (size_t)m * kp;
    int nb = 0;
    auto axpby = [&](double* y, const double* xx, const double* a, double sa, const double* b, bool sq) {
        WB_DISPATCH_G(G, lsmr_axpby_kernel<GV><<<gm, kBlock, 0, S.stream>>>(y, xx, a, sa, b, m, kp, sq ? part : nullptr));
        WB_CUDA(cudaGetLastError());
        S.gpu_launches++;
        if (sq) launch_reduce(S, part, gm, kp, red);
    };
    auto dot = [&](const double* a, const double* b) {
        launch_dot<double, double>(S, a, b, m, kp, part, nb);
        launch_reduce(S, part, nb, kp, red);
    };
    auto obs_axpy = [&](const double* xx, const double* scale) {  // u = sw .* xx + scale u, red = ||u||^2
        WB_DISPATCH_G(G, lsmr_obs_axpy_kernel<GV><<<gn, kBlock, 0, S.stream>>>(B.u.p, xx, sw, scale, n, kp, part));
        WB_CUDA(cudaGetLastError());
        S.gpu_launches++;
        launch_reduce(S, part, gn, kp, red);
    };
    auto scale_u = [&]() {  // u *= inv_alpha (a = inv_alpha, b = 0)
        WB_DISPATCH_G(G, lsmr_axpby_kernel<GV><<<gn, kBlock, 0, S.stream>>>(B.u.p, B.u.p, B.inv_alpha.p, 1.0, B.zeros.p,
                                                                             n, kp, nullptr));
        WB_CUDA(cudaGetLastError());
        S.gpu_launches++;
    };
    auto adjoint = [&](double* out) {  // out = D' (sw .* u)
        launch_obs<double, OBS_RHS>(S, kp, sw, nullptr, B.u.p, out, nullptr);
    };
    // ring of past (v, M v) pairs for the windowed reorthogonalization
    int r_next = 0, r_count = 0;
    auto ring_sweep = [&]() {
        const int start = r_count < cap ? 0 : r_next;
        for (int i = 0; i < r_count; ++i) {
            const int idx = (start + i) % cap;
            const double* vj = B.ring_v.p + (size_t)idx * mk;
            if (precond) {
                const double* pj = B.ring_p.p + (size_t)idx * mk;
                dot(B.v.p, pj);
                axpby(B.v.p, vj, red, -1.0, nullptr, false);
                axpby(B.pt.p, pj, red, -1.0, nullptr, false);
            } else {
                dot(B.v.p, vj);
                axpby(B.v.p, vj, red, -1.0, nullptr, false);
            }
        }
    };
    auto ring_push = [&]() {  // v (normalized) and p~ / alpha
        WB_CUDA(cudaMemcpyAsync(B.ring_v.p + (size_t)r_next * mk, B.v.p, sizeof(double) * mk, cudaMemcpyDeviceToDevice,
                                S.stream));
        if (precond) {
            double* pj = B.ring_p.p + (size_t)r_next * mk;
            axpby(pj, B.pt.p, B.inv_alpha.p, 1.0, B.zeros.p, false);
        }
        r_next = (r_next + 1) % cap;
        if (r_count < cap) ++r_count;
    };
    // --- init: beta_1 u_1 = b, alpha_1 v_1 = A'u_1 (or M^-1 A'u_1 with the M-norm)
    obs_axpy(yi, B.zeros.p);
    lsmr_init_kernel<<<1, 32, 0, S.stream>>>(s, red, kp);
    scale_u();
    if (!precond) {
        adjoint(B.v.p);
        dot(B.v.p, B.v.p);
    } else {
        adjoint(B.pt.p);
        int nbp = 0;
        apply_precond<double>(S, B.pt.p, B.v.p, kp, nullptr, nbp);
        dot(B.v.p, B.pt.p);
    }
    lsmr_alpha1_kernel<<<1, 32, 0, S.stream>>>(s, red, kp);
    axpby(B.v.p, B.v.p, B.inv_alpha.p, 1.0, B.zeros.p, false);  // v /= alpha_1
    if (cap) ring_push();
    WB_CUDA(cudaMemcpyAsync(B.h.p, B.v.p, sizeof(double) * mk, cudaMemcpyDeviceToDevice, S.stream));
    WB_CUDA(cudaMemsetAsync(B.hb.p, 0, sizeof(double) * mk, S.stream));
    WB_CUDA(cudaMemsetAsync(x, 0, sizeof(double) * mk, S.stream));
    publish_active(S, B.n_active.p);
    WB_CUDA(cudaStreamSynchronize(S.stream));
    S.gpu_launches += 2;
    for (int itn = 1; itn <= S.params.maxiter && *S.h_active > 0; ++itn) {
        // one pass over the observations: u_{k+1} = A v_k + scale u_k (into the other u
        // buffer), its squared norm per warp, and A'u_{k+1}
        const int nw = launch_obs<double, OBS_LSMR>(S, kp, sw, B.v.p, B.u.p, B.atu.p, B.av.p, B.scale.p, part);
        launch_reduce(S, part, nw, kp, red);
        std::swap(B.u, B.av);
        lsmr_beta_kernel<<<1, 32, 0, S.stream>>>(s, red, kp);
        S.gpu_launches++;
        if (!precond) {
            axpby(B.v.p, B.atu.p, B.pa.p, 1.0, B.pb.p, !cap);  // v = A'u / beta - beta v, red = ||v||^2
            if (cap) {
                ring_sweep();
                dot(B.v.p, B.v.p);
            }
        } else {
            axpby(B.pt.p, B.atu.p, B.pa.p, 1.0, B.pb.p, false);  // p~ = A'u / beta - (beta / alpha) p~
            int nbp = 0;
            apply_precond<double>(S, B.pt.p, B.v.p, kp, nullptr, nbp);
            if (cap) ring_sweep();
            dot(B.v.p, B.pt.p);
        }
        lsmr_step_kernel<<<1, 32, 0, S.stream>>>(s, red, kp, itn);
        S.gpu_launches++;
        axpby(B.v.p, B.v.p, B.inv_alpha.p, 1.0, B.zeros.p, false);  // v /= alpha_{k+1}
        if (cap) ring_push();
        WB_DISPATCH_G(G, lsmr_update_kernel<GV><<<gm, kBlock, 0, S.stream>>>(x, B.h.p, B.hb.p, B.v.p, B.coef.p, m, kp));
        WB_CUDA(cudaGetLastError());
        S.gpu_launches++;
        publish_active(S, B.n_active.p);
        WB_CUDA(cudaStreamSynchronize(S.stream));
    }
    conv.assign(kp, 0);
    iters.assign(kp, 0);
    read_small(S, conv.data(), B.conv.p, sizeof(int32_t) * kp);
    read_small(S, iters.data(), B.iters.p, sizeof(int32_t) * kp);
}

}  // namespace

// ---------------------------------------------------------------------------
// Solve drivers
// ---------------------------------------------------------------------------

namespace {

struct BatchOut {
    std::vector<int32_t> conv, iters;
    std::vector<double> fres;
};

std::vector<double> host_reduce(SolverImpl& S, int nb, int kp) {
    std::vector<double> hpart((size_t)nb * kp), out(kp, 0.0);
    read_small(S, hpart.data(), S.ws.part.p, sizeof(double) * nb * kp);
    for (int c = 0; c < kp; ++c)
        for (int b = 0; b < nb; ++b) out[c] += hpart[(size_t)b * kp + c];
    return out;
}

// Solve k <= 32 RHS with device inputs ycol (n x k RHS-major) into device outputs
// x (n_dofs x k RHS-major) and dem (n x k RHS-major).  Solver::solve semantics
// (solver.rs:209-238) batched over RHS, with the refinement residual b - G x (computed
// as D'W (y - D x) when that check may be the last).
#ifndef WB_MIXED_EXIT_MARGIN
#define WB_MIXED_EXIT_MARGIN 0.3
#endif
constexpr double kMixedExitMargin = WB_MIXED_EXIT_MARGIN;

void solve_chunk(SolverImpl& S, const double* ycol, int k, double* xcol, double* demcol, BatchOut& out) {
    const int kp = pad_kp(k);
    ensure_ws(S, kp);
    Workspace& w = S.ws;
    const int64_t n = S.d.n, m = S.d.ndofs;
    const uint32_t* perm = S.perm_identity ? nullptr : S.perm.p;
    // y -> interleaved, primary-sorted, padded to kp columns
    if (perm) {  // user order interleaved (coalesced), then the rows into primary order
        gather_interleave_kernel<double><<<xpose_blocks(n, S.n_sm), kXposeWarps * 32, xpose_smem(kp), S.stream>>>(ycol, n, k, kp, nullptr, w.e.p);
        permute_rows_kernel<<<S.nblk(n * kp / 2, 1), kBlock, 0, S.stream>>>(w.e.p, n, kp, perm, 0, w.yi.p);
        S.gpu_launches++;
    } else {
        gather_interleave_kernel<double><<<xpose_blocks(n, S.n_sm), kXposeWarps * 32, xpose_smem(kp), S.stream>>>(ycol, n, k, kp, nullptr, w.yi.p);
    }
    // b = D'W y (rmatvec_wdt, solver.rs:210-211)
    launch_obs<double, OBS_RHS>(S, kp, S.w64.p, nullptr, w.yi.p, w.b.p, nullptr);
    obs_autotune<double>(S, kp, S.w64.p, w.b.p, w.gx.p);  // FP64 passes: refinement and demeaning
    int nb = 0;
    launch_dot<double, double>(S, w.b.p, w.b.p, m, kp, w.part.p, nb);
    std::vector<double> bb = host_reduce(S, nb, kp);
    std::vector<double> rhs_norm(kp), abs_tol(kp);
    // Mixed precision refines until the FP64 residual is kMixedExitMargin x the tolerance:
    // its last correction is a short FP32 solve, whose error at a given residual is larger
    // than that of a CG that ran the whole way, so the margin keeps its result at least
    // as accurate as the FP64 solve's at the same tolerance.  `converged` is still judged
    // on tol (final FP64 residual).
    const double exit_margin = S.mixed() ? kMixedExitMargin : 1.0;
    for (int c = 0; c < kp; ++c) {
        rhs_norm[c] = std::max(std::sqrt(bb[c]), 1e-15);  // solver.rs:212
        abs_tol[c] = exit_margin * S.params.tol * rhs_norm[c];
    }
    std::vector<int32_t> conv(kp, 0), iters(kp, 0), part_of(kp, 0);
    std::vector<double> final_rr;  // set when w.e and w.r already hold the final e and D'W e
    for (int c = 0; c < k; ++c) part_of[c] = 1;
    std::vector<double> tol(kp, S.params.tol);
    if (S.params.krylov == WITHIN_KRYLOV_LSMR) {
        // Solver::solve, LSMR branch (solver.rs:162-203): mlsmr on W^(1/2) D, FP64, no
        // refinement; converged and iterations are LSMR's own
        if (!S.lsmr) S.lsmr = std::make_shared<LsmrBufs>();
        lsmr_device(S, *std::static_pointer_cast<LsmrBufs>(S.lsmr), kp, w.yi.p, w.x.p, part_of, conv, iters);
    } else {
        // One inner Krylov solve of G d = rhs on the RHS in `who` to relative tolerances tl,
        // then x += d on those RHS.
        auto run_inner = [&](const double* rhs, const std::vector<int32_t>& who, const std::vector<double>& tl,
                             std::vector<int32_t>& cv, std::vector<int32_t>& it) {
            write_small(S, w.st_part.p, who.data(), w.st_tol.p, tl.data(), kp);
            WB_CUDA(cudaMemsetAsync(w.st_conv.p, 0, sizeof(int32_t) * 32, S.stream));
            const int grid = S.nblk(m * kp, 1);
            if (S.params.krylov == WITHIN_KRYLOV_GMRES) {
                if (!S.gmres) S.gmres = std::make_shared<GmresBufs>();
                GmresBufs& B = *std::static_pointer_cast<GmresBufs>(S.gmres);
                if (!S.mixed()) gmres_device<double>(S, B, kp, rhs, w.cx.p, S.params.maxiter);
                else gmres_device<float>(S, B, kp, rhs, w.cx.p, S.params.maxiter);
                masked_axpy_kernel<double><<<grid, kBlock, 0, S.stream>>>(w.x.p, w.cx.p, w.st_part.p, m, kp);
                WB_CUDA(cudaMemcpyAsync(w.st_conv.p, B.conv.p, sizeof(int32_t) * kp, cudaMemcpyDeviceToDevice, S.stream));
                WB_CUDA(cudaMemcpyAsync(w.st_iters.p, B.iters.p, sizeof(int32_t) * kp, cudaMemcpyDeviceToDevice, S.stream));
            } else if (!S.mixed()) {
                cg_device<double>(S, kp, rhs, w.cx.p, w.cr.p, w.dz.p, w.dp.p, w.dap.p, S.params.maxiter);
                masked_axpy_kernel<double><<<grid, kBlock, 0, S.stream>>>(w.x.p, w.cx.p, w.st_part.p, m, kp);
            } else {
                convert_kernel<double, float><<<grid, kBlock, 0, S.stream>>>(rhs, w.frhs.p, m * kp);
                cg_device<float>(S, kp, w.frhs.p, w.fx.p, w.fr.p, w.fz.p, w.fp.p, w.fap.p, S.params.maxiter);
                masked_axpy_kernel<float><<<grid, kBlock, 0, S.stream>>>(w.x.p, w.fx.p, w.st_part.p, m, kp);
            }
            WB_CUDA(cudaGetLastError());
            S.gpu_launches += 2;
            cv.assign(kp, 0);
            it.assign(kp, 0);
            read_small(S, cv.data(), w.st_conv.p, sizeof(int32_t) * kp);
            read_small(S, it.data(), w.st_iters.p, sizeof(int32_t) * kp);
        };
        WB_CUDA(cudaMemsetAsync(w.x.p, 0, sizeof(double) * m * kp, S.stream));
        std::vector<int32_t> cv, it;
        // FP64: initial solve + max_refinements corrections (solver.rs:215-216, 296-333).
        // Mixed: FP32 inner solves to >= 1e-5 relative inside an FP64 refinement loop of up to
        // max_refinements + 4 corrections, stopping when ||b - G x|| <= tol ||b||.
        const int n_corr = S.mixed() ? S.params.max_refinements + 4 : S.params.max_refinements;
        if (!S.mixed()) {
            run_inner(w.b.p, part_of, tol, cv, it);
            conv = cv;
            iters = it;
        }
        std::vector<int32_t> done(kp, 0);
        for (int c = k; c < kp; ++c) done[c] = 1;
        for (int ref = 0; ref <= n_corr; ++ref) {
            if (!S.mixed() && ref == n_corr) break;
            const bool first_mixed = S.mixed() && ref == 0;
            const double* rhs = w.b.p;
            // The residual b - G x equals D'W (y - D x).  A mixed-precision check after the
            // first correction, likely the last, computes it that way, with e = y - D x, so
            // that when it ends the loop it is also the final demeaning below.  (FP64 runs
            // usually end with a correction after the last check, so theirs stay b - G x.)
            const bool resid = S.mixed() && ref >= 2;
            if (resid) {
                launch_obs<double, OBS_RESID>(S, kp, S.w64.p, w.x.p, w.yi.p, w.r.p, w.e.p);
                rhs = w.r.p;
            } else if (!first_mixed) {  // r = b - G x in FP64
                cudaEvent_t e0 = nullptr;
                S.prof_begin(e0);
                launch_gram<double>(S, kp, S.w64.p, w.x.p, w.gx.p);
                S.prof_end(0, e0);
                const int grid = S.nblk(m * kp, 1);
                sub_kernel<<<grid, kBlock, 0, S.stream>>>(w.b.p, w.gx.p, w.r.p, m * kp);
                WB_CUDA(cudaGetLastError());
                S.gpu_launches++;
                rhs = w.r.p;
            }
            launch_dot<double, double>(S, rhs, rhs, m, kp, w.part.p, nb);
            std::vector<double> rr = host_reduce(S, nb, kp);
            std::vector<int32_t> who(kp, 0);
            std::vector<double> ctol(kp, 1.0);
            int nwho = 0;
            for (int c = 0; c < k; ++c) {
                if (done[c]) continue;
                const double cn = std::sqrt(rr[c]);
                if (cn <= abs_tol[c]) { done[c] = 1; continue; }
                ctol[c] = std::min(abs_tol[c] / cn, 1.0);  // corr_tol (solver.rs:319-320)
                if (S.mixed()) ctol[c] = std::max(ctol[c], 1e-5);
                who[c] = 1;
                ++nwho;
            }
            if (nwho == 0 || ref == n_corr) {
                if (resid) final_rr = rr;  // x is unchanged since this check
                break;
            }
            run_inner(rhs, who, ctol, cv, it);
            for (int c = 0; c < k; ++c)
                if (who[c]) { iters[c] += it[c]; conv[c] = cv[c]; }
        }
        if (S.mixed()) {
            // converged when the FP64 residual met the tolerance
            for (int c = 0; c < k; ++c) conv[c] = done[c] ? 1 : 0;
        }
    }
    // final demeaned e = y - D x and ||D'W e|| / ||b|| (solver.rs:222-227, 335-339)
    if (final_rr.empty()) {
        launch_obs<double, OBS_RESID>(S, kp, S.w64.p, w.x.p, w.yi.p, w.r.p, w.e.p);
        launch_dot<double, double>(S, w.r.p, w.r.p, m, kp, w.part.p, nb);
    }
    if (perm) {  // the rows back into user order (yi is free now), then column-major
        permute_rows_kernel<<<S.nblk(n * kp / 2, 1), kBlock, 0, S.stream>>>(w.e.p, n, kp, perm, 1, w.yi.p);
        scatter_deinterleave_kernel<double><<<xpose_blocks(n, S.n_sm), kXposeWarps * 32, xpose_smem(kp), S.stream>>>(w.yi.p, n, k, kp, nullptr, demcol);
        S.gpu_launches++;
    } else {
        scatter_deinterleave_kernel<double><<<xpose_blocks(n, S.n_sm), kXposeWarps * 32, xpose_smem(kp), S.stream>>>(w.e.p, n, k, kp, nullptr, demcol);
    }
    scatter_deinterleave_kernel<double><<<xpose_blocks(m, S.n_sm), kXposeWarps * 32, xpose_smem(kp), S.stream>>>(w.x.p, m, k, kp, nullptr, xcol);
    WB_CUDA(cudaGetLastError());
    S.gpu_launches += 3;
    if (!final_rr.empty()) WB_CUDA(cudaStreamSynchronize(S.stream));  // as host_reduce would
    const std::vector<double> ee = final_rr.empty() ? host_reduce(S, nb, kp) : final_rr;
    S.prof_harvest();
    out.conv.assign(conv.begin(), conv.begin() + k);
    out.iters.assign(iters.begin(), iters.begin() + k);
    out.fres.resize(k);
    for (int c = 0; c < k; ++c) out.fres[c] = std::sqrt(ee[c]) / rhs_norm[c];
    if (S.mixed())
        for (int c = 0; c < k; ++c) out.conv[c] = out.fres[c] <= S.params.tol ? 1 : 0;
}

// ---------------------------------------------------------------------------
// Learned coarse space: the network's forward and backward passes on this solver's
// design, and the coarse correction it feeds (see coarse.cuh)
// ---------------------------------------------------------------------------

// Offsets of the parameter vector (FP32 masters; the forward pass reads BF16 copies).
struct CnLayout {
    int64_t W[kCnLayers], b[kCnLayers], Wo;
    CnLayout() {
        int64_t o = 0;
        int fin = kCnIn;
        for (int l = 0; l < kCnLayers; ++l) {
            W[l] = o; o += (int64_t)2 * fin * kCnHidden;
            b[l] = o; o += kCnHidden;
            fin = kCnHidden;
        }
        Wo = o;
    }
};

// Device buffers of one network evaluation on a design of m levels.
struct CnState {
    int64_t m = 0;
    DArr<double> d, cnt, isq;
    DArr<float> X, H[kCnLayers], P[kCnLayers], T, GT, Zt, w32;
    DArr<float> params;
    DArr<__nv_bfloat16> pb;
    // backward
    DArr<float> dZ, dH, dpre, dS, ones, grad, fpart;
    DArr<double> dpart, small;
};

int cn_blocks(int64_t n) { return (int)std::max<int64_t>(1, (n + 255) / 256); }

// diag(G), level counts and D^-1/2 of the design, on the device
void cn_design_stats(SolverImpl& S, CnState& C) {
    const Design& d = S.d;
    const int64_t m = d.ndofs;
    std::vector<double> dg((size_t)m, 0.0), cnt((size_t)m, 0.0), isq((size_t)m, 0.0);
    for (int q = 0; q < d.Q; ++q) {
        const uint32_t* c = d.codes.data() + (size_t)q * d.n;
        const int64_t o = d.off[q];
        for (int64_t i = 0; i < d.n; ++i) {
            dg[(size_t)(o + c[i])] += d.weight(i);
            cnt[(size_t)(o + c[i])] += 1.0;
        }
    }
    for (int64_t l = 0; l < m; ++l) isq[(size_t)l] = dg[(size_t)l] > 0.0 ? 1.0 / std::sqrt(dg[(size_t)l]) : 0.0;
    C.m = m;
    C.d.upload(dg);
    C.cnt.upload(cnt);
    C.isq.upload(isq);
}

// P[:, pc0:pc0+ncols] (+)= Ahat H[:, 0:ncols] (H has row stride F >= ncols, P row stride
// PF >= pc0 + ncols) via passes of the FP32 observation pass over column blocks of 16 or
// 32 (ncols a multiple of 16).
void cn_ahat(SolverImpl& S, CnState& C, const float* H, int F, int ncols, float* P, int PF, int pc0, bool accumulate) {
    const int64_t m = C.m;
    const float* w = S.w32.p ? S.w32.p : C.w32.p;  // null: unit weights
    for (int c0 = 0; c0 < ncols; c0 += 32) {
        const int kt = std::min(32, ncols - c0);
        cn_scale_cols_kernel<<<cn_blocks(m * kt), 256, 0, S.stream>>>(m, F, c0, kt, H, C.isq.p, C.T.p);
        launch_obs<float, OBS_GRAM>(S, kt, w, C.T.p, nullptr, C.GT.p, nullptr);
        cn_combine_kernel<<<cn_blocks(m * kt), 256, 0, S.stream>>>(m, F, c0, kt, C.GT.p, C.isq.p, H, P, PF, pc0 + c0,
                                                                   accumulate ? 1 : 0);
        WB_CUDA(cudaGetLastError());
        S.gpu_launches += 2;
    }
}

template <int N, int ACT>
void cn_dense(SolverImpl& S, int64_t m, const float* A0, int K0, const float* A1, int K1, const __nv_bfloat16* W,
              const float* bias, float* out) {
    const size_t smem = sizeof(__nv_bfloat16) * (size_t)(K0 + K1) * N;
    const int64_t warps = (m + 15) / 16;
    const int grid = (int)std::max<int64_t>(1, (warps + 3) / 4);
    cn_dense_fwd_kernel<N, ACT><<<grid, 128, smem, S.stream>>>(m, A0, K0, A1, K1, W, bias, out);
    WB_CUDA(cudaGetLastError());
    S.gpu_launches++;
}

// Buffers for a design (features once per seed) and the parameters (FP32 + BF16).
void cn_prepare(SolverImpl& S, CnState& C, const float* params, uint64_t seed) {
    if (C.m == 0) cn_design_stats(S, C);
    const int64_t m = C.m;
    if (S.w64.p && !S.w32.p && !C.w32.p) {  // FP32 weights for the FP32 observation pass
        C.w32.alloc((size_t)S.obs.ns);
        convert_kernel<double, float><<<S.nblk(S.obs.ns, 1), kBlock, 0, S.stream>>>(S.w64.p, C.w32.p, S.obs.ns);
        WB_CUDA(cudaGetLastError());
    }
    C.X.alloc((size_t)m * kCnIn);
    for (int l = 0; l < kCnLayers; ++l) {
        C.H[l].alloc((size_t)m * kCnHidden);
        C.P[l].alloc((size_t)m * (l == 0 ? kCnIn : kCnHidden));
    }
    C.T.alloc((size_t)m * 32);
    C.GT.alloc((size_t)m * 32);
    C.Zt.alloc((size_t)m * kCnOut);
    CnOffsets fo{};
    fo.Q = S.d.Q;
    for (int q = 0; q < S.d.Q; ++q) fo.off[q] = S.d.off[q];
    fo.off[S.d.Q] = m;
    cn_features_kernel<<<cn_blocks(m), 256, 0, S.stream>>>(m, fo, C.d.p, C.cnt.p, seed, C.X.p);
    C.params.alloc(kCnParams);
    C.pb.alloc(kCnParams);
    WB_CUDA(cudaMemcpyAsync(C.params.p, params, sizeof(float) * kCnParams, cudaMemcpyHostToDevice, S.stream));
    cn_to_bf16_kernel<<<cn_blocks(kCnParams), 256, 0, S.stream>>>(kCnParams, C.params.p, C.pb.p);
    WB_CUDA(cudaGetLastError());
    S.gpu_launches += 2;
}

// Zt = network(X): H_0 = X, H_{l+1} = tanh(bf16([Ahat H_l, H_l]) W_l + b_l), Zt = bf16(H_3) W_o
void cn_forward(SolverImpl& S, CnState& C) {
    static const CnLayout L;
    const int64_t m = C.m;
    const float* Hin = C.X.p;
    int F = kCnIn;
    for (int l = 0; l < kCnLayers; ++l) {
        cn_ahat(S, C, Hin, F, F, C.P[l].p, F, 0, false);
        cn_dense<kCnHidden, 1>(S, m, C.P[l].p, F, Hin, F, C.pb.p + L.W[l], C.params.p + L.b[l], C.H[l].p);
        Hin = C.H[l].p;
        F = kCnHidden;
    }
    cn_dense<kCnOut, 0>(S, m, C.H[kCnLayers - 1].p, kCnHidden, nullptr, 0, C.pb.p + L.Wo, nullptr, C.Zt.p);
}

// sum_rows a' b into out (K x N) with the block partials of cn_tn_partial_kernel
template <typename TACC, typename TOUT>
void cn_tn(SolverImpl& S, CnState& C, int64_t m, const float* A0, int K0, const float* A1, int K1, bool round_a,
           const float* B, int N, TOUT* out) {
    const int nb = (int)std::max<int64_t>(1, std::min<int64_t>((m + 255) / 256, (int64_t)S.n_sm * 2));
    const int64_t KN = (int64_t)(K0 + K1) * N;
    TACC* part;
    if (std::is_same<TACC, double>::value) {
        C.dpart.alloc((size_t)nb * KN);
        part = reinterpret_cast<TACC*>(C.dpart.p);
    } else {
        C.fpart.alloc((size_t)nb * KN);
        part = reinterpret_cast<TACC*>(C.fpart.p);
    }
    cn_tn_partial_kernel<TACC><<<nb, 256, 0, S.stream>>>(m, A0, K0, A1, K1, round_a ? 1 : 0, B, N, part);
    cn_reduce_partials_kernel<TACC, TOUT><<<cn_blocks(KN), 256, 0, S.stream>>>(part, nb, KN, out);
    WB_CUDA(cudaGetLastError());
    S.gpu_launches += 2;
}

// Loss L = 1 - tr(B'A^-1 B)/t (A = Zt'Zt + eps I, B = Zt'V) and the gradient of every
// parameter into grad (kCnParams, FP32).  V: the design's targets (m x t).
double cn_backward(SolverImpl& S, CnState& C, float* grad_host) {
    static const CnLayout L;
    const int64_t m = C.m;
    const int t = S.cn_t;
    const float* V = S.cn_targets.p;
    C.small.alloc((size_t)32 * 32 * 2 + 32 * 32 * 2);
    double* dA = C.small.p;              // 32 x 32
    double* dB = C.small.p + 32 * 32;    // 32 x t
    cn_tn<double, double>(S, C, m, C.Zt.p, kCnOut, nullptr, 0, false, C.Zt.p, kCnOut, dA);
    cn_tn<double, double>(S, C, m, C.Zt.p, kCnOut, nullptr, 0, false, V, t, dB);
    std::vector<double> A(32 * 32), B((size_t)32 * t);
    WB_CUDA(cudaMemcpyAsync(A.data(), dA, sizeof(double) * 32 * 32, cudaMemcpyDeviceToHost, S.stream));
    WB_CUDA(cudaMemcpyAsync(B.data(), dB, sizeof(double) * 32 * t, cudaMemcpyDeviceToHost, S.stream));
    WB_CUDA(cudaStreamSynchronize(S.stream));
    // A += eps I, A^-1 by Gauss-Jordan (32 x 32, SPD)
    double tr = 0.0;
    for (int i = 0; i < 32; ++i) tr += A[i * 32 + i];
    for (int i = 0; i < 32; ++i) A[i * 32 + i] += 1e-6 * tr / 32.0 + 1e-300;
    std::vector<double> Ai(32 * 32, 0.0);
    {
        std::vector<double> M(A);
        for (int i = 0; i < 32; ++i) Ai[i * 32 + i] = 1.0;
        for (int c = 0; c < 32; ++c) {
            int piv = c;
            for (int r = c + 1; r < 32; ++r)
                if (std::fabs(M[r * 32 + c]) > std::fabs(M[piv * 32 + c])) piv = r;
            if (piv != c)
                for (int j = 0; j < 32; ++j) { std::swap(M[c * 32 + j], M[piv * 32 + j]); std::swap(Ai[c * 32 + j], Ai[piv * 32 + j]); }
            const double inv = 1.0 / M[c * 32 + c];
            for (int j = 0; j < 32; ++j) { M[c * 32 + j] *= inv; Ai[c * 32 + j] *= inv; }
            for (int r = 0; r < 32; ++r) {
                if (r == c) continue;
                const double f = M[r * 32 + c];
                if (f == 0.0) continue;
                for (int j = 0; j < 32; ++j) { M[r * 32 + j] -= f * M[c * 32 + j]; Ai[r * 32 + j] -= f * Ai[c * 32 + j]; }
            }
        }
    }
    std::vector<double> AiB((size_t)32 * t, 0.0);  // 32 x t
    for (int i = 0; i < 32; ++i)
        for (int a = 0; a < 32; ++a)
            for (int j = 0; j < t; ++j) AiB[(size_t)i * t + j] += Ai[i * 32 + a] * B[(size_t)a * t + j];
    double trv = 0.0;
    for (int i = 0; i < 32; ++i)
        for (int j = 0; j < t; ++j) trv += B[(size_t)i * t + j] * AiB[(size_t)i * t + j];
    const double loss = 1.0 - trv / t;
    // dZ = V C1 + Z C2: C1 = -2/t (A^-1 B)' (t x 32), C2 = 2/t (A^-1 B)(A^-1 B)' (32 x 32)
    std::vector<double> C1((size_t)t * 32), C2(32 * 32, 0.0);
    for (int j = 0; j < t; ++j)
        for (int i = 0; i < 32; ++i) C1[(size_t)j * 32 + i] = -2.0 / t * AiB[(size_t)i * t + j];
    for (int i = 0; i < 32; ++i)
        for (int k = 0; k < 32; ++k) {
            double v = 0.0;
            for (int j = 0; j < t; ++j) v += AiB[(size_t)i * t + j] * AiB[(size_t)k * t + j];
            C2[i * 32 + k] = 2.0 / t * v;
        }
    WB_CUDA(cudaMemcpyAsync(dA, C1.data(), sizeof(double) * t * 32, cudaMemcpyHostToDevice, S.stream));
    WB_CUDA(cudaMemcpyAsync(dB, C2.data(), sizeof(double) * 32 * 32, cudaMemcpyHostToDevice, S.stream));
    C.dZ.alloc((size_t)m * kCnOut);
    C.dH.alloc((size_t)m * kCnHidden);
    C.dpre.alloc((size_t)m * kCnHidden);
    C.dS.alloc((size_t)m * 2 * kCnHidden);
    C.grad.alloc(kCnParams);
    if (C.ones.n < (size_t)m) {
        std::vector<float> one((size_t)m, 1.0f);
        C.ones.upload(one);
    }
    cn_dz_kernel<<<cn_blocks(m * 32), 256, 0, S.stream>>>(m, V, t, dA, C.Zt.p, dB, C.dZ.p);
    // W_o: H_3' dZ (H_3 rounded as the forward pass read it); dH_3 = dZ W_o'
    cn_tn<float, float>(S, C, m, C.H[kCnLayers - 1].p, kCnHidden, nullptr, 0, true, C.dZ.p, kCnOut, C.grad.p + L.Wo);
    {
        const size_t smem = sizeof(float) * kCnHidden * kCnOut;
        cn_matmul_nt_kernel<<<S.nblk(m * kCnHidden, 1), 256, smem, S.stream>>>(m, C.dZ.p, kCnOut, C.pb.p + L.Wo,
                                                                              kCnHidden, C.dH.p);
    }
    for (int l = kCnLayers - 1; l >= 0; --l) {
        const int F = l == 0 ? kCnIn : kCnHidden;
        const float* Hl = l == 0 ? C.X.p : C.H[l - 1].p;
        cn_dtanh_kernel<<<cn_blocks(m * kCnHidden), 256, 0, S.stream>>>(m * kCnHidden, C.dH.p, C.H[l].p, C.dpre.p);
        cn_tn<float, float>(S, C, m, C.P[l].p, F, Hl, F, true, C.dpre.p, kCnHidden, C.grad.p + L.W[l]);
        cn_tn<float, float>(S, C, m, C.ones.p, 1, nullptr, 0, false, C.dpre.p, kCnHidden, C.grad.p + L.b[l]);
        if (l == 0) break;
        // dS = dpre W_l' (m x 2F); dH_l = dS[:, F:] + Ahat dS[:, :F]
        const size_t smem = sizeof(float) * 2 * F * kCnHidden;
        if (smem > 48 * 1024) WB_CUDA(cudaFuncSetAttribute(cn_matmul_nt_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        cn_matmul_nt_kernel<<<S.nblk(m * 2 * F, 1), 256, smem, S.stream>>>(m, C.dpre.p, kCnHidden, C.pb.p + L.W[l],
                                                                           2 * F, C.dS.p);
        cn_copy_cols_kernel<<<cn_blocks(m * F), 256, 0, S.stream>>>(m, 2 * F, F, F, C.dS.p, C.dH.p, F, 0);
        cn_ahat(S, C, C.dS.p, 2 * F, F, C.dH.p, F, 0, true);
    }
    WB_CUDA(cudaGetLastError());
    S.gpu_launches += 8;
    WB_CUDA(cudaMemcpyAsync(grad_host, C.grad.p, sizeof(float) * kCnParams, cudaMemcpyDeviceToHost, S.stream));
    WB_CUDA(cudaStreamSynchronize(S.stream));
    return loss;
}

// Eigen-decomposition of a symmetric n x n matrix by cyclic Jacobi rotations (n <= 32):
// A is destroyed, eigenvalues into lam, eigenvectors into the columns of V.
void jacobi_eigen(std::vector<double>& A, int n, std::vector<double>& lam, std::vector<double>& V) {
    V.assign((size_t)n * n, 0.0);
    for (int i = 0; i < n; ++i) V[(size_t)i * n + i] = 1.0;
    for (int sweep = 0; sweep < 100; ++sweep) {
        double off = 0.0, tot = 0.0;
        for (int i = 0; i < n; ++i)
            for (int j = 0; j < n; ++j) {
                tot += A[(size_t)i * n + j] * A[(size_t)i * n + j];
                if (i != j) off += A[(size_t)i * n + j] * A[(size_t)i * n + j];
            }
        if (off <= 1e-30 * std::max(tot, 1e-300)) break;
        for (int p = 0; p < n; ++p)
            for (int q = p + 1; q < n; ++q) {
                const double apq = A[(size_t)p * n + q];
                if (std::fabs(apq) < 1e-300) continue;
                const double app = A[(size_t)p * n + p], aqq = A[(size_t)q * n + q];
                const double theta = (aqq - app) / (2.0 * apq);
                const double tt = (theta >= 0 ? 1.0 : -1.0) / (std::fabs(theta) + std::sqrt(theta * theta + 1.0));
                const double c = 1.0 / std::sqrt(tt * tt + 1.0), s = tt * c;
                for (int k = 0; k < n; ++k) {
                    const double akp = A[(size_t)k * n + p], akq = A[(size_t)k * n + q];
                    A[(size_t)k * n + p] = c * akp - s * akq;
                    A[(size_t)k * n + q] = s * akp + c * akq;
                }
                for (int k = 0; k < n; ++k) {
                    const double apk = A[(size_t)p * n + k], aqk = A[(size_t)q * n + k];
                    A[(size_t)p * n + k] = c * apk - s * aqk;
                    A[(size_t)q * n + k] = s * apk + c * aqk;
                }
                for (int k = 0; k < n; ++k) {
                    const double vkp = V[(size_t)k * n + p], vkq = V[(size_t)k * n + q];
                    V[(size_t)k * n + p] = c * vkp - s * vkq;
                    V[(size_t)k * n + q] = s * vkp + c * vkq;
                }
            }
    }
    lam.resize(n);
    for (int i = 0; i < n; ++i) lam[i] = A[(size_t)i * n + i];
}

// Installs the coarse space spanned by the columns of Z64 (m x 32 row-major, FP64, on the
// device): GZ = G Z and E = Z'GZ in FP64, E's pseudo-inverse (eigenvalues below 1e-10 of
// the largest dropped: null-space directions of G), and FP32 copies of Z and GZ for
// mixed precision.
void install_coarse(SolverImpl& S) {
    const int64_t m = S.d.ndofs;
    S.coarse_gz64.alloc((size_t)m * 32);
    launch_gram<double>(S, 32, S.w64.p, S.coarse_z64.p, S.coarse_gz64.p);
    const int nbc = coarse_blocks(S);
    S.coarse_part.alloc((size_t)nbc * 32 * 32);
    S.coarse_u.alloc(2 * 32 * 32);
    S.coarse_einv.alloc(32 * 32);
    coarse_tn_kernel<double><<<nbc, 256, 0, S.stream>>>(m, S.coarse_z64.p, S.coarse_gz64.p, 32, S.coarse_part.p);
    // E = the sum of the partials: coarse_solve with the identity as "E^+" gives u = E
    std::vector<double> I(32 * 32, 0.0);
    for (int i = 0; i < 32; ++i) I[i * 32 + i] = 1.0;
    WB_CUDA(cudaMemcpyAsync(S.coarse_einv.p, I.data(), sizeof(double) * 32 * 32, cudaMemcpyHostToDevice, S.stream));
    coarse_solve_kernel<<<1, kCoarseSolveThreads, 0, S.stream>>>(S.coarse_part.p, nbc, S.coarse_einv.p, 32, S.coarse_u.p);
    WB_CUDA(cudaGetLastError());
    S.gpu_launches += 2;
    std::vector<double> E(32 * 32);
    WB_CUDA(cudaMemcpyAsync(E.data(), S.coarse_u.p, sizeof(double) * 32 * 32, cudaMemcpyDeviceToHost, S.stream));
    WB_CUDA(cudaStreamSynchronize(S.stream));
    for (int i = 0; i < 32; ++i)
        for (int j = i + 1; j < 32; ++j) E[i * 32 + j] = E[j * 32 + i] = 0.5 * (E[i * 32 + j] + E[j * 32 + i]);
    std::vector<double> lam, V;
    jacobi_eigen(E, 32, lam, V);
    double lmax = 0.0;
    for (double v : lam) lmax = std::max(lmax, v);
    std::vector<double> Ei(32 * 32, 0.0);
    for (int k = 0; k < 32; ++k) {
        if (!(lam[k] > 1e-10 * lmax)) continue;
        const double inv = 1.0 / lam[k];
        for (int i = 0; i < 32; ++i)
            for (int j = 0; j < 32; ++j) Ei[i * 32 + j] += V[(size_t)i * 32 + k] * inv * V[(size_t)j * 32 + k];
    }
    WB_CUDA(cudaMemcpyAsync(S.coarse_einv.p, Ei.data(), sizeof(double) * 32 * 32, cudaMemcpyHostToDevice, S.stream));
    if (S.mixed()) {
        S.coarse_z32.alloc((size_t)m * 32);
        S.coarse_gz32.alloc((size_t)m * 32);
        convert_kernel<double, float><<<S.nblk(m * 32, 1), kBlock, 0, S.stream>>>(S.coarse_z64.p, S.coarse_z32.p, m * 32);
        convert_kernel<double, float><<<S.nblk(m * 32, 1), kBlock, 0, S.stream>>>(S.coarse_gz64.p, S.coarse_gz32.p, m * 32);
        WB_CUDA(cudaGetLastError());
    }
    WB_CUDA(cudaStreamSynchronize(S.stream));
    S.coarse_k = 32;
    if (S.cg_exec) {  // the captured CG iteration changes
        WB_CUDA(cudaGraphExecDestroy(S.cg_exec));
        S.cg_exec = nullptr;
    }
}

}  // namespace

}  // namespace wb

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------

using wb::SolverImpl;

struct within_solver {
    std::unique_ptr<SolverImpl> impl;
};

namespace {

int guard(const std::function<int()>& f) {
    try {
        const int rc = f();
        if (rc == WITHIN_OK) wb::g_last_error.clear();
        return rc;
    } catch (const wb::CudaError& e) {
        return wb::fail(WITHIN_ERR_CUDA, e.what());
    } catch (const std::bad_alloc&) {
        return wb::fail(WITHIN_ERR_OVERFLOW, "out of host memory");
    } catch (const std::exception& e) {
        return wb::fail(WITHIN_ERR_INVALID_ARGUMENT, e.what());
    }
}


// Device attributes, the solver's stream and its pinned status word.
void init_device(SolverImpl& S) {
    int dev = 0;
    WB_CUDA(cudaGetDevice(&dev));
    WB_CUDA(cudaDeviceGetAttribute(&S.n_sm, cudaDevAttrMultiProcessorCount, dev));
    int coop = 0;
    WB_CUDA(cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev));
    S.coop = coop != 0;
    WB_CUDA(cudaStreamCreateWithFlags(&S.stream, cudaStreamNonBlocking));
    WB_CUDA(cudaMallocHost(&S.h_active, sizeof(int32_t)));
}

// The device stages of the Schwarz preconditioner from the host subdomains: one stage of
// all subdomains (additive), or one per factor pair (multiplicative).
void build_precond_stages(SolverImpl& S) {
    if (S.pc.kind == 0 || S.subs.empty()) return;
    std::vector<std::vector<int32_t>> groups;
    if (S.pc.kind == 1) {
        groups.emplace_back(S.subs.size());
        std::iota(groups[0].begin(), groups[0].end(), 0);
    } else {
        for (int32_t i = 0; i < (int32_t)S.subs.size(); ++i) {
            if (groups.empty() || S.subs[groups.back()[0]].q != S.subs[i].q || S.subs[groups.back()[0]].r != S.subs[i].r)
                groups.emplace_back();
            groups.back().push_back(i);
        }
    }
    for (auto& g : groups) {
        const wb::StageHost h = wb::build_stage(S.subs, g, S.d.ndofs, S.pc.kind == 1);
        S.max_nsub = std::max(S.max_nsub, h.nsub);
        S.max_slots = std::max(S.max_slots, h.nslots);
        S.max_core_total = std::max(S.max_core_total, (int64_t)h.core_slot.size());
        S.stages64.emplace_back();
        wb::upload_stage(S.stages64.back(), h);
        if (S.mixed()) {
            S.stages32.emplace_back();
            wb::upload_stage(S.stages32.back(), h);
        }
    }
}

// The assembled Gramian on the device, with its row chunks for the explicit operator.
void install_gramian(SolverImpl& S, const std::vector<int64_t>& gp, const std::vector<uint32_t>& gi,
                     const std::vector<double>& gv) {
    S.g_ptr.upload(gp);
    S.g_idx.upload(gi);
    S.g_val64.upload(gv);
    if (S.mixed()) S.g_val32.upload_cast(gv);
    const int64_t m = S.d.ndofs;
    std::vector<uint32_t> rows((size_t)m);
    std::iota(rows.begin(), rows.end(), 0u);
    S.g_rows.upload(rows);
    const std::vector<wb::CsrChunk> ch = wb::make_chunks(gp, 0, m, 256, 1, true);
    S.g_chunks.upload(ch);
    S.g_nchunks = (int64_t)ch.size();
    S.explicit_op = true;
}

// img: a deserialized preconditioner to use instead of building one (Solver::with_preconditioner,
// solver.rs:433-446, from_design_with_preconditioner :137-154).
int build_solver(const uint32_t* codes, size_t n_obs, size_t n_factors, int64_t row_stride, int64_t col_stride,
                 const double* weights, const within_params* params, const within_preconditioner* precond,
                 std::unique_ptr<SolverImpl>& out, wb::PrecondImage* img = nullptr) {
    const double t0 = wb::now_s();
    auto S = std::make_unique<SolverImpl>();
    within_default_params(&S->params);
    if (params) S->params = *params;
    const within_params& p = S->params;
    if (p.krylov != WITHIN_KRYLOV_CG && p.krylov != WITHIN_KRYLOV_GMRES && p.krylov != WITHIN_KRYLOV_LSMR)
        return wb::fail(WITHIN_ERR_INVALID_ARGUMENT, "config must be CG, GMRES, or LSMR");
    if (p.krylov == WITHIN_KRYLOV_LSMR && p.lsmr_local_size < 0)
        return wb::fail(WITHIN_ERR_INVALID_ARGUMENT, "LSMR local_size must be >= 0");
    if (p.krylov == WITHIN_KRYLOV_GMRES && p.gmres_restart < 1)
        return wb::fail(WITHIN_ERR_INVALID_ARGUMENT, "GMRES restart must be >= 1");
    if (precond && precond->kind == WITHIN_PRECOND_MULTIPLICATIVE && p.krylov == WITHIN_KRYLOV_CG)
        return wb::fail(WITHIN_ERR_INVALID_ARGUMENT,
                        "CG requires a symmetric preconditioner; use 'additive' or switch to GMRES");
    if (precond && precond->kind == WITHIN_PRECOND_MULTIPLICATIVE && p.krylov == WITHIN_KRYLOV_LSMR)
        return wb::fail(WITHIN_ERR_INVALID_ARGUMENT,
                        "LSMR requires a symmetric preconditioner; use 'additive' or switch to GMRES");
    if (p.operator_repr != WITHIN_OPERATOR_IMPLICIT && p.operator_repr != WITHIN_OPERATOR_EXPLICIT)
        return wb::fail(WITHIN_ERR_INVALID_ARGUMENT, "operator must be Implicit or Explicit");
    if (p.precision != WITHIN_PRECISION_FP64 && p.precision != WITHIN_PRECISION_MIXED)
        return wb::fail(WITHIN_ERR_INVALID_ARGUMENT, "precision must be FP64 or MIXED");
    if (n_factors > (size_t)wb::kMaxQ) return wb::fail(WITHIN_ERR_INVALID_ARGUMENT, "at most 16 factors are supported");
    if (codes == nullptr && n_obs > 0) return wb::fail(WITHIN_ERR_INVALID_ARGUMENT, "categories pointer is null");
    wb::Status st = wb::build_design(codes, (int64_t)n_obs, (int)n_factors, row_stride, col_stride, weights, S->d);
    if (!st.ok()) return wb::fail(st.code, st.msg);
    S->pc.kind = precond ? precond->kind : 0;
    if (precond) {
        S->pc.ac_seed = precond->approx_chol_seed;
        S->pc.ac_split = precond->approx_chol_split < 1 ? 1 : precond->approx_chol_split;
        S->pc.approx_schur = precond->approx_schur_enabled != 0;
        S->pc.schur_seed = precond->approx_schur_seed;
        S->pc.schur_split = precond->approx_schur_split < 1 ? 1 : precond->approx_schur_split;
        S->pc.dense_threshold = precond->dense_threshold;
        if (precond->reduction_strategy < 0 || precond->reduction_strategy > 2)
            return wb::fail(WITHIN_ERR_INVALID_ARGUMENT, "reduction strategy must be 0 (Auto), 1 (AtomicScatter) or 2 (ParallelReduction)");
        S->reduction_strategy = precond->reduction_strategy;
    }
    if (img) {
        if (img->ndofs != S->d.ndofs)
            return wb::fail(WITHIN_ERR_INVALID_ARGUMENT, "the preconditioner has " + std::to_string(img->ndofs) +
                                                             " dofs, the design has " + std::to_string(S->d.ndofs));
        S->pc = img->cfg;
        S->pc.kind = img->kind;
        S->reduction_strategy = img->reduction;
        S->subs = std::move(img->subs);
    }
    int dev_count = 0;
    if (cudaGetDeviceCount(&dev_count) != cudaSuccess || dev_count == 0)
        return wb::fail(WITHIN_ERR_CUDA, "no CUDA device is available (the solve phase has no CPU path)");
    // the subdomains and their factors (host) are built while the design goes to the device
    std::future<wb::Status> subs_job;
    int dev = 0;
    WB_CUDA(cudaGetDevice(&dev));
    if (S->pc.kind != 0 && !img)
        subs_job = std::async(std::launch::async, [&S, dev]() { return wb::build_subdomains(S->d, S->pc, S->subs, dev); });
    init_device(*S);
    wb::upload_design(*S);
    if (subs_job.valid()) {
        st = subs_job.get();
        if (!st.ok()) return wb::fail(st.code, st.msg);
    }
    build_precond_stages(*S);
    // the assembled Gramian (solver.rs:103-121): for an explicit operator, and for the
    // multiplicative residual updates, which then also use it as the Krylov operator
    if (p.operator_repr == WITHIN_OPERATOR_EXPLICIT || S->pc.kind == 2) {
        if (img && !img->g_ptr.empty()) {
            install_gramian(*S, img->g_ptr, img->g_idx, img->g_val);
        } else {
            std::vector<int64_t> gp;
            std::vector<uint32_t> gi;
            std::vector<double> gv;
            wb::build_explicit_gramian(S->d, gp, gi, gv);
            install_gramian(*S, gp, gi, gv);
        }
    }
    WB_CUDA(cudaStreamSynchronize(S->stream));
    S->setup_time = wb::now_s() - t0;
    out = std::move(S);
    return WITHIN_OK;
}

// A handle that holds only a deserialized preconditioner (FePreconditioner::new from
// bytes, within-py/src/lib.rs:903-913): its apply, sizes and diagnostics, no design.
int build_precond_only(wb::PrecondImage& img, std::unique_ptr<SolverImpl>& out) {
    auto S = std::make_unique<SolverImpl>();
    within_default_params(&S->params);
    S->precond_only = true;
    S->d.ndofs = img.ndofs;
    S->pc = img.cfg;
    S->pc.kind = img.kind;
    S->reduction_strategy = img.reduction;
    S->subs = std::move(img.subs);
    int dev_count = 0;
    if (cudaGetDeviceCount(&dev_count) != cudaSuccess || dev_count == 0)
        return wb::fail(WITHIN_ERR_CUDA, "no CUDA device is available (the solve phase has no CPU path)");
    init_device(*S);
    build_precond_stages(*S);
    if (S->pc.kind == 2) install_gramian(*S, img.g_ptr, img.g_idx, img.g_val);
    WB_CUDA(cudaStreamSynchronize(S->stream));
    out = std::move(S);
    return WITHIN_OK;
}

int solve_device(SolverImpl& S, const double* d_ys, size_t k, double* d_x, double* d_dem, within_solve_stats* stats) {
    if (S.precond_only)
        return wb::fail(WITHIN_ERR_INVALID_ARGUMENT, "this handle holds only a preconditioner; build a Solver to solve");
    const int64_t n = S.d.n, m = S.d.ndofs;
    for (size_t c0 = 0; c0 < k; c0 += 32) {
        const int kc = (int)std::min<size_t>(32, k - c0);
        const double t0 = wb::now_s();
        wb::BatchOut bo;
        wb::solve_chunk(S, d_ys + c0 * n, kc, d_x + c0 * m, d_dem + c0 * n, bo);
        const double dt = wb::now_s() - t0;
        if (stats)
            for (int c = 0; c < kc; ++c) {
                within_solve_stats& s = stats[c0 + c];
                s.converged = bo.conv[c];
                s.iterations = bo.iters[c];
                s.final_residual = bo.fres[c];
                s.time_solve = dt;
                s.time_setup = 0.0;
                s.time_total = dt;
            }
    }
    // LocalSolveFailed inside CG's try_apply (schwarz-precond solve/cg.rs:69, 104) ends the
    // solve with an error (IterativeSolve)
    if (wb::sweeps_failed(S))
        return wb::fail(WITHIN_ERR_ITERATIVE_SOLVE,
                        "local solve failed: an approximate-Cholesky sweep's grid barrier wait ran out");
    return WITHIN_OK;
}

}  // namespace

extern "C" {

void within_default_params(within_params* p) {
    p->krylov = WITHIN_KRYLOV_CG;
    p->gmres_restart = 30;
    p->operator_repr = WITHIN_OPERATOR_IMPLICIT;
    p->lsmr_local_size = 0;
    p->tol = 1e-8;
    p->maxiter = 1000;
    p->max_refinements = 2;
    p->precision = WITHIN_PRECISION_FP64;
}

void within_default_preconditioner(within_preconditioner* p) {
    p->kind = WITHIN_PRECOND_ADDITIVE;
    p->approx_chol_seed = 0;
    p->approx_chol_split = 2;
    p->approx_schur_enabled = 1;
    p->approx_schur_seed = 0;
    p->approx_schur_split = 1;
    p->dense_threshold = 24;
    p->reduction_strategy = 0;
}

int within_solver_new_with_preconditioner(const uint32_t* codes, size_t n_obs, size_t n_factors, int64_t row_stride,
                                          int64_t col_stride, const double* weights, const within_params* params,
                                          const uint8_t* data, size_t len, within_solver** out) {
    if (!out) return wb::fail(WITHIN_ERR_INVALID_ARGUMENT, "out pointer is null");
    *out = nullptr;
    return guard([&]() -> int {
        wb::PrecondImage img;
        const wb::Status st = wb::deserialize_preconditioner(data, len, img);
        if (!st.ok()) return wb::fail(st.code, st.msg);
        std::unique_ptr<SolverImpl> S;
        const int rc = build_solver(codes, n_obs, n_factors, row_stride, col_stride, weights, params, nullptr, S, &img);
        if (rc != WITHIN_OK) return rc;
        *out = new within_solver{std::move(S)};
        return WITHIN_OK;
    });
}

int within_preconditioner_from_bytes(const uint8_t* data, size_t len, within_solver** out) {
    if (!out) return wb::fail(WITHIN_ERR_INVALID_ARGUMENT, "out pointer is null");
    *out = nullptr;
    return guard([&]() -> int {
        wb::PrecondImage img;
        const wb::Status st = wb::deserialize_preconditioner(data, len, img);
        if (!st.ok()) return wb::fail(st.code, st.msg);
        std::unique_ptr<SolverImpl> S;
        const int rc = build_precond_only(img, S);
        if (rc != WITHIN_OK) return rc;
        *out = new within_solver{std::move(S)};
        return WITHIN_OK;
    });
}

int within_solver_preconditioner_bytes(within_solver* s, uint8_t* buf, size_t* len) {
    if (!s || !len) return wb::fail(WITHIN_ERR_INVALID_ARGUMENT, "solver and len must not be null");
    SolverImpl& S = *s->impl;
    std::lock_guard<std::mutex> lk(S.mu);
    return guard([&]() -> int {
        if (S.pc.kind == 0) return wb::fail(WITHIN_ERR_INVALID_ARGUMENT, "the solver has no preconditioner");
        if (S.pc_bytes.empty()) {
            wb::PrecondImage img;
            img.ndofs = S.d.ndofs;
            img.kind = S.pc.kind;
            img.reduction = S.reduction_strategy;
            img.cfg = S.pc;
            if (S.pc.kind == 2) {  // the residual updater's Gramian, from the device copy
                img.g_ptr.resize(S.g_ptr.n);
                img.g_idx.resize(S.g_idx.n);
                img.g_val.resize(S.g_val64.n);
                WB_CUDA(cudaMemcpy(img.g_ptr.data(), S.g_ptr.p, sizeof(int64_t) * S.g_ptr.n, cudaMemcpyDeviceToHost));
                WB_CUDA(cudaMemcpy(img.g_idx.data(), S.g_idx.p, sizeof(uint32_t) * S.g_idx.n, cudaMemcpyDeviceToHost));
                WB_CUDA(cudaMemcpy(img.g_val.data(), S.g_val64.p, sizeof(double) * S.g_val64.n, cudaMemcpyDeviceToHost));
            }
            S.pc_bytes = wb::serialize_preconditioner(img, S.subs);
        }
        const size_t need = S.pc_bytes.size();
        if (buf) {
            if (*len < need) {
                *len = need;
                return wb::fail(WITHIN_ERR_INVALID_ARGUMENT, "buffer too small for the serialized preconditioner");
            }
            std::memcpy(buf, S.pc_bytes.data(), need);
        }
        *len = need;
        return WITHIN_OK;
    });
}

int32_t within_solver_preconditioner_kind(const within_solver* s) { return s ? (int32_t)s->impl->pc.kind : 0; }

int within_solver_new(const uint32_t* codes, size_t n_obs, size_t n_factors, int64_t row_stride, int64_t col_stride,
                      const double* weights, const within_params* params, const within_preconditioner* precond,
                      within_solver** out) {
    if (!out) return wb::fail(WITHIN_ERR_INVALID_ARGUMENT, "out pointer is null");
    *out = nullptr;
    return guard([&]() -> int {
        std::unique_ptr<SolverImpl> S;
        const int rc = build_solver(codes, n_obs, n_factors, row_stride, col_stride, weights, params,
                                    (precond && precond->kind != WITHIN_PRECOND_OFF) ? precond : nullptr, S);
        if (rc != WITHIN_OK) return rc;
        *out = new within_solver{std::move(S)};
        return WITHIN_OK;
    });
}

void within_solver_free(within_solver* s) { delete s; }

size_t within_solver_n_dofs(const within_solver* s) { return s ? (size_t)s->impl->d.ndofs : 0; }
size_t within_solver_n_obs(const within_solver* s) { return s ? (size_t)s->impl->d.n : 0; }
size_t within_solver_n_factors(const within_solver* s) { return s ? (size_t)s->impl->d.Q : 0; }

int within_solver_solve_batch_device(within_solver* s, const double* d_ys, size_t k, double* d_x, double* d_dem,
                                     within_solve_stats* stats, void* stream) {
    if (!s) return wb::fail(WITHIN_ERR_INVALID_ARGUMENT, "solver is null");
    SolverImpl& S = *s->impl;
    std::lock_guard<std::mutex> lk(S.mu);
    return guard([&]() -> int {
        if (stream) {
            cudaEvent_t ev;
            WB_CUDA(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
            WB_CUDA(cudaEventRecord(ev, (cudaStream_t)stream));
            WB_CUDA(cudaStreamWaitEvent(S.stream, ev, 0));
            WB_CUDA(cudaEventDestroy(ev));
        }
        const int rc = solve_device(S, d_ys, k, d_x, d_dem, stats);
        if (stream) {
            cudaEvent_t ev;
            WB_CUDA(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
            WB_CUDA(cudaEventRecord(ev, S.stream));
            WB_CUDA(cudaStreamWaitEvent((cudaStream_t)stream, ev, 0));
            WB_CUDA(cudaEventDestroy(ev));
        }
        return rc;
    });
}

int within_solver_solve_batch(within_solver* s, const double* ys, size_t k, double* x, double* dem,
                              within_solve_stats* stats) {
    if (!s) return wb::fail(WITHIN_ERR_INVALID_ARGUMENT, "solver is null");
    SolverImpl& S = *s->impl;
    return guard([&]() -> int {
        const double t0 = wb::now_s();
        if (k == 0) return WITHIN_OK;
        if (!ys || !x || !dem) return wb::fail(WITHIN_ERR_INVALID_ARGUMENT, "null buffer");
        if (S.precond_only)
            return wb::fail(WITHIN_ERR_INVALID_ARGUMENT, "this handle holds only a preconditioner; build a Solver to solve");
        const size_t n = (size_t)S.d.n, m = (size_t)S.d.ndofs;
        // this call's device buffers and copy stream (a slot kept by the solver); the
        // upload and the download run outside the solver's lock, so that calls from other
        // host threads overlap their copies with this solve and this one's with theirs
        wb::HostCall* hc = nullptr;
        {
            std::lock_guard<std::mutex> lc(S.calls_mu);
            for (auto& c : S.calls)
                if (!c->busy) { hc = c.get(); break; }
            if (!hc) {
                S.calls.push_back(std::make_unique<wb::HostCall>());
                hc = S.calls.back().get();
            }
            hc->busy = true;
        }
        struct Release {
            wb::SolverImpl& S;
            wb::HostCall* hc;
            ~Release() {
                std::lock_guard<std::mutex> lc(S.calls_mu);
                hc->busy = false;
            }
        } release{S, hc};
        if (!hc->stream) WB_CUDA(cudaStreamCreateWithFlags(&hc->stream, cudaStreamNonBlocking));
        hc->y.alloc(n * k);
        hc->x.alloc(m * k);
        hc->dem.alloc(n * k);
        cudaEvent_t up = nullptr, done = nullptr;
        WB_CUDA(cudaEventCreateWithFlags(&up, cudaEventDisableTiming));
        struct Events {
            cudaEvent_t &a, &b;
            ~Events() {
                if (a) cudaEventDestroy(a);
                if (b) cudaEventDestroy(b);
            }
        } evs{up, done};
        WB_CUDA(cudaEventCreateWithFlags(&done, cudaEventDisableTiming));
        WB_CUDA(cudaMemcpyAsync(hc->y.p, ys, sizeof(double) * n * k, cudaMemcpyHostToDevice, hc->stream));
        WB_CUDA(cudaEventRecord(up, hc->stream));
        {
            std::lock_guard<std::mutex> lk(S.mu);
            WB_CUDA(cudaStreamWaitEvent(S.stream, up, 0));
            const int rc = solve_device(S, hc->y.p, k, hc->x.p, hc->dem.p, stats);
            if (rc != WITHIN_OK) {
                WB_CUDA(cudaStreamSynchronize(S.stream));
                return rc;
            }
            WB_CUDA(cudaEventRecord(done, S.stream));
        }
        WB_CUDA(cudaStreamWaitEvent(hc->stream, done, 0));
        WB_CUDA(cudaMemcpyAsync(x, hc->x.p, sizeof(double) * m * k, cudaMemcpyDeviceToHost, hc->stream));
        WB_CUDA(cudaMemcpyAsync(dem, hc->dem.p, sizeof(double) * n * k, cudaMemcpyDeviceToHost, hc->stream));
        WB_CUDA(cudaStreamSynchronize(hc->stream));
        if (stats) stats[0].time_total = wb::now_s() - t0;
        return WITHIN_OK;
    });
}

int within_solver_solve(within_solver* s, const double* y, double* x, double* dem, within_solve_stats* stats) {
    return within_solver_solve_batch(s, y, 1, x, dem, stats);
}

int within_solve(const uint32_t* codes, size_t n_obs, size_t n_factors, int64_t row_stride, int64_t col_stride,
                 const double* y, const double* weights, const within_params* params,
                 const within_preconditioner* precond, double* x, double* dem, within_solve_stats* stats) {
    return within_solve_batch(codes, n_obs, n_factors, row_stride, col_stride, y, 1, weights, params, precond, x, dem,
                              stats);
}

int within_solve_batch(const uint32_t* codes, size_t n_obs, size_t n_factors, int64_t row_stride, int64_t col_stride,
                       const double* ys, size_t k, const double* weights, const within_params* params,
                       const within_preconditioner* precond, double* x, double* dem, within_solve_stats* stats) {
    const double t0 = wb::now_s();
    within_solver* s = nullptr;
    int rc = within_solver_new(codes, n_obs, n_factors, row_stride, col_stride, weights, params, precond, &s);
    if (rc != WITHIN_OK) return rc;
    const double t_setup = wb::now_s() - t0;
    rc = within_solver_solve_batch(s, ys, k, x, dem, stats);
    within_solver_free(s);
    if (rc == WITHIN_OK && stats)
        for (size_t c = 0; c < k; ++c) {
            stats[c].time_setup += t_setup;
            stats[c].time_total = wb::now_s() - t0;
        }
    return rc;
}

// --- operator applies on host vectors (parity tests) ---

static int apply_common(within_solver* s, const double* in, size_t k, double* out, int which) {
    if (!s) return wb::fail(WITHIN_ERR_INVALID_ARGUMENT, "solver is null");
    SolverImpl& S = *s->impl;
    std::lock_guard<std::mutex> lk(S.mu);
    return guard([&]() -> int {
        if (k == 0) return WITHIN_OK;
        if (k > 32) return wb::fail(WITHIN_ERR_INVALID_ARGUMENT, "at most 32 vectors per call");
        if (S.precond_only && which != 1)
            return wb::fail(WITHIN_ERR_INVALID_ARGUMENT, "this handle holds only a preconditioner");
        const int kk = (int)k, kp = wb::pad_kp(kk);
        wb::ensure_ws(S, kp);
        const size_t n = (size_t)S.d.n, m = (size_t)S.d.ndofs;
        const size_t in_rows = (which == 3) ? n : m;
        const size_t out_rows = (which == 2) ? n : m;
        wb::DArr<double> din, dout, iin, iout;
        din.alloc(in_rows * k);
        dout.alloc(out_rows * k);
        iin.alloc(in_rows * kp);
        iout.alloc(out_rows * kp);
        WB_CUDA(cudaMemcpyAsync(din.p, in, sizeof(double) * in_rows * k, cudaMemcpyHostToDevice, S.stream));
        const uint32_t* perm = S.perm_identity ? nullptr : S.perm.p;
        wb::gather_interleave_kernel<double><<<wb::xpose_blocks((int64_t)in_rows, S.n_sm), wb::kXposeWarps * 32, wb::xpose_smem(kp), S.stream>>>(
            din.p, (int64_t)in_rows, kk, kp, which == 3 ? perm : nullptr, iin.p);
        if (which == 0 || which == 1) {
            if (!S.mixed()) {
                if (which == 0) {
                    wb::launch_gram<double>(S, kp, S.w64.p, iin.p, iout.p);
                } else {
                    int nb = 0;
                    wb::apply_precond<double>(S, iin.p, iout.p, kp, nullptr, nb);
                }
            } else {
                wb::DArr<float> fi, fo;
                fi.alloc(m * kp);
                fo.alloc(m * kp);
                wb::convert_kernel<double, float><<<S.nblk(m * kp, 1), wb::kBlock, 0, S.stream>>>(iin.p, fi.p, m * kp);
                if (which == 0) {
                    wb::launch_gram<float>(S, kp, S.w32.p, fi.p, fo.p);
                } else {
                    int nb = 0;
                    wb::apply_precond<float>(S, fi.p, fo.p, kp, nullptr, nb);
                }
                wb::convert_kernel<float, double><<<S.nblk(m * kp, 1), wb::kBlock, 0, S.stream>>>(fo.p, iout.p, m * kp);
                WB_CUDA(cudaStreamSynchronize(S.stream));
            }
        } else if (which == 2) {  // D x
            wb::launch_obs<double, wb::OBS_DX>(S, kp, nullptr, iin.p, nullptr, nullptr, iout.p);
        } else {  // D'W r
            wb::launch_obs<double, wb::OBS_RHS>(S, kp, S.w64.p, nullptr, iin.p, iout.p, nullptr);
        }
        wb::scatter_deinterleave_kernel<double><<<wb::xpose_blocks((int64_t)out_rows, S.n_sm), wb::kXposeWarps * 32, wb::xpose_smem(kp), S.stream>>>(
            iout.p, (int64_t)out_rows, kk, kp, which == 2 ? perm : nullptr, dout.p);
        WB_CUDA(cudaGetLastError());
        WB_CUDA(cudaMemcpyAsync(out, dout.p, sizeof(double) * out_rows * k, cudaMemcpyDeviceToHost, S.stream));
        WB_CUDA(cudaStreamSynchronize(S.stream));
        // a local solve that did not complete left z all NaN, as the reference's apply
        // does (schwarz-precond additive/preconditioner.rs:197-201); the flag is cleared
        if (which == 1) wb::sweeps_failed(S);
        return WITHIN_OK;
    });
}

int within_solver_apply_gramian(within_solver* s, const double* x, size_t k, double* y) { return apply_common(s, x, k, y, 0); }
int within_solver_apply_preconditioner(within_solver* s, const double* r, size_t k, double* z) { return apply_common(s, r, k, z, 1); }
int within_solver_matvec_d(within_solver* s, const double* x, size_t k, double* y) { return apply_common(s, x, k, y, 2); }
int within_solver_rmatvec_wdt(within_solver* s, const double* r, size_t k, double* x) { return apply_common(s, r, k, x, 3); }

void within_solver_factor_meta(const within_solver* s, int64_t* n_levels, int64_t* offsets) {
    const wb::Design& d = s->impl->d;
    for (int q = 0; q < d.Q; ++q) { n_levels[q] = d.nlev[q]; offsets[q] = d.off[q]; }
}
int32_t within_solver_n_subdomains(const within_solver* s) { return (int32_t)s->impl->subs.size(); }
void within_solver_subdomain_info(const within_solver* s, int32_t i, int64_t* info) {
    const wb::Subdomain& sd = s->impl->subs[i];
    info[0] = sd.q; info[1] = sd.r; info[2] = sd.n_local(); info[3] = sd.n_q(); info[4] = sd.n_r();
    info[5] = sd.elim_q; info[6] = sd.kind; info[7] = sd.n_red;
}
void within_solver_subdomain_inner_work(const within_solver* s, int64_t* work) {
    const auto& subs = s->impl->subs;
    for (size_t i = 0; i < subs.size(); ++i) work[i] = wb::inner_parallel_work(subs[i]);
}
int within_solver_additive_diagnostics(const within_solver* s, int32_t threads, within_additive_diagnostics* out) {
    if (!s || !out) return wb::fail(WITHIN_ERR_INVALID_ARGUMENT, "solver and out must not be null");
    const SolverImpl& S = *s->impl;
    if (S.pc.kind != 1) return wb::fail(WITHIN_ERR_INVALID_ARGUMENT, "the solver has no additive Schwarz preconditioner");
    const int64_t t = threads > 0 ? threads : (int64_t)std::max(1u, std::thread::hardware_concurrency());
    const wb::AdditiveDiagnostics g = wb::additive_diagnostics(S.subs, S.d.ndofs, S.reduction_strategy, t);
    out->reduction_strategy = g.configured;
    out->resolved_reduction_strategy = g.resolved;
    out->n_subdomains = g.n_subdomains;
    out->n_dofs = g.n_dofs;
    out->total_inner_parallel_work = g.total_inner_work;
    out->max_inner_parallel_work = g.max_inner_work;
    out->total_scatter_dofs = g.total_scatter_dofs;
    out->outer_parallel_capacity = g.outer_parallel_capacity;
    out->scatter_overlap = g.scatter_overlap;
    wb::g_last_error.clear();
    return WITHIN_OK;
}
void within_solver_subdomain_indices(const within_solver* s, int32_t i, uint32_t* gidx, double* pou) {
    const wb::Subdomain& sd = s->impl->subs[i];
    std::memcpy(gidx, sd.gidx.data(), sizeof(uint32_t) * sd.gidx.size());
    for (size_t a = 0; a < sd.gidx.size(); ++a) pou[a] = sd.pou.empty() ? 1.0 : sd.pou[a];
}
void within_solver_ac_sizes(const within_solver* s, int32_t i, int64_t* sizes) {
    const wb::Subdomain& sd = s->impl->subs[i];
    for (int a = 0; a < 5; ++a) sizes[a] = 0;
    if (sd.kind != 1) return;
    sizes[0] = sd.ac.n; sizes[1] = sd.ac.nlev; sizes[2] = (int64_t)sd.ac.col_idx.size();
    sizes[3] = sd.ac.ncol; sizes[4] = sd.ac.ncore;
}
void within_solver_ac_arrays(const within_solver* s, int32_t i, int32_t* level_ptr, int32_t* col_vertex,
                             double* col_diag, int32_t* col_ptr, int32_t* col_idx, double* col_coef,
                             int32_t* core_vertex, double* core_z) {
    const wb::AcFactor& f = s->impl->subs[i].ac;
    std::copy(f.level_ptr.begin(), f.level_ptr.end(), level_ptr);
    std::copy(f.col_vertex.begin(), f.col_vertex.end(), col_vertex);
    std::copy(f.col_diag.begin(), f.col_diag.end(), col_diag);
    std::copy(f.col_ptr.begin(), f.col_ptr.end(), col_ptr);
    std::copy(f.col_idx.begin(), f.col_idx.end(), col_idx);
    std::copy(f.col_coef.begin(), f.col_coef.end(), col_coef);
    std::copy(f.core_vertex.begin(), f.core_vertex.end(), core_vertex);
    std::copy(f.core_z.begin(), f.core_z.end(), core_z);
}

int within_solver_inject_sweep_timeout(within_solver* s, int32_t on) {
    if (!s) return wb::fail(WITHIN_ERR_INVALID_ARGUMENT, "solver is null");
    SolverImpl& S = *s->impl;
    std::lock_guard<std::mutex> lk(S.mu);
    return guard([&]() -> int {
        bool sweeps = false;
        for (const auto& st : S.stages64) sweeps = sweeps || st.fwd_lp.size() > 2 || st.bwd_lp.size() > 2;
        if (!S.coop || !sweeps)
            return wb::fail(WITHIN_ERR_INVALID_ARGUMENT, "the preconditioner has no fused approximate-Cholesky sweeps");
        S.inject_sweep_timeout = on != 0;
        if (S.cg_exec) {  // the captured CG iteration holds the sweep parameters
            WB_CUDA(cudaGraphExecDestroy(S.cg_exec));
            S.cg_exec = nullptr;
        }
        return WITHIN_OK;
    });
}

int within_solver_set_sweep_cluster(within_solver* s, int64_t max_chunks) {
    if (!s || max_chunks < 0) return wb::fail(WITHIN_ERR_INVALID_ARGUMENT, "invalid argument");
    SolverImpl& S = *s->impl;
    std::lock_guard<std::mutex> lk(S.mu);
    return guard([&]() -> int {
        S.sweep_cluster_chunks = max_chunks;
        if (S.cg_exec) {  // the captured CG iteration holds the sweep launches
            WB_CUDA(cudaGraphExecDestroy(S.cg_exec));
            S.cg_exec = nullptr;
        }
        return WITHIN_OK;
    });
}

// --- learned coarse space ---

int32_t within_coarse_net_params(void) { return (int32_t)wb::kCnParams; }

static int coarse_common(within_solver* s, const std::function<int(SolverImpl&)>& f) {
    if (!s) return wb::fail(WITHIN_ERR_INVALID_ARGUMENT, "solver is null");
    SolverImpl& S = *s->impl;
    std::lock_guard<std::mutex> lk(S.mu);
    return guard([&]() -> int {
        if (S.precond_only) return wb::fail(WITHIN_ERR_INVALID_ARGUMENT, "this handle holds only a preconditioner");
        return f(S);
    });
}

int within_solver_set_coarse_net(within_solver* s, const float* params, size_t n_params, uint64_t seed) {
    return coarse_common(s, [&](SolverImpl& S) -> int {
        if (!params || n_params != (size_t)wb::kCnParams)
            return wb::fail(WITHIN_ERR_INVALID_ARGUMENT, "the coarse-space network has " +
                                                             std::to_string(wb::kCnParams) + " parameters");
        wb::CnState C;
        wb::cn_prepare(S, C, params, seed);
        wb::cn_forward(S, C);
        const int64_t m = S.d.ndofs;
        S.coarse_z64.alloc((size_t)m * 32);
        wb::cn_unscale_kernel<<<wb::cn_blocks(m * 32), 256, 0, S.stream>>>(m, C.Zt.p, C.isq.p, S.coarse_z64.p, nullptr);
        WB_CUDA(cudaGetLastError());
        S.gpu_launches++;
        wb::install_coarse(S);
        return WITHIN_OK;
    });
}

int within_solver_set_coarse_basis(within_solver* s, const double* Z, size_t k) {
    return coarse_common(s, [&](SolverImpl& S) -> int {
        if (!Z || k == 0 || k > 32) return wb::fail(WITHIN_ERR_INVALID_ARGUMENT, "a coarse basis has 1 to 32 columns");
        const size_t m = (size_t)S.d.ndofs;
        std::vector<double> zr(m * 32, 0.0);  // row-major, 32 columns
        for (size_t j = 0; j < k; ++j)
            for (size_t i = 0; i < m; ++i) zr[i * 32 + j] = Z[j * m + i];
        S.coarse_z64.upload(zr);
        wb::install_coarse(S);
        return WITHIN_OK;
    });
}

int within_solver_clear_coarse(within_solver* s) {
    return coarse_common(s, [&](SolverImpl& S) -> int {
        S.coarse_k = 0;
        if (S.cg_exec) {
            WB_CUDA(cudaGraphExecDestroy(S.cg_exec));
            S.cg_exec = nullptr;
        }
        return WITHIN_OK;
    });
}

int within_solver_coarse_basis(within_solver* s, double* Z) {
    return coarse_common(s, [&](SolverImpl& S) -> int {
        if (S.coarse_k == 0) return wb::fail(WITHIN_ERR_INVALID_ARGUMENT, "the solver has no coarse space");
        const size_t m = (size_t)S.d.ndofs;
        std::vector<double> zr(m * 32);
        WB_CUDA(cudaMemcpy(zr.data(), S.coarse_z64.p, sizeof(double) * m * 32, cudaMemcpyDeviceToHost));
        for (size_t j = 0; j < 32; ++j)
            for (size_t i = 0; i < m; ++i) Z[j * m + i] = zr[i * 32 + j];
        return WITHIN_OK;
    });
}

int within_solver_set_coarse_targets(within_solver* s, const double* V, size_t t) {
    return coarse_common(s, [&](SolverImpl& S) -> int {
        if (!V || t == 0 || t > 32) return wb::fail(WITHIN_ERR_INVALID_ARGUMENT, "targets have 1 to 32 columns");
        const size_t m = (size_t)S.d.ndofs;
        std::vector<float> vr(m * t);
        for (size_t j = 0; j < t; ++j)
            for (size_t i = 0; i < m; ++i) vr[i * t + j] = (float)V[j * m + i];
        S.cn_targets.upload(vr);
        S.cn_t = (int32_t)t;
        return WITHIN_OK;
    });
}

int within_coarse_net_grad(within_solver* s, const float* params, uint64_t seed, float* grad, double* loss,
                           float* zt) {
    return coarse_common(s, [&](SolverImpl& S) -> int {
        if (!params || !grad || !loss) return wb::fail(WITHIN_ERR_INVALID_ARGUMENT, "null buffer");
        if (S.cn_t == 0) return wb::fail(WITHIN_ERR_INVALID_ARGUMENT, "no training targets on this solver");
        if (!S.cn) S.cn = std::make_shared<wb::CnState>();
        wb::CnState& C = *std::static_pointer_cast<wb::CnState>(S.cn);
        wb::cn_prepare(S, C, params, seed);
        wb::cn_forward(S, C);
        *loss = wb::cn_backward(S, C, grad);
        if (zt) {
            const size_t m = (size_t)S.d.ndofs;
            std::vector<float> zr(m * 32);
            WB_CUDA(cudaMemcpy(zr.data(), C.Zt.p, sizeof(float) * m * 32, cudaMemcpyDeviceToHost));
            for (size_t j = 0; j < 32; ++j)
                for (size_t i = 0; i < m; ++i) zt[j * m + i] = zr[i * 32 + j];
        }
        return WITHIN_OK;
    });
}

int within_solver_release_coarse_training(within_solver* s) {
    return coarse_common(s, [&](SolverImpl& S) -> int {
        S.cn.reset();
        S.cn_targets.release();
        S.cn_t = 0;
        return WITHIN_OK;
    });
}

int within_solver_obs_config(const within_solver* s, int32_t k, int32_t elem_bytes, int32_t* obs_per_chunk,
                             int32_t* blocks_per_sm) {
    if (!s || k <= 0 || k > 32 || (elem_bytes != 4 && elem_bytes != 8) || !obs_per_chunk || !blocks_per_sm)
        return wb::fail(WITHIN_ERR_INVALID_ARGUMENT, "invalid argument");
    const int32_t c = s->impl->obs_choice[wb::kp_class(wb::pad_kp(k))][elem_bytes == 8 ? 1 : 0];
    *obs_per_chunk = c < 0 ? 32 : 16 << ((c % wb::kObsShapes) / 2);
    *blocks_per_sm = c < 0 ? 2 : 1 + c % 2;
    return c < 0 ? 1 : 0;
}

int32_t within_solver_obs_hot_global(const within_solver* s, int32_t k, int32_t elem_bytes) {
    if (!s || k <= 0 || k > 32 || (elem_bytes != 4 && elem_bytes != 8)) return -1;
    const int kp = wb::pad_kp(k);
    const int32_t c = s->impl->obs_choice[wb::kp_class(kp)][elem_bytes == 8 ? 1 : 0];
    if (c < 0) return -1;
    if (c % (2 * wb::kObsShapes) < wb::kObsShapes) return 0;
    wb::ObsParams P;
    wb::obs_params_for(*s->impl, kp, (size_t)elem_bytes, P, true);
    return P.hot_glob ? 1 : 0;
}

int32_t within_solver_obs_rhs_per_lane(const within_solver* s, int32_t k, int32_t elem_bytes) {
    if (!s || k <= 0 || k > 32 || (elem_bytes != 4 && elem_bytes != 8)) return -1;
    const int kp = wb::pad_kp(k);
    const int32_t c = s->impl->obs_choice[wb::kp_class(kp)][elem_bytes == 8 ? 1 : 0];
    if (c < 0) return -1;
    return (c >= 2 * wb::kObsShapes && wb::obs_wide_for(*s->impl, kp, (size_t)elem_bytes)) ? 8 : 4;
}

int within_solver_set_hybrid(within_solver* s, int32_t k, int32_t elem_bytes, int32_t on) {
    if (!s || k <= 0 || k > 32 || (elem_bytes != 4 && elem_bytes != 8) || on < 0 || on > 2)
        return wb::fail(WITHIN_ERR_INVALID_ARGUMENT, "invalid argument");
    wb::SolverImpl& S = *s->impl;
    std::lock_guard<std::mutex> lk(S.mu);
    return guard([&]() -> int {
        const int kp = wb::pad_kp(k);
        if (elem_bytes == 4 && !S.mixed())
            return wb::fail(WITHIN_ERR_INVALID_ARGUMENT, "the solver has no FP32 operator");
        int np = 0;
        const uint32_t smask = (on && wb::hybrid_possible(S)) ? wb::hybrid_smask(S, kp, (size_t)elem_bytes, np) : 0u;
        if (on && smask == 0)
            return wb::fail(WITHIN_ERR_INVALID_ARGUMENT,
                            "no hybrid operator apply for this solver (it needs an additive Schwarz preconditioner, "
                            "the implicit operator, and one or two factors in lane-group tables)");
        int32_t& cur = S.hyb_on[wb::kp_class(kp)][elem_bytes == 8 ? 1 : 0];
        if (on) {
            if (S.hyb && S.hyb->smask != smask) {
                cur = 0;
                if (wb::hybrid_in_use(S))
                    return wb::fail(WITHIN_ERR_INVALID_ARGUMENT, "the hybrid apply is in use with other small factors");
            }
            if (!S.hyb || S.hyb->smask != smask) wb::build_hybrid(S, smask);
            wb::PrimMmaParams M;
            if (on == 2 && !wb::mma_layout(S, kp, (size_t)elem_bytes, M)) {
                cur = 0;
                return wb::fail(WITHIN_ERR_INVALID_ARGUMENT,
                                "no tensor-core form of the hybrid apply here (it needs 16 RHS columns and at most "
                                "48 small-factor levels, each factor padded to 8)");
            }
        }
        cur = on;
        if (S.cg_exec) {  // the captured CG iteration holds the old operator
            WB_CUDA(cudaGraphExecDestroy(S.cg_exec));
            S.cg_exec = nullptr;
        }
        return 0;
    });
}

int32_t within_solver_hybrid(const within_solver* s, int32_t k, int32_t elem_bytes, float* ms) {
    if (!s || k <= 0 || k > 32 || (elem_bytes != 4 && elem_bytes != 8)) return -1;
    const int c = wb::kp_class(wb::pad_kp(k)), e = elem_bytes == 8 ? 1 : 0;
    if (ms) *ms = s->impl->hyb_ms[c][e];
    return s->impl->hyb_on[c][e];
}

int64_t within_solver_hybrid_bytes(const within_solver* s, int32_t k, int32_t elem_bytes) {
    if (!s || k <= 0 || k > 32 || (elem_bytes != 4 && elem_bytes != 8) || !s->impl->hyb) return 0;
    const wb::SolverImpl& S = *s->impl;
    const wb::HybridDev& H = *S.hyb;
    const int64_t e = elem_bytes, kp = wb::pad_kp(k), nP = S.d.nlev[S.primary];
    const int64_t ns = __builtin_popcount(H.smask), wt = S.d.w.empty() ? 0 : 1;
    const bool mma = S.hyb_on[wb::kp_class((int)kp)][elem_bytes == 8 ? 1 : 0] == 2;
    // per primary level: its C_PO row pointer (8) and its observation offset (4), or its
    // pieces (16 each) for the tensor-core form
    const int64_t lvl = mma ? (nP + 1) * 8 + H.npieces * 16 : (nP + 1) * (8 + 4);
    return S.d.n * (4 * ns + e * wt) + (int64_t)(H.pcol.n + H.ocol.n) * (4 + e) + lvl +
           (int64_t)H.rows.n * (4 + 8) + 2 * e * S.d.ndofs * kp;
}

int within_solver_obs_tune_times(const within_solver* s, int32_t k, int32_t elem_bytes, float* ms, int32_t n) {
    if (!s || k <= 0 || k > 32 || (elem_bytes != 4 && elem_bytes != 8) || !ms || n < 0)
        return wb::fail(WITHIN_ERR_INVALID_ARGUMENT, "invalid argument");
    const float* t = s->impl->obs_tune_ms[wb::kp_class(wb::pad_kp(k))][elem_bytes == 8 ? 1 : 0];
    for (int32_t c = 0; c < n && c < 4 * wb::kObsShapes; ++c) ms[c] = t[c];
    return 0;
}

int within_solver_set_obs_config(within_solver* s, int32_t k, int32_t elem_bytes, int32_t obs_per_chunk,
                                 int32_t blocks_per_sm, int32_t variant) {
    if (!s || k <= 0 || k > 32 || (elem_bytes != 4 && elem_bytes != 8) ||
        (obs_per_chunk != 16 && obs_per_chunk != 32 && obs_per_chunk != 64) || blocks_per_sm < 1 ||
        blocks_per_sm > 2 || variant < 0 || variant > 3)
        return wb::fail(WITHIN_ERR_INVALID_ARGUMENT, "invalid argument");
    if ((variant & 2) && !wb::obs_wide_for(*s->impl, wb::pad_kp(k), (size_t)elem_bytes))
        return wb::fail(WITHIN_ERR_INVALID_ARGUMENT, "no wide lanes for this precision, RHS count and design");
    const int32_t hot_global = variant & 1;
    wb::SolverImpl& S = *s->impl;
    std::lock_guard<std::mutex> lk(S.mu);
    return guard([&]() -> int {
        const int kp = wb::pad_kp(k);
        if (hot_global) wb::grow_obs_hot(S, wb::obs_hot_bytes(S, kp, (size_t)elem_bytes));
        if (S.cg_exec) {  // the captured CG iteration holds the pass's old shape
            WB_CUDA(cudaGraphExecDestroy(S.cg_exec));
            S.cg_exec = nullptr;
        }
        const int32_t ci = obs_per_chunk == 16 ? 0 : obs_per_chunk == 32 ? 1 : 2;
        S.obs_choice[wb::kp_class(kp)][elem_bytes == 8 ? 1 : 0] =
            ((variant & 2) ? 2 * wb::kObsShapes : 0) + (hot_global ? wb::kObsShapes : 0) + 2 * ci + (blocks_per_sm - 1);
        return 0;
    });
}

int64_t within_solver_schwarz_bytes(const within_solver* s, int32_t k, int32_t elem_bytes) {
    if (!s || k <= 0 || (elem_bytes != 4 && elem_bytes != 8)) return 0;
    const int64_t e = elem_bytes;
    int64_t b = 0;
    for (const wb::Subdomain& sd : s->impl->subs) {
        const int64_t nl = sd.n_local();
        b += 2 * (4 + e) * sd.ct.c.nnz();  // the cross block: reduced rhs and back substitution
        b += (4 + 8) * nl;                 // global index and partition-of-unity weight per slot
        b += 2 * e * nl * k;               // the local vector, gathered and scattered
        if (sd.kind == 0) {
            const int64_t r = std::max<int64_t>(sd.n_red - 1, 0);
            b += e * r * r;                // the anchored dense factor
        } else {
            b += 2 * (4 + e) * (int64_t)sd.ac.col_idx.size();  // AC forward and backward sweeps
            b += e * (int64_t)sd.ac.ncore * sd.ac.ncore;        // the dense core's inverse
        }
    }
    return b;
}

const char* within_last_error(void) { return wb::g_last_error.c_str(); }

int within_solve_many(within_problem* problems, size_t n_problems, const within_params* params,
                      const within_preconditioner* precond, int32_t concurrency) {
    if (n_problems == 0) return WITHIN_OK;
    if (!problems) return wb::fail(WITHIN_ERR_INVALID_ARGUMENT, "problems is null");
    int dev = 0;
    cudaError_t ce = cudaGetDevice(&dev);
    if (ce != cudaSuccess) return wb::fail(WITHIN_ERR_CUDA, std::string("cudaGetDevice: ") + cudaGetErrorString(ce));
    const size_t hw = std::max(1u, std::thread::hardware_concurrency());
    const size_t nt = std::min<size_t>(n_problems, concurrency > 0 ? (size_t)concurrency : hw);
    std::atomic<size_t> next{0};
    std::vector<std::string> msg(n_problems);
    // each host thread drives one problem at a time: setup on the host, then the solve on
    // the solver's own stream (the device is the caller's)
    auto worker = [&]() {
        cudaSetDevice(dev);
        wb::busy_threads().fetch_add(1);  // nested setup phases see this core as taken
        for (;;) {
            const size_t i = next.fetch_add(1);
            if (i >= n_problems) break;
            within_problem& p = problems[i];
            within_solver* sv = nullptr;
            int rc = within_solver_new(p.codes, p.n_obs, p.n_factors, p.row_stride, p.col_stride, p.weights, params,
                                       precond, &sv);
            if (rc == WITHIN_OK) {
                rc = within_solver_solve_batch(sv, p.ys, p.k, p.x, p.demeaned, p.stats);
                if (rc != WITHIN_OK) msg[i] = within_last_error();
                within_solver_free(sv);
            } else {
                msg[i] = within_last_error();
            }
            p.status = rc;
        }
        wb::busy_threads().fetch_sub(1);
    };
    std::vector<std::thread> pool;
    for (size_t t = 1; t < nt; ++t) pool.emplace_back(worker);
    worker();
    for (auto& t : pool) t.join();
    for (size_t i = 0; i < n_problems; ++i)
        if (problems[i].status != WITHIN_OK)
            return wb::fail(problems[i].status, "problem " + std::to_string(i) + ": " + msg[i]);
    wb::g_last_error.clear();
    return WITHIN_OK;
}

int64_t within_solver_gpu_launches(const within_solver* s) { return s ? s->impl->gpu_launches : 0; }
double within_solver_setup_time(const within_solver* s) { return s ? s->impl->setup_time : 0.0; }

void within_solver_set_profiling(within_solver* s, int32_t on) {
    if (!s) return;
    std::lock_guard<std::mutex> lk(s->impl->mu);
    s->impl->profiling = on != 0;
    for (int a = 0; a < 4; ++a) { s->impl->prof_count[a] = 0; s->impl->prof_ms[a] = 0.0; }
}
void within_solver_kernel_time(const within_solver* s, int32_t which, int64_t* launches, double* total_ms) {
    *launches = 0;
    *total_ms = 0.0;
    if (!s || which < 0 || which > 3) return;
    *launches = s->impl->prof_count[which];
    *total_ms = s->impl->prof_ms[which];
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Gramian apply that allocates nothing
// ---------------------------------------------------------------------------
//
// Some callers cannot allocate device memory while they run: host code under a fixed
// device-memory budget or a custom allocator that forbids outside allocations, and
// loops where an allocation's synchronisation is not acceptable.  within_solver_apply_gramian_noalloc serves them:
// its working space -- the RHS-interleaved copies of x and of y = G x -- lives in the
// static device array below instead of cudaMalloc'd buffers.  The array is 16 MiB and
// stays resident on every GPU that loads this library until the process exits.

namespace {
constexpr size_t kNoAllocScratchDoubles = (size_t)1 << 21;  // 16 MiB of FP64
__device__ __align__(256) double g_noalloc_scratch[kNoAllocScratchDoubles];
constexpr int kNoAllocMaxDevices = 64;
std::mutex g_noalloc_mu;
double* g_noalloc_addr[kNoAllocMaxDevices] = {};

// Device address of the scratch array on the current device, looked up once per
// device (host code may not use the symbol itself as a device pointer).
int noalloc_scratch(double** out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return wb::fail(WITHIN_ERR_CUDA, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
    if (dev < 0 || dev >= kNoAllocMaxDevices) return wb::fail(WITHIN_ERR_CUDA, "device index out of range");
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    if (!g_noalloc_addr[dev]) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p)
            return wb::fail(WITHIN_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
        g_noalloc_addr[dev] = static_cast<double*>(p);
    }
    *out = g_noalloc_addr[dev];
    return WITHIN_OK;
}

// The error mapping of guard() for a callable passed by template parameter (no
// std::function, so no host allocation on the success path).  No exception crosses the
// C ABI: anything other than a CUDA error or host memory exhaustion maps to
// WITHIN_ERR_CUDA, as only the device calls above can raise on this path.
template <typename F>
int noalloc_guard(F&& f) {
    try {
        const int rc = f();
        if (rc == WITHIN_OK) wb::g_last_error.clear();
        return rc;
    } catch (const wb::CudaError& e) {
        return wb::fail(WITHIN_ERR_CUDA, e.what());
    } catch (const std::bad_alloc&) {
        return wb::fail(WITHIN_ERR_OVERFLOW, "out of host memory");
    } catch (...) {
        return wb::fail(WITHIN_ERR_CUDA, "unexpected error in the no-allocation apply");
    }
}
}  // namespace

extern "C" int within_solver_apply_gramian_noalloc(within_solver* s, const double* d_x, size_t k, double* d_y,
                                                   void* stream) {
    if (!s) return wb::fail(WITHIN_ERR_INVALID_ARGUMENT, "solver is null");
    if (!d_x || !d_y) return wb::fail(WITHIN_ERR_INVALID_ARGUMENT, "null buffer");
    if (k == 0) return WITHIN_OK;
    if (k > 32) return wb::fail(WITHIN_ERR_INVALID_ARGUMENT, "at most 32 vectors per call");
    SolverImpl& S = *s->impl;
    // a handle rebuilt from preconditioner bytes has no design to apply
    if (S.precond_only)
        return wb::fail(WITHIN_ERR_INVALID_ARGUMENT, "this handle holds only a preconditioner");
    const int kk = (int)k, kp = wb::pad_kp(kk);
    const size_t m = (size_t)S.d.ndofs;
    const size_t need = 2 * m * (size_t)kp;
    if (need > kNoAllocScratchDoubles)
        return wb::fail(WITHIN_ERR_INVALID_ARGUMENT,
                        "n_dofs x k is too large for the no-allocation path: it needs " + std::to_string(need) +
                            " doubles of scratch (2 x n_dofs x k rounded up to 4, 8, 16 or 32), the limit is " +
                            std::to_string(kNoAllocScratchDoubles));
    std::lock_guard<std::mutex> lk(S.mu);
    // the solver's own stream comes back however this call leaves
    struct StreamRestore {
        SolverImpl& S;
        cudaStream_t saved;
        ~StreamRestore() { S.stream = saved; }
    } restore{S, S.stream};
    // guard() takes a std::function; this lambda is called directly so that nothing here
    // allocates on the host either
    return noalloc_guard([&]() -> int {
        double* scratch = nullptr;
        const int rc = noalloc_scratch(&scratch);
        if (rc != WITHIN_OK) return rc;
        double* xi = scratch;           // x, RHS-interleaved (m x kp)
        double* yi = scratch + m * kp;  // G x, RHS-interleaved (m x kp)
        if (stream) S.stream = (cudaStream_t)stream;
        wb::gather_interleave_kernel<double><<<wb::xpose_blocks((int64_t)m, S.n_sm), wb::kXposeWarps * 32, wb::xpose_smem(kp), S.stream>>>(
            d_x, (int64_t)m, kk, kp, nullptr, xi);
        wb::launch_obs<double, wb::OBS_GRAM>(S, kp, S.w64.p, xi, nullptr, yi, nullptr);
        wb::scatter_deinterleave_kernel<double><<<wb::xpose_blocks((int64_t)m, S.n_sm), wb::kXposeWarps * 32, wb::xpose_smem(kp), S.stream>>>(
            yi, (int64_t)m, kk, kp, nullptr, d_y);
        WB_CUDA(cudaGetLastError());
        S.gpu_launches += 2;
        return WITHIN_OK;
    });
}
