// Host-side setup of the solve phase: design metadata, factor-pair subdomains,
// Schur complements and approximate-Cholesky factors.  Integer outputs
// (level counts, offsets, subdomain membership and order) follow the
// reference exactly; the device layout is built from these in solver.cu.
#pragma once

#include <algorithm>
#include <atomic>
#include <cstdint>
#include <functional>
#include <thread>
#include <string>
#include <vector>

namespace wb {

// Host threads busy with setup work across the process: the workers of concurrent
// solves (which hold one each while they work) and the helpers of parallel_tasks.
// Nested parallel phases only take helpers while this stays below the core count, so
// that many concurrent solves do not oversubscribe the host.
inline std::atomic<int>& busy_threads() {
    static std::atomic<int> n{0};
    return n;
}

// One helper thread from the budget, if a core is idle (release it with release_helper).
inline bool try_take_helper() {
    const int hw = (int)std::max(1u, std::thread::hardware_concurrency());
    std::atomic<int>& busy = busy_threads();
    for (int cur = busy.load(); cur + 1 < hw;)
        if (busy.compare_exchange_weak(cur, cur + 1)) return true;
    return false;
}
inline void release_helper() { busy_threads().fetch_sub(1); }

// Runs fn(w, nw) on nw workers (the calling thread and up to max_workers - 1 helpers,
// as many as there are idle cores), w = 0..nw-1; with no idle core nw is 1.
inline void parallel_workers(int max_workers, const std::function<void(int, int)>& fn) {
    int got = 0;
    while (got + 1 < max_workers && try_take_helper()) ++got;
    const int nw = got + 1;
    std::vector<std::thread> th;
    for (int w = 1; w < nw; ++w) th.emplace_back([&, w] { fn(w, nw); });
    fn(0, nw);
    for (auto& x : th) x.join();
    for (int w = 0; w < got; ++w) release_helper();
}

// Runs fn(t) for t in [0, ntasks) on the calling thread and as many helper threads as
// there are idle cores (at most one per task).
inline void parallel_tasks(size_t ntasks, const std::function<void(size_t)>& fn) {
    const int hw = (int)std::max(1u, std::thread::hardware_concurrency());
    const int want = (int)std::min<size_t>(ntasks, (size_t)hw) - 1;
    int got = 0;
    std::atomic<int>& busy = busy_threads();
    while (got < want) {
        int cur = busy.load();
        if (cur + 1 >= hw) break;  // the calling thread keeps one core
        if (busy.compare_exchange_weak(cur, cur + 1)) ++got;
    }
    if (got == 0) {
        for (size_t t = 0; t < ntasks; ++t) fn(t);
        return;
    }
    std::atomic<size_t> next{0};
    auto worker = [&]() {
        for (size_t t; (t = next.fetch_add(1)) < ntasks;) fn(t);
    };
    std::vector<std::thread> th;
    for (int i = 0; i < got; ++i) th.emplace_back(worker);
    worker();
    for (auto& x : th) x.join();
    busy.fetch_sub(got);
}

struct Status {
    int code = 0;  // WITHIN_OK or a WITHIN_ERR_* value
    std::string msg;
    bool ok() const { return code == 0; }
};

// WeightedDesign (within/src/domain.rs:97-155).
struct Design {
    int64_t n = 0;
    int Q = 0;
    std::vector<uint32_t> codes;  // factor-major: codes[q*n + i]
    std::vector<double> w;        // empty = unit weights
    std::vector<int64_t> nlev, off;
    int64_t ndofs = 0;
    uint32_t level(int64_t i, int q) const { return codes[(size_t)q * n + i]; }
    double weight(int64_t i) const { return w.empty() ? 1.0 : w[i]; }
};

struct Csr {
    int32_t nrows = 0, ncols = 0;
    std::vector<uint32_t> ptr, idx;
    std::vector<double> val;
    int64_t nnz() const { return ptr.empty() ? 0 : (int64_t)ptr[nrows]; }
};

// Bipartite block [D_q C; C^T D_r] of one factor pair (gramian/cross_tab.rs:189-199).
struct CrossTab {
    Csr c, ct;
    std::vector<double> dq, dr;
};

// Rounds of the approximate Cholesky factor stop once at most this many vertices remain
// (they form the dense core), or once a round would eliminate fewer than
// max(kAcStallMin, remaining / kAcStallDiv) vertices: the remaining graph has turned
// dense, and if it is larger than a core, its vertices become one last level of pivots
// (the diagonal of the remaining Laplacian).
constexpr int32_t kAcCoreMax = 1024;
constexpr int64_t kAcStallMin = 32, kAcStallDiv = 128;

// Approximate Cholesky factor L D L^T of a Schur-complement Laplacian, eliminated in
// rounds of independent vertices.  Column c eliminates vertex col_vertex[c] with pivot
// col_diag[c] (0 = anchor) and entries (col_idx, col_coef = w/d) for its live neighbours.
// The last <= kAcCoreMax vertices form a dense core solved by its anchored inverse core_z.
struct AcFactor {
    int32_t n = 0, nlev = 0, ncol = 0, ncore = 0;
    std::vector<int32_t> level_ptr, col_vertex, col_ptr, col_idx;
    std::vector<double> col_diag, col_coef;
    std::vector<int32_t> core_vertex;  // ascending
    std::vector<double> core_z;        // ncore x ncore row-major
};

struct Subdomain {
    int q = 0, r = 0;
    std::vector<uint32_t> gidx;   // q-levels then r-levels (factor_pairs.rs:244-250)
    std::vector<double> pou;      // empty = uniform weights
    CrossTab ct;
    bool elim_q = true;           // n_q >= n_r (schur_complement.rs:174)
    std::vector<double> inv_diag; // 1 / D_elim
    int kind = 0;                 // 0 dense anchored Cholesky, 1 approximate Cholesky
    int32_t n_red = 0;            // reduced (kept) size
    std::vector<double> L;        // dense: (n_red-1)^2 row-major lower factor
    AcFactor ac;
    int32_t n_q() const { return ct.c.nrows; }
    int32_t n_r() const { return ct.c.ncols; }
    int32_t n_local() const { return ct.c.nrows + ct.c.ncols; }
};

struct PrecondConfig {
    int kind = 1;  // 0 off, 1 additive, 2 multiplicative
    uint64_t ac_seed = 0;
    uint32_t ac_split = 2;
    bool approx_schur = true;
    uint64_t schur_seed = 0;
    uint32_t schur_split = 1;
    int dense_threshold = 24;
};

struct Setup {
    Design d;
    std::vector<Subdomain> subs;
    // Explicit symmetric Gramian CSR (multiplicative Schwarz residual updates only).
    std::vector<int64_t> g_ptr;
    std::vector<uint32_t> g_idx;
    std::vector<double> g_val;
};

// Validates the inputs and builds the design (ArrayStore::new + from_store).
Status build_design(const uint32_t* codes, int64_t n, int Q, int64_t row_stride, int64_t col_stride,
                    const double* weights, Design& d);
// Builds subdomains and their local factors (build_local_domains + build_additive).
// device >= 0: the factor pairs' cross-tabulations of designs with at least
// kDeviceCrosstabMinObs observations are summed on that CUDA device (device_pair_sums);
// the result is identical to the host build, which is used otherwise or on any failure.
Status build_subdomains(const Design& d, const PrecondConfig& cfg, std::vector<Subdomain>& subs, int device = -1);
#ifndef WB_DEVICE_CROSSTAB_MIN_OBS
#define WB_DEVICE_CROSSTAB_MIN_OBS (1 << 15)
#endif
constexpr int64_t kDeviceCrosstabMinObs = WB_DEVICE_CROSSTAB_MIN_OBS;
// For the observations of a factor pair (q codes cq, r codes cr, weights w or null): the
// distinct keys qmap[cq] * nr + rmap[cr] in ascending order, with the sum of the weights of
// each key's observations taken in observation order (crosstab.cu).  False when the device
// path is unavailable or failed.
bool device_pair_sums(int device, int64_t n, const uint32_t* cq, const uint32_t* cr, const double* w,
                      const std::vector<uint32_t>& qmap, const std::vector<uint32_t>& rmap, uint32_t nq, uint32_t nr,
                      std::vector<uint64_t>& seg_key, std::vector<double>& seg_sum);
// Explicit Gramian for the multiplicative residual updater.
void build_explicit_gramian(const Design& d, std::vector<int64_t>& ptr, std::vector<uint32_t>& idx,
                            std::vector<double>& val);

// A built preconditioner as bytes (FePreconditioner pickling, within-py/src/lib.rs:890-913):
// the configuration, the subdomains with their local factors and, for multiplicative
// Schwarz, the explicit Gramian of its residual updates.  The format is this library's
// own: magic "WB200PC\0", a version, little-endian fields, length-prefixed arrays, an
// FNV-1a 64 checksum at the end.  Reading validates every count against the bytes left
// and every index against the sizes it addresses, so that nothing built from the bytes
// can address outside its arrays.
struct PrecondImage {
    int64_t ndofs = 0;
    int32_t kind = 1;       // 1 additive, 2 multiplicative
    int32_t reduction = 0;  // ReductionStrategy as configured
    PrecondConfig cfg;
    std::vector<Subdomain> subs;
    std::vector<int64_t> g_ptr;  // multiplicative only
    std::vector<uint32_t> g_idx;
    std::vector<double> g_val;
};
// img's subdomains are ignored in favour of `subs` (so that a solver's need not be copied).
std::vector<uint8_t> serialize_preconditioner(const PrecondImage& img, const std::vector<Subdomain>& subs);
Status deserialize_preconditioner(const uint8_t* data, size_t len, PrecondImage& img);

// LocalSolver::inner_parallelism_work_estimate of a block-elimination subdomain
// (within/src/operator/local_solver.rs:348-356).
int64_t inner_parallel_work(const Subdomain& sd);

// AdditiveSchwarzDiagnostics (schwarz-precond/src/schwarz/additive/planning.rs:141-210) and
// the strategy its scheduler resolves for `threads` worker threads (planning.rs:71-135).
// Strategies: 0 Auto, 1 AtomicScatter, 2 ParallelReduction.
struct AdditiveDiagnostics {
    int32_t configured = 0, resolved = 0;
    int64_t n_subdomains = 0, n_dofs = 0;
    int64_t total_inner_work = 0, max_inner_work = 0, total_scatter_dofs = 0;
    double outer_parallel_capacity = 0.0, scatter_overlap = 0.0;
};
AdditiveDiagnostics additive_diagnostics(const std::vector<Subdomain>& subs, int64_t n_dofs, int32_t configured,
                                         int64_t threads);

}  // namespace wb
