// Host-side setup of the solve phase (see setup.hpp).  Reference citations are
// relative to the reference's crates/ directory.
#include "setup.hpp"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <future>
#include <numeric>
#include <thread>

#include "../../include/within_b200.h"

namespace wb {

namespace {

// splitmix64 (Steele, Lea & Flood 2014): random stream of the clique-tree sampler.
struct SplitMix {
    uint64_t s;
    explicit SplitMix(uint64_t seed) : s(seed) {}
    uint64_t next() {
        uint64_t z = (s += 0x9E3779B97F4A7C15ULL);
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
        return z ^ (z >> 31);
    }
    double uniform() { return (double)(next() >> 11) * 0x1.0p-53; }
};
uint64_t hash64(uint64_t x) { return SplitMix(x).next(); }

Csr transpose(const Csr& a) {
    // Stable counting scatter: rows of the result come out column-sorted
    // (CsrBlock::transpose, operator/csr_block.rs:31-62).
    Csr t;
    t.nrows = a.ncols;
    t.ncols = a.nrows;
    const int64_t nnz = a.nnz();
    t.ptr.assign((size_t)t.nrows + 1, 0);
    t.idx.resize((size_t)nnz);
    t.val.resize((size_t)nnz);
    for (int64_t e = 0; e < nnz; ++e) t.ptr[a.idx[e] + 1]++;
    for (int32_t i = 0; i < t.nrows; ++i) t.ptr[i + 1] += t.ptr[i];
    std::vector<uint32_t> cursor(t.ptr.begin(), t.ptr.end() - 1);
    for (int32_t r = 0; r < a.nrows; ++r)
        for (uint32_t e = a.ptr[r]; e < a.ptr[r + 1]; ++e) {
            const uint32_t pos = cursor[a.idx[e]]++;
            t.idx[pos] = (uint32_t)r;
            t.val[pos] = a.val[e];
        }
    return t;
}

// One factor pair's cross-tab over active levels (CrossTab::build_for_pair_with_active,
// gramian/cross_tab.rs:246-265; bucket accumulation :568-664).  Returns false when a
// factor of the pair has no active level.
bool pair_crosstab(const Design& d, int q, int r, const std::vector<std::vector<uint8_t>>& active,
                   CrossTab& out, std::vector<uint32_t>& l2g, int32_t& nq_out, int device) {
    const int64_t Lq = d.nlev[q], Lr = d.nlev[r];
    std::vector<uint32_t> qmap((size_t)Lq, UINT32_MAX), rmap((size_t)Lr, UINT32_MAX);
    int32_t nq = 0, nr = 0;
    for (int64_t j = 0; j < Lq; ++j) if (active[q][j]) qmap[j] = (uint32_t)nq++;
    for (int64_t k = 0; k < Lr; ++k) if (active[r][k]) rmap[k] = (uint32_t)nr++;
    if (nq == 0 || nr == 0) return false;
    l2g.clear();
    l2g.reserve((size_t)nq + nr);
    for (int64_t j = 0; j < Lq; ++j) if (active[q][j]) l2g.push_back((uint32_t)(d.off[q] + j));
    for (int64_t k = 0; k < Lr; ++k) if (active[r][k]) l2g.push_back((uint32_t)(d.off[r] + k));

    const uint32_t* cq = d.codes.data() + (size_t)q * d.n;
    const uint32_t* cr = d.codes.data() + (size_t)r * d.n;
    std::vector<uint64_t> seg_key;
    std::vector<double> seg_sum;
    if (device >= 0 && d.n >= kDeviceCrosstabMinObs &&
        device_pair_sums(device, d.n, cq, cr, d.w.empty() ? nullptr : d.w.data(), qmap, rmap, (uint32_t)nq,
                         (uint32_t)nr, seg_key, seg_sum)) {
        // the device's distinct (row, column) keys in ascending order with their sums
        std::vector<double> dq((size_t)nq, 0.0), dr((size_t)nr, 0.0);
        for (int64_t i = 0; i < d.n; ++i) {
            const double w = d.weight(i);
            dq[qmap[cq[i]]] += w;
            dr[rmap[cr[i]]] += w;
        }
        Csr c;
        c.nrows = nq;
        c.ncols = nr;
        c.ptr.assign((size_t)nq + 1, 0);
        c.idx.reserve(seg_key.size());
        c.val.reserve(seg_key.size());
        for (size_t s = 0; s < seg_key.size(); ++s) {
            if (seg_sum[s] == 0.0) continue;  // as the host build drops exact zeros
            const uint64_t row = seg_key[s] / (uint64_t)nr;
            c.idx.push_back((uint32_t)(seg_key[s] % (uint64_t)nr));
            c.val.push_back(seg_sum[s]);
            c.ptr[row + 1]++;
        }
        for (int32_t j = 0; j < nq; ++j) c.ptr[j + 1] += c.ptr[j];
        out.ct = transpose(c);
        out.c = std::move(c);
        out.dq = std::move(dq);
        out.dr = std::move(dr);
        nq_out = nq;
        return true;
    }
    std::vector<double> dq((size_t)nq, 0.0), dr((size_t)nr, 0.0);
    std::vector<uint32_t> bptr((size_t)nq + 1, 0);
    for (int64_t i = 0; i < d.n; ++i) {
        const uint32_t j = qmap[cq[i]], k = rmap[cr[i]];
        const double w = d.weight(i);
        dq[j] += w;
        dr[k] += w;
        bptr[j + 1]++;
    }
    for (int32_t j = 0; j < nq; ++j) bptr[j + 1] += bptr[j];
    std::vector<uint32_t> bcol(bptr[nq]);
    std::vector<double> bval(bptr[nq]);
    {
        std::vector<uint32_t> cur(bptr.begin(), bptr.end() - 1);
        for (int64_t i = 0; i < d.n; ++i) {
            const uint32_t j = qmap[cq[i]];
            const uint32_t pos = cur[j]++;
            bcol[pos] = rmap[cr[i]];
            bval[pos] = d.weight(i);
        }
    }
    Csr c;
    c.nrows = nq;
    c.ncols = nr;
    c.ptr.assign((size_t)nq + 1, 0);
    c.idx.reserve(bcol.size());
    c.val.reserve(bcol.size());
    std::vector<double> work((size_t)nr, 0.0);
    std::vector<uint8_t> seen((size_t)nr, 0);
    std::vector<uint32_t> touched;
    for (int32_t row = 0; row < nq; ++row) {
        touched.clear();
        for (uint32_t e = bptr[row]; e < bptr[row + 1]; ++e) {
            const uint32_t col = bcol[e];
            if (!seen[col]) { seen[col] = 1; touched.push_back(col); }
            work[col] += bval[e];  // summed in observation order
        }
        std::sort(touched.begin(), touched.end());
        for (uint32_t col : touched) {
            if (work[col] != 0.0) { c.idx.push_back(col); c.val.push_back(work[col]); }
            work[col] = 0.0;
            seen[col] = 0;
        }
        c.ptr[row + 1] = (uint32_t)c.idx.size();
    }
    out.ct = transpose(c);
    out.c = std::move(c);
    out.dq = std::move(dq);
    out.dr = std::move(dr);
    nq_out = nq;
    return true;
}

struct Component {
    std::vector<int32_t> qi, ri;
};

// Connected components of the bipartite graph, in order of their smallest node
// (q-nodes numbered before r-nodes); members sorted.  Union-find gives the same sets
// and order as the reference's DFS (cross_tab.rs:381-444).
std::vector<Component> components(const CrossTab& x) {
    const int32_t nq = x.c.nrows, nr = x.c.ncols, n = nq + nr;
    std::vector<int32_t> parent((size_t)n);
    std::iota(parent.begin(), parent.end(), 0);
    auto find = [&](int32_t a) {
        while (parent[a] != a) { parent[a] = parent[parent[a]]; a = parent[a]; }
        return a;
    };
    for (int32_t i = 0; i < nq; ++i)
        for (uint32_t e = x.c.ptr[i]; e < x.c.ptr[i + 1]; ++e) {
            int32_t a = find(i), b = find(nq + (int32_t)x.c.idx[e]);
            if (a != b) parent[std::max(a, b)] = std::min(a, b);  // root = smallest node
        }
    std::vector<int32_t> comp_of((size_t)n, -1);
    std::vector<Component> comps;
    for (int32_t v = 0; v < n; ++v) {
        const int32_t root = find(v);
        if (comp_of[root] < 0) { comp_of[root] = (int32_t)comps.size(); comps.emplace_back(); }
        Component& c = comps[comp_of[root]];
        if (v < nq) c.qi.push_back(v); else c.ri.push_back(v - nq);
    }
    return comps;
}

// extract_component (cross_tab.rs:450-501).
CrossTab extract(const CrossTab& x, const Component& cp) {
    std::vector<uint32_t> rre((size_t)x.c.ncols, UINT32_MAX);
    for (size_t a = 0; a < cp.ri.size(); ++a) rre[cp.ri[a]] = (uint32_t)a;
    CrossTab o;
    o.dq.reserve(cp.qi.size());
    o.dr.reserve(cp.ri.size());
    for (int32_t i : cp.qi) o.dq.push_back(x.dq[i]);
    for (int32_t i : cp.ri) o.dr.push_back(x.dr[i]);
    Csr c;
    c.nrows = (int32_t)cp.qi.size();
    c.ncols = (int32_t)cp.ri.size();
    c.ptr.assign((size_t)c.nrows + 1, 0);
    for (int32_t a = 0; a < c.nrows; ++a) {
        const int32_t old = cp.qi[a];
        for (uint32_t e = x.c.ptr[old]; e < x.c.ptr[old + 1]; ++e) {
            const uint32_t nc = rre[x.c.idx[e]];
            if (nc != UINT32_MAX) { c.idx.push_back(nc); c.val.push_back(x.c.val[e]); }
        }
        c.ptr[a + 1] = (uint32_t)c.idx.size();
    }
    o.ct = transpose(c);
    o.c = std::move(c);
    return o;
}

// ---------------------------------------------------------------------------
// Schur complements (operator/schur_complement.rs)
// ---------------------------------------------------------------------------

struct Elim {
    bool elim_q;
    int32_t n_keep, n_elim;
    const std::vector<double>* diag_elim;
    const std::vector<double>* diag_keep;
    const Csr* k2e;  // keep rows -> elim columns
    const Csr* e2k;  // elim rows -> keep columns
};

Status make_elim(const CrossTab& x, Elim& e, std::vector<double>& inv) {
    const int32_t nq = x.c.nrows, nr = x.c.ncols;
    e.elim_q = nq >= nr;
    e.n_keep = e.elim_q ? nr : nq;
    e.n_elim = e.elim_q ? nq : nr;
    e.diag_elim = e.elim_q ? &x.dq : &x.dr;
    e.diag_keep = e.elim_q ? &x.dr : &x.dq;
    e.k2e = e.elim_q ? &x.ct : &x.c;
    e.e2k = e.elim_q ? &x.c : &x.ct;
    inv.resize((size_t)e.n_elim);
    for (int32_t i = 0; i < e.n_elim; ++i) {
        const double dd = (*e.diag_elim)[i];
        if (!(dd > 0.0)) {
            Status s;
            s.code = WITHIN_ERR_SINGULAR_DIAGONAL;
            s.msg = std::string("zero diagonal in ") + (e.elim_q ? "q (elim)" : "r (elim)") +
                    " block at index " + std::to_string(i);
            return s;
        }
        inv[i] = 1.0 / dd;
    }
    return {};
}

// Sparse symmetric matrix in CSR (only off-diagonal entries are used downstream).
struct SymCsr {
    int32_t n = 0;
    std::vector<uint32_t> ptr, idx;
    std::vector<double> val;
};

// Exact Schur complement by row workspace (SchurLaplacian::from_elimination, :394-412).
SymCsr schur_exact(const Elim& e, const std::vector<double>& inv) {
    SymCsr s;
    s.n = e.n_keep;
    s.ptr.assign((size_t)s.n + 1, 0);
    std::vector<double> work((size_t)s.n, 0.0);
    std::vector<uint8_t> in((size_t)s.n, 0);
    std::vector<int32_t> touched;
    for (int32_t i = 0; i < s.n; ++i) {
        touched.clear();
        work[i] = (*e.diag_keep)[i];
        touched.push_back(i);
        in[i] = 1;
        for (uint32_t f = e.k2e->ptr[i]; f < e.k2e->ptr[i + 1]; ++f) {
            const uint32_t k = e.k2e->idx[f];
            const double scale = e.k2e->val[f] * inv[k];
            for (uint32_t b = e.e2k->ptr[k]; b < e.e2k->ptr[k + 1]; ++b) {
                const uint32_t j = e.e2k->idx[b];
                if (!in[j]) { in[j] = 1; touched.push_back((int32_t)j); }
                work[j] -= scale * e.e2k->val[b];
            }
        }
        std::sort(touched.begin(), touched.end());
        for (int32_t j : touched) {
            if (work[j] != 0.0 || j == i) { s.idx.push_back((uint32_t)j); s.val.push_back(work[j]); }
            work[j] = 0.0;
            in[j] = 0;
        }
        s.ptr[i + 1] = (uint32_t)s.idx.size();
    }
    return s;
}

// Top-left (n_keep-1)^2 minor of the exact Schur complement (:490-527).
std::vector<double> schur_anchored_minor(const Elim& e, const std::vector<double>& inv) {
    const int32_t n = e.n_keep;
    if (n <= 1) return {};
    const int32_t m = n - 1;
    std::vector<double> a((size_t)m * m, 0.0);
    for (int32_t i = 0; i < m; ++i) a[(size_t)i * m + i] = (*e.diag_keep)[i];
    for (int32_t i = 0; i < m; ++i)
        for (uint32_t f = e.k2e->ptr[i]; f < e.k2e->ptr[i + 1]; ++f) {
            const uint32_t k = e.k2e->idx[f];
            const double scale = e.k2e->val[f] * inv[k];
            for (uint32_t b = e.e2k->ptr[k]; b < e.e2k->ptr[k + 1]; ++b) {
                const uint32_t j = e.e2k->idx[b];
                if ((int32_t)j < m) a[(size_t)i * m + j] -= scale * e.e2k->val[b];
            }
        }
    return a;
}

struct Edge {
    uint32_t lo, hi;
    double w;
};
struct Nbr {
    uint32_t col;
    double w;
};

// Sampled clique tree of one eliminated vertex (Gao, Kyng & Spielman,
// arXiv:2303.00709).  Neighbours split into `split` copies of weight w/split are
// ordered by (weight, column); copy i links to a later copy j drawn with
// probability w_j / S_i (S_i = weight after i) with edge weight w_i S_i / d, so the
// expected tree equals the clique with weights w_a w_b / d.  One uniform draw per
// copy; links between copies of one neighbour are dropped (self-loops).
class CliqueTreeSampler {
public:
    void sample(const Nbr* nb, int32_t deg, uint32_t split, double d, uint64_t seed,
                std::vector<Edge>& out) {
        if (split < 1) split = 1;
        const int32_t m = deg * (int32_t)split;
        v_.resize((size_t)m);
        cum_.resize((size_t)m);
        suf_.resize((size_t)m);
        for (int32_t a = 0, p = 0; a < deg; ++a)
            for (uint32_t s = 0; s < split; ++s, ++p) v_[p] = Nbr{nb[a].col, nb[a].w / (double)split};
        std::sort(v_.begin(), v_.end(), [](const Nbr& x, const Nbr& y) {
            if (x.w != y.w) return x.w < y.w;
            return x.col < y.col;
        });
        double acc = 0.0;
        for (int32_t a = 0; a < m; ++a) { acc += v_[a].w; cum_[a] = acc; }
        acc = 0.0;
        for (int32_t a = m - 1; a >= 0; --a) { suf_[a] = acc; acc += v_[a].w; }
        SplitMix rng(seed);
        for (int32_t i = 0; i + 1 < m; ++i) {
            const double u = rng.uniform();
            if (!(suf_[i] > 0.0)) continue;
            const double target = cum_[i] + u * suf_[i];
            // first j in (i, m-1] with cum[j] > target
            const int32_t j = (int32_t)(std::upper_bound(cum_.begin() + i + 1, cum_.begin() + m - 1, target) -
                                        cum_.begin());
            if (v_[j].col == v_[i].col) continue;
            const uint32_t a = v_[i].col, b = v_[j].col;
            out.push_back(Edge{std::min(a, b), std::max(a, b), v_[i].w * suf_[i] / d});
        }
    }

private:
    std::vector<Nbr> v_;
    std::vector<double> cum_, suf_;
};

// Stable sort by (lo, hi), then sum duplicates in emission order.
void sort_merge_edges(std::vector<Edge>& e) {
    std::stable_sort(e.begin(), e.end(), [](const Edge& a, const Edge& b) {
        return a.lo != b.lo ? a.lo < b.lo : a.hi < b.hi;
    });
    size_t w = 0;
    for (size_t a = 0; a < e.size(); ++a) {
        if (w > 0 && e[w - 1].lo == e[a].lo && e[w - 1].hi == e[a].hi) e[w - 1].w += e[a].w;
        else e[w++] = e[a];
    }
    e.resize(w);
}

// Approximate Schur complement: each eliminated star of degree > 1 emits a clique
// tree with seed = seed + k (ApproxSchurComplement::compute, :697-711 and :128-139).
SymCsr schur_approx(const Elim& e, uint64_t seed, uint32_t split) {
    std::vector<Edge> edges;
    CliqueTreeSampler sampler;
    std::vector<Nbr> nb;
    for (int32_t k = 0; k < e.n_elim; ++k) {
        const uint32_t b = e.e2k->ptr[k], en = e.e2k->ptr[k + 1];
        const int32_t deg = (int32_t)(en - b);
        if (deg <= 1) continue;
        nb.resize((size_t)deg);
        for (int32_t a = 0; a < deg; ++a) nb[a] = Nbr{e.e2k->idx[b + a], e.e2k->val[b + a]};
        sampler.sample(nb.data(), deg, split, (*e.diag_elim)[k], seed + (uint64_t)k, edges);
    }
    sort_merge_edges(edges);
    // Laplacian CSR (build_laplacian_csr, :534-586); only off-diagonals are consumed.
    SymCsr s;
    s.n = e.n_keep;
    std::vector<uint32_t> lc((size_t)s.n, 0), uc((size_t)s.n, 0);
    std::vector<double> dg((size_t)s.n, 0.0);
    for (const Edge& x : edges) { uc[x.lo]++; lc[x.hi]++; dg[x.lo] += x.w; dg[x.hi] += x.w; }
    s.ptr.assign((size_t)s.n + 1, 0);
    for (int32_t i = 0; i < s.n; ++i) s.ptr[i + 1] = s.ptr[i] + lc[i] + 1 + uc[i];
    s.idx.resize(s.ptr[s.n]);
    s.val.resize(s.ptr[s.n]);
    std::vector<uint32_t> lcur((size_t)s.n), ucur((size_t)s.n);
    for (int32_t i = 0; i < s.n; ++i) {
        lcur[i] = s.ptr[i];
        ucur[i] = s.ptr[i] + lc[i] + 1;
        s.idx[s.ptr[i] + lc[i]] = (uint32_t)i;
        s.val[s.ptr[i] + lc[i]] = dg[i];
    }
    for (const Edge& x : edges) {
        uint32_t p = ucur[x.lo]++;
        s.idx[p] = x.hi;
        s.val[p] = -x.w;
        p = lcur[x.hi]++;
        s.idx[p] = x.lo;
        s.val[p] = -x.w;
    }
    return s;
}

// ---------------------------------------------------------------------------
// Approximate Cholesky in rounds of independent vertices
// ---------------------------------------------------------------------------

// Sort neighbour records by column (stable) and merge duplicates, dropping dead ones.
// compact_adj for a list whose first `sorted` entries are already sorted by column and
// merged (the last compaction's output) and whose tail holds entries appended since:
// the tail is sorted and merged into the prefix stably, which orders the entries exactly
// as a stable sort of the whole list would.  Returns the list's new length (all sorted).
size_t compact_adj_tail(std::vector<Nbr>& l, size_t sorted, const std::vector<uint8_t>& dead,
                        std::vector<Nbr>& scratch) {
    size_t m = 0, mp = 0;
    for (size_t a = 0; a < l.size(); ++a) {
        if (dead[l[a].col]) continue;
        if (a < sorted) ++mp;
        l[m++] = l[a];
    }
    l.resize(m);
    auto by_col = [](const Nbr& a, const Nbr& b) { return a.col < b.col; };
    if (mp < m) {
        std::stable_sort(l.begin() + (ptrdiff_t)mp, l.end(), by_col);
        scratch.resize(m);
        std::merge(l.begin(), l.begin() + (ptrdiff_t)mp, l.begin() + (ptrdiff_t)mp, l.end(), scratch.begin(), by_col);
        std::copy(scratch.begin(), scratch.begin() + (ptrdiff_t)m, l.begin());
    }
    size_t w = 0;
    for (size_t a = 0; a < m; ++a) {
        if (w > 0 && l[w - 1].col == l[a].col) l[w - 1].w += l[a].w;
        else l[w++] = l[a];
    }
    l.resize(w);
    return w;
}

void compact_adj(std::vector<Nbr>& l, const std::vector<uint8_t>& dead) {
    size_t m = 0;
    for (size_t a = 0; a < l.size(); ++a)
        if (!dead[l[a].col]) l[m++] = l[a];
    l.resize(m);
    std::stable_sort(l.begin(), l.end(), [](const Nbr& a, const Nbr& b) { return a.col < b.col; });
    size_t w = 0;
    for (size_t a = 0; a < m; ++a) {
        if (w > 0 && l[w - 1].col == l[a].col) l[w - 1].w += l[a].w;
        else l[w++] = l[a];
    }
    l.resize(w);
}

bool dense_cholesky(std::vector<double>& a, int32_t m);

// SPD inverse through the Cholesky factor: A = L L^T, A^-1 = L^-T L^-1.
bool spd_inverse(std::vector<double>& a, int32_t m) {
    if (!dense_cholesky(a, m)) return false;
    // L^-1 row by row (row i = (e_i - sum_{k<i} L_ik row_k) / L_ii): contiguous row updates
    std::vector<double> li((size_t)m * m, 0.0);
    for (int32_t i = 0; i < m; ++i) {
        double* ri = li.data() + (size_t)i * m;
        const double* lrow = a.data() + (size_t)i * m;
        for (int32_t k = 0; k < i; ++k) {
            const double c = lrow[k];
            if (c == 0.0) continue;
            const double* rk = li.data() + (size_t)k * m;
            for (int32_t j = 0; j <= k; ++j) ri[j] -= c * rk[j];
        }
        ri[i] += 1.0;
        const double inv = 1.0 / lrow[i];
        for (int32_t j = 0; j <= i; ++j) ri[j] *= inv;
    }
    // A^-1 = L^-T L^-1 = sum_k row_k^T row_k, accumulated row by row into the lower half
    std::vector<double> z((size_t)m * m, 0.0);
    for (int32_t k = 0; k < m; ++k) {
        const double* rk = li.data() + (size_t)k * m;
        for (int32_t i = 0; i <= k; ++i) {
            const double c = rk[i];
            if (c == 0.0) continue;
            double* zi = z.data() + (size_t)i * m;
            for (int32_t j = 0; j <= i; ++j) zi[j] += c * rk[j];
        }
    }
    for (int32_t i = 0; i < m; ++i)
        for (int32_t j = 0; j < i; ++j) z[(size_t)j * m + i] = z[(size_t)i * m + j];
    a.swap(z);
    return true;
}

// Dense core: live vertices ascending, exact Laplacian of the remaining graph, anchored
// inverse per connected component (anchor = the component's largest vertex).
void ac_core(AcFactor& f, std::vector<std::vector<Nbr>>& g, const std::vector<uint8_t>& dead) {
    const int32_t n = f.n;
    std::vector<int32_t> loc((size_t)n, -1);
    int32_t r = 0;
    for (int32_t v = 0; v < n; ++v) if (!dead[v]) { loc[v] = r++; f.core_vertex.push_back(v); }
    f.ncore = r;
    f.core_z.assign((size_t)r * r, 0.0);
    if (r == 0) return;
    std::vector<double> S((size_t)r * r, 0.0);
    std::vector<int32_t> parent((size_t)r);
    std::iota(parent.begin(), parent.end(), 0);
    auto find = [&](int32_t a) { while (parent[a] != a) a = parent[a]; return a; };
    for (int32_t a = 0; a < r; ++a) {
        std::vector<Nbr>& L = g[f.core_vertex[a]];
        compact_adj(L, dead);
        for (const Nbr& x : L) {
            const int32_t c = loc[x.col];
            S[(size_t)a * r + c] -= x.w;
            S[(size_t)a * r + a] += x.w;
            const int32_t ra = find(a), rc = find(c);
            if (ra != rc) parent[std::max(ra, rc)] = std::min(ra, rc);
        }
    }
    std::vector<int32_t> root((size_t)r);
    for (int32_t a = 0; a < r; ++a) root[a] = find(a);
    std::vector<uint8_t> done((size_t)r, 0);
    std::vector<int32_t> mem;
    for (int32_t a = 0; a < r; ++a) {
        if (done[root[a]]) continue;
        done[root[a]] = 1;
        mem.clear();
        for (int32_t b = a; b < r; ++b) if (root[b] == root[a]) mem.push_back(b);
        const int32_t m = (int32_t)mem.size() - 1;  // last member anchors the component
        if (m <= 0) continue;
        std::vector<double> A((size_t)m * m);
        for (int32_t i = 0; i < m; ++i)
            for (int32_t j = 0; j < m; ++j) A[(size_t)i * m + j] = S[(size_t)mem[i] * r + mem[j]];
        if (spd_inverse(A, m))
            for (int32_t i = 0; i < m; ++i)
                for (int32_t j = 0; j < m; ++j) f.core_z[(size_t)mem[i] * r + mem[j]] = A[(size_t)i * m + j];
    }
}

AcFactor ac_factor(const SymCsr& s, uint64_t seed, uint32_t split) {
    const int32_t n = s.n;
    AcFactor f;
    f.n = n;
    std::vector<std::vector<Nbr>> g((size_t)n);
    for (int32_t i = 0; i < n; ++i)
        for (uint32_t e = s.ptr[i]; e < s.ptr[i + 1]; ++e)
            if ((int32_t)s.idx[e] != i && s.val[e] < 0.0) g[i].push_back(Nbr{s.idx[e], -s.val[e]});
    std::vector<uint8_t> dead((size_t)n, 0), blocked((size_t)n, 0);
    struct Rank {
        int32_t deg;
        uint64_t h;
        int32_t v;
    };
    std::vector<Rank> rank;
    std::vector<int32_t> picked;
    f.col_vertex.reserve((size_t)n);
    f.col_diag.reserve((size_t)n);
    f.col_ptr.reserve((size_t)n + 1);
    int32_t remaining = n;
    // A vertex's list changes only when a neighbour is eliminated (the neighbour dies, fill
    // edges arrive), so only those "dirty" lists are compacted in the next round; a clean
    // list is already sorted and merged, where compacting it again would change nothing.
    std::vector<uint8_t> dirty((size_t)n, 1);
    std::vector<size_t> sorted_len((size_t)n, 0);  // leading entries already sorted and merged
    std::vector<uint64_t> vhash((size_t)n);
    for (int32_t v = 0; v < n; ++v) vhash[v] = hash64(seed ^ ((uint64_t)v * 0xD1B54A32D192ED03ULL));
    std::vector<int32_t> live((size_t)n);  // live vertices, ascending
    std::iota(live.begin(), live.end(), 0);
    std::vector<int32_t> todo;
    std::vector<std::vector<Edge>> fills;
    // vertices per task of the parallel phases (small: the late rounds pick few vertices
    // of high degree, whose lists and samples are the long ones)
    constexpr size_t kCompactTask = 64, kSampleTask = 16, kColTask = 256;
    std::vector<size_t> col_off;
    while (remaining > kAcCoreMax) {
        // compact the dirty lists (each list alone: independent across vertices)
        todo.clear();
        for (int32_t v : live)
            if (dirty[v]) todo.push_back(v);
        parallel_tasks((todo.size() + kCompactTask - 1) / kCompactTask, [&](size_t t) {
            std::vector<Nbr> scr;
            for (size_t a = t * kCompactTask; a < std::min(todo.size(), (t + 1) * kCompactTask); ++a) {
                const int32_t v = todo[a];
                sorted_len[v] = compact_adj_tail(g[v], sorted_len[v], dead, scr);
                dirty[v] = 0;
            }
        });
        rank.clear();
        for (int32_t v : live) rank.push_back(Rank{(int32_t)g[v].size(), vhash[v], v});
        std::sort(rank.begin(), rank.end(), [](const Rank& a, const Rank& b) {
            if (a.deg != b.deg) return a.deg < b.deg;
            if (a.h != b.h) return a.h < b.h;
            return a.v < b.v;
        });
        picked.clear();
        for (const Rank& rk : rank) {
            if (blocked[rk.v]) continue;
            picked.push_back(rk.v);
            blocked[rk.v] = 1;
            for (const Nbr& x : g[rk.v]) blocked[x.col] = 1;
        }
        if ((int64_t)picked.size() < std::max<int64_t>(kAcStallMin, remaining / kAcStallDiv)) {
            // the remaining graph has turned dense: rounds would eliminate a few vertices
            // each; stop here (the tail below)
            for (const Rank& rk : rank) blocked[rk.v] = 0;
            break;
        }
        f.level_ptr.push_back((int32_t)f.col_vertex.size());
        // the picked vertices are independent: no fill edge touches another picked vertex's
        // list, so every clique tree is sampled from the lists as they are now (in parallel,
        // each with its own seed) and the fill is then added in pick order
        fills.resize(picked.size());
        parallel_tasks((picked.size() + kSampleTask - 1) / kSampleTask, [&](size_t t) {
            CliqueTreeSampler smp;
            for (size_t a = t * kSampleTask; a < std::min(picked.size(), (t + 1) * kSampleTask); ++a) {
                const int32_t v = picked[a];
                const std::vector<Nbr>& L = g[v];
                fills[a].clear();
                if (L.size() <= 1) continue;
                double d = 0.0;
                for (const Nbr& x : L) d += x.w;
                smp.sample(L.data(), (int32_t)L.size(), split, d, seed + (uint64_t)v, fills[a]);
            }
        });
        // the picked vertices' columns: sized first, then written in parallel (each column
        // at its offset, with the same arithmetic as an append in pick order)
        {
            const size_t c0 = f.col_vertex.size(), i0 = f.col_idx.size(), np = picked.size();
            col_off.assign(np + 1, 0);
            for (size_t a = 0; a < np; ++a) col_off[a + 1] = col_off[a] + g[picked[a]].size();
            f.col_vertex.resize(c0 + np);
            f.col_diag.resize(c0 + np);
            f.col_ptr.resize(c0 + np);
            f.col_idx.resize(i0 + col_off[np]);
            f.col_coef.resize(i0 + col_off[np]);
            parallel_tasks((np + kColTask - 1) / kColTask, [&](size_t t) {
                for (size_t a = t * kColTask; a < std::min(np, (t + 1) * kColTask); ++a) {
                    const int32_t v = picked[a];
                    const std::vector<Nbr>& L = g[v];
                    double d = 0.0;
                    for (const Nbr& x : L) d += x.w;
                    f.col_vertex[c0 + a] = v;
                    f.col_diag[c0 + a] = L.empty() ? 0.0 : d;
                    f.col_ptr[c0 + a] = (int32_t)(i0 + col_off[a]);
                    for (size_t j = 0; j < L.size(); ++j) {
                        f.col_idx[i0 + col_off[a] + j] = (int32_t)L[j].col;
                        f.col_coef[i0 + col_off[a] + j] = L[j].w / d;
                    }
                }
            });
        }
        // the fill, appended in emission order: worker w of nw owns the target vertices
        // u with u % nw == w and scans every edge, so each list receives its entries in
        // the same order as one sequential pass (nw = 1) appends them
        parallel_workers(8, [&](int w, int nw) {
            const uint32_t uw = (uint32_t)w, un = (uint32_t)nw;
            for (size_t a = 0; a < picked.size(); ++a)
                for (const Edge& e : fills[a]) {
                    if (e.lo % un == uw) g[e.lo].push_back(Nbr{e.hi, e.w});
                    if (e.hi % un == uw) g[e.hi].push_back(Nbr{e.lo, e.w});
                }
        });
        for (int32_t v : picked)
            for (const Nbr& x : g[v]) dirty[x.col] = 1;
        for (int32_t v : picked) { dead[v] = 1; std::vector<Nbr>().swap(g[v]); }
        live.erase(std::remove_if(live.begin(), live.end(), [&](int32_t v) { return dead[v] != 0; }), live.end());
        for (const Rank& rk : rank) blocked[rk.v] = 0;
        remaining -= (int32_t)picked.size();
        f.nlev++;
    }
    if (remaining > kAcCoreMax) {
        // stalled with more vertices than a dense core holds: one last level of pivots,
        // each remaining vertex's weighted degree in the remaining graph (the diagonal
        // of the remaining Laplacian) and no off-diagonal entries
        f.level_ptr.push_back((int32_t)f.col_vertex.size());
        for (int32_t v = 0; v < n; ++v) {
            if (dead[v]) continue;
            compact_adj(g[v], dead);
            double d = 0.0;
            for (const Nbr& x : g[v]) d += x.w;
            f.col_vertex.push_back(v);
            f.col_diag.push_back(g[v].empty() ? 0.0 : d);
            f.col_ptr.push_back((int32_t)f.col_idx.size());
        }
        for (int32_t v = 0; v < n; ++v) dead[v] = 1;
        f.nlev++;
    }
    f.level_ptr.push_back((int32_t)f.col_vertex.size());
    f.col_ptr.push_back((int32_t)f.col_idx.size());
    f.ncol = (int32_t)f.col_vertex.size();
    ac_core(f, g, dead);
    return f;
}

// Lower Cholesky of an SPD row-major matrix; false when a pivot is not positive.
bool dense_cholesky(std::vector<double>& a, int32_t m) {
    // dot products with four partial sums (vectorisable; rounding differs from a strict
    // left-to-right sum only in the last bits)
    auto dot = [](const double* x, const double* y, int32_t n) {
        double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;
        int32_t k = 0;
        for (; k + 4 <= n; k += 4) {
            s0 += x[k] * y[k];
            s1 += x[k + 1] * y[k + 1];
            s2 += x[k + 2] * y[k + 2];
            s3 += x[k + 3] * y[k + 3];
        }
        for (; k < n; ++k) s0 += x[k] * y[k];
        return (s0 + s1) + (s2 + s3);
    };
    for (int32_t j = 0; j < m; ++j) {
        double* rj = a.data() + (size_t)j * m;
        const double s = rj[j] - dot(rj, rj, j);
        if (!(s > 0.0)) return false;
        const double ljj = std::sqrt(s);
        rj[j] = ljj;
        for (int32_t i = j + 1; i < m; ++i) {
            double* ri = a.data() + (size_t)i * m;
            ri[j] = (ri[j] - dot(ri, rj, j)) / ljj;
        }
        for (int32_t i = 0; i < j; ++i) a[(size_t)i * m + j] = 0.0;
    }
    return true;
}

// build_reduced_schur_factor (operator/schwarz.rs:274-303).
Status build_local_factor(Subdomain& sd, const PrecondConfig& cfg) {
    Elim e;
    Status st = make_elim(sd.ct, e, sd.inv_diag);
    if (!st.ok()) return st;
    sd.elim_q = e.elim_q;
    if (cfg.dense_threshold > 0 && e.n_keep <= cfg.dense_threshold) {
        std::vector<double> minor = schur_anchored_minor(e, sd.inv_diag);
        if (e.n_keep <= 1 || dense_cholesky(minor, e.n_keep - 1)) {
            sd.kind = 0;
            sd.n_red = e.n_keep;
            sd.L = std::move(minor);
            return {};
        }
    }
    SymCsr s = cfg.approx_schur ? schur_approx(e, cfg.schur_seed, cfg.schur_split) : schur_exact(e, sd.inv_diag);
    sd.kind = 1;
    sd.n_red = e.n_keep;
    sd.ac = ac_factor(s, cfg.ac_seed, cfg.ac_split < 1 ? 1 : cfg.ac_split);
    return {};
}

}  // namespace

Status build_design(const uint32_t* codes, int64_t n, int Q, int64_t row_stride, int64_t col_stride,
                    const double* weights, Design& d) {
    Status st;
    if (n <= 0) { st.code = WITHIN_ERR_EMPTY_OBSERVATIONS; st.msg = "no observations provided"; return st; }
    if (Q <= 0) { st.code = WITHIN_ERR_INVALID_ARGUMENT; st.msg = "categories must have at least one factor column"; return st; }
    if ((uint64_t)n > 0xFFFFFFFFull) { st.code = WITHIN_ERR_OVERFLOW; st.msg = "more than 2^32-1 observations"; return st; }
    d.n = n;
    d.Q = Q;
    d.codes.resize((size_t)n * Q);
    if (weights) d.w.resize((size_t)n);
    // copy and per-factor maxima over ranges of observations (a maximum does not depend
    // on the order it is taken in)
    constexpr int64_t kRange = 1 << 20;
    const int64_t nr = (n + kRange - 1) / kRange;
    std::vector<uint32_t> mx((size_t)nr * Q, 0);
    parallel_tasks((size_t)nr, [&](size_t t) {
        const int64_t i0 = (int64_t)t * kRange, i1 = std::min(n, i0 + kRange);
        for (int q = 0; q < Q; ++q) {
            uint32_t* dst = d.codes.data() + (size_t)q * n;
            if (row_stride == 1) {
                std::memcpy(dst + i0, codes + q * col_stride + i0, sizeof(uint32_t) * (size_t)(i1 - i0));
            } else {
                for (int64_t i = i0; i < i1; ++i) dst[i] = codes[i * row_stride + q * col_stride];
            }
            uint32_t m = 0;
            for (int64_t i = i0; i < i1; ++i) m = std::max(m, dst[i]);
            mx[t * Q + q] = m;
        }
        if (weights) std::memcpy(d.w.data() + i0, weights + i0, sizeof(double) * (size_t)(i1 - i0));
    });
    d.nlev.resize(Q);
    d.off.resize(Q);
    int64_t off = 0;
    for (int q = 0; q < Q; ++q) {
        uint32_t m = 0;
        for (int64_t t = 0; t < nr; ++t) m = std::max(m, mx[(size_t)t * Q + q]);
        d.nlev[q] = (int64_t)m + 1;
        d.off[q] = off;
        off += d.nlev[q];
    }
    if ((uint64_t)off > 0xFFFFFFFFull) { st.code = WITHIN_ERR_OVERFLOW; st.msg = "more than 2^32-1 fixed-effect levels"; return st; }
    d.ndofs = off;
    return st;
}

Status build_subdomains(const Design& d, const PrecondConfig& cfg, std::vector<Subdomain>& subs, int device) {
    subs.clear();
    std::vector<std::vector<uint8_t>> active((size_t)d.Q);
    for (int q = 0; q < d.Q; ++q) {  // find_all_active_levels (cross_tab.rs:75-89)
        active[q].assign((size_t)d.nlev[q], 0);
        const uint32_t* c = d.codes.data() + (size_t)q * d.n;
        // observation ranges mark their own flags, which are then or-ed level by level
        constexpr int64_t kRange = 1 << 21;
        const int64_t nr = (d.n + kRange - 1) / kRange;
        if (nr <= 1 || nr * d.nlev[q] > ((int64_t)1 << 26)) {  // one pass, or flags too large
            for (int64_t i = 0; i < d.n; ++i) active[q][c[i]] = 1;
            continue;
        }
        const int64_t L = d.nlev[q];
        std::vector<uint8_t> part((size_t)nr * L, 0);
        parallel_tasks((size_t)nr, [&](size_t t) {
            uint8_t* a = part.data() + t * L;
            for (int64_t i = (int64_t)t * kRange; i < std::min(d.n, ((int64_t)t + 1) * kRange); ++i) a[c[i]] = 1;
        });
        const int64_t nl = (L + kRange - 1) / kRange;
        parallel_tasks((size_t)nl, [&](size_t b) {
            for (int64_t j = (int64_t)b * kRange; j < std::min(L, ((int64_t)b + 1) * kRange); ++j)
                for (int64_t t = 0; t < nr; ++t)
                    if (part[(size_t)t * L + j]) { active[q][j] = 1; break; }
        });
    }
    // Pairs (q < r) in lexicographic order (factor_pairs.rs:252-260); components in
    // order; indices q-levels then r-levels (:244-250).  The pairs are independent and
    // built concurrently (each pair's arithmetic is unchanged), then appended in order.
    // A pair's local factors (which do not depend on the partition of unity) are built
    // as soon as its subdomains exist: the large ones on threads of their own, the rest
    // on the pair's thread.
    std::vector<std::pair<int, int>> pairs;
    for (int q = 0; q < d.Q; ++q)
        for (int r = q + 1; r < d.Q; ++r) pairs.emplace_back(q, r);
    std::vector<std::vector<Subdomain>> per_pair(pairs.size());
    std::vector<std::vector<Status>> per_status(pairs.size());
    // (threads come from the process-wide budget: try_take_helper)
    auto factor_pair = [&](size_t p) {
        std::vector<Subdomain>& v = per_pair[p];
        std::vector<Status>& status = per_status[p];
        status.assign(v.size(), Status{});
        std::vector<std::future<void>> jobs;
        for (size_t i = 0; i < v.size(); ++i) {
            if (v[i].n_local() > 4096 && try_take_helper()) {
                jobs.push_back(std::async(std::launch::async, [&, i] {
                    status[i] = build_local_factor(v[i], cfg);
                    release_helper();
                }));
            } else {
                status[i] = build_local_factor(v[i], cfg);
            }
        }
        for (auto& j : jobs) j.get();
    };
    auto build_pair = [&](size_t p) {
        const int q = pairs[p].first, r = pairs[p].second;
        CrossTab full;
        std::vector<uint32_t> l2g;
        int32_t nqf = 0;
        if (!pair_crosstab(d, q, r, active, full, l2g, nqf, device)) return;
        std::vector<Component> comps = components(full);
        for (size_t c = 0; c < comps.size(); ++c) {
            Subdomain sd;
            sd.q = q;
            sd.r = r;
            sd.gidx.reserve(comps[c].qi.size() + comps[c].ri.size());
            for (int32_t i : comps[c].qi) sd.gidx.push_back(l2g[i]);
            for (int32_t i : comps[c].ri) sd.gidx.push_back(l2g[nqf + i]);
            sd.ct = comps.size() == 1 ? std::move(full) : extract(full, comps[c]);
            per_pair[p].push_back(std::move(sd));
        }
        factor_pair(p);
    };
    {
        std::vector<std::future<void>> pj;
        for (size_t p = 0; p < pairs.size(); ++p) {
            if (p + 1 < pairs.size() && try_take_helper())
                pj.push_back(std::async(std::launch::async, [&, p] {
                    build_pair(p);
                    release_helper();
                }));
            else
                build_pair(p);
        }
        for (auto& j : pj) j.get();
    }
    for (const auto& v : per_status)
        for (const Status& st : v)
            if (!st.ok()) return st;
    for (auto& v : per_pair)
        for (auto& sd : v) subs.push_back(std::move(sd));
    // Partition-of-unity weights (compute_partition_weights, factor_pairs.rs:272-304).
    std::vector<uint32_t> count((size_t)d.ndofs, 0);
    for (const Subdomain& sd : subs)
        for (uint32_t g : sd.gidx) count[g]++;
    for (Subdomain& sd : subs) {
        bool unique = true;
        for (uint32_t g : sd.gidx) if (count[g] > 1) { unique = false; break; }
        if (!unique) {
            sd.pou.resize(sd.gidx.size());
            for (size_t a = 0; a < sd.gidx.size(); ++a) sd.pou[a] = 1.0 / std::sqrt((double)count[sd.gidx[a]]);
        }
    }
    return {};
}

void build_explicit_gramian(const Design& d, std::vector<int64_t>& ptr, std::vector<uint32_t>& idx,
                            std::vector<double>& val) {
    // Gramian::build (gramian/explicit.rs:207): G = D'WD as symmetric CSR, columns
    // ascending, each row = its diagonal plus every cross-pair entry.
    const int64_t m = d.ndofs;
    std::vector<double> diag((size_t)m, 0.0);
    for (int q = 0; q < d.Q; ++q)
        for (int64_t i = 0; i < d.n; ++i) diag[d.off[q] + d.level(i, q)] += d.weight(i);
    std::vector<std::vector<std::pair<uint32_t, double>>> rows((size_t)m);
    for (int q = 0; q < d.Q; ++q)
        for (int r = q + 1; r < d.Q; ++r) {
            const int64_t Lq = d.nlev[q];
            std::vector<int64_t> bp((size_t)Lq + 1, 0);
            for (int64_t i = 0; i < d.n; ++i) bp[d.level(i, q) + 1]++;
            for (int64_t j = 0; j < Lq; ++j) bp[j + 1] += bp[j];
            std::vector<int64_t> cur(bp.begin(), bp.end() - 1);
            std::vector<std::pair<uint32_t, double>> b((size_t)d.n);
            for (int64_t i = 0; i < d.n; ++i)
                b[cur[d.level(i, q)]++] = {(uint32_t)(d.off[r] + d.level(i, r)), d.weight(i)};
            for (int64_t j = 0; j < Lq; ++j) {
                std::stable_sort(b.begin() + bp[j], b.begin() + bp[j + 1],
                                 [](const auto& x, const auto& y) { return x.first < y.first; });
                const uint32_t gq = (uint32_t)(d.off[q] + j);
                for (int64_t e = bp[j]; e < bp[j + 1];) {
                    const uint32_t col = b[e].first;
                    double w = 0.0;
                    while (e < bp[j + 1] && b[e].first == col) { w += b[e].second; ++e; }
                    if (w == 0.0) continue;
                    rows[gq].push_back({col, w});
                    rows[col].push_back({gq, w});
                }
            }
        }
    ptr.assign((size_t)m + 1, 0);
    for (int64_t i = 0; i < m; ++i) ptr[i + 1] = ptr[i] + (int64_t)rows[i].size() + 1;
    idx.resize((size_t)ptr[m]);
    val.resize((size_t)ptr[m]);
    for (int64_t i = 0; i < m; ++i) {
        rows[i].push_back({(uint32_t)i, diag[i]});
        std::sort(rows[i].begin(), rows[i].end(), [](const auto& x, const auto& y) { return x.first < y.first; });
        for (size_t a = 0; a < rows[i].size(); ++a) {
            idx[ptr[i] + a] = rows[i][a].first;
            val[ptr[i] + a] = rows[i][a].second;
        }
        std::vector<std::pair<uint32_t, double>>().swap(rows[i]);
    }
}

namespace {

constexpr char kPcMagic[8] = {'W', 'B', '2', '0', '0', 'P', 'C', '\0'};
constexpr uint32_t kPcVersion = 1;

uint64_t fnv1a(const uint8_t* p, size_t n) {
    uint64_t h = 1469598103934665603ull;
    for (size_t i = 0; i < n; ++i) { h ^= p[i]; h *= 1099511628211ull; }
    return h;
}

struct Writer {
    std::vector<uint8_t> b;
    template <typename T> void put(T v) {
        const uint8_t* p = reinterpret_cast<const uint8_t*>(&v);
        b.insert(b.end(), p, p + sizeof(T));
    }
    template <typename T> void vec(const std::vector<T>& v) {
        put<uint64_t>(v.size());
        const uint8_t* p = reinterpret_cast<const uint8_t*>(v.data());
        b.insert(b.end(), p, p + sizeof(T) * v.size());
    }
    void csr(const Csr& c) { put<int32_t>(c.nrows); put<int32_t>(c.ncols); vec(c.ptr); vec(c.idx); vec(c.val); }
};

struct Reader {
    const uint8_t* p;
    size_t left;
    bool ok = true;
    template <typename T> T get() {
        T v{};
        if (!ok || left < sizeof(T)) { ok = false; return v; }
        std::memcpy(&v, p, sizeof(T));
        p += sizeof(T);
        left -= sizeof(T);
        return v;
    }
    template <typename T> void vec(std::vector<T>& v) {
        const uint64_t n = get<uint64_t>();
        if (!ok || n > left / sizeof(T)) { ok = false; v.clear(); return; }
        v.resize((size_t)n);
        if (n) std::memcpy(v.data(), p, sizeof(T) * (size_t)n);
        p += sizeof(T) * (size_t)n;
        left -= sizeof(T) * (size_t)n;
    }
    void csr(Csr& c) { c.nrows = get<int32_t>(); c.ncols = get<int32_t>(); vec(c.ptr); vec(c.idx); vec(c.val); }
};

// CSR structure: rows + 1 non-decreasing pointers from 0 to nnz, columns below ncols.
bool csr_valid(const Csr& c) {
    if (c.nrows < 0 || c.ncols < 0 || c.ptr.size() != (size_t)c.nrows + 1 || c.ptr[0] != 0) return false;
    for (int32_t i = 0; i < c.nrows; ++i)
        if (c.ptr[i + 1] < c.ptr[i]) return false;
    if ((size_t)c.ptr[c.nrows] != c.idx.size() || c.idx.size() != c.val.size()) return false;
    for (uint32_t j : c.idx)
        if ((int64_t)j >= c.ncols) return false;
    return true;
}
template <typename I> bool ptr_valid(const std::vector<I>& ptr, size_t rows, size_t total) {
    if (ptr.size() != rows + 1 || ptr[0] != 0) return false;
    for (size_t i = 0; i < rows; ++i)
        if (ptr[i + 1] < ptr[i]) return false;
    return (size_t)ptr[rows] == total;
}
template <typename I> bool all_below(const std::vector<I>& v, int64_t bound) {
    for (I x : v)
        if ((int64_t)x < 0 || (int64_t)x >= bound) return false;
    return true;
}

// Everything the device layout is built from (build_stage) indexes within its arrays.
std::string subdomain_invalid(const Subdomain& sd, int64_t ndofs) {
    const int64_t nq = sd.ct.c.nrows, nr = sd.ct.c.ncols;
    if (sd.q < 0 || sd.r <= sd.q || sd.r >= 64) return "factor pair";
    if (!csr_valid(sd.ct.c) || !csr_valid(sd.ct.ct) || sd.ct.ct.nrows != nr || sd.ct.ct.ncols != nq)
        return "cross-tab structure";
    if (sd.ct.c.idx.size() != sd.ct.ct.idx.size()) return "cross-tab transpose size";
    if ((int64_t)sd.gidx.size() != nq + nr || !all_below(sd.gidx, ndofs)) return "global indices";
    if (!sd.pou.empty() && (int64_t)sd.pou.size() != nq + nr) return "partition-of-unity weights";
    if ((int64_t)sd.ct.dq.size() != nq || (int64_t)sd.ct.dr.size() != nr) return "cross-tab diagonals";
    const int64_t n_keep = sd.elim_q ? nr : nq, n_elim = sd.elim_q ? nq : nr;
    if ((int64_t)sd.inv_diag.size() != n_elim) return "eliminated-block diagonal";
    if (sd.n_red != n_keep) return "reduced size";
    if (sd.kind == 0) {
        const int64_t m1 = n_keep >= 1 ? n_keep - 1 : 0;
        if ((int64_t)sd.L.size() != m1 * m1) return "dense factor size";
    } else if (sd.kind == 1) {
        const AcFactor& f = sd.ac;
        if (f.n != n_keep || f.nlev < 0 || f.ncol < 0 || f.ncore < 0 || f.ncore > kAcCoreMax) return "factor sizes";
        if (!ptr_valid(f.level_ptr, (size_t)f.nlev, (size_t)f.ncol)) return "factor levels";
        if (f.col_vertex.size() != (size_t)f.ncol || f.col_diag.size() != (size_t)f.ncol || !all_below(f.col_vertex, f.n))
            return "factor columns";
        if (!ptr_valid(f.col_ptr, (size_t)f.ncol, f.col_idx.size()) || f.col_idx.size() != f.col_coef.size() ||
            !all_below(f.col_idx, f.n))
            return "factor entries";
        if (f.core_vertex.size() != (size_t)f.ncore || !all_below(f.core_vertex, f.n) ||
            f.core_z.size() != (size_t)f.ncore * (size_t)f.ncore)
            return "factor core";
    } else {
        return "local solver kind";
    }
    return {};
}

}  // namespace

std::vector<uint8_t> serialize_preconditioner(const PrecondImage& img, const std::vector<Subdomain>& subs) {
    Writer w;
    for (char c : kPcMagic) w.put<char>(c);
    w.put<uint32_t>(kPcVersion);
    w.put<int64_t>(img.ndofs);
    w.put<int32_t>(img.kind);
    w.put<int32_t>(img.reduction);
    w.put<uint64_t>(img.cfg.ac_seed);
    w.put<uint32_t>(img.cfg.ac_split);
    w.put<int32_t>(img.cfg.approx_schur ? 1 : 0);
    w.put<uint64_t>(img.cfg.schur_seed);
    w.put<uint32_t>(img.cfg.schur_split);
    w.put<int32_t>(img.cfg.dense_threshold);
    w.put<uint64_t>(subs.size());
    for (const Subdomain& sd : subs) {
        w.put<int32_t>(sd.q); w.put<int32_t>(sd.r); w.put<int32_t>(sd.elim_q ? 1 : 0);
        w.put<int32_t>(sd.kind); w.put<int32_t>(sd.n_red);
        w.vec(sd.gidx); w.vec(sd.pou);
        w.csr(sd.ct.c); w.csr(sd.ct.ct);
        w.vec(sd.ct.dq); w.vec(sd.ct.dr); w.vec(sd.inv_diag); w.vec(sd.L);
        const AcFactor& f = sd.ac;
        w.put<int32_t>(f.n); w.put<int32_t>(f.nlev); w.put<int32_t>(f.ncol); w.put<int32_t>(f.ncore);
        w.vec(f.level_ptr); w.vec(f.col_vertex); w.vec(f.col_ptr); w.vec(f.col_idx);
        w.vec(f.col_diag); w.vec(f.col_coef); w.vec(f.core_vertex); w.vec(f.core_z);
    }
    w.vec(img.g_ptr); w.vec(img.g_idx); w.vec(img.g_val);
    w.put<uint64_t>(fnv1a(w.b.data(), w.b.size()));
    return std::move(w.b);
}

Status deserialize_preconditioner(const uint8_t* data, size_t len, PrecondImage& img) {
    Status st;
    auto bad = [&](const std::string& what) {
        st.code = WITHIN_ERR_INVALID_ARGUMENT;
        st.msg = "failed to deserialize preconditioner: " + what;
        return st;
    };
    if (!data || len < sizeof(kPcMagic) + sizeof(uint32_t) + sizeof(uint64_t)) return bad("too short");
    if (std::memcmp(data, kPcMagic, sizeof(kPcMagic)) != 0) return bad("not a serialized preconditioner");
    uint64_t sum = 0;
    std::memcpy(&sum, data + len - sizeof(uint64_t), sizeof(uint64_t));
    if (sum != fnv1a(data, len - sizeof(uint64_t))) return bad("checksum mismatch (corrupted bytes)");
    Reader r{data + sizeof(kPcMagic), len - sizeof(kPcMagic) - sizeof(uint64_t)};
    if (r.get<uint32_t>() != kPcVersion) return bad("unsupported version");
    img.ndofs = r.get<int64_t>();
    img.kind = r.get<int32_t>();
    img.reduction = r.get<int32_t>();
    img.cfg.kind = img.kind;
    img.cfg.ac_seed = r.get<uint64_t>();
    img.cfg.ac_split = r.get<uint32_t>();
    img.cfg.approx_schur = r.get<int32_t>() != 0;
    img.cfg.schur_seed = r.get<uint64_t>();
    img.cfg.schur_split = r.get<uint32_t>();
    img.cfg.dense_threshold = r.get<int32_t>();
    const uint64_t nsub = r.get<uint64_t>();
    if (!r.ok) return bad("truncated header");
    if (img.ndofs <= 0 || img.ndofs > 0xFFFFFFFFll) return bad("dof count");
    if (img.kind != 1 && img.kind != 2) return bad("preconditioner kind");
    if (img.reduction < 0 || img.reduction > 2) return bad("reduction strategy");
    if (nsub > r.left / 64) return bad("subdomain count");
    img.subs.resize((size_t)nsub);
    for (uint64_t i = 0; i < nsub; ++i) {
        Subdomain& sd = img.subs[i];
        sd.q = r.get<int32_t>(); sd.r = r.get<int32_t>(); sd.elim_q = r.get<int32_t>() != 0;
        sd.kind = r.get<int32_t>(); sd.n_red = r.get<int32_t>();
        r.vec(sd.gidx); r.vec(sd.pou);
        r.csr(sd.ct.c); r.csr(sd.ct.ct);
        r.vec(sd.ct.dq); r.vec(sd.ct.dr); r.vec(sd.inv_diag); r.vec(sd.L);
        AcFactor& f = sd.ac;
        f.n = r.get<int32_t>(); f.nlev = r.get<int32_t>(); f.ncol = r.get<int32_t>(); f.ncore = r.get<int32_t>();
        r.vec(f.level_ptr); r.vec(f.col_vertex); r.vec(f.col_ptr); r.vec(f.col_idx);
        r.vec(f.col_diag); r.vec(f.col_coef); r.vec(f.core_vertex); r.vec(f.core_z);
        if (!r.ok) return bad("truncated subdomain " + std::to_string(i));
        const std::string why = subdomain_invalid(sd, img.ndofs);
        if (!why.empty()) return bad("subdomain " + std::to_string(i) + ": " + why);
    }
    r.vec(img.g_ptr); r.vec(img.g_idx); r.vec(img.g_val);
    if (!r.ok || r.left != 0) return bad("trailing or truncated data");
    if (img.kind == 2) {
        if (!ptr_valid(img.g_ptr, (size_t)img.ndofs, img.g_idx.size()) || img.g_idx.size() != img.g_val.size() ||
            !all_below(img.g_idx, img.ndofs))
            return bad("explicit Gramian");
    } else if (!img.g_ptr.empty() || !img.g_idx.empty() || !img.g_val.empty()) {
        return bad("explicit Gramian of an additive preconditioner");
    }
    return st;
}

// A subdomain's local solve goes inner-parallel in the reference only when its larger
// side has more rows than both parallel thresholds (PAR_BACKSUB_THRESHOLD,
// local_solver.rs:78, and PAR_SPMV_THRESHOLD, csr_block.rs:4: 10,000 each); its work is
// then two passes over the cross block plus the local vector.
int64_t inner_parallel_work(const Subdomain& sd) {
    constexpr int32_t kParThreshold = 10000;
    if (std::max(sd.n_q(), sd.n_r()) <= kParThreshold) return 0;
    return 2 * sd.ct.c.nnz() + sd.n_local();
}

AdditiveDiagnostics additive_diagnostics(const std::vector<Subdomain>& subs, int64_t n_dofs, int32_t configured,
                                         int64_t threads) {
    // AdditiveScheduler constants (planning.rs:213-218)
    constexpr int64_t kMinInnerWork = 200000;
    constexpr double kOuterCapacityTarget = 0.75, kSweepFactor = 1.1, kInnerSweepFactor = 6.0, kOverlap = 4.0;
    AdditiveDiagnostics g;
    g.configured = configured;
    g.n_subdomains = (int64_t)subs.size();
    g.n_dofs = n_dofs;
    for (const Subdomain& sd : subs) {  // from_entries (planning.rs:151-172)
        const int64_t w = inner_parallel_work(sd);
        g.total_inner_work += w;
        g.max_inner_work = std::max(g.max_inner_work, w);
        g.total_scatter_dofs += (int64_t)sd.gidx.size();
    }
    g.outer_parallel_capacity = g.max_inner_work == 0 ? 0.0 : (double)g.total_inner_work / (double)g.max_inner_work;
    g.scatter_overlap = (double)g.total_scatter_dofs / (double)std::max<int64_t>(n_dofs, 1);
    threads = std::max<int64_t>(threads, 1);
    // allow_inner_parallelism (planning.rs:84-90)
    const bool inner = g.max_inner_work >= kMinInnerWork && g.outer_parallel_capacity < (double)threads * kOuterCapacityTarget;
    if (configured == 1 || configured == 2) {
        g.resolved = configured;
    } else {  // pick_auto_strategy, reduction_sweep_to_scatter (planning.rs:105-135)
        const int64_t active = std::max<int64_t>(std::min<int64_t>(threads, g.n_subdomains), 1);
        const double ratio = (double)(active * n_dofs) / (double)std::max<int64_t>(g.total_scatter_dofs, 1);
        if (ratio <= kSweepFactor || (inner && ratio <= kInnerSweepFactor) || g.scatter_overlap >= kOverlap)
            g.resolved = 2;
        else
            g.resolved = 1;
    }
    return g;
}

}  // namespace wb
