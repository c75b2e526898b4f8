"""Helpers shared by the GPU parity tests (and the accuracy report of bench.py)."""
import numpy as np
import scipy.sparse as sp
from scipy.sparse.csgraph import connected_components


def make_normalizer(cats):
    """A function x -> x modulo the null space of G: in every connected component of the
    level graph, each factor q >= 1 is centred and its mean moved onto factor 0 (D x is
    unchanged).  The component structure is computed once per design."""
    cats = np.asarray(cats)
    n, Q = cats.shape
    nlev = cats.max(axis=0).astype(np.int64) + 1
    off = np.concatenate([[0], np.cumsum(nlev)[:-1]])
    m = int(nlev.sum())
    rows = np.concatenate([off[0] + cats[:, 0].astype(np.int64)] * (Q - 1)) if Q > 1 else np.array([], np.int64)
    cols = np.concatenate([off[q] + cats[:, q].astype(np.int64) for q in range(1, Q)]) if Q > 1 else np.array([], np.int64)
    g = sp.coo_matrix((np.ones(len(rows)), (rows, cols)), shape=(m, m))
    ncomp, lab = connected_components(g, directed=False)
    active = np.zeros(m, bool)
    for q in range(Q):
        active[off[q] + np.unique(cats[:, q])] = True
    fac = np.concatenate([np.full(nlev[q], q) for q in range(Q)])
    sel = [(fac == q) & active for q in range(Q)]
    cnt = [np.bincount(lab[s], minlength=ncomp) for s in sel]

    def normalize(x):
        x = np.asarray(x, dtype=np.float64).copy()
        for q in range(1, Q):
            s = sel[q]
            sums = np.bincount(lab[s], weights=x[s], minlength=ncomp)
            mean = np.where(cnt[q] > 0, sums / np.maximum(cnt[q], 1), 0.0)
            x[s] -= mean[lab[s]]
            x[sel[0]] += mean[lab[sel[0]]]
        x[~active] = 0.0
        return x

    return normalize


def normalize_x(cats, x):
    """x modulo the null space of G (see make_normalizer)."""
    return make_normalizer(cats)(x)


def rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))
