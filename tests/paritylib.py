"""Helpers shared by the GPU parity tests."""
import numpy as np
import scipy.sparse as sp
from scipy.sparse.csgraph import connected_components


def normalize_x(cats, x):
    """x modulo the null space of G: in every connected component of the level graph,
    each factor q >= 1 is centred and its mean moved onto factor 0 (D x is unchanged)."""
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
    x = np.asarray(x, dtype=np.float64).copy()
    fac = np.concatenate([np.full(nlev[q], q) for q in range(Q)])
    for q in range(1, Q):
        sel = (fac == q) & active
        sums = np.bincount(lab[sel], weights=x[sel], minlength=ncomp)
        cnt = np.bincount(lab[sel], minlength=ncomp)
        mean = np.where(cnt > 0, sums / np.maximum(cnt, 1), 0.0)
        x[sel] -= mean[lab[sel]]
        s0 = (fac == 0) & active
        x[s0] += mean[lab[s0]]
    x[~active] = 0.0
    return x


def rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))
