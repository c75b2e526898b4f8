"""CPU oracle of the learned coarse space: the message-passing network, its loss against
Ritz-vector targets, and its gradients (numpy, FP64 arithmetic with the device's BF16
roundings emulated).

TEST INFRASTRUCTURE ONLY: imported by the tests and the training script's gradient
check, never by the ``within_b200`` package.  There is no counterpart in the
reference: the coarse space augments its additive Schwarz preconditioner
(schwarz-precond/src/schwarz/additive/executor.rs:59-147) inside its CG
(schwarz-precond/src/solve/cg.rs:45-133).

The network, on the level graph of a design (one node per level of every factor; the
edge weight between two levels is the weighted count of the observations that carry
both, i.e. the off-diagonal of G = D'WD):

    d = diag(G),  Ahat h = D^-1/2 (G - diag(G)) D^-1/2 h     (0 on unobserved levels)
    X  = features (m x 16): one-hot of min(factor, 3), log1p(d)/8, log1p(count)/8,
         10 probe channels of +-1 from a splitmix64 hash of (level, channel)
    for l = 0, 1, 2:   S_l = [Ahat H_l, H_l];  H_{l+1} = tanh(bf16(S_l) @ bf16(W_l) + b_l)
    Zt = bf16(H_3) @ bf16(W_o)     (m x 32, in the D^1/2-scaled space; Z = D^-1/2 Zt)

Loss against targets Vt (m x t, orthonormal columns in the scaled space):
    A = Zt'Zt + eps I,  B = Zt'Vt,  L = 1 - tr(B' A^-1 B) / t
the fraction of the targets' energy outside span(Zt).
"""
from __future__ import annotations

import numpy as np
import scipy.sparse as sp

F_IN, HIDDEN, K_OUT, N_LAYERS = 16, 64, 32, 3
N_PROBE = 10
_M64 = (1 << 64) - 1


def bf16(a):
    """Round to BF16 (round to nearest even) and back to float64."""
    f = np.asarray(a, dtype=np.float32)
    b = f.view(np.uint32).astype(np.uint64)
    b = (b + 0x7FFF + ((b >> 16) & 1)) & 0xFFFF0000
    return b.astype(np.uint32).view(np.float32).astype(np.float64)


def probe_sign(level, channel, seed=0):
    """+-1 from the splitmix64 finalizer of level * 64 + channel (+ seed)."""
    z = (np.asarray(level, dtype=np.uint64) * np.uint64(64) + np.uint64(channel)
         + np.uint64((0x9E3779B97F4A7C15 * (seed + 1)) & _M64))
    with np.errstate(over="ignore"):
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        z = z ^ (z >> np.uint64(31))
    return np.where((z & np.uint64(1)) == 1, 1.0, -1.0)


class Design:
    """Level graph of a design: G = D'WD as a sparse matrix, its diagonal and counts."""

    def __init__(self, cats, weights=None):
        cats = np.asarray(cats)
        n, Q = cats.shape
        self.nlev = cats.max(axis=0).astype(np.int64) + 1
        self.off = np.concatenate([[0], np.cumsum(self.nlev)[:-1]]).astype(np.int64)
        self.m = int(self.nlev.sum())
        w = np.ones(n) if weights is None else np.asarray(weights, dtype=np.float64)
        lev = np.concatenate([self.off[q] + cats[:, q].astype(np.int64) for q in range(Q)])  # factor-major
        obs = np.tile(np.arange(n), Q)
        Dm = sp.csr_matrix((np.ones(n * Q), (obs, lev)), shape=(n, self.m))
        self.G = (Dm.T @ sp.diags(w) @ Dm).tocsr()
        self.d = self.G.diagonal().copy()
        self.count = np.asarray((Dm.T @ np.ones(n))).ravel()
        self.factor = np.concatenate([np.full(self.nlev[q], q) for q in range(Q)])
        self.isq = np.where(self.d > 0, 1.0 / np.sqrt(np.where(self.d > 0, self.d, 1.0)), 0.0)

    def ahat(self, H):
        """D^-1/2 (G - diag G) D^-1/2 H."""
        S = self.isq[:, None] * H
        return self.isq[:, None] * (self.G @ S - self.d[:, None] * S)

    def features(self, seed=0):
        X = np.zeros((self.m, F_IN))
        X[np.arange(self.m), np.minimum(self.factor, 3)] = 1.0
        X[:, 4] = np.log1p(self.d) / 8.0
        X[:, 5] = np.log1p(self.count) / 8.0
        lev = np.arange(self.m)
        for c in range(N_PROBE):
            X[:, 6 + c] = probe_sign(lev, c, seed)
        return X.astype(np.float32).astype(np.float64)


def init_params(seed=0):
    """Glorot-uniform weights (FP32 masters), zero biases."""
    rng = np.random.default_rng(seed)
    P = {}
    fin = F_IN
    for l in range(N_LAYERS):
        lim = np.sqrt(6.0 / (2 * fin + HIDDEN))
        P[f"W{l}"] = rng.uniform(-lim, lim, (2 * fin, HIDDEN)).astype(np.float32)
        P[f"b{l}"] = np.zeros(HIDDEN, np.float32)
        fin = HIDDEN
    lim = np.sqrt(6.0 / (HIDDEN + K_OUT))
    P["Wo"] = rng.uniform(-lim, lim, (HIDDEN, K_OUT)).astype(np.float32)
    return P


PARAM_ORDER = [f"{p}{l}" for l in range(N_LAYERS) for p in ("W", "b")] + ["Wo"]


def flatten(P):
    return np.concatenate([np.asarray(P[k], np.float32).ravel() for k in PARAM_ORDER])


def unflatten(v):
    P, o = {}, 0
    fin = F_IN
    for l in range(N_LAYERS):
        P[f"W{l}"] = v[o:o + 2 * fin * HIDDEN].reshape(2 * fin, HIDDEN); o += 2 * fin * HIDDEN
        P[f"b{l}"] = v[o:o + HIDDEN]; o += HIDDEN
        fin = HIDDEN
    P["Wo"] = v[o:o + HIDDEN * K_OUT].reshape(HIDDEN, K_OUT); o += HIDDEN * K_OUT
    assert o == v.size
    return P


def forward(P, design, X):
    """Zt and the cache of the backward pass."""
    H = X
    cache = []
    for l in range(N_LAYERS):
        S = np.hstack([design.ahat(H), H])
        Sb = bf16(S)
        pre = Sb @ bf16(P[f"W{l}"]) + np.asarray(P[f"b{l}"], np.float64)
        Hn = np.tanh(pre)
        cache.append((H, Sb, Hn))
        H = Hn
    Hb = bf16(H)
    Z = Hb @ bf16(P["Wo"])
    cache.append(Hb)
    return Z, cache


def loss_and_grad_z(Z, V, eps_rel=1e-6):
    """L = 1 - tr(B'A^-1 B)/t and dL/dZ, A = Z'Z + eps I, B = Z'V."""
    t = V.shape[1]
    A = Z.T @ Z
    A = A + eps_rel * np.trace(A) / A.shape[0] * np.eye(A.shape[0])
    B = Z.T @ V
    Ai = np.linalg.inv(A)
    AiB = Ai @ B
    L = 1.0 - np.trace(B.T @ AiB) / t
    # d tr(B'A^-1B) = 2 tr(dZ' V B'A^-1) - 2 tr(dZ' Z A^-1 B B' A^-1)
    C1 = AiB.T                    # t x k:  B'A^-1
    C2 = AiB @ AiB.T              # k x k:  A^-1 B B' A^-1
    dZ = -(2.0 / t) * (V @ C1 - Z @ C2)
    return L, dZ, C1, C2


def backward(P, design, cache, dZ):
    """Gradients of every parameter (FP64) from dL/dZt."""
    g = {}
    Hb = cache[-1]
    g["Wo"] = Hb.T @ dZ
    dH = dZ @ bf16(P["Wo"]).T
    for l in reversed(range(N_LAYERS)):
        H, Sb, Hn = cache[l]
        dpre = dH * (1.0 - Hn * Hn)
        g[f"W{l}"] = Sb.T @ dpre
        g[f"b{l}"] = dpre.sum(axis=0)
        if l == 0:
            break
        dS = dpre @ bf16(P[f"W{l}"]).T
        f = H.shape[1]
        dH = dS[:, f:] + design.ahat(dS[:, :f])
    return g


def loss(P, design, X, V):
    Z, _ = forward(P, design, X)
    return loss_and_grad_z(Z, V)[0]


def ritz_targets(design, Mf, steps=80, nev=32, seed=0):
    """The nev lowest Ritz vectors of M^-1 G (Lanczos with full reorthogonalization,
    M^-1 = Mf) outside the null space, in the scaled space (D^1/2 v), orthonormalized."""
    m = design.m
    rng = np.random.default_rng(seed)
    Gf = lambda v: design.G @ v
    r = rng.standard_normal(m)
    z = Mf(r)
    bn = np.sqrt(r @ z)
    r, z = r / bn, z / bn
    R, Zs, al, be = [], [], [], []
    r_prev, beta = np.zeros(m), 0.0
    for _ in range(steps):
        R.append(r); Zs.append(z)
        w = Gf(z)
        a = w @ z
        w = w - a * r - beta * r_prev
        Rm, Zm = np.array(R), np.array(Zs)
        for _ in range(2):
            w = w - Rm.T @ (Zm @ w)
        zn = Mf(w)
        bnew = np.sqrt(max(w @ zn, 1e-300))
        al.append(a); be.append(bnew)
        r_prev, r, z, beta = r, w / bnew, zn / bnew, bnew
    T = np.diag(al) + np.diag(be[:-1], 1) + np.diag(be[:-1], -1)
    lam, S = np.linalg.eigh(T)
    keep = lam > 1e-8 * lam[-1]
    Y = np.array(Zs).T @ S[:, keep][:, :nev]
    Vt = np.sqrt(design.d)[:, None] * Y
    q, _ = np.linalg.qr(Vt)
    return q, lam[keep][:nev]
