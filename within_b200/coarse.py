"""Learned coarse space for CG: training targets, training and the shipped network.

The solver's CG preconditioner can be augmented with a coarse space Z (n_dofs x 32):
M^-1 r + Z (Z'GZ)^+ Z' r, which stays symmetric positive semi-definite, so CG keeps its
guarantees and every solve still runs to the same tolerance.  Z comes from a small
message-passing network over the level graph (``within_solver_set_coarse_net``; its
layers are documented in ``include/within_b200.h``), evaluated and differentiated by the
library's own sm_100a kernels.  The reference has no counterpart: the correction
augments its additive Schwarz apply (schwarz-precond/src/schwarz/additive/
executor.rs:59-147) inside its CG (schwarz-precond/src/solve/cg.rs:45-133).

Training targets are the lowest Ritz vectors of the preconditioned operator M^-1 G of
each training design, from a Lanczos run (full reorthogonalization) that uses the
solver's own operator and Schwarz applies on the GPU.  The loss is the fraction of the
targets outside span(Z) in the D^1/2-scaled space (D = diag G); the optimizer is Adam.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import _lib

HERE = os.path.dirname(os.path.abspath(__file__))
WEIGHTS = os.path.join(HERE, "coarse_net_weights.npy")
N_IN, HIDDEN, K_OUT, LAYERS = 16, 64, 32, 3


def n_params() -> int:
    return int(_lib.load().within_coarse_net_params())


def init_params(seed: int = 0) -> np.ndarray:
    """Glorot-uniform weights, zero biases, in the library's parameter order."""
    rng = np.random.default_rng(seed)
    parts = []
    fin = N_IN
    for _ in range(LAYERS):
        lim = np.sqrt(6.0 / (2 * fin + HIDDEN))
        parts += [rng.uniform(-lim, lim, 2 * fin * HIDDEN), np.zeros(HIDDEN)]
        fin = HIDDEN
    lim = np.sqrt(6.0 / (HIDDEN + K_OUT))
    parts.append(rng.uniform(-lim, lim, HIDDEN * K_OUT))
    p = np.concatenate(parts).astype(np.float32)
    assert p.size == n_params()
    return p


class CoarseNet:
    """Parameters of the coarse-space network (FP32) and the probe seed."""

    def __init__(self, params: np.ndarray, seed: int = 0):
        params = np.ascontiguousarray(params, dtype=np.float32)
        if params.size != n_params():
            raise ValueError(f"the coarse-space network has {n_params()} parameters, got {params.size}")
        self.params, self.seed = params, int(seed)

    @classmethod
    def trained(cls) -> "CoarseNet":
        """The network trained by ``train_default`` and shipped with the package."""
        if not os.path.exists(WEIGHTS):
            raise FileNotFoundError(f"{WEIGHTS} is missing; run within_b200.coarse.train_default()")
        return cls(np.load(WEIGHTS), 0)


def level_diagonal(categories, weights=None) -> np.ndarray:
    """diag(G) = the weighted count of every level (n_dofs)."""
    cats = np.asarray(categories)
    nlev = cats.max(axis=0).astype(np.int64) + 1
    off = np.concatenate([[0], np.cumsum(nlev)[:-1]])
    w = np.ones(cats.shape[0]) if weights is None else np.asarray(weights, np.float64)
    return np.concatenate([np.bincount(cats[:, q], weights=w, minlength=nlev[q]) for q in range(cats.shape[1])])


def ritz_targets(solver, diag: np.ndarray, steps: int = 72, nev: int = 32, seed: int = 0):
    """The nev lowest Ritz vectors of M^-1 G outside its null space, from `steps` Lanczos
    steps in the M^-1 inner product with full reorthogonalization (G and M^-1 are the
    solver's own device applies), scaled by D^1/2 and orthonormalized.  Returns the
    targets (n_dofs x t) and the Ritz values."""
    m = solver.n_dofs
    pre = solver.preconditioner()
    rng = np.random.default_rng(seed)
    r = rng.standard_normal(m)
    r -= r.mean()
    z = pre.apply(r)
    bn = np.sqrt(max(r @ z, 1e-300))
    r, z = r / bn, z / bn
    R = np.zeros((steps, m))
    Zs = np.zeros((steps, m))
    al, be = [], []
    r_prev, beta = np.zeros(m), 0.0
    for j in range(steps):
        R[j], Zs[j] = r, z
        w = solver.apply_gramian(z)
        a = float(w @ z)
        w = w - a * r - beta * r_prev
        for _ in range(2):  # full reorthogonalization: w -= R (Z' w)
            w -= R[:j + 1].T @ (Zs[:j + 1] @ w)
        zn = pre.apply(w)
        bnew = float(np.sqrt(max(w @ zn, 1e-300)))
        al.append(a)
        be.append(bnew)
        r_prev, r, z, beta = r, w / bnew, zn / bnew, bnew
    T = np.diag(al) + np.diag(be[:-1], 1) + np.diag(be[:-1], -1)
    lam, S = np.linalg.eigh(T)
    keep = lam > 1e-8 * lam[-1]
    Y = Zs.T @ S[:, keep][:, :nev]
    q, _ = np.linalg.qr(np.sqrt(diag)[:, None] * Y)
    return q, lam[keep][:nev]


def grad(solver, params: np.ndarray, seed: int = 0, want_z: bool = False):
    """Loss and gradient of the network on the solver's design against the targets set
    with ``set_targets`` (device forward and backward passes)."""
    L = _lib.load()
    g = np.empty(params.size, np.float32)
    loss = C.c_double()
    zt = np.empty((solver.n_dofs, K_OUT), np.float32, order="F") if want_z else None
    p = np.ascontiguousarray(params, dtype=np.float32)
    rc = L.within_coarse_net_grad(solver._h, p.ctypes.data_as(C.c_void_p), seed, g.ctypes.data_as(C.c_void_p),
                                  C.byref(loss), None if zt is None else zt.ctypes.data_as(C.c_void_p))
    if rc != 0:
        raise RuntimeError(_lib.last_error())
    return (loss.value, g, zt) if want_z else (loss.value, g)


def set_targets(solver, V: np.ndarray) -> None:
    V = np.asfortranarray(V, dtype=np.float64)
    rc = _lib.load().within_solver_set_coarse_targets(solver._h, V.ctypes.data_as(C.c_void_p), V.shape[1])
    if rc != 0:
        raise RuntimeError(_lib.last_error())


def release_training(solver) -> None:
    _lib.load().within_solver_release_coarse_training(solver._h)


class Adam:
    """Adam (Kingma & Ba 2015) on the FP32 parameter vector."""

    def __init__(self, n, lr=1e-3, b1=0.9, b2=0.999, eps=1e-8):
        self.m1, self.m2 = np.zeros(n), np.zeros(n)
        self.lr, self.b1, self.b2, self.eps, self.t = lr, b1, b2, eps, 0

    def step(self, p, g):
        self.t += 1
        self.m1 = self.b1 * self.m1 + (1 - self.b1) * g
        self.m2 = self.b2 * self.m2 + (1 - self.b2) * g * g
        mh = self.m1 / (1 - self.b1 ** self.t)
        vh = self.m2 / (1 - self.b2 ** self.t)
        return (p - self.lr * mh / (np.sqrt(vh) + self.eps)).astype(np.float32)


def training_designs(n_designs: int, seed: int = 0, min_obs: float = 1e5, max_obs: float = 5e5):
    """Worker-firm-year panels of the benchmark generator: n_obs log-uniform on
    [min_obs, max_obs] (10 years per worker, firms = workers / 10), switch probability
    uniform on [0.01, 0.3], lognormal weights on every other design."""
    from . import synthetic
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n_designs):
        n = float(np.exp(rng.uniform(np.log(min_obs), np.log(max_obs))))
        W = max(int(n / 10), 100)
        p = float(rng.uniform(0.01, 0.3))
        cats = synthetic.worker_firm_year(W, max(W // 10, 10), 10, 20, p, seed=int(rng.integers(0, 2**31)))
        w = rng.lognormal(0.0, 1.0, cats.shape[0]) if i % 2 else None
        out.append((cats, w, p))
    return out


def train(designs, epochs: int = 20, lr: float = 2e-3, seed: int = 0, params=None, log=print, nev: int = 32,
          steps: int = 72):
    """Trains the network on the designs (each: (categories, weights, label)); returns the
    parameters and the per-epoch mean loss."""
    from . import Solver
    solvers = []
    for i, (cats, w, _) in enumerate(designs):
        s = Solver(cats, weights=w)
        V, lam = ritz_targets(s, level_diagonal(cats, w), steps=steps, nev=nev, seed=i)
        set_targets(s, V)
        solvers.append(s)
    p = init_params(seed) if params is None else np.asarray(params, np.float32).copy()
    opt = Adam(p.size, lr=lr)
    rng = np.random.default_rng(seed)
    hist = []
    for ep in range(epochs):
        losses = []
        for i in rng.permutation(len(solvers)):
            loss, g = grad(solvers[i], p, 0)
            losses.append(loss)
            p = opt.step(p, g.astype(np.float64))
        hist.append(float(np.mean(losses)))
        log(f"epoch {ep}: mean loss {hist[-1]:.4f}")
    for s in solvers:
        release_training(s)
    return p, hist


def install_judged(solver, coarse, n_probe: int = 2, seed: int = 0) -> dict:
    """Installs `coarse` (a CoarseNet or a basis) on the solver only if CG with it solves
    probe right-hand sides (seeded N(0,1), n_probe columns) in less time than with plain
    additive Schwarz; otherwise the solver keeps plain Schwarz.  Plain Schwarz is both
    the fallback and the judge: every solve runs to the same tolerance either way.
    Returns the probe measurements and whether the coarse space was kept."""
    import time
    y = np.asfortranarray(np.random.default_rng(seed).standard_normal((solver.n_obs, n_probe)))

    def timed():
        solver.solve_batch(y)  # the first solve captures the CG iteration
        t0 = time.perf_counter()
        r = solver.solve_batch(y)
        return time.perf_counter() - t0, r.iterations

    solver.clear_coarse_space()
    t_plain, it_plain = timed()
    solver.set_coarse_space(coarse)
    t_coarse, it_coarse = timed()
    kept = t_coarse < t_plain
    if not kept:
        solver.clear_coarse_space()
    return {"kept": kept, "plain_s": t_plain, "coarse_s": t_coarse, "plain_iterations": it_plain,
            "coarse_iterations": it_coarse}


def train_default(out: str = WEIGHTS, n_designs: int = 96, epochs: int = 40, log=print):
    """Trains the shipped network: 96 generated worker-firm-year designs (1e5 to 5e5
    observations, switch probability 0.01 to 0.3, seed 2024), 32 Ritz targets each, 40
    epochs of Adam (learning rate 3e-3); saves the parameters to `out`."""
    designs = training_designs(n_designs, seed=2024)
    p, hist = train(designs, epochs=epochs, lr=3e-3, log=log)
    np.save(out, p)
    return p, hist


if __name__ == "__main__":
    import sys
    train_default(sys.argv[1] if len(sys.argv) > 1 else WEIGHTS)
