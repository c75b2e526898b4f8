"""Seeded synthetic fixed-effects designs with the shapes of the reference's benchmarks.

No public dataset is used by the reference's benchmarks; these generators stand in
for them.  The worker-firm-year panel follows the reference's AKM generator
(benchmarks/_problems.py:417-539): Zipf(1.1) firm sizes (weights rank^-1.1) and a
per-year switch to a Zipf-drawn firm with probability p; year codes are a
consecutive window per worker.
"""
from __future__ import annotations

import numpy as np


def uniform_design(n_obs: int, n_levels, seed: int = 0):
    """Codes uniform on [0, L_q) per factor, Fortran-ordered uint32 (n_obs, Q)."""
    rng = np.random.default_rng(seed)
    cols = [rng.integers(0, L, size=n_obs, dtype=np.uint32) for L in n_levels]
    return np.asfortranarray(np.column_stack(cols).astype(np.uint32))


def worker_firm_year(n_workers: int, n_firms: int, years_per_worker: int, n_years: int,
                     switch_prob: float, seed: int = 0, zipf_s: float = 1.1):
    """Worker-firm-year panel: returns (categories (n,3) F-order uint32, fe values dict).

    Observations are worker-major (each worker's consecutive years together).
    """
    rng = np.random.default_rng(seed)
    W, T = n_workers, years_per_worker
    p_firm = np.arange(1, n_firms + 1, dtype=np.float64) ** (-zipf_s)
    p_firm /= p_firm.sum()
    cdf = np.cumsum(p_firm)
    cdf[-1] = 1.0

    def draw(k):
        return np.searchsorted(cdf, rng.random(k), side="right").astype(np.uint32)

    firms = np.empty((W, T), dtype=np.uint32)
    firms[:, 0] = draw(W)
    for t in range(1, T):
        sw = rng.random(W) < switch_prob
        firms[:, t] = firms[:, t - 1]
        ns = int(sw.sum())
        if ns:
            firms[sw, t] = draw(ns)
    max_start = max(n_years - T, 0)
    start = rng.integers(0, max_start + 1, size=W, dtype=np.uint32) if max_start > 0 else np.zeros(W, np.uint32)
    years = (start[:, None] + np.arange(T, dtype=np.uint32)[None, :]).astype(np.uint32)
    workers = np.repeat(np.arange(W, dtype=np.uint32), T)
    cats = np.asfortranarray(np.column_stack([workers, firms.ravel(), years.ravel()]).astype(np.uint32))
    return cats


def akm_panel(n_workers: int, n_firms: int, years_per_worker: int, n_years: int,
              switch_prob: float, n_x: int, weighted: bool, seed: int = 0):
    """Panel plus responses: y = worker_fe + firm_fe + year_fe + N(0,1) and n_x N(0,1) columns.

    Returns (categories, Y (n, 1+n_x) F-order float64, weights or None).
    """
    cats = worker_firm_year(n_workers, n_firms, years_per_worker, n_years, switch_prob, seed)
    rng = np.random.default_rng(seed + 1)
    n = cats.shape[0]
    fe_w = rng.standard_normal(n_workers)
    fe_f = rng.standard_normal(n_firms)
    fe_y = rng.standard_normal(n_years)
    Y = np.empty((n, 1 + n_x), order="F")
    Y[:, 0] = fe_w[cats[:, 0]] + fe_f[cats[:, 1]] + fe_y[cats[:, 2]] + rng.standard_normal(n)
    for j in range(n_x):
        Y[:, 1 + j] = rng.standard_normal(n)
    w = rng.lognormal(0.0, 1.0, size=n) if weighted else None
    return cats, Y, w


# Named workloads (sizes of the five benchmark configurations).
def config1(seed: int = 0):
    """100k obs, codes U[0,500) x U[0,200), y ~ N(0,1), unit weights."""
    cats = uniform_design(100_000, [500, 200], seed)
    y = np.random.default_rng(seed + 1).standard_normal(100_000)
    return cats, y[:, None].copy(order="F"), None


def config2(seed: int = 0, scale: float = 1.0):
    """200k workers x 10 years, 20k Zipf(1.1) firms, p_switch 0.1, 20 years, 9 RHS."""
    W = max(int(200_000 * scale), 10)
    F = max(int(20_000 * scale), 5)
    return akm_panel(W, F, 10, 20, 0.1, 8, False, seed)


def config3(seed: int = 0, scale: float = 1.0):
    """500k workers x 20 years (10M obs), 100k Zipf(1.1) firms, lognormal weights, 16 RHS."""
    W = max(int(500_000 * scale), 10)
    F = max(int(100_000 * scale), 5)
    return akm_panel(W, F, 20, 20, 0.1, 15, True, seed)


def config4(seed: int = 0, n_problems: int = 256, max_obs: int = 1_000_000):
    """Uneven batch: n_problems independent designs, n_obs log-uniform on [1e3, max_obs],
    2-4 factors with level counts log-uniform on [n/50, n/5] and uniform codes, 1-8
    N(0,1) right-hand sides each.  Returns a list of (categories, Y)."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n_problems):
        n = int(np.exp(rng.uniform(np.log(1e3), np.log(max_obs))))
        q = int(rng.integers(2, 5))
        lv = [max(2, int(np.exp(rng.uniform(np.log(n / 50), np.log(n / 5))))) for _ in range(q)]
        cats = uniform_design(n, lv, seed=int(rng.integers(0, 2**31)))
        k = int(rng.integers(1, 9))
        Y = np.asfortranarray(rng.standard_normal((n, k)))
        out.append((cats, Y))
    return out
