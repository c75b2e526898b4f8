"""AdditiveSchwarzDiagnostics and subdomain_inner_parallel_work.

The reference computes these scheduling metrics from its built subdomains
(schwarz-precond/src/schwarz/additive/planning.rs:141-218,
within/src/operator/local_solver.rs:348-356) and exposes them through
within-py (lib.rs:200-260, 872-881).  The CPU tests pin the oracle's restatement
with answers worked out by hand from the designs; the GPU tests check the C ABI
against the oracle on the same builds.
"""
import numpy as np
import pytest

import oracle
from oracle import additive_diagnostics, inner_parallel_work
from within_b200 import synthetic


def _two_factor(n, a, b, seed):
    rng = np.random.default_rng(seed)
    return np.asfortranarray(np.column_stack([rng.integers(0, a, n), rng.integers(0, b, n)]).astype(np.uint32))


# ---------------------------------------------------------------- CPU: the oracle


def test_reference_diagnostics_case():
    # tests/test_properties.py:302-316: 300 observations, 10 x 10 levels
    cats = _two_factor(300, 10, 10, 5)
    o = oracle.OracleSolver(cats)
    d = o.additive_diagnostics(threads=8)
    assert d["total_inner_parallel_work"] >= 0 and d["total_scatter_dofs"] >= 0
    # one connected pair of 20 levels: no inner work (10 rows <= 10,000), no overlap;
    # one active buffer sweeps 20 dofs for 20 scattered: ParallelReduction
    assert d["n_subdomains"] == 1 and d["total_scatter_dofs"] == 20
    assert d["total_inner_parallel_work"] == 0 and d["outer_parallel_capacity"] == 0.0
    assert d["scatter_overlap"] == 1.0 and d["resolved_reduction_strategy"] == 2
    assert o.subdomain_inner_parallel_work() == [0]


def test_inner_work_of_a_large_pair():
    # 20,000 x 40 levels: the larger side is above 10,000 rows, so the work is
    # 2 nnz(C) + n_local, with nnz(C) = distinct (q, r) pairs and n_local = observed
    # levels (the cross-tab keeps only levels that occur)
    cats = _two_factor(120_000, 20_000, 40, 7)
    o = oracle.OracleSolver(cats)
    nnz = np.unique(cats[:, 0].astype(np.int64) * 40 + cats[:, 1]).size
    n_local = np.unique(cats[:, 0]).size + np.unique(cats[:, 1]).size
    assert n_local < 20_040  # some of the 20,000 levels are never drawn
    assert o.subdomain_inner_parallel_work() == [2 * nnz + n_local]
    d = o.additive_diagnostics(threads=8)
    assert d["max_inner_parallel_work"] == d["total_inner_parallel_work"] == 2 * nnz + n_local
    assert d["outer_parallel_capacity"] == 1.0
    # one subdomain covering every dof once: ratio 1 <= 1.1, ParallelReduction
    assert d["resolved_reduction_strategy"] == 2


def test_auto_rule_branches():
    # planning.rs:105-135 on hand-made inputs
    m = 1000
    # three pairs of a 3-factor design: every dof in two subdomains, 3 threads:
    # ratio 3m / 2m = 1.5 > 1.1, no inner work, overlap 2 < 4: AtomicScatter
    d = additive_diagnostics([0, 0, 0], [700, 700, 600], m, 0, threads=3)
    assert d["scatter_overlap"] == 2.0 and d["resolved_reduction_strategy"] == 1
    # one thread: ratio 1000 / 2000 = 0.5: ParallelReduction
    assert additive_diagnostics([0, 0, 0], [700, 700, 600], m, 0, threads=1)["resolved_reduction_strategy"] == 2
    # inner parallelism allowed (max work >= 200k, capacity 1 < 0.75 threads) and ratio <= 6
    d = additive_diagnostics([300_000, 0], [1000, 1000], 1000, 0, threads=4)
    assert d["outer_parallel_capacity"] == 1.0 and d["resolved_reduction_strategy"] == 2
    # the same with capacity 2 >= 0.75 x 2 threads: no inner parallelism, ratio 1: still <= 1.1
    d = additive_diagnostics([300_000, 300_000], [1000, 1000], 1000, 0, threads=2)
    assert d["resolved_reduction_strategy"] == 2
    # overlap >= 4 forces ParallelReduction even with many threads
    d = additive_diagnostics([0] * 8, [500] * 8, 1000, 0, threads=64)
    assert d["scatter_overlap"] == 4.0 and d["resolved_reduction_strategy"] == 2
    # configured strategies are kept as they are
    for s in (1, 2):
        assert additive_diagnostics([0], [10], 10, s, threads=8)["resolved_reduction_strategy"] == s
    assert inner_parallel_work(10_000, 5, 50) == 0 and inner_parallel_work(10_001, 5, 50) == 100 + 10_006


# ------------------------------------------------------ GPU: the C ABI vs the oracle

DESIGNS = {
    "small": lambda: (_two_factor(300, 10, 10, 5), None),
    "large_pair": lambda: (_two_factor(120_000, 20_000, 40, 7), None),
    "akm_w": lambda: (lambda c, Y, w: (c, w))(*synthetic.config2(scale=0.1)),
    "three_factor": lambda: (synthetic.uniform_design(60_000, [15_000, 800, 30], seed=3), None),
}


@pytest.mark.gpu
@pytest.mark.parametrize("name", list(DESIGNS))
@pytest.mark.parametrize("strategy", [0, 1, 2])
def test_diagnostics_match_oracle(name, strategy):
    import ctypes as C

    import within_b200 as wb
    from within_b200 import _lib

    cats, w = DESIGNS[name]()
    s = wb.Solver(cats, weights=w, preconditioner=wb.AdditiveSchwarz(reduction=wb.ReductionStrategy(strategy)))
    o = oracle.OracleSolver(cats, w)
    p = s.preconditioner()
    assert p.subdomain_inner_parallel_work == o.subdomain_inner_parallel_work()
    for threads in (1, 8, 64):
        d = _lib.AdditiveDiagnostics()
        assert _lib.load().within_solver_additive_diagnostics(s._h, threads, C.byref(d)) == 0
        e = o.additive_diagnostics(configured=strategy, threads=threads)
        for key, v in e.items():
            assert getattr(d, key) == v, (key, threads)
    d = p.additive_schwarz_diagnostics()
    assert d.reduction_strategy == wb.ReductionStrategy(strategy)
    assert isinstance(d.resolved_reduction_strategy, wb.ReductionStrategy)
    assert repr(d).startswith("AdditiveSchwarzDiagnostics(reduction_strategy=")


@pytest.mark.gpu
def test_diagnostics_only_for_additive():
    import within_b200 as wb

    cats = _two_factor(300, 10, 10, 5)
    s = wb.Solver(cats, wb.GMRES(), preconditioner=wb.Preconditioner.Multiplicative)
    p = s.preconditioner()
    assert p.additive_schwarz_diagnostics() is None
    assert p.subdomain_inner_parallel_work == [0]
    assert wb.Solver(cats, preconditioner=wb.Preconditioner.Off).preconditioner() is None
