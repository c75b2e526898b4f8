"""OperatorRepr.Explicit: the Krylov operator is the assembled Gramian G (CSR SpMV)
instead of the observation pass (within/src/solver.rs:103-121, 350-360), through the
C ABI, against the CPU oracle."""
import numpy as np
import pytest

import oracle
import within_b200 as wb
from within_b200 import synthetic
from paritylib import normalize_x, rel

pytestmark = pytest.mark.gpu

DESIGNS = {
    # year-like factor with long G rows (split into pieces added atomically)
    "uniform3w": lambda: (synthetic.uniform_design(80_000, [900, 300, 25], seed=1),
                          np.random.default_rng(5).lognormal(0, 1, 80_000)),
    "akm": lambda: synthetic.config2(scale=0.05)[0::2],
    "uniform4w": lambda: (synthetic.uniform_design(50_000, [600, 250, 40, 6], seed=11),
                          np.random.default_rng(6).lognormal(0, 1, 50_000)),
}


def _explicit(cats, w, krylov="cg", precision="fp64", **kw):
    cfg = (wb.CG if krylov == "cg" else wb.GMRES)(operator=wb.OperatorRepr.Explicit, precision=precision)
    return wb.Solver(cats, cfg, weights=w, **kw)


@pytest.mark.parametrize("name", list(DESIGNS))
@pytest.mark.parametrize("k", [1, 5, 16, 32])
def test_explicit_operator_apply(name, k):
    cats, w = DESIGNS[name]()
    g = _explicit(cats, w)
    o = oracle.OracleSolver(cats, w)
    X = np.random.default_rng(k).standard_normal((g.n_dofs, k))
    GX = g.apply_gramian(X)
    for c in range(k):
        # tolerance 1e-13 relative: the CSR rows sum in another order than the oracle
        assert rel(GX[:, c], o.apply_gramian(X[:, c])) < 1e-13


@pytest.mark.parametrize("name", list(DESIGNS))
@pytest.mark.parametrize("krylov,precision", [("cg", "fp64"), ("cg", "mixed"), ("gmres", "fp64")])
def test_explicit_solve_matches_oracle(name, krylov, precision):
    cats, w = DESIGNS[name]()
    y = np.random.default_rng(11).standard_normal(cats.shape[0])
    g = _explicit(cats, w, krylov, precision).solve(y)
    o = oracle.OracleSolver(cats, w, krylov=krylov).solve(y)
    assert g.converged and g.residual <= 1e-8
    assert abs(g.iterations - o.iterations) <= 2
    # tolerance 1e-8 relative (demeaned) against the oracle at the same tol
    assert rel(g.demeaned, o.demeaned) < 1e-8
    assert rel(normalize_x(cats, g.x), normalize_x(cats, o.x)) < 1e-6


def test_explicit_batch_equals_implicit():
    cats, w = DESIGNS["uniform3w"]()
    Y = np.asfortranarray(np.random.default_rng(3).standard_normal((cats.shape[0], 16)))
    e = _explicit(cats, w, precision="mixed").solve_batch(Y)
    i = wb.Solver(cats, wb.CG(precision="mixed"), weights=w).solve_batch(Y)
    assert all(e.converged) and max(e.residual) <= 1e-8
    for c in range(16):
        assert rel(e.demeaned[:, c], i.demeaned[:, c]) < 1e-7


def test_explicit_without_preconditioner():
    cats = synthetic.uniform_design(60_000, [500, 200], seed=0)
    y = np.random.default_rng(2).standard_normal(cats.shape[0])
    g = _explicit(cats, None, preconditioner=wb.Preconditioner.Off).solve(y)
    o = oracle.OracleSolver(cats, None, preconditioner="off").solve(y)
    assert g.converged and o.converged
    assert rel(g.demeaned, o.demeaned) < 1e-7
