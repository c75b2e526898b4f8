"""LSMR (KrylovMethod::Lsmr; schwarz-precond/src/solve/lsmr.rs) through the C ABI
against the CPU oracle: min ||W^(1/2)(y - D x)||, batched over RHS columns."""
import numpy as np
import pytest

import oracle
import within_b200 as wb
from within_b200 import synthetic
from paritylib import normalize_x, rel

pytestmark = pytest.mark.gpu

DESIGNS = {
    "uniform3w": lambda: (synthetic.uniform_design(80_000, [900, 300, 25], seed=1),
                          np.random.default_rng(5).lognormal(0, 1, 80_000)),
    "akm": lambda: synthetic.config2(scale=0.05)[0::2],
    "uniform4w": lambda: (synthetic.uniform_design(50_000, [600, 250, 40, 6], seed=11),
                          np.random.default_rng(6).lognormal(0, 1, 50_000)),
}


def _pre(kind):
    return None if kind == "additive" else wb.Preconditioner.Off


@pytest.mark.parametrize("name", list(DESIGNS))
@pytest.mark.parametrize("pre", ["additive", "off"])
@pytest.mark.parametrize("local_size", [None, 5])
def test_lsmr_matches_oracle(name, pre, local_size):
    cats, w = DESIGNS[name]()
    y = np.random.default_rng(11).standard_normal(cats.shape[0])
    g = wb.Solver(cats, wb.LSMR(local_size=local_size), weights=w, preconditioner=_pre(pre)).solve(y)
    o = oracle.OracleSolver(cats, w, krylov="lsmr", preconditioner=pre, local_size=local_size).solve(y)
    assert g.converged == o.converged
    # the same recurrences in another summation order: the stop iteration may move by one,
    # and by a few percent over the hundreds of unpreconditioned iterations of a short
    # recurrence (rounding shifts where the stop test first passes)
    assert abs(g.iterations - o.iterations) <= max(1, 0.05 * o.iterations)
    # tolerance: 1e-6 relative on the demeaned residuals against the oracle at the same tol,
    # and the error against the least-squares solution (oracle CG at tol 1e-13) of the
    # oracle's own size
    truth = oracle.OracleSolver(cats, w, tol=1e-13).solve(y)
    err_o = rel(o.demeaned, truth.demeaned)
    assert rel(g.demeaned, o.demeaned) < max(1e-6, 10 * err_o)
    assert rel(g.demeaned, truth.demeaned) < max(10 * err_o, 1e-9)
    if g.iterations == o.iterations:
        assert abs(g.residual - o.residual) <= 1e-3 * o.residual + 1e-14
    xo, xt = normalize_x(cats, o.x), normalize_x(cats, truth.x)
    assert rel(normalize_x(cats, g.x), xo) < max(1e-4, 10 * rel(xo, xt))


def test_lsmr_batch_columns_are_independent():
    cats, w = DESIGNS["uniform3w"]()
    rng = np.random.default_rng(3)
    Y = np.asfortranarray(rng.standard_normal((cats.shape[0], 6)))
    Y[:, 2] = 0.0  # a zero right-hand side stops at iteration 0
    s = wb.Solver(cats, wb.LSMR(), weights=w)
    b = s.solve_batch(Y)
    assert b.converged[2] and b.iterations[2] == 0 and not b.x[:, 2].any()
    o = oracle.OracleSolver(cats, w, krylov="lsmr")
    for c in (0, 1, 3, 5):
        r = o.solve(Y[:, c])
        assert b.converged[c] == r.converged and abs(b.iterations[c] - r.iterations) <= 1
        assert rel(b.demeaned[:, c], r.demeaned) < 1e-6
        one = s.solve(Y[:, c])
        assert one.iterations == b.iterations[c]
        assert rel(b.demeaned[:, c], one.demeaned) < 1e-10


def test_lsmr_maxiter_and_validation():
    cats, w = DESIGNS["akm"]()
    y = np.random.default_rng(4).standard_normal(cats.shape[0])
    r = wb.Solver(cats, wb.LSMR(maxiter=3, tol=1e-14), preconditioner=wb.Preconditioner.Off).solve(y)
    o = oracle.OracleSolver(cats, None, krylov="lsmr", maxiter=3, tol=1e-14, preconditioner="off").solve(y)
    assert not r.converged and r.iterations == 3 == o.iterations
    assert rel(r.demeaned, o.demeaned) < 1e-9
    with pytest.raises(ValueError, match="LSMR requires a symmetric preconditioner"):
        wb.Solver(cats, wb.LSMR(), preconditioner=wb.Preconditioner.Multiplicative)
    # y in the column space of D: the least-squares residual is zero
    oc = oracle.OracleSolver(cats, None)
    yy = oc.matvec_d(np.random.default_rng(5).standard_normal(oc.n_dofs))
    r = wb.Solver(cats, wb.LSMR()).solve(yy)
    assert r.converged and np.abs(r.demeaned).max() < 1e-6 * np.abs(yy).max()
