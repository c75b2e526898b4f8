"""Parity at the stated sizes of the benchmark configurations 1 and 2, against the CPU
oracle at the same tolerance and at tol 1e-13 (the "truth").

Criteria (relative 2-norm errors):
- FP64, the drop-in, runs the reference's algorithm: its demeaned residuals and its x
  (after removing the null-space shift) are within 1e-8 of the oracle's at tol 1e-8.
- Mixed precision runs a different iteration to the same tolerance, so it cannot track
  the oracle's iterates.  The reference's own solve at tol 1e-8 is itself up to ~1e-7
  away from the tol-1e-13 solution on these designs (7.4e-8 on config 2's first RHS),
  so the bar is accuracy: its error against the truth is at most twice the oracle's own
  (demeaned residuals and x), plus 1e-9.  (It refines to 0.3 x the tolerance, which on
  these designs puts it below the oracle's error on most RHS.)
"""
import numpy as np
import pytest

import oracle
import within_b200 as wb
from within_b200 import synthetic
from paritylib import make_normalizer, rel

pytestmark = pytest.mark.gpu


def _check(cats, w, Y, g, o, truth, precision):
    NZ = make_normalizer(cats)
    k = Y.shape[1]
    assert all(g.converged) and max(g.residual) <= 1e-8
    for c in range(k):
        if precision == "fp64":
            assert rel(g.demeaned[:, c], o.demeaned[:, c]) < 1e-8
            assert rel(NZ(g.x[:, c]), NZ(o.x[:, c])) < 1e-8
    for c in range(truth.x.shape[1]):
        e_o = rel(o.demeaned[:, c], truth.demeaned[:, c])
        x_o = rel(NZ(o.x[:, c]), NZ(truth.x[:, c]))
        assert rel(g.demeaned[:, c], truth.demeaned[:, c]) <= 2 * e_o + 1e-9
        assert rel(NZ(g.x[:, c]), NZ(truth.x[:, c])) <= 2 * x_o + 1e-9


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("split", [1, 2])
def test_config1_stated_size(split, precision):
    """100k observations, codes U[0,500) x U[0,200), y ~ N(0,1), unit weights, CG tol
    1e-8, AdditiveSchwarz(SchurComplement(ApproxCholConfig(seed=0, split))) with the
    Python class's exact Schur complement (python/within/_within.pyi:490-513); split 1
    as stated, split 2 the Python default."""
    cats, Y, w = synthetic.config1()
    pre = wb.AdditiveSchwarz(local_solver=wb.SchurComplement(approx_chol=wb.ApproxCholConfig(seed=0, split=split)))
    g = wb.Solver(cats, wb.CG(precision=precision), weights=w, preconditioner=pre).solve_batch(Y)
    kw = dict(approx_chol_split=split, approx_schur=None)
    o = oracle.OracleSolver(cats, w, **kw).solve_batch(Y)
    truth = oracle.OracleSolver(cats, w, tol=1e-13, **kw).solve_batch(Y)
    _check(cats, w, Y, g, o, truth, precision)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_config2_stated_size(precision):
    """200k workers x 10 years (2M observations), 20k Zipf(1.1) firms, switch
    probability 0.1, 9 RHS (y and 8 N(0,1) columns), default additive Schwarz."""
    cats, Y, w = synthetic.config2()
    Y = np.asfortranarray(Y)
    g = wb.Solver(cats, wb.CG(precision=precision), weights=w).solve_batch(Y)
    o = oracle.OracleSolver(cats, w).solve_batch(Y)
    truth = oracle.OracleSolver(cats, w, tol=1e-13).solve_batch(Y[:, :3])
    _check(cats, w, Y, g, o, truth, precision)
