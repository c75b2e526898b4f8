"""Mixed-precision refinement (solver.rs:296-347 with FP32 inner solves): a check after
the first correction computes D'W(y - D x) with the demeaned e = y - D x, and when it
ends the loop it is also the final demeaning.  Whatever ends the loop (tolerance met,
corrections or inner iterations exhausted), the returned x, demeaned and
final_residual must describe one and the same solution."""
import numpy as np
import pytest

import oracle
import within_b200 as wb
from within_b200 import synthetic
from paritylib import rel

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("maxiter,max_refinements", [(1000, 2), (1000, 0), (3, 0), (3, 2), (2, 6)])
def test_mixed_outputs_describe_one_solution(maxiter, max_refinements):
    cats = synthetic.uniform_design(80_000, [900, 300, 25], seed=1)
    w = np.random.default_rng(5).lognormal(0, 1, 80_000)
    Y = np.asfortranarray(np.random.default_rng(7).standard_normal((cats.shape[0], 5)))
    s = wb.Solver(cats, wb.CG(precision="mixed", maxiter=maxiter, max_refinements=max_refinements), weights=w)
    r = s.solve_batch(Y)
    o = oracle.OracleSolver(cats, w)
    for c in range(Y.shape[1]):
        e = Y[:, c] - o.matvec_d(r.x[:, c])
        # tolerance 1e-10 relative: FP64 demeaning of the returned x against the oracle's
        assert rel(r.demeaned[:, c], e) < 1e-10
        fr = np.linalg.norm(o.rmatvec_wdt(e)) / np.linalg.norm(o.rmatvec_wdt(Y[:, c]))
        # the reported residual is ||D'W e|| / ||D'W y|| of that same e, to 1e-6 relative
        # (it is a difference of nearly equal sums when the solve has converged)
        assert abs(r.residual[c] - fr) <= 1e-6 * fr + 1e-13
        assert bool(r.converged[c]) == (r.residual[c] <= 1e-8)
    if maxiter >= 1000 and max_refinements >= 2:
        assert all(r.converged)
