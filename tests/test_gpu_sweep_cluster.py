"""The small trailing levels of the approximate-Cholesky sweeps in one thread-block cluster.

The reference solves an approximate-Cholesky factor sequentially
(approx_chol::Factor::solve_in_place, called from operator/local_solver.rs:182-198); here
each elimination round is one level of a level-scheduled sweep.  The large levels run in
a cooperative grid launch with grid barriers between them; the trailing run of small
levels runs in one cluster launch with the cluster's hardware barrier between them.  The
arithmetic and its order are the same either way, so the preconditioner apply and the
solve agree with the all-grid form (to the rounding that the subdomain atomics leave) and
with the oracle.
"""
import numpy as np
import pytest

import oracle
import within_b200 as wb
from within_b200 import _lib, synthetic
from paritylib import rel

pytestmark = pytest.mark.gpu


def _designs():
    # 5000 x 3000 uniform levels: 17 elimination rounds on the kept side, several small;
    # default limit of 512 row pieces per cluster level
    yield "uniform", synthetic.uniform_design(60_000, [5000, 3000], seed=21), None, 512
    # the worker-firm-year panel at a fifth of its size (4 rounds of 11765, 2264, 721 and
    # 343 firms): the last three in the cluster
    cats, _, w = synthetic.config3(seed=4, scale=0.2)
    yield "panel", cats, w, 4096


@pytest.mark.parametrize("which", ["uniform", "panel"])
def test_cluster_levels_match_grid_levels_and_oracle(which):
    name, cats, w, chunks = next(d for d in _designs() if d[0] == which)
    L = _lib.load()
    s = wb.Solver(cats, wb.CG(), weights=w)
    p = s.preconditioner()
    rng = np.random.default_rng(5)
    r = rng.standard_normal(s.n_dofs)
    y = rng.standard_normal(cats.shape[0])

    assert L.within_solver_set_sweep_cluster(s._h, 0) == 0, _lib.last_error()
    n0 = L.within_solver_gpu_launches(s._h)
    z_grid = p.apply(r)
    launches_grid = L.within_solver_gpu_launches(s._h) - n0
    res_grid = s.solve(y)

    assert L.within_solver_set_sweep_cluster(s._h, chunks) == 0, _lib.last_error()
    n0 = L.within_solver_gpu_launches(s._h)
    z_cl = p.apply(r)
    launches_cl = L.within_solver_gpu_launches(s._h) - n0
    res_cl = s.solve(y)

    # the cluster path ran: one more launch per sweep direction that has a small tail
    assert launches_cl > launches_grid
    assert rel(z_cl, z_grid) < 1e-10
    assert res_cl.converged and res_cl.residual <= 1e-8
    assert rel(res_cl.demeaned, res_grid.demeaned) < 1e-9
    o = oracle.OracleSolver(cats, w)
    assert rel(res_cl.demeaned, o.solve(y).demeaned) < 1e-8
    assert rel(z_cl, o.apply_precond(r)) < 1e-10
