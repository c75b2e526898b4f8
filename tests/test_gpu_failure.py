"""Failure path of a local solve on the device, made on the host without a GPU fault.

The reference tests it with a LocalSolver stub that always fails
(schwarz-precond/tests/schwarz.rs:947-1001): Preconditioner::apply then fills z with
NaN, and CG's try_apply ends the solve with LocalSolveFailed (solve/cg.rs:69, 104;
IterativeSolve in within).  Here the failure is a test hook that makes the
approximate-Cholesky sweeps' grid barriers wait for one block more than the grid has,
with a short limit: the waits run out, the device error flag is set, and the launches end
normally.  Afterwards the same solver (and CUDA context) works again.
"""
import numpy as np
import pytest

import oracle
import within_b200 as wb
from within_b200 import _lib, synthetic
from paritylib import rel

pytestmark = pytest.mark.gpu


def _design():
    # 5000 x 3000 uniform levels: the kept side's AC factor has 17 elimination rounds, so
    # the sweeps run as cooperative launches with grid barriers between rounds
    return synthetic.uniform_design(60_000, [5000, 3000], seed=21)


@pytest.mark.parametrize("kind", ["additive", "multiplicative"])
def test_failed_local_solve_gives_nan_apply_and_a_solve_error(kind):
    cats = _design()
    cfg, pre = (wb.CG(), wb.AdditiveSchwarz()) if kind == "additive" else (wb.GMRES(), wb.MultiplicativeSchwarz())
    s = wb.Solver(cats, cfg, preconditioner=pre)
    rng = np.random.default_rng(3)
    r = rng.standard_normal(s.n_dofs)
    y = rng.standard_normal(cats.shape[0])
    p = s.preconditioner()
    z0 = p.apply(r)
    assert np.isfinite(z0).all()
    L = _lib.load()
    assert L.within_solver_inject_sweep_timeout(s._h, 1) == 0, _lib.last_error()
    z = p.apply(r)
    assert np.isnan(z).all()
    with pytest.raises(wb.WithinError) as e:
        s.solve(y)
    assert e.value.code == 8 and "local solve failed" in str(e.value)
    assert L.within_solver_inject_sweep_timeout(s._h, 0) == 0
    # the solver and the context are usable again
    assert rel(p.apply(r), z0) < 1e-10
    res = s.solve(y)
    assert res.converged and res.residual <= 1e-8
    o = oracle.OracleSolver(cats, None, krylov="cg" if kind == "additive" else "gmres", preconditioner=kind).solve(y)
    assert rel(res.demeaned, o.demeaned) < 1e-8


def test_injection_needs_fused_sweeps():
    cats = synthetic.uniform_design(3_000, [30, 20], seed=2)  # dense core only: no sweep levels
    s = wb.Solver(cats)
    assert _lib.load().within_solver_inject_sweep_timeout(s._h, 1) == 9
