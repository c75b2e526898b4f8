"""The FP32 observation pass with wide lanes (8 RHS per lane, a lane group of kp/8 lanes
per observation stream; within_solver_set_obs_config with variant 2 or 3).  The operator
apply G x = D'W D x (the reference's GramianOperator::apply, operator/gramian.rs:84-89,
over domain.rs:312-417) matches the CPU oracle to FP32 rounding and the 4-RHS lanes to
the rounding that the order of the atomic additions leaves, for every block shape and
both forms of the hot-level tables; a mixed-precision solve on it stays within the
oracle's own error."""
import numpy as np
import pytest

import oracle
import within_b200 as wb
from within_b200 import _lib, synthetic
from paritylib import make_normalizer, rel
from test_gpu_parity import DESIGNS

pytestmark = pytest.mark.gpu

# FP32 operator: x and the weights rounded to FP32, sums in FP32
FP32_TOL = 5e-6


def _pin(s, k, per, bps, variant):
    L = _lib.load()
    assert L.within_solver_set_obs_config(s._h, k, 4, per, bps, variant) == 0, L.within_last_error()


@pytest.mark.parametrize("name", ["uniform2", "uniform3w", "akm", "akm_w", "shuffled", "uniform4w"])
@pytest.mark.parametrize("k", [5, 16, 32])
def test_wide_lanes_match_oracle_and_narrow_lanes(name, k):
    cats, w = DESIGNS[name]()
    g = wb.Solver(cats, wb.CG(precision="mixed"), weights=w)
    o = oracle.OracleSolver(cats, w)
    L = _lib.load()
    X = np.random.default_rng(k + 300).standard_normal((g.n_dofs, k))
    want = [o.apply_gramian(X[:, c]) for c in range(k)]
    for per, bps in ((16, 1), (32, 2), (64, 2)):
        for hot in (0, 1):
            _pin(g, k, per, bps, hot)
            narrow = g.apply_gramian(X)
            _pin(g, k, per, bps, 2 + hot)
            assert L.within_solver_obs_rhs_per_lane(g._h, k, 4) == 8
            wide = g.apply_gramian(X)
            for c in range(k):
                assert rel(wide[:, c], want[c]) < FP32_TOL, (per, bps, hot, c)
                assert rel(wide[:, c], narrow[:, c]) < FP32_TOL, (per, bps, hot, c)


def test_wide_lanes_rejected_where_they_do_not_exist():
    L = _lib.load()
    cats, w = DESIGNS["akm"]()
    g = wb.Solver(cats, wb.CG(precision="mixed"), weights=w)
    assert L.within_solver_set_obs_config(g._h, 4, 4, 32, 2, 2) != 0  # 4 RHS: one lane per row already
    assert L.within_solver_set_obs_config(g._h, 16, 8, 32, 2, 2) != 0  # FP64
    assert L.within_solver_set_obs_config(g._h, 16, 4, 32, 2, 4) != 0  # no such variant
    cats5, _ = DESIGNS["uniform5"]()  # 5 factors: generic kernel, no wide form
    g5 = wb.Solver(cats5, wb.CG(precision="mixed"))
    assert L.within_solver_set_obs_config(g5._h, 16, 4, 32, 2, 2) != 0


def test_mixed_solve_with_wide_lanes():
    cats, Y, w = synthetic.config3(scale=0.01)
    s = wb.Solver(cats, wb.CG(precision="mixed"), weights=w)
    _pin(s, 16, 32, 2, 3)
    r = s.solve_batch(Y)
    assert _lib.load().within_solver_obs_rhs_per_lane(s._h, 16, 4) == 8
    assert all(r.converged) and max(r.residual) <= 1e-8
    truth = oracle.OracleSolver(cats, w, tol=1e-13)
    same_tol = oracle.OracleSolver(cats, w)
    NZ = make_normalizer(cats)
    for c in (0, 7, 15):
        t = truth.solve(Y[:, c])
        o = same_tol.solve(Y[:, c])
        assert rel(r.demeaned[:, c], t.demeaned) <= 2 * rel(o.demeaned, t.demeaned) + 1e-9
        assert rel(NZ(r.x[:, c]), NZ(t.x)) <= 2 * rel(NZ(o.x), NZ(t.x)) + 1e-9
