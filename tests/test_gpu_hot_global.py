"""The observation pass with its hot-level tables in per-block global copies instead of
shared memory (within_solver_set_obs_config with hot_global = 1): the operator apply and
D'W y match the CPU oracle for every block shape on the parity designs, and a
mixed-precision solve on it stays within the oracle's own error."""
import numpy as np
import pytest

import oracle
import within_b200 as wb
from within_b200 import _lib, synthetic
from paritylib import make_normalizer, rel
from test_gpu_parity import DESIGNS

pytestmark = pytest.mark.gpu


def _pin(s, k, elem, per, bps, hot_global):
    L = _lib.load()
    assert L.within_solver_set_obs_config(s._h, k, elem, per, bps, hot_global) == 0, L.within_last_error()


@pytest.mark.parametrize("name", list(DESIGNS))
@pytest.mark.parametrize("k", [1, 5, 16, 32])
def test_global_hot_tables_match_oracle(name, k):
    cats, w = DESIGNS[name]()
    g = wb.Solver(cats, weights=w)
    o = oracle.OracleSolver(cats, w)
    rng = np.random.default_rng(k + 200)
    X = rng.standard_normal((g.n_dofs, k))
    R = rng.standard_normal((g.n_obs, k))
    want_gx = [o.apply_gramian(X[:, c]) for c in range(k)]
    want_dr = [o.rmatvec_wdt(R[:, c]) for c in range(k)]
    for per, bps in ((16, 1), (32, 2), (64, 2)):
        _pin(g, k, 8, per, bps, 1)
        assert _lib.load().within_solver_obs_hot_global(g._h, k, 8) in (0, 1)
        GX = g.apply_gramian(X)
        DR = g.rmatvec_wdt(R)
        for c in range(k):
            assert rel(GX[:, c], want_gx[c]) < 1e-13, (per, bps, c)
            assert rel(DR[:, c], want_dr[c]) < 1e-13, (per, bps, c)


def test_hot_global_reported():
    cats, w = DESIGNS["akm"]()  # Zipf firms: more than 256 levels outside the primary factor
    g = wb.Solver(cats, weights=w)
    L = _lib.load()
    assert L.within_solver_obs_hot_global(g._h, 16, 8) == -1  # not tuned yet
    _pin(g, 16, 8, 32, 2, 1)
    assert L.within_solver_obs_hot_global(g._h, 16, 8) == 1
    _pin(g, 16, 8, 32, 2, 0)
    assert L.within_solver_obs_hot_global(g._h, 16, 8) == 0
    assert L.within_solver_set_obs_config(g._h, 16, 8, 48, 2, 0) != 0
    assert L.within_solver_set_obs_config(g._h, 16, 8, 32, 3, 0) != 0


def test_mixed_solve_with_global_hot_tables():
    cats, Y, w = synthetic.config3(scale=0.01)
    s = wb.Solver(cats, wb.CG(precision="mixed"), weights=w)
    _pin(s, 16, 4, 32, 2, 1)
    r = s.solve_batch(Y)
    assert _lib.load().within_solver_obs_hot_global(s._h, 16, 4) == 1
    assert all(r.converged) and max(r.residual) <= 1e-8
    truth = oracle.OracleSolver(cats, w, tol=1e-13)
    same_tol = oracle.OracleSolver(cats, w)
    NZ = make_normalizer(cats)
    for c in (0, 9, 15):
        t = truth.solve(Y[:, c])
        o = same_tol.solve(Y[:, c])
        assert rel(r.demeaned[:, c], t.demeaned) <= 2 * rel(o.demeaned, t.demeaned) + 1e-9
        assert rel(NZ(r.x[:, c]), NZ(t.x)) <= 2 * rel(NZ(o.x), NZ(t.x)) + 1e-9
