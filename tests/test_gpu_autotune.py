"""The observation pass's autotuner: after a solve the block shape is one of the
candidates, a solver of the same shape class reuses it, and the operator apply under the
tuned shape still matches the CPU oracle."""
import ctypes as C

import numpy as np
import pytest

import oracle
import within_b200 as wb
from within_b200 import _lib, synthetic
from paritylib import rel

pytestmark = pytest.mark.gpu


def _config(s, k, elem):
    per, bps = C.c_int32(), C.c_int32()
    rc = _lib.load().within_solver_obs_config(s._h, k, elem, C.byref(per), C.byref(bps))
    return rc, per.value, bps.value


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_autotuned_shape_is_a_candidate_and_shared(precision):
    cats, Y, w = synthetic.config2(scale=0.05)
    s = wb.Solver(cats, wb.CG(precision=precision), weights=w)
    assert _config(s, 9, 8)[0] == 1  # not tuned before a solve
    r = s.solve_batch(np.asfortranarray(Y))
    assert all(r.converged)
    elem = 4 if precision == "mixed" else 8
    rc, per, bps = _config(s, 9, elem)
    assert rc == 0 and per in (16, 32, 64) and bps in (1, 2)
    # same shape class (observation count within a factor of two, same factors and kp)
    cats2, Y2, w2 = synthetic.config2(seed=5, scale=0.05)
    s2 = wb.Solver(cats2, wb.CG(precision=precision), weights=w2)
    s2.solve_batch(np.asfortranarray(Y2))
    assert _config(s2, 9, elem) == (0, per, bps)
    # the same variant of the hot tables runs in both (the second allocates its own copies)
    L = _lib.load()
    assert L.within_solver_obs_hot_global(s._h, 9, elem) in (0, 1)
    assert L.within_solver_obs_hot_global(s2._h, 9, elem) == L.within_solver_obs_hot_global(s._h, 9, elem)
    # the tuner's table: every shared-memory candidate timed by the first solver, none by
    # the second (it reused the choice)
    t1, t2 = (C.c_float * 12)(), (C.c_float * 12)()
    assert L.within_solver_obs_tune_times(s._h, 9, elem, t1, 12) == 0
    assert L.within_solver_obs_tune_times(s2._h, 9, elem, t2, 12) == 0
    assert all(t1[c] > 0 for c in range(6)) and all(t2[c] == 0 for c in range(12))
    # the operator apply under the tuned shape (FP64 solvers tune their FP64 pass)
    if precision == "fp64":
        o = oracle.OracleSolver(cats, w)
        X = np.random.default_rng(2).standard_normal((s.n_dofs, 9))
        GX = s.apply_gramian(X)
        for c in range(9):
            assert rel(GX[:, c], o.apply_gramian(X[:, c])) < 1e-13
