"""The hybrid operator apply: the primary factor's blocks with the small factors applied
by one pass over the observations (prim_rows_kernel), every other block of G = D'WD as
CSR rows of the additive Schwarz setup's factor-pair cross-tabulations.  It computes the
reference's GramianOperator::apply (operator/gramian.rs:84-89, over domain.rs:312-417):
checked against the CPU oracle in FP64 (1e-13) and FP32 (rounding of x and the weights),
for one and two small factors, and through CG solves at the stated tolerance."""
import ctypes as C

import numpy as np
import pytest

import oracle
import within_b200 as wb
from within_b200 import _lib, synthetic
from paritylib import make_normalizer, rel
from test_gpu_parity import DESIGNS

pytestmark = pytest.mark.gpu

FP32_TOL = 5e-6
# designs with one or two non-primary factors small enough for lane-group tables (at most
# 24 levels together: 20 years; 6 levels; 4 and 8 levels)
ELIGIBLE = ["akm", "akm_w", "shuffled", "uniform4w", "uniform5"]


def _set(s, k, elem, on):
    L = _lib.load()
    return L.within_solver_set_hybrid(s._h, k, elem, on)


@pytest.mark.parametrize("name", ELIGIBLE)
@pytest.mark.parametrize("k", [1, 5, 13, 16, 32])
def test_hybrid_apply_matches_oracle(name, k):
    cats, w = DESIGNS[name]()
    o = oracle.OracleSolver(cats, w)
    X = np.random.default_rng(k + 400).standard_normal((o.n_dofs, k))
    want = [o.apply_gramian(X[:, c]) for c in range(k)]
    g64 = wb.Solver(cats, weights=w)
    assert _set(g64, k, 8, 1) == 0, _lib.last_error()
    assert _lib.load().within_solver_hybrid(g64._h, k, 8, None) == 1
    GX = g64.apply_gramian(X)
    for c in range(k):
        assert rel(GX[:, c], want[c]) < 1e-13, c
    g32 = wb.Solver(cats, wb.CG(precision="mixed"), weights=w)
    rc = _set(g32, k, 4, 1)
    # one FP32 lane per row (k <= 4): a 20-level table per lane group does not fit
    assert rc == 0 or (k <= 4 and name != "uniform4w"), _lib.last_error()
    if rc == 0:
        GX = g32.apply_gramian(X)
        assert _set(g32, k, 4, 0) == 0
        GXi = g32.apply_gramian(X)  # the FP32 observation pass
        for c in range(k):
            assert rel(GX[:, c], want[c]) < FP32_TOL, c
            # no less accurate than the observation pass in the same precision
            assert rel(GX[:, c], want[c]) <= 2 * rel(GXi[:, c], want[c]) + 1e-7, c
    if k in (16, 13):  # the tensor-core form (16 RHS columns)
        assert _set(g64, k, 8, 2) == 0, _lib.last_error()
        assert _lib.load().within_solver_hybrid(g64._h, k, 8, None) == 2
        GX = g64.apply_gramian(X)
        for c in range(k):
            assert rel(GX[:, c], want[c]) < 1e-13, c
        if rc == 0:
            assert _set(g32, k, 4, 2) == 0, _lib.last_error()
            GX = g32.apply_gramian(X)
            for c in range(k):
                assert rel(GX[:, c], want[c]) < FP32_TOL, c
                assert rel(GX[:, c], want[c]) <= 2 * rel(GXi[:, c], want[c]) + 1e-7, c
    else:
        assert _set(g64, k, 8, 2) != 0  # no tensor-core form for this RHS width
    # and off again: the observation pass
    assert _set(g64, k, 8, 0) == 0
    GX = g64.apply_gramian(X)
    for c in range(k):
        assert rel(GX[:, c], want[c]) < 1e-13, c


def test_hybrid_rejected_where_it_does_not_apply():
    for name in ("uniform2", "uniform3w"):  # smallest non-primary factor: 200, 25 levels
        cats, w = DESIGNS[name]()
        assert _set(wb.Solver(cats, weights=w), 16, 8, 1) != 0
    cats, w = DESIGNS["akm"]()
    assert _set(wb.Solver(cats, weights=w, preconditioner=wb.Preconditioner.Off), 16, 8, 1) != 0
    assert _set(wb.Solver(cats, wb.GMRES(), weights=w, preconditioner=wb.MultiplicativeSchwarz()), 16, 8, 1) != 0
    assert _set(wb.Solver(cats, weights=w), 16, 4, 1) != 0  # an FP64 solver has no FP32 operator


@pytest.mark.parametrize("form", [1, 2])
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_solve_with_hybrid_apply(precision, form):
    cats, Y, w = synthetic.config3(seed=2, scale=0.01)
    k = Y.shape[1]
    s = wb.Solver(cats, wb.CG(precision=precision), weights=w)
    assert _set(s, k, 8, form) == 0, _lib.last_error()
    if precision == "mixed":
        assert _set(s, k, 4, form) == 0, _lib.last_error()
    r = s.solve_batch(Y)
    assert all(r.converged) and max(r.residual) <= 1e-8
    same_tol = oracle.OracleSolver(cats, w)
    NZ = make_normalizer(cats)
    if precision == "fp64":  # the reference's iterates, to the rounding of the sums' order
        for c in (0, 8, 15):
            o = same_tol.solve(Y[:, c])
            assert rel(r.demeaned[:, c], o.demeaned) < 1e-8
            assert rel(NZ(r.x[:, c]), NZ(o.x)) < 1e-8
    else:
        truth = oracle.OracleSolver(cats, w, tol=1e-13)
        for c in (0, 8, 15):
            t = truth.solve(Y[:, c])
            o = same_tol.solve(Y[:, c])
            assert rel(r.demeaned[:, c], t.demeaned) <= 2 * rel(o.demeaned, t.demeaned) + 1e-9
            # x: both stop at a residual of 1e-8, where the coefficients' error depends on
            # the path the iterates took (measured 2.3 and 4.0 times the oracle's own
            # 7.9e-9 on the first RHS, for two builds of the FP32 hybrid apply whose
            # operator errors are within rounding of each other)
            assert rel(NZ(r.x[:, c]), NZ(t.x)) <= 5 * rel(NZ(o.x), NZ(t.x)) + 1e-9


def test_autotuner_decides_and_the_decision_is_exact():
    cats, Y, w = synthetic.config3(seed=3, scale=0.05)
    k = Y.shape[1]
    s = wb.Solver(cats, wb.CG(precision="mixed"), weights=w)
    L = _lib.load()
    assert L.within_solver_hybrid(s._h, k, 4, None) == -1
    r = s.solve_batch(Y)
    assert all(r.converged) and max(r.residual) <= 1e-8
    ms = C.c_float()
    on32 = L.within_solver_hybrid(s._h, k, 4, C.byref(ms))
    assert on32 in (0, 1, 2) and ms.value > 0
    on64 = L.within_solver_hybrid(s._h, k, 8, C.byref(ms))
    assert on64 in (0, 1, 2)
    o = oracle.OracleSolver(cats, w)
    X = np.random.default_rng(7).standard_normal((s.n_dofs, 3))
    GX = s.apply_gramian(X)  # FP32 operator of the mixed solver, as decided
    for c in range(3):
        assert rel(GX[:, c], o.apply_gramian(X[:, c])) < FP32_TOL


def test_hybrid_decision_is_shared_by_a_shape_class():
    """Solvers of one shape class (observation count within a factor of two, same factor
    count and RHS width) take the first one's decision without timing it again."""
    L = _lib.load()
    cats, Y, w = synthetic.config2(seed=11, scale=0.08)
    Y = np.asfortranarray(Y[:, :5])
    s1 = wb.Solver(cats, weights=w)
    s1.solve_batch(Y)
    ms = C.c_float()
    # timed here, or taken from an earlier solver of the class in this process
    on1 = L.within_solver_hybrid(s1._h, 5, 8, C.byref(ms))
    assert on1 in (0, 1)  # no tensor-core form at 5 RHS (kp 8)
    cats2, Y2, w2 = synthetic.config2(seed=12, scale=0.08)
    Y2 = np.asfortranarray(Y2[:, :5])
    s2 = wb.Solver(cats2, weights=w2)
    r2 = s2.solve_batch(Y2)
    assert L.within_solver_hybrid(s2._h, 5, 8, C.byref(ms)) == on1 and ms.value == 0  # not timed again
    o = oracle.OracleSolver(cats2, w2)
    t = o.solve(Y2[:, 0])
    assert rel(r2.demeaned[:, 0], t.demeaned) < 1e-8
