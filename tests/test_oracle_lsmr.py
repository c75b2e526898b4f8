"""The oracle's LSMR (a restatement of schwarz-precond/src/solve/lsmr.rs, lsmr/bidiag.rs,
lsmr/recurrence.rs) pinned by the reference's own known-answer cases
(lsmr/tests.rs) and by dense least squares on small designs."""
import numpy as np
import pytest

import oracle
from oracle import lsmr_dense

# lsmr/tests.rs:8-52: A = [1 0 0; 0 1 0; 0 0 1; 1 1 0], M^-1 = diag(1/2, 1/2, 1)
OVER = np.array([[1, 0, 0], [0, 1, 0], [0, 0, 1], [1, 1, 0]], float)
DIAG = np.diag([0.5, 0.5, 1.0])


def _normal_residual(a, x, b):
    return np.linalg.norm(a.T @ (b - a @ x))


def test_unpreconditioned_and_preconditioned():
    # lsmr/tests.rs:64-93: b consistent with x = (1, 2, 3)
    b = np.array([1.0, 2.0, 3.0, 3.0])
    for minv in (None, DIAG):
        x, conv, it, stop = lsmr_dense(OVER, b, minv, 1e-10, 100)
        assert conv and np.linalg.norm(x - [1, 2, 3]) < 1e-6


def test_inconsistent_system():
    # lsmr/tests.rs:95-108
    b = np.array([1.0, 2.0, 3.0, 0.0])
    x, conv, _, _ = lsmr_dense(OVER, b, None, 1e-10, 100)
    assert conv and _normal_residual(OVER, x, b) < 1e-6


def test_underdetermined_rank_deficient_degenerate():
    # lsmr/tests.rs:110-194: minimum-norm solutions
    x, conv, _, _ = lsmr_dense(np.array([[1.0, 0, 0], [0, 1, 0]]), np.array([1.0, 2.0]), None, 1e-12, 100)
    assert conv and abs(x[0] - 1) < 1e-10 and abs(x[1] - 2) < 1e-10 and abs(x[2]) < 1e-10
    a = np.array([[1.0, 1.0], [2.0, 2.0]])
    x, conv, _, _ = lsmr_dense(a, np.array([3.0, 6.0]), None, 1e-12, 100)
    assert conv and abs(x.sum() - 3) < 1e-10 and _normal_residual(a, x, [3.0, 6.0]) < 1e-10
    a = np.array([[1.0, 0.0], [0.0, 0.0]])
    x, conv, _, _ = lsmr_dense(a, np.array([2.0, 3.0]), None, 1e-12, 100)
    assert conv and abs(x[0] - 2) < 1e-10 and abs(x[1]) < 1e-10


def test_mid_stream_breakdown_and_maxiter():
    # lsmr/tests.rs:196-237
    x, conv, _, stop = lsmr_dense(np.array([[1.0, 0.0], [0.0, 0.0]]), np.array([5.0, 0.0]), None, 1e-12, 100)
    assert conv and abs(x[0] - 5) < 1e-12 and abs(x[1]) < 1e-12
    x, conv, it, stop = lsmr_dense(OVER, np.array([1.0, 2.0, 3.0, 3.0]), None, 1e-15, 1)
    assert not conv and it == 1 and stop == "MaxIterations"
    x, conv, it, stop = lsmr_dense(OVER, np.zeros(4), None, 1e-8, 10)
    assert conv and it == 0 and stop == "ZeroRhs" and not x.any()


def test_identity_preconditioner_matches_plain():
    # lsmr/tests.rs:275-310: Golub-Kahan and Modified Golub-Kahan with M = I agree
    b = np.array([1.0, 2.0, 3.0, 3.0])
    x0, c0, i0, _ = lsmr_dense(OVER, b, None, 1e-12, 100)
    x1, c1, i1, _ = lsmr_dense(OVER, b, np.eye(3), 1e-12, 100)
    assert c0 and c1 and abs(i0 - i1) <= 1 and np.linalg.norm(x0 - x1) < 1e-10
    for ls in (1, 3):  # windowed reorthogonalization leaves the answer
        x2, c2, _, _ = lsmr_dense(OVER, b, np.eye(3), 1e-12, 100, ls)
        assert c2 and np.linalg.norm(x2 - x1) < 1e-10


def _dense_design(cats):
    cols = []
    for q in range(cats.shape[1]):
        m = np.zeros((cats.shape[0], int(cats[:, q].max()) + 1))
        m[np.arange(cats.shape[0]), cats[:, q]] = 1.0
        cols.append(m)
    return np.hstack(cols)


@pytest.mark.parametrize("weighted", [False, True])
@pytest.mark.parametrize("kw", [dict(preconditioner="off"), dict(), dict(local_size=5),
                                dict(preconditioner="off", local_size=5)])
def test_design_least_squares(weighted, kw):
    # Solver::solve's LSMR branch (solver.rs:162-203): min ||W^(1/2)(y - D x)||
    rng = np.random.default_rng(1)
    n = 400
    cats = np.asfortranarray(np.column_stack([rng.integers(0, 15, n), rng.integers(0, 8, n),
                                              rng.integers(0, 5, n)]).astype(np.uint32))
    w = rng.lognormal(0, 1, n) if weighted else None
    y = rng.standard_normal(n)
    d = _dense_design(cats)
    sw = np.sqrt(w) if weighted else np.ones(n)
    e_ls = y - d @ np.linalg.lstsq(sw[:, None] * d, sw * y, rcond=None)[0]
    r = oracle.OracleSolver(cats, w, krylov="lsmr", tol=1e-10, **kw).solve(y)
    assert r.converged and r.iterations > 0
    assert np.linalg.norm(r.demeaned - e_ls) / np.linalg.norm(e_ls) < 1e-8
    # the preconditioned process needs fewer iterations
    if kw.get("preconditioner") != "off":
        r0 = oracle.OracleSolver(cats, w, krylov="lsmr", tol=1e-10, preconditioner="off").solve(y)
        assert r.iterations < r0.iterations


def test_design_edge_cases():
    rng = np.random.default_rng(2)
    n = 300
    cats = np.asfortranarray(np.column_stack([rng.integers(0, 12, n), rng.integers(0, 7, n)]).astype(np.uint32))
    o = oracle.OracleSolver(cats, None, krylov="lsmr")
    r = o.solve(np.zeros(n))
    assert r.converged and r.iterations == 0 and not r.x.any()
    y = _dense_design(cats) @ rng.standard_normal(19)  # y in the column space of D
    r = o.solve(y)
    assert r.converged and np.abs(r.demeaned).max() < 1e-6
    # (unpreconditioned: on two factors the Schwarz preconditioner is an exact solve)
    r = oracle.OracleSolver(cats, None, krylov="lsmr", maxiter=2, tol=1e-14,
                            preconditioner="off").solve(rng.standard_normal(n))
    assert not r.converged and r.iterations == 2
