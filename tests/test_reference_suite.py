"""The reference's Python test suite (tests/test_solve.py, test_properties.py,
test_edge_cases.py, test_error_handling.py, test_preconditioner.py), restated against
this package: the same problems, calls and expectations, each test citing the one it
follows.  Argument errors are raised before anything touches a device, so those tests
run on CPU; the others are GPU tests.

Deliberate differences, each stated where it applies: results are reproducible to
rounding, not bit for bit (subdomain and operator sums are accumulated with atomics,
so their order varies between runs); where the reference compares with exact
equality, the test uses 1e-10 relative.
"""
import pickle
import warnings

import numpy as np
import pytest

from within_b200 import (CG, GMRES, AdditiveSchwarz, FePreconditioner, MultiplicativeSchwarz, OperatorRepr,
                         Preconditioner, ReductionStrategy, Solver, solve, solve_batch)
from within_b200._within import ApproxCholConfig, ApproxSchurConfig, SchurComplement
from conftest import generate_synthetic_data


def _cats(cols):
    return np.asfortranarray(np.column_stack(cols).astype(np.uint32))


def _problem():
    """tests/test_solve.py:28-37: two factors of 50 levels, 10k observations (seed 42)."""
    rng = np.random.RandomState(42)
    cats = [rng.randint(0, 50, size=10_000), rng.randint(0, 50, size=10_000)]
    return cats, rng.randn(10_000)


def _design_times(cats, x):
    out, off = np.zeros(cats.shape[0]), 0
    for q in range(cats.shape[1]):
        out += x[off + cats[:, q]]
        off += int(cats[:, q].max()) + 1
    return out


def _relclose(a, b, tol=1e-10):
    return np.linalg.norm(np.asarray(a) - np.asarray(b)) <= tol * max(np.linalg.norm(b), 1e-300)


# ----------------------------------------------------------------- argument errors (CPU)

SMALL = _cats([np.array([0, 1, 0]), np.array([0, 0, 1])])


def test_error_handling():
    # tests/test_error_handling.py:15-94
    with pytest.raises(ValueError):
        solve(np.empty((0, 2), dtype=np.uint32, order="F"), np.array([], dtype=np.float64))
    with pytest.raises(ValueError):
        solve(SMALL, np.array([1.0, 2.0, 3.0]), weights=np.array([1.0, 2.0]))
    with pytest.raises(TypeError):
        solve(np.array([[0.0, 0.0], [1.0, 1.0]], order="F"), np.array([1.0, 2.0]))
    with pytest.raises(TypeError):
        solve(SMALL, np.array([1, 2, 3], dtype=np.int32))
    with pytest.raises(TypeError):
        solve(np.array([0, 1, 2], dtype=np.uint32), np.array([1.0, 2.0, 3.0]))
    with pytest.raises(TypeError):
        solve(SMALL, np.array([1.0, 2.0, 3.0]), config="invalid")
    with pytest.raises(TypeError):
        solve(SMALL, np.array([1.0, 2.0, 3.0]), preconditioner="invalid")
    with pytest.raises((ValueError, OverflowError)):
        ApproxCholConfig(split=0)
    with pytest.raises((ValueError, OverflowError)):
        ApproxSchurConfig(split=0)


def test_config_classes():
    # tests/test_preconditioner.py:43-61
    assert (ApproxCholConfig().seed, ApproxCholConfig().split) == (0, 1)
    c = ApproxCholConfig(seed=42, split=2)
    assert (c.seed, c.split) == (42, 2)
    assert (ApproxSchurConfig().seed, ApproxSchurConfig().split) == (0, 1)
    assert SchurComplement().dense_threshold == 24


def test_argument_checks_before_the_device():
    # tests/test_solve.py:65-76 and test_edge_cases.py:373-385: CG with a multiplicative
    # preconditioner; test_preconditioner.py:113-115: bytes that are not a preconditioner
    cats, y = _problem()
    with pytest.raises(ValueError):
        solve(_cats(cats), y, CG(), preconditioner=Preconditioner.Multiplicative)
    with pytest.raises(ValueError):
        FePreconditioner(b"garbage")


# ------------------------------------------------------------------------ solves (GPU)


@pytest.mark.gpu
def test_solve_configurations():
    # tests/test_solve.py:41-147, test_preconditioner.py:63-72
    cats, y = _problem()
    c = _cats(cats)
    w = np.random.RandomState(0).uniform(0.5, 2.0, size=10_000)
    runs = [
        solve(c, y),
        solve(c, y, CG(operator=OperatorRepr.Explicit)),
        solve(c, y, GMRES(), preconditioner=Preconditioner.Multiplicative),
        solve(c, y, CG(), preconditioner=Preconditioner.Off),
        solve(c, y, GMRES(), preconditioner=Preconditioner.Off),
        solve(c, y, weights=w),
        solve(c, y, CG(), preconditioner=AdditiveSchwarz()),
        solve(c, y, GMRES(), preconditioner=MultiplicativeSchwarz()),
        solve(c, y, CG(), preconditioner=AdditiveSchwarz(local_solver=SchurComplement())),
        solve(c, y, CG(), preconditioner=AdditiveSchwarz(local_solver=SchurComplement(
            approx_chol=ApproxCholConfig(seed=3, split=2), approx_schur=ApproxSchurConfig(seed=1), dense_threshold=8))),
    ]
    for r in runs:
        assert r.converged
        assert r.x.shape == (100,) and r.demeaned.shape == (10_000,)
        assert r.iterations >= 1 and r.residual >= 0.0
        assert r.time_total >= 0 and r.time_setup >= 0 and r.time_solve >= 0


@pytest.mark.gpu
def test_demeaning_properties():
    # tests/test_solve.py:150-203
    cats, x_true, y = generate_synthetic_data([50, 50], 10_000, seed=7)  # (n, Q) uint32, F-order
    r = solve(cats, y)
    assert r.converged
    off = 0
    for n in (50, 50):  # x is identified up to a constant per factor
        bh, bt = r.x[off:off + n], x_true[off:off + n]
        np.testing.assert_allclose(bh - bh.mean(), bt - bt.mean(), atol=1e-4)
        off += n
    rng = np.random.RandomState(99)
    cats = [rng.randint(0, nl, size=5_000) for nl in (30, 40)]
    y = rng.randn(5_000)
    c = _cats(cats)
    r = solve(c, y)
    resid = y - _design_times(c, r.x)
    for q in range(2):  # D' (y - D x) = 0
        assert np.abs(np.bincount(c[:, q], weights=resid)).max() < 1e-6
    np.testing.assert_allclose(r.demeaned, resid, atol=1e-10)


@pytest.mark.gpu
def test_contiguity_warnings_and_solver_reuse():
    # tests/test_solve.py:206-285
    cats, y = _problem()
    c = _cats(cats)
    with pytest.warns(UserWarning):
        solve(np.ascontiguousarray(c), y)
    with warnings.catch_warnings():
        warnings.simplefilter("error")
        solve(c, y)
    s = Solver(c)
    r1, r2 = s.solve(y), solve(c, y)
    assert _relclose(r1.x, r2.x) and _relclose(s.solve(y).x, r1.x)
    assert s.n_dofs == 100 and s.n_obs == 10_000
    assert Solver(c, preconditioner=Preconditioner.Off).solve(y).converged
    assert Solver(c, GMRES(), preconditioner=Preconditioner.Multiplicative).solve(y).converged


@pytest.mark.gpu
def test_batches():
    # tests/test_solve.py:287-440, test_properties.py:322-410
    cats, y = _problem()
    c = _cats(cats)
    rng = np.random.RandomState(5)
    Y = np.column_stack([y, rng.randn(10_000), rng.randn(10_000)])
    s = Solver(c)
    b = s.solve_batch(Y)
    assert b.x.shape == (100, 3) and b.demeaned.shape == (10_000, 3)
    assert len(b.converged) == len(b.iterations) == len(b.residual) == len(b.time_solve) == 3
    assert all(b.converged) and b.time_total >= 0
    for k in range(3):
        assert _relclose(b.x[:, k], s.solve(Y[:, k]).x, 1e-8)
    w = rng.uniform(0.5, 2.0, size=10_000)
    assert all(solve_batch(c, Y, weights=w).converged)
    one = solve_batch(c, y[:, None])
    assert one.x.shape == (100, 1) and _relclose(one.x[:, 0], solve(c, y).x, 1e-8)
    same = s.solve_batch(np.column_stack([y, y, y]))
    np.testing.assert_allclose(same.x[:, 0], same.x[:, 1], atol=1e-12)
    np.testing.assert_allclose(same.x[:, 1], same.x[:, 2], atol=1e-12)
    zero = s.solve_batch(np.zeros((10_000, 2)))
    assert not zero.x.any() and all(zero.converged)


@pytest.mark.gpu
def test_preconditioner_objects():
    # tests/test_preconditioner.py:75-122, test_solve.py:321-385, test_properties.py:76-95
    cats, y = _problem()
    c = _cats(cats)
    s = Solver(c)
    p = s.preconditioner()
    x = np.random.RandomState(1).randn(p.nrows)
    r = p.apply(x)
    assert r.shape == (p.nrows,) and np.isfinite(r).all()
    with pytest.raises(ValueError):
        p.apply(np.random.randn(p.nrows + 5))
    assert "Additive" in repr(p) and p.nrows == p.ncols == s.n_dofs
    q = pickle.loads(pickle.dumps(p))
    # the reference compares applies with exact equality; here to rounding (atomic sums)
    assert _relclose(q.apply(x), p.apply(x)) and _relclose(p.apply(x), p.apply(x))
    r0 = s.solve(y)
    r1 = Solver(c, preconditioner=q).solve(y)
    assert r1.converged and _relclose(r1.x, r0.x, 1e-8)
    pm = Solver(c, GMRES(), preconditioner=Preconditioner.Multiplicative).preconditioner()
    assert "Multiplicative" in repr(pm)
    assert Solver(c, preconditioner=Preconditioner.Off).preconditioner() is None
    assert solve(c, y, preconditioner=Preconditioner.Additive).converged
    assert solve(c, y, GMRES(), preconditioner=Preconditioner.Multiplicative).converged


@pytest.mark.gpu
@pytest.mark.parametrize("seed", [0, 1, 2])
def test_properties(seed):
    # tests/test_properties.py:13-218 (a few fixed draws of its random problems)
    rng = np.random.default_rng(seed)
    q = int(rng.integers(2, 4))
    levels = [int(rng.integers(2, 51)) for _ in range(q)]
    n = int(rng.integers(50, 2001))
    c = np.asfortranarray(np.column_stack([rng.integers(0, nl, size=n, dtype=np.uint32) for nl in levels]))
    y = rng.standard_normal(n)
    r1, r2 = solve(c, y), solve(c, y)
    # the reference asks atol 1e-14 of two solves; atomic accumulation leaves rounding-level
    # differences, so the same comparison is made at 1e-10 relative
    assert _relclose(r1.x, r2.x)
    resid = y - _design_times(c, r1.x)
    for k in range(q):
        assert np.abs(np.bincount(c[:, k], weights=resid)).max() < 1e-6 * max(1.0, np.abs(y).sum())
    np.testing.assert_allclose(r1.demeaned, resid, atol=1e-10)
    e = solve(c, y, CG(operator=OperatorRepr.Explicit))
    np.testing.assert_allclose(e.demeaned, r1.demeaned, atol=1e-6)
    u = solve(c, y, weights=np.ones(n))
    np.testing.assert_allclose(u.demeaned, r1.demeaned, atol=1e-10)
    s = Solver(c)
    assert s.n_dofs == len(r1.x) and s.n_obs == n
    assert r1.residual >= 0 and r1.time_total >= 0 and r1.time_setup >= 0 and r1.time_solve >= 0
    if np.abs(r1.demeaned).max() > 1e-10:
        assert r1.iterations >= 1
    for pre in (AdditiveSchwarz(), AdditiveSchwarz(reduction=ReductionStrategy.AtomicScatter),
                AdditiveSchwarz(reduction=ReductionStrategy.ParallelReduction)):
        rr = solve(c, y, preconditioner=pre)
        assert rr.converged and np.abs(rr.x - r1.x).max() < 1e-4 * max(1.0, np.abs(r1.x).max())
    assert solve(c, y, GMRES(), preconditioner=MultiplicativeSchwarz()).converged
    d = s.preconditioner().additive_schwarz_diagnostics()
    assert d is not None and d.total_inner_parallel_work >= 0 and d.total_scatter_dofs >= 0


@pytest.mark.gpu
def test_edge_cases_non_finite_and_weights():
    # tests/test_edge_cases.py:25-118
    c = SMALL
    assert np.isnan(solve(c, np.array([1.0, np.nan, 3.0])).x).any()
    assert not np.isfinite(solve(c, np.array([1.0, np.inf, 3.0])).x).all()
    y = np.array([1.0, 2.0, 3.0])
    for bad in (np.array([1.0, np.nan, 1.0]), np.array([1.0, np.inf, 1.0])):
        try:  # raise, or a non-finite / non-converged result
            r = solve(c, y, weights=bad)
            assert not np.isfinite(r.x).all() or not r.converged
        except ValueError:
            pass
    try:
        r = solve(c, y, weights=np.zeros(3))
        assert not r.converged or not np.isfinite(r.x).all()
    except ValueError:
        pass
    rng = np.random.RandomState(0)
    cc = _cats([rng.randint(0, 10, 500), rng.randint(0, 10, 500)])
    yy = rng.randn(500)
    try:
        solve(cc, yy, weights=-np.ones(500))  # no crash required
    except ValueError:
        pass
    for w in (np.full(500, 1e-12), np.full(500, 1e12)):
        assert np.isfinite(solve(cc, yy, weights=w).x).all()


@pytest.mark.gpu
def test_edge_cases_degenerate_problems():
    # tests/test_edge_cases.py:121-275
    rng = np.random.RandomState(1)
    c = _cats([rng.randint(0, 20, 1000), rng.randint(0, 20, 1000)])
    r = solve(c, np.zeros(1000))
    assert r.converged and not r.x.any()
    r = solve(c, np.full(1000, 3.5))
    assert np.abs(r.demeaned).max() < 1e-8
    same = _cats([np.zeros(100, int), np.zeros(100, int)])
    assert np.isfinite(solve(same, rng.randn(100)).x).all()
    assert np.isfinite(solve(c, rng.randn(1000), CG(maxiter=1)).x).all()
    hard = _cats([rng.randint(0, 300, 3000), rng.randint(0, 300, 3000)])
    r = solve(hard, rng.randn(3000), CG(maxiter=2, tol=1e-15), preconditioner=Preconditioner.Off)
    assert not r.converged
    assert np.isfinite(solve(c, rng.randn(1000), CG(tol=1e-14)).x).all()
    r = solve(c, rng.randn(1000), CG(tol=1.0))
    assert r.converged and r.iterations <= 2
    assert np.isfinite(solve(c, rng.randn(1000), GMRES(maxiter=1)).x).all()
    solve(c, rng.randn(1000), CG(tol=0.0, maxiter=50))        # no crash required
    solve(c, rng.randn(1000), CG(tol=float("nan"), maxiter=50))
    solve(_cats([np.array([0]), np.array([0])]), np.array([1.0]))
    solve(_cats([np.array([0, 1]), np.array([0, 1])]), np.array([1.0, 2.0]))
    two = _cats([rng.randint(0, 2, 200), rng.randint(0, 2, 200)])
    assert solve(two, rng.randn(200)).converged


@pytest.mark.gpu
def test_edge_cases_layouts_and_preconditioner_off():
    # tests/test_edge_cases.py:278-370
    rng = np.random.RandomState(2)
    c = _cats([rng.randint(0, 30, 2000), rng.randint(0, 25, 2000)])
    big = rng.randn(2000, 3)
    y_nc, y_c = big[:, 1], np.ascontiguousarray(big[:, 1])
    assert _relclose(solve(c, y_nc).x, solve(c, y_c).x)
    wbig = rng.uniform(0.5, 2.0, size=(2000, 2))
    assert _relclose(solve(c, y_c, weights=wbig[:, 0]).x, solve(c, y_c, weights=np.ascontiguousarray(wbig[:, 0])).x)
    with pytest.warns(UserWarning):
        solve(np.ascontiguousarray(c), y_c)
    r = solve(c, y_c, preconditioner=Preconditioner.Off)
    assert r.converged and np.isfinite(r.x).all()
    assert Solver(c, preconditioner=Preconditioner.Off).preconditioner() is None


@pytest.mark.gpu
def test_synthetic_data_helpers():
    # tests/test_solve.py:442-455
    cats, x_true, y = generate_synthetic_data([100, 100], 10_000)
    assert solve(cats, y).converged
    c1, x1, y1 = generate_synthetic_data([50, 50], 5_000, seed=123)
    c2, x2, y2 = generate_synthetic_data([50, 50], 5_000, seed=123)
    np.testing.assert_array_equal(y1, y2)
