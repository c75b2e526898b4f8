"""Parity of the sm_100a path (through the C ABI) with the CPU oracle."""
import numpy as np
import pytest

import oracle
import within_b200 as wb
from within_b200 import synthetic
from conftest import fmajor, generate_synthetic_data
from paritylib import make_normalizer, normalize_x, rel

pytestmark = pytest.mark.gpu

DESIGNS = {
    "uniform2": lambda: (synthetic.uniform_design(60_000, [500, 200], seed=0), None),
    "uniform3w": lambda: (synthetic.uniform_design(80_000, [900, 300, 25], seed=1),
                          np.random.default_rng(5).lognormal(0, 1, 80_000)),
    "akm": lambda: synthetic.config2(scale=0.05)[0::2],
    "akm_w": lambda: (lambda c, Y, w: (c, np.random.default_rng(3).lognormal(0, 1, c.shape[0])))(*synthetic.config2(scale=0.03)),
    "shuffled": lambda: (np.asfortranarray(synthetic.config2(scale=0.02)[0][np.random.default_rng(9).permutation(40_000)]), None),
    # four factors, weighted; five factors (the generic factor-count kernels)
    "uniform4w": lambda: (synthetic.uniform_design(50_000, [600, 250, 40, 6], seed=11),
                          np.random.default_rng(6).lognormal(0, 1, 50_000)),
    "uniform5": lambda: (synthetic.uniform_design(30_000, [350, 120, 30, 8, 4], seed=12), None),
    # primary factor with most of its levels unobserved (empty levels inside chunks)
    "sparse_primary": lambda: (np.asfortranarray(np.column_stack([
        np.random.default_rng(13).integers(0, 5000, 3000), np.random.default_rng(14).integers(0, 50, 3000)]).astype(np.uint32)), None),
}


def _pair(name, **kw):
    cats, w = DESIGNS[name]()
    return cats, w, wb.Solver(cats, wb.CG(**{k: v for k, v in kw.items() if k in ("tol", "maxiter", "precision", "max_refinements")}), weights=w), oracle.OracleSolver(cats, w, **{k: v for k, v in kw.items() if k in ("tol", "maxiter", "max_refinements")})


@pytest.mark.parametrize("name", list(DESIGNS))
def test_setup_is_bit_exact(name):
    cats, w = DESIGNS[name]()
    g = wb.Solver(cats, weights=w)
    o = oracle.OracleSolver(cats, w)
    gn, go = g.factor_meta(), o.factor_meta()
    assert gn[0].tolist() == go[0].tolist() and gn[1].tolist() == go[1].tolist()
    gs, os_ = g.subdomains(), o.subdomains()
    assert len(gs) == len(os_)
    for a, b in zip(gs, os_):
        for key in ("pair", "n_q", "n_r", "eliminate_q", "reduced_kind", "n_reduced"):
            assert a[key] == b[key], key
        np.testing.assert_array_equal(a["global_indices"], b["global_indices"])
        np.testing.assert_array_equal(a["pou"], b["pou"])
        if "ac" in b:
            for key in ("level_ptr", "col_vertex", "col_ptr", "col_idx", "core_vertex"):
                np.testing.assert_array_equal(a["ac"][key], b["ac"][key], err_msg=key)
            np.testing.assert_array_equal(a["ac"]["col_diag"], b["ac"]["col_diag"])
            np.testing.assert_array_equal(a["ac"]["col_coef"], b["ac"]["col_coef"])
            np.testing.assert_allclose(a["ac"]["core_z"], b["ac"]["core_z"], rtol=1e-10, atol=1e-14)


@pytest.mark.parametrize("name", list(DESIGNS))
@pytest.mark.parametrize("k", [1, 5, 16, 32])
def test_operator_applies(name, k):
    cats, w = DESIGNS[name]()
    g = wb.Solver(cats, weights=w)
    o = oracle.OracleSolver(cats, w)
    rng = np.random.default_rng(k)
    X = rng.standard_normal((g.n_dofs, k))
    R = rng.standard_normal((g.n_obs, k))
    GX = g.apply_gramian(X)
    DX = g.matvec_d(X)
    DR = g.rmatvec_wdt(R)
    for c in range(k):
        assert rel(GX[:, c], o.apply_gramian(X[:, c])) < 1e-13
        assert rel(DX[:, c], o.matvec_d(X[:, c])) < 1e-15
        assert rel(DR[:, c], o.rmatvec_wdt(R[:, c])) < 1e-13


@pytest.mark.parametrize("name", list(DESIGNS))
@pytest.mark.parametrize("k", [1, 16])
def test_preconditioner_apply(name, k):
    cats, w = DESIGNS[name]()
    g = wb.Solver(cats, weights=w)
    o = oracle.OracleSolver(cats, w)
    R = np.random.default_rng(7).standard_normal((g.n_dofs, k))
    Z = g.preconditioner().apply(R)
    for c in range(k):
        assert rel(Z[:, c], o.apply_precond(R[:, c])) < 1e-10


@pytest.mark.parametrize("name", list(DESIGNS))
def test_solve_matches_oracle(name):
    cats, w = DESIGNS[name]()
    y = np.random.default_rng(11).standard_normal(cats.shape[0])
    g = wb.Solver(cats, weights=w).solve(y)
    os_ = oracle.OracleSolver(cats, w)
    o = os_.solve(y)
    truth = oracle.OracleSolver(cats, w, tol=1e-13).solve(y)
    assert g.converged and g.residual <= 1e-8
    assert abs(g.iterations - o.iterations) <= 2
    # tolerance 1e-8 relative (demeaned) against the oracle at the same tol
    assert rel(g.demeaned, o.demeaned) < 1e-8
    # the error against the FP64 truth (tol 1e-13) is of the same size as the oracle's own
    assert rel(g.demeaned, truth.demeaned) < max(10 * rel(o.demeaned, truth.demeaned), 1e-9)
    # x after removing the null-space shift: the same iterates as the oracle's
    assert rel(normalize_x(cats, g.x), normalize_x(cats, o.x)) < 1e-8
    # the demeaned output is y - D x of the returned x
    assert rel(g.demeaned, y - os_.matvec_d(g.x)) < 1e-12


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_batch_16_rhs(precision):
    cats, Y, w = synthetic.config3(scale=0.01)
    s = wb.Solver(cats, wb.CG(precision=precision), weights=w)
    r = s.solve_batch(Y)
    truth = oracle.OracleSolver(cats, w, tol=1e-13)
    assert all(r.converged) and max(r.residual) <= 1e-8
    assert r.x.shape == (s.n_dofs, 16) and r.demeaned.shape == (s.n_obs, 16)
    same_tol = oracle.OracleSolver(cats, w)
    NZ = make_normalizer(cats)
    for c in (0, 7, 15):
        t = truth.solve(Y[:, c])
        o = same_tol.solve(Y[:, c])
        if precision == "fp64":  # the reference's iterates
            assert rel(r.demeaned[:, c], o.demeaned) < 1e-8
            assert rel(NZ(r.x[:, c]), NZ(o.x)) < 1e-8
        # within twice the reference's own error at the same tolerance
        assert rel(r.demeaned[:, c], t.demeaned) <= 2 * rel(o.demeaned, t.demeaned) + 1e-9
        assert rel(NZ(r.x[:, c]), NZ(t.x)) <= 2 * rel(NZ(o.x), NZ(t.x)) + 1e-9
    if precision == "fp64":
        one = s.solve(Y[:, 3])
        assert rel(one.demeaned, r.demeaned[:, 3]) < 1e-10


def test_reference_python_tests_semantics():
    # tests/test_solve.py:150-203 of the reference, run against the device path
    cats, x_true, y = generate_synthetic_data([50, 50], 10_000, seed=7)
    r = wb.solve(cats, y)
    assert r.converged
    off = 0
    for n in (50, 50):
        b, t = r.x[off:off + n], x_true[off:off + n]
        np.testing.assert_allclose(b - b.mean(), t - t.mean(), atol=1e-4)
        off += n
    o = oracle.OracleSolver(cats)
    np.testing.assert_allclose(r.demeaned, y - o.matvec_d(r.x), atol=1e-10)
    assert np.abs(o.rmatvec_dt(r.demeaned)).max() < 1e-4


def test_edge_cases():
    cats = synthetic.uniform_design(3_000, [30, 20], seed=2)
    s = wb.Solver(cats)
    r = s.solve(np.zeros(3_000))
    assert r.converged and r.iterations == 0 and not r.x.any()
    r = s.solve(np.full(3_000, 2.5))
    assert np.abs(r.demeaned).max() < 1e-8
    # reference tests/test_edge_cases.py:161-180 (50 x 50 levels, tol 1e-15)
    rng = np.random.default_rng(42)
    hard = np.asfortranarray(np.column_stack([rng.integers(0, 50, 1000), rng.integers(0, 50, 1000)]).astype(np.uint32))
    yh = rng.standard_normal(1000)
    for it in (1, 2):
        r = wb.solve(hard, yh, wb.CG(maxiter=it, tol=1e-15))
        assert not r.converged and np.all(np.isfinite(r.x))
    r = wb.solve(hard, yh, wb.CG(tol=1.0))
    assert r.converged
    r = wb.solve(cats, np.random.default_rng(0).standard_normal(3_000), preconditioner=wb.Preconditioner.Off)
    assert r.converged
    # single observation / two observations (reference tests/test_edge_cases.py:244-262)
    r = wb.solve(np.zeros((1, 2), np.uint32, order="F"), np.array([3.0]))
    assert np.all(np.isfinite(r.x))
    r = wb.solve(fmajor([[0, 1], [0, 1]]), np.array([1.0, 2.0]))
    assert np.all(np.isfinite(r.x))
    with pytest.raises(wb.WithinError, match="expected 3000"):
        s.solve(np.zeros(10))
    # more than 32 RHS (chunked) and C-order categories
    Y = np.random.default_rng(4).standard_normal((3_000, 35))
    b = wb.solve_batch(np.ascontiguousarray(cats), Y)
    assert all(b.converged) and b.x.shape[1] == 35


@pytest.mark.parametrize("local", [
    wb.SchurComplement(approx_schur=None),
    wb.SchurComplement(approx_chol=wb.ApproxCholConfig(seed=3, split=1), approx_schur=wb.ApproxSchurConfig(seed=1, split=2)),
    wb.SchurComplement(dense_threshold=0),
])
def test_local_solver_variants(local):
    cats = synthetic.uniform_design(50_000, [700, 300], seed=4)
    y = np.random.default_rng(6).standard_normal(50_000)
    r = wb.solve(cats, y, preconditioner=wb.AdditiveSchwarz(local_solver=local))
    t = oracle.OracleSolver(cats, tol=1e-13).solve(y)
    assert r.converged
    assert rel(r.demeaned, t.demeaned) < 1e-7


@pytest.mark.parametrize("pre", ["multiplicative", "additive"])
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_gmres(pre, precision):
    cats = synthetic.uniform_design(40_000, [400, 150, 12], seed=8)
    w = np.random.default_rng(2).lognormal(0, 1, 40_000)
    y = np.random.default_rng(3).standard_normal(40_000)
    p = wb.MultiplicativeSchwarz() if pre == "multiplicative" else wb.AdditiveSchwarz()
    r = wb.solve(cats, y, wb.GMRES(restart=30, precision=precision), weights=w, preconditioner=p)
    o = oracle.OracleSolver(cats, w, krylov="gmres", preconditioner=pre).solve(y)
    t = oracle.OracleSolver(cats, w, tol=1e-13).solve(y)
    assert r.converged and o.converged and r.residual <= 1e-8
    assert rel(r.demeaned, o.demeaned) < 1e-8
    assert rel(r.demeaned, t.demeaned) < 1e-7
    if precision == "fp64":
        assert abs(r.iterations - o.iterations) <= 2


def test_multiplicative_preconditioner_apply():
    cats = synthetic.uniform_design(30_000, [300, 120, 10], seed=9)
    g = wb.Solver(cats, wb.GMRES(), preconditioner=wb.MultiplicativeSchwarz())
    o = oracle.OracleSolver(cats, krylov="gmres", preconditioner="multiplicative")
    R = np.random.default_rng(1).standard_normal((g.n_dofs, 3))
    Z = g.preconditioner().apply(R)
    for c in range(3):
        assert rel(Z[:, c], o.apply_precond(R[:, c])) < 1e-10


def test_gmres_batch_and_edges():
    cats = synthetic.uniform_design(20_000, [200, 100, 9], seed=10)
    Y = np.random.default_rng(4).standard_normal((20_000, 5))
    Y[:, 2] = 0.0
    r = wb.solve_batch(cats, Y, wb.GMRES(restart=10))
    assert all(r.converged) and r.iterations[2] == 0 and not r.x[:, 2].any()
    one = wb.solve(cats, Y[:, 1], wb.GMRES(restart=10))
    assert rel(one.demeaned, r.demeaned[:, 1]) < 1e-9
    r1 = wb.solve(cats, Y[:, 0], wb.GMRES(restart=30, maxiter=1, tol=1e-15, max_refinements=0))
    assert not r1.converged and r1.iterations == 1 and np.all(np.isfinite(r1.x))
