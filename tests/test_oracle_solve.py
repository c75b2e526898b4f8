"""End-to-end properties of the oracle's solve (reference test strategy, tests/test_solve.py)."""
import numpy as np
import pytest

import oracle
from conftest import generate_synthetic_data
from within_b200 import synthetic


def test_recovers_fixed_effects():
    # reference tests/test_solve.py:150-167 (atol 1e-4 per-factor demeaned)
    cats, x_true, y = generate_synthetic_data([50, 50], 10_000, seed=7)
    r = oracle.OracleSolver(cats).solve(y)
    assert r.converged
    off = 0
    for n in (50, 50):
        b, t = r.x[off:off + n], x_true[off:off + n]
        np.testing.assert_allclose(b - b.mean(), t - t.mean(), atol=1e-4)
        off += n


@pytest.mark.parametrize("pre", ["additive", "off"])
def test_residual_orthogonal_and_demeaned(pre):
    rng = np.random.default_rng(99)
    cats = synthetic.uniform_design(5_000, [30, 40], seed=3)
    y = rng.standard_normal(5_000)
    s = oracle.OracleSolver(cats, preconditioner=pre)
    r = s.solve(y)
    assert r.converged and r.residual < 1e-8
    np.testing.assert_allclose(r.demeaned, y - s.matvec_d(r.x), atol=1e-10)
    assert np.abs(s.rmatvec_dt(r.demeaned)).max() < 1e-4


def test_gmres_multiplicative_and_additive_agree():
    cats = synthetic.uniform_design(20_000, [200, 80, 15], seed=5)
    y = np.random.default_rng(1).standard_normal(20_000)
    ra = oracle.OracleSolver(cats).solve(y)
    rm = oracle.OracleSolver(cats, krylov="gmres", preconditioner="multiplicative").solve(y)
    rg = oracle.OracleSolver(cats, krylov="gmres").solve(y)
    assert ra.converged and rm.converged and rg.converged
    for r in (rm, rg):
        np.testing.assert_allclose(r.demeaned, ra.demeaned, atol=1e-6 * np.abs(y).max())


def test_batch_matches_individual():
    cats, Y, w = synthetic.config2(scale=0.02)
    s = oracle.OracleSolver(cats, w)
    b = s.solve_batch(Y[:, :3], threads=2)
    for c in range(3):
        r = s.solve(Y[:, c])
        np.testing.assert_array_equal(b.x[:, c], r.x)
        np.testing.assert_array_equal(b.demeaned[:, c], r.demeaned)


def test_exact_schur_and_split_variants():
    cats = synthetic.uniform_design(30_000, [400, 300], seed=11)
    y = np.random.default_rng(2).standard_normal(30_000)
    ref = oracle.OracleSolver(cats, tol=1e-13).solve(y)
    for kw in (dict(approx_schur=None), dict(approx_schur=(0, 2), approx_chol_split=1),
               dict(approx_chol_seed=7, dense_threshold=0)):
        r = oracle.OracleSolver(cats, **kw).solve(y)
        assert r.converged
        np.testing.assert_allclose(r.demeaned, ref.demeaned, atol=1e-7 * np.abs(y).max())


def test_ac_factor_is_deterministic_and_complete():
    cats, Y, w = synthetic.config2(scale=0.05)
    a = oracle.OracleSolver(cats, w).subdomains()
    b = oracle.OracleSolver(cats, w).subdomains()
    acs = [(x["ac"], y["ac"]) for x, y in zip(a, b) if "ac" in x]
    assert acs
    for fa, fb in acs:
        for key in ("level_ptr", "col_vertex", "col_ptr", "col_idx", "core_vertex"):
            np.testing.assert_array_equal(fa[key], fb[key])
        np.testing.assert_array_equal(fa["col_coef"], fb["col_coef"])
        # every vertex is eliminated exactly once or belongs to the core
        verts = np.concatenate([fa["col_vertex"], fa["core_vertex"]])
        assert sorted(verts.tolist()) == list(range(fa["n"]))
        # coefficients of a column are the neighbour weights over the pivot: they sum to 1
        cp = fa["col_ptr"]
        sums = np.add.reduceat(fa["col_coef"], cp[:-1]) if len(cp) > 1 and cp[-1] else np.array([])
        nz = np.diff(cp) > 0
        np.testing.assert_allclose(sums[nz[: len(sums)]], 1.0, rtol=1e-12)


def test_zero_rhs_and_constant_y():
    cats = synthetic.uniform_design(2_000, [20, 10], seed=1)
    s = oracle.OracleSolver(cats)
    r = s.solve(np.zeros(2_000))
    assert r.converged and r.iterations == 0 and not r.x.any()
    r = s.solve(np.full(2_000, 3.5))
    assert np.abs(r.demeaned).max() < 1e-8
