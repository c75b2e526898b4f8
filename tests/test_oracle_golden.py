"""The CPU oracle against the literal vectors of the reference's own unit tests."""
import numpy as np
import pytest

import oracle
from conftest import fmajor


def test_design5_operators(golden):
    g = golden["design5"]
    s = oracle.OracleSolver(fmajor(g["categories_factor_major"]), preconditioner="off")
    nl, off = s.factor_meta()
    assert nl.tolist() == g["n_levels"] and off.tolist() == g["offsets"]
    assert s.n_dofs == g["n_dofs"]
    assert s.matvec_d(g["x"]).tolist() == g["dx"]
    assert s.rmatvec_dt(g["r"]).tolist() == g["dtr"]
    assert s.rmatvec_wdt(g["r"]).tolist() == g["dtr"]       # unweighted: D'W = D'
    assert s.gramian_diagonal().tolist() == g["diag"]


def test_weighted4(golden):
    g = golden["weighted4"]
    s = oracle.OracleSolver(fmajor(g["categories_factor_major"]), weights=g["weights"], preconditioner="off")
    assert s.rmatvec_wdt(g["r"]).tolist() == g["dtwr"]
    assert s.gramian_diagonal().tolist() == g["diag"]


def test_csr_transpose(golden):
    g = golden["csr_transpose"]
    tp, ti, td = oracle.csr_transpose(g["nrows"], g["ncols"], g["indptr"], g["indices"], g["data"])
    assert tp.tolist() == g["t_indptr"] and ti.tolist() == g["t_indices"] and td.tolist() == g["t_data"]
    # round trip
    p2, i2, d2 = oracle.csr_transpose(g["ncols"], g["nrows"], tp, ti, td)
    assert p2.tolist() == g["indptr"] and i2.tolist() == g["indices"] and d2.tolist() == g["data"]


def test_two_components(golden):
    g = golden["two_components"]
    s = oracle.OracleSolver(fmajor(g["categories_factor_major"]))
    subs = s.subdomains()
    assert len(subs) == 2
    # component q-levels then r-levels (global r offset = 4)
    for sd, comp in zip(subs, g["components"]):
        assert sd["global_indices"].tolist() == comp["q"] + [4 + v for v in comp["r"]]
        assert sd["pou"].tolist() == [1.0] * 4


def test_three_factor_pou(golden):
    g = golden["three_factor6"]
    cats = fmajor(g["categories_factor_major"])
    s = oracle.OracleSolver(cats)
    subs = s.subdomains()
    assert len(subs) >= g["min_domains"]
    wsq = np.zeros(s.n_dofs)
    covered = np.zeros(s.n_dofs, bool)
    for sd in subs:
        wsq[sd["global_indices"]] += sd["pou"] ** 2
        covered[sd["global_indices"]] = True
    assert covered.all()
    np.testing.assert_allclose(wsq[wsq > 0], 1.0, rtol=0, atol=1e-12)


def test_large_design_adjoint(golden):
    g = golden["large_design"]
    n = g["n_obs"]
    i = np.arange(n)
    cats = np.asfortranarray(np.column_stack([i % 50, i % 50]).astype(np.uint32))
    s = oracle.OracleSolver(cats, preconditioner="off")
    x = np.sin(np.arange(s.n_dofs) * 0.17 + 1.0)
    r = np.cos(np.arange(n) * 0.23 + 2.0)
    assert abs(s.matvec_d(x) @ r - x @ s.rmatvec_dt(r)) < g["adjoint_tol"]
    assert np.all(s.rmatvec_dt(np.ones(n)) == g["dt_ones_per_level"])


def test_cg_spd3(golden):
    g = golden["spd3"]
    a, b = np.array(g["a"]), np.array(g["b"])
    x, conv, it, _ = oracle.dense_krylov(a, b, tol=g["tol"], maxiter=100)
    assert conv and it <= g["max_iterations_unpreconditioned"]
    assert np.linalg.norm(a @ x - b) < g["residual_tol"]
    x2, conv2, _, _ = oracle.dense_krylov(a, b, m_inv_diag=g["jacobi_inv_diag"], tol=g["tol"], maxiter=100)
    assert conv2 and np.linalg.norm(a @ x2 - b) < g["residual_tol"]
    # zero rhs: converged at iteration 0 with x = 0
    x0, c0, i0, r0 = oracle.dense_krylov(a, np.zeros(3))
    assert c0 and i0 == 0 and r0 == 0.0 and not x0.any()
    # maxiter exhaustion
    _, c1, i1, r1 = oracle.dense_krylov(a, b, tol=1e-15, maxiter=1)
    assert not c1 and i1 == 1 and r1 > 0


def test_cg_indefinite(golden):
    g = golden["neg_diag3"]
    _, conv, it, _ = oracle.dense_krylov(np.array(g["a"]), np.array(g["b"]))
    assert conv == g["converged"] and it == g["iterations"]


def test_gmres_known_answers(golden):
    g = golden["gmres_diag3"]
    x, conv, it, _ = oracle.dense_krylov(np.array(g["a"]), np.array(g["b"]), tol=g["tol"], method="gmres")
    assert conv and it <= g["max_iterations"]
    np.testing.assert_allclose(x, g["x"], atol=1e-10)
    a = np.array(golden["spd3"]["a"]); b = np.array(golden["spd3"]["b"])
    for restart in (1, 2, 50):
        x, conv, it, _ = oracle.dense_krylov(a, b, tol=1e-10, method="gmres", restart=restart)
        assert conv and np.linalg.norm(a @ x - b) < 1e-8
    x, conv, it, rn = oracle.dense_krylov(a, np.zeros(3), method="gmres")
    assert conv and it == 0 and rn == 0.0
