"""Host-buffer solves from several host threads on one solver (Solver::solve_batch,
solver.rs:241-277, called concurrently): each call has its own device buffers and copy
stream and the solves take turns, so every call returns the same result as the same call
made alone, and the oracle's."""
import threading

import numpy as np
import pytest

import oracle
import within_b200 as wb
from within_b200 import synthetic
from paritylib import make_normalizer, rel

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_concurrent_host_calls_match_sequential_ones(precision):
    cats, Y, w = synthetic.config3(seed=6, scale=0.02)
    s = wb.Solver(cats, wb.CG(precision=precision), weights=w)
    rng = np.random.default_rng(8)
    batches = [np.asfortranarray(Y * (1.0 + 0.25 * j) + rng.standard_normal(Y.shape)) for j in range(6)]
    alone = [s.solve_batch(b) for b in batches]
    out = [None] * len(batches)
    errors = []

    def worker(idx):
        try:
            for j in idx:
                out[j] = s.solve_batch(batches[j])
        except Exception as e:  # reported below
            errors.append(e)

    th = [threading.Thread(target=worker, args=(list(range(t, len(batches), 3)),)) for t in range(3)]
    for t in th:
        t.start()
    for t in th:
        t.join()
    assert not errors, errors
    NZ = make_normalizer(cats)  # x up to each connected component's constant shift
    for j, (a, b) in enumerate(zip(alone, out)):
        assert all(b.converged) and max(b.residual) <= 1e-8
        # same solve; the order of the atomic additions leaves rounding-level differences
        # (FP64), or FP32 inner iterates that differ by FP32 rounding and end at another
        # point within the tolerance (mixed: measured 2e-10)
        bound = 1e-10 if precision == "fp64" else 1e-8
        assert rel(b.demeaned, a.demeaned) < bound, j
        for c in (0, 7, 15):
            assert rel(NZ(b.x[:, c]), NZ(a.x[:, c])) < bound * 10, (j, c)
    o = oracle.OracleSolver(cats, w)
    if precision == "fp64":  # the reference's iterates
        for j in (0, 5):
            t = o.solve(batches[j][:, 0])
            assert rel(out[j].demeaned[:, 0], t.demeaned) < 1e-8
            assert rel(NZ(out[j].x[:, 0]), NZ(t.x)) < 1e-8
    else:  # accuracy against the tol-1e-13 truth, against the oracle's own at tol 1e-8
        truth = oracle.OracleSolver(cats, w, tol=1e-13)
        for j in (0, 5):
            t, ob = truth.solve(batches[j][:, 0]), o.solve(batches[j][:, 0])
            assert rel(out[j].demeaned[:, 0], t.demeaned) <= 2 * rel(ob.demeaned, t.demeaned) + 1e-9
