"""Uneven batch of independent problems (within_solve_many) against the CPU oracle and
against solving each problem on its own."""
import numpy as np
import pytest

import oracle
import within_b200 as wb
from within_b200 import synthetic
from paritylib import make_normalizer, rel

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_solve_many_matches_oracle(precision):
    probs = synthetic.config4(seed=3, n_problems=7, max_obs=30_000)
    res = wb.solve_many(probs, wb.CG(precision=precision), concurrency=4)
    assert len(res) == len(probs)
    for (cats, Y), r in zip(probs, res):
        assert r.x.shape == (sum(int(cats[:, j].max()) + 1 for j in range(cats.shape[1])), Y.shape[1])
        o = oracle.OracleSolver(cats, None).solve_batch(Y, threads=4)
        t = oracle.OracleSolver(cats, None, tol=1e-13).solve_batch(Y, threads=4)
        NZ = make_normalizer(cats)
        for c in range(Y.shape[1]):
            assert r.converged[c] and r.residual[c] <= 1e-8
            if precision == "fp64":  # the reference's iterates: within 1e-8 of the oracle
                assert rel(r.demeaned[:, c], o.demeaned[:, c]) < 1e-8
                # x of these uniform designs is ill-conditioned: the order of the atomic
                # additions alone moved one x by 1.06e-8 from the oracle's; such an x must
                # then still be within twice the oracle's own error
                ex = rel(NZ(r.x[:, c]), NZ(o.x[:, c]))
                assert ex < 1e-8 or rel(NZ(r.x[:, c]), NZ(t.x[:, c])) <= 2 * rel(NZ(o.x[:, c]), NZ(t.x[:, c])) + 1e-9
            # within twice the reference's own error at the same tolerance
            assert rel(r.demeaned[:, c], t.demeaned[:, c]) <= 2 * rel(o.demeaned[:, c], t.demeaned[:, c]) + 1e-9
            assert rel(NZ(r.x[:, c]), NZ(t.x[:, c])) <= 2 * rel(NZ(o.x[:, c]), NZ(t.x[:, c])) + 1e-9


def test_solve_many_equals_single_solves_and_weights():
    probs = synthetic.config4(seed=5, n_problems=5, max_obs=20_000)
    rng = np.random.default_rng(2)
    wprobs = [(c, Y, rng.lognormal(0, 1, c.shape[0])) for c, Y in probs]
    many = wb.solve_many(wprobs, concurrency=3)
    for (c, Y, w), r in zip(wprobs, many):
        one = wb.solve_batch(c, Y, weights=w)
        for j in range(Y.shape[1]):
            assert rel(r.demeaned[:, j], one.demeaned[:, j]) < 1e-10
            assert r.iterations[j] == one.iterations[j] or abs(r.iterations[j] - one.iterations[j]) <= 1


def test_solve_many_reports_the_failing_problem():
    good = synthetic.config4(seed=7, n_problems=2, max_obs=5_000)
    bad = (good[0][0], good[0][1][:-1])  # one observation short
    with pytest.raises(wb.WithinError):
        wb.solve_many([good[1], bad], concurrency=2)
    assert wb.solve_many([]) == []
