"""The Gramian apply that allocates nothing, checked against the one that allocates and
against the CPU oracle.

within_solver_apply_gramian_noalloc is for callers that cannot allocate device memory
while they run: code under a fixed device-memory budget or a custom allocator that
forbids outside allocations, and loops that cannot take an allocation's
synchronisation.  Its working space is a static device array instead of cudaMalloc'd
buffers.  Its arithmetic is FP64 through the implicit observation pass whatever the
solver's precision and operator, so each case is compared with the oracle at the FP64
operator tolerance, and with the allocating apply at the tolerance that apply has in
that configuration.  This file is named to be collected last.
"""
import ctypes as C

import numpy as np
import pytest

import oracle
import within_b200 as wb
from within_b200 import _lib, synthetic

pytestmark = pytest.mark.gpu


def _noalloc(solver, X, stream=None):
    import torch
    dx = torch.from_numpy(np.ascontiguousarray(X.T)).cuda()  # RHS-major: column c at c * n_dofs
    dy = torch.full_like(dx, np.nan)
    torch.cuda.synchronize()
    rc = _lib.load().within_solver_apply_gramian_noalloc(solver._h, C.c_void_p(dx.data_ptr()), X.shape[1],
                                                         C.c_void_p(dy.data_ptr()), stream)
    assert rc == 0, _lib.last_error()
    torch.cuda.synchronize()  # the call only queues work
    return dy.cpu().numpy().T


def _rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


# (solver config, weighted, tolerance against the allocating apply of the same solver):
# the allocating apply runs the observation pass in FP64 (1e-13: only the order of the
# atomic additions differs), the CSR SpMV of the assembled Gramian in FP64 (1e-12: a
# different summation order), or the observation pass in FP32 (1e-6).
CASES = {
    "fp64_weighted": (lambda: wb.CG(), True, 1e-13),
    "fp64_unweighted": (lambda: wb.CG(), False, 1e-13),
    "mixed_weighted": (lambda: wb.CG(precision="mixed"), True, 1e-6),
    "explicit_weighted": (lambda: wb.CG(operator=wb.OperatorRepr.Explicit), True, 1e-12),
}


@pytest.mark.parametrize("case", list(CASES))
def test_noalloc_matches_allocating_apply_on_two_calls(case):
    import torch
    cfg, weighted, tol = CASES[case]
    cats, _, _ = synthetic.config2(scale=0.02)
    w = np.random.default_rng(1).lognormal(0.0, 1.0, cats.shape[0]) if weighted else None
    s = wb.Solver(cats, cfg(), weights=w)
    o = oracle.OracleSolver(cats, w)
    rng = np.random.default_rng(7)
    streams = [None, C.c_void_p(torch.cuda.current_stream().cuda_stream)]
    for call in range(2):  # the second call reuses the scratch the first one left behind
        X = rng.standard_normal((s.n_dofs, 5 + 4 * call))
        got = _noalloc(s, X, streams[call])
        ref = s.apply_gramian(X)
        for c in range(X.shape[1]):
            assert _rel(got[:, c], ref[:, c]) < tol
            assert _rel(got[:, c], o.apply_gramian(X[:, c])) < 1e-13


def test_noalloc_rejects_sizes_beyond_its_scratch():
    cats = synthetic.uniform_design(50_000, [40_000, 30_000], seed=3)
    s = wb.Solver(cats, preconditioner=wb.Preconditioner.Off)  # n_dofs = 70k: 2 x 70k x 16 > 2^21
    import torch
    dx = torch.zeros((16, s.n_dofs), dtype=torch.float64, device="cuda")
    dy = torch.zeros_like(dx)
    L = _lib.load()
    rc = L.within_solver_apply_gramian_noalloc(s._h, C.c_void_p(dx.data_ptr()), 16, C.c_void_p(dy.data_ptr()), None)
    assert rc == 9 and "too large for the no-allocation path" in _lib.last_error()
    rc = L.within_solver_apply_gramian_noalloc(s._h, C.c_void_p(dx.data_ptr()), 33, C.c_void_p(dy.data_ptr()), None)
    assert rc == 9 and "at most 32" in _lib.last_error()


def test_noalloc_rejects_a_preconditioner_only_handle():
    """A handle rebuilt from preconditioner bytes has no design: the call is refused on
    the host before any launch."""
    import torch
    cats = synthetic.uniform_design(20_000, [300, 100], seed=5)
    s = wb.Solver(cats)
    p = wb.FePreconditioner(s.preconditioner()._bytes())
    dx = torch.zeros((4, s.n_dofs), dtype=torch.float64, device="cuda")
    dy = torch.zeros_like(dx)
    rc = _lib.load().within_solver_apply_gramian_noalloc(p._h, C.c_void_p(dx.data_ptr()), 4,
                                                         C.c_void_p(dy.data_ptr()), None)
    assert rc == 9 and "holds only a preconditioner" in _lib.last_error()
