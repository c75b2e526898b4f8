"""The Gramian apply that allocates nothing, checked against the one that allocates.

within_solver_apply_gramian_noalloc is for callers that cannot allocate device memory
while they run: code inside a CUDA stream capture (an allocation there breaks the
capture), code under a fixed device-memory budget or a custom allocator.  Its working
space is a static device array instead of cudaMalloc'd buffers.  This file is named to
be collected last.
"""
import ctypes as C

import numpy as np
import pytest

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


def test_noalloc_matches_allocating_apply_on_two_calls():
    import torch
    cats, _, w = synthetic.config2(scale=0.02)
    w = np.random.default_rng(1).lognormal(0.0, 1.0, cats.shape[0])
    s = wb.Solver(cats, weights=w)  # FP64 solver, additive Schwarz
    rng = np.random.default_rng(7)
    streams = [None, C.c_void_p(torch.cuda.current_stream().cuda_stream)]
    for call in range(2):  # the second call reuses the scratch the first one left behind
        X = rng.standard_normal((s.n_dofs, 5 + 4 * call))
        got = _noalloc(s, X, streams[call])
        ref = s.apply_gramian(X)
        for c in range(X.shape[1]):
            assert _rel(got[:, c], ref[:, c]) < 1e-13


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
