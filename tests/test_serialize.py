"""Preconditioner persistence: FePreconditioner pickling and FePreconditioner(bytes)
(within-py/src/lib.rs:890-913), Solver::with_preconditioner (within/src/solver.rs:433-446).

The CPU tests feed hand-made byte strings to the reader, which must reject every
malformed or inconsistent one on the host before anything reaches a device.  The GPU
tests round-trip real preconditioners and check that the rebuilt ones act identically.
"""
import pickle
import struct

import numpy as np
import pytest

import within_b200 as wb
from within_b200 import synthetic
from paritylib import rel


def _fnv(b: bytes) -> int:
    h = 1469598103934665603
    for x in b:
        h = ((h ^ x) * 1099511628211) & 0xFFFFFFFFFFFFFFFF
    return h


def _vec(fmt, vals):
    return struct.pack("<Q", len(vals)) + struct.pack("<%d%s" % (len(vals), fmt), *vals)


def _csr(nrows, ncols, ptr, idx, val):
    return struct.pack("<ii", nrows, ncols) + _vec("I", ptr) + _vec("I", idx) + _vec("d", val)


def _blob(ndofs=3, gidx=(0, 1, 2), kind=1, version=1, tamper=None):
    """One 1 x 2 subdomain (q-level 0 eliminated into two kept r-levels), dense factor."""
    head = b"WB200PC\0" + struct.pack("<I", version) + struct.pack("<qii", ndofs, kind, 0)
    head += struct.pack("<QIiQIi", 0, 1, 1, 0, 1, 24) + struct.pack("<Q", 1)
    sub = struct.pack("<iiiii", 0, 1, 1, 0, 2)                      # q, r, elim_q, kind, n_red
    sub += _vec("I", list(gidx)) + _vec("d", [])
    sub += _csr(1, 2, [0, 2], [0, 1], [1.0, 1.0]) + _csr(2, 1, [0, 1, 2], [0, 0], [1.0, 1.0])
    sub += _vec("d", [2.0]) + _vec("d", [1.0, 1.0]) + _vec("d", [0.5]) + _vec("d", [1.0])
    sub += struct.pack("<iiii", 0, 0, 0, 0) + _vec("i", []) * 4 + _vec("d", []) * 2 + _vec("i", []) + _vec("d", [])
    tail = _vec("q", []) + _vec("I", []) + _vec("d", [])
    body = head + sub + tail
    if tamper:
        body = tamper(body)
    return body + struct.pack("<Q", _fnv(body))


def _reject(data, what):
    with pytest.raises(ValueError, match=what):
        wb.FePreconditioner(data)


def test_reader_rejects_malformed_bytes():
    _reject(b"", "too short")
    _reject(b"not a preconditioner at all", "not a serialized preconditioner")
    good = _blob()
    flipped = bytearray(good)
    flipped[40] ^= 0xFF
    _reject(bytes(flipped), "checksum")
    _reject(good[:-9] + good[-8:], "checksum")
    _reject(_blob(version=7), "unsupported version")
    _reject(_blob(gidx=(0, 1, 3)), "global indices")           # a dof beyond n_dofs
    _reject(_blob(ndofs=0), "dof count")
    _reject(_blob(kind=5), "preconditioner kind")
    _reject(_blob(tamper=lambda b: b[:-10]), "truncated|trailing")
    # a CSR column beyond the block's columns
    _reject(_blob(tamper=lambda b: b.replace(_csr(1, 2, [0, 2], [0, 1], [1.0, 1.0]),
                                             _csr(1, 2, [0, 2], [0, 2], [1.0, 1.0]))), "cross-tab")


def test_reader_accepts_a_consistent_blob_up_to_the_device():
    # a well-formed blob passes every check; without a GPU only the device step fails
    import torch
    if torch.cuda.is_available():
        p = wb.FePreconditioner(_blob())
        assert p.nrows == 3 and p.n_subdomains == 1
    else:
        with pytest.raises(ValueError, match="CUDA device"):
            wb.FePreconditioner(_blob())


DESIGNS = {
    "uniform3w": lambda: (synthetic.uniform_design(60_000, [700, 250, 25], seed=1),
                          np.random.default_rng(5).lognormal(0, 1, 60_000)),
    "akm": lambda: synthetic.config2(scale=0.04)[0::2],
}


@pytest.mark.gpu
@pytest.mark.parametrize("name", list(DESIGNS))
@pytest.mark.parametrize("kind", ["additive", "multiplicative"])
def test_pickle_round_trip(name, kind):
    cats, w = DESIGNS[name]()
    cfg = wb.CG() if kind == "additive" else wb.GMRES()
    pre = None if kind == "additive" else wb.Preconditioner.Multiplicative
    s = wb.Solver(cats, cfg, weights=w, preconditioner=pre)
    p = s.preconditioner()
    q = pickle.loads(pickle.dumps(p))
    assert isinstance(q, wb.FePreconditioner) and q.nrows == p.nrows == s.n_dofs
    assert q.n_subdomains == p.n_subdomains and repr(q) == repr(p)
    assert q.subdomain_inner_parallel_work == p.subdomain_inner_parallel_work
    # same factors, same kernels; the applies add subdomain results with atomics, so two
    # applies of one preconditioner already differ in the last bits: tolerance 1e-10
    R = np.random.default_rng(2).standard_normal((s.n_dofs, 5))
    for c in range(5):
        assert rel(q.apply(R[:, c]), p.apply(R[:, c])) < 1e-10
    # a solver that reuses the preconditioner solves as the one that built it
    y = np.random.default_rng(3).standard_normal(cats.shape[0])
    r0 = s.solve(y)
    s2 = wb.Solver(cats, cfg, weights=w, preconditioner=q)
    r1 = s2.solve(y)
    assert r1.converged and abs(r1.iterations - r0.iterations) <= 1
    assert rel(r1.demeaned, r0.demeaned) < 1e-8
    if kind == "additive":
        assert repr(q.additive_schwarz_diagnostics()) == repr(p.additive_schwarz_diagnostics())
    else:
        assert q.additive_schwarz_diagnostics() is None


@pytest.mark.gpu
def test_reuse_across_precisions_and_errors():
    cats, w = DESIGNS["uniform3w"]()
    p = wb.Solver(cats, weights=w).preconditioner()
    data = pickle.dumps(p)
    Y = np.asfortranarray(np.random.default_rng(4).standard_normal((cats.shape[0], 4)))
    b0 = wb.Solver(cats, wb.CG(precision="mixed"), weights=w).solve_batch(Y)
    b1 = wb.Solver(cats, wb.CG(precision="mixed"), weights=w, preconditioner=pickle.loads(data)).solve_batch(Y)
    for c in range(4):
        assert rel(b1.demeaned[:, c], b0.demeaned[:, c]) < 1e-8
    # a preconditioner for another design (other dof count) is rejected
    other = synthetic.uniform_design(20_000, [300, 90, 7], seed=2)
    with pytest.raises(ValueError, match="dofs"):
        wb.Solver(other, preconditioner=pickle.loads(data))
    # the bytes-only handle applies but does not solve
    q = pickle.loads(data)
    with pytest.raises(ValueError, match="only a preconditioner"):
        wb._lib.load()  # the handle rejects operator applies through the C ABI
        from within_b200 import _apply_handle
        _apply_handle(q._h, "within_solver_apply_gramian", np.zeros(q.nrows), q.nrows)
    # no preconditioner, nothing to serialize
    assert wb.Solver(cats, preconditioner=wb.Preconditioner.Off).preconditioner() is None


def test_reader_fuzz():
    """Random mutations of a consistent blob, checksum re-signed so that the structural
    checks are reached: every outcome is a ValueError (malformed bytes, or on a machine
    without a GPU the device step) or, with a GPU, a handle; never a crash.  The dof
    count is left alone: it is taken as given (it may exceed the subdomains' dofs when
    levels are unobserved), and it sizes the handle's arrays."""
    import torch
    rng = np.random.default_rng(0)
    good = bytearray(_blob()[:-8])
    for trial in range(300):
        b = bytearray(good)
        for _ in range(int(rng.integers(1, 4))):
            # every byte after the magic except the dof count (bytes 12-19): the reader
            # bounds every index by it, and a bytes-only handle sizes host arrays by it
            pos = int(rng.integers(8, len(b) - 8))
            pos = pos + 8 if pos >= 12 else pos
            b[pos] = int(rng.integers(0, 256))
        if rng.random() < 0.2:  # also truncate or extend
            cut = int(rng.integers(8, len(b)))
            b = b[:cut] if rng.random() < 0.5 else b + bytes(int(rng.integers(1, 64)))
        data = bytes(b) + struct.pack("<Q", _fnv(bytes(b)))
        try:
            p = wb.FePreconditioner(data)
            assert torch.cuda.is_available() and p.nrows > 0
        except ValueError:
            pass
