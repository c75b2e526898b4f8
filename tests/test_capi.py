"""The C-ABI library loads and exports every symbol include/within_b200.h declares;
host-side validation works without a device."""
import ctypes as C
import os
import re

import numpy as np
import pytest

import within_b200 as wb
from within_b200 import _lib
from conftest import ROOT


def header_symbols():
    text = open(os.path.join(ROOT, "include", "within_b200.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(within_\w+)\s*\(", text)))


def test_library_exports_every_header_symbol():
    L = _lib.load()
    syms = header_symbols()
    assert len(syms) >= 20
    missing = [s for s in syms if not hasattr(L, s)]
    assert not missing, missing
    assert sorted(_lib.EXPORTED) == syms


def test_defaults_match_reference():
    p = _lib.Params()
    _lib.load().within_default_params(C.byref(p))
    assert (p.krylov, p.tol, p.maxiter, p.max_refinements, p.gmres_restart) == (0, 1e-8, 1000, 2, 30)
    q = _lib.Precond()
    _lib.load().within_default_preconditioner(C.byref(q))
    # LocalSolverConfig::solver_default(): split_merge 2, approx Schur (seed 0, split 1), dense 24
    assert (q.kind, q.approx_chol_split, q.approx_schur_enabled, q.approx_schur_split, q.dense_threshold) == (1, 2, 1, 1, 24)


def test_config_validation_before_device():
    cats = np.zeros((4, 2), dtype=np.uint32, order="F")
    with pytest.raises(ValueError, match="CG requires a symmetric preconditioner"):
        wb.Solver(cats, wb.CG(), preconditioner=wb.Preconditioner.Multiplicative)
    with pytest.raises(TypeError):
        wb.Solver(cats, config="cg")
    with pytest.raises(TypeError):
        wb.Solver(cats, preconditioner="additive")
    with pytest.raises(TypeError):
        wb.Solver(cats, preconditioner=wb.AdditiveSchwarz(local_solver=object()))
    with pytest.raises(ValueError):
        wb.ApproxCholConfig(split=0)
    with pytest.raises(ValueError):
        wb.CG(precision="fp16")
    with pytest.raises(TypeError):  # 1-D categories (reference tests/test_error_handling.py:51-56)
        wb.Solver(np.zeros(4, np.uint32))
    with pytest.raises(wb.WithinError, match="weights has length 3, expected 4"):
        wb.Solver(cats, weights=np.ones(3))


def test_empty_observations_error():
    with pytest.raises(wb.WithinError, match="no observations") as e:
        wb.Solver(np.zeros((0, 2), np.uint32, order="F"))
    assert e.value.kind == "EmptyObservations"


def test_c_order_warning():
    cats = np.zeros((4, 2), dtype=np.uint32)  # C-order
    with pytest.warns(UserWarning, match="not F-contiguous"):
        try:
            wb.Solver(cats, preconditioner=wb.Preconditioner.Off)
        except wb.WithinError:
            pass  # no device here


def test_no_device_fails_loudly():
    import torch
    if torch.cuda.is_available():
        pytest.skip("device present")
    cats = np.asfortranarray(np.array([[0, 0], [1, 1], [0, 1]], np.uint32))
    with pytest.raises(wb.WithinError) as e:
        wb.Solver(cats)
    assert e.value.kind == "Cuda"
