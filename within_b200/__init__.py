"""B200-native solve phase of `within` with the `within_py` Python API.

Mirrors ``within`` (python/within/__init__.py, within-py/src/lib.rs:62-1074):
``solve``, ``solve_batch``, ``Solver``, the configuration classes ``CG``,
``GMRES``, ``AdditiveSchwarz``, ``MultiplicativeSchwarz``, ``SchurComplement``,
``ApproxCholConfig``, ``ApproxSchurConfig`` and the enums ``OperatorRepr``,
``Preconditioner``, ``ReductionStrategy``.  Every solve runs on the current CUDA
device through ``libwithin_b200.so``; invalid input raises ``ValueError``, a bad
configuration type ``TypeError`` (as within-py does, lib.rs:480-483, 516, 590).

Additions: ``CG``/``GMRES`` take ``precision="fp64"`` (the drop-in: every
step in FP64) or ``precision="mixed"`` (FP32 operator and Schwarz applies inside
an FP64 iterative-refinement loop; same tolerance on the FP64 residual);
``Solver.set_coarse_space`` adds a coarse space to CG's preconditioner (a basis, or
the message-passing network of ``within_b200.coarse``).
"""
from __future__ import annotations

import ctypes as C
import time
import warnings
from enum import IntEnum

import numpy as np

from . import _lib

__all__ = [
    "OperatorRepr", "Preconditioner", "ReductionStrategy", "CG", "GMRES", "LSMR", "ApproxCholConfig",
    "ApproxSchurConfig", "SchurComplement", "AdditiveSchwarz", "MultiplicativeSchwarz", "SolveResult",
    "BatchSolveResult", "AdditiveSchwarzDiagnostics", "FePreconditioner", "Solver", "solve", "solve_batch", "solve_many", "WithinError",
]


class WithinError(ValueError):
    """Error raised by the native library (a ValueError, like within-py's errors)."""

    def __init__(self, code: int, message: str):
        super().__init__(message)
        self.code = code
        self.kind = _lib.ERR_NAMES.get(code, "Unknown")


class OperatorRepr(IntEnum):
    Implicit = 0
    Explicit = 1


class Preconditioner(IntEnum):
    Additive = 0
    Multiplicative = 1
    Off = 2


class ReductionStrategy(IntEnum):
    Auto = 0
    AtomicScatter = 1
    ParallelReduction = 2


_PRECISIONS = {"fp64": 0, "mixed": 1}


class CG:
    """Conjugate gradient on the normal equations (within-py CG, lib.rs:262-300)."""

    def __init__(self, tol: float = 1e-8, maxiter: int = 1000, operator: OperatorRepr = OperatorRepr.Implicit,
                 max_refinements: int = 2, precision: str = "fp64"):
        if precision not in _PRECISIONS:
            raise ValueError("precision must be 'fp64' or 'mixed'")
        self.tol, self.maxiter, self.operator = float(tol), int(maxiter), OperatorRepr(operator)
        self.max_refinements, self.precision = int(max_refinements), precision

    def __repr__(self):
        return f"CG(tol={self.tol}, maxiter={self.maxiter}, operator={self.operator.name}, precision={self.precision!r})"


class GMRES:
    """Right-preconditioned GMRES(restart) (within-py GMRES, lib.rs:302-346)."""

    def __init__(self, tol: float = 1e-8, maxiter: int = 1000, restart: int = 30,
                 operator: OperatorRepr = OperatorRepr.Implicit, max_refinements: int = 2,
                 precision: str = "fp64"):
        if precision not in _PRECISIONS:
            raise ValueError("precision must be 'fp64' or 'mixed'")
        self.tol, self.maxiter, self.restart = float(tol), int(maxiter), int(restart)
        self.operator, self.max_refinements, self.precision = OperatorRepr(operator), int(max_refinements), precision

    def __repr__(self):
        return f"GMRES(tol={self.tol}, maxiter={self.maxiter}, restart={self.restart})"


class LSMR:
    """Modified LSMR on the rectangular problem min ||W^(1/2)(y - D x)|| (within-py LSMR,
    lib.rs:399-425; schwarz-precond/src/solve/lsmr.rs).  Runs in FP64 with no iterative
    refinement; with a preconditioner, one M^-1 apply per iteration."""

    def __init__(self, tol: float = 1e-8, maxiter: int = 1000, local_size: int | None = None):
        if local_size is not None and int(local_size) < 0:
            raise OverflowError("local_size must be a non-negative integer")
        self.tol, self.maxiter = float(tol), int(maxiter)
        self.local_size = None if local_size is None else int(local_size)

    def __repr__(self):
        return f"LSMR(tol={self.tol}, maxiter={self.maxiter}, local_size={self.local_size})"


class ApproxCholConfig:
    """Approximate Cholesky parameters; split > 1 means split_merge=Some(split) (lib.rs:62-98)."""

    def __init__(self, seed: int = 0, split: int = 1):
        if split < 1:
            raise ValueError("split must be >= 1")
        self.seed, self.split = int(seed), int(split)


class ApproxSchurConfig:
    """Sampled Schur complement parameters (lib.rs:100-128)."""

    def __init__(self, seed: int = 0, split: int = 1):
        if split < 1:
            raise ValueError("split must be >= 1")
        self.seed, self.split = int(seed), int(split)


class SchurComplement:
    """Local solver: Schur complement + approximate Cholesky (lib.rs:130-180)."""

    def __init__(self, approx_chol: ApproxCholConfig | None = None, approx_schur: ApproxSchurConfig | None = None,
                 dense_threshold: int = 24):
        self.approx_chol, self.approx_schur, self.dense_threshold = approx_chol, approx_schur, int(dense_threshold)


class AdditiveSchwarz:
    def __init__(self, local_solver: SchurComplement | None = None,
                 reduction: ReductionStrategy = ReductionStrategy.Auto):
        self.local_solver, self.reduction = local_solver, ReductionStrategy(reduction)


class MultiplicativeSchwarz:
    def __init__(self, local_solver: SchurComplement | None = None):
        self.local_solver = local_solver


def _default_local() -> _lib.Precond:
    p = _lib.Precond()
    _lib.load().within_default_preconditioner(C.byref(p))  # LocalSolverConfig::solver_default()
    return p


def _local_config(p: _lib.Precond, local) -> None:
    if local is None:
        return
    if not isinstance(local, SchurComplement):
        raise TypeError("local_solver must be SchurComplement or None")
    ac = local.approx_chol or ApproxCholConfig()   # unwrap_or_default: seed 0, split_merge None
    p.approx_chol_seed, p.approx_chol_split = ac.seed, ac.split
    if local.approx_schur is None:
        p.approx_schur_enabled = 0
    else:
        p.approx_schur_enabled, p.approx_schur_seed = 1, local.approx_schur.seed
        p.approx_schur_split = local.approx_schur.split
    p.dense_threshold = local.dense_threshold


def _precond_struct(preconditioner):
    """extract_preconditioner_config (within-py/src/lib.rs:542-594)."""
    if isinstance(preconditioner, FePreconditioner):
        raise TypeError("a built FePreconditioner applies to one design: pass it to Solver(...)")
    p = _default_local()
    if preconditioner is None:
        return p
    if isinstance(preconditioner, Preconditioner):
        if preconditioner == Preconditioner.Off:
            p.kind = 0
        elif preconditioner == Preconditioner.Multiplicative:
            p.kind = 2
        return p
    if isinstance(preconditioner, AdditiveSchwarz):
        _local_config(p, preconditioner.local_solver)
        p.kind, p.reduction_strategy = 1, int(preconditioner.reduction)
        return p
    if isinstance(preconditioner, MultiplicativeSchwarz):
        _local_config(p, preconditioner.local_solver)
        p.kind = 2
        return p
    raise TypeError("preconditioner must be Preconditioner.Additive, Preconditioner.Multiplicative, "
                    "Preconditioner.Off, AdditiveSchwarz(...), MultiplicativeSchwarz(...), or None")


def _params_struct(config):
    p = _lib.Params()
    _lib.load().within_default_params(C.byref(p))
    if config is None:
        return p
    if isinstance(config, LSMR):  # extract_solver_params (lib.rs:621-632)
        p.krylov, p.lsmr_local_size = 2, config.local_size or 0
        p.tol, p.maxiter, p.max_refinements = config.tol, config.maxiter, 0
        return p
    if isinstance(config, CG):
        p.krylov = 0
    elif isinstance(config, GMRES):
        p.krylov, p.gmres_restart = 1, config.restart
    else:
        raise TypeError("config must be CG, GMRES, or LSMR")
    p.operator_repr, p.tol, p.maxiter = int(config.operator), config.tol, config.maxiter
    p.max_refinements, p.precision = config.max_refinements, _PRECISIONS[config.precision]
    return p


def _validate(params, pre) -> None:
    """validate_cg_preconditioner (within-py/src/lib.rs:639-656)."""
    if params.krylov in (0, 2) and pre.kind == 2:
        method = "CG" if params.krylov == 0 else "LSMR"
        raise ValueError(f"{method} requires a symmetric preconditioner; use 'additive' or switch to GMRES")


def _categories(categories) -> np.ndarray:
    cats = np.asarray(categories)
    if cats.ndim != 2:  # within-py extracts a 2-D uint32 array (a TypeError otherwise)
        raise TypeError("categories must be a 2-D array of shape (n_obs, n_factors)")
    if cats.dtype != np.uint32:
        raise TypeError("categories must have dtype uint32")
    if cats.strides[0] != cats.itemsize and cats.shape[0] > 1 and cats.shape[1] > 1:
        warnings.warn("categories array is not F-contiguous (column-major). "
                      "Use np.asfortranarray(categories) for faster solves.", UserWarning, stacklevel=3)
    return cats


def _f64(a, name):
    """A float64 array; other numpy dtypes are a TypeError, as within-py's float64 array
    arguments are (lists and scalars are converted)."""
    if isinstance(a, np.ndarray) and a.dtype != np.float64:
        raise TypeError(f"{name} must have dtype float64, got {a.dtype}")
    return np.asarray(a, dtype=np.float64)


def _check(rc: int) -> None:
    if rc != _lib.WITHIN_OK:
        raise WithinError(rc, _lib.last_error())


class SolveResult:
    """Single-RHS result (orchestrate.rs:37-54; within-py SolveResult)."""

    def __init__(self, x, demeaned, converged, iterations, residual, time_total, time_setup, time_solve):
        self.x, self.demeaned, self.converged = x, demeaned, bool(converged)
        self.iterations, self.residual = int(iterations), float(residual)
        self.time_total, self.time_setup, self.time_solve = time_total, time_setup, time_solve

    def __repr__(self):
        return (f"SolveResult(converged={self.converged}, iterations={self.iterations}, "
                f"residual={self.residual:.3e})")


class BatchSolveResult:
    """Batch result: x (n_dofs, k) and demeaned (n_obs, k) F-order (within-py lib.rs:690-714)."""

    def __init__(self, x, demeaned, converged, iterations, residual, time_solve, time_total):
        self.x, self.demeaned = x, demeaned
        self.converged, self.iterations, self.residual = converged, iterations, residual
        self.time_solve, self.time_total = time_solve, time_total

    def __repr__(self):
        return f"BatchSolveResult(n_rhs={len(self.converged)}, converged={self.converged})"


class AdditiveSchwarzDiagnostics:
    """Build-time scheduling metrics of an additive Schwarz preconditioner
    (within-py PyAdditiveSchwarzDiagnostics, lib.rs:200-260; planning.rs:141-210).

    ``resolved_reduction_strategy`` is what the reference's CPU scheduler would pick for
    this build with one worker thread per host core (planning.rs:71-135).  The device
    executor has a single reduction (atomic adds of the subdomain results), whichever
    strategy is configured.
    """

    def __init__(self, d: "_lib.AdditiveDiagnostics"):
        self.reduction_strategy = ReductionStrategy(d.reduction_strategy)
        self.resolved_reduction_strategy = ReductionStrategy(d.resolved_reduction_strategy)
        self.total_inner_parallel_work = int(d.total_inner_parallel_work)
        self.max_inner_parallel_work = int(d.max_inner_parallel_work)
        self.total_scatter_dofs = int(d.total_scatter_dofs)
        self.outer_parallel_capacity = float(d.outer_parallel_capacity)
        self.scatter_overlap = float(d.scatter_overlap)

    def __repr__(self):
        return (f"AdditiveSchwarzDiagnostics(reduction_strategy={self.reduction_strategy.name}, "
                f"resolved_reduction_strategy={self.resolved_reduction_strategy.name}, "
                f"total_inner_parallel_work={self.total_inner_parallel_work}, "
                f"max_inner_parallel_work={self.max_inner_parallel_work}, "
                f"total_scatter_dofs={self.total_scatter_dofs}, "
                f"outer_parallel_capacity={self.outer_parallel_capacity:.3f}, "
                f"scatter_overlap={self.scatter_overlap:.3f})")


class FePreconditioner:
    """A built Schwarz preconditioner (within-py PyFePreconditioner, lib.rs:825-914).

    Obtained from ``Solver.preconditioner()``, or rebuilt from bytes with
    ``FePreconditioner(data)``, which is what ``pickle`` calls (``__reduce__``).  Passing
    it to ``Solver(..., preconditioner=p)`` reuses its factors instead of building them
    (``Solver::with_preconditioner``); the design must have the same number of dofs.  The
    bytes are this library's own format (see ``within_solver_preconditioner_bytes``).
    """

    def __init__(self, data: bytes):
        data = bytes(data)
        h = C.c_void_p()
        buf = (C.c_ubyte * len(data)).from_buffer_copy(data) if data else None
        rc = _lib.load().within_preconditioner_from_bytes(buf, len(data), C.byref(h))
        if rc != _lib.WITHIN_OK:
            raise ValueError(_lib.last_error())
        self._h, self._solver, self._own, self._data = h, None, True, data

    @classmethod
    def _of(cls, solver: "Solver") -> "FePreconditioner":
        p = cls.__new__(cls)
        p._h, p._solver, p._own, p._data = solver._h, solver, False, None
        return p

    def __del__(self):
        if getattr(self, "_own", False) and getattr(self, "_h", None):
            _lib.load().within_solver_free(self._h)
            self._h = None

    def _bytes(self) -> bytes:
        if self._data is None:
            L = _lib.load()
            n = C.c_size_t(0)
            _check(L.within_solver_preconditioner_bytes(self._h, None, C.byref(n)))
            buf = (C.c_ubyte * n.value)()
            _check(L.within_solver_preconditioner_bytes(self._h, buf, C.byref(n)))
            self._data = bytes(buf)
        return self._data

    def __reduce__(self):
        return (FePreconditioner, (self._bytes(),))

    @property
    def _kind(self) -> int:
        return int(_lib.load().within_solver_preconditioner_kind(self._h))

    def apply(self, x) -> np.ndarray:
        return _apply_handle(self._h, "within_solver_apply_preconditioner", x, self.nrows)

    @property
    def nrows(self) -> int:
        return int(_lib.load().within_solver_n_dofs(self._h))

    @property
    def ncols(self) -> int:
        return self.nrows

    @property
    def n_subdomains(self) -> int:
        return int(_lib.load().within_solver_n_subdomains(self._h))

    @property
    def subdomain_inner_parallel_work(self) -> list[int]:
        """Per-subdomain inner parallel work estimate (preconditioner.rs:64-79)."""
        work = np.zeros(self.n_subdomains, np.int64)
        _lib.load().within_solver_subdomain_inner_work(self._h, work)
        return [int(v) for v in work]

    def additive_schwarz_diagnostics(self) -> AdditiveSchwarzDiagnostics | None:
        """Diagnostics if this is an additive preconditioner, else None (preconditioner.rs:98-106)."""
        if self._kind != 1:
            return None
        d = _lib.AdditiveDiagnostics()
        _check(_lib.load().within_solver_additive_diagnostics(self._h, 0, C.byref(d)))
        return AdditiveSchwarzDiagnostics(d)

    def __repr__(self):
        kind = {1: "Additive", 2: "Multiplicative"}.get(self._kind, "Off")
        return f"FePreconditioner({kind}, n={self.nrows})"


def _apply_handle(h, fn, v, rows, in_rows=None):
    """out (rows x k) = fn(v); v has in_rows rows (default: rows), else a ValueError."""
    v = np.asarray(v, dtype=np.float64)
    one = v.ndim == 1
    want = rows if in_rows is None else in_rows
    if v.ndim not in (1, 2) or v.shape[0] != want:
        raise ValueError(f"expected {want} rows, got shape {v.shape}")
    V = np.asfortranarray(v.reshape(v.shape[0], -1))
    out = np.empty((rows, V.shape[1]), order="F")
    _check(getattr(_lib.load(), fn)(h, _lib.ptr(V), V.shape[1], _lib.ptr(out)))
    return out[:, 0] if one else out


class Solver:
    """Persistent solver (Solver::new / solve / solve_batch, within/src/solver.rs:82-447)."""

    def __init__(self, categories, config=None, weights=None, preconditioner=None):
        t0 = time.perf_counter()
        L = _lib.load()
        cats = _categories(categories)
        self._params = _params_struct(config)
        built = isinstance(preconditioner, FePreconditioner)
        if not built:  # a built preconditioner skips the configuration checks (lib.rs:963-972)
            self._pre = _precond_struct(preconditioner)
            _validate(self._params, self._pre)
        n, q = cats.shape
        self._w = None
        if weights is not None:
            self._w = np.ascontiguousarray(_f64(weights, "weights"))
            if self._w.ndim != 1 or self._w.shape[0] != n:
                raise WithinError(3, f"weights has length {self._w.shape[0] if self._w.ndim else 0}, expected {n}")
        isz = cats.itemsize
        h = C.c_void_p()
        if built:  # Solver::with_preconditioner (solver.rs:433-446)
            data = preconditioner._bytes()
            buf = (C.c_ubyte * len(data)).from_buffer_copy(data)
            rc = L.within_solver_new_with_preconditioner(cats.ctypes.data_as(C.c_void_p), n, q, cats.strides[0] // isz,
                                                         cats.strides[1] // isz, _lib.ptr(self._w),
                                                         C.byref(self._params), buf, len(data), C.byref(h))
        else:
            pre = None if self._pre.kind == 0 else C.byref(self._pre)
            rc = L.within_solver_new(cats.ctypes.data_as(C.c_void_p), n, q, cats.strides[0] // isz,
                                     cats.strides[1] // isz, _lib.ptr(self._w), C.byref(self._params), pre,
                                     C.byref(h))
        _check(rc)
        self._h = h
        self.n_obs, self.n_dofs, self.n_factors = n, int(L.within_solver_n_dofs(h)), q
        self.time_setup = time.perf_counter() - t0

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            _lib.load().within_solver_free(h)
            self._h = None

    def _y(self, y, ndim):
        y = _f64(y, "y")
        if y.ndim != ndim:
            raise ValueError(f"expected a {ndim}-D array")
        if y.shape[0] != self.n_obs:
            raise WithinError(2, f"y has {y.shape[0]} observations, expected {self.n_obs}")
        return y

    def solve(self, y) -> SolveResult:
        y = np.ascontiguousarray(self._y(y, 1))
        x = np.empty(self.n_dofs)
        d = np.empty(self.n_obs)
        st = _lib.Stats()
        _check(_lib.load().within_solver_solve(self._h, _lib.ptr(y), _lib.ptr(x), _lib.ptr(d), C.byref(st)))
        return SolveResult(x, d, st.converged, st.iterations, st.final_residual, st.time_total,
                           self.time_setup, st.time_solve)

    def solve_batch(self, Y) -> BatchSolveResult:
        Y = np.asfortranarray(self._y(Y, 2))
        k = Y.shape[1]
        x = np.empty((self.n_dofs, k), order="F")
        d = np.empty((self.n_obs, k), order="F")
        st = (_lib.Stats * max(k, 1))()
        _check(_lib.load().within_solver_solve_batch(self._h, _lib.ptr(Y), k, _lib.ptr(x), _lib.ptr(d), st))
        return BatchSolveResult(x, d, [bool(st[c].converged) for c in range(k)],
                                [int(st[c].iterations) for c in range(k)],
                                [float(st[c].final_residual) for c in range(k)],
                                [float(st[c].time_solve) for c in range(k)], float(st[0].time_total) if k else 0.0)

    def preconditioner(self) -> FePreconditioner | None:
        return None if _lib.load().within_solver_preconditioner_kind(self._h) == 0 else FePreconditioner._of(self)

    # --- operator access (kernel-level parity checks) ---
    def _apply(self, fn, v, out_rows=None, in_rows=None):
        return _apply_handle(self._h, fn, v, out_rows or self.n_dofs, in_rows or self.n_dofs)

    def apply_gramian(self, x):
        return self._apply("within_solver_apply_gramian", x)

    def matvec_d(self, x):
        return self._apply("within_solver_matvec_d", x, self.n_obs)

    def rmatvec_wdt(self, r):
        return self._apply("within_solver_rmatvec_wdt", r, self.n_dofs, self.n_obs)

    def factor_meta(self):
        nl = np.zeros(self.n_factors, np.int64)
        off = np.zeros(self.n_factors, np.int64)
        _lib.load().within_solver_factor_meta(self._h, nl, off)
        return nl, off

    def subdomains(self):
        """Setup structure in the oracle's format (pair, indices, weights, factors)."""
        L = _lib.load()
        out = []
        for i in range(L.within_solver_n_subdomains(self._h)):
            info = np.zeros(8, np.int64)
            L.within_solver_subdomain_info(self._h, i, info)
            q, r, nloc, nq, nr, eq, kind, nred = (int(v) for v in info)
            g = np.zeros(nloc, np.uint32)
            w = np.zeros(nloc)
            L.within_solver_subdomain_indices(self._h, i, g, w)
            d = dict(pair=(q, r), global_indices=g, pou=w, n_q=nq, n_r=nr, eliminate_q=bool(eq),
                     reduced_kind="dense" if kind == 0 else "ac", n_reduced=nred)
            if kind == 1:
                sz = np.zeros(5, np.int64)
                L.within_solver_ac_sizes(self._h, i, sz)
                n, nlev, nnz, ncol, ncore = (int(v) for v in sz)
                lp = np.zeros(nlev + 1, np.int32); cv = np.zeros(max(ncol, 1), np.int32)
                cd = np.zeros(max(ncol, 1)); cp = np.zeros(ncol + 1, np.int32)
                ci = np.zeros(max(nnz, 1), np.int32); cc = np.zeros(max(nnz, 1))
                core = np.zeros(max(ncore, 1), np.int32); z = np.zeros(max(ncore * ncore, 1))
                L.within_solver_ac_arrays(self._h, i, lp, cv, cd, cp, ci, cc, core, z)
                d["ac"] = dict(n=n, level_ptr=lp, col_vertex=cv[:ncol], col_diag=cd[:ncol], col_ptr=cp,
                               col_idx=ci[:nnz], col_coef=cc[:nnz], core_vertex=core[:ncore],
                               core_z=z[:ncore * ncore].reshape(ncore, ncore))
            out.append(d)
        return out

    @property
    def gpu_launches(self) -> int:
        return int(_lib.load().within_solver_gpu_launches(self._h))

    # --- coarse space for CG (an addition: the reference has none) ---
    def set_coarse_space(self, coarse) -> None:
        """CG's preconditioner becomes M^-1 r + Z (Z'GZ)^+ Z' r.  ``coarse``: a
        ``coarse.CoarseNet`` (its network is evaluated on this design on the GPU) or a
        basis (n_dofs x k array, k <= 32).  GMRES and LSMR ignore it."""
        from .coarse import CoarseNet
        L = _lib.load()
        if isinstance(coarse, CoarseNet):
            rc = L.within_solver_set_coarse_net(self._h, coarse.params.ctypes.data_as(C.c_void_p), coarse.params.size,
                                                coarse.seed)
        else:
            Z = np.asfortranarray(coarse, dtype=np.float64)
            if Z.ndim != 2 or Z.shape[0] != self.n_dofs:
                raise ValueError(f"a coarse basis has {self.n_dofs} rows")
            rc = L.within_solver_set_coarse_basis(self._h, _lib.ptr(Z), Z.shape[1])
        _check(rc)

    def clear_coarse_space(self) -> None:
        _check(_lib.load().within_solver_clear_coarse(self._h))

    def coarse_basis(self) -> np.ndarray:
        """The installed coarse basis (n_dofs x 32)."""
        Z = np.empty((self.n_dofs, 32), order="F")
        _check(_lib.load().within_solver_coarse_basis(self._h, _lib.ptr(Z)))
        return Z


def solve(categories, y, config=None, weights=None, preconditioner=None) -> SolveResult:
    """orchestrate::solve (within/src/orchestrate.rs:151-166)."""
    t0 = time.perf_counter()
    y = _f64(y, "y")  # argument types are checked before anything is built
    s = Solver(categories, config, weights, preconditioner)
    r = s.solve(y)
    r.time_setup = s.time_setup
    r.time_total = time.perf_counter() - t0
    return r


def solve_many(problems, config=None, preconditioner=None, concurrency: int = 0) -> list:
    """Many independent problems of uneven size, each like ``solve_batch``.

    ``problems`` is a sequence of ``(categories, Y)`` or ``(categories, Y, weights)``
    with Y of shape (n_obs, k) (or (n_obs,) for one RHS).  Up to ``concurrency``
    problems (0: one per host core) are solved at once, each with its own solver and
    CUDA stream, so that
    small problems share the GPU.  Returns one BatchSolveResult per problem; raises
    WithinError naming the first problem that failed.
    """
    L = _lib.load()
    params = _params_struct(config)
    pre = _precond_struct(preconditioner)
    _validate(params, pre)
    keep, arr = [], (_lib.Problem * max(len(problems), 1))()
    outs = []
    for i, prob in enumerate(problems):
        cats, Y = prob[0], prob[1]
        w = prob[2] if len(prob) > 2 else None
        cats = _categories(cats)
        n, q = cats.shape
        Y = np.asarray(Y, dtype=np.float64)
        Y = np.asfortranarray(Y.reshape(n, -1) if Y.ndim == 1 else Y)
        if Y.shape[0] != n:
            raise WithinError(2, f"problem {i}: y has {Y.shape[0]} observations, expected {n}")
        k = Y.shape[1]
        m = int(sum(int(cats[:, j].max()) + 1 for j in range(q))) if n > 0 else 0
        if w is not None:
            w = np.ascontiguousarray(w, dtype=np.float64)
            if w.ndim != 1 or w.shape[0] != n:
                raise WithinError(3, f"problem {i}: weights has length {w.shape[0] if w.ndim else 0}, expected {n}")
        x = np.empty((m, k), order="F")
        d = np.empty((n, k), order="F")
        st = (_lib.Stats * max(k, 1))()
        isz = cats.itemsize
        arr[i] = _lib.Problem(cats.ctypes.data, n, q, cats.strides[0] // isz, cats.strides[1] // isz,
                              w.ctypes.data if w is not None else None, Y.ctypes.data, k, x.ctypes.data, d.ctypes.data,
                              C.cast(st, C.c_void_p), 0)
        keep.append((cats, Y, w))
        outs.append((x, d, st, k))
    rc = L.within_solve_many(arr, len(problems), C.byref(params), None if pre.kind == 0 else C.byref(pre),
                             int(concurrency))
    _check(rc)
    res = []
    for x, d, st, k in outs:
        res.append(BatchSolveResult(x, d, [bool(st[c].converged) for c in range(k)],
                                    [int(st[c].iterations) for c in range(k)],
                                    [float(st[c].final_residual) for c in range(k)],
                                    [float(st[c].time_solve) for c in range(k)], float(st[0].time_total) if k else 0.0))
    return res


def solve_batch(categories, Y, config=None, weights=None, preconditioner=None) -> BatchSolveResult:
    """orchestrate::solve_batch (within/src/orchestrate.rs:172-184)."""
    t0 = time.perf_counter()
    Y = _f64(Y, "Y")
    s = Solver(categories, config, weights, preconditioner)
    r = s.solve_batch(Y)
    r.time_total = time.perf_counter() - t0
    return r


def shard_problems(sizes, world: int) -> list:
    """Assignment of independent problems to ``world`` ranks (one GPU each), balanced by
    observation count: the largest problem first, each to the rank with the least work
    so far (ties: the lowest rank).  ``sizes`` are the problems' observation counts.
    Returns one ascending index list per rank; together they hold every index once.

    Independent problems share nothing, so ranks solve their shards with no exchange
    (``solve_many`` on each); only the job's time is combined (its slowest rank's).
    """
    if world < 1:
        raise ValueError("world must be at least 1")
    load = [0] * world
    out = [[] for _ in range(world)]
    for i in sorted(range(len(sizes)), key=lambda j: (-int(sizes[j]), j)):
        r = min(range(world), key=lambda q: (load[q], q))
        out[r].append(i)
        load[r] += int(sizes[i])
    return [sorted(o) for o in out]
