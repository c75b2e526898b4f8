"""ctypes binding of libwithin_b200.so (the C ABI in include/within_b200.h).

The shared library is built in-tree by ``within_b200.build``.  There is no CPU
fallback: a missing library raises ImportError, a missing device makes every
solver call fail with a CUDA error.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libwithin_b200.so")

WITHIN_OK = 0
ERR_NAMES = {
    1: "EmptyObservations", 2: "ObservationCountMismatch", 3: "WeightCountMismatch", 4: "Overflow",
    5: "SingularDiagonal", 6: "LocalSolverBuild", 7: "PreconditionerBuild", 8: "IterativeSolve",
    9: "InvalidArgument", 10: "Cuda",
}


class Params(C.Structure):
    _fields_ = [("krylov", C.c_int32), ("gmres_restart", C.c_int32), ("operator_repr", C.c_int32),
                ("tol", C.c_double), ("maxiter", C.c_int32), ("max_refinements", C.c_int32),
                ("precision", C.c_int32), ("lsmr_local_size", C.c_int32)]


class Precond(C.Structure):
    _fields_ = [("kind", C.c_int32), ("approx_chol_seed", C.c_uint64), ("approx_chol_split", C.c_uint32),
                ("approx_schur_enabled", C.c_int32), ("approx_schur_seed", C.c_uint64),
                ("approx_schur_split", C.c_uint32), ("dense_threshold", C.c_int32),
                ("reduction_strategy", C.c_int32)]


class Stats(C.Structure):
    _fields_ = [("converged", C.c_int32), ("iterations", C.c_int32), ("final_residual", C.c_double),
                ("time_total", C.c_double), ("time_setup", C.c_double), ("time_solve", C.c_double)]


class Problem(C.Structure):
    _fields_ = [("codes", C.c_void_p), ("n_obs", C.c_size_t), ("n_factors", C.c_size_t),
                ("row_stride", C.c_int64), ("col_stride", C.c_int64), ("weights", C.c_void_p),
                ("ys", C.c_void_p), ("k", C.c_size_t), ("x", C.c_void_p), ("demeaned", C.c_void_p),
                ("stats", C.c_void_p), ("status", C.c_int32)]


class AdditiveDiagnostics(C.Structure):
    _fields_ = [("reduction_strategy", C.c_int32), ("resolved_reduction_strategy", C.c_int32),
                ("n_subdomains", C.c_int64), ("n_dofs", C.c_int64), ("total_inner_parallel_work", C.c_int64),
                ("max_inner_parallel_work", C.c_int64), ("total_scatter_dofs", C.c_int64),
                ("outer_parallel_capacity", C.c_double), ("scatter_overlap", C.c_double)]


_u32p = np.ctypeslib.ndpointer(dtype=np.uint32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_i32p = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_i64p = np.ctypeslib.ndpointer(dtype=np.int64, flags="C_CONTIGUOUS")

# Every symbol declared in include/within_b200.h.
EXPORTED = [
    "within_default_params", "within_default_preconditioner", "within_solver_new", "within_solver_free",
    "within_solver_n_dofs", "within_solver_n_obs", "within_solver_n_factors", "within_solver_solve",
    "within_solver_solve_batch", "within_solver_solve_batch_device", "within_solve", "within_solve_batch",
    "within_solver_apply_gramian", "within_solver_apply_preconditioner", "within_solver_matvec_d",
    "within_solver_rmatvec_wdt", "within_solver_factor_meta", "within_solver_n_subdomains",
    "within_solver_subdomain_info", "within_solver_subdomain_indices", "within_solver_ac_sizes",
    "within_solver_ac_arrays", "within_solver_gpu_launches", "within_solver_setup_time", "within_last_error",
    "within_solver_set_profiling", "within_solver_kernel_time", "within_solver_apply_gramian_noalloc",
    "within_solve_many", "within_solver_subdomain_inner_work", "within_solver_additive_diagnostics",
    "within_solver_preconditioner_bytes", "within_solver_new_with_preconditioner",
    "within_preconditioner_from_bytes", "within_solver_preconditioner_kind", "within_solver_schwarz_bytes",
    "within_coarse_net_params", "within_solver_set_coarse_net", "within_solver_set_coarse_basis",
    "within_solver_clear_coarse", "within_solver_coarse_basis", "within_solver_set_coarse_targets",
    "within_coarse_net_grad", "within_solver_release_coarse_training", "within_solver_inject_sweep_timeout", "within_solver_set_sweep_cluster",
    "within_solver_obs_config", "within_solver_obs_hot_global", "within_solver_obs_rhs_per_lane", "within_solver_set_hybrid", "within_solver_hybrid", "within_solver_hybrid_bytes", "within_solver_set_obs_config",
    "within_solver_obs_tune_times",
]

_lib = None


def load():
    """Load the library (building it first if the sources are newer)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        try:
            from . import build as _build
            _build.build()
        except Exception as e:  # pragma: no cover - build environment specific
            raise ImportError(f"libwithin_b200.so is missing and could not be built: {e}") from e
    L = C.CDLL(LIB_PATH)
    vp = C.c_void_p
    L.within_default_params.argtypes = [C.POINTER(Params)]
    L.within_default_preconditioner.argtypes = [C.POINTER(Precond)]
    L.within_solver_new.argtypes = [vp, C.c_size_t, C.c_size_t, C.c_int64, C.c_int64, vp,
                                    C.POINTER(Params), C.POINTER(Precond), C.POINTER(vp)]
    L.within_solver_new.restype = C.c_int
    L.within_solver_free.argtypes = [vp]
    for f in ("within_solver_n_dofs", "within_solver_n_obs", "within_solver_n_factors"):
        getattr(L, f).argtypes = [vp]
        getattr(L, f).restype = C.c_size_t
    L.within_solver_solve.argtypes = [vp, vp, vp, vp, C.POINTER(Stats)]
    L.within_solver_solve_batch.argtypes = [vp, vp, C.c_size_t, vp, vp, C.POINTER(Stats)]
    L.within_solver_solve_batch_device.argtypes = [vp, vp, C.c_size_t, vp, vp, C.POINTER(Stats), vp]
    L.within_solve.argtypes = [vp, C.c_size_t, C.c_size_t, C.c_int64, C.c_int64, vp, vp,
                               C.POINTER(Params), C.POINTER(Precond), vp, vp, C.POINTER(Stats)]
    L.within_solve_batch.argtypes = [vp, C.c_size_t, C.c_size_t, C.c_int64, C.c_int64, vp, C.c_size_t, vp,
                                     C.POINTER(Params), C.POINTER(Precond), vp, vp, C.POINTER(Stats)]
    for f in ("within_solver_apply_gramian", "within_solver_apply_preconditioner", "within_solver_matvec_d",
              "within_solver_rmatvec_wdt"):
        getattr(L, f).argtypes = [vp, vp, C.c_size_t, vp]
    L.within_solver_factor_meta.argtypes = [vp, _i64p, _i64p]
    L.within_solver_n_subdomains.argtypes = [vp]
    L.within_solver_n_subdomains.restype = C.c_int32
    L.within_solver_subdomain_info.argtypes = [vp, C.c_int32, _i64p]
    L.within_solver_subdomain_indices.argtypes = [vp, C.c_int32, _u32p, _f64p]
    L.within_solver_preconditioner_bytes.argtypes = [vp, vp, C.POINTER(C.c_size_t)]
    L.within_solver_preconditioner_bytes.restype = C.c_int
    L.within_solver_new_with_preconditioner.argtypes = [vp, C.c_size_t, C.c_size_t, C.c_int64, C.c_int64, vp,
                                                        C.POINTER(Params), vp, C.c_size_t, C.POINTER(vp)]
    L.within_solver_new_with_preconditioner.restype = C.c_int
    L.within_preconditioner_from_bytes.argtypes = [vp, C.c_size_t, C.POINTER(vp)]
    L.within_preconditioner_from_bytes.restype = C.c_int
    L.within_solver_preconditioner_kind.argtypes = [vp]
    L.within_solver_preconditioner_kind.restype = C.c_int32
    L.within_solver_subdomain_inner_work.argtypes = [vp, _i64p]
    L.within_solver_additive_diagnostics.argtypes = [vp, C.c_int32, C.POINTER(AdditiveDiagnostics)]
    L.within_solver_additive_diagnostics.restype = C.c_int
    L.within_solver_ac_sizes.argtypes = [vp, C.c_int32, _i64p]
    L.within_solver_ac_arrays.argtypes = [vp, C.c_int32, _i32p, _i32p, _f64p, _i32p, _i32p, _f64p, _i32p, _f64p]
    L.within_solver_gpu_launches.argtypes = [vp]
    L.within_solver_gpu_launches.restype = C.c_int64
    L.within_solver_setup_time.argtypes = [vp]
    L.within_solver_setup_time.restype = C.c_double
    L.within_last_error.restype = C.c_char_p
    L.within_solve_many.argtypes = [C.POINTER(Problem), C.c_size_t, vp, vp, C.c_int32]
    L.within_solve_many.restype = C.c_int
    L.within_solver_apply_gramian_noalloc.argtypes = [vp, vp, C.c_size_t, vp, vp]
    L.within_solver_apply_gramian_noalloc.restype = C.c_int
    L.within_solver_set_profiling.argtypes = [vp, C.c_int32]
    L.within_solver_kernel_time.argtypes = [vp, C.c_int32, C.POINTER(C.c_int64), C.POINTER(C.c_double)]
    L.within_solver_schwarz_bytes.argtypes = [vp, C.c_int32, C.c_int32]
    L.within_solver_schwarz_bytes.restype = C.c_int64
    L.within_coarse_net_params.restype = C.c_int32
    L.within_solver_set_coarse_net.argtypes = [vp, vp, C.c_size_t, C.c_uint64]
    L.within_solver_set_coarse_basis.argtypes = [vp, vp, C.c_size_t]
    L.within_solver_clear_coarse.argtypes = [vp]
    L.within_solver_coarse_basis.argtypes = [vp, vp]
    L.within_solver_set_coarse_targets.argtypes = [vp, vp, C.c_size_t]
    L.within_coarse_net_grad.argtypes = [vp, vp, C.c_uint64, vp, C.POINTER(C.c_double), vp]
    L.within_solver_release_coarse_training.argtypes = [vp]
    L.within_solver_inject_sweep_timeout.argtypes = [vp, C.c_int32]
    L.within_solver_inject_sweep_timeout.restype = C.c_int
    L.within_solver_set_sweep_cluster.argtypes = [vp, C.c_int64]
    L.within_solver_set_sweep_cluster.restype = C.c_int
    L.within_solver_obs_config.argtypes = [vp, C.c_int32, C.c_int32, C.POINTER(C.c_int32), C.POINTER(C.c_int32)]
    L.within_solver_obs_config.restype = C.c_int
    L.within_solver_obs_hot_global.argtypes = [vp, C.c_int32, C.c_int32]
    L.within_solver_obs_hot_global.restype = C.c_int32
    L.within_solver_obs_rhs_per_lane.argtypes = [vp, C.c_int32, C.c_int32]
    L.within_solver_obs_rhs_per_lane.restype = C.c_int32
    L.within_solver_set_hybrid.argtypes = [vp, C.c_int32, C.c_int32, C.c_int32]
    L.within_solver_set_hybrid.restype = C.c_int
    L.within_solver_hybrid.argtypes = [vp, C.c_int32, C.c_int32, C.POINTER(C.c_float)]
    L.within_solver_hybrid.restype = C.c_int32
    L.within_solver_hybrid_bytes.argtypes = [vp, C.c_int32, C.c_int32]
    L.within_solver_hybrid_bytes.restype = C.c_int64
    L.within_solver_set_obs_config.argtypes = [vp, C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_int32]
    L.within_solver_set_obs_config.restype = C.c_int
    L.within_solver_obs_tune_times.argtypes = [vp, C.c_int32, C.c_int32, C.POINTER(C.c_float), C.c_int32]
    L.within_solver_obs_tune_times.restype = C.c_int
    for f in ("within_solver_set_coarse_net", "within_solver_set_coarse_basis", "within_solver_clear_coarse",
              "within_solver_coarse_basis", "within_solver_set_coarse_targets", "within_coarse_net_grad",
              "within_solver_release_coarse_training"):
        getattr(L, f).restype = C.c_int
    _lib = L
    return L


def last_error() -> str:
    return load().within_last_error().decode(errors="replace")


def ptr(a: np.ndarray | None):
    return None if a is None else a.ctypes.data_as(C.c_void_p)
