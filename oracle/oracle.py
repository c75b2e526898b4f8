"""ctypes front end of the CPU oracle (``liboracle.so``).

TEST INFRASTRUCTURE ONLY: imported by the tests, ``__graft_entry__.smoke()`` and
the CPU-baseline leg of ``bench.py``.  The ``within_b200`` package never imports
it.  See ``oracle.h`` for what is restated from which reference file.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from dataclasses import dataclass

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle.so")
_lib = None

u32p = np.ctypeslib.ndpointer(dtype=np.uint32, flags="C_CONTIGUOUS")
f64p = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
i32p = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
i64p = np.ctypeslib.ndpointer(dtype=np.int64, flags="C_CONTIGUOUS")


class OracleParams(C.Structure):
    _fields_ = [
        ("krylov", C.c_int32),
        ("gmres_restart", C.c_int32),
        ("tol", C.c_double),
        ("maxiter", C.c_int32),
        ("max_refinements", C.c_int32),
        ("precond_kind", C.c_int32),
        ("approx_chol_seed", C.c_uint64),
        ("approx_chol_split", C.c_uint32),
        ("approx_schur_enabled", C.c_int32),
        ("approx_schur_seed", C.c_uint64),
        ("approx_schur_split", C.c_uint32),
        ("dense_threshold", C.c_int32),
        ("lsmr_local_size", C.c_int32),
    ]


def build() -> None:
    """Compile liboracle.so from oracle.c with the committed Makefile."""
    subprocess.run(["make", "-C", _HERE, "-s"], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = C.CDLL(_LIB_PATH)
        vp = C.c_void_p
        L.oracle_solver_new.argtypes = [u32p, C.c_int64, C.c_int32, C.c_int64, C.c_int64, C.c_void_p,
                                        C.POINTER(OracleParams), C.POINTER(vp), C.c_char_p, C.c_int]
        L.oracle_solver_new.restype = C.c_int
        L.oracle_solver_free.argtypes = [vp]
        L.oracle_n_dofs.argtypes = [vp]; L.oracle_n_dofs.restype = C.c_int64
        L.oracle_n_obs.argtypes = [vp]; L.oracle_n_obs.restype = C.c_int64
        L.oracle_factor_meta.argtypes = [vp, i64p, i64p]
        L.oracle_solve.argtypes = [vp, f64p, f64p, f64p, i32p, i32p, f64p, C.c_char_p, C.c_int]
        L.oracle_solve_batch.argtypes = [vp, f64p, C.c_int32, f64p, f64p, i32p, i32p, f64p, C.c_int32,
                                         C.c_char_p, C.c_int]
        for name in ("oracle_matvec_d", "oracle_rmatvec_wdt", "oracle_rmatvec_dt", "oracle_apply_gramian"):
            getattr(L, name).argtypes = [vp, f64p, f64p]
        L.oracle_apply_precond.argtypes = [vp, f64p, f64p]
        L.oracle_gramian_diagonal.argtypes = [vp, f64p]
        L.oracle_n_subdomains.argtypes = [vp]; L.oracle_n_subdomains.restype = C.c_int32
        L.oracle_subdomain_info.argtypes = [vp, C.c_int32, i64p]
        L.oracle_subdomain_indices.argtypes = [vp, C.c_int32, u32p, f64p]
        L.oracle_ac_sizes.argtypes = [vp, C.c_int32, i64p]
        L.oracle_ac_arrays.argtypes = [vp, C.c_int32, i32p, i32p, f64p, i32p, i32p, f64p, i32p, f64p]
        L.oracle_crosstab_nnz.argtypes = [vp, C.c_int32]; L.oracle_crosstab_nnz.restype = C.c_int64
        L.oracle_crosstab.argtypes = [vp, C.c_int32, u32p, u32p, f64p, f64p, f64p]
        L.oracle_csr_transpose.argtypes = [C.c_int32, C.c_int32, u32p, u32p, f64p, u32p, u32p, f64p]
        L.oracle_dense_cg.argtypes = [C.c_int32, C.c_void_p, C.c_void_p, f64p, C.c_double, C.c_int32, f64p,
                                      i32p, i32p, f64p]
        L.oracle_dense_gmres.argtypes = [C.c_int32, C.c_void_p, C.c_void_p, f64p, C.c_double, C.c_int32,
                                         C.c_int32, f64p, i32p, i32p, f64p]
        L.oracle_lsmr_dense.argtypes = [f64p, C.c_int64, C.c_int64, C.c_void_p, f64p, C.c_double, C.c_int32,
                                        C.c_int32, f64p, i32p, i32p, i32p]
        _lib = L
    return _lib


LSMR_STOPS = ("ZeroRhs", "InitialNormalEquationResidualZero", "ResidualTolerance", "NormalEquationTolerance",
              "BidiagonalizationBreakdown", "MaxIterations")


def lsmr_dense(a, b, minv=None, tol=1e-10, maxiter=100, local_size=0):
    """The oracle's LSMR (lsmr.rs) on a dense operator: (x, converged, iterations, stop reason)."""
    a = np.ascontiguousarray(a, dtype=np.float64)
    rows, cols = a.shape
    mi = None if minv is None else np.ascontiguousarray(minv, dtype=np.float64)
    x = np.zeros(cols)
    cv, it, st = np.zeros(1, np.int32), np.zeros(1, np.int32), np.zeros(1, np.int32)
    lib().oracle_lsmr_dense(a.ravel(), rows, cols, None if mi is None else mi.ctypes.data_as(C.c_void_p),
                            np.ascontiguousarray(b, dtype=np.float64), tol, maxiter, local_size, x, cv, it, st)
    return x, bool(cv[0]), int(it[0]), LSMR_STOPS[int(st[0])]


def make_params(krylov="cg", tol=1e-8, maxiter=1000, max_refinements=2, restart=30,
                preconditioner="additive", approx_chol_seed=0, approx_chol_split=2,
                approx_schur=(0, 1), dense_threshold=24, local_size=None) -> OracleParams:
    """Reference defaults: CG, tol 1e-8, maxiter 1000, 2 refinements (within/src/config.rs:227-236),
    additive Schwarz with LocalSolverConfig::solver_default() (config.rs:108-117)."""
    p = OracleParams()
    p.krylov = {"cg": 0, "gmres": 1, "lsmr": 2}[krylov]
    p.lsmr_local_size = 0 if local_size is None else int(local_size)
    p.gmres_restart = restart
    p.tol = tol
    p.maxiter = maxiter
    p.max_refinements = max_refinements
    p.precond_kind = {"off": 0, "additive": 1, "multiplicative": 2}[preconditioner]
    p.approx_chol_seed = approx_chol_seed
    p.approx_chol_split = max(1, approx_chol_split)
    if approx_schur is None:
        p.approx_schur_enabled = 0
    else:
        p.approx_schur_enabled = 1
        p.approx_schur_seed, p.approx_schur_split = approx_schur
    p.dense_threshold = dense_threshold
    return p


@dataclass
class OracleResult:
    x: np.ndarray
    demeaned: np.ndarray
    converged: object
    iterations: object
    residual: object


class OracleSolver:
    def __init__(self, categories, weights=None, **kw):
        L = lib()
        cats = np.asarray(categories)
        if cats.ndim != 2:
            raise ValueError("categories must be 2-D")
        codes = np.ascontiguousarray(np.asfortranarray(cats.astype(np.uint32)).T)  # factor-major
        n, q = cats.shape
        self.n_obs, self.n_factors = n, q
        self._w = None if weights is None else np.ascontiguousarray(weights, dtype=np.float64)
        self.params = make_params(**kw)
        h = C.c_void_p()
        err = C.create_string_buffer(512)
        # codes[i*row_stride + q*col_stride] with a factor-major buffer: row_stride 1, col_stride n
        rc = L.oracle_solver_new(codes.ravel(), n, q, 1, n,
                                 None if self._w is None else self._w.ctypes.data_as(C.c_void_p),
                                 C.byref(self.params), C.byref(h), err, 512)
        if rc != 0:
            raise ValueError(err.value.decode())
        self._h = h
        self.n_dofs = int(L.oracle_n_dofs(h))

    def __del__(self):
        if getattr(self, "_h", None):
            lib().oracle_solver_free(self._h)
            self._h = None

    def factor_meta(self):
        nl = np.zeros(self.n_factors, np.int64); off = np.zeros(self.n_factors, np.int64)
        lib().oracle_factor_meta(self._h, nl, off)
        return nl, off

    def solve(self, y) -> OracleResult:
        y = np.ascontiguousarray(y, dtype=np.float64)
        x = np.zeros(self.n_dofs); d = np.zeros(self.n_obs)
        cv = np.zeros(1, np.int32); it = np.zeros(1, np.int32); fr = np.zeros(1)
        lib().oracle_solve(self._h, y, x, d, cv, it, fr, None, 0)
        return OracleResult(x, d, bool(cv[0]), int(it[0]), float(fr[0]))

    def solve_batch(self, Y, threads=None) -> OracleResult:
        Y = np.asarray(Y, dtype=np.float64)
        k = Y.shape[1]
        ys = np.ascontiguousarray(Y.T)
        x = np.zeros((k, self.n_dofs)); d = np.zeros((k, self.n_obs))
        cv = np.zeros(k, np.int32); it = np.zeros(k, np.int32); fr = np.zeros(k)
        threads = threads or os.cpu_count() or 1
        lib().oracle_solve_batch(self._h, ys.ravel(), k, x.ravel(), d.ravel(), cv, it, fr, threads, None, 0)
        return OracleResult(x.T.copy(), d.T.copy(), [bool(c) for c in cv], [int(i) for i in it],
                            [float(f) for f in fr])

    def _vec(self, name, v, n_out):
        v = np.ascontiguousarray(v, dtype=np.float64)
        out = np.zeros(n_out)
        getattr(lib(), name)(self._h, v, out)
        return out

    def matvec_d(self, x): return self._vec("oracle_matvec_d", x, self.n_obs)
    def rmatvec_wdt(self, r): return self._vec("oracle_rmatvec_wdt", r, self.n_dofs)
    def rmatvec_dt(self, r): return self._vec("oracle_rmatvec_dt", r, self.n_dofs)
    def apply_gramian(self, x): return self._vec("oracle_apply_gramian", x, self.n_dofs)
    def apply_precond(self, r): return self._vec("oracle_apply_precond", r, self.n_dofs)

    def gramian_diagonal(self):
        out = np.zeros(self.n_dofs)
        lib().oracle_gramian_diagonal(self._h, out)
        return out

    def subdomains(self):
        """List of dicts: pair, global indices, PoU weights, elimination and factor data."""
        L = lib()
        out = []
        for i in range(L.oracle_n_subdomains(self._h)):
            info = np.zeros(8, np.int64)
            L.oracle_subdomain_info(self._h, i, info)
            q, r, nloc, nq, nr, eq, kind, nred = (int(v) for v in info)
            g = np.zeros(nloc, np.uint32); w = np.zeros(nloc)
            L.oracle_subdomain_indices(self._h, i, g, w)
            d = dict(pair=(q, r), global_indices=g, pou=w, n_q=nq, n_r=nr, eliminate_q=bool(eq),
                     reduced_kind="dense" if kind == 0 else "ac", n_reduced=nred)
            nnz = int(L.oracle_crosstab_nnz(self._h, i))
            ip = np.zeros(nq + 1, np.uint32); ix = np.zeros(max(nnz, 1), np.uint32); dv = np.zeros(max(nnz, 1))
            dq = np.zeros(max(nq, 1)); dr = np.zeros(max(nr, 1))
            L.oracle_crosstab(self._h, i, ip, ix, dv, dq, dr)
            d.update(c_indptr=ip, c_indices=ix[:nnz], c_data=dv[:nnz], diag_q=dq[:nq], diag_r=dr[:nr])
            if kind == 1:
                sz = np.zeros(5, np.int64)
                L.oracle_ac_sizes(self._h, i, sz)
                n, nlev, annz, ncol, ncore = (int(v) for v in sz)
                lp = np.zeros(nlev + 1, np.int32); cv = np.zeros(max(ncol, 1), np.int32); cd = np.zeros(max(ncol, 1))
                cp = np.zeros(ncol + 1, np.int32); ci = np.zeros(max(annz, 1), np.int32); cc = np.zeros(max(annz, 1))
                core = np.zeros(max(ncore, 1), np.int32); z = np.zeros(max(ncore * ncore, 1))
                L.oracle_ac_arrays(self._h, i, lp, cv, cd, cp, ci, cc, core, z)
                d["ac"] = dict(n=n, level_ptr=lp, col_vertex=cv[:ncol], col_diag=cd[:ncol], col_ptr=cp,
                               col_idx=ci[:annz], col_coef=cc[:annz], core_vertex=core[:ncore],
                               core_z=z[:ncore * ncore].reshape(ncore, ncore))
            out.append(d)
        return out

    def subdomain_inner_parallel_work(self):
        """FePreconditioner::subdomain_inner_parallel_work (within/src/operator/preconditioner.rs:64-79)."""
        L = lib()
        out = []
        for i in range(L.oracle_n_subdomains(self._h)):
            info = np.zeros(8, np.int64)
            L.oracle_subdomain_info(self._h, i, info)
            out.append(inner_parallel_work(int(info[3]), int(info[4]), int(L.oracle_crosstab_nnz(self._h, i))))
        return out

    def additive_diagnostics(self, configured=0, threads=1):
        """AdditiveSchwarzDiagnostics of this build (see ``additive_diagnostics``)."""
        L = lib()
        scatter = []
        for i in range(L.oracle_n_subdomains(self._h)):
            info = np.zeros(8, np.int64)
            L.oracle_subdomain_info(self._h, i, info)
            scatter.append(int(info[2]))
        return additive_diagnostics(self.subdomain_inner_parallel_work(), scatter, self.n_dofs, configured, threads)


# Subdomains go inner-parallel only above both thresholds (PAR_BACKSUB_THRESHOLD,
# within/src/operator/local_solver.rs:78; PAR_SPMV_THRESHOLD, operator/csr_block.rs:4).
PAR_THRESHOLD = 10_000
# AdditiveScheduler constants (schwarz-precond/src/schwarz/additive/planning.rs:213-218).
MIN_INNER_PARALLEL_WORK = 200_000
OUTER_CAPACITY_TARGET = 0.75
AUTO_REDUCTION_SWEEP_FACTOR = 1.1
AUTO_INNER_REDUCTION_SWEEP_FACTOR = 6.0
AUTO_OVERLAP_FOR_REDUCTION = 4.0


def inner_parallel_work(n_q, n_r, cross_nnz):
    """BlockElimSolver::estimated_inner_parallel_work (local_solver.rs:348-356)."""
    if max(n_q, n_r) <= PAR_THRESHOLD:
        return 0
    return 2 * cross_nnz + n_q + n_r


def additive_diagnostics(work, scatter, n_dofs, configured=0, threads=1):
    """AdditiveSchwarzDiagnostics::from_entries and its accessors (planning.rs:151-210),
    and the strategy AdditiveScheduler::reduction_plan resolves (planning.rs:71-135).
    work: per-subdomain inner work; scatter: per-subdomain local sizes.  Strategies:
    0 Auto, 1 AtomicScatter, 2 ParallelReduction."""
    total, mx, tsc = sum(work), max(work, default=0), sum(scatter)
    cap = 0.0 if mx == 0 else total / mx
    overlap = tsc / max(n_dofs, 1)
    threads = max(threads, 1)
    inner = mx >= MIN_INNER_PARALLEL_WORK and cap < threads * OUTER_CAPACITY_TARGET
    if configured in (1, 2):
        resolved = configured
    else:
        active = max(min(threads, len(work)), 1)
        ratio = (active * n_dofs) / max(tsc, 1)
        if ratio <= AUTO_REDUCTION_SWEEP_FACTOR:
            resolved = 2
        elif inner and ratio <= AUTO_INNER_REDUCTION_SWEEP_FACTOR:
            resolved = 2
        elif overlap >= AUTO_OVERLAP_FOR_REDUCTION:
            resolved = 2
        else:
            resolved = 1
    return dict(reduction_strategy=configured, resolved_reduction_strategy=resolved, n_subdomains=len(work),
                n_dofs=n_dofs, total_inner_parallel_work=total, max_inner_parallel_work=mx,
                total_scatter_dofs=tsc, outer_parallel_capacity=cap, scatter_overlap=overlap)


def csr_transpose(nrows, ncols, indptr, indices, data):
    indptr = np.ascontiguousarray(indptr, np.uint32); indices = np.ascontiguousarray(indices, np.uint32)
    data = np.ascontiguousarray(data, np.float64)
    nnz = int(indptr[-1])
    tp = np.zeros(ncols + 1, np.uint32); ti = np.zeros(max(nnz, 1), np.uint32); td = np.zeros(max(nnz, 1))
    lib().oracle_csr_transpose(nrows, ncols, indptr, indices, data, tp, ti, td)
    return tp, ti[:nnz], td[:nnz]


def dense_krylov(a, b, m_inv_diag=None, tol=1e-10, maxiter=100, method="cg", restart=30):
    a = np.ascontiguousarray(a, np.float64); b = np.ascontiguousarray(b, np.float64)
    n = len(b)
    x = np.zeros(n); cv = np.zeros(1, np.int32); it = np.zeros(1, np.int32); rn = np.zeros(1)
    mp = None
    if m_inv_diag is not None:
        m_inv_diag = np.ascontiguousarray(m_inv_diag, np.float64)
        mp = m_inv_diag.ctypes.data_as(C.c_void_p)
    if method == "cg":
        lib().oracle_dense_cg(n, a.ctypes.data_as(C.c_void_p), mp, b, tol, maxiter, x, cv, it, rn)
    else:
        lib().oracle_dense_gmres(n, a.ctypes.data_as(C.c_void_p), mp, b, tol, maxiter, restart, x, cv, it, rn)
    return x, bool(cv[0]), int(it[0]), float(rn[0])
