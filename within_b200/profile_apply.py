"""Per-apply timing of the operator and Schwarz applies on the weighted worker-firm-year
panel (config 3's generator), for profiling runs:

    PRECS=mixed SCALE=0.5 python -m within_b200.profile_apply

For each precision in PRECS (``mixed``, ``fp64``; default both) it builds a solver on the
panel at SCALE (1 = 10M observations, 16 RHS), solves once (the autotuner times its
candidates here), solves again with event timing on, and prints one JSON line: the
average operator apply (``<prec>_obs_us``) and Schwarz apply (``<prec>_sch_us``) in µs,
the observation pass's chosen shape and the autotuner's timing table, the hybrid apply's
form and time, iterations and the final residual.  HYB=0|1|2 fixes the operator (the
observation pass, the hybrid apply with lane-group tables, or its tensor-core form);
FORCE=smem|glob:<obs per chunk>:<blocks per SM> pins the observation pass's shape;
TAG labels the line.
"""
import ctypes as C
import json
import os
import time

import numpy as np
import torch

import within_b200 as wb
from within_b200 import _lib, synthetic


def main():
    L = _lib.load()
    scale = float(os.environ.get("SCALE", "1"))
    force = os.environ.get("FORCE", "")
    cats, Y, w = synthetic.config3(seed=0, scale=scale)
    n, k = Y.shape
    out = {"tag": os.environ.get("TAG", force or "auto")}
    precs = os.environ.get("PRECS", "mixed,fp64")
    for prec, which in [p for p in (("mixed", 1), ("fp64", 0)) if p[0] in precs]:
        s = wb.Solver(cats, wb.CG(precision=prec, maxiter=int(os.environ.get("MAXIT", "200"))), weights=w)
        elem = 4 if prec == "mixed" else 8
        if os.environ.get("HYB") in ("0", "1", "2"):
            for e in ((4, 8) if prec == "mixed" else (8,)):
                rc = L.within_solver_set_hybrid(s._h, k, e, int(os.environ["HYB"]))
                assert rc == 0, L.within_last_error()
        if force:
            kind, per, bps = force.split(":")
            rc = L.within_solver_set_obs_config(s._h, k, elem, int(per), int(bps), 1 if kind == "glob" else 0)
            assert rc == 0, L.within_last_error()
        dY = torch.from_numpy(np.ascontiguousarray(Y.T)).cuda()
        dX = torch.empty((k, s.n_dofs), dtype=torch.float64, device="cuda")
        dD = torch.empty((k, n), dtype=torch.float64, device="cuda")
        st = (_lib.Stats * k)()

        def step():
            rc = L.within_solver_solve_batch_device(s._h, C.c_void_p(dY.data_ptr()), k, C.c_void_p(dX.data_ptr()),
                                                    C.c_void_p(dD.data_ptr()), st, None)
            assert rc == 0, L.within_last_error()

        t0 = time.time()
        step()
        torch.cuda.synchronize()
        out[prec + "_first_s"] = round(time.time() - t0, 3)
        L.within_solver_set_profiling(s._h, 1)
        step()
        torch.cuda.synchronize()
        cnt, ms = C.c_int64(), C.c_double()
        L.within_solver_kernel_time(s._h, which, C.byref(cnt), C.byref(ms))
        out[prec + "_obs_us"] = round(1000 * ms.value / max(1, cnt.value), 1)
        L.within_solver_kernel_time(s._h, which + 2, C.byref(cnt), C.byref(ms))
        out[prec + "_sch_us"] = round(1000 * ms.value / max(1, cnt.value), 1)
        L.within_solver_set_profiling(s._h, 0)
        per, bps = C.c_int32(), C.c_int32()
        L.within_solver_obs_config(s._h, k, elem, C.byref(per), C.byref(bps))
        out[prec + "_cfg"] = [L.within_solver_obs_hot_global(s._h, k, elem), per.value, bps.value,
                              L.within_solver_obs_rhs_per_lane(s._h, k, elem)]
        tm = (C.c_float * 24)()
        L.within_solver_obs_tune_times(s._h, k, elem, tm, 24)
        out[prec + "_tune_us"] = [round(1000 * v, 1) for v in tm]
        hm = C.c_float()
        out[prec + "_hyb32"] = [L.within_solver_hybrid(s._h, k, 4, C.byref(hm)), round(1000 * hm.value, 1)]
        out[prec + "_hyb64"] = [L.within_solver_hybrid(s._h, k, 8, C.byref(hm)), round(1000 * hm.value, 1)]
        out[prec + "_iters"] = max(int(st[c].iterations) for c in range(k))
        out[prec + "_res"] = max(float(st[c].final_residual) for c in range(k))
        del s
        torch.cuda.synchronize()
    print(json.dumps(out), flush=True)


if __name__ == "__main__":
    main()
