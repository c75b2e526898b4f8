"""Benchmark of the solve phase: RHS solved/sec at tol 1e-8 on the weighted 3-FE panel
(10M observations: 500k workers x 20 years, 100k Zipf(1.1) firms, lognormal weights,
16 right-hand sides).

    python bench.py [--gpus N --steps K --warmup W] [--impl ours|reference]

A step is one batched solve of the 16 RHS (Solver::solve_batch semantics, each RHS to
final_residual <= 1e-8).  `value` is measured with the inputs resident in HBM through
within_solver_solve_batch_device; `e2e` through within_solver_solve_batch with host
buffers (pinned), the host<->device copies inside the timed region.  Multi-GPU runs are
independent replicas (weak scaling; the path has no exchange step).  The reference arm
times the CPU oracle (a restatement of the reference's Rust path) on the host cores.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "RHS solved/sec at tol 1e-8, 10M obs 3 FE; speedup vs plain FP64 GPU PCG"
PEAKS = os.path.join(ROOT, "MEASURED_PEAKS.json")


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--scale", type=float, default=1.0, help="problem scale (1.0 = 10M observations)")
    ap.add_argument("--precision", default="mixed", choices=["mixed", "fp64"])
    ap.add_argument("--krylov", default="cg", choices=["cg", "lsmr"],
                    help="cg (default): CG on the normal equations; lsmr: LSMR on W^(1/2) D (FP64)")
    ap.add_argument("--operator", default="implicit", choices=["implicit", "explicit"],
                    help="Krylov operator: the observation pass (default) or the assembled Gramian (CSR)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-dropin", action="store_true", help="skip the FP64 drop-in comparison run")
    ap.add_argument("--workload", default="panel", choices=["panel", "uneven"],
                    help="panel: the 10M-obs weighted 3-FE panel (the headline); uneven: 256 independent "
                         "problems of 1e3-1e6 observations, 2-4 factors, 1-8 RHS each (solve_many)")
    ap.add_argument("--problems", type=int, default=256, help="number of problems of the uneven workload")
    return ap.parse_args()


def max_over_ranks(dist, value: float, device: str = "cuda") -> float:
    """The largest of every rank's value (the job's time is its slowest rank's)."""
    if dist is None:
        return value
    import torch
    t = torch.tensor([value], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def dist_info():
    return int(os.environ.get("RANK", 0)), int(os.environ.get("LOCAL_RANK", 0)), int(os.environ.get("WORLD_SIZE", 1))


def workload(scale):
    from within_b200 import synthetic
    cats, Y, w = synthetic.config3(seed=0, scale=scale)
    return cats, np.asfortranarray(Y), w


def config_dict(cats, k, scale, precision, operator="implicit"):
    return {"workload": "weighted 3-FE worker-firm-year panel (10M obs: 500k workers x 20 years, 100k Zipf(1.1) "
                        "firms, p_switch 0.1, lognormal weights), 16 RHS, CG + additive Schwarz, tol 1e-8"
            if scale == 1.0 else f"weighted 3-FE panel at scale {scale}",
            "n_obs": int(cats.shape[0]), "n_factors": int(cats.shape[1]), "n_rhs": int(k),
            "precision": precision, "operator": operator,
            "l2": "inputs larger than L2 (Y is n_obs x 16 FP64 = 1.28 GB)"}


class Clocks:
    """SM clocks, power and clock-event reasons sampled during the timed region.

    NVML is read from a thread every 10 ms, with one sample when sampling starts and one
    when it stops, so short timed regions still carry several samples; the device is
    found by the UUID torch reports for cuda:`index` (CUDA_VISIBLE_DEVICES-safe).  Only
    reads: no setting of the GPU is changed.  Without NVML, nvidia-smi is sampled instead.
    """

    # nvmlClocksEventReasons bits
    _BITS = {"sw_power_cap": 0x4, "hw_slowdown": 0x8, "sw_thermal_slowdown": 0x20, "hw_thermal_slowdown": 0x40}

    def __init__(self, index):
        import threading
        self.samples, self.reasons, self.max_mhz = [], set(), None
        self.p = self.nv = None
        try:
            import pynvml as nv
            import torch
            nv.nvmlInit()
            try:
                uuid = str(torch.cuda.get_device_properties(index).uuid)
                h = nv.nvmlDeviceGetHandleByUUID(uuid if uuid.startswith("GPU-") else "GPU-" + uuid)
            except Exception:
                h = nv.nvmlDeviceGetHandleByIndex(index)
            self.nv, self.h = nv, h
            self.max_mhz = float(nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM))
            self._sample()
            self.done = threading.Event()
            self.t = threading.Thread(target=self._loop, daemon=True)
            self.t.start()
        except Exception:
            self.nv = None
            self._smi(index)

    def _sample(self):
        nv, h = self.nv, self.h
        self.samples.append(float(nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)))
        try:
            bits = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
        except Exception:
            bits = nv.nvmlDeviceGetCurrentClocksThrottleReasons(h)
        for name, bit in self._BITS.items():
            if bits & bit:
                self.reasons.add(name)

    def _loop(self):
        while not self.done.wait(0.01):
            try:
                self._sample()
            except Exception:
                return

    def _smi(self, index):
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        try:
            self.p = subprocess.Popen(["nvidia-smi", f"--id={index}", f"--query-gpu={q}", "--format=csv,noheader,nounits",
                                       "-lms", "100"], stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None

    def stop(self):
        if self.nv is not None:
            self.done.set()
            self.t.join()
            try:
                self._sample()
            except Exception:
                pass
            return {"sm_mhz": statistics.median(self.samples) if self.samples else None, "sm_max_mhz": self.max_mhz,
                    "reasons": sorted(self.reasons), "samples": len(self.samples), "source": "nvml, 10 ms"}
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.p.terminate()
        self.p.wait()
        self.f.flush()
        self.f.seek(0)
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.f.read().splitlines():
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx.append(float(parts[2]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        os.unlink(self.f.name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm), "source": "nvidia-smi"}


def cpu_baseline_run(cats, Y, w, n_rhs, threads):
    """The oracle (CPU restatement of the reference path) on a bounded sample."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    t0 = time.perf_counter()
    s = oracle.OracleSolver(cats, w)
    t_setup = time.perf_counter() - t0
    t0 = time.perf_counter()
    r = s.solve_batch(Y[:, :n_rhs], threads=threads)
    dt = time.perf_counter() - t0
    return {"value": n_rhs / dt, "unit": "RHS/s", "cores": threads, "kind": "port",
            "sample": f"{n_rhs} of the 16 RHS on the same 10M-obs design, one RHS per thread (solve_batch), "
                      f"setup {t_setup:.1f}s excluded",
            "converged": all(r.converged), "max_residual": max(r.residual)}


def reference_arm(args):
    rank, _, world = dist_info()
    if rank != 0:
        return
    cats, Y, w = workload(args.scale)
    threads = max(1, min(16, os.cpu_count() or 1))
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    s = oracle.OracleSolver(cats, w)
    times = []
    for step in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        s.solve_batch(Y[:, :threads], threads=threads)
        if step >= args.warmup:
            times.append(time.perf_counter() - t0)
    total = sum(times)
    value = threads * len(times) / total
    line = {"metric": METRIC, "value": value, "unit": "RHS/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1000 * total / len(times), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)",
            # the workload is our arm's (all its RHS); each step is a bounded sample of it
            "config": dict(config_dict(cats, Y.shape[1], args.scale, args.precision, args.operator),
                           krylov=args.krylov),
            "impl": "reference",
            "cpu_baseline": {"value": value, "unit": "RHS/s", "cores": threads, "kind": "port",
                             "sample": f"each step solves {threads} of the 16 RHS, one per host thread"},
            "e2e": {"value": value, "unit": "RHS/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def uneven(args):
    """Many independent problems of uneven size through within_solve_many.  A step solves
    every problem from scratch (setup included: each problem is a one-shot solve), timed
    on the host around the whole call with the device synchronised on both sides (the
    problems run on many streams at once, which one stream's events do not cover)."""
    import torch
    import within_b200 as wb
    from within_b200 import synthetic
    torch.cuda.set_device(0)
    probs = synthetic.config4(seed=0, n_problems=args.problems, max_obs=1_000_000)
    n_rhs = sum(Y.shape[1] for _, Y in probs)
    n_obs = sum(c.shape[0] for c, _ in probs)
    cfg = wb.CG(precision=args.precision)
    for _ in range(max(1, args.warmup)):
        wb.solve_many(probs, cfg)
    clocks = Clocks(0)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        res = wb.solve_many(probs, cfg)
    torch.cuda.synchronize()
    el = time.perf_counter() - t0
    clk = clocks.stop()
    conv = all(all(r.converged) for r in res)
    worst = max(max(r.residual) for r in res)
    line = {"metric": "RHS solved/sec at tol 1e-8, uneven batch of independent problems (setup included)",
            "value": args.steps * n_rhs / el, "unit": "RHS/s", "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1000.0 * el / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None,
            "dtype": "f32 inner / f64 refinement" if args.precision == "mixed" else "f64",
            "data": "synthetic (seeded log-uniform sizes, uniform codes)",
            "config": {"workload": f"{len(probs)} independent problems, n_obs log-uniform on [1e3, 1e6] "
                                   f"(total {n_obs}), 2-4 factors with levels log-uniform on [n/50, n/5], "
                                   f"1-8 RHS each (total {n_rhs}), CG + additive Schwarz, tol 1e-8, "
                                   f"{os.cpu_count()} problems in flight (one per host core)",
                       "timing": "host wall clock, device synchronised"},
            "clocks": clk, "accuracy": {"converged": conv, "max_final_residual": worst}}
    print(json.dumps(line), flush=True)


def ours(args):
    if args.workload == "uneven":
        return uneven(args)
    import torch
    rank, local, world = dist_info()
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=600))
    import within_b200 as wb
    from within_b200 import _lib
    L = _lib.load()

    cats, Y, w = workload(args.scale)
    n, k = Y.shape
    t0 = time.perf_counter()
    op = wb.OperatorRepr.Explicit if args.operator == "explicit" else wb.OperatorRepr.Implicit
    cfg = wb.LSMR() if args.krylov == "lsmr" else wb.CG(precision=args.precision, operator=op)
    solver = wb.Solver(cats, cfg, weights=w)
    setup_s = time.perf_counter() - t0
    m = solver.n_dofs
    dY = torch.from_numpy(np.ascontiguousarray(Y.T)).cuda()       # (k, n) = RHS-major
    dX = torch.empty((k, m), dtype=torch.float64, device="cuda")
    dD = torch.empty((k, n), dtype=torch.float64, device="cuda")
    st = (_lib.Stats * k)()

    def step():
        rc = L.within_solver_solve_batch_device(solver._h, C.c_void_p(dY.data_ptr()), k, C.c_void_p(dX.data_ptr()),
                                                C.c_void_p(dD.data_ptr()), st, None)
        if rc != 0:
            raise RuntimeError(_lib.last_error())

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    clocks = Clocks(local)
    launches0 = solver.gpu_launches
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    ev0.record()
    for _ in range(args.steps):
        step()
    ev1.record()
    torch.cuda.synchronize()
    clk = clocks.stop()
    elapsed_ms = ev0.elapsed_time(ev1)
    launches = solver.gpu_launches - launches0
    conv = [bool(st[c].converged) for c in range(k)]
    res = [float(st[c].final_residual) for c in range(k)]
    iters = [int(st[c].iterations) for c in range(k)]
    # one more (untimed) step with per-launch event timing of the operator and Schwarz
    # applies; event timing runs the CG iterations launch by launch instead of as the
    # captured graph, so it stays out of the timed region
    L.within_solver_set_profiling(solver._h, 1)
    step()
    torch.cuda.synchronize()
    kt = {}
    for which in range(4):
        cnt, ms = C.c_int64(), C.c_double()
        L.within_solver_kernel_time(solver._h, which, C.byref(cnt), C.byref(ms))
        kt[which] = (cnt.value, ms.value)
    L.within_solver_set_profiling(solver._h, 0)
    if dist:
        elapsed_ms = max_over_ranks(dist, elapsed_ms)
    value = world * args.steps * k / (elapsed_ms / 1000.0)

    # end-to-end through the host C ABI (pinned buffers; copies inside the timed region)
    hY = torch.from_numpy(np.ascontiguousarray(Y.T)).pin_memory()
    hX = torch.empty((k, m), dtype=torch.float64).pin_memory()
    hD = torch.empty((k, n), dtype=torch.float64).pin_memory()
    e2e_steps = max(1, min(args.steps, 3))

    def host_step():
        rc = L.within_solver_solve_batch(solver._h, C.c_void_p(hY.data_ptr()), k, C.c_void_p(hX.data_ptr()),
                                         C.c_void_p(hD.data_ptr()), st)
        if rc != 0:
            raise RuntimeError(_lib.last_error())

    host_step()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(e2e_steps):
        host_step()
    e1.record()
    torch.cuda.synchronize()
    e2e_ms = e0.elapsed_time(e1)
    if dist:
        e2e_ms = max_over_ranks(dist, e2e_ms)
    e2e_value = world * e2e_steps * k / (e2e_ms / 1000.0)

    # roofline of the dominant kernel: the operator apply G x = D'W(D x)
    peaks = json.load(open(PEAKS)) if os.path.exists(PEAKS) else {}
    peak = float(peaks.get("hbm_gbs", 6650.0))
    peak_src = "of measured" if "hbm_gbs" in peaks else "of fallback"
    Q = cats.shape[1]
    which = 1 if args.precision == "mixed" else 0
    s_b = 4 if which == 1 else 8
    op_bytes = n * (4 * Q + s_b * (1 if w is not None else 0)) + 2 * s_b * m * k
    cnt, ms = kt[which]
    achieved = op_bytes / (ms / cnt / 1000.0) / 1e9 if cnt else None
    roofline = {"bound": "hbm", "kernel": "obs_pass_kernel (operator apply D'W(D x), %s)" % ("FP32" if which else "FP64"),
                "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": (achieved / peak) if achieved else None, "peak_source": peak_src,
                "algorithmic_bytes_per_launch": op_bytes, "launches": cnt,
                "avg_launch_us": 1000.0 * ms / cnt if cnt else None, "traffic": None,
                "schwarz_apply_avg_us": 1000.0 * kt[which + 2][1] / kt[which + 2][0] if kt[which + 2][0] else None}
    if args.operator == "explicit":
        # CSR SpMV of G: row pointers, column indices and values once, x read and y
        # written once (nnz(G) = m + 2 x distinct level pairs of every factor pair)
        nnz = m
        for a in range(Q):
            for b in range(a + 1, Q):
                nnz += 2 * int(np.unique(cats[:, a].astype(np.int64) * (int(cats[:, b].max()) + 1) + cats[:, b]).size)
        op_bytes = (m + 1) * 8 + nnz * (4 + s_b) + 2 * s_b * m * k
        achieved = op_bytes / (ms / cnt / 1000.0) / 1e9 if cnt else None
        roofline.update({"kernel": "csr_rows_kernel (explicit Gramian SpMV, %s)" % ("FP32" if which else "FP64"),
                         "achieved": achieved, "frac": (achieved / peak) if achieved else None,
                         "algorithmic_bytes_per_launch": op_bytes, "gramian_nnz": nnz})
    # DRAM bytes (dram__bytes_read.sum + write.sum) of one FP32 operator apply, from an ncu
    # capture of the same panel at half size (5M observations), scaled by the observations
    if which == 1 and abs(args.scale - 1.0) < 1e-9 and args.operator == "implicit":
        roofline["traffic"] = int(2 * 111.6e6)
        roofline["traffic_source"] = "ncu dram__bytes_read+write at 5M observations, x2 (scales with n)"

    line = {"metric": METRIC, "value": value, "unit": "RHS/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": elapsed_ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None,
            "dtype": "f32 inner / f64 refinement" if args.precision == "mixed" else "f64",
            "data": "synthetic (seeded generator with the reference benchmark's AKM shapes)",
            "config": dict(config_dict(cats, k, args.scale, args.precision, args.operator), krylov=args.krylov),
            "e2e": {"value": e2e_value, "unit": "RHS/s", "h2d_bytes_per_step": int(n * k * 8),
                    "d2h_bytes_per_step": int((m + n) * k * 8)},
            "gpu_launches": int(launches), "roofline": roofline, "clocks": clk,
            "accuracy": {"converged": all(conv), "max_final_residual": max(res), "iterations": iters},
            "setup_s": setup_s}

    # the plain FP64 drop-in on the same inputs (the metric's denominator)
    if args.precision == "mixed" and not args.no_dropin and args.krylov == "cg":
        d64 = wb.Solver(cats, wb.CG(precision="fp64"), weights=w)
        for _ in range(max(1, args.warmup - 1)):
            L.within_solver_solve_batch_device(d64._h, C.c_void_p(dY.data_ptr()), k, C.c_void_p(dX.data_ptr()),
                                               C.c_void_p(dD.data_ptr()), st, None)
        torch.cuda.synchronize()
        a0, a1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a0.record()
        for _ in range(args.steps):
            L.within_solver_solve_batch_device(d64._h, C.c_void_p(dY.data_ptr()), k, C.c_void_p(dX.data_ptr()),
                                               C.c_void_p(dD.data_ptr()), st, None)
        a1.record()
        torch.cuda.synchronize()
        d_ms = a0.elapsed_time(a1)
        if dist:
            d_ms = max_over_ranks(dist, d_ms)
        line["fp64_dropin"] = {"value": world * args.steps * k / (d_ms / 1000.0), "unit": "RHS/s",
                               "ms_per_step": d_ms / args.steps,
                               "converged": all(bool(st[c].converged) for c in range(k)),
                               "max_final_residual": max(float(st[c].final_residual) for c in range(k))}
        line["speedup_vs_fp64_dropin"] = line["fp64_dropin"]["ms_per_step"] / line["ms_per_step"]
        del d64

    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        threads = max(1, min(4, os.cpu_count() or 1))
        line["cpu_baseline"] = cpu_baseline_run(cats, Y, w, threads, threads)
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


def main():
    args = parse()
    if args.impl == "reference":
        reference_arm(args)
    else:
        ours(args)


if __name__ == "__main__":
    main()
