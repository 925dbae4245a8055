#!/usr/bin/env python
"""Benchmark: CG solves/s to relative residual 1e-10 on one B200.

Workload (default): the 3D 7-point 128^3 configuration (n = 2,097,152,
nnz = 14,581,760; off-diagonals -(f_i+f_j)/2 with f = 10^U[-3,0], diagonal
row |sum| + 1e-3, b = A x*, x* ~ U[-1,1], seed 1).  One step = one full solve
from x0 = 0 to ||b - A x|| / ||b|| <= 1e-10 with the matrix resident in HBM.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl mf|reference]

--impl mf        this library (value: device-resident solves; e2e: the
                 host-buffer C-ABI call mf_cg_solve_host, b in and x out
                 through pinned host memory every step)
--impl reference the reference's own CPU tiled path (Tile_create +
                 blockspmv_cpu from the reference sources, with a CG loop
                 around it), timed on the host cores on a bounded sample

N > 1 runs independent replicas, one per GPU (a single system does not
shard), timed with CUDA events and reported as the max over
ranks.
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
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "CG solves/sec at rel-res 1e-10: learned/batched vs plain FP64 tiled, 1 B200"
UNIT = "solves/s"
GRID = 128
SEED = 1
TOL = 1e-10
# FP64 CG iterations to 1e-10 on this configuration, from the CPU oracle
# (tests/test_config_iterations.py pins it); used to scale the CPU sample.
FP64_ITERS_ORACLE = 598


def load_peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def ncu_traffic(kernel):
    """Per-iteration DRAM bytes of `kernel` from the committed ncu summary."""
    p = ROOT / "profiles" / "ncu_traffic.json"
    if not p.exists():
        return None
    d = json.loads(p.read_text())
    return d.get(kernel)


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index):
        self.dev = device_index
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(prefix="mf_clocks_", suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-lms", "100",
                 "-i", str(self.dev)], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
            time.sleep(0.3)
        except FileNotFoundError:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            time.sleep(0.15)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if not self.path or not os.path.exists(self.path):
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        os.unlink(self.path)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


def build_problem(mf):
    A = mf.synth_poisson3d_scaled(GRID, SEED)
    xs = mf.synth_xstar(SEED, A.n_rows)
    b = A.matvec(xs)
    return A, xs, b


class CpuReference:
    """The reference CPU tiled path (its Tile_create + blockspmv_cpu, compiled
    from its sources into oracle/_ref) with a CG loop around it; each sample
    is a bounded number of CG iterations."""

    def __init__(self, A, b, threads=None):
        sys.path.insert(0, str(ROOT / "tests"))
        import oracle_lib as ol  # CPU-baseline leg only

        self.ref = ref = ol.reference()
        if ref is None:
            return
        ref.ref_cg_iterations.argtypes = [C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p,
                                          C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int, C.POINTER(C.c_double)]
        ref.ref_cg_iterations.restype = C.c_double
        self.threads = threads or os.cpu_count() or 1
        self.A = A
        csr = ol.Csr(A.n_rows, A.n_cols, A.rowptr, A.colidx, A.val)
        t0 = time.perf_counter()
        sizes, _ = ol.reference_tiles(csr)
        self.setup_s = time.perf_counter() - t0
        ref.ref_encode_last()
        nx = sizes["tilen"] * 16
        self.x, self.r, self.p, self.q, self.b = (np.zeros(nx) for _ in range(5))
        self.b[: A.n_rows] = b
        self.rho = C.c_double(0.0)
        self._run(1, start=1)

    def _run(self, iters, start=0):
        A = self.A
        return self.ref.ref_cg_iterations(A.n_rows, A.n_cols, A.nnz, self.b.ctypes.data, self.x.ctypes.data,
                                          self.r.ctypes.data, self.p.ctypes.data, self.q.ctypes.data, iters,
                                          self.threads, start, C.byref(self.rho))

    def seconds_per_iteration(self, iters):
        return self._run(iters) / iters

    def auto_iters(self, budget_s):
        one = self._run(1)
        return int(max(3, min(500, budget_s / max(one, 1e-6))))


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    import __graft_entry__ as ge

    mf = ge.load_package()
    A, xs, b = build_problem(mf)
    iters = FP64_ITERS_ORACLE
    cpu = CpuReference(A, b)
    if cpu.ref is None:
        print(json.dumps({"impl": "reference", "unavailable": "reference CPU code not built (oracle/_ref)"}))
        return 0
    # each step is a bounded sample of CG iterations sized so the whole run
    # stays within a few minutes
    per_step = cpu.auto_iters(max(1.0, 60.0 / max(1, args.warmup + args.steps)))
    step_vals = []
    for s in range(args.warmup + args.steps):
        t = cpu.seconds_per_iteration(per_step)
        if s >= args.warmup:
            step_vals.append(1.0 / (t * iters))
    v = statistics.median(step_vals)
    line = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 / v, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": f"poisson3d_scaled_{GRID}^3 CG to 1e-10", "n": A.n_rows, "nnz": A.nnz, "seed": SEED,
                   "l2": "inputs larger than L2", "reference_setup_s": cpu.setup_s},
        "cpu_baseline": {"value": v, "unit": UNIT, "cores": cpu.threads, "kind": "reference",
                         "sample": f"{per_step} CG iterations per step (reference blockspmv_cpu, serial, "
                                   f"+ OpenMP vector loops), scaled by {iters} FP64 iterations to 1e-10"},
        "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))
    return 0


def run_mf(args):
    import torch
    import torch.distributed as dist

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta

        dist.init_process_group("nccl", timeout=timedelta(seconds=300), device_id=torch.device("cuda", local))
    import __graft_entry__ as ge

    mf = ge.load_package()
    L = mf.lib()
    A, xs, b = build_problem(mf)
    t0 = time.perf_counter()
    M = mf.Matrix(A)
    torch.cuda.synchronize()
    setup_ms = (time.perf_counter() - t0) * 1e3
    n = A.n_rows
    db = torch.from_numpy(b).cuda()
    dx = torch.zeros(n, dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream()
    if args.iters:
        opts = mf.solve_opts(tol=-1.0, maxiter=args.iters, policy=args.policy)
    else:
        opts = mf.solve_opts(tol=TOL, maxiter=20000, policy=args.policy)
    rep = mf.SolveReport()

    def solve():
        st = L.mf_cg_solve(M.h, db.data_ptr(), dx.data_ptr(), C.byref(opts), C.byref(rep), None, stream.cuda_stream)
        if st != 0:
            mf.check(st)

    for _ in range(args.warmup):
        solve()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    launches0 = L.mf_kernel_launches()
    kernel_ms, iters, bytes_moved = [], [], []
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        ev0.record(stream)
        for _ in range(args.steps):
            solve()
            kernel_ms.append(rep.kernel_ms)
            iters.append(rep.iterations)
            bytes_moved.append(rep.bytes_moved)
        ev1.record(stream)
        torch.cuda.synchronize()
    launches = L.mf_kernel_launches() - launches0
    ms = ev0.elapsed_time(ev1)
    if world > 1:
        t = torch.tensor([ms], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    value = args.steps * world / (ms * 1e-3)
    if args.profile:
        if rank == 0:
            print(json.dumps({"profile_run": True, "ms_per_step": ms / args.steps, "iterations": rep.iterations,
                              "kernel_ms": rep.kernel_ms, "launches": int(launches)}))
        M.close()
        if world > 1:
            dist.destroy_process_group()
        return 0
    relres_true = rep.relres_true
    x_err = float(torch.max(torch.abs(dx.cpu() - torch.from_numpy(xs))).item())

    # e2e: the host-buffer C-ABI call, pinned b in and x out every step
    b_pin = torch.from_numpy(b).pin_memory()
    x_pin = torch.zeros(n, dtype=torch.float64).pin_memory()
    erep = mf.SolveReport()
    for _ in range(1):
        L.mf_cg_solve_host(M.h, b_pin.data_ptr(), x_pin.data_ptr(), C.byref(opts), C.byref(erep))
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        st = L.mf_cg_solve_host(M.h, b_pin.data_ptr(), x_pin.data_ptr(), C.byref(opts), C.byref(erep))
        if st != 0:
            mf.check(st)
    torch.cuda.synchronize()
    e2e_s = time.perf_counter() - t0
    if world > 1:
        t = torch.tensor([e2e_s], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_s = float(t.item())
    e2e = args.steps * world / e2e_s

    peak, peak_kind = load_peaks()
    mean_ms = statistics.mean(kernel_ms)
    per_launch_bytes = statistics.mean(bytes_moved)
    achieved = per_launch_bytes / (mean_ms * 1e-3) / 1e9
    kname = "k_cg_fp64" if args.policy == "fp64" else "k_cg_mixed"
    tr = ncu_traffic(kname)
    traffic = None if tr is None else tr["dram_bytes_per_iteration"] * statistics.mean(iters)
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "traffic": traffic, "peak_kind": peak_kind, "kernel": kname,
                "algorithmic_bytes_per_launch": per_launch_bytes, "launch_ms": mean_ms}
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64" if args.policy == "fp64" else "mixed(f16/f32 tiles, f32 accumulate, f64 refinement)",
        "data": "synthetic",
        "config": {"workload": f"poisson3d_scaled_{GRID}^3 CG to 1e-10", "n": n, "nnz": A.nnz, "seed": SEED,
                   "policy": args.policy, "iterations": int(statistics.mean(iters)), "relres_true": relres_true,
                   "max_abs_err_vs_xstar": x_err, "setup_ms": setup_ms, "parallelism": f"replicas x{world}",
                   "l2": "inputs larger than L2 (matrix ~200 MB vs 126 MB L2); no flush"},
        "roofline": roofline,
        "e2e": {"value": e2e, "unit": UNIT, "h2d_bytes_per_step": 8 * n, "d2h_bytes_per_step": 8 * n},
        "gpu_launches": int(launches),
        "clocks": clk.summary(),
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = CpuReference(A, b)
        if cpu.ref is not None:
            k = cpu.auto_iters(15.0)
            t = cpu.seconds_per_iteration(k)
            line["cpu_baseline"] = {"value": 1.0 / (t * FP64_ITERS_ORACLE), "unit": UNIT, "cores": cpu.threads,
                                    "kind": "reference",
                                    "sample": f"{k} CG iterations (reference blockspmv_cpu, serial, + OpenMP vector "
                                              f"loops on {cpu.threads} threads), scaled by {FP64_ITERS_ORACLE} "
                                              f"FP64 iterations to 1e-10; reference Tile_create {cpu.setup_s:.1f} s "
                                              f"not timed"}
    if rank == 0:
        print(json.dumps(line))
    M.close()
    if world > 1:
        dist.destroy_process_group()
    return 0


def main():
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["mf", "reference"], default="mf")
    ap.add_argument("--policy", default="fp64", choices=["fp64", "static", "rule", "learned"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--profile", action="store_true",
                    help="device solves only (no e2e, clocks or CPU baseline): the command profiled with ncu")
    ap.add_argument("--iters", type=int, default=0,
                    help="run a fixed number of CG iterations per solve instead of stopping at 1e-10 (profiling)")
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference(args)
    return run_mf(args)


if __name__ == "__main__":
    sys.exit(main())
