#!/usr/bin/env python
"""Benchmark: CG solves/s to relative residual 1e-10 on one B200.

Workloads (--workload):
  batched (default) 512 random SPD systems, n ~ log-uniform[1k, 64k], seeds
                  100-611 (random symmetric pattern, 8-32 draws per row,
                  values N(0,1) x row scale 10^U[-4,4], diagonal row |sum| +
                  1; b = A x*, x* ~ U[-1,1] from the system's seed), solved
                  by one graph-captured batched launch per step with the
                  learned per-chunk precision policy (--policy learned,
                  policy file mille-feuille_b200/policies/randspd_batched.mfpol,
                  trained on seeds 2000-2063); the static and rule policies
                  of the same batched solver and the plain FP64 tiled solves
                  of the same 512 systems one after another are timed in the
                  same run (static, rule and fp64 keys).  One step = every
                  system from x0 = 0 to ||b - A x|| / ||b|| <= 1e-10.
  poisson3d       3D 7-point 128^3 (n = 2,097,152, nnz = 14,581,760;
                  off-diagonals -(f_i+f_j)/2 with f = 10^U[-3,0], diagonal
                  row |sum| + 1e-3, b = A x*, x* ~ U[-1,1], seed 1), solved
                  with tile mixed precision and FP64 refinement (--policy
                  static); the plain FP64 tiled solve of the same system is
                  timed in the same run (fp64 key).  One step = one solve
                  from x0 = 0 to ||b - A x|| / ||b|| <= 1e-10, matrix
                  resident in HBM.
  lap2d           CG on the 2D 5-point Laplacian 128^2 (seed 0) to 1e-10: small
                  enough to live in L2; reports the latency-bound regime.
  convdiff        BiCGSTAB on the 96^3 convection-diffusion system to 1e-9.
  aniso           160^3 anisotropic diffusion (seed 3) with a learned policy
                  file (--policy-file), the rule policy and plain FP64.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl mf|reference]

--impl mf        this library (value: device-resident solves; e2e: the
                 host-buffer call, b in and x out through pinned host memory
                 every step)
--impl reference the reference's own CPU tiled path (Tile_create +
                 blockspmv_cpu from the reference sources, with a CG loop
                 around it) on the chosen workload, timed on the host cores
                 on a bounded sample (batched: a sample of the systems, one
                 per host core at once, scaled by the FP64 oracle's
                 iteration counts of all 512 systems)

N > 1: the batched workload is sharded -- rank r solves its own 512
systems (seeds 100 + 512 r ...), no collective on the data path -- and the
single-system workloads run independent replicas (a single system does not
shard); timed with CUDA events and reported as the max over ranks, value =
the systems of all ranks / that time (weak scaling).
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
# FP64 CG iterations to 1e-10 of the FP64 CPU oracle on the single-system
# configurations (tests/golden/config_iterations.json, recomputed by
# tests/test_config_iterations.py); they scale the CPU-baseline samples.
CONFIG_ITERS = json.loads((ROOT / "tests" / "golden" / "config_iterations.json").read_text())
FP64_ITERS_ORACLE = CONFIG_ITERS["poisson3d_scaled_128"]["iterations"]


def oracle_iterations(workload):
    """The FP64 oracle's iteration count for a single-system workload (None
    where no CPU baseline is scaled)."""
    key = {"poisson3d": "poisson3d_scaled_128", "lap2d": "laplace2d_128"}.get(workload)
    return CONFIG_ITERS[key]["iterations"] if key else None


def load_peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def ncu_traffic(kernel, workload, policy):
    """Per-iteration DRAM bytes of `kernel` from the committed ncu summary,
    only when that capture ran the same workload and precision policy (the
    figure belongs to one matrix and one payload)."""
    p = ROOT / "profiles" / "ncu_traffic.json"
    if not p.exists():
        return None
    e = json.loads(p.read_text()).get(kernel)
    if e is None or e.get("workload") != workload or (e.get("policy") is not None and e.get("policy") != policy):
        return None
    return e


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


BATCH_ORACLE = ROOT / "tests" / "golden" / "batched_oracle.json"
BATCH_POLICY = ROOT / "mille-feuille_b200" / "policies" / "randspd_batched.mfpol"


def _ref_batch_worker(task):
    """One sampled system of the batched configuration on one host thread:
    the reference's Tile_create and blockspmv_cpu (compiled from its sources
    into oracle/_ref) inside a CG loop, for about `budget_s` seconds; returns
    (seed, n, nnz, seconds per iteration).  The system comes from the
    oracle's restatement of the generator (no product library loaded)."""
    seed, budget_s = task
    sys.path.insert(0, str(ROOT / "tests"))
    import oracle_lib as ol  # CPU-baseline leg only

    ref = ol.reference()
    ref.ref_cg_iterations.argtypes = [C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p,
                                      C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int, C.POINTER(C.c_double)]
    ref.ref_cg_iterations.restype = C.c_double
    A = ol.oracle_random_spd(seed)
    b = A.to_scipy() @ ol.oracle_xstar(seed, A.n_rows)
    sizes, _ = ol.reference_tiles(A)
    ref.ref_encode_last()
    nx = sizes["tilen"] * 16
    x, r, p, q, bb = (np.zeros(nx) for _ in range(5))
    bb[: A.n_rows] = b
    rho = C.c_double(0.0)

    def run(k, start=0):
        return ref.ref_cg_iterations(A.n_rows, A.n_cols, A.nnz, bb.ctypes.data, x.ctypes.data, r.ctypes.data,
                                     p.ctypes.data, q.ctypes.data, k, 1, start, C.byref(rho))

    one = run(1, start=1)
    k = int(max(3, min(5000, budget_s / max(one, 1e-7))))
    return seed, A.n_rows, A.nnz, run(k) / k


class CpuBatchReference:
    """The reference CPU tiled path on the batched configuration, timed on a
    sample of its systems (evenly spaced in size), one system per host core
    at once (each on one thread, as blockspmv_cpu is serial), and scaled to
    the whole batch by the FP64 oracle's iteration counts of all 512 systems
    (tests/golden/batched_oracle.json): seconds per (entry x iteration) under
    that load times the batch's sum of iterations x entries, divided by the
    cores used.  The reference Tile_create is not timed (matrices resident,
    as on the GPU)."""

    def __init__(self, sample=16, budget_s=4.0, workers=None):
        import multiprocessing as mp

        fixture = json.loads(BATCH_ORACLE.read_text())
        self.systems = fixture["systems"]
        order = sorted(self.systems, key=lambda s: s["nnz"])
        idx = np.unique(np.linspace(0, len(order) - 1, sample).round().astype(int))
        self.seeds = [order[i]["seed"] for i in idx]
        self.cores = max(1, min(workers or os.cpu_count() or 1, len(self.seeds)))
        self.budget_s = budget_s
        self.work = sum(s["iterations"] * s["nnz"] for s in self.systems)
        self.pool = mp.get_context("spawn").Pool(self.cores)

    def measure(self, budget_s=None):
        """Seconds for the whole batch on the cores (one sample)."""
        b = budget_s or self.budget_s
        res = self.pool.map(_ref_batch_worker, [(s, b) for s in self.seeds])
        alpha = statistics.median(t / nnz for _, _, nnz, t in res)
        self.last = res
        return alpha * self.work / self.cores

    def close(self):
        self.pool.close()
        self.pool.join()

    def describe(self):
        return (f"{len(self.seeds)} of the 512 systems (evenly spaced in size), one per host core at once, each "
                f"timed for ~{self.budget_s:.0f} s of reference blockspmv_cpu CG iterations on one thread; seconds "
                f"per entry-iteration (median) x the batch's {self.work:.3e} entry-iterations (FP64 oracle "
                f"iteration counts) / {self.cores} cores; reference Tile_create not timed")


def run_reference_spmv(args):
    """The reference arm of --workload spmv: the reference's own
    blockspmv_cpu (serial, as the reference runs it, its schedule arrays
    allocated per call) on the same matrix and x, timed per call."""
    sys.path.insert(0, str(ROOT / "tests"))
    import oracle_lib as ol  # reference arm: the reference's own CPU code

    ref = ol.reference()
    if ref is None:
        print(json.dumps({"impl": "reference", "unavailable": "reference CPU code not built (oracle/_ref)"}))
        return 0
    import __graft_entry__ as ge

    mf = ge.load_package()
    A = mf.synth_poisson3d_scaled(GRID, SEED)
    csr = ol.Csr(A.n_rows, A.n_cols, A.rowptr, A.colidx, A.val)
    sizes, _ = ol.reference_tiles(csr)
    ref.ref_encode_last()
    nx = sizes["tilen"] * 16
    x = np.ascontiguousarray(mf.synth_xstar(SEED, nx))
    y = np.zeros(nx)
    p1 = np.zeros(sizes["tilenum"] + 1, np.int32)
    p2 = np.zeros(sizes["tilenum"] + 1, np.int32)
    vals = []
    for s in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        ref.ref_blockspmv(A.n_rows, A.n_cols, A.nnz, x, y, p1, p2, None, None, None)
        t = time.perf_counter() - t0
        if s >= args.warmup:
            vals.append(1.0 / t)
    v = statistics.median(vals)
    line = {"impl": "reference",
            "metric": "FP64 tiled SpMV/s (mf_spmv, bit-identical to the reference's blockspmv_cpu), 1 B200",
            "value": v, "unit": "spmv/s", "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1e3 / v, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64", "data": "synthetic",
            "config": {"workload": f"poisson3d_scaled_{GRID}^3 mf_spmv", "n": A.n_rows, "nnz": A.nnz},
            "cpu_baseline": {"value": v, "unit": "spmv/s", "cores": 1, "kind": "reference",
                             "sample": "one reference blockspmv_cpu call per step (serial), schedule included"},
            "e2e": {"value": v, "unit": "spmv/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    if args.workload == "batched":
        sys.path.insert(0, str(ROOT / "tests"))
        import oracle_lib as ol  # reference arm: the reference's own CPU code

        if ol.reference() is None:
            print(json.dumps({"impl": "reference", "unavailable": "reference CPU code not built (oracle/_ref)"}))
            return 0
        steps = args.warmup + args.steps
        cpu = CpuBatchReference(budget_s=max(0.5, min(8.0, 60.0 / max(1, steps))))
        vals = []
        try:
            for s in range(steps):
                t = cpu.measure()
                if s >= args.warmup:
                    vals.append(len(cpu.systems) / t)
        finally:
            cpu.close()
        v = statistics.median(vals)
        line = {
            "impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 / v * len(cpu.systems),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": BATCH_NAME, "systems": len(cpu.systems),
                       "l2": "host cores only (no device cache involved)"},
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": cpu.cores, "kind": "reference",
                             "sample": cpu.describe()},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        }
        print(json.dumps(line))
        return 0
    if args.workload == "spmv":
        return run_reference_spmv(args)
    if args.workload not in ("poisson3d",):
        print(json.dumps({"impl": "reference", "unavailable": f"no reference arm for --workload {args.workload} "
                                                              "(the reference arm measures batched, poisson3d, spmv)"}))
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
                   "l2": "host cores only (no device cache involved)", "reference_setup_s": cpu.setup_s},
        "cpu_baseline": {"value": v, "unit": UNIT, "cores": cpu.threads, "kind": "reference",
                         "sample": f"{per_step} CG iterations per step (reference blockspmv_cpu, serial, "
                                   f"+ OpenMP vector loops), scaled by {iters} FP64 iterations to 1e-10"},
        "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))
    return 0


L2_FLUSH_BYTES = 256 << 20  # twice the B200's 126 MB L2
L2_NOTE = "L2 flushed (256 MB write) before every timed step, outside its timed events"

_flush_buf = None


def _flush_l2(stream):
    """Overwrites a buffer twice the L2 size on `stream`, so that no input of
    the next step is served from L2."""
    import torch

    global _flush_buf
    if _flush_buf is None:
        _flush_buf = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device="cuda")
    with torch.cuda.stream(stream):
        _flush_buf.fill_(1)


def _timed(stream, fn, steps):
    """Device time of `steps` calls of fn: CUDA events on the launching stream
    around each call, L2 flushed before each (outside the events)."""
    import torch

    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    total = 0.0
    for _ in range(steps):
        _flush_l2(stream)
        ev0.record(stream)
        fn()
        ev1.record(stream)
        torch.cuda.synchronize()
        total += ev0.elapsed_time(ev1)
    return total


def _max_over_ranks(v, world):
    if world == 1:
        return v
    import torch
    import torch.distributed as dist

    # NCCL reduces device tensors; gloo (the CPU tests of this path) host ones
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([v], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def _barrier(world):
    if world > 1:
        import torch.distributed as dist

        dist.barrier()


def tiles_of(A):
    """Number of non-empty 16x16 tiles of a host CSR matrix."""
    rows = np.repeat(np.arange(A.n_rows, dtype=np.int64), np.diff(A.rowptr))
    key = (rows // 16) * ((A.n_cols + 15) // 16) + A.colidx.astype(np.int64) // 16
    return int(np.unique(key).size)


def workload_single(args, mf, world, local):
    """poisson3d / convdiff / aniso: one system, device-resident solves."""
    import torch

    L = mf.lib()
    method = "bicgstab" if args.workload == "convdiff" else "cg"
    if args.workload == "poisson3d":
        A = mf.synth_poisson3d_scaled(GRID, SEED)
        seed, tol, name = SEED, TOL, f"poisson3d_scaled_{GRID}^3 CG to 1e-10"
    elif args.workload == "lap2d":
        A = mf.synth_laplace2d(128, 128)
        seed, tol, name = 0, TOL, "laplace2d_128^2 CG to 1e-10 (L2-resident, latency-bound)"
    elif args.workload == "convdiff":
        A = mf.synth_convdiff3d(96)
        seed, tol, name = 2, 1e-9, "convdiff3d_96^3 BiCGSTAB to 1e-9"
    else:
        A = mf.synth_aniso3d(160, 3)
        seed, tol, name = 3, TOL, "aniso3d_160^3 (lognormal k, sigma 2, corr 8, k_z x100) CG to 1e-10"
    xs = mf.synth_xstar(seed, A.n_rows)
    b = A.matvec(xs)
    t0 = time.perf_counter()
    M = mf.Matrix(A)
    torch.cuda.synchronize()
    setup_ms = (time.perf_counter() - t0) * 1e3
    pol = None
    if args.policy == "learned":
        if not args.policy_file:
            raise SystemExit("--policy learned needs --policy-file")
        pol = mf.Policy.load(args.policy_file)
        M.attach_policy(pol)
    n = A.n_rows
    db = torch.from_numpy(b).cuda()
    dx = torch.zeros(n, dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream()
    fn_dev = L.mf_bicgstab_solve if method == "bicgstab" else L.mf_cg_solve
    fn_host = L.mf_bicgstab_solve_host if method == "bicgstab" else L.mf_cg_solve_host

    maxiter = 400000 if args.workload == "aniso" else 50000

    def opts_for(policy):
        if args.iters:
            return mf.solve_opts(tol=-1.0, maxiter=args.iters, policy=policy)
        return mf.solve_opts(tol=tol, maxiter=maxiter, policy=policy)

    def make_solve(policy, rep):
        o = opts_for(policy)

        def solve():
            st = fn_dev(M.h, db.data_ptr(), dx.data_ptr(), C.byref(o), C.byref(rep), None, stream.cuda_stream)
            if st != 0:
                mf.check(st)
        return solve

    rep = mf.SolveReport()
    solve = make_solve(args.policy, rep)
    for _ in range(args.warmup):
        solve()
    torch.cuda.synchronize()
    _barrier(world)
    torch.cuda.synchronize()
    launches0 = L.mf_kernel_launches()
    kernel_ms, iters, bytes_moved = [], [], []

    def step():
        solve()
        kernel_ms.append(rep.kernel_ms)
        iters.append(rep.iterations)
        bytes_moved.append(rep.bytes_moved)

    with ClockSampler(local) as clk:
        ms = _timed(stream, step, args.steps)
    launches = L.mf_kernel_launches() - launches0
    ms = _max_over_ranks(ms, world)
    value = args.steps * world / (ms * 1e-3)
    result = {"rep": rep, "ms": ms, "value": value, "launches": launches, "clocks": clk.summary(),
              "kernel_ms": kernel_ms, "iters": iters, "bytes_moved": bytes_moved}
    if args.profile:
        return result, None
    relres_true = rep.relres_true
    x_err = float(torch.max(torch.abs(dx.cpu() - torch.from_numpy(xs))).item())
    info = {"workload": name, "n": n, "nnz": A.nnz, "seed": seed, "policy": args.policy,
            "iterations": int(statistics.mean(iters)), "refinements": int(rep.refinements),
            "relres_true": relres_true, "max_abs_err_vs_xstar": x_err, "setup_ms": setup_ms,
            "parallelism": f"replicas x{world}",
            "l2": L2_NOTE}
    # the plain FP64 tiled solve of the same system, same box, same run
    if args.policy != "fp64" and not args.iters:
        rep64 = mf.SolveReport()
        s64 = make_solve("fp64", rep64)
        s64()
        torch.cuda.synchronize()
        _barrier(world)
        k = max(3, args.steps // 2)
        ms64 = _max_over_ranks(_timed(stream, s64, k), world)
        info["fp64"] = {"value": k * world / (ms64 * 1e-3), "unit": UNIT, "iterations": rep64.iterations,
                        "relres_true": rep64.relres_true, "steps": k}
        if args.workload == "aniso" and args.policy == "learned":
            repr_ = mf.SolveReport()
            sr = make_solve("rule", repr_)
            sr()
            torch.cuda.synchronize()
            msr = _max_over_ranks(_timed(stream, sr, k), world)
            info["rule"] = {"value": k * world / (msr * 1e-3), "unit": UNIT, "iterations": repr_.iterations,
                            "relres_true": repr_.relres_true, "steps": k}
    # e2e: the host-buffer C-ABI call, pinned b in and x out every step
    o = opts_for(args.policy)
    b_pin = torch.from_numpy(b).pin_memory()
    x_pin = torch.zeros(n, dtype=torch.float64).pin_memory()
    erep = mf.SolveReport()
    fn_host(M.h, b_pin.data_ptr(), x_pin.data_ptr(), C.byref(o), C.byref(erep))
    torch.cuda.synchronize()
    _barrier(world)
    e2e_s = 0.0
    for _ in range(args.steps):
        _flush_l2(stream)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        st = fn_host(M.h, b_pin.data_ptr(), x_pin.data_ptr(), C.byref(o), C.byref(erep))
        if st != 0:
            mf.check(st)
        torch.cuda.synchronize()
        e2e_s += time.perf_counter() - t0
    e2e_s = _max_over_ranks(e2e_s, world)
    result["e2e"] = {"value": args.steps * world / e2e_s, "unit": UNIT, "h2d_bytes_per_step": 8 * n,
                     "d2h_bytes_per_step": 8 * n}
    mean_ms = statistics.mean(kernel_ms)
    per_launch = statistics.mean(bytes_moved)
    kname = ("k_bicgstab" if method == "bicgstab" else "k_cg") + ("_fp64" if args.policy == "fp64" else "_mixed")
    result["roofline_in"] = (per_launch, mean_ms, kname, statistics.mean(iters))
    result["dtype"] = "f64" if args.policy == "fp64" else "mixed(f32/f16/i8 tiles, f32 accumulate, f64 refinement)"
    # FP64 CG iterations to 1e-10 from the CPU oracle (scale of the CPU sample)
    oracle_iters = oracle_iterations(args.workload)
    result["cpu"] = (A, b, oracle_iters) if oracle_iters else None
    M.close()
    return result, info


def workload_spmv(args, mf, world, local):
    """The standalone FP64 tiled SpMV (mf_spmv, k_spmv_fp64) on the
    poisson3d matrix; value = SpMVs per second.  Algorithmic bytes of one
    SpMV: nnz x (8-byte value + 1-byte in-tile column) + 24 bytes per tile
    (tile column, entry offset, 16 row pointers) + x read once and y written
    once (16 bytes per row)."""
    import torch

    L = mf.lib()
    A = mf.synth_poisson3d_scaled(GRID, SEED)
    M = mf.Matrix(A)
    inf = M.info()
    n, T = A.n_rows, inf.tilenum
    xs = mf.synth_xstar(SEED, inf.tilen * 16)
    dx = torch.from_numpy(xs).cuda()
    dy = torch.zeros(n, dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream()
    reps = 20  # SpMVs per step

    def spmv():
        for _ in range(reps):
            st = L.mf_spmv(M.h, dx.data_ptr(), dy.data_ptr(), stream.cuda_stream)
            if st != 0:
                mf.check(st)

    for _ in range(args.warmup):
        spmv()
    torch.cuda.synchronize()
    _barrier(world)
    launches0 = L.mf_kernel_launches()
    with ClockSampler(local) as clk:
        ms = _timed(stream, spmv, args.steps)
    launches = L.mf_kernel_launches() - launches0
    ms = _max_over_ranks(ms, world)
    value = reps * args.steps * world / (ms * 1e-3)
    result = {"ms": ms, "value": value, "launches": launches, "clocks": clk.summary(),
              "metric": "FP64 tiled SpMV/s (mf_spmv, bit-identical to the reference's blockspmv_cpu), 1 B200",
              "unit": "spmv/s"}
    if args.profile:
        return result, None
    y = dy.cpu().numpy()
    err = float(np.max(np.abs(y - A.matvec(xs[:n]))) / max(1e-300, np.max(np.abs(y))))
    bytes_spmv = A.nnz * 9 + 24 * T + 16 * n
    info = {"workload": f"poisson3d_scaled_{GRID}^3 mf_spmv", "n": n, "nnz": A.nnz, "tiles": T,
            "spmv_per_step": reps, "rel_diff_vs_scipy": err, "parallelism": f"replicas x{world}",
            "l2": "matrix (186 MB) larger than L2; no flush between SpMVs"}
    # e2e: x from pinned host memory, one SpMV, y back, every step
    x_pin = torch.from_numpy(xs).pin_memory()
    y_pin = torch.zeros(n, dtype=torch.float64).pin_memory()
    e2e_s = 0.0
    for _ in range(args.steps):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        dx.copy_(x_pin, non_blocking=True)
        L.mf_spmv(M.h, dx.data_ptr(), dy.data_ptr(), stream.cuda_stream)
        y_pin.copy_(dy, non_blocking=True)
        torch.cuda.synchronize()
        e2e_s += time.perf_counter() - t0
    e2e_s = _max_over_ranks(e2e_s, world)
    result["e2e"] = {"value": args.steps * world / e2e_s, "unit": "spmv/s", "h2d_bytes_per_step": 8 * len(xs),
                     "d2h_bytes_per_step": 8 * n}
    result["roofline_in"] = (bytes_spmv, ms / (reps * args.steps), "k_spmv_fp64", None)
    result["dtype"] = "f64"
    result["cpu"] = None
    M.close()
    return result, info


def workload_spmm_f16(args, mf, world, local):
    """mf_spmm_f16 (16 right-hand sides, the dense 16x16 tiles on the tensor
    cores) on a block-structured matrix of 32,768 block rows (a dense
    diagonal block and 3 random dense blocks per block row, 2 random sparse
    entries per row); value = SpMMs per second, the FP64 mf_spmm of the same
    product beside it.  Algorithmic bytes per launch: 512 per dense tile
    (FP16) + 5 per sparse entry (FP32 value, in-tile column) + 24 per tile +
    X read (FP64, 128 B per row) and packed (FP16, 32 B per row written and
    read) + Y written (FP64, 128 B per row)."""
    import torch

    L = mf.lib()
    H = mf.synth_block_dense(32768, 3, 2, 7)
    M = mf.Matrix(H)
    inf = M.info()
    n, k = H.n_rows, 16
    X = torch.from_numpy(np.random.default_rng(7).normal(size=(k, n))).cuda()
    Y = torch.zeros(k, n, dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream()
    nd = C.c_int()
    reps = 20

    def f16():
        for _ in range(reps):
            st = L.mf_spmm_f16(M.h, k, X.data_ptr(), n, Y.data_ptr(), n, 0, C.byref(nd), stream.cuda_stream)
            if st != 0:
                mf.check(st)

    def f64():
        for _ in range(reps):
            st = L.mf_spmm(M.h, k, X.data_ptr(), n, Y.data_ptr(), n, stream.cuda_stream)
            if st != 0:
                mf.check(st)

    for _ in range(args.warmup):
        f16()
    torch.cuda.synchronize()
    _barrier(world)
    launches0 = L.mf_kernel_launches()
    with ClockSampler(local) as clk:
        ms = _timed(stream, f16, args.steps)
    launches = L.mf_kernel_launches() - launches0
    ms = _max_over_ranks(ms, world)
    result = {"ms": ms, "value": reps * args.steps * world / (ms * 1e-3), "launches": launches,
              "clocks": clk.summary(), "unit": "spmm/s",
              "metric": "SpMM/s, 16 right-hand sides, dense tiles on tensor cores (mf_spmm_f16), 1 B200"}
    if args.profile:
        return result, None
    y16 = Y.cpu().numpy().copy()
    f64()
    torch.cuda.synchronize()
    ms64 = _max_over_ranks(_timed(stream, f64, max(3, args.steps // 2)), world)
    y64 = Y.cpu().numpy()
    dense_entries = 256 * nd.value
    sparse_entries = H.nnz - dense_entries
    npad = inf.tilen * 16
    bytes_launch = 512 * nd.value + 5 * sparse_entries + 24 * inf.tilenum + 128 * n + 64 * npad + 128 * n
    info = {"workload": "block-dense 32768 x (16x16 diagonal + 3 dense blocks) + 2 sparse per row, k = 16",
            "n": n, "nnz": H.nnz, "tiles": inf.tilenum, "dense_tiles": nd.value,
            "max_rel_diff_vs_fp64_spmm": float(np.max(np.abs(y16 - y64)) / np.max(np.abs(y64))),
            "fp64_spmm": {"value": reps * max(3, args.steps // 2) * world / (ms64 * 1e-3), "unit": "spmm/s",
                          "what": "mf_spmm of the same product (FP64, SIMT)"},
            "tensor_tflops": 2 * 16 * 16 * 16 * nd.value / (ms / (reps * args.steps) * 1e-3) / 1e12,
            "parallelism": f"replicas x{world}", "l2": "matrix larger than L2; no flush between SpMMs"}
    # e2e: X from pinned host memory, one SpMM, Y back, every step
    x_pin = X.cpu().pin_memory()
    y_pin = torch.zeros_like(x_pin).pin_memory()
    e2e_s = 0.0
    for _ in range(args.steps):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        X.copy_(x_pin, non_blocking=True)
        L.mf_spmm_f16(M.h, k, X.data_ptr(), n, Y.data_ptr(), n, 0, None, stream.cuda_stream)
        y_pin.copy_(Y, non_blocking=True)
        torch.cuda.synchronize()
        e2e_s += time.perf_counter() - t0
    e2e_s = _max_over_ranks(e2e_s, world)
    result["e2e"] = {"value": args.steps * world / e2e_s, "unit": "spmm/s", "h2d_bytes_per_step": 8 * k * n,
                     "d2h_bytes_per_step": 8 * k * n}
    result["roofline_in"] = (bytes_launch, ms / (reps * args.steps), "k_spmm_tc", None)
    result["dtype"] = "mixed(f16 dense tiles and x on tensor cores, f32 sparse tiles, f32 accumulate)"
    result["cpu"] = None
    M.close()
    return result, info


BATCH_NAME = ("batched random SPD x512 (n ~ log-uniform[1k,64k], seeds 100-611, 8-32 draws per row, "
              "row scale 10^U[-4,4]) CG to 1e-10")


def batch_seeds(rank, count):
    """The seeds of rank `rank`'s shard of the batched workload: rank 0 has
    the benchmark's 100 .. 100 + count - 1, rank r the next `count` after
    rank r - 1's (disjoint shards of one larger batch)."""
    return [100 + rank * count + k for k in range(count)]


def workload_batched(args, mf, world, local):
    """512 random SPD systems per GPU in one graph-captured batched launch
    (rank r: its own shard of systems, batch_seeds)."""
    import torch
    from concurrent.futures import ThreadPoolExecutor

    L = mf.lib()
    N = args.systems
    rank = int(os.environ.get("RANK", "0"))
    seeds = batch_seeds(rank, N)
    with ThreadPoolExecutor(16) as ex:
        systems = list(ex.map(lambda k: mf.synth_random_spd(seeds[k]), range(N)))
        xs = list(ex.map(lambda k: mf.synth_xstar(seeds[k], systems[k].n_rows), range(N)))
    bs = [A.matvec(x) for A, x in zip(systems, xs)]
    t0 = time.perf_counter()
    B = mf.Batch(systems)
    setup_ms = (time.perf_counter() - t0) * 1e3
    pol = None
    if args.policy == "learned":
        pol = mf.Policy.load(args.policy_file or BATCH_POLICY)
        B.attach_policy(pol)
    bstack = B.stack(bs)
    db = torch.from_numpy(bstack).cuda()
    dx = torch.zeros_like(db)
    stream = torch.cuda.current_stream()

    def make_solve(policy, rep):
        o = mf.solve_opts(tol=TOL, maxiter=50000, policy=policy)

        def solve():
            st = L.mf_batch_cg_solve(B.h, db.data_ptr(), dx.data_ptr(), C.byref(o), 1, C.byref(rep),
                                     stream.cuda_stream)
            if st != 0:
                mf.check(st)
        return solve

    rep = mf.BatchReport()
    solve = make_solve(args.policy, rep)
    for _ in range(args.warmup):
        solve()
    torch.cuda.synchronize()
    _barrier(world)
    launches0 = L.mf_kernel_launches()
    kernel_ms, bytes_moved = [], []

    def step():
        solve()
        kernel_ms.append(rep.kernel_ms)
        bytes_moved.append(rep.bytes_moved)

    with ClockSampler(local) as clk:
        ms = _timed(stream, step, args.steps)
    launches = L.mf_kernel_launches() - launches0
    ms = _max_over_ranks(ms, world)
    its, rr = B.results()
    value = N * args.steps * world / (ms * 1e-3)
    result = {"rep": rep, "ms": ms, "value": value, "launches": launches, "clocks": clk.summary()}
    if args.profile:
        return result, None
    # accuracy: FP64 true residual of every system, the error against x*,
    # and against the FP64 CPU oracle's solution on the four smallest systems
    x = dx.cpu().numpy()
    xparts = B.split(x)
    err_xs = max(float(np.max(np.abs(xp - xv))) for xp, xv in zip(xparts, xs))
    sys.path.insert(0, str(ROOT / "tests"))
    import oracle_lib as ol  # checker only

    fixture = json.loads(BATCH_ORACLE.read_text())["systems"] if BATCH_ORACLE.exists() else None
    small = sorted(range(N), key=lambda k: systems[k].n_rows)[:4]
    err_or = 0.0
    for k in small:
        A = systems[k]
        _, x_o, _ = ol.oracle_cg(ol.Csr(A.n_rows, A.n_cols, A.rowptr, A.colidx, A.val), bs[k], 50000, TOL)
        err_or = max(err_or, float(np.max(np.abs(xparts[k] - x_o))))
    info = {"workload": BATCH_NAME, "systems": N, "rows_total": int(sum(A.n_rows for A in systems)),
            "nnz_total": int(sum(A.nnz for A in systems)), "policy": args.policy,
            "policy_file": str(Path(args.policy_file or BATCH_POLICY).relative_to(ROOT)) if pol else None,
            "iterations_total": int(its.sum()), "iterations_max": int(its.max()),
            "relres_true_max": float(rep.relres_true_max), "failed": int(rep.failed),
            "fp16_share": float(rep.fp16_share), "max_abs_err_vs_xstar": err_xs,
            "max_abs_err_vs_fp64_oracle_4_smallest": err_or, "setup_ms": setup_ms,
            "lanes_per_row": int(rep.lanes_per_row), "cluster_ctas": int(rep.cluster_ctas),
            "parallelism": f"sharded x{world} (disjoint systems per GPU)", "l2": L2_NOTE}
    if fixture is not None and N == len(fixture) and rank == 0:
        it_o = np.array([s["iterations"] for s in fixture])
        info["iterations_vs_fp64_oracle"] = float(its.sum() / it_o.sum())
        info["oracle_max_abs_err_vs_xstar"] = max(s["max_abs_err_vs_xstar"] for s in fixture)
    # the other policies of the same batched solver, same run
    k = max(2, args.steps // 4)
    for other in ("static", "rule"):
        if other == args.policy:
            continue
        orep = mf.BatchReport()
        osolve = make_solve(other, orep)
        osolve()
        torch.cuda.synchronize()
        oms = _max_over_ranks(_timed(stream, osolve, k), world)
        info[other] = {"value": N * k * world / (oms * 1e-3), "unit": UNIT, "iterations_total": int(orep.iterations_total),
                       "relres_true_max": float(orep.relres_true_max), "fp16_share": float(orep.fp16_share),
                       "steps": k}
    # the plain FP64 tiled solves of the same systems, one after another
    if not args.no_fp64_baseline:
        dbs = [torch.from_numpy(bv).cuda() for bv in bs]
        mats = [mf.Matrix(A) for A in systems]
        o64 = mf.solve_opts(tol=TOL, maxiter=50000, policy="fp64")
        r64 = mf.SolveReport()
        xk = torch.zeros(max(A.n_rows for A in systems), dtype=torch.float64, device="cuda")
        it64 = []

        def seq():
            it64.clear()
            for M_, d in zip(mats, dbs):
                L.mf_cg_solve(M_.h, d.data_ptr(), xk.data_ptr(), C.byref(o64), C.byref(r64), None,
                              stream.cuda_stream)
                it64.append(r64.iterations)

        seq()
        torch.cuda.synchronize()
        ms64 = _max_over_ranks(_timed(stream, seq, 1), world)
        info["fp64"] = {"value": N * world / (ms64 * 1e-3), "unit": UNIT, "iterations_total": int(sum(it64)),
                        "what": "the same 512 systems solved one after another by the plain FP64 tiled CG"}
        for M_ in mats:
            M_.close()
    # e2e: stacked b from pinned host memory, solve, x back, every step
    b_pin = torch.from_numpy(bstack).pin_memory()
    x_pin = torch.zeros_like(b_pin).pin_memory()
    _barrier(world)
    e2e_s = 0.0
    for _ in range(args.steps):
        _flush_l2(stream)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        db.copy_(b_pin, non_blocking=True)
        solve()
        x_pin.copy_(dx, non_blocking=True)
        torch.cuda.synchronize()
        e2e_s += time.perf_counter() - t0
    e2e_s = _max_over_ranks(e2e_s, world)
    result["e2e"] = {"value": N * args.steps * world / e2e_s, "unit": UNIT,
                     "h2d_bytes_per_step": 8 * len(bstack), "d2h_bytes_per_step": 8 * len(bstack)}
    # roofline numerator: the kernel's own count of the bytes its passes
    # stream (each chunk in its working class: values + 16-bit columns + row
    # pointers, + row scale and diagonal for FP16 chunks), the vector
    # streams of each iteration and the FP64 reliable updates
    result["roofline_in"] = (statistics.mean(bytes_moved), statistics.mean(kernel_ms), "k_batched_cg", None)
    result["dtype"] = ("f64" if args.policy == "fp64" else
                       "mixed(fp32 / row-scaled fp16 chunks, f32 accumulate, f64 refinement)")
    result["cpu_batch"] = N == 512
    result["cpu"] = None
    B.close()
    return result, info


def workload_multi(args, mf, world, local):
    """k right-hand sides of the poisson3d system solved together by
    mf_cg_solve_multi (FP64, one pass over the matrix per iteration for all
    of them); value = right-hand sides solved per second."""
    import torch

    L = mf.lib()
    k = args.rhs
    A = mf.synth_poisson3d_scaled(GRID, SEED)
    n = A.n_rows
    B = np.stack([A.matvec(mf.synth_xstar(SEED + j, n)) for j in range(k)])  # k x n: column-major n x k
    t0 = time.perf_counter()
    M = mf.Matrix(A)
    torch.cuda.synchronize()
    setup_ms = (time.perf_counter() - t0) * 1e3
    dB = torch.from_numpy(B).cuda()
    dX = torch.zeros((k, n), dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream()
    reps = (mf.SolveReport * k)()
    o = (mf.solve_opts(tol=-1.0, maxiter=args.iters) if args.iters else mf.solve_opts(tol=TOL, maxiter=50000))

    def solve():
        st = L.mf_cg_solve_multi(M.h, k, dB.data_ptr(), n, dX.data_ptr(), n, C.byref(o), reps, stream.cuda_stream)
        if st != 0:
            mf.check(st)

    for _ in range(args.warmup):
        solve()
    torch.cuda.synchronize()
    _barrier(world)
    launches0 = L.mf_kernel_launches()
    kernel_ms, bytes_moved, iters = [], [], []

    def step():
        solve()
        kernel_ms.append(reps[0].kernel_ms)
        bytes_moved.append(reps[0].bytes_moved)
        iters.append(max(r.iterations for r in reps))

    with ClockSampler(local) as clk:
        ms = _timed(stream, step, args.steps)
    launches = L.mf_kernel_launches() - launches0
    ms = _max_over_ranks(ms, world)
    value = k * args.steps * world / (ms * 1e-3)
    result = {"ms": ms, "value": value, "launches": launches, "clocks": clk.summary()}
    if args.profile:
        return result, None
    its = [r.iterations for r in reps]
    info = {"workload": f"poisson3d_scaled_{GRID}^3, {k} right-hand sides (x* seeds {SEED}-{SEED + k - 1}) "
                        f"CG to 1e-10 together", "n": n, "nnz": A.nnz, "rhs": k, "policy": "fp64",
            "iterations_min": min(its), "iterations_max": max(its),
            "relres_true_max": max(r.relres_true for r in reps), "setup_ms": setup_ms,
            "parallelism": f"replicas x{world}", "l2": L2_NOTE}
    if not args.no_fp64_baseline:
        rep1 = mf.SolveReport()
        db1 = dB[0].contiguous()
        dx1 = torch.zeros(n, dtype=torch.float64, device="cuda")
        o1 = mf.solve_opts(tol=TOL, maxiter=50000, policy="fp64")

        def s1():
            st = L.mf_cg_solve(M.h, db1.data_ptr(), dx1.data_ptr(), C.byref(o1), C.byref(rep1), None,
                               stream.cuda_stream)
            if st != 0:
                mf.check(st)

        s1()
        torch.cuda.synchronize()
        ms1 = _max_over_ranks(_timed(stream, s1, 3), world)
        info["fp64_single"] = {"value": 3 * world / (ms1 * 1e-3), "unit": UNIT, "iterations": rep1.iterations,
                               "what": "the first right-hand side alone by the single-vector FP64 CG"}
    # e2e: pinned host B in and X out every step through mf_cg_solve_multi_host
    b_pin = torch.from_numpy(B).pin_memory()
    x_pin = torch.zeros((k, n), dtype=torch.float64).pin_memory()
    ereps = (mf.SolveReport * k)()
    L.mf_cg_solve_multi_host(M.h, k, b_pin.data_ptr(), x_pin.data_ptr(), C.byref(o), ereps)
    _barrier(world)
    e2e_s = 0.0
    for _ in range(args.steps):
        _flush_l2(stream)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        st = L.mf_cg_solve_multi_host(M.h, k, b_pin.data_ptr(), x_pin.data_ptr(), C.byref(o), ereps)
        if st != 0:
            mf.check(st)
        e2e_s += time.perf_counter() - t0
    e2e_s = _max_over_ranks(e2e_s, world)
    result["e2e"] = {"value": k * args.steps * world / e2e_s, "unit": UNIT, "h2d_bytes_per_step": 8 * n * k,
                     "d2h_bytes_per_step": 8 * n * k}
    result["roofline_in"] = (statistics.mean(bytes_moved), statistics.mean(kernel_ms), "k_mr_spmm+k_mr_update+"
                             "k_mr_pupdate (multi-RHS FP64 CG)", statistics.mean(iters))
    result["dtype"] = "f64"
    result["cpu"] = None
    M.close()
    return result, info


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
    if args.workload == "batched":
        res, info = workload_batched(args, mf, world, local)
    elif args.workload == "multirhs":
        res, info = workload_multi(args, mf, world, local)
    elif args.workload == "spmv":
        res, info = workload_spmv(args, mf, world, local)
    elif args.workload == "spmm_f16":
        res, info = workload_spmm_f16(args, mf, world, local)
    else:
        res, info = workload_single(args, mf, world, local)
    if args.profile:
        if rank == 0:
            print(json.dumps({"profile_run": True, "ms_per_step": res["ms"] / args.steps,
                              "launches": int(res["launches"])}))
        if world > 1:
            dist.destroy_process_group()
        return 0
    peak, peak_kind = load_peaks()
    per_launch, mean_ms, kname, mean_iters = res["roofline_in"]
    achieved = per_launch / (mean_ms * 1e-3) / 1e9
    tr = ncu_traffic(kname, args.workload, args.policy)
    traffic = None
    if tr is not None and "dram_bytes_per_launch" in tr:
        traffic = tr["dram_bytes_per_launch"]
    elif tr is not None and mean_iters is not None:
        traffic = tr["dram_bytes_per_iteration"] * mean_iters
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "traffic": traffic, "peak_kind": peak_kind, "kernel": kname,
                "algorithmic_bytes_per_launch": per_launch, "launch_ms": mean_ms}
    line = {
        "metric": res.get("metric", METRIC), "value": res["value"], "unit": res.get("unit", UNIT), "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": res["ms"] / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": res["dtype"], "data": "synthetic", "config": info, "roofline": roofline,
        "e2e": res["e2e"], "gpu_launches": int(res["launches"]), "clocks": res["clocks"],
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline and res["cpu"] is not None:
        A, b, oracle_iters = res["cpu"]
        cpu = CpuReference(A, b)
        if cpu.ref is not None:
            k = min(cpu.auto_iters(15.0), oracle_iters)
            t = cpu.seconds_per_iteration(k)
            line["cpu_baseline"] = {"value": 1.0 / (t * oracle_iters), "unit": UNIT, "cores": cpu.threads,
                                    "kind": "reference",
                                    "sample": f"{k} CG iterations (reference blockspmv_cpu, serial, + OpenMP vector "
                                              f"loops on {cpu.threads} threads), scaled by {oracle_iters} "
                                              f"FP64 iterations to 1e-10; reference Tile_create {cpu.setup_s:.1f} s "
                                              f"not timed"}
    if rank == 0 and world == 1 and not args.no_cpu_baseline and res.get("cpu_batch"):
        sys.path.insert(0, str(ROOT / "tests"))
        import oracle_lib as ol  # CPU-baseline leg only

        if ol.reference() is not None:
            cpu = CpuBatchReference(budget_s=8.0)
            try:
                t = cpu.measure()
            finally:
                cpu.close()
            line["cpu_baseline"] = {"value": len(cpu.systems) / t, "unit": UNIT, "cores": cpu.cores,
                                    "kind": "reference", "sample": cpu.describe()}
    if rank == 0:
        print(json.dumps(line))
    if world > 1:
        dist.destroy_process_group()
    return 0


def main():
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["mf", "reference"], default="mf")
    ap.add_argument("--workload", default="batched",
                    choices=["batched", "poisson3d", "lap2d", "convdiff", "aniso", "multirhs", "spmv", "spmm_f16"])
    ap.add_argument("--rhs", type=int, default=16, help="multirhs workload: right-hand sides (1-16)")
    ap.add_argument("--policy", default=None, choices=["fp64", "static", "rule", "learned", "static_fp16"],
                    help="precision policy (default: learned for batched, static otherwise)")
    ap.add_argument("--policy-file", default=None,
                    help="learned policy (mf_policy_save format; batched default: "
                         "mille-feuille_b200/policies/randspd_batched.mfpol)")
    ap.add_argument("--no-fp64-baseline", action="store_true")
    ap.add_argument("--systems", type=int, default=512, help="batched workload: number of systems (seeds 100..)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--profile", action="store_true",
                    help="device solves only (no e2e, clocks or CPU baseline): the command profiled with ncu")
    ap.add_argument("--iters", type=int, default=0,
                    help="run a fixed number of CG iterations per solve instead of stopping at 1e-10 (profiling)")
    args = ap.parse_args()
    if args.policy is None:
        args.policy = "learned" if args.workload == "batched" else "static"
    if args.impl == "reference":
        return run_reference(args)
    return run_mf(args)


if __name__ == "__main__":
    sys.exit(main())
