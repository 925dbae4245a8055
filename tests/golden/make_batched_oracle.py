"""Generates tests/golden/batched_oracle.json: the FP64 CPU oracle's CG on
every system of the batched configuration (512 random SPD systems, seeds
100-611, n ~ log-uniform[1k, 64k], b = A x*, x* ~ U[-1, 1] from the system's
seed, x0 = 0, stop at ||r|| <= 1e-10 ||b||).

Per system it records n, nnz, the oracle's iteration count, its recurrence
and true relative residuals and max |x - x*|.  The GPU batched-solver test
compares per-system iterations and accuracy with these figures, and the
reference arm of bench.py scales its timed iteration samples by the
iteration counts (a full 512-system CPU solve takes tens of minutes).

    python tests/golden/make_batched_oracle.py [--workers N]
"""
import argparse
import json
import multiprocessing as mp
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "tests"))

SEEDS = range(100, 612)
TOL = 1e-10
MAXITER = 50000


def solve(seed):
    import __graft_entry__ as ge
    import oracle_lib as ol

    mf = ge.load_package()
    A = mf.synth_random_spd(seed)
    xs = mf.synth_xstar(seed, A.n_rows)
    b = A.matvec(xs)
    csr = ol.Csr(A.n_rows, A.n_cols, A.rowptr, A.colidx, A.val)
    t0 = time.perf_counter()
    it, x, rr = ol.oracle_cg(csr, b, MAXITER, TOL)
    return {"seed": seed, "n": A.n_rows, "nnz": A.nnz, "iterations": int(it), "relres": rr,
            "relres_true": ol.oracle_true_relres(csr, b, x), "max_abs_err_vs_xstar": float(np.max(np.abs(x - xs))),
            "cpu_s": time.perf_counter() - t0}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--workers", type=int, default=8)
    args = ap.parse_args()
    ctx = mp.get_context("spawn")
    with ctx.Pool(args.workers) as pool:
        # largest systems first so the pool's tail is short
        import __graft_entry__ as ge

        mf = ge.load_package()
        order = sorted(SEEDS, key=lambda s: -mf.lib().mf_synth_random_spd_size(s))
        rows = {r["seed"]: r for r in pool.imap_unordered(solve, order)}
    out = {"what": "FP64 CPU oracle CG (oracle/mf_oracle.c orc_cg) on the batched configuration",
           "tol": TOL, "systems": [rows[s] for s in SEEDS]}
    (Path(__file__).resolve().parent / "batched_oracle.json").write_text(json.dumps(out, indent=0) + "\n")


if __name__ == "__main__":
    main()
