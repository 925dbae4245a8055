"""Generates tests/golden/config_iterations.json: the FP64 CPU oracle's CG
iteration counts (and accuracy) on the single-system configurations.

    python tests/golden/make_config_iterations.py

Config 1: 2D 5-point Laplacian 128^2, x* seed 0; config 2: 3D 7-point
Poisson 128^3 with per-row scaled off-diagonals, seed 1; both b = A x*,
x0 = 0, stop at ||r|| <= 1e-10 ||b||.  bench.py scales its CPU-baseline
samples by these counts; tests/test_config_iterations.py recomputes them.
"""
import json
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "tests"))

CONFIGS = {
    "laplace2d_128": ("laplace2d", (128, 128), 0),
    "poisson3d_scaled_128": ("poisson3d", (128, 1), 1),
}


def compute(name):
    import __graft_entry__ as ge
    import oracle_lib as ol

    mf = ge.load_package()
    kind, args, seed = CONFIGS[name]
    A = mf.synth_laplace2d(*args) if kind == "laplace2d" else mf.synth_poisson3d_scaled(*args)
    xs = mf.synth_xstar(seed, A.n_rows)
    b = A.matvec(xs)
    it, x, rr = ol.oracle_cg(ol.Csr(A.n_rows, A.n_cols, A.rowptr, A.colidx, A.val), b, 50000, 1e-10)
    return {"iterations": int(it), "relres": rr, "max_abs_err_vs_xstar": float(np.max(np.abs(x - xs))),
            "n": A.n_rows, "nnz": A.nnz}


def main():
    out = {name: compute(name) for name in CONFIGS}
    (Path(__file__).resolve().parent / "config_iterations.json").write_text(json.dumps(out, indent=1) + "\n")


if __name__ == "__main__":
    main()
