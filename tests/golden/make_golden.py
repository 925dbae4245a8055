"""Generates tests/golden/tiles.json from the reference's own CPU code.

Runs the reference Tile_create (src/csr2block.h:267) and blockspmv_cpu
(src/blockspmv_cpu.h:2, after filling csr_compressedIdx with the
reference's encode, src/encode.h:29) -- compiled from the reference sources
into oracle/_ref/libmfref.so by oracle/Makefile -- on every test matrix of
tests/matrices.py, and records SHA-256 digests of each output array.  The
committed JSON pins the oracle and the GPU path where the reference build is
absent.

    python tests/golden/make_golden.py
"""
import hashlib
import json
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "tests"))

import __graft_entry__ as ge  # noqa: E402
import matrices  # noqa: E402
import oracle_lib as ol  # noqa: E402


def digest(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def spmv_input(n):
    # deterministic x with distinct values per column
    i = np.arange(n, dtype=np.float64)
    return np.sin(0.37 * i + 0.1) + 0.01 * i


def main():
    mf = ge.load_package()
    ref = ol.reference()
    assert ref is not None, "oracle/_ref/libmfref.so missing: run make -C oracle with the reference sources present"
    out = {}
    for name, A in matrices.all_matrices(mf).items():
        sizes, arrs = ol.reference_tiles(A)
        entry = {"sizes": sizes, "csr_digest": digest(np.concatenate([A.rowptr.view(np.uint8), A.colidx.view(np.uint8),
                                                                       A.val.view(np.uint8)]))}
        entry["arrays"] = {k: digest(v) for k, v in arrs.items()}
        # blockspmv_cpu with the encoded column index
        ref.ref_encode_last()
        T = sizes["tilenum"]
        x = spmv_input(sizes["tilen"] * 16)
        y = np.zeros(sizes["tilem"] * 16, np.float64)
        p1 = np.zeros(max(T, 1), np.int32)
        p2 = np.zeros(max(T, 1), np.int32)
        ref.ref_blockspmv(A.n_rows, A.n_cols, A.nnz, x, y, p1, p2, None, None, None)
        entry["blockspmv_y"] = digest(y[: A.n_rows])
        entry["ptroffset1"] = digest(p1[:T])
        entry["ptroffset2"] = digest(p2[:T])
        out[name] = entry
        print(name, sizes)
    (ROOT / "tests" / "golden" / "tiles.json").write_text(json.dumps(out, indent=1, sort_keys=True) + "\n")


if __name__ == "__main__":
    main()
