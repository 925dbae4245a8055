"""Deterministic test matrices shared by the CPU and GPU parity tests.

Edge cases follow what the tiled format has to get right: empty rows and
empty tile-rows, unsorted and duplicate column indices, a row count that is
not a multiple of 16, more columns than rows, a full 16x16 tile (256 entries:
the u8 entry count wraps to 0), a tile-row large enough for the global-memory
sort path, and the seeded synthetic configurations at small sizes.
"""
from __future__ import annotations

import numpy as np

from oracle_lib import Csr


def _from_rows(n_rows, n_cols, rows):
    rp = [0]
    ci, v = [], []
    for r in rows:
        for c, x in r:
            ci.append(c)
            v.append(x)
        rp.append(len(ci))
    return Csr(n_rows, n_cols, np.array(rp, np.int32), np.array(ci, np.int32), np.array(v, np.float64))


def edge_empty_rows():
    rng = np.random.default_rng(11)
    rows = []
    for i in range(64):
        if i % 5 == 0 or 16 <= i < 32:  # scattered empty rows and a fully empty tile-row
            rows.append([])
            continue
        cols = sorted(set(rng.integers(0, 64, size=4).tolist() + [i]))
        rows.append([(c, float(rng.normal())) for c in cols])
    return _from_rows(64, 64, rows)


def edge_unsorted_duplicates():
    rng = np.random.default_rng(12)
    rows = []
    for i in range(48):
        cols = rng.integers(0, 48, size=9).tolist()  # unsorted, may repeat
        cols += [cols[0]]  # a guaranteed duplicate
        rows.append([(int(c), float(rng.normal())) for c in cols])
    return _from_rows(48, 48, rows)


def edge_ragged_rect():
    """37 rows (not a multiple of 16), 50 columns."""
    rng = np.random.default_rng(13)
    rows = []
    for i in range(37):
        k = int(rng.integers(0, 8))
        cols = rng.choice(50, size=k, replace=False).tolist()
        rows.append([(int(c), float(rng.uniform(-2, 2))) for c in cols])
    return _from_rows(37, 50, rows)


def edge_full_tile():
    """A dense 16x16 diagonal block (256 entries in one tile) plus a band."""
    rows = []
    for i in range(32):
        if i < 16:
            r = [(c, 1.0 + i + c / 16.0) for c in range(16)] + [(16 + i, -0.5)]
        else:
            r = [(i - 16, -0.5), (i, 4.0)] + ([(i + 1, -1.0)] if i + 1 < 32 else [])
        rows.append(r)
    return _from_rows(32, 32, rows)


def edge_big_tilerow():
    """One tile-row with 16 x 400 entries (above the shared-memory sort cap)."""
    rng = np.random.default_rng(14)
    n = 64 * 16
    rows = []
    for i in range(32):
        if i < 16:
            cols = rng.choice(n, size=400, replace=False).tolist()
        else:
            cols = sorted(set([i, (i * 7) % n, (i * 13 + 5) % n]))
        rows.append([(int(c), float(rng.normal())) for c in cols])
    return _from_rows(32, n, rows)


def edge_single():
    return _from_rows(16, 16, [[(0, 2.0)]] + [[] for _ in range(15)])


def edge_integer_valued():
    """Integer-valued tiles (the int8 class) next to large values (fp64 class)."""
    rows = []
    for i in range(32):
        r = [(i, 4.0)]
        if i > 0:
            r.insert(0, (i - 1, -1.0))
        if i + 1 < 32:
            r.append((i + 1, -1.0))
        if i >= 16:
            r.append(((i + 8) % 16, 1e300 if i == 20 else 3e-39 if i == 21 else 0.5))
        rows.append(sorted(r))
    return _from_rows(32, 32, rows)


def synth_matrices(mf):
    """Seeded synthetic configurations at small sizes (as oracle Csr)."""
    out = {}
    for name, A in (
        ("lap2d_32", mf.synth_laplace2d(32, 32)),
        ("poisson3d_12", mf.synth_poisson3d_scaled(12, 1)),
        ("convdiff_10", mf.synth_convdiff3d(10)),
        ("randspd_1500", mf.synth_random_spd(105, 1500)),
        ("aniso_12", mf.synth_aniso3d(12, 3)),
    ):
        out[name] = Csr(A.n_rows, A.n_cols, A.rowptr, A.colidx, A.val)
    return out


EDGE_CASES = {
    "empty_rows": edge_empty_rows,
    "unsorted_duplicates": edge_unsorted_duplicates,
    "ragged_rect": edge_ragged_rect,
    "full_tile": edge_full_tile,
    "big_tilerow": edge_big_tilerow,
    "single": edge_single,
    "integer_valued": edge_integer_valued,
}


def all_matrices(mf):
    out = {k: f() for k, f in EDGE_CASES.items()}
    out.update(synth_matrices(mf))
    return out
