"""Helpers for the drop-in entry points: a ctypes Tile_matrix built from the
field list in include/Mille-feuille-tile.h, loaders for the solver entry
libraries and a Matrix Market writer."""
from __future__ import annotations

import ctypes as C
import re
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent.parent
LIB = ROOT / "mille-feuille_b200" / "lib"
BIN = ROOT / "mille-feuille_b200" / "bin"
TILE_H = ROOT / "include" / "Mille-feuille-tile.h"


def tile_fields():
    """(name, is_pointer) of Tile_matrix's fields in declaration order."""
    text = TILE_H.read_text()
    body = text[text.index("typedef struct {"): text.index("} Tile_matrix;")]
    body = re.sub(r"/\*.*?\*/", "", body, flags=re.S)
    out = []
    for m in re.finditer(r"^\s*([A-Za-z_][\w ]*?)\s*(\*?)\s*([A-Za-z_]\w*);", body, re.M):
        out.append((m.group(3), m.group(2) == "*"))
    return out


class TileMatrix(C.Structure):
    _fields_ = [(n, C.c_void_p if p else C.c_int) for n, p in tile_fields()]

    def array(self, name, dtype, count):
        p = getattr(self, name)
        if count == 0:
            return np.zeros(0, dtype)
        buf = (C.c_char * (count * np.dtype(dtype).itemsize)).from_address(p)
        return np.frombuffer(buf, dtype=dtype, count=count).copy()


ARRAYS = {  # field -> (dtype, length key)
    "tile_ptr": (np.int32, "tilem+1"),
    "tile_columnidx": (np.int32, "tilenum"),
    "tile_nnz": (np.int32, "tilenum+1"),
    "blknnz": (np.int32, "tilenum+1"),
    "blknnznnz": (np.uint8, "tilenum+1"),
    "csr_offset": (np.int32, "tilenum+1"),
    "csrptr_offset": (np.int32, "tilenum+1"),
    "Blockcsr_Val": (np.float64, "csrsize"),
    "Blockcsr_Val_Low": (np.float32, "csrsize"),
    "Tile_csr_Col": (np.uint8, "csrsize"),
    "Blockcsr_Ptr": (np.uint8, "csrptrlen"),
}


def length(tm: TileMatrix, key: str) -> int:
    if key.endswith("+1"):
        return getattr(tm, key[:-2]) + 1
    return getattr(tm, key)


_solvers = {}


def solvers(mixed: bool) -> C.CDLL:
    name = "libmf_solvers_mixed.so" if mixed else "libmf_solvers.so"
    if name not in _solvers:
        L = C.CDLL(str(LIB / name))
        vp = C.c_void_p
        for f in ("cg_solve_inc", "cg_solve_sync", "cg_solve_reduce"):
            fn = getattr(L, f)
            fn.argtypes = [vp, vp, vp, vp, vp, vp, C.c_int, vp, C.c_int, C.c_double, C.c_char_p, C.c_int, C.c_int]
            fn.restype = None
        for f in ("bicgstab", "bicgstab_sync", "bicgstab_inc"):
            fn = getattr(L, f)
            fn.argtypes = [vp, vp, vp, vp, vp, C.c_int, C.c_char_p, C.c_int]
            fn.restype = C.c_int
        _solvers[name] = L
    return _solvers[name]


def write_mtx(path, csr, symmetric=False):
    """Writes a general (or lower-triangle symmetric) coordinate file."""
    lines = []
    for i in range(csr.n_rows):
        for j in range(csr.rowptr[i], csr.rowptr[i + 1]):
            c = int(csr.colidx[j])
            if symmetric and c > i:
                continue
            lines.append(f"{i + 1} {c + 1} {float(csr.val[j])!r}")
    kind = "symmetric" if symmetric else "general"
    Path(path).write_text(f"%%MatrixMarket matrix coordinate real {kind}\n"
                          f"{csr.n_rows} {csr.n_cols} {len(lines)}\n" + "\n".join(lines) + "\n")
