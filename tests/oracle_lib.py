"""ctypes bindings for the CPU oracle (oracle/liboracle.so) and for the
reference's own CPU code compiled from the reference sources
(oracle/_ref/libmfref.so).

Test infrastructure: imported by tests/, by ``__graft_entry__.smoke()`` and by
the CPU-baseline leg of ``bench.py`` only, and only as the checker.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent.parent
ORACLE_SO = ROOT / "oracle" / "liboracle.so"
REF_SO = ROOT / "oracle" / "_ref" / "libmfref.so"


def reference_root():
    """The reference checkout: $MF_REFERENCE_ROOT, else a `reference`
    directory beside this repository; None when neither exists (tests that
    read its files then skip)."""
    env = os.environ.get("MF_REFERENCE_ROOT")
    cand = Path(env) if env else ROOT.parent / "reference"
    return cand if cand.is_dir() else None

_i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
_u32p = np.ctypeslib.ndpointer(np.uint32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
_f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
_u8p = np.ctypeslib.ndpointer(np.uint8, flags="C_CONTIGUOUS")
_u16p = np.ctypeslib.ndpointer(np.uint16, flags="C_CONTIGUOUS")
_i8p = np.ctypeslib.ndpointer(np.int8, flags="C_CONTIGUOUS")


class _OrcTiles(C.Structure):
    _fields_ = [(n, C.c_int) for n in ("tilem", "tilen", "tilenum", "csrsize", "csrptrlen")] + [
        ("tile_ptr", C.POINTER(C.c_int)),
        ("tile_columnidx", C.POINTER(C.c_int)),
        ("tile_nnz", C.POINTER(C.c_int)),
        ("blknnz", C.POINTER(C.c_int)),
        ("blknnznnz", C.POINTER(C.c_ubyte)),
        ("csr_offset", C.POINTER(C.c_int)),
        ("csrptr_offset", C.POINTER(C.c_int)),
        ("Blockcsr_Val", C.POINTER(C.c_double)),
        ("Blockcsr_Val_Low", C.POINTER(C.c_float)),
        ("Tile_csr_Col", C.POINTER(C.c_ubyte)),
        ("Blockcsr_Ptr", C.POINTER(C.c_ubyte)),
    ]


# array name -> (struct field, length key)
TILE_ARRAYS = {
    "tile_ptr": ("tile_ptr", "tilem+1"),
    "tile_columnidx": ("tile_columnidx", "tilenum"),
    "tile_nnz": ("tile_nnz", "tilenum+1"),
    "blknnz": ("blknnz", "tilenum+1"),
    "blknnznnz": ("blknnznnz", "tilenum+1"),
    "csr_offset": ("csr_offset", "tilenum+1"),
    "csrptr_offset": ("csrptr_offset", "tilenum+1"),
    "Blockcsr_Val": ("Blockcsr_Val", "csrsize"),
    "Blockcsr_Val_Low": ("Blockcsr_Val_Low", "csrsize"),
    "Tile_csr_Col": ("Tile_csr_Col", "csrsize"),
    "Blockcsr_Ptr": ("Blockcsr_Ptr", "csrptrlen"),
}


def _len(sizes: dict, key: str) -> int:
    if key.endswith("+1"):
        return sizes[key[:-2]] + 1
    return sizes[key]


_orc = None
_ref = None


def oracle() -> C.CDLL:
    global _orc
    if _orc is None:
        if not ORACLE_SO.exists():
            raise RuntimeError(f"{ORACLE_SO} not built (run make -C oracle)")
        lib = C.CDLL(str(ORACLE_SO))
        lib.orc_tile_create.argtypes = [C.c_int, C.c_int, _i32p, _i32p, _f64p, C.c_void_p, C.POINTER(_OrcTiles)]
        lib.orc_tile_create.restype = C.c_int
        lib.orc_tiles_free.argtypes = [C.POINTER(_OrcTiles)]
        lib.orc_encode.argtypes = [_u8p, _u8p, C.c_int, C.c_int]
        lib.orc_decode.argtypes = [_u8p, _u8p, C.c_int]
        lib.orc_rowblkblock_count.argtypes = [C.POINTER(_OrcTiles)]
        lib.orc_blockspmv.argtypes = [C.POINTER(_OrcTiles), C.c_int, C.c_int, _u8p, _i32p, _i32p,
                                      _u32p, _i32p, _i32p, _f64p, _f64p]
        lib.orc_tiled_spmv.argtypes = [C.POINTER(_OrcTiles), C.c_int, _f64p, _f64p]
        lib.orc_nonzero_rows_count.argtypes = [C.POINTER(_OrcTiles), C.c_int]
        lib.orc_nonzero_rows.argtypes = [C.POINTER(_OrcTiles), C.c_int, _i32p, _i32p, _u8p, _u8p, _i32p]
        lib.orc_balance.argtypes = [C.POINTER(_OrcTiles), C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int),
                                    _i32p, _i32p, _i32p, C.POINTER(C.c_int), C.POINTER(C.c_int)]
        lib.orc_f32_to_f16_bits.argtypes = [C.c_float]
        lib.orc_f32_to_f16_bits.restype = C.c_uint16
        lib.orc_payload_casts.argtypes = [_f64p, C.c_int, _f32p, _u16p, _i8p]
        lib.orc_rule_class.argtypes = [C.c_double]
        lib.orc_rule_tiles.argtypes = [C.c_int, C.c_int, C.c_int, _i32p, _u8p, C.c_void_p, _f32p, _f32p, C.c_int, _u8p,
                                       _u8p]
        lib.orc_rule_tiles.restype = None
        lib.orc_f64_to_f16_bits.argtypes = [C.c_double]
        lib.orc_f64_to_f16_bits.restype = C.c_uint16
        lib.orc_batch_rows.argtypes = [C.c_int, _i32p, _i32p, _f64p, _u16p, _f32p, _f32p, _u8p, _f32p]
        lib.orc_batch_rows.restype = None
        lib.orc_pn_forward.argtypes = [_f32p, _f32p, _f32p]
        lib.orc_pn_forward.restype = None
        lib.orc_batch_classify.argtypes = [C.c_int, _i32p, _i32p, _f64p, C.c_int, _i32p, _i32p, _f64p, _f64p,
                                           _f64p, _f64p, C.c_double, C.c_int, C.c_int, _f32p, _f32p, _f32p, _u8p,
                                           _f64p]
        lib.orc_batch_classify.restype = None
        lib.orc_random_spd_size.argtypes = [C.c_uint64]
        lib.orc_random_spd_size.restype = C.c_int
        lib.orc_random_spd.argtypes = [C.c_uint64, C.c_int, C.POINTER(C.c_int), C.POINTER(C.POINTER(C.c_int)),
                                       C.POINTER(C.POINTER(C.c_int)), C.POINTER(C.POINTER(C.c_double))]
        lib.orc_random_spd.restype = C.c_int
        lib.orc_xstar.argtypes = [C.c_uint64, C.c_int, _f64p]
        lib.orc_xstar.restype = None
        lib.orc_free.argtypes = [C.c_void_p]
        lib.orc_free.restype = None
        lib.orc_csr_spmv.argtypes = [C.c_int, _i32p, _i32p, _f64p, _f64p, _f64p]
        lib.orc_cg.argtypes = [C.c_int, _i32p, _i32p, _f64p, _f64p, _f64p, C.c_int, C.c_double,
                               C.POINTER(C.c_double), C.c_void_p]
        lib.orc_cg.restype = C.c_int
        lib.orc_bicgstab.argtypes = [C.c_int, _i32p, _i32p, _f64p, _f64p, _f64p, C.c_int, C.c_double,
                                     C.POINTER(C.c_double)]
        lib.orc_bicgstab.restype = C.c_int
        lib.orc_true_relres.argtypes = [C.c_int, _i32p, _i32p, _f64p, _f64p, _f64p]
        lib.orc_true_relres.restype = C.c_double
        lib.orc_mlp_grad.argtypes = [_f32p, _f32p, np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS"), C.c_int,
                                     _f64p]
        lib.orc_mlp_grad.restype = C.c_double
        _orc = lib
    return _orc


def reference():
    """The reference's own CPU code, or None where it was not compiled."""
    global _ref
    if _ref is None:
        if not REF_SO.exists():
            return None
        lib = C.CDLL(str(REF_SO))

        class Sizes(C.Structure):
            _fields_ = [(n, C.c_int) for n in ("tilem", "tilen", "tilenum", "csrsize", "csrptrlen")]

        lib.Sizes = Sizes
        lib.ref_tile_create.argtypes = [C.c_int, C.c_int, C.c_int, _i32p, _i32p, _f64p, _f32p, C.POINTER(Sizes)]
        lib.ref_tile_fetch.argtypes = [_i32p, _i32p, _i32p, _i32p, _u8p, _i32p, _i32p, _f64p, _f32p, _u8p, _u8p, _u8p]
        lib.ref_encode.argtypes = [_u8p, _u8p, C.c_int, C.c_int]
        lib.ref_encode_last.argtypes = []
        lib.ref_blockspmv.argtypes = [C.c_int, C.c_int, C.c_int, _f64p, _f64p, _i32p, _i32p, C.c_void_p,
                                      C.c_void_p, C.c_void_p]
        lib.ref_blockspmv.restype = C.c_int
        lib.ref_read_mtx.argtypes = [C.c_char_p, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int)]
        lib.ref_read_mtx_fetch.argtypes = [_i32p, _i32p, _f64p]
        _ref = lib
    return _ref


class Csr:
    """A CSR matrix held in numpy arrays (int32 indices, float64 values)."""

    def __init__(self, n_rows, n_cols, rowptr, colidx, val):
        self.n_rows = int(n_rows)
        self.n_cols = int(n_cols)
        self.rowptr = np.ascontiguousarray(rowptr, dtype=np.int32)
        self.colidx = np.ascontiguousarray(colidx, dtype=np.int32)
        self.val = np.ascontiguousarray(val, dtype=np.float64)

    @property
    def nnz(self):
        return int(self.rowptr[-1])

    def truncated(self, rows):
        """First `rows` rows (the reference truncates n to a multiple of 16)."""
        rp = self.rowptr[: rows + 1].copy()
        return Csr(rows, self.n_cols, rp, self.colidx[: rp[-1]].copy(), self.val[: rp[-1]].copy())

    def to_scipy(self):
        import scipy.sparse as sp

        return sp.csr_matrix((self.val, self.colidx, self.rowptr), shape=(self.n_rows, self.n_cols))


def oracle_tiles(csr: Csr, val_low=None):
    """Runs the oracle Tile_create; returns (sizes dict, arrays dict)."""
    lib = oracle()
    t = _OrcTiles()
    vl = None if val_low is None else np.ascontiguousarray(val_low, np.float32)
    rc = lib.orc_tile_create(csr.n_rows, csr.n_cols, csr.rowptr, csr.colidx, csr.val,
                             None if vl is None else vl.ctypes.data, C.byref(t))
    if rc != 0:
        lib.orc_tiles_free(C.byref(t))
        raise ValueError("oracle tile_create rejected the input")
    sizes = {k: getattr(t, k) for k in ("tilem", "tilen", "tilenum", "csrsize", "csrptrlen")}
    arrays = {}
    for name, (field, key) in TILE_ARRAYS.items():
        n = _len(sizes, key)
        ptr = getattr(t, field)
        arrays[name] = np.ctypeslib.as_array(ptr, shape=(max(n, 1),))[:n].copy() if n > 0 else \
            np.zeros(0, dtype=np.ctypeslib.as_array(ptr, shape=(1,)).dtype)
    return sizes, arrays, t


def free_oracle_tiles(t):
    oracle().orc_tiles_free(C.byref(t))


def reference_tiles(csr: Csr, val_low=None):
    """Runs the reference Tile_create (compiled from its sources)."""
    lib = reference()
    if lib is None:
        return None
    vl = (csr.val.astype(np.float32) if val_low is None else np.ascontiguousarray(val_low, np.float32))
    sz = lib.Sizes()
    lib.ref_tile_create(csr.n_rows, csr.n_cols, csr.nnz, csr.rowptr, csr.colidx, csr.val, vl, C.byref(sz))
    sizes = {k: getattr(sz, k) for k in ("tilem", "tilen", "tilenum", "csrsize", "csrptrlen")}
    T = sizes["tilenum"]
    a = {
        "tile_ptr": np.zeros(sizes["tilem"] + 1, np.int32),
        "tile_columnidx": np.zeros(max(T, 1), np.int32),
        "tile_nnz": np.zeros(T + 1, np.int32),
        "blknnz": np.zeros(T + 1, np.int32),
        "blknnznnz": np.zeros(T + 1, np.uint8),
        "csr_offset": np.zeros(T + 1, np.int32),
        "csrptr_offset": np.zeros(T + 1, np.int32),
        "Blockcsr_Val": np.zeros(max(sizes["csrsize"], 1), np.float64),
        "Blockcsr_Val_Low": np.zeros(max(sizes["csrsize"], 1), np.float32),
        "Tile_csr_Col": np.zeros(max(sizes["csrsize"], 1), np.uint8),
        "Blockcsr_Ptr": np.zeros(max(sizes["csrptrlen"], 1), np.uint8),
        "csr_compressedIdx": np.zeros(max((sizes["csrsize"] + 1) // 2, 1), np.uint8),
    }
    lib.ref_tile_fetch(a["tile_ptr"], a["tile_columnidx"], a["tile_nnz"], a["blknnz"], a["blknnznnz"],
                       a["csr_offset"], a["csrptr_offset"], a["Blockcsr_Val"], a["Blockcsr_Val_Low"],
                       a["Tile_csr_Col"], a["Blockcsr_Ptr"], a["csr_compressedIdx"])
    a["tile_columnidx"] = a["tile_columnidx"][:T]
    for k in ("Blockcsr_Val", "Blockcsr_Val_Low", "Tile_csr_Col"):
        a[k] = a[k][: sizes["csrsize"]]
    a["Blockcsr_Ptr"] = a["Blockcsr_Ptr"][: sizes["csrptrlen"]]
    a["csr_compressedIdx"] = a["csr_compressedIdx"][: (sizes["csrsize"] + 1) // 2]
    return sizes, a


def reference_read_mtx(path) -> Csr:
    lib = reference()
    m, n, nnz = C.c_int(), C.c_int(), C.c_int()
    lib.ref_read_mtx(str(path).encode(), C.byref(m), C.byref(n), C.byref(nnz))
    rp = np.zeros(m.value + 1, np.int32)
    ci = np.zeros(nnz.value, np.int32)
    v = np.zeros(nnz.value, np.float64)
    lib.ref_read_mtx_fetch(rp, ci, v)
    return Csr(m.value, n.value, rp, ci, v)


def oracle_cg(csr: Csr, b, maxiter, tol, want_hist=False):
    lib = oracle()
    x = np.zeros(csr.n_rows, np.float64)
    rr = C.c_double()
    hist = np.zeros(maxiter + 1, np.float64) if want_hist else None
    it = lib.orc_cg(csr.n_rows, csr.rowptr, csr.colidx, csr.val, np.ascontiguousarray(b, np.float64), x,
                    maxiter, tol, C.byref(rr), None if hist is None else hist.ctypes.data)
    if want_hist:
        return it, x, rr.value, hist[: it + 1]
    return it, x, rr.value


def oracle_bicgstab(csr: Csr, b, maxiter, tol):
    lib = oracle()
    x = np.zeros(csr.n_rows, np.float64)
    rr = C.c_double()
    it = lib.orc_bicgstab(csr.n_rows, csr.rowptr, csr.colidx, csr.val, np.ascontiguousarray(b, np.float64), x,
                          maxiter, tol, C.byref(rr))
    return it, x, rr.value


def oracle_true_relres(csr: Csr, b, x) -> float:
    return oracle().orc_true_relres(csr.n_rows, csr.rowptr, csr.colidx, csr.val,
                                    np.ascontiguousarray(b, np.float64), np.ascontiguousarray(x, np.float64))


def oracle_rule_tiles(n, tilen, tile_col, static_cls, pn, po, scaled=False, f16ok=None):
    """Per-tile rule decision and working class (the restatement of the
    reference's partial-convergence rule, src/main-cg-mixed.cu:415-460);
    f16ok (u8 per tile, None: all finite) marks tiles whose FP16 payload is
    finite."""
    T = len(tile_col)
    dec = np.zeros(max(T, 1), np.uint8)
    work = np.zeros(max(T, 1), np.uint8)
    ok = None if f16ok is None else np.ascontiguousarray(f16ok, np.uint8)
    oracle().orc_rule_tiles(n, tilen, T, np.ascontiguousarray(tile_col, np.int32),
                            np.ascontiguousarray(static_cls, np.uint8), None if ok is None else ok.ctypes.data,
                            np.ascontiguousarray(pn, np.float32),
                            np.ascontiguousarray(po, np.float32), 1 if scaled else 0, dec, work)
    return dec[:T], work[:T]


def oracle_batch_rows(csr: Csr):
    """The batched solver's per-row storage of one system: FP16 bits of the
    row-scaled off-diagonals, row scales, FP32 diagonal, flags, row stats."""
    n = csr.n_rows
    nz = int(csr.rowptr[-1])
    v16 = np.zeros(max(nz, 1), np.uint16)
    rs = np.zeros(n, np.float32)
    d32 = np.zeros(n, np.float32)
    fl = np.zeros(n, np.uint8)
    st = np.zeros(4 * n, np.float32)
    oracle().orc_batch_rows(n, csr.rowptr, csr.colidx, csr.val, v16, rs, d32, fl, st)
    return v16[:nz], rs, d32, fl, st.reshape(n, 4)


def oracle_batch_classify(csr: Csr, crow, cent, r, pn, po, q, relres, refs, have_prev, prev, w):
    """The batched chunk policy on one system (see orc_batch_classify);
    returns (features [nch, 16], classes, decision margins); prev (float32,
    4 per chunk) is read when have_prev and overwritten."""
    nch = len(crow) - 1
    feat = np.zeros((max(nch, 1), 16), np.float32)
    cls = np.zeros(max(nch, 1), np.uint8)
    mar = np.zeros(max(nch, 1), np.float64)
    oracle().orc_batch_classify(csr.n_rows, csr.rowptr, csr.colidx, csr.val, nch,
                                np.ascontiguousarray(crow, np.int32), np.ascontiguousarray(cent, np.int32),
                                *(np.ascontiguousarray(v, np.float64) for v in (r, pn, po, q)), float(relres),
                                int(refs), int(have_prev), prev, np.ascontiguousarray(w, np.float32), feat, cls, mar)
    return feat[:nch], cls[:nch], mar[:nch]


def oracle_random_spd(seed, n=0) -> Csr:
    """The batched configuration's random SPD system of `seed` (the C
    restatement of the library's generator)."""
    lib = oracle()
    nnz = C.c_int()
    rp, ci, v = C.POINTER(C.c_int)(), C.POINTER(C.c_int)(), C.POINTER(C.c_double)()
    n = lib.orc_random_spd(seed, n, C.byref(nnz), C.byref(rp), C.byref(ci), C.byref(v))
    out = Csr(n, n, np.ctypeslib.as_array(rp, shape=(n + 1,)).copy(),
              np.ctypeslib.as_array(ci, shape=(max(nnz.value, 1),))[: nnz.value].copy(),
              np.ctypeslib.as_array(v, shape=(max(nnz.value, 1),))[: nnz.value].copy())
    for p in (rp, ci, v):
        lib.orc_free(C.cast(p, C.c_void_p))
    return out


def oracle_xstar(seed, n):
    out = np.zeros(n, np.float64)
    oracle().orc_xstar(seed, n, out)
    return out
