"""Python bindings (ctypes) for libmf, the B200 (sm_100a) Mille-feuille
tiled sparse solver library.  The product is the C ABI in include/mf.h; this
module only marshals numpy arrays to it for tests, benchmarks and scripts.

Load it with ``load_package()`` from ``__graft_entry__`` (the directory name
is not a Python identifier).
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "lib" / "libmf.so"

MF_OK = 0
STATUS_NAMES = {
    0: "MF_OK", 1: "MF_ERR_INVALID_ARG", 2: "MF_ERR_CUDA", 3: "MF_ERR_NO_MEMORY", 4: "MF_ERR_TIMEOUT",
    5: "MF_ERR_BREAKDOWN", 6: "MF_ERR_NOT_CONVERGED", 7: "MF_ERR_IO", 8: "MF_ERR_UNSUPPORTED",
    9: "MF_ERR_NO_DEVICE",
}
POLICY = {"fp64": 0, "static": 1, "rule": 2, "learned": 3, "rule_scaled": 4, "static_fp16": 5}
CLASS_NAMES = {0: "fp64", 1: "bypass", 2: "int8", 3: "fp16", 4: "fp32"}


class MfError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {msg}")
        self.status = status


class MatrixInfo(C.Structure):
    _fields_ = [(n, C.c_int) for n in ("rows", "cols", "nnz", "tilem", "tilen", "tilenum", "csrsize",
                                       "csrptrlen", "nonzero_rows", "rowblkblock")] + [
        ("class_tiles", C.c_int * 5), ("max_tile_nnz", C.c_int), ("device_bytes", C.c_size_t)]


class SolveOpts(C.Structure):
    _fields_ = [("maxiter", C.c_int), ("tol", C.c_double), ("policy", C.c_int), ("refine_delta", C.c_double),
                ("wait_budget_s", C.c_double), ("record_history", C.c_int), ("phase_times", C.c_int),
                ("precond", C.c_int)]


class BatchReport(C.Structure):
    _fields_ = [("systems", C.c_int), ("failed", C.c_int), ("iterations_total", C.c_longlong),
                ("iterations_max", C.c_int), ("refinements_total", C.c_int), ("relres_true_max", C.c_double),
                ("kernel_ms", C.c_double), ("lanes_per_row", C.c_int), ("cluster_ctas", C.c_int),
                ("status", C.c_int), ("bytes_moved", C.c_longlong), ("fp16_share", C.c_double)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class SolveReport(C.Structure):
    _fields_ = [("iterations", C.c_int), ("status", C.c_int), ("refinements", C.c_int), ("relres", C.c_double),
                ("relres_true", C.c_double), ("kernel_ms", C.c_double), ("bytes_moved", C.c_longlong),
                ("grid_ctas", C.c_int), ("phase_us", C.c_double * 9), ("layout", C.c_int),
                ("fallback_iteration", C.c_int)]

    def as_dict(self):
        d = {k: getattr(self, k) for k, _ in self._fields_}
        d["phase_us"] = list(self.phase_us)
        return d


ARRAY_DTYPES = {
    "tile_ptr": np.int32, "tile_columnidx": np.int32, "tile_nnz": np.int32, "blknnz": np.int32,
    "csr_offset": np.int32, "csrptr_offset": np.int32, "ptroffset1": np.int32, "ptroffset2": np.int32,
    "blknnznnz": np.uint8, "Blockcsr_Val": np.float64, "Blockcsr_Val_Low": np.float32, "Tile_csr_Col": np.uint8,
    "Blockcsr_Ptr": np.uint8, "csr_compressedIdx": np.uint8, "nonzero_row_new": np.int32, "tile_rowidx": np.int32,
    "block_signal": np.int32, "blockrowid_new": np.uint8, "blockcsr_ptr_new": np.uint8,
    "rowblkblock_rowidx": np.uint32, "rowblkblock_colstart": np.int32, "rowblkblock_colstop": np.int32,
    "tile_class": np.uint8, "tile_f16ok": np.uint8, "payload_f16": np.uint16, "payload_i8": np.int8,
}

_lib = None


def lib() -> C.CDLL:
    """The loaded libmf (raises if it was not built)."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise RuntimeError(f"libmf not built: {LIB_PATH} missing (run __graft_entry__.build())")
        L = C.CDLL(str(LIB_PATH))
        vp, ip, dp = C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_double)
        L.mf_last_error.restype = C.c_char_p
        L.mf_version.restype = C.c_char_p
        L.mf_kernel_launches.restype = C.c_longlong
        L.mf_matrix_create.argtypes = [C.c_int, C.c_int, vp, vp, vp, vp, C.c_int, vp, C.POINTER(vp)]
        L.mf_matrix_destroy.argtypes = [vp]
        L.mf_matrix_get_info.argtypes = [vp, C.POINTER(MatrixInfo)]
        L.mf_matrix_array_bytes.argtypes = [vp, C.c_char_p, C.POINTER(C.c_size_t)]
        L.mf_matrix_export.argtypes = [vp, C.c_char_p, vp, C.c_size_t]
        L.mf_encode_column_index.argtypes = [vp, vp]
        L.mf_spmv.argtypes = [vp, vp, vp, vp]
        L.mf_residual_norm.argtypes = [vp, vp, vp, vp, vp]
        L.mf_residual_norm_noalloc.argtypes = [vp, vp, vp, vp, vp]
        L.mf_rule_classes.argtypes = [vp, C.c_int, vp, vp, vp, vp, vp]
        L.mf_solve_opts_default.argtypes = [C.POINTER(SolveOpts)]
        L.mf_solve_opts_default.restype = None
        L.mf_cg_solve.argtypes = [vp, vp, vp, C.POINTER(SolveOpts), C.POINTER(SolveReport), vp, vp]
        L.mf_cg_solve_host.argtypes = [vp, vp, vp, C.POINTER(SolveOpts), C.POINTER(SolveReport)]
        L.mf_bicgstab_solve.argtypes = [vp, vp, vp, C.POINTER(SolveOpts), C.POINTER(SolveReport), vp, vp]
        L.mf_bicgstab_solve_host.argtypes = [vp, vp, vp, C.POINTER(SolveOpts), C.POINTER(SolveReport)]
        L.mf_spmm.argtypes = [vp, C.c_int, vp, C.c_int, vp, C.c_int, vp]
        L.mf_cg_solve_multi.argtypes = [vp, C.c_int, vp, C.c_int, vp, C.c_int, C.POINTER(SolveOpts),
                                        C.POINTER(SolveReport), vp]
        L.mf_cg_solve_multi_host.argtypes = [vp, C.c_int, vp, vp, C.POINTER(SolveOpts), C.POINTER(SolveReport)]
        L.mf_read_matrix_market.argtypes = [C.c_char_p, ip, ip, ip, C.POINTER(ip), C.POINTER(ip), C.POINTER(dp), ip]
        L.mf_matrix_create_mtx.argtypes = [C.c_char_p, vp, C.POINTER(vp), ip]
        L.mf_spmm_f16.argtypes = [vp, C.c_int, vp, C.c_int, vp, C.c_int, C.c_int, ip, vp]
        L.mf_read_matrix.argtypes = [C.c_char_p, ip, ip, ip, C.POINTER(ip), C.POINTER(ip), C.POINTER(dp), ip]
        L.mf_read_cbd.argtypes = [C.c_char_p, ip, ip, ip, C.POINTER(ip), C.POINTER(ip), C.POINTER(dp)]
        L.mf_write_cbd.argtypes = [C.c_char_p, C.c_int, C.c_int, C.c_int, vp, vp, vp]
        L.mf_free_host.argtypes = [vp]
        L.mf_free_host.restype = None
        L.mf_rng_u01.argtypes = [C.c_uint64, C.c_uint64, C.c_uint64]
        L.mf_rng_u01.restype = C.c_double
        L.mf_rng_normal.argtypes = [C.c_uint64, C.c_uint64, C.c_uint64]
        L.mf_rng_normal.restype = C.c_double
        L.mf_synth_xstar.argtypes = [C.c_uint64, C.c_int, vp]
        L.mf_synth_random_spd_size.argtypes = [C.c_uint64]
        L.mf_synth_random_spd_size.restype = C.c_int
        L.mf_batch_create.argtypes = [C.c_int, vp, vp, vp, vp, C.POINTER(vp)]
        L.mf_batch_destroy.argtypes = [vp]
        L.mf_batch_info.argtypes = [vp, C.POINTER(C.c_longlong), C.POINTER(C.c_longlong), vp]
        L.mf_batch_cg_solve.argtypes = [vp, vp, vp, C.POINTER(SolveOpts), C.c_int, C.POINTER(BatchReport), vp]
        L.mf_batch_results.argtypes = [vp, vp, vp]
        L.mf_batch_tune.argtypes = [vp, vp, vp, C.POINTER(SolveOpts), C.POINTER(C.c_int), C.POINTER(C.c_int), vp]
        L.mf_batch_set_schedule.argtypes = [vp, C.c_int, C.c_int]
        L.mf_batch_chunk_count.argtypes = [vp, ip, ip, ip]
        L.mf_batch_export.argtypes = [vp, C.c_char_p, vp, C.c_size_t]
        L.mf_batch_attach_policy.argtypes = [vp, vp]
        L.mf_batch_policy_collect.argtypes = [vp, vp, vp, C.c_int, C.c_int, C.c_longlong, C.POINTER(C.c_longlong)]
        L.mf_batch_policy_classify.argtypes = [vp, vp, vp, vp, vp, vp, vp, C.c_int, vp, vp]
        L.mf_policy_param_count.restype = C.c_int
        L.mf_policy_create.argtypes = [C.c_uint64, C.POINTER(vp)]
        L.mf_policy_destroy.argtypes = [vp]
        L.mf_policy_get_params.argtypes = [vp, vp, C.c_int]
        L.mf_policy_set_params.argtypes = [vp, vp, C.c_int]
        L.mf_policy_save.argtypes = [vp, C.c_char_p]
        L.mf_policy_load.argtypes = [C.c_char_p, C.POINTER(vp)]
        L.mf_policy_collect.argtypes = [vp, vp, vp, C.c_int, C.c_int, C.c_longlong, C.POINTER(C.c_longlong)]
        L.mf_policy_label_counts.argtypes = [vp, vp]
        L.mf_policy_train.argtypes = [vp, C.c_int, C.c_int, C.c_float, C.c_uint64, dp, dp]
        L.mf_policy_eval_grad.argtypes = [vp, vp, vp, C.c_int, vp, dp]
        L.mf_matrix_attach_policy.argtypes = [vp, vp]
        gen = [ip, ip, C.POINTER(ip), C.POINTER(ip), C.POINTER(dp)]
        L.mf_synth_laplace2d.argtypes = [C.c_int, C.c_int] + gen
        L.mf_synth_poisson3d_scaled.argtypes = [C.c_int, C.c_uint64] + gen
        L.mf_synth_convdiff3d.argtypes = [C.c_int, C.c_double, C.c_double, C.c_double, C.c_double] + gen
        L.mf_synth_random_spd.argtypes = [C.c_int, C.c_uint64] + gen
        L.mf_synth_aniso3d.argtypes = [C.c_int, C.c_uint64, C.c_double, C.c_double, C.c_double] + gen
        _lib = L
    return _lib


def check(status):
    if status != MF_OK:
        raise MfError(status, lib().mf_last_error().decode(errors="replace"))


class HostCsr:
    """CSR matrix in numpy arrays (int32 indices, float64 values)."""

    def __init__(self, n_rows, n_cols, rowptr, colidx, val):
        self.n_rows, self.n_cols = int(n_rows), int(n_cols)
        self.rowptr = np.ascontiguousarray(rowptr, np.int32)
        self.colidx = np.ascontiguousarray(colidx, np.int32)
        self.val = np.ascontiguousarray(val, np.float64)

    @property
    def nnz(self):
        return int(self.rowptr[-1])

    def truncated(self, rows):
        rp = self.rowptr[: rows + 1].copy()
        return HostCsr(rows, self.n_cols, rp, self.colidx[: rp[-1]].copy(), self.val[: rp[-1]].copy())

    def matvec(self, x):
        import scipy.sparse as sp

        A = sp.csr_matrix((self.val, self.colidx, self.rowptr), shape=(self.n_rows, self.n_cols))
        return A @ x


def _take_csr(n, nnz, rp, ci, v, n_cols=None):
    L = lib()
    out = HostCsr(n, n if n_cols is None else n_cols,
                  np.ctypeslib.as_array(rp, shape=(n + 1,)).copy(),
                  np.ctypeslib.as_array(ci, shape=(max(nnz, 1),))[:nnz].copy(),
                  np.ctypeslib.as_array(v, shape=(max(nnz, 1),))[:nnz].copy())
    for p in (rp, ci, v):
        L.mf_free_host(C.cast(p, C.c_void_p))
    return out


def _gen(fn, *args):
    n, nnz = C.c_int(), C.c_int()
    rp, ci = C.POINTER(C.c_int)(), C.POINTER(C.c_int)()
    v = C.POINTER(C.c_double)()
    check(fn(*args, C.byref(n), C.byref(nnz), C.byref(rp), C.byref(ci), C.byref(v)))
    return _take_csr(n.value, nnz.value, rp, ci, v)


def synth_laplace2d(nx, ny):
    return _gen(lib().mf_synth_laplace2d, nx, ny)


def synth_poisson3d_scaled(g, seed):
    return _gen(lib().mf_synth_poisson3d_scaled, g, seed)


def synth_convdiff3d(g, peclet=10.0, v=(1.0, 0.5, 0.25)):
    return _gen(lib().mf_synth_convdiff3d, g, peclet, v[0], v[1], v[2])


def synth_random_spd(seed, n=0):
    return _gen(lib().mf_synth_random_spd, n, seed)


def synth_aniso3d(g, seed, log_sigma=2.0, corr_len=8.0, aniso=100.0):
    return _gen(lib().mf_synth_aniso3d, g, seed, log_sigma, corr_len, aniso)


def synth_block_dense(nb, dense_per_row, sparse_per_row, seed, ragged=0):
    """A block-structured matrix (HostCsr) for the tensor-core SpMM: nb block
    rows of 16 (the last one `ragged` rows short); per block row a dense
    diagonal 16x16 block and `dense_per_row` dense blocks at random block
    columns (values N(0,1) x 10^U[-2,2] per block), plus `sparse_per_row`
    random N(0,1) entries per row; duplicates summed, columns sorted (NumPy
    PCG64 seeded with `seed`)."""
    import scipy.sparse as sp

    rng = np.random.default_rng(seed)
    n = 16 * nb - ragged
    rows, cols, vals = [], [], []
    base = np.arange(16)
    for b in range(nb):
        for bc in sorted({b} | set(rng.integers(0, nb, dense_per_row).tolist())):
            rows.append(np.repeat(base + 16 * b, 16))
            cols.append(np.tile(base + 16 * bc, 16))
            vals.append(rng.normal(size=256) * 10.0 ** rng.uniform(-2, 2))
    r = rng.integers(0, 16 * nb, 16 * nb * sparse_per_row)
    c = rng.integers(0, 16 * nb, 16 * nb * sparse_per_row)
    rows.append(r)
    cols.append(c)
    vals.append(rng.normal(size=r.size))
    rows, cols, vals = np.concatenate(rows), np.concatenate(cols), np.concatenate(vals)
    keep = (rows < n) & (cols < n)
    A = sp.coo_matrix((vals[keep], (rows[keep], cols[keep])), shape=(n, n)).tocsr()
    A.sum_duplicates()
    A.sort_indices()
    return HostCsr(n, n, A.indptr, A.indices, A.data)


def synth_xstar(seed, n):
    out = np.zeros(n, np.float64)
    check(lib().mf_synth_xstar(seed, n, out.ctypes.data))
    return out


def read_matrix_market(path):
    L = lib()
    m, n, nnz, sym = C.c_int(), C.c_int(), C.c_int(), C.c_int()
    rp, ci = C.POINTER(C.c_int)(), C.POINTER(C.c_int)()
    v = C.POINTER(C.c_double)()
    check(L.mf_read_matrix_market(str(path).encode(), C.byref(m), C.byref(n), C.byref(nnz), C.byref(rp),
                                  C.byref(ci), C.byref(v), C.byref(sym)))
    return _take_csr(m.value, nnz.value, rp, ci, v, n_cols=n.value)


def matrix_from_mtx(path, stream=None):
    """A Matrix from a Matrix Market file, the CSR built on the GPU
    (mf_matrix_create_mtx); returns (Matrix, is_symmetric)."""
    h = C.c_void_p()
    sym = C.c_int()
    check(lib().mf_matrix_create_mtx(str(path).encode(), stream, C.byref(h), C.byref(sym)))
    return Matrix(None, _handle=h), sym.value


def read_matrix(path):
    """.mtx or .cbd by extension (mf_read_matrix); returns (HostCsr, is_symmetric)."""
    L = lib()
    m, n, nnz, sym = C.c_int(), C.c_int(), C.c_int(), C.c_int()
    rp, ci = C.POINTER(C.c_int)(), C.POINTER(C.c_int)()
    v = C.POINTER(C.c_double)()
    check(L.mf_read_matrix(str(path).encode(), C.byref(m), C.byref(n), C.byref(nnz), C.byref(rp), C.byref(ci),
                           C.byref(v), C.byref(sym)))
    return _take_csr(m.value, nnz.value, rp, ci, v, n_cols=n.value), sym.value


def read_cbd(path):
    """A binary CSR (.cbd) file (mf_read_cbd)."""
    L = lib()
    m, n, nnz = C.c_int(), C.c_int(), C.c_int()
    rp, ci = C.POINTER(C.c_int)(), C.POINTER(C.c_int)()
    v = C.POINTER(C.c_double)()
    check(L.mf_read_cbd(str(path).encode(), C.byref(m), C.byref(n), C.byref(nnz), C.byref(rp), C.byref(ci),
                        C.byref(v)))
    return _take_csr(m.value, nnz.value, rp, ci, v, n_cols=n.value)


def write_cbd(path, A):
    """Writes A as a binary CSR (.cbd) file (mf_write_cbd)."""
    check(lib().mf_write_cbd(str(path).encode(), A.n_rows, A.n_cols, A.nnz, A.rowptr.ctypes.data,
                             A.colidx.ctypes.data, A.val.ctypes.data))


def solve_opts(**kw):
    o = SolveOpts()
    lib().mf_solve_opts_default(C.byref(o))
    for k, val in kw.items():
        if k == "policy" and isinstance(val, str):
            val = POLICY[val]
        setattr(o, k, val)
    return o


class Matrix:
    """A device-resident tiled matrix (mf_matrix handle)."""

    def __init__(self, csr: HostCsr, rows=None, cols=None, val_low=None, _handle=None):
        if _handle is not None:  # a handle made by another entry point (matrix_from_mtx)
            self._keep = None
            self.h = _handle
            return
        L = lib()
        rows = csr.n_rows if rows is None else rows
        cols = csr.n_cols if cols is None else cols
        h = C.c_void_p()
        self._keep = (csr, None if val_low is None else np.ascontiguousarray(val_low, np.float32))
        vl = None if val_low is None else self._keep[1].ctypes.data
        check(L.mf_matrix_create(rows, cols, csr.rowptr.ctypes.data, csr.colidx.ctypes.data, csr.val.ctypes.data,
                                 vl, 0, None, C.byref(h)))
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            lib().mf_matrix_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def info(self) -> MatrixInfo:
        inf = MatrixInfo()
        check(lib().mf_matrix_get_info(self.h, C.byref(inf)))
        return inf

    def export(self, name):
        L = lib()
        nb = C.c_size_t()
        check(L.mf_matrix_array_bytes(self.h, name.encode(), C.byref(nb)))
        dt = np.dtype(ARRAY_DTYPES[name])
        out = np.zeros(nb.value // dt.itemsize, dt)
        check(L.mf_matrix_export(self.h, name.encode(), out.ctypes.data if out.size else None, nb.value))
        return out

    def encode_column_index(self):
        check(lib().mf_encode_column_index(self.h, None))

    def attach_policy(self, policy):
        """Uses `policy` (a Policy, or None to detach) for MF_POLICY_LEARNED."""
        check(lib().mf_matrix_attach_policy(self.h, None if policy is None else policy.h))
        self._policy = policy

    def solve_host(self, b, method="cg", **opts):
        """CG (or BiCGSTAB) with host b/x through mf_*_solve_host; returns
        (x, report)."""
        b = np.ascontiguousarray(b, np.float64)
        x = np.zeros(self.info().rows, np.float64)
        rep = SolveReport()
        o = solve_opts(**opts)
        fn = lib().mf_bicgstab_solve_host if method == "bicgstab" else lib().mf_cg_solve_host
        st = fn(self.h, b.ctypes.data, x.ctypes.data, C.byref(o), C.byref(rep))
        if st not in (MF_OK, 6):
            check(st)
        return x, rep


def solve_multi_host(M, B, **opts):
    """k <= 16 right-hand sides at once (mf_cg_solve_multi_host): B is
    rows x k; returns (status, X rows x k, list of k SolveReport)."""
    B = np.asarray(B, np.float64)
    if B.ndim == 1:
        B = B[:, None]
    n, k = B.shape
    Bc = np.asfortranarray(B)
    X = np.zeros((n, k), np.float64, order="F")
    reps = (SolveReport * max(k, 1))()
    o = solve_opts(**opts)
    st = lib().mf_cg_solve_multi_host(M.h, k, Bc.ctypes.data, X.ctypes.data, C.byref(o), reps)
    return st, np.ascontiguousarray(X), list(reps)[:k]


class Batch:
    """Many independent systems solved by one batched launch (mf_batch)."""

    def __init__(self, systems):
        self.systems = list(systems)
        cnt = len(self.systems)
        n = np.array([A.n_rows for A in self.systems], np.int32)
        self._keep = [(A.rowptr, A.colidx, A.val) for A in self.systems]
        rp = (C.c_void_p * cnt)(*[A.rowptr.ctypes.data for A in self.systems])
        ci = (C.c_void_p * cnt)(*[A.colidx.ctypes.data for A in self.systems])
        va = (C.c_void_p * cnt)(*[A.val.ctypes.data for A in self.systems])
        h = C.c_void_p()
        check(lib().mf_batch_create(cnt, n.ctypes.data, rp, ci, va, C.byref(h)))
        self.h = h
        self.n = n
        self.offsets = np.concatenate([[0], np.cumsum(n.astype(np.int64))])

    def close(self):
        if getattr(self, "h", None):
            lib().mf_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def stack(self, parts):
        return np.ascontiguousarray(np.concatenate(parts), np.float64)

    def split(self, v):
        return [v[self.offsets[k]:self.offsets[k + 1]] for k in range(len(self.systems))]

    def solve_device(self, db_ptr, dx_ptr, use_graph=1, stream=None, **opts):
        rep = BatchReport()
        o = solve_opts(**opts)
        st = lib().mf_batch_cg_solve(self.h, db_ptr, dx_ptr, C.byref(o), use_graph, C.byref(rep), stream)
        return st, rep

    def results(self):
        it = np.zeros(len(self.systems), np.int32)
        rr = np.zeros(len(self.systems), np.float64)
        check(lib().mf_batch_results(self.h, it.ctypes.data, rr.ctypes.data))
        return it, rr

    def tune(self, db_ptr, dx_ptr, **opts):
        o = solve_opts(**opts)
        la, cl = C.c_int(), C.c_int()
        check(lib().mf_batch_tune(self.h, db_ptr, dx_ptr, C.byref(o), C.byref(la), C.byref(cl), None))
        return la.value, cl.value

    def chunk_count(self):
        """(chunks, chunks exact in FP16, chunks that can be held in FP16)."""
        a, b, c = C.c_int(), C.c_int(), C.c_int()
        check(lib().mf_batch_chunk_count(self.h, C.byref(a), C.byref(b), C.byref(c)))
        return a.value, b.value, c.value

    def export(self, name):
        nch = self.chunk_count()[0]
        nz = int(sum(A.nnz for A in self.systems))
        rows = int(self.offsets[-1])
        spec = {"chunk_class": (np.uint8, nch), "chunk_static": (np.uint8, nch),
                "chunk_features_static": (np.float32, 6 * nch), "chunk_start": (np.int32, len(self.systems) + 1),
                "chunk_rows": (np.int32, nch + len(self.systems)), "chunk_ends": (np.int32, nch + len(self.systems)),
                "val16": (np.uint16, nz),
                "val32": (np.float32, nz), "val": (np.float64, nz), "row_scale": (np.float32, rows),
                "diag32": (np.float32, rows), "col": (np.uint16, nz)}
        dt, cnt = spec[name]
        out = np.zeros(cnt, dt)
        check(lib().mf_batch_export(self.h, name.encode(), out.ctypes.data if cnt else None, out.nbytes))
        return out

    def attach_policy(self, policy):
        check(lib().mf_batch_attach_policy(self.h, None if policy is None else policy.h))
        self._policy = policy

    def collect(self, policy, db_ptr, checkpoint_every=20, sample_stride=1, max_samples=1 << 20):
        got = C.c_longlong()
        check(lib().mf_batch_policy_collect(policy.h, self.h, db_ptr, checkpoint_every, sample_stride, max_samples,
                                            C.byref(got)))
        return got.value


class Policy:
    """The learned per-tile precision policy (mf_learned handle)."""

    def __init__(self, seed=0, _handle=None):
        if _handle is None:
            _handle = C.c_void_p()
            check(lib().mf_policy_create(seed, C.byref(_handle)))
        self.h = _handle

    @classmethod
    def load(cls, path):
        h = C.c_void_p()
        check(lib().mf_policy_load(str(path).encode(), C.byref(h)))
        return cls(_handle=h)

    @staticmethod
    def param_count():
        return lib().mf_policy_param_count()

    def close(self):
        if getattr(self, "h", None):
            lib().mf_policy_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def params(self):
        w = np.zeros(self.param_count(), np.float32)
        check(lib().mf_policy_get_params(self.h, w.ctypes.data, w.size))
        return w

    def set_params(self, w):
        w = np.ascontiguousarray(w, np.float32)
        check(lib().mf_policy_set_params(self.h, w.ctypes.data, w.size))

    def save(self, path):
        check(lib().mf_policy_save(self.h, str(path).encode()))

    def collect(self, matrix, b_dev_ptr, checkpoint_every=10, sample_stride=1, max_samples=1 << 20):
        """Appends samples from an FP64 solve of matrix with device rhs; returns the sample count."""
        n = C.c_longlong()
        check(lib().mf_policy_collect(self.h, matrix.h, b_dev_ptr, checkpoint_every, sample_stride, max_samples,
                                      C.byref(n)))
        return n.value

    def label_counts(self):
        c = np.zeros(4, np.int64)
        check(lib().mf_policy_label_counts(self.h, c.ctypes.data))
        return c

    def train(self, epochs=5, batch=1024, lr=3e-3, seed=0):
        """Adam over the collected samples; returns (first batch loss, last epoch mean loss)."""
        l0, l1 = C.c_double(), C.c_double()
        check(lib().mf_policy_train(self.h, epochs, batch, lr, seed, C.byref(l0), C.byref(l1)))
        return l0.value, l1.value

    def eval_grad(self, X, Y):
        """Mean cross-entropy loss and its gradient at the current weights."""
        X = np.ascontiguousarray(X, np.float32)
        Y = np.ascontiguousarray(Y, np.int32)
        g = np.zeros(self.param_count(), np.float32)
        loss = C.c_double()
        check(lib().mf_policy_eval_grad(self.h, X.ctypes.data, Y.ctypes.data, len(Y), g.ctypes.data,
                                        C.byref(loss)))
        return loss.value, g
