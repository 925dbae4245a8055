"""The reference's own entry points served by libmf (needs a B200):
Tile_create / Tile_destroy / blockspmv_cpu against the CPU oracle, the
cg_solve_* and bicgstab* calls against the FP64 oracle at the reference's
fixed iteration counts and to a tolerance, and the four CLIs end to end."""
import ctypes as C
import os
import subprocess

import numpy as np
import pytest

import dropin
import matrices
import oracle_lib as ol

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def tile_lib(mf):
    L = mf.lib()
    L.Tile_create.argtypes = [C.POINTER(dropin.TileMatrix), C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_void_p,
                              C.c_void_p, C.c_void_p]
    L.Tile_create.restype = None
    L.Tile_destroy.argtypes = [C.POINTER(dropin.TileMatrix)]
    L.Tile_destroy.restype = None
    vp = C.c_void_p
    L.blockspmv_cpu.argtypes = [C.POINTER(dropin.TileMatrix), vp, vp, C.POINTER(C.c_int), C.POINTER(vp),
                                C.POINTER(vp), C.POINTER(vp), C.c_int, C.c_int, C.c_int, vp, vp, vp, vp, vp, vp]
    L.blockspmv_cpu.restype = None
    return L


@pytest.fixture(scope="module")
def mats(mf):
    return matrices.all_matrices(mf)


def _tile_create(L, A):
    tm = dropin.TileMatrix()
    L.Tile_create(C.byref(tm), A.n_rows, A.n_cols, A.nnz, A.rowptr.ctypes.data, A.colidx.ctypes.data,
                  A.val.ctypes.data, None)
    return tm


@pytest.mark.parametrize("name", sorted(matrices.EDGE_CASES) + ["lap2d_32", "poisson3d_12", "aniso_12"])
def test_tile_create_matches_oracle(tile_lib, mats, name):
    A = mats[name]
    tm = _tile_create(tile_lib, A)
    sizes, orc, t = ol.oracle_tiles(A)
    try:
        assert {k: getattr(tm, k) for k in sizes} == sizes
        for field, (dt, key) in dropin.ARRAYS.items():
            got = tm.array(field, dt, dropin.length(tm, key))
            assert np.array_equal(got.view(np.uint8), orc[field].view(np.uint8)), field
        # allocated and zero-filled as in the reference (src/csr2block.h:387-389)
        assert not tm.array("csr_compressedIdx", np.uint8, (tm.csrsize + 1) // 2).any()
        assert tm.mf_handle and not tm.coo_offset and tm.coosize == 0
    finally:
        ol.free_oracle_tiles(t)
        tile_lib.Tile_destroy(C.byref(tm))
    assert tm.tile_ptr is None and tm.mf_handle is None and tm.tilenum == 0


def _blockspmv(L, tm, A, x):
    T = tm.tilenum
    p1 = np.zeros(max(T, 1), np.int32)
    p2 = np.zeros(max(T, 1), np.int32)
    rbb = C.c_int()
    ri, cs, ce = C.c_void_p(), C.c_void_p(), C.c_void_p()
    y = np.zeros(tm.tilem * 16 + 1, np.float64)
    L.blockspmv_cpu(C.byref(tm), p1.ctypes.data, p2.ctypes.data, C.byref(rbb), C.byref(ri), C.byref(cs),
                    C.byref(ce), A.n_rows, A.n_cols, A.nnz, A.rowptr.ctypes.data, A.colidx.ctypes.data,
                    A.val.ctypes.data, x.ctypes.data, y.ctypes.data, None)
    n = rbb.value
    assert n >= 0
    get = lambda p, dt: np.frombuffer((C.c_char * (4 * max(n, 1))).from_address(p.value), dt, n).copy()
    out = (p1[:T], p2[:T], get(ri, np.uint32), get(cs, np.int32), get(ce, np.int32), y[: A.n_rows])
    libc = C.CDLL(None)
    for p in (ri, cs, ce):
        libc.free(p)
    return out


@pytest.mark.parametrize("encoded", [False, True])
@pytest.mark.parametrize("name", ["empty_rows", "ragged_rect", "big_tilerow", "full_tile", "lap2d_32",
                                  "poisson3d_12"])
def test_blockspmv_cpu_matches_oracle(tile_lib, mats, name, encoded):
    """Schedule, offsets and y = A x bit-identical to blockspmv_cpu: with the
    zero csr_compressedIdx Tile_create leaves (every entry read as column 0,
    as the reference does), and after the caller encodes the columns."""
    A = mats[name]
    lib = ol.oracle()
    tm = _tile_create(tile_lib, A)
    sizes, orc, t = ol.oracle_tiles(A)
    try:
        cidx = np.zeros((tm.csrsize + 1) // 2 + 1, np.uint8)
        if encoded:
            lib.orc_encode(np.ascontiguousarray(orc["Tile_csr_Col"]), cidx, tm.csrsize, 0)
            C.memmove(tm.csr_compressedIdx, cidx.ctypes.data, (tm.csrsize + 1) // 2)
        i = np.arange(tm.tilen * 16, dtype=np.float64)
        x = np.sin(0.37 * i + 0.1) + 0.01 * i
        p1, p2, ri, cs, ce, y = _blockspmv(tile_lib, tm, A, x)
        T = sizes["tilenum"]
        rbb = lib.orc_rowblkblock_count(t)
        o1, o2 = np.zeros(max(T, 1), np.int32), np.zeros(max(T, 1), np.int32)
        ori = np.zeros(max(rbb, 1), np.uint32)
        ocs, oce = np.zeros(max(rbb, 1), np.int32), np.zeros(max(rbb, 1), np.int32)
        yo = np.zeros(sizes["tilem"] * 16, np.float64)
        lib.orc_blockspmv(t, A.n_rows, A.n_cols, cidx, o1, o2, ori, ocs, oce, x, yo)
        assert np.array_equal(p1, o1[:T]) and np.array_equal(p2, o2[:T])
        assert ri.size == rbb and np.array_equal(ri, ori[:rbb])
        assert np.array_equal(cs, ocs[:rbb]) and np.array_equal(ce, oce[:rbb])
        assert np.array_equal(y, yo[: A.n_rows])
    finally:
        ol.free_oracle_tiles(t)
        tile_lib.Tile_destroy(C.byref(tm))


def _csv_rows(path):
    return [l.split(",") for l in path.read_text().splitlines()]


@pytest.fixture()
def workdir(tmp_path, monkeypatch):
    (tmp_path / "data").mkdir()
    monkeypatch.chdir(tmp_path)
    monkeypatch.delenv("MF_SHIM_TOL", raising=False)
    monkeypatch.delenv("MF_SHIM_MAXITER", raising=False)
    monkeypatch.delenv("MF_SHIM_POLICY", raising=False)
    return tmp_path


def _cg_call(fn, A, b, n, ori):
    x = np.full(n, 7.0)  # zeroed on entry by the call
    it = C.c_int(-1)
    vl = A.val.astype(np.float32)
    fn(A.rowptr.ctypes.data, A.colidx.ctypes.data, A.val.ctypes.data, vl.ctypes.data, x.ctypes.data,
       b.ctypes.data, n, C.byref(it), 10, 1e-5, b"lap.mtx", A.nnz, ori)
    return x, it.value


@pytest.mark.parametrize("entry,iters", [("cg_solve_inc", 100), ("cg_solve_sync", 100)])
def test_cg_entry_fixed_iterations_match_oracle(mf, workdir, entry, iters):
    A = mf.synth_laplace2d(40, 40)
    Ac = ol.Csr(A.n_rows, A.n_cols, A.rowptr, A.colidx, A.val)
    b = A.matvec(np.ones(A.n_rows))
    x, it = _cg_call(getattr(dropin.solvers(False), entry), A, b, A.n_rows, A.n_rows)
    it_o, x_o, _ = ol.oracle_cg(Ac, b, iters, -1.0)
    assert it == iters == it_o
    assert np.max(np.abs(x - x_o)) <= 1e-9 * np.max(np.abs(x_o))
    rows = _csv_rows(workdir / "data" / "cg_performance.csv")
    assert len(rows) == 1 and rows[0][0] == "lap.mtx" and rows[0][1] == "100" and rows[0][3] == str(A.nnz)
    assert abs(float(rows[0][4]) - ol.oracle_true_relres(Ac, b, x)) <= 1e-12 + 1e-6 * float(rows[0][4])


def test_cg_reduce_runs_past_convergence(mf, workdir):
    """cg_solve_reduce runs 10000 iterations; an exactly zero residual ends
    the run early instead of dividing 0 by 0."""
    A = mf.synth_laplace2d(16, 16)
    b = A.matvec(np.ones(A.n_rows))
    x, it = _cg_call(dropin.solvers(False).cg_solve_reduce, A, b, A.n_rows, A.n_rows)
    assert np.all(np.isfinite(x)) and np.max(np.abs(x - 1.0)) <= 1e-10
    assert 0 < it <= 10000


def test_cg_entry_tolerance_override_and_truncation(mf, workdir, monkeypatch):
    """MF_SHIM_TOL stops at the tolerance.  n = 37 * 37 = 1369 rows are
    truncated to 1360: the leading block is solved, the tail of x stays 0."""
    monkeypatch.setenv("MF_SHIM_TOL", "1e-10")
    A = mf.synth_laplace2d(37, 37)
    n = A.n_rows // 16 * 16
    b = A.matvec(np.ones(A.n_rows))
    x, it = _cg_call(dropin.solvers(False).cg_solve_sync, A, b, n, A.n_rows)
    L = ol.Csr(A.n_rows, A.n_cols, A.rowptr, A.colidx, A.val).truncated(n)
    keep = L.colidx < n
    rp = np.concatenate([[0], np.cumsum([keep[L.rowptr[i]:L.rowptr[i + 1]].sum() for i in range(n)])])
    Lb = ol.Csr(n, n, rp.astype(np.int32), L.colidx[keep], L.val[keep])
    assert ol.oracle_true_relres(Lb, b[:n], x[:n]) <= 1.01e-10
    assert 0 < it < 1000
    rows = _csv_rows(workdir / "data" / "cg_performance.csv")
    assert float(rows[-1][4]) <= 1.01e-10


def test_cg_entry_mixed_library_to_tolerance(mf, workdir, monkeypatch):
    monkeypatch.setenv("MF_SHIM_TOL", "1e-10")
    A = mf.synth_poisson3d_scaled(16, 1)
    b = A.matvec(mf.synth_xstar(1, A.n_rows))
    x, it = _cg_call(dropin.solvers(True).cg_solve_inc, A, b, A.n_rows, A.n_rows)
    Ac = ol.Csr(A.n_rows, A.n_cols, A.rowptr, A.colidx, A.val)
    assert ol.oracle_true_relres(Ac, b, x) <= 1.01e-10


def _bicg_call(fn, A, x0, n):
    rhs = np.ones(A.n_rows)
    x = np.array(x0, np.float64)
    rc = fn(A.rowptr.ctypes.data, A.colidx.ctypes.data, A.val.ctypes.data, rhs.ctypes.data, x.ctypes.data,
            A.nnz, b"cd.mtx", n)
    return rc, rhs, x


@pytest.mark.parametrize("entry", ["bicgstab_sync", "bicgstab_inc"])
def test_bicgstab_entry_fixed_iterations(mf, workdir, entry):
    """rhs becomes the row sums (src/main-bicg.cu:480-487); 50 iterations;
    the solution matches the FP64 oracle's 50 iterations."""
    A = mf.synth_convdiff3d(8)
    Ac = ol.Csr(A.n_rows, A.n_cols, A.rowptr, A.colidx, A.val)
    rc, rhs, x = _bicg_call(getattr(dropin.solvers(False), entry), A, np.zeros(A.n_rows), A.n_rows)
    assert np.array_equal(rhs, np.array([A.val[A.rowptr[i]:A.rowptr[i + 1]].sum() for i in range(A.n_rows)]))
    it_o, x_o, _ = ol.oracle_bicgstab(Ac, rhs, 50, -1.0)
    assert rc == 1 and it_o == 50
    assert np.max(np.abs(x - x_o)) <= 1e-7 * np.max(np.abs(x_o))
    rows = _csv_rows(workdir / "data" / "bicg_performance.csv")
    assert rows[-1][0] == "cd.mtx" and rows[-1][1] == "50"


def test_bicgstab_entry_initial_guess_and_tolerance(mf, workdir, monkeypatch):
    monkeypatch.setenv("MF_SHIM_TOL", "1e-10")
    A = mf.synth_convdiff3d(8)
    Ac = ol.Csr(A.n_rows, A.n_cols, A.rowptr, A.colidx, A.val)
    rc, rhs, x = _bicg_call(dropin.solvers(False).bicgstab, A, np.full(A.n_rows, 0.5), A.n_rows)
    assert rc == 0
    assert ol.oracle_true_relres(Ac, rhs, x) <= 2e-10
    rc, rhs, x = _bicg_call(dropin.solvers(True).bicgstab, A, np.zeros(A.n_rows), A.n_rows)
    assert rc == 0 and ol.oracle_true_relres(Ac, rhs, x) <= 2e-10


def _run(cli, args, cwd, env=None):
    e = dict(os.environ)
    e.update(env or {})
    return subprocess.run([str(dropin.BIN / cli)] + args, capture_output=True, text=True, timeout=300, cwd=cwd,
                          env=e)


@pytest.mark.parametrize("cli,csv,tag", [("main-cg", "cg_performance.csv", "time_cg="),
                                         ("main-cg-mixed", "cg_performance.csv", "time_cg="),
                                         ("main-bicg", "bicg_performance.csv", "time_bicg="),
                                         ("main-bicg-mixed", "bicg_performance.csv", "time_bicg=")])
def test_cli_end_to_end(mf, tmp_path, cli, csv, tag):
    """A symmetric Matrix Market file (Laplacian 30x30 = 900 rows, truncated
    to 896): the CLI prints its time line and appends one CSV row, and with
    MF_SHIM_TOL the row reports a converged true residual."""
    (tmp_path / "data").mkdir()
    A = mf.synth_laplace2d(30, 30)
    f = tmp_path / "lap30.mtx"
    dropin.write_mtx(f, ol.Csr(A.n_rows, A.n_cols, A.rowptr, A.colidx, A.val), symmetric=True)
    p = _run(cli, [str(f)], tmp_path)
    assert p.returncode == 0, p.stderr
    assert p.stdout.startswith(tag), p.stdout
    p = _run(cli, [str(f)], tmp_path, {"MF_SHIM_TOL": "1e-10"})
    assert p.returncode == 0, p.stderr
    rows = _csv_rows(tmp_path / "data" / csv)
    assert len(rows) == 2 and rows[0][0] == str(f) and int(rows[0][3]) == A.nnz
    assert float(rows[1][4]) <= 2e-10


@pytest.mark.parametrize("cli,csv,tag", [("main-cg", "cg_performance.csv", "time_cg="),
                                         ("main-bicg-mixed", "bicg_performance.csv", "time_bicg=")])
def test_cli_end_to_end_binary_csr(mf, tmp_path, cli, csv, tag):
    """The same Laplacian as a binary CSR (.cbd) file, which the reference's
    CLIs also take: announced on stdout, then the solve as from the .mtx."""
    (tmp_path / "data").mkdir()
    A = mf.synth_laplace2d(30, 30)
    f = tmp_path / "lap30.cbd"
    mf.write_cbd(f, A)
    p = _run(cli, [str(f)], tmp_path)
    assert p.returncode == 0, p.stderr
    first, rest = p.stdout.split("\n", 1)
    assert first == f"read binary file {f}" and rest.startswith(tag), p.stdout
    rows = _csv_rows(tmp_path / "data" / csv)
    assert len(rows) == 1 and rows[0][0] == str(f) and int(rows[0][3]) == A.nnz
