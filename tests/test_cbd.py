"""Binary CSR (.cbd) files, the reference's cache of a parsed matrix
(binary_read_csr / binary_write_csr, src/biio2.0/src/biio.h:22-94), and the
extension-dispatching reader the CLIs use (read_Dmatrix_32, biio.h:153).
Host only."""
import subprocess

import numpy as np
import pytest

import dropin
from oracle_lib import Csr


def ref_bytes(A):
    """The file the reference's binary_write_csr produces for A, built field
    by field: int32 rows, int32 cols, int64 nnz, int64 row_ptr[rows+1],
    int32 col_idx[nnz], double val[nnz] (little-endian, as on this host)."""
    return (np.array([A.n_rows, A.n_cols], "<i4").tobytes() + np.array([A.nnz], "<i8").tobytes() +
            A.rowptr.astype("<i8").tobytes() + A.colidx.astype("<i4").tobytes() + A.val.astype("<f8").tobytes())


def same(A, B):
    return (A.n_rows, A.n_cols) == (B.n_rows, B.n_cols) and np.array_equal(A.rowptr, B.rowptr) and \
        np.array_equal(A.colidx, B.colidx) and np.array_equal(A.val.view(np.uint64), B.val.view(np.uint64))


@pytest.fixture
def mats(mf):
    return [mf.synth_laplace2d(9, 7), mf.synth_random_spd(3, 500), mf.synth_poisson3d_scaled(5, 2)]


def test_write_is_the_reference_layout(mf, mats, tmp_path):
    for k, A in enumerate(mats):
        f = tmp_path / f"a{k}.cbd"
        mf.write_cbd(f, A)
        assert f.read_bytes() == ref_bytes(A)


def test_read_reference_layout_round_trip(mf, mats, tmp_path):
    for k, A in enumerate(mats):
        f = tmp_path / f"a{k}.cbd"
        f.write_bytes(ref_bytes(A))
        assert same(mf.read_cbd(f), A)
        B, sym = mf.read_matrix(f)
        assert same(B, A) and sym == 0


def test_mtx_and_cbd_read_the_same(mf, tmp_path):
    """A symmetric Matrix Market file is expanded on reading; its .cbd copy
    (what the reference caches next to it) reads back to the same arrays."""
    A = mf.synth_laplace2d(6, 5)
    f = tmp_path / "lap.mtx"
    dropin.write_mtx(f, Csr(A.n_rows, A.n_cols, A.rowptr, A.colidx, A.val), symmetric=True)
    M, sym = mf.read_matrix(f)
    assert sym == 1 and M.nnz == A.nnz
    g = tmp_path / "lap.cbd"
    mf.write_cbd(g, M)
    B, sym2 = mf.read_matrix(g)
    assert sym2 == 0 and same(B, M)


def test_empty_matrix(mf, tmp_path):
    A = mf.HostCsr(4, 3, np.zeros(5, np.int32), np.zeros(0, np.int32), np.zeros(0))
    f = tmp_path / "e.cbd"
    mf.write_cbd(f, A)
    B = mf.read_cbd(f)
    assert (B.n_rows, B.n_cols, B.nnz) == (4, 3, 0) and np.array_equal(B.rowptr, A.rowptr)


def _bad(mf, path):
    with pytest.raises(mf.MfError) as e:
        mf.read_cbd(path)
    return e.value.status


def test_malformed_files(mf, tmp_path):
    A = mf.synth_laplace2d(4, 4)
    good = ref_bytes(A)
    cases = {
        "truncated": good[:-8],
        "trailing": good + b"\0" * 8,
        "short_header": good[:10],
    }
    rp = A.rowptr.copy()
    rp[3], rp[4] = rp[4], rp[3]  # decreasing
    B = mf.HostCsr(A.n_rows, A.n_cols, rp, A.colidx, A.val)
    cases["decreasing_rowptr"] = ref_bytes(B)
    rp0 = A.rowptr.copy()
    rp0[0] = 1
    cases["rowptr_start"] = ref_bytes(mf.HostCsr(A.n_rows, A.n_cols, rp0, A.colidx, A.val))
    ci = A.colidx.copy()
    ci[5] = A.n_cols
    cases["column_out_of_range"] = ref_bytes(mf.HostCsr(A.n_rows, A.n_cols, A.rowptr, ci, A.val))
    neg = bytearray(good)
    neg[0:4] = np.array([-1], "<i4").tobytes()
    cases["negative_rows"] = bytes(neg)
    for name, data in cases.items():
        f = tmp_path / f"{name}.cbd"
        f.write_bytes(data)
        assert _bad(mf, f) == 7, name  # MF_ERR_IO
    huge = bytearray(good)
    huge[8:16] = np.array([1 << 31], "<i8").tobytes()
    f = tmp_path / "huge.cbd"
    f.write_bytes(bytes(huge))
    assert _bad(mf, f) == 8  # MF_ERR_UNSUPPORTED: more than 2^31-1 entries
    assert _bad(mf, tmp_path / "missing.cbd") == 7


def test_read_matrix_rejects_other_extensions(mf, tmp_path):
    f = tmp_path / "a.txt"
    f.write_text("%%MatrixMarket matrix coordinate real general\n1 1 1\n1 1 1.0\n")
    with pytest.raises(mf.MfError) as e:
        mf.read_matrix(f)
    assert e.value.status == 7


@pytest.mark.parametrize("cli,out", [("main-cg", "unequal\n"), ("main-cg-mixed", "")])
def test_cli_reads_cbd(mf, cli, out, tmp_path):
    """The CLIs take .cbd files as the reference's do, announcing them on
    stdout (biio.h:160) before the non-square early exit."""
    A = mf.HostCsr(3, 4, np.array([0, 1, 2, 3], np.int32), np.array([0, 1, 3], np.int32), np.ones(3))
    f = tmp_path / "rect.cbd"
    mf.write_cbd(f, A)
    p = subprocess.run([str(dropin.BIN / cli), str(f)], capture_output=True, text=True, timeout=60, cwd=tmp_path)
    assert p.returncode == 0 and p.stdout == f"read binary file {f}\n" + out
