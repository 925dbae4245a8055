"""GPU tile conversion and SpMV parity (needs a B200).

The GPU Tile_create must be bit-exact with the oracle (and, through the
committed digests, with the reference's own CPU code) on every array, and the
FP64 SpMV bit-identical to blockspmv_cpu's summation order."""
import hashlib
import json
from pathlib import Path

import numpy as np
import pytest

import matrices
import oracle_lib as ol

pytestmark = pytest.mark.gpu

GOLDEN = json.loads((Path(__file__).parent / "golden" / "tiles.json").read_text())


def digest(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


@pytest.fixture(scope="module")
def mats(mf):
    return matrices.all_matrices(mf)


def host(mf, A):
    return mf.HostCsr(A.n_rows, A.n_cols, A.rowptr, A.colidx, A.val)


@pytest.mark.parametrize("name", sorted(GOLDEN))
def test_gpu_tiles_bit_exact(mf, mats, name):
    A = mats[name]
    M = mf.Matrix(host(mf, A))
    g = GOLDEN[name]
    inf = M.info()
    assert (inf.tilem, inf.tilen, inf.tilenum, inf.csrsize, inf.csrptrlen) == tuple(
        g["sizes"][k] for k in ("tilem", "tilen", "tilenum", "csrsize", "csrptrlen"))
    for k, d in g["arrays"].items():
        assert digest(M.export(k)) == d, f"{name}:{k}"
    assert digest(M.export("ptroffset1")) == g["ptroffset1"]
    assert digest(M.export("ptroffset2")) == g["ptroffset2"]
    M.close()


@pytest.mark.parametrize("name", sorted(GOLDEN))
def test_gpu_derived_arrays_match_oracle(mf, mats, name):
    A = mats[name]
    M = mf.Matrix(host(mf, A))
    lib = ol.oracle()
    sizes, arrs, t = ol.oracle_tiles(A)
    try:
        T, tilem = sizes["tilenum"], sizes["tilem"]
        cnt = lib.orc_nonzero_rows_count(t, A.n_rows)
        nzr = np.zeros(T + 1, np.int32)
        tri = np.zeros(max(T, 1), np.int32)
        rid = np.zeros(cnt + 1, np.uint8)
        pn = np.zeros(cnt + 1, np.uint8)
        bs = np.zeros(tilem + 1, np.int32)
        lib.orc_nonzero_rows(t, A.n_rows, nzr, tri, rid, pn, bs)
        assert M.info().nonzero_rows == cnt
        assert np.array_equal(M.export("nonzero_row_new"), nzr)
        assert np.array_equal(M.export("tile_rowidx"), tri[:T])
        assert np.array_equal(M.export("blockrowid_new"), rid)
        assert np.array_equal(M.export("blockcsr_ptr_new"), pn)
        assert np.array_equal(M.export("block_signal"), bs)
        rbb = lib.orc_rowblkblock_count(t)
        assert M.info().rowblkblock == rbb
        ri = np.zeros(max(rbb, 1), np.uint32)
        cs = np.zeros(max(rbb, 1), np.int32)
        ce = np.zeros(max(rbb, 1), np.int32)
        p1 = np.zeros(max(T, 1), np.int32)
        p2 = np.zeros(max(T, 1), np.int32)
        x = np.zeros(sizes["tilen"] * 16)
        y = np.zeros(tilem * 16)
        cidx = np.zeros((sizes["csrsize"] + 1) // 2 + 1, np.uint8)
        lib.orc_blockspmv(t, A.n_rows, A.n_cols, cidx, p1, p2, ri, cs, ce, x, y)
        assert np.array_equal(M.export("rowblkblock_rowidx"), ri[:rbb])
        assert np.array_equal(M.export("rowblkblock_colstart"), cs[:rbb])
        assert np.array_equal(M.export("rowblkblock_colstop"), ce[:rbb])
        # payload casts (src/main-cg-mixed.cu:2333-2336)
        f32 = np.zeros(max(A.nnz, 1), np.float32)
        f16 = np.zeros(max(A.nnz, 1), np.uint16)
        i8 = np.zeros(max(A.nnz, 1), np.int8)
        vals = np.ascontiguousarray(arrs["Blockcsr_Val"])
        if vals.size:
            lib.orc_payload_casts(vals, vals.size, f32, f16, i8)
        assert np.array_equal(M.export("payload_f16"), f16[: vals.size])
        assert np.array_equal(M.export("payload_i8"), i8[: vals.size])
        # encode on the GPU equals the reference encode
        M.encode_column_index()
        enc = np.zeros((sizes["csrsize"] + 1) // 2 + 1, np.uint8)
        lib.orc_encode(np.ascontiguousarray(arrs["Tile_csr_Col"]), enc, sizes["csrsize"], 0)
        assert np.array_equal(M.export("csr_compressedIdx"), enc[: (sizes["csrsize"] + 1) // 2])
    finally:
        ol.free_oracle_tiles(t)
        M.close()


@pytest.mark.parametrize("name", sorted(GOLDEN))
def test_gpu_spmv_bit_identical(mf, mats, name):
    import torch

    A = mats[name]
    M = mf.Matrix(host(mf, A))
    inf = M.info()
    i = np.arange(inf.tilen * 16, dtype=np.float64)
    x = np.sin(0.37 * i + 0.1) + 0.01 * i
    dx = torch.from_numpy(x).cuda()
    dy = torch.zeros(max(A.n_rows, 1), dtype=torch.float64, device="cuda")
    mf.check(mf.lib().mf_spmv(M.h, dx.data_ptr(), dy.data_ptr(), None))
    torch.cuda.synchronize()
    y = dy.cpu().numpy()[: A.n_rows]
    assert digest(y) == GOLDEN[name]["blockspmv_y"]
    M.close()


def test_gpu_rejects_overfull_tile(mf):
    # 300 entries in one 16x16 tile (duplicates): the u8 row pointers cannot
    # describe it; the reference silently corrupts it, libmf refuses it.
    rows = 16
    rp = np.arange(0, rows * 20 + 1, 20, dtype=np.int32)
    ci = np.tile(np.arange(16, dtype=np.int32), rows * 20 // 16 + 1)[: rows * 20]
    v = np.ones(rows * 20)
    with pytest.raises(mf.MfError) as e:
        mf.Matrix(mf.HostCsr(rows, 16, rp, ci, v))
    assert e.value.status == 8


def test_gpu_rejects_bad_columns(mf):
    rp = np.array([0, 1, 2], np.int32)
    ci = np.array([0, 5], np.int32)
    with pytest.raises(mf.MfError) as e:
        mf.Matrix(mf.HostCsr(2, 4, rp, ci, np.ones(2)))
    assert e.value.status == 1


def test_gpu_config_sized_tiles_match_oracle(mf):
    """A 64^3 instance of the 3D configuration: every canonical array equal
    to the oracle's (sizes where the CPU oracle still takes seconds)."""
    A = mf.synth_poisson3d_scaled(64, 1)
    Ac = ol.Csr(A.n_rows, A.n_cols, A.rowptr, A.colidx, A.val)
    M = mf.Matrix(A)
    sizes, arrs, t = ol.oracle_tiles(Ac)
    try:
        for k in ol.TILE_ARRAYS:
            assert np.array_equal(M.export(k).view(np.uint8), arrs[k].view(np.uint8)), k
    finally:
        ol.free_oracle_tiles(t)
        M.close()


@pytest.mark.parametrize("name", ["lap2d_32", "poisson3d_12", "convdiff_10", "ragged_rect", "empty_rows"])
def test_gpu_residual_norm_matches_oracle(mf, mats, name):
    """mf_residual_norm (the reference's FP64 post-solve check) against the
    CPU oracle's sequential FP64 residual, on square test matrices."""
    import torch

    A = mats[name]
    if A.n_rows != A.n_cols:
        pytest.skip("square systems only")
    M = mf.Matrix(host(mf, A))
    rng = np.random.default_rng(3)
    x = rng.uniform(-1, 1, A.n_cols)
    b = rng.uniform(-1, 1, A.n_rows)
    out = torch.zeros(3, dtype=torch.float64, device="cuda")
    db, dx = torch.from_numpy(b).cuda(), torch.from_numpy(x).cuda()  # held alive across the call
    mf.check(mf.lib().mf_residual_norm(M.h, db.data_ptr(), dx.data_ptr(), out.data_ptr(), None))
    got = out.cpu().numpy()
    want = ol.oracle_true_relres(A, b, x)
    assert abs(got[0] - want) <= 1e-13 * max(1.0, want)
    assert abs(got[2] - np.linalg.norm(b)) <= 1e-12 * np.linalg.norm(b)
    M.close()
