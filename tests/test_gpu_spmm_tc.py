"""mf_spmm_f16: Y = A X with the dense 16x16 tiles on the tensor cores (FP16
inputs, FP32 accumulation), against the exact FP64 product: every entry
within the FP16 rounding bound 2^-9 (|A| |X|), on a block-structured matrix
(dense diagonal and off-diagonal 16x16 blocks plus sparse couplings), on a
stencil without dense tiles, with every tile forced dense, for k = 1, 8, 9
and 16 with padded leading dimensions; run to run bit identity; rejected
arguments."""
import ctypes as C

import numpy as np
import pytest
import scipy.sparse as sp
import torch

pytestmark = pytest.mark.gpu


def block_matrix(nb, dense_per_row, sparse_per_row, seed, ragged=0):
    import __graft_entry__ as ge

    H = ge.load_package().synth_block_dense(nb, dense_per_row, sparse_per_row, seed, ragged)
    return sp.csr_matrix((H.val, H.colidx, H.rowptr), shape=(H.n_rows, H.n_cols))


def host(mf, A):
    return mf.HostCsr(A.shape[0], A.shape[1], A.indptr.astype(np.int32), A.indices.astype(np.int32),
                      A.data.astype(np.float64))


def dense_tiles_of(A, fill):
    coo = A.tocoo()
    key = (coo.row // 16).astype(np.int64) * ((A.shape[1] + 15) // 16) + coo.col // 16
    _, cnt = np.unique(key, return_counts=True)
    return int(np.count_nonzero(cnt >= fill))


def run(mf, M, A, X, k, fill=0, pad=(3, 5)):
    n, m = A.shape
    ldx, ldy = m + pad[0], n + pad[1]
    Xd = np.zeros((k, ldx))
    Xd[:, :m] = X[:, :k].T
    dX = torch.from_numpy(Xd).cuda()
    dY = torch.full((k, ldy), np.nan, dtype=torch.float64, device="cuda")
    nd = C.c_int(-1)
    st = mf.lib().mf_spmm_f16(M.h, k, dX.data_ptr(), ldx, dY.data_ptr(), ldy, fill, C.byref(nd), None)
    assert st == 0, mf.lib().mf_last_error()
    torch.cuda.synchronize()
    Y = dY.cpu().numpy()
    assert np.all(np.isnan(Y[:, n:]))  # past the rows: untouched
    return Y[:, :n].T, nd.value


def check_accuracy(A, X, Y, k):
    ref = A @ X[:, :k]
    bound = abs(A) @ np.abs(X[:, :k])
    err = np.abs(Y - ref)
    assert np.all(err <= 2.0 ** -9 * bound + 1e-300), float(np.max(err / np.maximum(bound, 1e-300)))


@pytest.mark.parametrize("k", [1, 8, 9, 16])
def test_block_matrix_dense_tiles_on_tensor_cores(mf, k):
    A = block_matrix(300, 3, 2, seed=k, ragged=5)
    M = mf.Matrix(host(mf, A))
    X = np.random.default_rng(100 + k).normal(size=(A.shape[1], 16)) * 10.0 ** np.arange(-8, 8)
    Y, nd = run(mf, M, A, X, k)
    assert nd == dense_tiles_of(A, 64) and nd >= 300
    check_accuracy(A, X, Y, k)
    Y2, _ = run(mf, M, A, X, k)
    assert np.array_equal(Y.view(np.uint64), Y2.view(np.uint64))  # deterministic
    M.close()


def test_stencil_without_dense_tiles_and_all_tiles_dense(mf):
    A0 = mf.synth_poisson3d_scaled(12, 1)
    A = sp.csr_matrix((A0.val, A0.colidx, A0.rowptr), shape=(A0.n_rows, A0.n_cols))
    M = mf.Matrix(A0)
    X = np.random.default_rng(1).normal(size=(A.shape[1], 16))
    Y, nd = run(mf, M, A, X, 16)
    assert nd == 0
    check_accuracy(A, X, Y, 16)
    Y1, nd1 = run(mf, M, A, X, 16, fill=1)  # every tile dense (FP16 values)
    assert nd1 == dense_tiles_of(A, 1)
    check_accuracy(A, X, Y1, 16)
    M.close()


def test_rejects(mf):
    A = block_matrix(4, 1, 1, seed=0)
    M = mf.Matrix(host(mf, A))
    n = A.shape[0]
    L = mf.lib()
    d = torch.zeros(16 * (n + 1), dtype=torch.float64, device="cuda")
    for k, fill, ld in [(0, 0, n), (17, 0, n), (4, 257, n), (4, 0, n - 1)]:
        assert L.mf_spmm_f16(M.h, k, d.data_ptr(), ld, d.data_ptr(), ld, fill, None, None) == 1
    M.close()
