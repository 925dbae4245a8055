"""Several right-hand sides at once: mf_spmm (k <= 16 columns, one pass over
the matrix) against mf_spmv column by column, bit for bit, and
mf_cg_solve_multi (k independent FP64 CG recurrences sharing each SpMM)
against the CG oracle and the single-vector solver, with the edge cases of
the interface (zero right-hand sides, maxiter, fixed iteration counts,
determinism, rejected options)."""
import ctypes as C

import numpy as np
import pytest

import matrices
import oracle_lib as ol

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def mats(mf):
    return matrices.all_matrices(mf)


def host(mf, A):
    return mf.HostCsr(A.n_rows, A.n_cols, A.rowptr, A.colidx, A.val)


@pytest.mark.parametrize("k", [1, 5, 16])
@pytest.mark.parametrize("name", sorted(matrices.EDGE_CASES) + ["lap2d_32", "poisson3d_12", "randspd_1500"])
def test_spmm_columns_equal_spmv(mf, mats, name, k):
    import torch

    A = mats[name]
    M = mf.Matrix(host(mf, A))
    inf = M.info()
    rng = np.random.default_rng(7 + k)
    ldx, ldy = A.n_cols + 3, A.n_rows + 5
    X = rng.standard_normal((k, ldx))  # column j of X is row j here (column-major)
    dX = torch.from_numpy(X.copy()).cuda()
    dY = torch.full((k, ldy), np.nan, dtype=torch.float64, device="cuda")
    st = mf.lib().mf_spmm(M.h, k, dX.data_ptr(), ldx, dY.data_ptr(), ldy, None)
    assert st == 0, mf.lib().mf_last_error()
    torch.cuda.synchronize()
    Y = dY.cpu().numpy()
    for j in range(k):
        xp = np.zeros(inf.tilen * 16)
        xp[: A.n_cols] = X[j, : A.n_cols]
        dx = torch.from_numpy(xp).cuda()
        dy = torch.zeros(max(A.n_rows, 1), dtype=torch.float64, device="cuda")
        mf.check(mf.lib().mf_spmv(M.h, dx.data_ptr(), dy.data_ptr(), None))
        torch.cuda.synchronize()
        y1 = dy.cpu().numpy()[: A.n_rows]
        assert np.array_equal(Y[j, : A.n_rows].view(np.uint64), y1.view(np.uint64)), (name, j)
        assert np.all(np.isnan(Y[j, A.n_rows:]))  # past the rows: untouched
    M.close()


CG_CASES = [
    ("poisson3d_16", lambda mf: mf.synth_poisson3d_scaled(16, 1), 5),
    ("laplace2d_37x29", lambda mf: mf.synth_laplace2d(37, 29), 3),
    ("randspd_2000", lambda mf: mf.synth_random_spd(111, 2000), 16),
    ("aniso_12", lambda mf: mf.synth_aniso3d(12, 3), 8),
]


def _rhs(mf, A, k, seed0=20):
    return np.stack([A.matvec(mf.synth_xstar(seed0 + j, A.n_rows)) for j in range(k)], axis=1)


@pytest.mark.parametrize("name,make,k", CG_CASES)
def test_multi_cg_matches_oracle(mf, name, make, k):
    A = make(mf)
    B = _rhs(mf, A, k)
    M = mf.Matrix(A)
    st, X, reps = mf.solve_multi_host(M, B, tol=1e-10, maxiter=20000)
    assert st == 0, mf.lib().mf_last_error()
    csr = ol.Csr(A.n_rows, A.n_cols, A.rowptr, A.colidx, A.val)
    for j in range(k):
        it_o, x_o, _ = ol.oracle_cg(csr, B[:, j], 20000, 1e-10)
        r = reps[j]
        assert r.status == 0
        assert abs(r.iterations - it_o) <= max(2, it_o // 50), (j, r.iterations, it_o)
        assert r.relres <= 1e-10
        assert r.relres_true <= 1.05e-10, r.relres_true
        assert abs(ol.oracle_true_relres(csr, B[:, j], X[:, j]) - r.relres_true) <= 1e-12
        assert np.max(np.abs(X[:, j] - x_o)) <= 1e-6 * max(1.0, np.max(np.abs(x_o)))
    M.close()


def test_multi_cg_columns_match_single_solves(mf):
    A = mf.synth_poisson3d_scaled(20, 2)
    B = _rhs(mf, A, 6, seed0=40)
    M = mf.Matrix(A)
    st, X, reps = mf.solve_multi_host(M, B, tol=1e-10, maxiter=20000)
    assert st == 0
    for j in range(6):
        x1, r1 = M.solve_host(B[:, j], tol=1e-10, maxiter=20000, policy="fp64")
        assert r1.status == 0
        assert abs(reps[j].iterations - r1.iterations) <= 2, (reps[j].iterations, r1.iterations)
        assert np.max(np.abs(X[:, j] - x1)) <= 1e-7 * max(1.0, np.max(np.abs(x1)))
    M.close()


def test_multi_zero_column_and_maxiter(mf):
    A = mf.synth_laplace2d(40, 40)
    B = _rhs(mf, A, 4)
    B[:, 2] = 0.0
    M = mf.Matrix(A)
    st, X, reps = mf.solve_multi_host(M, B, tol=1e-10, maxiter=20000)
    assert st == 0
    assert reps[2].iterations == 0 and reps[2].status == 0 and not np.any(X[:, 2])
    # too few iterations: the other columns report not converged
    st, X, reps = mf.solve_multi_host(M, B, tol=1e-10, maxiter=5)
    assert st == 6  # MF_ERR_NOT_CONVERGED
    for j in (0, 1, 3):
        assert reps[j].status == 6 and reps[j].iterations == 5
    assert reps[2].status == 0 and reps[2].iterations == 0
    M.close()


def test_multi_fixed_iteration_count(mf):
    A = mf.synth_poisson3d_scaled(12, 3)
    B = _rhs(mf, A, 3)
    M = mf.Matrix(A)
    st, X, reps = mf.solve_multi_host(M, B, tol=-1.0, maxiter=7)
    assert st == 0
    assert [r.iterations for r in reps] == [7, 7, 7]
    M.close()


def test_multi_cg_deterministic_and_device_equals_host(mf):
    import torch

    A = mf.synth_random_spd(112, 1500)
    k = 7
    B = _rhs(mf, A, k)
    M = mf.Matrix(A)
    st1, X1, _ = mf.solve_multi_host(M, B, tol=1e-10, maxiter=20000)
    st2, X2, _ = mf.solve_multi_host(M, B, tol=1e-10, maxiter=20000)
    assert st1 == st2 == 0
    assert np.array_equal(X1.view(np.uint64), X2.view(np.uint64))
    n, ld = A.n_rows, A.n_rows + 9
    Bd = np.zeros((k, ld))
    Bd[:, :n] = B.T
    dB = torch.from_numpy(Bd).cuda()
    dX = torch.zeros((k, ld), dtype=torch.float64, device="cuda")
    reps = (mf.SolveReport * k)()
    o = mf.solve_opts(tol=1e-10, maxiter=20000)
    st = mf.lib().mf_cg_solve_multi(M.h, k, dB.data_ptr(), ld, dX.data_ptr(), ld, C.byref(o), reps, None)
    assert st == 0
    torch.cuda.synchronize()
    Xd = dX.cpu().numpy()[:, :n].T
    assert np.array_equal(np.ascontiguousarray(Xd).view(np.uint64), X1.view(np.uint64))
    M.close()


def test_multi_rejects(mf):
    A = mf.synth_laplace2d(16, 16)
    M = mf.Matrix(A)
    n = A.n_rows
    L = mf.lib()
    B = np.ones((n, 17))
    X = np.zeros((n, 17))
    reps = (mf.SolveReport * 17)()
    for k in (0, 17):
        o = mf.solve_opts()
        assert L.mf_cg_solve_multi_host(M.h, k, B.ctypes.data, X.ctypes.data, C.byref(o), reps) == 1
    # a solve run first leaves the staging buffer holding a solution ...
    o = mf.solve_opts()
    assert L.mf_cg_solve_multi_host(M.h, 2, B.ctypes.data, X.ctypes.data, C.byref(o), reps) == 0
    for kw in (dict(policy="static"), dict(precond=1)):
        # ... which an UNSUPPORTED call must not copy into the caller's X
        X[:] = 7.25
        o = mf.solve_opts(**kw)
        assert L.mf_cg_solve_multi_host(M.h, 2, B.ctypes.data, X.ctypes.data, C.byref(o), reps) == 8
        assert np.all(X == 7.25)
    o = mf.solve_opts()
    assert L.mf_cg_solve_multi(M.h, 2, None, n - 1, None, n, C.byref(o), reps, None) == 1
    assert L.mf_spmm(M.h, 0, None, n, None, n, None) == 1
    assert L.mf_spmm(M.h, 2, None, n - 1, None, n, None) == 1
    M.close()
