"""Jacobi-preconditioned CG (mf_solve_opts.precond = 1) on the GPU against a
float64 NumPy/SciPy restatement of the same method (test-side checker: the
preconditioned method has no counterpart in the reference)."""
import ctypes as C

import numpy as np
import pytest

import oracle_lib as ol
from pcg_ref import pcg_jacobi

pytestmark = pytest.mark.gpu


CASES = [
    ("poisson3d_24", lambda mf: mf.synth_poisson3d_scaled(24, 1), 1),
    ("aniso_16", lambda mf: mf.synth_aniso3d(16, 3), 3),
    ("randspd_3000", lambda mf: mf.synth_random_spd(107, 3000), 107),
    ("laplace2d_37x29", lambda mf: mf.synth_laplace2d(37, 29), 0),
]


@pytest.mark.parametrize("name,make,seed", CASES)
def test_jacobi_fp64_matches_checker(mf, name, make, seed):
    A = make(mf)
    b = A.matvec(mf.synth_xstar(seed, A.n_rows))
    M = mf.Matrix(A)
    x, rep = M.solve_host(b, tol=1e-10, maxiter=20000, precond=1)
    it_o, x_o = pcg_jacobi(A, b, 1e-10, 20000)
    assert rep.status == 0, rep.as_dict()
    assert abs(rep.iterations - it_o) <= max(2, it_o // 50), (rep.iterations, it_o)
    assert ol.oracle_true_relres(ol.Csr(A.n_rows, A.n_cols, A.rowptr, A.colidx, A.val), b, x) <= 1.05e-10
    assert np.max(np.abs(x - x_o)) <= 1e-6 * max(1.0, np.max(np.abs(x_o)))
    M.close()


@pytest.mark.parametrize("policy", ["static", "rule"])
@pytest.mark.parametrize("name,make,seed", CASES[:2])
def test_jacobi_mixed_reaches_fp64_accuracy(mf, policy, name, make, seed):
    A = make(mf)
    b = A.matvec(mf.synth_xstar(seed, A.n_rows))
    M = mf.Matrix(A)
    x, rep = M.solve_host(b, tol=1e-10, maxiter=50000, policy=policy, precond=1)
    it_o, _ = pcg_jacobi(A, b, 1e-10, 50000)
    assert rep.status == 0 and rep.refinements >= 1, rep.as_dict()
    assert ol.oracle_true_relres(ol.Csr(A.n_rows, A.n_cols, A.rowptr, A.colidx, A.val), b, x) <= 1.05e-10
    assert rep.iterations <= 2 * it_o + 50, (rep.iterations, it_o)
    M.close()


def test_jacobi_cuts_iterations_on_scaled_rows(mf):
    """Rows scaled by 10^U[-3,0]: the diagonal scaling removes most of the
    spread, so the preconditioned solve needs far fewer iterations."""
    A = mf.synth_poisson3d_scaled(32, 1)
    b = A.matvec(mf.synth_xstar(1, A.n_rows))
    M = mf.Matrix(A)
    _, r0 = M.solve_host(b, tol=1e-10, maxiter=20000)
    _, r1 = M.solve_host(b, tol=1e-10, maxiter=20000, precond=1)
    assert r0.status == r1.status == 0
    assert r1.iterations < 0.8 * r0.iterations, (r1.iterations, r0.iterations)
    M.close()


@pytest.mark.parametrize("policy", ["static", "rule"])
def test_jacobi_staged_equals_slots(mf, monkeypatch, policy):
    A = mf.synth_poisson3d_scaled(24, 2)
    b = A.matvec(mf.synth_xstar(2, A.n_rows))
    M = mf.Matrix(A)
    monkeypatch.setenv("MF_SOLVER_LAYOUT", "staged")
    x2, r2 = M.solve_host(b, tol=1e-10, maxiter=20000, policy=policy, precond=1)
    monkeypatch.setenv("MF_SOLVER_LAYOUT", "slots")
    x1, r1 = M.solve_host(b, tol=1e-10, maxiter=20000, policy=policy, precond=1)
    assert r2.layout == 2 and r1.layout == 1 and r1.status == r2.status == 0
    assert r1.iterations == r2.iterations
    assert np.array_equal(x1.view(np.uint64), x2.view(np.uint64))
    M.close()


def test_jacobi_rejected_by_bicgstab(mf):
    A = mf.synth_convdiff3d(16)
    M = mf.Matrix(A)
    b = np.ones(A.n_rows)
    x = np.zeros(A.n_rows)
    rep = mf.SolveReport()
    o = mf.solve_opts(tol=1e-9, maxiter=100, precond=1)
    st = mf.lib().mf_bicgstab_solve_host(M.h, b.ctypes.data, x.ctypes.data, C.byref(o), C.byref(rep))
    assert st == 8  # MF_ERR_UNSUPPORTED
    M.close()


def test_jacobi_rejected_by_batch_and_bad_value(mf):
    import torch

    systems = [mf.synth_laplace2d(16, 16), mf.synth_laplace2d(8, 24)]
    B = mf.Batch(systems)
    nt = int(B.offsets[-1])
    db = torch.ones(nt, dtype=torch.float64, device="cuda")
    dx = torch.zeros(nt, dtype=torch.float64, device="cuda")
    st, _ = B.solve_device(db.data_ptr(), dx.data_ptr(), use_graph=0, tol=1e-9, maxiter=100, precond=1)
    assert st == 8  # MF_ERR_UNSUPPORTED
    B.close()
    A = mf.synth_laplace2d(16, 16)
    M = mf.Matrix(A)
    b = np.ones(A.n_rows)
    x = np.zeros(A.n_rows)
    rep = mf.SolveReport()
    o = mf.solve_opts(tol=1e-9, maxiter=100, precond=2)
    st = mf.lib().mf_cg_solve_host(M.h, b.ctypes.data, x.ctypes.data, C.byref(o), C.byref(rep))
    assert st == 1  # MF_ERR_INVALID_ARG
    M.close()
