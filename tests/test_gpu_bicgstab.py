"""Persistent BiCGSTAB on the GPU against the FP64 CPU oracle (needs a B200)."""
import numpy as np
import pytest

import oracle_lib as ol

pytestmark = pytest.mark.gpu


def _oc(A):
    return ol.Csr(A.n_rows, A.n_cols, A.rowptr, A.colidx, A.val)


@pytest.mark.parametrize("policy", ["fp64", "static"])
@pytest.mark.parametrize("g", [12, 24])
def test_bicgstab_convdiff_matches_oracle(mf, policy, g):
    """The nonsymmetric convection-diffusion configuration at small sizes:
    stop at 1e-9 on the recurrence; the FP64 true residual and the error
    against the oracle solution are checked."""
    A = mf.synth_convdiff3d(g)
    xs = mf.synth_xstar(2, A.n_rows)
    b = A.matvec(xs)
    M = mf.Matrix(A)
    x, rep = M.solve_host(b, method="bicgstab", tol=1e-9, maxiter=5000, policy=policy)
    it_o, x_o, rr_o = ol.oracle_bicgstab(_oc(A), b, 5000, 1e-9)
    assert rep.status == 0, rep.as_dict()
    true_rr = ol.oracle_true_relres(_oc(A), b, x)
    assert true_rr <= 2e-9, (true_rr, rep.as_dict())
    assert rep.iterations <= int(1.5 * it_o) + 10, (rep.iterations, it_o)
    err_o = np.max(np.abs(x_o - xs))
    assert np.max(np.abs(x - x_o)) <= 10 * err_o + 1e-9
    M.close()


def test_bicgstab_fixed_iterations_like_reference(mf):
    """tol < 0 runs exactly maxiter iterations (the reference's persistent
    BiCGSTAB runs a fixed 50, src/Mille-feuille-bicg.h:272)."""
    A = mf.synth_convdiff3d(10)
    b = A.matvec(np.ones(A.n_rows))
    M = mf.Matrix(A)
    x, rep = M.solve_host(b, method="bicgstab", tol=-1.0, maxiter=20)
    it_o, x_o, _ = ol.oracle_bicgstab(_oc(A), b, 20, -1.0)
    assert rep.iterations == 20 == it_o
    assert np.max(np.abs(x - x_o)) <= 1e-8 * max(1.0, np.max(np.abs(x_o)))
    M.close()


def test_bicgstab_spd_system(mf):
    A = mf.synth_poisson3d_scaled(16, 1)
    b = A.matvec(mf.synth_xstar(1, A.n_rows))
    M = mf.Matrix(A)
    x, rep = M.solve_host(b, method="bicgstab", tol=1e-10, maxiter=5000)
    assert rep.status == 0
    assert ol.oracle_true_relres(_oc(A), b, x) <= 2e-10
    M.close()
