"""The FP64 CG oracle (oracle/mf_oracle.c orc_cg) pinned against SciPy's
conjugate gradient: the iterate after a fixed number of iterations, and the
iteration count to the relative residual 1e-10 (CPU only)."""
import numpy as np
import pytest
import scipy.sparse.linalg as spla

import oracle_lib as ol


def _system(mf, name):
    if name == "laplace2d_64":
        A, seed = mf.synth_laplace2d(64, 64), 0
    elif name == "poisson3d_20":
        A, seed = mf.synth_poisson3d_scaled(20, 1), 1
    else:
        A, seed = mf.synth_random_spd(105, 1500), 105
    b = A.matvec(mf.synth_xstar(seed, A.n_rows))
    return ol.Csr(A.n_rows, A.n_cols, A.rowptr, A.colidx, A.val), b


def _scipy_cg(csr, b, maxiter, rtol):
    its = [0]

    def cb(_):
        its[0] += 1

    x, info = spla.cg(csr.to_scipy(), b, x0=np.zeros_like(b), rtol=rtol, atol=0.0, maxiter=maxiter, callback=cb)
    return x, its[0], info


@pytest.mark.parametrize("name", ["laplace2d_64", "poisson3d_20", "randspd_1500"])
def test_oracle_cg_fixed_iterations_match_scipy(mf, name):
    csr, b = _system(mf, name)
    for k in (1, 3, 5):
        it, x, _ = ol.oracle_cg(csr, b, k, -1.0)
        xs, its, _ = _scipy_cg(csr, b, k, 1e-300)
        assert it == k == its
        # the same textbook recurrence with a different summation order (the
        # rounding differences grow with the iterations on ill-conditioned
        # systems, so the iterates are compared over the first few)
        assert np.max(np.abs(x - xs)) <= 1e-11 * max(1.0, np.max(np.abs(xs)))


@pytest.mark.parametrize("name", ["laplace2d_64", "poisson3d_20", "randspd_1500"])
def test_oracle_cg_iterations_to_tolerance_match_scipy(mf, name):
    csr, b = _system(mf, name)
    it, x, rr = ol.oracle_cg(csr, b, 20000, 1e-10)
    xs, its, info = _scipy_cg(csr, b, 20000, 1e-10)
    assert info == 0 and rr <= 1e-10
    assert abs(it - its) <= 1 + its // 100, (it, its)
    assert np.max(np.abs(x - xs)) <= 1e-7 * max(1.0, np.max(np.abs(xs)))
