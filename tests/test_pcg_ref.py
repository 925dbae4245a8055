"""Pins the test-side Jacobi-PCG checker (tests/pcg_ref.py) that the GPU
preconditioner tests compare against: same iterations (within one) and
solution as SciPy's preconditioned CG with the same diagonal preconditioner,
and the FP64 true residual at the tolerance."""
import numpy as np
import pytest
import scipy.sparse as sp
import scipy.sparse.linalg as spla

from pcg_ref import pcg_jacobi

CASES = [
    ("poisson3d_12", lambda mf: mf.synth_poisson3d_scaled(12, 1), 1),
    ("aniso_10", lambda mf: mf.synth_aniso3d(10, 3), 3),
    ("randspd_800", lambda mf: mf.synth_random_spd(107, 800), 107),
    ("laplace2d_20x17", lambda mf: mf.synth_laplace2d(20, 17), 0),
]


@pytest.mark.parametrize("name,make,seed", CASES)
def test_pcg_checker_matches_scipy(mf, name, make, seed):
    A = make(mf)
    b = A.matvec(mf.synth_xstar(seed, A.n_rows))
    it, x = pcg_jacobi(A, b, 1e-10, 5000)
    M = sp.csr_matrix((A.val, A.colidx, A.rowptr), shape=(A.n_rows, A.n_cols))
    d = M.diagonal()
    dinv = np.where(d != 0, 1.0 / np.where(d != 0, d, 1.0), 1.0)
    P = spla.LinearOperator(M.shape, matvec=lambda v: dinv * v)
    count = [0]

    def cb(_):
        count[0] += 1

    xs, info = spla.cg(M, b, rtol=1e-10, atol=0.0, maxiter=5000, M=P, callback=cb)
    assert info == 0
    assert abs(it - count[0]) <= 1, (it, count[0])
    scale = max(1.0, np.max(np.abs(xs)))
    assert np.max(np.abs(x - xs)) <= 1e-8 * scale
    assert np.linalg.norm(b - M @ x) <= 1.05e-10 * np.linalg.norm(b)


def test_pcg_checker_fewer_iterations_on_scaled_rows(mf):
    """Rows scaled by 10^U[-3,0]: the diagonal preconditioner removes most of
    the scaling, so the checker needs far fewer iterations than plain CG."""
    A = mf.synth_poisson3d_scaled(16, 1)
    b = A.matvec(mf.synth_xstar(1, A.n_rows))
    it_pc, _ = pcg_jacobi(A, b, 1e-10, 20000)
    M = sp.csr_matrix((A.val, A.colidx, A.rowptr), shape=(A.n_rows, A.n_cols))
    count = [0]
    spla.cg(M, b, rtol=1e-10, atol=0.0, maxiter=20000, callback=lambda _: count.__setitem__(0, count[0] + 1))
    assert it_pc < 0.8 * count[0], (it_pc, count[0])
