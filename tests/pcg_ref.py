"""Float64 restatement of Jacobi-preconditioned CG (test-side checker for
mf_solve_opts.precond; the reference has no preconditioner): z = D^-1 r with
1 where the diagonal is 0, p = z + beta p, alpha = r.z / p.q, beta = r.z_new /
r.z, stop on ||r|| <= tol ||b||."""
import numpy as np
import scipy.sparse as sp


def pcg_jacobi(A, b, tol, maxiter):
    """z = D^-1 r (1 where the diagonal is 0), p = z + beta p, beta =
    r.z / r.z_old, stop on ||r|| <= tol ||b||; returns (iterations, x)."""
    M = sp.csr_matrix((A.val, A.colidx, A.rowptr), shape=(A.n_rows, A.n_cols))
    d = M.diagonal()
    dinv = np.where(d != 0, 1.0 / np.where(d != 0, d, 1.0), 1.0)
    x = np.zeros(A.n_rows)
    r = b.copy()
    z = dinv * r
    p = np.zeros(A.n_rows)
    rz = r @ z
    beta = 0.0
    nb = np.linalg.norm(b)
    for it in range(maxiter + 1):
        if np.linalg.norm(r) <= tol * nb:
            return it, x
        p = z + beta * p
        q = M @ p
        alpha = rz / (p @ q)
        x += alpha * p
        r -= alpha * q
        z = dinv * r
        rz_new = r @ z
        beta = rz_new / rz
        rz = rz_new
    return maxiter, x
