"""mf_residual_norm_noalloc: the residual check for callers that may not
allocate device memory (fixed device-memory budgets, caller-owned allocators,
no tolerance for the synchronisation an allocation can cause).  Called through
the C ABI, it must give the same value as mf_residual_norm, call after call,
and refuse matrices beyond its fixed scratch limit.  Collected last on
purpose; it depends on no other test."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = 1e-13  # relative, as the residual tests use


def _norms(mf, fn, M, db, dx):
    import torch

    out = torch.full((3,), -1.0, dtype=torch.float64, device="cuda")
    st = fn(M.h, db.data_ptr(), dx.data_ptr(), out.data_ptr(), None)
    torch.cuda.synchronize()
    return st, out.cpu().numpy()


def test_noalloc_matches_allocating_entry_point_twice(mf):
    import torch

    lib = mf.lib()
    rng = np.random.default_rng(11)
    cases = [mf.synth_poisson3d_scaled(24, 1), mf.synth_laplace2d(100, 37)]
    for A in cases:  # two calls in a row, on different systems and sizes
        M = mf.Matrix(A)
        x = torch.from_numpy(rng.uniform(-1, 1, A.n_cols)).cuda()
        b = torch.from_numpy(A.matvec(rng.uniform(-1, 1, A.n_cols))).cuda()
        st_ref, ref = _norms(mf, lib.mf_residual_norm, M, b, x)
        for _ in range(2):
            st, got = _norms(mf, lib.mf_residual_norm_noalloc, M, b, x)
            assert st == 0 and st_ref == 0, lib.mf_last_error()
            assert np.all(np.abs(got - ref) <= TOL * np.maximum(1.0, np.abs(ref)))
            assert got[0] > 0.0
        M.close()


def test_noalloc_rejects_matrices_beyond_its_limit(mf):
    import torch

    lib = mf.lib()
    A = mf.synth_laplace2d(1025, 1024)  # 1,049,600 rows > 1,048,576
    M = mf.Matrix(A)
    x = torch.zeros(A.n_cols, dtype=torch.float64, device="cuda")
    st, out = _norms(mf, lib.mf_residual_norm_noalloc, M, x, x)
    assert st == 1  # MF_ERR_INVALID_ARG
    assert b"1048576" in lib.mf_last_error()
    assert np.all(out == -1.0)  # nothing was written
    M.close()
