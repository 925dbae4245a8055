"""Staged row-slot chunks (the vector runs each chunk reads copied into shared
memory next to its slots) against the plain row slots, on the GPU.

Both layouts run the same operations in the same order, so every solve must
be bit-identical: same iterations, refinements and solution bits.  The
layout each solve ran is read from mf_solve_report.layout (1 plain row
slots, 2 staged)."""
import ctypes as C

import numpy as np
import pytest

import oracle_lib as ol

pytestmark = pytest.mark.gpu


def stencil27(g):
    """3D 27-point stencil, diagonal 27, neighbours -1 (SPD): 27 entries per
    interior row, so several half-warps share a strip."""
    rp, ci, va = [0], [], []
    for z in range(g):
        for y in range(g):
            for x in range(g):
                i = (z * g + y) * g + x
                for dz in (-1, 0, 1):
                    for dy in (-1, 0, 1):
                        for dx in (-1, 0, 1):
                            zz, yy, xx = z + dz, y + dy, x + dx
                            if 0 <= zz < g and 0 <= yy < g and 0 <= xx < g:
                                j = (zz * g + yy) * g + xx
                                ci.append(j)
                                va.append(27.0 if j == i else -1.0)
                rp.append(len(ci))
    return rp, ci, va


def _solve(mf, M, b, monkeypatch, layout, **opts):
    if layout is None:
        monkeypatch.delenv("MF_SOLVER_LAYOUT", raising=False)
    else:
        monkeypatch.setenv("MF_SOLVER_LAYOUT", layout)
    return M.solve_host(b, **opts)


def _same(r1, x1, r2, x2):
    assert r1.status == r2.status == 0, (r1.as_dict(), r2.as_dict())
    assert r1.iterations == r2.iterations and r1.refinements == r2.refinements
    assert np.array_equal(x1.view(np.uint64), x2.view(np.uint64))


CASES = [
    ("poisson3d_24", lambda mf: mf.synth_poisson3d_scaled(24, 1), 1),
    ("poisson3d_33", lambda mf: mf.synth_poisson3d_scaled(33, 2), 2),
    ("laplace2d_64", lambda mf: mf.synth_laplace2d(64, 64), 0),
    ("ragged_37x29", lambda mf: mf.synth_laplace2d(37, 29), 0),
    ("aniso_20", lambda mf: mf.synth_aniso3d(20, 3), 3),
]


@pytest.mark.parametrize("policy", ["static", "rule"])
@pytest.mark.parametrize("name,make,seed", CASES)
def test_staged_mixed_bit_identical_to_slots(mf, monkeypatch, policy, name, make, seed):
    A = make(mf)
    b = A.matvec(mf.synth_xstar(seed, A.n_rows))
    M = mf.Matrix(A)
    x2, r2 = _solve(mf, M, b, monkeypatch, None, tol=1e-10, maxiter=20000, policy=policy)
    x1, r1 = _solve(mf, M, b, monkeypatch, "slots", tol=1e-10, maxiter=20000, policy=policy)
    assert r2.layout == 2 and r1.layout == 1
    _same(r1, x1, r2, x2)
    assert ol.oracle_true_relres(ol.Csr(A.n_rows, A.n_cols, A.rowptr, A.colidx, A.val), b, x2) <= 1.05e-10
    M.close()


@pytest.mark.parametrize("name,make,seed", CASES[:3])
def test_staged_fp64_bit_identical_to_slots(mf, monkeypatch, name, make, seed):
    """The FP64 kernel on staged chunks (forced; its default is the plain
    slots) sums every row exactly as blockspmv_cpu: the solve is the same bit
    for bit.  The two-reduction kernel is forced (small systems would take
    the single-reduction one)."""
    monkeypatch.setenv("MF_CG_VARIANT", "2")
    A = make(mf)
    b = A.matvec(mf.synth_xstar(seed, A.n_rows))
    M = mf.Matrix(A)
    x2, r2 = _solve(mf, M, b, monkeypatch, "staged", tol=1e-10, maxiter=20000)
    x1, r1 = _solve(mf, M, b, monkeypatch, "slots", tol=1e-10, maxiter=20000)
    assert r2.layout == 2 and r1.layout == 1
    _same(r1, x1, r2, x2)
    M.close()


def test_staged_long_rows_share_strips(mf, monkeypatch):
    """27 entries per row: chunks of 4 strips, 4 half-warps per strip whose
    partial sums are added in order."""
    g = 14
    rp, ci, va = stencil27(g)
    n = g ** 3
    A = mf.HostCsr(n, n, np.array(rp), np.array(ci), np.array(va))
    b = A.matvec(mf.synth_xstar(5, n))
    M = mf.Matrix(A)
    for policy in ("static", "rule"):
        x2, r2 = _solve(mf, M, b, monkeypatch, None, tol=1e-10, maxiter=5000, policy=policy)
        x1, r1 = _solve(mf, M, b, monkeypatch, "slots", tol=1e-10, maxiter=5000, policy=policy)
        assert r2.layout == 2 and r1.layout == 1
        _same(r1, x1, r2, x2)
    M.close()


def test_scattered_columns_fall_back_to_slots(mf, monkeypatch):
    """Random SPD rows touch columns all over the matrix: no chunk's columns
    fit the staged vectors, the solve runs (correctly) from the plain
    slots."""
    A = mf.synth_random_spd(7, 4000)
    b = A.matvec(mf.synth_xstar(7, A.n_rows))
    M = mf.Matrix(A)
    x, r = _solve(mf, M, b, monkeypatch, None, tol=1e-10, maxiter=20000, policy="static")
    assert r.layout == 1 and r.status == 0
    assert ol.oracle_true_relres(ol.Csr(A.n_rows, A.n_cols, A.rowptr, A.colidx, A.val), b, x) <= 1.05e-10
    M.close()


def test_staged_fixed_iterations_and_tiny_budget(mf, monkeypatch):
    """A fixed-count staged solve equals the plain one; with a 1 ns wait
    budget a staged solve ends with MF_OK or MF_ERR_TIMEOUT (copies in flight
    drained before a CTA leaves) and the next solve runs normally."""
    A = mf.synth_poisson3d_scaled(32, 1)
    b = A.matvec(mf.synth_xstar(1, A.n_rows))
    M = mf.Matrix(A)
    x2, r2 = _solve(mf, M, b, monkeypatch, None, tol=-1.0, maxiter=77, policy="static")
    x1, r1 = _solve(mf, M, b, monkeypatch, "slots", tol=-1.0, maxiter=77, policy="static")
    assert r2.layout == 2 and r1.iterations == r2.iterations == 77
    assert np.array_equal(x1.view(np.uint64), x2.view(np.uint64))
    monkeypatch.delenv("MF_SOLVER_LAYOUT", raising=False)
    x = np.zeros(A.n_rows)
    rep = mf.SolveReport()
    o = mf.solve_opts(tol=1e-10, maxiter=5000, policy="static", wait_budget_s=1e-9)
    st = mf.lib().mf_cg_solve_host(M.h, b.ctypes.data, x.ctypes.data, C.byref(o), C.byref(rep))
    assert st in (0, 4) and rep.status == st
    x, rep = M.solve_host(b, tol=1e-10, maxiter=5000, policy="static")
    assert rep.status == 0 and rep.layout == 2 and rep.relres_true <= 1.05e-10
    M.close()


@pytest.mark.parametrize("g", [24, 33])
def test_staged_bicgstab_bit_identical_to_slots(mf, monkeypatch, g):
    """Mixed BiCGSTAB on staged chunks (w = p - omega v stored by the update
    pass, so each SpMV stages two vectors) equals the plain slots bit for
    bit on the nonsymmetric convection-diffusion system."""
    A = mf.synth_convdiff3d(g)
    b = A.matvec(mf.synth_xstar(2, A.n_rows))
    M = mf.Matrix(A)
    x2, r2 = _solve(mf, M, b, monkeypatch, None, method="bicgstab", tol=1e-9, maxiter=5000, policy="static")
    x1, r1 = _solve(mf, M, b, monkeypatch, "slots", method="bicgstab", tol=1e-9, maxiter=5000, policy="static")
    assert r2.layout == 2 and r1.layout == 1
    assert r1.status == r2.status == 0 and r1.iterations == r2.iterations
    assert np.array_equal(x1.view(np.uint64), x2.view(np.uint64))
    assert ol.oracle_true_relres(ol.Csr(A.n_rows, A.n_cols, A.rowptr, A.colidx, A.val), b, x2) <= 1.05e-9
    M.close()
