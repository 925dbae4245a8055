"""The rule policies' per-tile classes on the GPU against the CPU
restatement, bit for bit.

MF_POLICY_RULE is the reference's partial-convergence decision
(src/main-cg-mixed.cu:415-460): per 16-row segment of p, the largest
|p_new - p_old| in FP64 against the absolute thresholds 1e-5 / 1e-6 / 1e-7 /
1e-8 (FP64 / FP32 / FP16 / INT8 / BYPASS), and each tile takes the decision of
its column segment.  The direction vectors are fixed, seeded inputs whose
per-segment changes span every class, including values on the thresholds.
"""
import numpy as np
import pytest

import oracle_lib as ol

pytestmark = pytest.mark.gpu


def _directions(n, seed):
    """p_old ~ U[-1, 1]; p_new = p_old + d with per-segment magnitudes
    10^U[-10, -3] (random signs), a few elements placed on the thresholds."""
    rng = np.random.default_rng(seed)
    po = rng.uniform(-1, 1, n).astype(np.float32)
    nseg = (n + 15) // 16
    mag = 10.0 ** rng.uniform(-10, -3, nseg)
    d = rng.uniform(-1, 1, n) * np.repeat(mag, 16)[:n]
    pn = (po.astype(np.float64) + d).astype(np.float32)
    # segments whose directions did not change at all, and one of each
    # threshold hit as closely as FP32 allows
    pn[: 16 * 3] = po[: 16 * 3]
    for k, t in enumerate((1e-5, 1e-6, 1e-7, 1e-8)):
        j = 16 * (5 + k)
        if j < n:
            po[j] = np.float32(0.0)
            pn[j] = np.float32(t)
    return pn, po


def _run(mf, A, policy, seed):
    import torch

    lib = mf.lib()
    M = mf.Matrix(A)
    info = M.info()
    pn, po = _directions(A.n_cols, seed)
    T = info.tilenum
    d_pn = torch.from_numpy(np.pad(pn, (0, 16))).cuda()
    d_po = torch.from_numpy(np.pad(po, (0, 16))).cuda()
    dec = torch.full((T,), 255, dtype=torch.uint8, device="cuda")
    wrk = torch.full((T,), 255, dtype=torch.uint8, device="cuda")
    st = lib.mf_rule_classes(M.h, mf.POLICY[policy], d_pn.data_ptr(), d_po.data_ptr(), dec.data_ptr(),
                             wrk.data_ptr(), None)
    torch.cuda.synchronize()
    assert st == 0, lib.mf_last_error()
    tile_col = M.export("tile_columnidx")
    static_cls = M.export("tile_class")
    f16ok = M.export("tile_f16ok")
    # f16ok against the FP16 payload itself: bit 0 clear exactly where a
    # value is inf, bit 1 set where also no nonzero value became zero or
    # subnormal
    tnz = M.export("tile_nnz")
    f16 = M.export("payload_f16")
    val = M.export("Blockcsr_Val")
    per_tile = lambda bad: np.diff(np.concatenate([[0], np.cumsum(bad)])[tnz])
    n_inf = per_tile((f16 & 0x7C00) == 0x7C00)
    n_sub = per_tile(((f16 & 0x7C00) == 0) & (val != 0))
    want_ok = (n_inf == 0).astype(np.uint8) | (((n_inf == 0) & (n_sub == 0)).astype(np.uint8) << 1)
    assert np.array_equal(f16ok, want_ok)
    want_dec, want_wrk = ol.oracle_rule_tiles(A.n_cols, info.tilen, tile_col, static_cls, pn, po,
                                              scaled=(policy == "rule_scaled"), f16ok=f16ok)
    got_dec, got_wrk = dec.cpu().numpy(), wrk.cpu().numpy()
    M.close()
    return got_dec, got_wrk, want_dec, want_wrk


CASES = [
    ("poisson3d_64", lambda mf: mf.synth_poisson3d_scaled(64, 1)),
    ("laplace2d_128", lambda mf: mf.synth_laplace2d(128, 128)),
    ("laplace2d_ragged", lambda mf: mf.synth_laplace2d(37, 29)),
    ("aniso_64", lambda mf: mf.synth_aniso3d(64, 3)),  # values beyond binary16's range
]


@pytest.mark.parametrize("name,make", CASES)
@pytest.mark.parametrize("policy", ["rule", "rule_scaled"])
def test_rule_classes_match_restatement(mf, name, make, policy):
    A = make(mf)
    got_dec, got_wrk, want_dec, want_wrk = _run(mf, A, policy, seed=sum(map(ord, name)))
    assert np.array_equal(got_dec, want_dec), np.flatnonzero(got_dec != want_dec)[:10]
    assert np.array_equal(got_wrk, want_wrk), np.flatnonzero(got_wrk != want_wrk)[:10]
    if policy == "rule":
        # the changes span every decision of the reference's rule
        assert set(np.unique(got_dec).tolist()) == {0, 1, 2, 3, 4}


def test_rule_rejects_other_policies(mf):
    import torch

    lib = mf.lib()
    A = mf.synth_laplace2d(16, 16)
    M = mf.Matrix(A)
    p = torch.zeros(A.n_cols + 16, dtype=torch.float32, device="cuda")
    for pol in ("fp64", "static", "learned"):
        assert lib.mf_rule_classes(M.h, mf.POLICY[pol], p.data_ptr(), p.data_ptr(), None, None, None) == 1
    M.close()
