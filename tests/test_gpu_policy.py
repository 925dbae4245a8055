"""The learned per-tile precision policy on the GPU: its training gradient
against the FP64 CPU oracle of the same network, sample collection from FP64
solver traces, training, and LEARNED solves to the FP64 tolerance (needs a
B200)."""
import numpy as np
import pytest

import oracle_lib as ol

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch():
    import torch as t

    return t


def test_policy_gradient_matches_oracle(mf):
    P = mf.Policy(seed=3)
    w = P.params()
    assert w.size == mf.Policy.param_count() == 1732
    rng = np.random.default_rng(4)
    n = 300  # three training blocks, the last one partial
    X = rng.normal(size=(n, 16)).astype(np.float32)
    Y = rng.integers(0, 4, size=n).astype(np.int32)
    loss, g = P.eval_grad(X, Y)
    go = np.zeros(w.size)
    lo = ol.oracle().orc_mlp_grad(w, X, Y, n, go)
    # FP32 forward/backward against FP64: relative to the gradient's scale
    assert abs(loss - lo) <= 1e-5 * max(1.0, abs(lo))
    assert np.max(np.abs(g - go)) <= 1e-4 * np.max(np.abs(go)) + 1e-7
    # deterministic: the same bits twice
    loss2, g2 = P.eval_grad(X, Y)
    assert loss2 == loss and np.array_equal(g, g2)
    P.close()


def test_policy_save_load_roundtrip(mf, tmp_path):
    P = mf.Policy(seed=9)
    f = tmp_path / "p.mfpol"
    P.save(f)
    Q = mf.Policy.load(f)
    assert np.array_equal(P.params(), Q.params())
    bad = tmp_path / "bad.mfpol"
    bad.write_bytes(b"not a policy")
    with pytest.raises(mf.MfError):
        mf.Policy.load(bad)
    P.close()
    Q.close()


def test_learned_requires_attached_policy(mf):
    A = mf.synth_laplace2d(32, 32)
    M = mf.Matrix(A)
    with pytest.raises(mf.MfError):
        M.solve_host(A.matvec(np.ones(A.n_rows)), policy="learned")
    M.close()


@pytest.fixture(scope="module")
def trained(mf, torch):
    """A policy trained on traces of FP64 solves of random SPD systems whose
    rows mix magnitudes over 8 decades (2000 rows, seeds 1000..1007): the
    tiles of small entries are the ones an accuracy-preserving label may
    demote."""
    P = mf.Policy(seed=1)
    total = 0
    for seed in range(1000, 1008):
        A = mf.synth_random_spd(seed, 2000)
        xs = mf.synth_xstar(seed, A.n_rows)
        b = torch.tensor(A.matvec(xs), dtype=torch.float64, device="cuda")
        M = mf.Matrix(A)
        total = P.collect(M, b.data_ptr(), checkpoint_every=20, sample_stride=2, max_samples=1 << 22)
        torch.cuda.synchronize()
        M.close()
    counts = P.label_counts()
    l0, l1 = P.train(epochs=20, batch=1024, lr=3e-3, seed=7)
    return P, total, counts, l0, l1


def test_policy_collect_and_train(trained):
    P, total, counts, l0, l1 = trained
    assert total > 1000 and counts.sum() == total
    assert np.count_nonzero(counts) >= 2, counts
    assert l1 < l0, (l0, l1)


def test_learned_policy_gain_over_static(mf, trained):
    """An unseen system (seed 2000, 4000 rows): the LEARNED policy reaches the
    1e-10 FP64 true relative residual like the STATIC value-range policy
    (the method without the network) and moves fewer bytes: the network
    demotes tiles whose contribution is below the rows' FP32 rounding."""
    P = trained[0]
    A = mf.synth_random_spd(2000, 4000)
    xs = mf.synth_xstar(2000, A.n_rows)
    b = A.matvec(xs)
    M = mf.Matrix(A)
    M.attach_policy(P)
    x, rep = M.solve_host(b, tol=1e-10, maxiter=50000, policy="learned")
    assert rep.status == 0, rep.as_dict()
    assert rep.relres_true <= 1e-10 * (1 + 1e-6)
    assert ol.oracle_true_relres(ol.Csr(A.n_rows, A.n_cols, A.rowptr, A.colidx, A.val), b, x) <= 2e-10
    xs_, reps = M.solve_host(b, tol=1e-10, maxiter=50000, policy="static")
    x64, rep64 = M.solve_host(b, tol=1e-10, maxiter=50000, policy="fp64")
    assert reps.status == 0 and rep64.status == 0
    per_it = lambda r: r.bytes_moved / max(1, r.iterations)
    assert per_it(rep) < per_it(reps) < per_it(rep64), (per_it(rep), per_it(reps), per_it(rep64))
    assert rep.bytes_moved < reps.bytes_moved, (rep.as_dict(), reps.as_dict())
    M.close()
