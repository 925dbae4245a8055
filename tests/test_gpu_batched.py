"""Batched CG over many uneven random SPD systems (needs a B200): every
system against the FP64 CPU oracle, graph replay, autotuner, mixed policy."""
import numpy as np
import pytest
import torch

import oracle_lib as ol

pytestmark = pytest.mark.gpu


def _systems(mf, count, lo=800, hi=3000):
    rng = np.random.default_rng(7)
    sizes = rng.integers(lo, hi, size=count)
    return [mf.synth_random_spd(100 + k, int(sizes[k])) for k in range(count)]


def _rhs(mf, systems):
    xs = [mf.synth_xstar(100 + k, A.n_rows) for k, A in enumerate(systems)]
    bs = [A.matvec(x) for A, x in zip(systems, xs)]
    return xs, bs


@pytest.fixture(scope="module")
def batch(mf):
    systems = _systems(mf, 12)
    B = mf.Batch(systems)
    yield B, systems
    B.close()


@pytest.mark.parametrize("policy", ["fp64", "static"])
def test_batched_matches_oracle(mf, batch, policy):
    B, systems = batch
    xs, bs = _rhs(mf, systems)
    db = torch.from_numpy(B.stack(bs)).cuda()
    dx = torch.zeros_like(db)
    st, rep = B.solve_device(db.data_ptr(), dx.data_ptr(), use_graph=1, tol=1e-10, maxiter=20000, policy=policy)
    assert st == 0, rep.as_dict()
    assert rep.relres_true_max <= 1.2e-10, rep.as_dict()
    its, rrs = B.results()
    x = dx.cpu().numpy()
    for k, (A, b, xk) in enumerate(zip(systems, bs, B.split(x))):
        Ac = ol.Csr(A.n_rows, A.n_cols, A.rowptr, A.colidx, A.val)
        it_o, x_o, _ = ol.oracle_cg(Ac, b, 20000, 1e-10)
        assert ol.oracle_true_relres(Ac, b, xk) <= 1.2e-10
        err_o = np.max(np.abs(x_o - xs[k]))
        assert np.max(np.abs(xk - x_o)) <= 10 * err_o + 1e-9
        if policy == "fp64":
            assert abs(int(its[k]) - it_o) <= max(3, it_o // 20), (k, its[k], it_o)


def test_batched_graph_replay_and_determinism(mf, batch):
    B, systems = batch
    xs, bs = _rhs(mf, systems)
    db = torch.from_numpy(B.stack(bs)).cuda()
    dx1 = torch.zeros_like(db)
    st, r1 = B.solve_device(db.data_ptr(), dx1.data_ptr(), use_graph=1, tol=1e-10, maxiter=20000)
    st2, r2 = B.solve_device(db.data_ptr(), dx1.data_ptr(), use_graph=1, tol=1e-10, maxiter=20000)  # replay
    dx3 = torch.zeros_like(db)
    st3, r3 = B.solve_device(db.data_ptr(), dx3.data_ptr(), use_graph=0, tol=1e-10, maxiter=20000)
    assert st == st2 == st3 == 0
    assert r1.iterations_total == r2.iterations_total == r3.iterations_total
    assert torch.equal(dx1, dx3)


def test_batched_autotuner_picks_a_schedule(mf, batch):
    B, systems = batch
    xs, bs = _rhs(mf, systems)
    db = torch.from_numpy(B.stack(bs)).cuda()
    dx = torch.zeros_like(db)
    lanes, cluster = B.tune(db.data_ptr(), dx.data_ptr(), tol=1e-10, maxiter=20000)
    assert lanes in (4, 8, 16, 32) and cluster in (1, 2, 4, 8, 16)
    st, rep = B.solve_device(db.data_ptr(), dx.data_ptr(), use_graph=1, tol=1e-10, maxiter=20000)
    assert st == 0 and rep.lanes_per_row == lanes and rep.cluster_ctas == cluster


def test_batched_rejects_bad_input(mf):
    A = mf.synth_random_spd(100, 500)
    A.colidx[3] = 10**6
    with pytest.raises(mf.MfError):
        mf.Batch([A])
