"""Trains the learned precision policies on plain FP64 CG traces.

    python mille-feuille_b200/train_policy.py --grid 64 --instances 200 --seed0 1000 \
        --out aniso64.mfpol
    python mille-feuille_b200/train_policy.py --family batched --instances 64 --seed0 2000 \
        --every 25 --stride 4 --out randspd_batched.mfpol

Family batched: the chunk policy of the batched solver.  The instances are
random SPD systems of the batched configuration's family (n ~
log-uniform[1k, 64k], seeds seed0 ...), solved together by one plain FP64
batched solve that samples (chunk features, label) every `--every`
iterations (mf_batch_policy_collect).

Each instance is a seeded 3D anisotropic diffusion system (lognormal
coefficients, log-sigma 2, correlation length 8 cells, k_z = 100 k; family
aniso) or a random SPD system with row scales 10^U[-4,4] (family randspd),
with b = A x*; its FP64 CG solve to 1e-10 is traced every `--every` iterations and
about one tile in `--stride` becomes a (features, label) sample
(mf_policy_collect).  The network is then trained on the GPU with Adam
(mf_policy_train) and saved (mf_policy_save).
"""
from __future__ import annotations

import argparse
import json
import sys
import time
from pathlib import Path


def _package():
    here = Path(__file__).resolve().parent
    sys.path.insert(0, str(here.parent))
    import __graft_entry__ as ge

    return ge.load_package()


def make_system(mf, family, size, seed):
    """One training system: 'aniso' (3D anisotropic diffusion, grid `size`) or
    'randspd' (random SPD with row scales 10^U[-4,4], `size` rows)."""
    if family == "aniso":
        return mf.synth_aniso3d(size, seed)
    return mf.synth_random_spd(seed, size)


def train(grid=64, instances=200, seed0=1000, every=500, stride=256, max_samples=1 << 23, epochs=5, batch=4096,
          lr=3e-3, init_seed=1, out=None, log=print, family="aniso"):
    import torch

    mf = _package()
    P = mf.Policy(seed=init_seed)
    t0 = time.time()
    n = 0
    if family == "batched":
        systems = [mf.synth_random_spd(seed0 + k) for k in range(instances)]
        B = mf.Batch(systems)
        b = B.stack([A.matvec(mf.synth_xstar(seed0 + k, A.n_rows)) for k, A in enumerate(systems)])
        db = torch.from_numpy(b).cuda()
        n = B.collect(P, db.data_ptr(), checkpoint_every=every, sample_stride=stride, max_samples=max_samples)
        torch.cuda.synchronize()
        B.close()
        grid = int(sum(A.n_rows for A in systems))
        instances_done = instances
    else:
        instances_done = 0
    for k in range(instances_done, instances):
        seed = seed0 + k
        A = make_system(mf, family, grid, seed)
        b = torch.tensor(A.matvec(mf.synth_xstar(seed, A.n_rows)), dtype=torch.float64, device="cuda")
        M = mf.Matrix(A)
        n = P.collect(M, b.data_ptr(), checkpoint_every=every, sample_stride=stride, max_samples=max_samples)
        torch.cuda.synchronize()
        M.close()
        if (k + 1) % 20 == 0:
            log(f"instances {k + 1}/{instances}: {n} samples, {time.time() - t0:.1f} s")
    counts = P.label_counts()
    t1 = time.time()
    l0, l1 = P.train(epochs=epochs, batch=batch, lr=lr, seed=7)
    summary = {"family": family, "instances": instances, "size": grid, "seed0": seed0, "samples": int(n),
               "labels": [int(c) for c in counts], "loss_first": l0, "loss_last": l1,
               "collect_s": t1 - t0, "train_s": time.time() - t1}
    if out:
        P.save(out)
    return P, summary


def main():
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--family", choices=["aniso", "randspd", "batched"], default="aniso")
    ap.add_argument("--grid", type=int, default=64, help="grid side (aniso) or rows (randspd)")
    ap.add_argument("--instances", type=int, default=200)
    ap.add_argument("--seed0", type=int, default=1000)
    ap.add_argument("--every", type=int, default=500)
    ap.add_argument("--stride", type=int, default=256)
    ap.add_argument("--epochs", type=int, default=5)
    ap.add_argument("--batch", type=int, default=4096)
    ap.add_argument("--lr", type=float, default=3e-3)
    ap.add_argument("--out", required=True)
    a = ap.parse_args()
    _, summary = train(a.grid, a.instances, a.seed0, a.every, a.stride, 1 << 23, a.epochs, a.batch, a.lr, 1, a.out,
                       log=lambda s: print(s, flush=True), family=a.family)
    print(json.dumps(summary))


if __name__ == "__main__":
    main()
