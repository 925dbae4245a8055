"""The seeded generators of the benchmark configurations (csrc/synth.cpp),
pinned bit for bit against their Python restatement (tests/synth_mirror.py)
at small sizes."""
import numpy as np
import pytest

import synth_mirror as sm


def _same(A, ref):
    rp, ci, v = ref
    assert np.array_equal(A.rowptr, rp) and np.array_equal(A.colidx, ci)
    assert np.array_equal(A.val.view(np.uint64), v.view(np.uint64))


@pytest.mark.parametrize("seed,stream", [(0, 1), (1, 2), (611, 5), (2 ** 40 + 7, 7)])
def test_rng_matches_mirror(mf, seed, stream):
    for i in (0, 1, 2, 1000, 123456):
        assert mf.lib().mf_rng_u01(seed, stream, i) == sm.u01(sm.stream_key(seed, stream), i)
        assert mf.lib().mf_rng_normal(seed, stream, i) == sm.normal01(sm.stream_key(seed, stream), i)


def test_xstar(mf):
    assert np.array_equal(mf.synth_xstar(3, 500), sm.xstar(3, 500))


def test_laplace2d(mf):
    _same(mf.synth_laplace2d(12, 9), sm.laplace2d(12, 9))


def test_poisson3d_scaled(mf):
    _same(mf.synth_poisson3d_scaled(7, 1), sm.poisson3d_scaled(7, 1))


def test_convdiff3d(mf):
    _same(mf.synth_convdiff3d(6), sm.convdiff3d(6))


@pytest.mark.parametrize("seed", [100, 101, 611])
def test_random_spd(mf, seed):
    assert mf.lib().mf_synth_random_spd_size(seed) == sm.random_spd_size(seed)
    _same(mf.synth_random_spd(seed, 300), sm.random_spd(seed, 300))


def test_aniso3d(mf):
    _same(mf.synth_aniso3d(6, 3), sm.aniso3d(6, 3))


@pytest.mark.parametrize("seed,n", [(100, 0), (101, 0), (3001, 2000), (611, 0)])
def test_oracle_random_spd_matches_library(mf, seed, n):
    """The oracle's C restatement of the random SPD generator (used by the
    CPU baseline, which loads no product library) equals the library's."""
    import oracle_lib as ol

    A = mf.synth_random_spd(seed, n)
    B = ol.oracle_random_spd(seed, n)
    assert A.n_rows == B.n_rows
    assert np.array_equal(A.rowptr, B.rowptr) and np.array_equal(A.colidx, B.colidx)
    assert np.array_equal(A.val, B.val)
    assert np.array_equal(mf.synth_xstar(seed, A.n_rows), ol.oracle_xstar(seed, A.n_rows))
    assert ol.oracle().orc_random_spd_size(seed) == mf.lib().mf_synth_random_spd_size(seed)
