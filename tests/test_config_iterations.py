"""The FP64 CPU oracle's iteration counts on configurations 1 and 2, which
bench.py uses to scale its CPU-baseline samples, recomputed and compared
with the committed fixture (tests/golden/config_iterations.json)."""
import json
from pathlib import Path

import pytest

import make_config_iterations_path  # noqa: F401  (puts tests/golden on the path)
import make_config_iterations as mci

GOLDEN = Path(__file__).resolve().parent / "golden" / "config_iterations.json"


@pytest.mark.parametrize("name", sorted(mci.CONFIGS))
def test_oracle_iterations_match_fixture(name):
    want = json.loads(GOLDEN.read_text())[name]
    got = mci.compute(name)
    assert got["iterations"] == want["iterations"]
    assert got["relres"] <= 1e-10 and got["n"] == want["n"] and got["nnz"] == want["nnz"]


def test_bench_reads_the_fixture():
    import bench

    d = json.loads(GOLDEN.read_text())
    assert bench.FP64_ITERS_ORACLE == d["poisson3d_scaled_128"]["iterations"]
    assert bench.oracle_iterations("lap2d") == d["laplace2d_128"]["iterations"]
