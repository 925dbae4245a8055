"""Host logic of bench.py that needs no GPU: which committed ncu traffic
figure a bench line may carry, and the timing notes it reports."""
import json
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parent.parent
sys.path.insert(0, str(ROOT))

import bench  # noqa: E402


def test_traffic_only_for_the_captured_workload_and_policy():
    d = json.loads((ROOT / "profiles" / "ncu_traffic.json").read_text())
    for kernel, e in d.items():
        # a figure per iteration (persistent solves) or per launch (a batch,
        # one SpMV)
        key = "dram_bytes_per_iteration" if "dram_bytes_per_iteration" in e else "dram_bytes_per_launch"
        assert e[key] > 0 and e["workload"]
        got = bench.ncu_traffic(kernel, e["workload"], e["policy"] or "static")
        assert got is not None and got[key] == e[key]
        # the figure of one matrix and payload is not reused for another
        assert bench.ncu_traffic(kernel, "lap2d" if e["workload"] != "lap2d" else "poisson3d", e["policy"]) is None
        if e["policy"] is not None:  # a figure that depends on the precision policy
            other = "rule" if e["policy"] != "rule" else "static"
            assert bench.ncu_traffic(kernel, e["workload"], other) is None
    assert bench.ncu_traffic("k_no_such_kernel", "poisson3d", "static") is None


def test_l2_flush_is_larger_than_l2():
    assert bench.L2_FLUSH_BYTES >= 2 * 126 * 10**6
    assert "flushed" in bench.L2_NOTE


def test_batched_reference_baseline_runs_on_host():
    """The reference arm of the batched workload: the reference's own CPU
    code on a sample of the systems, scaled by the committed FP64 oracle
    iteration counts (no product library loaded in its workers)."""
    import pytest

    sys.path.insert(0, str(ROOT / "tests"))
    import oracle_lib as ol

    if ol.reference() is None:
        pytest.skip("reference CPU code not built")
    cpu = bench.CpuBatchReference(sample=2, budget_s=0.2, workers=2)
    try:
        t = cpu.measure()
    finally:
        cpu.close()
    assert t > 0 and len(cpu.systems) == 512 and cpu.cores == 2
    assert all(nnz > 0 and s > 0 for _, _, nnz, s in cpu.last)
    assert "512 systems" in cpu.describe() or "of the 512" in cpu.describe()


def test_batch_shards_are_disjoint_and_rank0_is_the_benchmark():
    n = 512
    shards = [bench.batch_seeds(r, n) for r in range(8)]
    assert shards[0] == list(range(100, 612))
    flat = [s for sh in shards for s in sh]
    assert len(set(flat)) == len(flat) == 8 * n
