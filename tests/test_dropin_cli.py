"""The reference-compatible CLIs on the host side (no GPU needed): usage
errors and the non-square early exit happen before any device call."""
import subprocess

import numpy as np
import pytest

import dropin
from oracle_lib import Csr

CLIS = ["main-cg", "main-cg-mixed", "main-bicg", "main-bicg-mixed"]


@pytest.mark.parametrize("cli", CLIS)
def test_cli_usage(cli):
    p = subprocess.run([str(dropin.BIN / cli)], capture_output=True, text=True, timeout=60)
    assert p.returncode == 1 and "usage" in p.stderr


@pytest.mark.parametrize("cli", CLIS)
def test_cli_missing_file(cli, tmp_path):
    p = subprocess.run([str(dropin.BIN / cli), str(tmp_path / "nope.mtx")], capture_output=True, text=True,
                       timeout=60)
    assert p.returncode == 1 and p.stderr.strip()


@pytest.mark.parametrize("cli,out", [("main-cg", "unequal\n"), ("main-cg-mixed", "")])
def test_cg_cli_rejects_non_square(cli, out, tmp_path):
    """src/main-cg.cu:1638-1642 prints "unequal"; the mixed driver returns
    silently (src/main-cg-mixed.cu:3014-3015)."""
    A = Csr(3, 4, np.array([0, 1, 2, 3], np.int32), np.array([0, 1, 3], np.int32), np.ones(3))
    f = tmp_path / "rect.mtx"
    dropin.write_mtx(f, A)
    p = subprocess.run([str(dropin.BIN / cli), str(f)], capture_output=True, text=True, timeout=60, cwd=tmp_path)
    assert p.returncode == 0 and p.stdout == out
