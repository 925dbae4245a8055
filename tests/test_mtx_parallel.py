"""The Matrix Market reader's parallel entry parser against its serial one
(MF_MTX_THREADS=1): the same arrays, bit for bit, on every value format, and
the serial parser's errors where a file is malformed.  Host only."""
import os
import subprocess
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

# each case runs in a child process: the thread count is read from the
# environment at every call, but the child keeps this process's environment
# untouched
CHILD = r"""
import sys, json
sys.path.insert(0, sys.argv[1])
import numpy as np
import __graft_entry__ as ge
mf = ge.load_package()
try:
    A = mf.read_matrix_market(sys.argv[2])
    print(json.dumps({"ok": 1, "rp": A.rowptr.tolist(), "ci": A.colidx.tolist(),
                      "v": A.val.view(np.uint64).tolist(), "shape": [A.n_rows, A.n_cols]}))
except mf.MfError as e:
    print(json.dumps({"ok": 0, "status": e.status, "msg": str(e)}))
"""


def read(path, threads):
    env = dict(os.environ, MF_MTX_THREADS=str(threads))
    p = subprocess.run([sys.executable, "-c", CHILD, ROOT, str(path)], capture_output=True, text=True, env=env,
                       timeout=120)
    assert p.returncode == 0, p.stderr
    import json

    return json.loads(p.stdout.strip().splitlines()[-1])


def write(path, header, lines, crlf=False):
    nl = "\r\n" if crlf else "\n"
    path.write_text(nl.join([header] + lines) + nl)


def entries(n, rng, fmt):
    i = rng.integers(1, n + 1, 3000)
    j = rng.integers(1, n + 1, 3000)
    out = []
    for a, b in zip(i, j):
        x = rng.normal() * 10.0 ** rng.integers(-30, 30)
        if fmt == "real":
            s = rng.choice([f"{x:.17g}", f"{x:+.6e}", f"{x:.3f}", repr(float(x))])
            out.append(f"{a} {b} {s}")
        elif fmt == "integer":
            out.append(f"{a} {b} {int(rng.integers(-1000, 1000))}")
        elif fmt == "complex":
            out.append(f"{a} {b} {x:.17g} {-x:.5g}")
        else:
            out.append(f"{a} {b}")
    return out


@pytest.mark.parametrize("fmt,sym,crlf", [("real", "general", False), ("real", "symmetric", True),
                                          ("integer", "general", False), ("complex", "hermitian", False),
                                          ("pattern", "symmetric", False)])
def test_parallel_equals_serial(tmp_path, fmt, sym, crlf):
    rng = np.random.default_rng(7)
    n = 500
    lines = entries(n, rng, fmt)
    if sym != "general":  # lower triangle, as symmetric files store it
        fixed = []
        for ln in lines:
            parts = ln.split()
            a, b = int(parts[0]), int(parts[1])
            fixed.append(" ".join([str(max(a, b)), str(min(a, b))] + parts[2:]))
        lines = fixed
    f = tmp_path / "m.mtx"
    write(f, f"%%MatrixMarket matrix coordinate {fmt} {sym}", ["% comment", f"{n} {n} {len(lines)}"] + lines,
          crlf=crlf)
    ref = read(f, 1)
    assert ref["ok"] == 1
    for t in (2, 3, 8):
        assert read(f, t) == ref


def test_entries_spanning_lines_fall_back(tmp_path):
    """Numbers of one entry on two lines: the pieces do not hold whole
    entries, so the reader parses serially (the same result)."""
    f = tmp_path / "m.mtx"
    write(f, "%%MatrixMarket matrix coordinate real general", ["4 4 4", "1 1", "2.5", "2 2 3.5", "3", "3 1.25",
                                                               "4 4 -1e-3"])
    ref = read(f, 1)
    assert ref["ok"] == 1 and ref["rp"] == [0, 1, 2, 3, 4]
    assert read(f, 4) == ref


@pytest.mark.parametrize("body,status", [(["3 3 3", "1 1 1.0", "2 2 2.0"], 7),
                                         (["3 3 2", "1 1 1.0", "4 2 2.0"], 7),
                                         (["3 3 2", "1 1 1.0", "2 2 x"], 7)])
def test_malformed_same_error(tmp_path, body, status):
    f = tmp_path / "m.mtx"
    write(f, "%%MatrixMarket matrix coordinate real general", body)
    ref = read(f, 1)
    assert ref["ok"] == 0 and ref["status"] == status
    assert read(f, 4) == ref
