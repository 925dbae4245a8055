"""mf_matrix_create_mtx (Matrix Market file -> CSR built on the GPU -> tiled
matrix) against the host reader followed by mf_matrix_create: every tile
array bit for bit (the tile arrays keep each row's entry order, so the CSR
order is checked too), on general, symmetric, pattern, integer and
rectangular files, duplicates and unsorted columns included, a file large
enough for the parallel parser, an empty one, and the reference's add20.mtx
where the reference tree is present."""
import numpy as np
import pytest

import oracle_lib as ol

pytestmark = pytest.mark.gpu

ARRAYS = ["tile_ptr", "tile_columnidx", "tile_nnz", "blknnz", "blknnznnz", "csr_offset", "csrptr_offset",
          "Blockcsr_Val", "Blockcsr_Val_Low", "Tile_csr_Col", "Blockcsr_Ptr", "tile_class"]


def write_mtx(path, fmt, sym, m, n, entries):
    lines = [f"%%MatrixMarket matrix coordinate {fmt} {sym}", "% generated", f"{m} {n} {len(entries)}"]
    lines += entries
    path.write_text("\n".join(lines) + "\n")


def random_entries(rng, m, n, count, fmt, lower):
    i = rng.integers(1, m + 1, count)
    j = rng.integers(1, n + 1, count)
    if lower:
        i, j = np.maximum(i, j), np.minimum(i, j)
    out = []
    for a, b in zip(i, j):
        if fmt == "real":
            out.append(f"{a} {b} {rng.normal() * 10.0 ** rng.integers(-6, 6):.17g}")
        elif fmt == "integer":
            out.append(f"{a} {b} {int(rng.integers(-100, 100))}")
        elif fmt == "complex":
            out.append(f"{a} {b} {rng.normal():.17g} {rng.normal():.6g}")
        else:
            out.append(f"{a} {b}")
    return out


def same_matrix(mf, path):
    Md, sym_d = mf.matrix_from_mtx(path)
    A, sym_h = mf.read_matrix(path)
    Mh = mf.Matrix(A)
    try:
        assert sym_d == sym_h
        ia, ib = Md.info(), Mh.info()
        for f in ("rows", "cols", "nnz", "tilem", "tilen", "tilenum"):
            assert getattr(ia, f) == getattr(ib, f), f
        for name in ARRAYS:
            a, b = Md.export(name), Mh.export(name)
            assert a.dtype == b.dtype and np.array_equal(a.view(np.uint8), b.view(np.uint8)), name
        return ia
    finally:
        Md.close()
        Mh.close()


@pytest.mark.parametrize("fmt,sym,m,n,count", [
    ("real", "general", 3000, 3000, 40000),
    ("real", "symmetric", 2500, 2500, 30000),
    ("pattern", "symmetric", 1000, 1000, 8000),
    ("integer", "general", 777, 777, 9000),
    ("complex", "hermitian", 900, 900, 7000),  # real parts
    ("real", "general", 1200, 900, 15000),   # rectangular
])
def test_device_csr_equals_host_csr(mf, tmp_path, fmt, sym, m, n, count):
    rng = np.random.default_rng(count)
    ents = random_entries(rng, m, n, count, fmt, lower=(sym != "general"))
    ents += ents[:50]  # duplicate entries: kept, in file order
    f = tmp_path / "m.mtx"
    write_mtx(f, fmt, sym, m, n, ents)
    info = same_matrix(mf, f)
    assert info.nnz >= count


def test_device_csr_large_file(mf, tmp_path):
    """300,000 entries: parsed by the host threads, the CSR on the GPU."""
    rng = np.random.default_rng(3)
    m = 40000
    i = rng.integers(1, m + 1, 300000)
    j = rng.integers(1, m + 1, 300000)
    i, j = np.maximum(i, j), np.minimum(i, j)
    v = rng.normal(size=300000)
    f = tmp_path / "big.mtx"
    with open(f, "w") as fh:
        fh.write(f"%%MatrixMarket matrix coordinate real symmetric\n{m} {m} {len(v)}\n")
        fh.writelines(f"{a} {b} {x:.17g}\n" for a, b, x in zip(i, j, v))
    same_matrix(mf, f)


def test_device_csr_empty_and_errors(mf, tmp_path):
    f = tmp_path / "e.mtx"
    write_mtx(f, "real", "general", 40, 40, [])
    info = same_matrix(mf, f)
    assert info.nnz == 0
    with pytest.raises(mf.MfError) as e:
        mf.matrix_from_mtx(tmp_path / "missing.mtx")
    assert e.value.status == 7  # MF_ERR_IO
    bad = tmp_path / "bad.mtx"
    write_mtx(bad, "real", "general", 4, 4, ["1 1 1.0", "5 1 2.0"])  # row out of range
    with pytest.raises(mf.MfError) as e:
        mf.matrix_from_mtx(bad)
    assert e.value.status == 7


def test_device_csr_add20(mf):
    root = ol.reference_root()
    f = root / "test" / "add20.mtx" if root is not None else None
    if f is None or not f.exists():
        pytest.skip("reference tree not present")
    same_matrix(mf, f)
