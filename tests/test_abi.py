"""The C-ABI library loads and exports every function include/*.h declares
(no GPU needed: nothing is called that touches a device)."""
import ctypes
import re
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
DECL = re.compile(r"^\s*(?:const\s+)?(?:unsigned\s+)?[A-Za-z_][\w]*\s*\**\s*\b([A-Za-z_]\w*)\s*\(([^;{}]*)\)\s*;",
                  re.M | re.S)


# headers whose functions live in the solver entry libraries rather than libmf.so
SOLVER_HEADERS = ("Mille-feuille-cg.h", "Mille-feuille-bicg.h")


def declared_functions(headers=None):
    names = set()
    for h in sorted((ROOT / "include").glob("*.h")):
        if headers is not None and h.name not in headers:
            continue
        if headers is None and h.name in SOLVER_HEADERS:
            continue
        text = re.sub(r"/\*.*?\*/", "", h.read_text(), flags=re.S)
        text = re.sub(r"//[^\n]*", "", text)
        for m in DECL.finditer(text):
            if m.group(1) not in ("if", "while", "for", "return", "sizeof"):
                names.add(m.group(1))
    return sorted(names)


def test_headers_declare_functions():
    names = declared_functions()
    assert "mf_matrix_create" in names and "mf_cg_solve" in names
    assert len(names) >= 20


@pytest.mark.parametrize("name", declared_functions())
def test_symbol_exported(mf, name):
    lib = mf.lib()
    assert hasattr(lib, name), f"{name} declared in include/ but not exported by libmf.so"


def test_version_and_error_strings(mf):
    assert b"sm_100a" in mf.lib().mf_version()
    assert isinstance(mf.lib().mf_last_error(), bytes)


def test_invalid_arguments_rejected_without_device(mf):
    # argument validation happens before any device call
    h = ctypes.c_void_p()
    st = mf.lib().mf_matrix_create(-1, 4, None, None, None, None, 0, None, ctypes.byref(h))
    assert st == 1  # MF_ERR_INVALID_ARG
    st = mf.lib().mf_matrix_export(None, b"tile_ptr", None, 0)
    assert st == 1

    # the multi-right-hand-side entry points: null handle, k outside 1..16
    L = mf.lib()
    reps = (mf.SolveReport * 16)()
    o = mf.solve_opts()
    assert L.mf_spmm(None, 4, None, 8, None, 8, None) == 1
    assert L.mf_cg_solve_multi(None, 4, None, 8, None, 8, ctypes.byref(o), reps, None) == 1
    assert L.mf_cg_solve_multi_host(None, 4, None, None, ctypes.byref(o), reps) == 1
    assert b"null" in L.mf_last_error()


def test_noalloc_residual_argument_checks_without_device(mf):
    """mf_residual_norm_noalloc rejects a null matrix, vector or output
    before it touches a device (the scratch lookup and the matrix's device
    check come after these)."""
    L = mf.lib()
    buf = (ctypes.c_double * 3)()
    p = ctypes.cast(buf, ctypes.c_void_p)
    for args in [(None, p, p, p), (p, None, p, p), (p, p, None, p), (p, p, p, None)]:
        assert L.mf_residual_norm_noalloc(*args, None) == 1  # MF_ERR_INVALID_ARG
        assert b"null argument" in L.mf_last_error()
    assert list(buf) == [0.0, 0.0, 0.0]


def test_tensor_core_spmm_rejects_null_without_device(mf):
    assert mf.lib().mf_spmm_f16(None, 4, None, 8, None, 8, 0, None, None) == 1


def test_device_mtx_reader_rejects_before_device(mf, tmp_path):
    """mf_matrix_create_mtx: a null path or handle pointer, a missing file
    and a malformed one are reported before any device work."""
    L = mf.lib()
    h = ctypes.c_void_p()
    assert L.mf_matrix_create_mtx(None, None, ctypes.byref(h), None) == 1
    assert L.mf_matrix_create_mtx(b"x.mtx", None, None, None) == 1
    assert L.mf_matrix_create_mtx(str(tmp_path / "missing.mtx").encode(), None, ctypes.byref(h), None) == 7
    bad = tmp_path / "bad.mtx"
    bad.write_text("%%MatrixMarket matrix coordinate real general\n3 3 2\n1 1 1.0\n")  # truncated
    assert L.mf_matrix_create_mtx(str(bad).encode(), None, ctypes.byref(h), None) == 7
    assert h.value is None


@pytest.mark.parametrize("libname", ["libmf_solvers.so", "libmf_solvers_mixed.so"])
def test_solver_entry_libraries_export_reference_names(mf, libname):
    """cg_solve_inc/sync/reduce and bicgstab/_sync/_inc, as declared in
    Mille-feuille-cg.h and Mille-feuille-bicg.h."""
    names = declared_functions(SOLVER_HEADERS)
    assert set(names) == {"cg_solve_inc", "cg_solve_sync", "cg_solve_reduce", "bicgstab", "bicgstab_sync",
                          "bicgstab_inc"}
    lib = ctypes.CDLL(str(ROOT / "mille-feuille_b200" / "lib" / libname))
    for n in names:
        assert hasattr(lib, n), n


def test_tile_matrix_layout_matches_reference_field_order():
    """Tile_matrix keeps the reference's 69 fields in order (src/format.h:14-86)
    and appends mf_handle."""
    import dropin

    f = dropin.tile_fields()
    assert len(f) == 70 and f[-1] == ("mf_handle", True)
    names = [n for n, _ in f]
    assert names[:6] == ["tilem", "tilen", "tilenum", "tile_ptr", "tile_columnidx", "tile_nnz"]
    assert names.index("csrsize") == names.index("csr_compressedIdx") + 1
    import oracle_lib

    root = oracle_lib.reference_root()
    ref = root / "src" / "format.h" if root is not None else None
    if ref is not None and ref.exists():
        body = ref.read_text()
        body = body[body.index("typedef struct\n{"): body.index("} Tile_matrix;")]
        import re as _re

        ref_names = _re.findall(r"\b([A-Za-z_]\w*);", body)
        assert ref_names == names[:-1]
