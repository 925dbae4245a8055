"""The C-ABI library loads and exports every function include/*.h declares
(no GPU needed: nothing is called that touches a device)."""
import ctypes
import re
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
DECL = re.compile(r"^\s*(?:const\s+)?(?:unsigned\s+)?[A-Za-z_][\w]*\s*\**\s*\b([A-Za-z_]\w*)\s*\(([^;{}]*)\)\s*;",
                  re.M | re.S)


def declared_functions():
    names = set()
    for h in sorted((ROOT / "include").glob("*.h")):
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
