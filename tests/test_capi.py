"""The C-ABI library loads and exports every entry point include/*.h declares
(no compute calls: this runs without a GPU)."""
import ctypes as C
import re
import subprocess
from pathlib import Path

import pytest

from golap_public_b200 import _lib as L

ROOT = Path(__file__).resolve().parent.parent


def declared_functions():
    names = set()
    for h in (ROOT / "include").glob("*.h"):
        text = re.sub(r"/\*.*?\*/", "", h.read_text(), flags=re.S)
        # prototypes only (declarations ending in ';'), not inline helpers
        names |= set(re.findall(r"\b(gx_[a-z0-9_]+)\s*\([^;{}]*\)\s*;", text))
    return names


def test_library_exports_all_declared_symbols():
    lib = C.CDLL(str(L.LIB_PATH))
    missing = [n for n in sorted(declared_functions()) if not hasattr(lib, n)]
    assert not missing, missing
    out = subprocess.run(["nm", "-D", "--defined-only", str(L.LIB_PATH)], capture_output=True, text=True).stdout
    exported = set(re.findall(r" T (gx_[a-z0-9_]+)", out))
    assert declared_functions() <= exported


def test_python_binding_covers_header():
    # every binding refers to a declared function, and every declared one is bound
    assert set(L.exported_symbols()) == declared_functions()


def test_status_strings_and_errors():
    lib = L.lib()
    assert lib.gx_status_str(0) == b"GX_OK"
    assert lib.gx_status_str(L.GX_ERR_CORRUPT) == b"GX_ERR_CORRUPT"
    assert lib.gx_version().startswith(b"gx")
    o = L.EncodeOpts()
    assert lib.gx_encode_opts_default(C.byref(o)) == 0
    assert o.rows_per_block == 16384 and o.lz4_segments == 128
    h = C.c_void_p()
    assert lib.gx_column_encode(None, 10, C.byref(o), C.byref(h)) == L.GX_ERR_INVALID
    assert "null" in L.last_error()
    assert lib.gx_hashtable_create(0, C.byref(h)) == L.GX_ERR_INVALID
    assert lib.gx_scan(None, None) == L.GX_ERR_INVALID
    with pytest.raises(L.GxError):
        L.check(L.GX_ERR_INVALID)


def test_product_has_no_oracle_dependency():
    out = subprocess.run(["ldd", str(L.LIB_PATH)], capture_output=True, text=True).stdout
    assert "oracle" not in out and "golapref" not in out
    src = "".join(p.read_text() for p in (ROOT / "golap_public_b200").rglob("*.py"))
    assert "import oracle" not in src and "from oracle" not in src
