"""The C-ABI library loads and exports every entry point include/*.h declares
(no compute calls: this runs without a GPU)."""
import ctypes as C
import re
import subprocess
from pathlib import Path

import numpy as np
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


def test_device_encoder_argument_checks():
    # the GPU ingest encoder rejects bad arguments before touching the device
    lib = L.lib()
    o = L.EncodeOpts()
    assert lib.gx_encode_opts_default(C.byref(o)) == 0
    h = C.c_void_p()
    fake = C.c_void_p(0x1000)  # never dereferenced: every call below fails its argument checks
    assert lib.gx_column_encode_device(None, 10, C.byref(o), C.byref(h), None) == L.GX_ERR_INVALID
    assert lib.gx_column_encode_device(fake, 0, C.byref(o), C.byref(h), None) == L.GX_ERR_INVALID
    o.codec = L.GX_CODEC_LZ4
    o.lz4_min_match = 0  # match-finding LZ4 stays on the host encoder
    assert lib.gx_column_encode_device(fake, 10, C.byref(o), C.byref(h), None) == L.GX_ERR_INVALID
    assert "GX_LZ4_LITERAL" in L.last_error()
    o.lz4_min_match = L.GX_LZ4_LITERAL
    o.lz4_segments = 3
    assert lib.gx_column_encode_device(fake, 10, C.byref(o), C.byref(h), None) == L.GX_ERR_INVALID
    o.lz4_segments = 128
    o.rows_per_block = 0
    assert lib.gx_column_encode_device(fake, 10, C.byref(o), C.byref(h), None) == L.GX_ERR_INVALID
    o.rows_per_block = 16384
    o.codec = 7
    assert lib.gx_column_encode_device(fake, 10, C.byref(o), C.byref(h), None) == L.GX_ERR_INVALID


def test_device_encoder_wants_a_cuda_tensor():
    import torch

    from golap_public_b200 import api

    with pytest.raises(TypeError):
        api.Column.from_device(torch.arange(10, dtype=torch.int32))  # a host tensor
    with pytest.raises(TypeError):
        api.Column.from_device(np.arange(10, dtype=np.int32))


def test_block_zone_maps_of_the_host_encoder():
    # per-block-slot min/max, absent slots of a short chunk hold the empty range
    from golap_public_b200 import api

    rng = np.random.default_rng(3)
    v = rng.integers(-1000, 1000, 25_001).astype(np.int32)
    col = api.Column(v, "cascaded", rows_per_chunk=10_000, rows_per_block=3_000)
    mins, maxs = col.block_minmax()
    i = col.info
    assert len(mins) == i.n_chunks * i.blocks_per_chunk == 3 * 4
    for c in range(i.n_chunks):
        for j in range(i.blocks_per_chunk):
            lo = c * 10_000 + j * 3_000
            hi = min(c * 10_000 + min((j + 1) * 3_000, 10_000), len(v))
            s = c * i.blocks_per_chunk + j
            if lo >= hi:
                assert (mins[s], maxs[s]) == (np.iinfo(np.int32).max, np.iinfo(np.int32).min)
            else:
                assert (mins[s], maxs[s]) == (v[lo:hi].min(), v[lo:hi].max())
    cm, cx = col.minmax()
    assert list(cm) == [v[k:k + 10_000].min() for k in range(0, len(v), 10_000)]
    assert list(cx) == [v[k:k + 10_000].max() for k in range(0, len(v), 10_000)]
