"""GPU ingest encoder parity (prepare_compressed's per-chunk compress plus
MinMaxMeta::init_chunk, core/apps.cuh:149-255 and core/metadata.cuh:157-160):
a column encoded from HBM by gx_column_encode_device must be byte-identical to
the host encoder's column for the same values and options -- payload, block
directory, page / segment index, chunk min/max and block zone maps -- and the
device copies it leaves in HBM must decode and prune like an uploaded column."""
import ctypes as C

import numpy as np
import pytest

from golap_public_b200 import _lib as L
from golap_public_b200 import api, datagen, queries
from golap_public_b200._lib import GxError
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _wrap(handle, codec):
    col = api.Column.__new__(api.Column)
    col.handle = handle
    col.name = ""
    col.codec = codec
    return col


def _encode_pair(torch, values, codec, rpc=1_000_000, rpb=16384, S=128, rle=1, delta=1, bp=1):
    """The same values and options through the host encoder and the device encoder."""
    o = L.EncodeOpts()
    L.check(L.lib().gx_encode_opts_default(C.byref(o)))
    o.codec = api.CODECS[codec]
    o.rows_per_chunk = rpc
    o.rows_per_block = rpb
    o.lz4_segments = S
    o.lz4_min_match = L.GX_LZ4_LITERAL
    o.casc_rle, o.casc_delta, o.casc_bitpack = rle, delta, bp
    values = np.ascontiguousarray(values, dtype=np.int32)
    hh = C.c_void_p()
    L.check(L.lib().gx_column_encode(values.ctypes.data_as(C.c_void_p), len(values), C.byref(o), C.byref(hh)))
    dev = torch.from_numpy(values).cuda()
    hd = C.c_void_p()
    L.check(L.lib().gx_column_encode_device(C.c_void_p(dev.data_ptr()), len(values), C.byref(o), C.byref(hd),
                                            C.c_void_p(torch.cuda.current_stream().cuda_stream)))
    return _wrap(hh, codec), _wrap(hd, codec)


def _assert_identical(a, b, tag):
    ia, ib = a.info, b.info
    for f in ("n_rows", "comp_bytes", "meta_bytes", "codec", "rows_per_chunk", "rows_per_block", "n_chunks",
              "blocks_per_chunk", "n_blocks", "lz4_segments"):
        assert getattr(ia, f) == getattr(ib, f), (tag, f)
    assert ib.on_device == 1, tag
    assert np.array_equal(a.blocks(), b.blocks()), tag
    assert np.array_equal(a.seg_index(), b.seg_index()), tag
    for x, y in zip(a.minmax(), b.minmax()):
        assert np.array_equal(x, y), tag
    for x, y in zip(a.block_minmax(), b.block_minmax()):
        assert np.array_equal(x, y), tag
    pa, pb = a.payload_view(), b.payload_view()
    assert pa.shape == pb.shape, tag
    if not np.array_equal(pa, pb):
        bad = np.flatnonzero(pa != pb)
        raise AssertionError(f"{tag}: {bad.size} payload bytes differ, first at {bad[0]}")


def _distributions(n, seed):
    rng = np.random.default_rng(seed)
    f = datagen.fact_q1(n, True)
    runs = np.repeat(rng.integers(-1000, 1000, n // 7 + 1), 7)[:n]
    return {
        "date_sorted": f["date_key"],
        "discount": f["discount"],
        "random": rng.integers(-2**31, 2**31 - 1, n, dtype=np.int64).astype(np.int32),
        "runs": runs.astype(np.int32),
        # long runs of slowly rising values: RLE + delta pages
        "stairs": (np.arange(n, dtype=np.int64) // 300 * 5 - 90_000).astype(np.int32),
        "const": np.full(n, -3, np.int32),
        # wraps around int32: delta entries of the full 32-bit range
        "extremes": np.where(np.arange(n) % 2 == 0, 2**31 - 1, -2**31).astype(np.int32),
    }


CONFIGS = [
    # (codec, options): default chunks (1M rows, 62 blocks of 16384, the last one 576 rows)
    ("none", {}),
    ("lz4", {"S": 1}),
    ("lz4", {"S": 32}),
    ("lz4", {"S": 128}),
    ("cascaded", {}),
    ("cascaded", {"delta": 0}),
    ("cascaded", {"rle": 0}),
    ("cascaded", {"bp": 0}),
    ("cascaded", {"rle": 0, "delta": 0, "bp": 0}),
    # ragged layouts: short chunks, blocks that are not whole pages or segments
    ("cascaded", {"rpc": 50_000, "rpb": 3000}),
    ("cascaded", {"rpc": 7_001, "rpb": 2048}),
    ("lz4", {"rpc": 10_000, "rpb": 4096, "S": 4}),
    ("lz4", {"rpc": 70_000, "rpb": 16384, "S": 128}),
    ("none", {"rpc": 2_500, "rpb": 1000}),
]


@pytest.mark.parametrize("codec,opts", CONFIGS, ids=[f"{c}-{'-'.join(f'{k}{v}' for k, v in o.items())}"
                                                     for c, o in CONFIGS])
def test_device_encode_byte_identical(cuda, codec, opts):
    for name, v in _distributions(2_345_679, 5).items():
        a, b = _encode_pair(cuda, v, codec, **opts)
        _assert_identical(a, b, (codec, opts, name))


@pytest.mark.parametrize("n", [1, 2, 3, 4, 5, 17, 2047, 2048, 2049, 16383, 16385])
def test_device_encode_tiny(cuda, n):
    rng = np.random.default_rng(n)
    v = rng.integers(-50, 50, n).astype(np.int32)
    for codec, opts in (("none", {}), ("lz4", {"S": 1}), ("lz4", {"S": 128}), ("cascaded", {}),
                        ("cascaded", {"rpb": 3000, "rpc": 4000})):
        a, b = _encode_pair(cuda, v, codec, **opts)
        _assert_identical(a, b, (codec, opts, n))


def test_device_encode_max_runs(cuda):
    # pages with exactly the RLE run limit, one run more, and every row its own run
    lim = 512
    page = 2048
    over = np.concatenate([np.repeat(np.arange(lim - 1), 4), [9000, 9000, 9001, 9001]])  # lim + 1 runs
    v = np.concatenate([np.repeat(np.arange(lim), page // lim), over, np.arange(page)]).astype(np.int32)
    assert len(v) == 3 * page
    v = np.tile(v, 20)
    for opts in ({}, {"delta": 0}, {"bp": 0}):
        a, b = _encode_pair(cuda, v, "cascaded", **opts)
        _assert_identical(a, b, opts)


def test_device_encoded_columns_decode_and_prune(cuda):
    torch = cuda
    f = datagen.fact_q1(3_000_000, True)
    dd = datagen.date_dim()
    codecs = {"date_key": "cascaded", "discount": "lz4", "quantity": "none", "extended_price": "lz4"}
    cols = {k: api.Column.from_device(torch.from_numpy(v).cuda(), codecs[k], lz4_segments=128, name=k)
            for k, v in f.items()}
    for k, c in cols.items():
        out = torch.full((len(f[k]),), -7, dtype=torch.int32, device="cuda")
        api.ChunkDecompressor(c).chunks(0, c.info.n_chunks, out)
        api.scan_check()
        assert np.array_equal(out.cpu().numpy(), f[k]), k
    fact = queries.FactTable(cols, len(f["date_key"]))
    ok = dd["d_yearmonthnum"] == 199401
    q = queries.Q1Query(fact, dd, ok, 19940101, 19940131, 4, 6, 26, 35, prune=True)
    want = O.q1(f["date_key"], f["discount"], f["quantity"], f["extended_price"], dd["d_key"], ok, 4, 6, 26, 35)
    assert q.run() == want


def test_device_encode_rejects(cuda):
    torch = cuda
    v = torch.arange(1000, dtype=torch.int32, device="cuda")
    o = L.EncodeOpts()
    L.check(L.lib().gx_encode_opts_default(C.byref(o)))
    o.codec = L.GX_CODEC_LZ4
    o.lz4_min_match = 0  # match-finding policies stay on the host encoder
    h = C.c_void_p()
    s = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    assert L.lib().gx_column_encode_device(C.c_void_p(v.data_ptr()), 1000, C.byref(o), C.byref(h), s) == \
        L.GX_ERR_INVALID
    o.lz4_min_match = L.GX_LZ4_LITERAL
    assert L.lib().gx_column_encode_device(C.c_void_p(v.data_ptr()), 0, C.byref(o), C.byref(h), s) == \
        L.GX_ERR_INVALID
    o.rows_per_block = 16385
    assert L.lib().gx_column_encode_device(C.c_void_p(v.data_ptr()), 1000, C.byref(o), C.byref(h), s) == \
        L.GX_ERR_INVALID
    with pytest.raises(TypeError):
        api.Column.from_device(v.to(torch.int64))
    with pytest.raises(GxError):
        api.Column.from_device(v, "lz4", lz4_segments=3)


def test_device_encoded_host_copy_on_demand(cuda):
    # the payload stays in HBM until a caller needs the host copy; releasing the
    # device copy or moving the column to pinned host memory reads it back first
    torch = cuda
    rng = np.random.default_rng(11)
    v = rng.integers(0, 1 << 20, 1_500_001).astype(np.int32)
    host = api.Column(v, "lz4", lz4_segments=32, lz4_min_match=L.GX_LZ4_LITERAL)
    for step in ("release", "pinned", "payload"):
        col = api.Column.from_device(torch.from_numpy(v).cuda(), "lz4", lz4_segments=32)
        if step == "release":
            col.release_device()
            assert col.info.on_device == 0
            col.to_device("hbm")
        elif step == "pinned":
            col.to_device("pinned")
        else:
            assert np.array_equal(col.payload_view(), host.payload_view())
        out = torch.full((len(v),), -7, dtype=torch.int32, device="cuda")
        api.ChunkDecompressor(col).chunks(0, col.info.n_chunks, out)
        api.scan_check()
        assert np.array_equal(out.cpu().numpy(), v), step
        assert np.array_equal(col.payload_view(), host.payload_view()), step
        col.free()
