"""Host encoder (libgx.so, no GPU needed) against the CPU checkers.

Every encoded block must decode, with the oracle and with system liblz4
(an independent LZ4 implementation), to exactly the input values; segmented
LZ4 blocks must also decode segment by segment from their side index.
Mirrors the round-trip checks of core/test/comp_tests.cu:18-59 and the
decompressed-value comparison of core/test/apps_tests.cu:244-348.
"""
import ctypes as C

import numpy as np
import pytest

from golap_public_b200 import api, datagen
from golap_public_b200 import _lib as L
from golap_public_b200._lib import GxError
from oracle import oracle as O

_lz4 = C.CDLL("liblz4.so.1")
_lz4.LZ4_decompress_safe.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_int]
_lz4.LZ4_decompress_safe.restype = C.c_int


def _slots(col, rows_per_chunk, n):
    info = col.info
    bpc = info.blocks_per_chunk
    for s in range(info.n_chunks * bpc):
        c, j = divmod(s, bpc)
        r0 = c * rows_per_chunk + j * info.rows_per_block
        r1 = min(n, (c + 1) * rows_per_chunk)
        if r0 < r1:
            yield s, r0, min(info.rows_per_block, r1 - r0)


def _first_literal(blk):
    """Offset of the first literal byte of an LZ4 block that opens with literals, else None."""
    if len(blk) == 0 or (blk[0] >> 4) == 0:
        return None
    p = 1
    if (blk[0] >> 4) == 15:
        while blk[p] == 255:
            p += 1
        p += 1
    return p


def _check_alignment(codec, off, blk):
    if codec == "lz4":
        # an LZ4 block that opens with literals is placed so that its first
        # literal byte is 16-byte aligned (row tiles of a literal run are then
        # aligned byte ranges); other blocks may start anywhere
        lit = _first_literal(blk)
        assert lit is None or (off + lit) % 16 == 0
    else:
        assert off % 16 == 0


def _check_pages(blk, ent, rows):
    """Cascaded block: the page table in the stream equals the side index; pages are 16-byte aligned."""
    n_pages, page_rows = (int(x) for x in blk[:8].view(np.uint32))
    assert page_rows == 2048 and n_pages == -(-rows // 2048)
    offs = blk[8:8 + 4 * (n_pages + 1)].view(np.uint32).astype(np.int64)
    assert offs[-1] == len(blk)
    for p in range(n_pages):
        assert offs[p] % 16 == 0
        assert int(ent[2 * p]) == offs[p] and int(ent[2 * p + 1]) == offs[p + 1] - offs[p]


def roundtrip(vals, codec, rows_per_chunk=100_000, rows_per_block=16384, S=32, **kw):
    col = api.Column(vals, codec, rows_per_chunk=rows_per_chunk, rows_per_block=rows_per_block, lz4_segments=S, **kw)
    info = col.info
    pl, blocks, seg = col.payload(), col.blocks(), col.seg_index()
    assert info.n_rows == len(vals)
    assert len(blocks) == info.n_blocks
    mins, maxs = col.minmax()
    em, ex = O.chunk_minmax(np.ascontiguousarray(vals, np.int32), rows_per_chunk)
    assert np.array_equal(mins, em) and np.array_equal(maxs, ex)
    for k, (s, r0, rows) in enumerate(_slots(col, rows_per_chunk, len(vals))):
        off, size, used, tuples = (int(x) for x in blocks[k])
        assert tuples == rows and size >= used
        blk = pl[off:off + used]
        _check_alignment(codec, off, blk)
        want = np.ascontiguousarray(vals[r0:r0 + rows], np.int32)
        if codec == "lz4":
            got = O.lz4_decode(blk, rows * 4)
            assert got is not None and np.array_equal(got.view(np.int32), want)
            ref = np.zeros(rows * 4, np.uint8)
            assert _lz4.LZ4_decompress_safe(blk.ctypes.data, ref.ctypes.data, used, rows * 4) == rows * 4
            assert np.array_equal(ref.view(np.int32), want)
            if S > 1:
                ent = np.ascontiguousarray(seg[2 * S * s: 2 * S * (s + 1)])
                rc = O.lib().or_lz4_check_segments(O._ptr(blk), used, O._ptr(ent), S, rows_per_block // S, rows,
                                                   O._ptr(want.view(np.uint8)))
                assert rc == 0, f"segment {rc - 1} of slot {s}"
        elif codec == "cascaded":
            got = O.casc_decode(blk, rows)
            assert got is not None and np.array_equal(got, want)
            pages = -(-rows_per_block // 2048)
            _check_pages(blk, seg[2 * pages * s: 2 * pages * (s + 1)], rows)
        else:
            assert np.array_equal(blk.view(np.int32), want)
    return col


CODECS = [("lz4", 32), ("lz4", 1), ("lz4", 128), ("lz4", 2), ("cascaded", 1), ("none", 1)]


@pytest.mark.parametrize("codec,S", CODECS)
@pytest.mark.parametrize("kind", ["sorted_date", "discount", "quantity", "price", "random", "constant", "negative"])
def test_roundtrip_distributions(codec, S, kind):
    rng = np.random.default_rng(hash(kind) % 2**32)
    n = 250_000
    if kind == "sorted_date":
        v = datagen.fact_q1(n, True)["date_key"]
    elif kind == "discount":
        v = rng.integers(0, 11, n, dtype=np.int32)
    elif kind == "quantity":
        v = rng.integers(1, 51, n, dtype=np.int32)
    elif kind == "price":
        v = rng.integers(90_000, 10_494_951, n, dtype=np.int32)
    elif kind == "random":
        v = rng.integers(-2**31, 2**31 - 1, n, dtype=np.int64).astype(np.int32)
    elif kind == "constant":
        v = np.full(n, 7, np.int32)
    else:
        v = -rng.integers(0, 1000, n, dtype=np.int32) * 1000
    roundtrip(v, codec, S=S)


@pytest.mark.parametrize("codec,S", CODECS)
@pytest.mark.parametrize("n", [1, 2, 3, 5, 31, 577, 16384, 16385, 100_001])
def test_roundtrip_ragged_sizes(codec, S, n):
    rng = np.random.default_rng(n)
    v = rng.integers(0, 5, n, dtype=np.int32)
    roundtrip(v, codec, S=S)


@pytest.mark.parametrize("codec", ["lz4", "cascaded", "none"])
def test_roundtrip_extremes(codec):
    v = np.array([np.iinfo(np.int32).min, np.iinfo(np.int32).max, 0, -1, 1] * 5000, np.int32)
    roundtrip(v, codec)
    roundtrip(np.sort(v), codec)


def test_small_blocks_and_chunks():
    rng = np.random.default_rng(3)
    v = rng.integers(0, 3, 10_000, dtype=np.int32)
    for rpc, rpb, S in [(1000, 256, 8), (999, 128, 4), (10_000, 4096, 128), (1, 1, 1)]:
        for codec in ("lz4", "cascaded"):
            roundtrip(v[:3000] if rpb == 1 else v, codec, rows_per_chunk=rpc, rows_per_block=rpb,
                      S=S if codec == "lz4" else 1)


def test_lz4_min_match_and_depth_knobs():
    rng = np.random.default_rng(5)
    v = rng.integers(0, 11, 100_000, dtype=np.int32)
    sizes = []
    for mm in (4, 8, 16):
        sizes.append(roundtrip(v, "lz4", lz4_min_match=mm).info.comp_bytes)
    assert sizes[0] <= sizes[1] <= sizes[2]
    roundtrip(v, "lz4", lz4_search_depth=1)


def test_invalid_encode_options():
    v = np.arange(100, dtype=np.int32)
    with pytest.raises(GxError):
        api.Column(v, "lz4", lz4_segments=3)  # not a power of two
    with pytest.raises(GxError):
        api.Column(v, "lz4", rows_per_block=20000)  # > 64 KiB of int32
    with pytest.raises(GxError):
        api.Column(v, "lz4", lz4_min_match=6)
    with pytest.raises(GxError):
        api.Column(v[:0], "lz4")


def test_block_directory_matches_reference_blockinfo_layout():
    # BlockInfo{offset,size,payload,tuples} (core/comp.cuh:23-32); chunks of
    # 250k/250k/... rows as in core/test/apps_tests.cu:67-242.
    v = np.arange(1_000_000, dtype=np.int32)
    col = api.Column(v, "lz4", rows_per_chunk=250_000)
    b = col.blocks()
    info = col.info
    assert info.n_chunks == 4 and info.blocks_per_chunk == 16
    assert int(b[:, 3].sum()) == 1_000_000
    pl = col.payload()
    for off, _, used, _ in b:
        _check_alignment("lz4", int(off), pl[int(off):int(off) + int(used)])
    assert np.all(b[1:, 0] >= b[:-1, 0] + b[:-1, 2])


@pytest.mark.parametrize("S", [1, 4, 32, 128])
def test_literal_policy_blocks(S):
    # lz4_min_match = GX_LZ4_LITERAL (the GPU ingest encoder's LZ4 policy): every
    # block is one literal run that liblz4 and the oracle decode, placed so that
    # its first literal byte is 16-byte aligned
    rng = np.random.default_rng(S)
    for v in (rng.integers(0, 11, 250_001).astype(np.int32), np.arange(3, dtype=np.int32),
              np.full(70_000, 5, np.int32)):
        col = roundtrip(v, "lz4", S=S, lz4_min_match=L.GX_LZ4_LITERAL)
        pl, blocks = col.payload(), col.blocks()
        for off, size, used, tuples in blocks.astype(np.int64):
            lit = _first_literal(pl[off:off + used])
            assert lit is not None and used == lit + 4 * tuples
