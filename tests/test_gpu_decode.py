"""GPU decompression parity (ChunkDecompressor::step, core/comp.cuh:171-195):
decoded device bytes must equal the encoder input exactly, for every codec,
segment count, ragged size and residency; LZ4 blocks made by liblz4 (the
reference's LZ4CPUManager::compress) must decode through the raw entry
point; corrupt streams must be reported, not fault."""
import ctypes as C
from pathlib import Path

import numpy as np
import pytest

from golap_public_b200 import _lib as L
from golap_public_b200 import api, datagen
from golap_public_b200._lib import GxError

pytestmark = pytest.mark.gpu
GOLDEN = Path(__file__).parent / "golden"


def _decode_all(col, torch):
    n = col.info.n_rows
    out = torch.full((n,), -7, dtype=torch.int32, device="cuda")
    api.ChunkDecompressor(col).chunks(0, col.info.n_chunks, out)
    api.scan_check()
    return out.cpu().numpy()


@pytest.mark.parametrize("codec,S", [("lz4", 32), ("lz4", 1), ("lz4", 128), ("lz4", 4), ("cascaded", 1), ("none", 1)])
def test_decompress_distributions(cuda, codec, S):
    f = datagen.fact_q1(2_500_000, True)
    rng = np.random.default_rng(1)
    cols = dict(f, random=rng.integers(-2**31, 2**31 - 1, 2_500_000, dtype=np.int64).astype(np.int32),
                const=np.full(2_500_000, -3, np.int32),
                # strictly increasing: cascaded picks delta without RLE (tile prefix sums)
                ramp=(np.arange(2_500_000, dtype=np.int64) * 3 + rng.integers(0, 3, 2_500_000) - 7).astype(np.int32))
    for name, v in cols.items():
        col = api.Column(v, codec, lz4_segments=S).to_device()
        got = _decode_all(col, cuda)
        assert np.array_equal(got, v), (codec, S, name)


@pytest.mark.parametrize("codec,S", [("lz4", 32), ("lz4", 1), ("cascaded", 1), ("none", 1)])
@pytest.mark.parametrize("n", [1, 7, 16383, 16385, 1_000_001])
def test_decompress_ragged(cuda, codec, S, n):
    v = np.random.default_rng(n).integers(0, 9, n, dtype=np.int32)
    col = api.Column(v, codec, lz4_segments=S).to_device()
    assert np.array_equal(_decode_all(col, cuda), v)


def test_decompress_single_chunk_offsets(cuda):
    v = np.arange(3_300_000, dtype=np.int32) * 3
    col = api.Column(v, "lz4").to_device()
    out = cuda.zeros(1_000_000, dtype=cuda.int32, device="cuda")
    d = api.ChunkDecompressor(col)
    for c in range(4):
        d.step(c, out)
        api.scan_check()
        rows = min(1_000_000, 3_300_000 - c * 1_000_000)
        assert np.array_equal(out[:rows].cpu().numpy(), v[c * 1_000_000: c * 1_000_000 + rows])


def test_decompress_pinned_host_residency(cuda):
    v = datagen.fact_q1(1_200_000, True)["discount"]
    col = api.Column(v, "lz4").to_device("pinned")
    assert col.info.on_device == 2
    assert np.array_equal(_decode_all(col, cuda), v)


def test_raw_lz4_blocks_from_liblz4(cuda):
    z = np.load(GOLDEN / "lz4_reference_blocks.npz")
    names = sorted({k[:-4] for k in z.files})
    comps = [z[n + "_lz4"] for n in names]
    raws = [z[n + "_raw"] for n in names]
    coff = np.concatenate([[0], np.cumsum([len(c) for c in comps])]).astype(np.uint64)
    ooff = np.concatenate([[0], np.cumsum([len(r) for r in raws])]).astype(np.uint64)
    comp_d = cuda.from_numpy(np.concatenate(comps)).cuda()
    out_d = cuda.zeros(int(ooff[-1]), dtype=cuda.uint8, device="cuda")
    st = cuda.full((len(names),), -1, dtype=cuda.int32, device="cuda")
    coff_d = cuda.from_numpy(coff.view(np.int64)).cuda()
    ooff_d = cuda.from_numpy(ooff.view(np.int64)).cuda()
    L.check(L.lib().gx_lz4_decompress_raw(C.c_void_p(comp_d.data_ptr()), C.c_void_p(coff_d.data_ptr()),
                                          C.c_void_p(out_d.data_ptr()), C.c_void_p(ooff_d.data_ptr()), len(names),
                                          C.c_void_p(st.data_ptr()), None))
    cuda.cuda.synchronize()
    assert st.cpu().tolist() == [0] * len(names)
    assert np.array_equal(out_d.cpu().numpy(), np.concatenate(raws))
    # a truncated block is reported per block, the others still decode
    comps[1] = comps[1][:-5]
    coff = np.concatenate([[0], np.cumsum([len(c) for c in comps])]).astype(np.uint64)
    comp_d = cuda.from_numpy(np.concatenate(comps)).cuda()
    coff_d = cuda.from_numpy(coff.view(np.int64)).cuda()
    L.check(L.lib().gx_lz4_decompress_raw(C.c_void_p(comp_d.data_ptr()), C.c_void_p(coff_d.data_ptr()),
                                          C.c_void_p(out_d.data_ptr()), C.c_void_p(ooff_d.data_ptr()), len(names),
                                          C.c_void_p(st.data_ptr()), None))
    cuda.cuda.synchronize()
    s = st.cpu().tolist()
    assert s[1] == L.GX_ERR_CORRUPT and s[0] == 0 and s[2:] == [0] * (len(names) - 2)


def _corrupt_payload(col, offset, value):
    p = L.u8p()
    n = C.c_uint64()
    L.check(L.lib().gx_column_payload(col.handle, C.byref(p), C.byref(n)))
    assert offset < n.value
    p[offset] = value


@pytest.mark.parametrize("codec,S", [("lz4", 32), ("lz4", 1), ("cascaded", 1)])
def test_corrupt_blocks_are_reported(cuda, codec, S):
    # fixed 4-byte matches: a token-heavy LZ4 stream (with the default policy
    # these values encode as one literal run, whose last token's match nibble
    # no decoder reads)
    kw = {"lz4_min_match": 4} if codec == "lz4" else {}
    v = np.random.default_rng(2).integers(0, 11, 300_000, dtype=np.int32)
    rng = np.random.default_rng(9)
    reported = 0
    for trial in range(12):
        col = api.Column(v, codec, lz4_segments=S, **kw)
        blocks = col.blocks()
        b = blocks[trial % len(blocks)]
        off = int(b[0]) + int(rng.integers(0, int(b[2])))
        _corrupt_payload(col, off, int(rng.integers(0, 256)))
        col.to_device()
        out = cuda.zeros(300_000, dtype=cuda.int32, device="cuda")
        api.ChunkDecompressor(col).chunks(0, col.info.n_chunks, out)
        try:
            api.scan_check()
            got = out.cpu().numpy()  # a byte flip inside literals decodes to different values, legitimately
            assert got.shape == v.shape
        except GxError as e:
            assert e.status == L.GX_ERR_CORRUPT
            reported += 1
    # a flip inside packed values or literals legitimately decodes to other
    # values; a broken header / token stream must be reported
    col = api.Column(v, codec, lz4_segments=S, **kw)
    first = int(col.blocks()[0][0])
    if codec == "lz4" and S > 1:
        # segment decoders start from the side index (entry 0 resumes inside the
        # first literal run): break the first match's offset, which they read
        lit_pos, info = (int(x) for x in col.seg_index()[:2])
        assert info & 16
        _corrupt_payload(col, first + lit_pos + (info >> 5), 0xFF)
        _corrupt_payload(col, first + lit_pos + (info >> 5) + 1, 0xFF)
    elif codec == "cascaded":
        # the first page's run count (pages are located through the side index)
        page = int(col.seg_index()[0])
        _corrupt_payload(col, first + page + 5, 0xFF)
    else:
        _corrupt_payload(col, first, 0xFF)  # first token
    col.to_device()
    out = cuda.zeros(300_000, dtype=cuda.int32, device="cuda")
    api.ChunkDecompressor(col).chunks(0, col.info.n_chunks, out)
    with pytest.raises(GxError) as e:
        api.scan_check()
    assert e.value.status == L.GX_ERR_CORRUPT
    # the device stays usable afterwards
    col = api.Column(v, codec, lz4_segments=S).to_device()
    assert np.array_equal(_decode_all(col, cuda), v)
