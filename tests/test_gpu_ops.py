"""GPU operators against the oracle and the reference's own known answers:
min/max pruning (core/test/metadata_tests.cu), join count/probe
(core/test/join_tests.cu:71-107), group-by sums
(core/test/group_by_tests.cu:75-132)."""
import ctypes as C

import numpy as np
import pytest

from golap_public_b200 import _lib as L
from golap_public_b200 import api
from golap_public_b200._lib import GxError
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def test_check_minmax_and_combine(cuda):
    rng = np.random.default_rng(4)
    v = np.sort(rng.integers(0, 10_000, 2_000_000, dtype=np.int32))
    col = api.Column(v, "cascaded", rows_per_chunk=50_000).to_device()
    mins, maxs = col.minmax()
    n = col.info.n_chunks
    for lo, hi in [(0, 0), (5000, 5000), (-10, -1), (9999, 20000), (1234, 4321), (10_000, 10_000)]:
        flags = cuda.zeros(n, dtype=cuda.uint16, device="cuda")
        L.check(L.lib().gx_check_minmax(col.handle, lo, hi, C.c_void_p(flags.data_ptr()), None))
        cuda.cuda.synchronize()
        assert flags.cpu().numpy().tolist() == O.minmax_keep(mins, maxs, lo, hi).tolist()
    a = cuda.zeros(n, dtype=cuda.uint16, device="cuda")
    b = cuda.zeros(n, dtype=cuda.uint16, device="cuda")
    L.check(L.lib().gx_check_minmax(col.handle, 0, 6000, C.c_void_p(a.data_ptr()), None))
    L.check(L.lib().gx_check_minmax(col.handle, 4000, 9000, C.c_void_p(b.data_ptr()), None))
    L.check(L.lib().gx_combine_and(C.c_void_p(a.data_ptr()), C.c_void_p(a.data_ptr()), C.c_void_p(b.data_ptr()), n, None))
    cuda.cuda.synchronize()
    want = O.minmax_keep(mins, maxs, 4000, 9000, keep=O.minmax_keep(mins, maxs, 0, 6000))
    assert a.cpu().numpy().tolist() == want.tolist()


def test_metachecker_known_answers(cuda):
    # integer version of core/test/metadata_tests.cu:210-272: three chunks of 8
    # rows, {h0..h7}, {h8..h15}, {Dec1996/Feb1992} -> {0..7}, {8..15}, {1992,1996}
    v = np.array(list(range(16)) + [1996, 1992] * 4, np.int32)
    col = api.Column(v, "lz4", rows_per_chunk=8, rows_per_block=8, lz4_segments=1).to_device()
    keep = cuda.zeros(3, dtype=cuda.uint16, device="cuda")
    for lo, hi, want in [(5, 5, [1, 0, 0]), (15, 15, [0, 1, 0]), (1997, 1997, [0, 0, 0]), (1992, 1992, [0, 0, 1]),
                         (7, 1993, [1, 1, 1])]:
        api.MetaChecker(3).add_minmax(col, lo, hi).run(keep)
        assert keep.cpu().tolist() == want
    # AND of two predicates: [0,100] keeps chunks 0,1; [8,2000] keeps chunks 1,2
    api.MetaChecker(3).add_minmax(col, 0, 100).add_minmax(col, 8, 2000).run(keep)
    assert keep.cpu().tolist() == [0, 1, 0]


@pytest.mark.parametrize("layout", ["linear", "bucket", "dense"])
def test_join_count_1to1(cuda, layout):
    # join_tests.cu:71-107: build 500k ids, probe 10M rows id = i % 500k -> 10M hits
    build = cuda.arange(500_000, dtype=cuda.int32, device="cuda")
    probe = (cuda.arange(10_000_000, dtype=cuda.int64, device="cuda") % 500_000).to(cuda.int32)
    hm = api.HashMap(500_000, layout).build(build)
    assert hm.count() == 500_000
    hits = cuda.zeros(1, dtype=cuda.int64, device="cuda")
    pay = cuda.empty(10_000_000, dtype=cuda.int32, device="cuda")
    hm.probe(probe, pay, hits)
    assert int(hits.item()) == 10_000_000
    assert cuda.equal(pay, probe)  # payload defaults to the build row id


@pytest.mark.parametrize("layout", ["linear", "bucket", "dense"])
def test_filtered_build_and_probe_vs_oracle(cuda, layout):
    rng = np.random.default_rng(8)
    n_b, n_p = 200_000, 3_000_000
    keys = rng.permutation(np.arange(1, 4 * n_b, 4, dtype=np.int32))[:n_b]
    region = rng.integers(0, 5, n_b, dtype=np.int32)
    nation = rng.integers(0, 25, n_b, dtype=np.int32)
    probe = rng.integers(0, 4 * n_b + 10, n_p, dtype=np.int32)
    kd, rd, nd, pd = (cuda.from_numpy(x).cuda() for x in (keys, region, nation, probe))
    hm = api.HashMap(n_b, layout).build(kd, nd, preds=[(rd, 2, 3)])
    ok = (region >= 2) & (region <= 3)
    assert hm.count() == int(ok.sum())
    out = cuda.empty(n_p, dtype=cuda.int32, device="cuda")
    hits = cuda.zeros(1, dtype=cuda.int64, device="cuda")
    hm.probe(pd, out, hits)
    rid = O.join_probe(keys, ok, probe)
    want = np.where(rid >= 0, nation[np.maximum(rid, 0)], np.iinfo(np.int32).min)
    assert np.array_equal(out.cpu().numpy(), want)
    assert int(hits.item()) == int((rid >= 0).sum())


@pytest.mark.parametrize("layout", ["linear", "bucket", "dense"])
def test_hashtable_reserved_key_and_capacity(cuda, layout):
    keys = cuda.tensor([1, 2, np.iinfo(np.int32).min, 3], dtype=cuda.int32, device="cuda")
    hm = api.HashMap(4, layout).build(keys)
    with pytest.raises(GxError) as e:
        hm.count()
    assert e.value.status == L.GX_ERR_CAPACITY
    # more keys than max_entries: reported, never hangs
    many = cuda.arange(100, dtype=cuda.int32, device="cuda")
    hm2 = api.HashMap(8, layout).build(many)
    with pytest.raises(GxError):
        hm2.count()


def test_dense_table_edges(cuda):
    # negative keys, duplicates (the first insert wins), probes at and just
    # outside the range ends, the reserved key, an empty build, sparse keys
    keys = cuda.tensor([-5, 7, -5, 0, 12, 7], dtype=cuda.int32, device="cuda")
    pay = cuda.tensor([10, 11, 12, 13, 14, 15], dtype=cuda.int32, device="cuda")
    hm = api.HashMap(8, "dense").build(keys, pay)
    assert hm.count() == 4
    probe = cuda.tensor([-6, -5, 0, 7, 12, 13, 3, np.iinfo(np.int32).min, np.iinfo(np.int32).max],
                        dtype=cuda.int32, device="cuda")
    out = cuda.empty(9, dtype=cuda.int32, device="cuda")
    hits = cuda.zeros(1, dtype=cuda.int64, device="cuda")
    hm.probe(probe, out, hits)
    miss = np.iinfo(np.int32).min
    got = out.cpu().tolist()
    assert got[0] == miss and got[1] in (10, 12) and got[2] == 13 and got[3] in (11, 15) and got[4] == 14
    assert got[5:] == [miss] * 4 and int(hits.item()) == 4
    # predicates that pass no row: every probe misses
    reg = cuda.zeros(6, dtype=cuda.int32, device="cuda")
    hm.build(keys, pay, preds=[(reg, 1, 1)])
    assert hm.count() == 0
    hits.zero_()
    hm.probe(probe, out, hits)
    assert int(hits.item()) == 0 and out.cpu().tolist() == [miss] * 9
    # rebuilt over a wider range: the table grows
    wide = cuda.arange(0, 900_000, 3, dtype=cuda.int32, device="cuda")
    hm.build(wide)
    hits.zero_()
    hm.probe(wide[::1000].contiguous(), None, hits)
    assert int(hits.item()) == wide[::1000].numel()
    # keys too sparse for a dense table
    sparse = cuda.tensor([0, 1 << 30], dtype=cuda.int32, device="cuda")
    with pytest.raises(GxError) as e:
        api.HashMap(2, "dense").build(sparse)
    assert e.value.status == L.GX_ERR_INVALID and "span" in str(e.value)


def test_groupby_exact_sums(cuda):
    # group_by_tests.cu:75-132 at 2^27 rows: 64 groups, each sums to 2^27/64
    n, g = 1 << 27, 64
    keys = cuda.arange(n, dtype=cuda.int64, device="cuda") % g
    vals = cuda.ones(n, dtype=cuda.int64, device="cuda")
    agg = api.HashAggregate(g)
    agg.add(keys, vals)
    res = agg.read()
    assert len(res) == g and all(v == n // g for v in res.values())
    del keys, vals


def test_groupby_vs_oracle_and_overflow(cuda):
    rng = np.random.default_rng(12)
    k = rng.integers(0, 5000, 2_000_000).astype(np.int64)
    v = rng.integers(-10**9, 10**9, 2_000_000).astype(np.int64)
    agg = api.HashAggregate(5000)
    agg.add(cuda.from_numpy(k).cuda(), cuda.from_numpy(v).cuda())
    got = agg.read()
    want = np.zeros(5000, np.int64)
    assert O.lib().or_group_sum_dense(O._ptr(k), O._ptr(v), len(k), O._ptr(want), 5000) == 0
    assert got == {i: int(want[i]) for i in range(5000) if (k == i).any()}
    small = api.HashAggregate(10)  # 32 slots
    small.add(cuda.from_numpy(k[:1000]).cuda(), cuda.from_numpy(v[:1000]).cuda())
    with pytest.raises(GxError) as e:
        api.scan_check()
    assert e.value.status == L.GX_ERR_CAPACITY


@pytest.mark.parametrize("layout", ["linear", "bucket", "dense"])
def test_hashtable_keys_collects_filtered_build_keys(cuda, layout):
    # collect_hashmap_keys (core/dev_structs.cuh:136-150): the keys of the rows
    # the filtered build inserted, in any order, count on the device
    rng = np.random.default_rng(12)
    keys = rng.permutation(np.arange(100, 100 + 50_000, dtype=np.int32))
    flag = rng.integers(0, 3, len(keys), dtype=np.int32)
    kd, fd = cuda.from_numpy(keys).cuda(), cuda.from_numpy(flag).cuda()
    hm = api.HashMap(len(keys), layout).build(kd, None, preds=[(fd, 1, 1)])
    out = cuda.empty(len(keys), dtype=cuda.int32, device="cuda")
    cnt = cuda.zeros(1, dtype=cuda.int64, device="cuda")
    hm.keys(out, cnt)
    n = int(cnt.item())
    assert sorted(out[:n].cpu().numpy().tolist()) == sorted(keys[flag == 1].tolist())
    # a too-small output: the count is still the full count, nothing written past cap
    small = cuda.full((10,), -7, dtype=cuda.int32, device="cuda")
    hm.keys(small, cnt)
    assert int(cnt.item()) == n and set(small.cpu().numpy().tolist()) <= set(keys[flag == 1].tolist())


def test_join_pruning_points_vs_oracle(cuda):
    # check_mmmeta_multiple_pts (core/metadata.cuh:550-560) behind --join_prune
    # (usecases/ssb/queries/01.hpp:246-270): a chunk stays when one of the
    # build side's keys lies in its min/max
    rng = np.random.default_rng(5)
    v = np.sort(rng.integers(0, 1_000_000, 3_000_000, dtype=np.int32))
    col = api.Column(v, "cascaded", rows_per_chunk=20_000).to_device()
    mins, maxs = col.minmax()
    n = col.info.n_chunks
    for keys in (np.array([5, 500_000, 999_999], np.int32), rng.integers(-5, 1_100_000, 5000, dtype=np.int32),
                 np.zeros(0, np.int32), rng.integers(0, 1_000_000, 3000, dtype=np.int32)):
        kd = cuda.from_numpy(np.ascontiguousarray(keys)).cuda() if len(keys) else cuda.zeros(1, dtype=cuda.int32,
                                                                                           device="cuda")
        cnt = cuda.tensor([len(keys)], dtype=cuda.int64, device="cuda")
        keep = cuda.zeros(n, dtype=cuda.uint16, device="cuda")
        api.MetaChecker(n).add_points(col, kd, cnt, keep)
        assert keep.cpu().numpy().tolist() == O.minmax_points_keep(mins, maxs, keys).tolist()


def test_minmax_reduce_and_clear(cuda):
    # MinMaxMeta::init_chunk (core/metadata.cuh:157-160) on device data
    rng = np.random.default_rng(8)
    for n in (1, 3, 1000, 1 << 20, 3_000_001):
        v = rng.integers(-2**31, 2**31 - 1, n, dtype=np.int64).astype(np.int32)
        vd = cuda.from_numpy(v).cuda()
        for off in (0, 1):  # aligned and unaligned starts
            if off >= n:
                continue
            r = cuda.zeros(2, dtype=cuda.int32, device="cuda")
            L.check(L.lib().gx_minmax_reduce(C.c_void_p(vd.data_ptr() + 4 * off), n - off, C.c_void_p(r.data_ptr()),
                                             None))
            assert r.cpu().numpy().tolist() == [int(v[off:].min()), int(v[off:].max())]
    hm = api.HashMap(1000).build(cuda.arange(1000, dtype=cuda.int32, device="cuda"))
    assert hm.count() == 1000
    L.check(L.lib().gx_hashtable_clear(hm.handle, None))
    assert hm.count() == 0
    hits = cuda.zeros(1, dtype=cuda.int64, device="cuda")
    hm.probe(cuda.arange(1000, dtype=cuda.int32, device="cuda"), None, hits)
    assert int(hits.item()) == 0


@pytest.mark.parametrize("layout", ["linear", "bucket"])
@pytest.mark.parametrize("carry,key_codec", [(True, "cascaded"), (False, "lz4"), (True, "lz4")])
def test_build_from_compressed_dimension(cuda, layout, carry, key_codec):
    # GX_AGG_BUILD: pipeline_customer_q3 (usecases/ssb/queries/03.cuh:94-116)
    # fused with the decompression of the customer chunks -- filter on region,
    # insert key -> nation (CARRY) or key -> row number
    from golap_public_b200 import datagen, queries

    n = 1_200_000
    cust = datagen.dim_geo(n, datagen.SEED, 21)
    keys = cust["key"] if key_codec == "cascaded" else np.random.default_rng(3).permutation(cust["key"])
    cc = queries.encode_fact({"key": keys, "nation": cust["nation"], "region": cust["region"]},
                             {"key": key_codec, "nation": "cascaded", "region": "cascaded"}, rows_per_chunk=500_000)
    ht = api.HashMap(n, layout)
    queries.build_from_compressed(ht, cc.cols["key"], cc.cols["nation"] if carry else None,
                                  [(cc.cols["region"], 2, 2)])
    sel = cust["region"] == 2
    assert ht.count() == int(sel.sum())
    probe = cuda.from_numpy(keys).cuda()
    out = cuda.empty_like(probe)
    ht.probe(probe, out)
    exp = np.where(sel, cust["nation"] if carry else np.arange(n, dtype=np.int32), np.iinfo(np.int32).min)
    assert np.array_equal(out.cpu().numpy(), exp)
    # a dense table cannot be filled this way (it sizes itself from the key range)
    with pytest.raises(GxError):
        queries.build_from_compressed(api.HashMap(n, "dense"), cc.cols["key"], None)


@pytest.mark.parametrize("kind", ["sorted_date", "random", "constant_chunks"])
def test_histogram_metadata_vs_oracle(cuda, kind):
    # EqHistogram + fill_hist / check_hist (core/metadata.cuh:225-382, 573-595)
    from golap_public_b200 import datagen

    rng = np.random.default_rng(21)
    n, rpc = 1_000_000, 100_000
    if kind == "sorted_date":
        v = datagen.fact_q1(n, True)["date_key"]
    elif kind == "random":
        v = rng.integers(-50_000, 50_000, n, dtype=np.int32)
    else:
        v = np.repeat(rng.integers(0, 100, n // rpc, dtype=np.int32), rpc)
    col = api.Column(v, "cascaded" if kind != "random" else "lz4", rows_per_chunk=rpc).to_device()
    for nb in (1, 16, 1000):
        col.build_hist(nb)
        h, _, _ = col.meta()
        want = O.hist_counts(v, rpc, nb)
        assert np.array_equal(h, want)
        mins, maxs = col.minmax()
        med = int(np.median(v))
        for lo, hi in [(int(v.min()), int(v.min())), (int(v.max()), int(v.max())), (med, med + 3),
                       (int(v.min()) - 10, int(v.min()) - 1), (-100, 100), (19940101, 19940131)]:
            flags = cuda.zeros(len(mins), dtype=cuda.uint16, device="cuda")
            api.MetaChecker(len(mins)).add_hist(col, lo, hi, flags)
            assert flags.cpu().numpy().tolist() == O.hist_keep(mins, maxs, want, lo, hi).tolist()


@pytest.mark.parametrize("m_bytes,p", [(64, 0.05), (1024, 0.01), (8192, 0.001)])
def test_bloom_metadata_vs_oracle(cuda, m_bytes, p):
    # BloomMeta + fill_bloom / check_bloom (core/metadata.cuh:385-537, 602-620)
    rng = np.random.default_rng(22)
    n, rpc = 600_000, 50_000
    v = rng.integers(0, 200_000, n, dtype=np.int32)
    col = api.Column(v, "lz4", rows_per_chunk=rpc).to_device().build_bloom(m_bytes, p)
    _, w, k = col.meta()
    want_w, want_k = O.bloom_words(v, rpc, m_bytes, p)
    assert k == want_k and np.array_equal(w, want_w)
    nc = col.info.n_chunks
    for val in [int(v[0]), int(v[-1]), -1, 123_456, 199_999, int(v[rpc * 3 + 7])]:
        flags = cuda.zeros(nc, dtype=cuda.uint16, device="cuda")
        api.MetaChecker(nc).add_bloom(col, val, flags)
        got = flags.cpu().numpy()
        assert got.tolist() == O.bloom_keep(want_w, m_bytes, k, val).tolist()
        present = np.array([(v[c * rpc:(c + 1) * rpc] == val).any() for c in range(nc)])
        assert np.all(got[present] == 1)  # no false negatives
