"""Fused scan parity: GPU results must equal the oracle bit for bit, and on
the reference's SSB data the reference's own results (Q1.1/Q1.2/Q1.3 sums and
the Q3.1 group count/total in tests/golden/ssb_sf1_reference.json).

Shapes: pipeline_q1_lineorder (usecases/ssb/queries/01.cuh:27-54) and
pipeline_q3 (usecases/ssb/queries/03.cuh:119-170)."""
import json
from pathlib import Path

import numpy as np
import pytest

from golap_public_b200 import _lib as L
from golap_public_b200 import api, datagen, queries
from golap_public_b200._lib import GxError
from oracle import oracle as O

pytestmark = pytest.mark.gpu
GOLDEN = json.loads((Path(__file__).parent / "golden" / "ssb_sf1_reference.json").read_text())


@pytest.fixture(scope="module")
def sf1():
    return O.ssb_generate(1)


def _fact_sf1(t, codec_date="cascaded", codec_other="lz4", S=32):
    data = {"date_key": t["lo_orderdate"], "discount": t["lo_discount"], "quantity": t["lo_quantity"],
            "extended_price": t["lo_extendedprice"], "cust_key": t["lo_custkey"], "supp_key": t["lo_suppkey"],
            "revenue": t["lo_revenue"]}
    codecs = {k: codec_other for k in data}
    codecs["date_key"] = codec_date
    return queries.encode_fact(data, codecs, lz4_segments=S)


@pytest.mark.parametrize("codec_date,codec_other,S", [("cascaded", "lz4", 32), ("none", "none", 1),
                                                      ("lz4", "lz4", 1), ("cascaded", "cascaded", 1),
                                                      ("lz4", "lz4", 128)])
def test_ssb_sf1_matches_reference(cuda, sf1, codec_date, codec_other, S):
    fact = _fact_sf1(sf1, codec_date, codec_other, S)
    date = {"d_key": sf1["d_key"], "d_year": sf1["d_year"], "d_yearmonthnum": sf1["d_yearmonthnum"]}
    cases = [
        ("q1_1", sf1["d_year"] == 1993, 1, 3, 0, 24),
        ("q1_2", sf1["d_yearmonthnum"] == 199401, 4, 6, 26, 35),
        ("q1_3", (sf1["d_weeknuminyear"] == 6) & (sf1["d_year"] == 1994), 5, 7, 26, 35),
    ]
    for name, ok, dlo, dhi, qlo, qhi in cases:
        dk = sf1["d_key"][ok]
        for prune in (False, True):
            q = queries.Q1Query(fact, date, ok, int(dk.min()), int(dk.max()), dlo, dhi, qlo, qhi, prune=prune)
            assert q.run() == GOLDEN[name], (name, prune)
    # Q3.1: customer/supplier region ASIA (2), years 1992..1997, keys 0-based
    cust = {"key": sf1["c_key"], "nation": sf1["c_nation"], "region": sf1["c_region"]}
    supp = {"key": sf1["s_key"], "nation": sf1["s_nation"], "region": sf1["s_region"]}
    q3 = queries.Q3Query(fact, cust, supp, date, 2, 1992, 1997)
    got = q3.run()
    assert len(got) == GOLDEN["q3_1_groups"] and sum(got.values()) == GOLDEN["q3_1_sum"]
    sums, counts = O.ssb_queries(sf1)["q3_1_cells"]
    want = {(c, s, 1992 + y): int(sums[c, s, y]) for c, s, y in zip(*np.nonzero(counts))}
    assert got == want


def _oracle_q1(f, dd, ok, dlo, dhi, qlo, qhi, keep=None, rpc=1):
    return O.q1(f["date_key"], f["discount"], f["quantity"], f["extended_price"], dd["d_key"], ok, dlo, dhi, qlo, qhi,
                keep_chunk=keep, rows_per_chunk=rpc)


def test_q1_config0_uncompressed(cuda):
    # 6M unsorted rows, uncompressed, 1M-row chunks, no pruning; year 1993,
    # discount 1..3, quantity < 25
    f = datagen.fact_q1(6_000_000, False)
    dd = datagen.date_dim()
    fact = queries.encode_fact(f, {k: "none" for k in f})
    ok = dd["d_year"] == 1993
    q = queries.Q1Query(fact, dd, ok, 19930101, 19931231, 1, 3, 0, 24, prune=False)
    assert q.run() == _oracle_q1(f, dd, ok, 1, 3, 0, 24)


@pytest.mark.parametrize("S", [32, 128])
def test_q1_config1_sorted_pruned(cuda, S):
    # 60M rows sorted by date; cascaded date, LZ4 others; January 1994
    f = datagen.fact_q1(60_000_000, True)
    dd = datagen.date_dim()
    fact = queries.encode_fact(f, {"date_key": "cascaded"}, lz4_segments=S)
    ok = dd["d_yearmonthnum"] == 199401
    want = _oracle_q1(f, dd, ok, 4, 6, 26, 35)
    for prune in (True, False):
        q = queries.Q1Query(fact, dd, ok, 19940101, 19940131, 4, 6, 26, 35, prune=prune)
        assert q.run() == want
        if prune:
            kept = int(q.keep.sum().item())
            assert 1 <= kept <= 3  # ~98% of the 60 chunks pruned
            mins, maxs = fact.cols["date_key"].minmax()
            assert q.keep.cpu().numpy().tolist() == O.minmax_keep(mins, maxs, 19940101, 19940131).tolist()


def test_q1_join_pruning(cuda):
    # join pruning (usecases/ssb/queries/01.hpp:246-270): the filtered date
    # table's keys prune the chunks whose date_key min/max holds none of them;
    # two months three years apart keep only their own chunks, where min/max
    # pruning on the key range would keep everything in between
    f = datagen.fact_q1(30_000_000, True)
    dd = datagen.date_dim()
    fact = queries.encode_fact(f, {"date_key": "cascaded"})
    ok = np.isin(dd["d_yearmonthnum"], [199302, 199607])
    want = _oracle_q1(f, dd, ok, 4, 6, 26, 35)
    q = queries.Q1Query(fact, dd, ok, int(dd["d_key"][ok].min()), int(dd["d_key"][ok].max()), 4, 6, 26, 35,
                        prune=True, join_prune=True)
    assert q.run() == want
    mins, maxs = fact.cols["date_key"].minmax()
    jk = q.join_keep.cpu().numpy()
    assert jk.tolist() == O.minmax_points_keep(mins, maxs, dd["d_key"][ok]).tolist()
    range_keep = O.minmax_keep(mins, maxs, int(dd["d_key"][ok].min()), int(dd["d_key"][ok].max()))
    assert jk.sum() < range_keep.sum() // 4
    # keep_out = join flags AND the plan's own min/max pruning
    assert q.keep.cpu().numpy().tolist() == (jk & range_keep).tolist()


def test_q1_keep_chunks_in_and_out(cuda):
    # per-chunk keep flags handed to the scan (MetaChecker output) combine with
    # the plan's own min/max pruning; keep_out receives keep_in AND min/max
    f = datagen.fact_q1(7_500_000, True)
    dd = datagen.date_dim()
    fact = queries.encode_fact(f, {"date_key": "cascaded"})
    ok = dd["d_year"] == 1993
    keep_in = np.array([1, 1, 0, 1, 1, 0, 1, 1], dtype=np.uint16)
    q = queries.Q1Query(fact, dd, ok, 19930101, 19931231, 1, 3, 0, 24, prune=True)
    q.plan.keep_chunks = cuda.from_numpy(keep_in).cuda()
    got = q.run()
    assert got == _oracle_q1(f, dd, ok, 1, 3, 0, 24, keep=keep_in, rpc=1_000_000)
    assert got != _oracle_q1(f, dd, ok, 1, 3, 0, 24)  # the dropped chunks held qualifying rows
    mins, maxs = fact.cols["date_key"].minmax()
    assert q.keep.cpu().numpy().tolist() == O.minmax_keep(mins, maxs, 19930101, 19931231, keep=keep_in).tolist()


def test_q1_pinned_host_residency(cuda):
    # compressed columns in pinned host memory, read by the kernels over
    # PCIe: the same results as HBM residency, pruned and over every date
    f = datagen.fact_q1(8_000_000, True)
    dd = datagen.date_dim()
    fact = queries.encode_fact(f, {"date_key": "cascaded"}, residency="pinned")
    assert all(c.info.on_device == 2 for c in fact.cols.values())
    ok = dd["d_yearmonthnum"] == 199301
    q = queries.Q1Query(fact, dd, ok, 19930101, 19930131, 4, 6, 26, 35, prune=True)
    assert q.run() == _oracle_q1(f, dd, ok, 4, 6, 26, 35)
    ok_all = np.ones(len(dd["d_key"]), dtype=bool)
    qa = queries.Q1Query(fact, dd, ok_all, int(dd["d_key"].min()), int(dd["d_key"].max()), 4, 6, 26, 35, prune=False)
    assert qa.run() == _oracle_q1(f, dd, ok_all, 4, 6, 26, 35)


@pytest.mark.parametrize("group", [1, 3, 16])
def test_q1_streamed_from_pinned_host(cuda, group):
    # gx_scan_streamed: surviving chunks' bytes are staged in HBM group by
    # group; results and chunk flags equal the oracle's, pruned and unpruned
    f = datagen.fact_q1(9_500_000, True)
    dd = datagen.date_dim()
    fact = queries.encode_fact(f, {"date_key": "cascaded"}, residency="pinned", lz4_segments=32)
    for ym, lo, hi in ((199301, 19930101, 19930131), (199712, 19971201, 19971231)):
        ok = dd["d_yearmonthnum"] == ym
        q = queries.Q1Query(fact, dd, ok, lo, hi, 4, 6, 26, 35, prune=True)
        q.stream_group = group
        assert q.run() == _oracle_q1(f, dd, ok, 4, 6, 26, 35)
        mins, maxs = fact.cols["date_key"].minmax()
        assert q.keep.cpu().numpy().tolist() == O.minmax_keep(mins, maxs, lo, hi).tolist()
    ok_all = np.ones(len(dd["d_key"]), dtype=bool)
    qa = queries.Q1Query(fact, dd, ok_all, int(dd["d_key"].min()), int(dd["d_key"].max()), 1, 3, 0, 24, prune=False)
    qa.stream_group = group
    assert qa.run() == _oracle_q1(f, dd, ok_all, 1, 3, 0, 24)


def test_q3_streamed_from_pinned_host(cuda):
    f = datagen.fact_q3(5_000_000, True, n_customer=300_000, n_supplier=20_000)
    cust = datagen.dim_geo(300_000, datagen.SEED, 21)
    supp = datagen.dim_geo(20_000, datagen.SEED, 22)
    dd = datagen.date_dim()
    fact = queries.encode_fact(f, {"date_key": "cascaded"}, residency="pinned", lz4_segments=32)
    q = queries.Q3Query(fact, cust, supp, dd, 2, 1994, 1995)
    q.stream_group = 2
    sums, counts = O.q3(f["cust_key"], f["supp_key"], f["date_key"], f["revenue"], cust["key"], cust["nation"],
                        cust["region"] == 2, supp["key"], supp["nation"], supp["region"] == 2, dd["d_key"],
                        dd["d_year"], (dd["d_year"] >= 1994) & (dd["d_year"] <= 1995), 0, 25, 0, 25, 1994, 2)
    assert q.run() == {(c, s, 1994 + y): int(sums[c, s, y]) for c, s, y in zip(*np.nonzero(counts))}


def test_streamed_rejects_hbm_only_shapes(cuda):
    f = datagen.fact_q1(300_000, True)
    dd = datagen.date_dim()
    fact = queries.encode_fact(f, {"date_key": "cascaded"}, residency="pinned", lz4_segments=1)
    q = queries.Q1Query(fact, dd, dd["d_yearmonthnum"] == 199301, 19930101, 19930131, 4, 6, 26, 35)
    q.stream_group = 4
    with pytest.raises(GxError):
        q.run()  # plain LZ4 blocks: not a pipelined-kernel shape


def test_q3_star_join_groupby(cuda):
    # configs[2] shape at 20M fact rows with full-size dimensions
    f = datagen.fact_q3(20_000_000, True)
    cust = datagen.dim_geo(3_000_000, datagen.SEED, 21)
    supp = datagen.dim_geo(200_000, datagen.SEED, 22)
    dd = datagen.date_dim()
    fact = queries.encode_fact(f, {"date_key": "cascaded"})
    for region, layout in ((1, "linear"), (3, "linear"), (3, "bucket")):
        q = queries.Q3Query(fact, cust, supp, dd, region, 1992, 1997, ht_layout=layout)
        got = q.run()
        sums, counts = O.q3(f["cust_key"], f["supp_key"], f["date_key"], f["revenue"],
                            cust["key"], cust["nation"], cust["region"] == region,
                            supp["key"], supp["nation"], supp["region"] == region,
                            dd["d_key"], dd["d_year"], (dd["d_year"] >= 1992) & (dd["d_year"] <= 1997),
                            0, 25, 0, 25, 1992, 6)
        want = {(c, s, 1992 + y): int(sums[c, s, y]) for c, s, y in zip(*np.nonzero(counts))}
        assert got == want
        assert 100 <= len(got) <= 150


def test_q3_customer_from_compressed_chunks(cuda):
    # the customer join table filled from compressed customer columns in one
    # fused launch (GX_AGG_BUILD), then the star join: same groups as the oracle
    f = datagen.fact_q3(6_000_000, True)
    cust = datagen.dim_geo(3_000_000, datagen.SEED, 21)
    supp = datagen.dim_geo(200_000, datagen.SEED, 22)
    dd = datagen.date_dim()
    fact = queries.encode_fact(f, {"date_key": "cascaded"})
    cc = queries.encode_fact(cust, {"key": "cascaded", "nation": "cascaded", "region": "cascaded"})
    for region in (0, 3):
        q = queries.Q3Query(fact, cc, supp, dd, region, 1993, 1996)
        got = q.run()
        sums, counts = O.q3(f["cust_key"], f["supp_key"], f["date_key"], f["revenue"],
                            cust["key"], cust["nation"], cust["region"] == region,
                            supp["key"], supp["nation"], supp["region"] == region,
                            dd["d_key"], dd["d_year"], (dd["d_year"] >= 1993) & (dd["d_year"] <= 1996),
                            0, 25, 0, 25, 1993, 4)
        want = {(c, s, 1993 + y): int(sums[c, s, y]) for c, s, y in zip(*np.nonzero(counts))}
        assert got == want
        q.build_customer()  # rebuilt in place: the same table again
        assert q.hc.count() == int((cust["region"] == region).sum())
        assert q.run() == want


def test_scan_plan_validation(cuda):
    f = datagen.fact_q1(100_000, False)
    fact = queries.encode_fact(f, {})
    res = cuda.zeros(1, dtype=cuda.int64, device="cuda")
    p = api.ScanPlan(agg=L.GX_AGG_SUM_PRODUCT, result=res).filter(fact.cols["discount"], 0, 10)
    with pytest.raises(GxError):
        p.launch()  # no VALUE step
    p.value(fact.cols["extended_price"])
    with pytest.raises(GxError):
        p.launch()  # SUM_PRODUCT without CARRY
    other = api.Column(np.arange(10, dtype=np.int32), "lz4").to_device()
    with pytest.raises(GxError):
        api.ScanPlan(result=res).value(other).filter(fact.cols["discount"], 0, 1).launch()  # layout mismatch


def test_scan_count_and_sum_aggregates(cuda):
    f = datagen.fact_q1(3_000_000, False)
    fact = queries.encode_fact(f, {"date_key": "cascaded"})
    res = cuda.zeros(1, dtype=cuda.int64, device="cuda")
    api.ScanPlan(agg=L.GX_AGG_COUNT, result=res).filter(fact.cols["quantity"], 10, 20).value(
        fact.cols["discount"], 2, 5).run_sync()
    m = (f["quantity"] >= 10) & (f["quantity"] <= 20) & (f["discount"] >= 2) & (f["discount"] <= 5)
    assert int(res.item()) == int(m.sum())
    res.zero_()
    api.ScanPlan(agg=L.GX_AGG_SUM, result=res).filter(fact.cols["quantity"], 10, 20).value(
        fact.cols["extended_price"]).run_sync()
    m = (f["quantity"] >= 10) & (f["quantity"] <= 20)
    assert int(res.item()) == int(f["extended_price"][m].astype(np.int64).sum())


def test_scan_reports_corrupt_tile_and_recovers(cuda):
    import ctypes as C

    f = datagen.fact_q1(2_000_000, False)
    dd = datagen.date_dim()
    good = queries.encode_fact(f, {"date_key": "cascaded"})
    data = dict(f)
    bad_cols = {}
    for k, v in data.items():
        c = api.Column(v, "cascaded" if k == "date_key" else "lz4")
        if k == "date_key":
            p = L.u8p()
            n = C.c_uint64()
            L.check(L.lib().gx_column_payload(c.handle, C.byref(p), C.byref(n)))
            off = int(c.blocks()[3][0])
            pages = -(-c.info.rows_per_block // 2048)
            page = int(c.seg_index()[2 * pages * 3])  # first page of block 3 (side index entry)
            p[off + page + 4] = 0xFF  # its n_runs -> invalid page header
        bad_cols[k] = c.to_device()
    bad = queries.FactTable(bad_cols, len(f["date_key"]))
    ok = dd["d_year"] == 1995
    q = queries.Q1Query(bad, dd, ok, 19950101, 19951231, 0, 10, 0, 50, prune=False)
    with pytest.raises(GxError) as e:
        q.run()
    assert e.value.status == L.GX_ERR_CORRUPT
    q2 = queries.Q1Query(good, dd, ok, 19950101, 19951231, 0, 10, 0, 50, prune=False)
    assert q2.run() == _oracle_q1(f, dd, ok, 0, 10, 0, 50)


def test_scan_group_overflow_reports_capacity(cuda):
    # high-cardinality groups into a too-small global table: reported, no hang
    rng = np.random.default_rng(3)
    n = 2_000_000
    key = rng.integers(0, 1000, n, dtype=np.int32)
    val = rng.integers(0, 100, n, dtype=np.int32)
    kc = api.Column(key, "lz4").to_device()
    vc = api.Column(val, "lz4").to_device()
    ids = cuda.arange(1000, dtype=cuda.int32, device="cuda")
    ht = api.HashMap(1000).build(ids)
    agg = api.HashAggregate(16)
    res = cuda.zeros(1, dtype=cuda.int64, device="cuda")
    p = api.ScanPlan(agg=L.GX_AGG_SUM, groupby=agg, result=res).probe(kc, ht, 0, 1000).value(vc)
    with pytest.raises(GxError) as e:
        p.run_sync()
    assert e.value.status == L.GX_ERR_CAPACITY
    agg2 = api.HashAggregate(1000)
    api.ScanPlan(agg=L.GX_AGG_SUM, groupby=agg2).probe(kc, ht, 0, 1000).value(vc).run_sync()
    got = agg2.read()
    want = np.bincount(key, weights=val, minlength=1000).astype(np.int64)
    assert got == {i: int(want[i]) for i in range(1000) if (key == i).any()}
