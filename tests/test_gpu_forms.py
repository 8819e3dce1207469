"""Every kernel form of the single-plan scan gives the oracle's results.

gx_scan picks the warp-tile form (one warp per 1024-row tile), the pipelined
form (producer warp + 16 consumer warps), the shared form (one CTA per
2048-row tile) or the queue form (any plan); gx_scan_set_form forces one.
Each form runs the same plans here -- the Q1 shape (pipeline_q1_lineorder,
usecases/ssb/queries/01.cuh:27-54), the Q3 star join with group-by
(pipeline_q3, 03.cuh:119-170) and the Q4 profit shape (04.cuh:100) -- over
column encodings that take every read path of the warp-tile form: raw rows,
LZ4 literal runs read in place, LZ4 ranges with matches decoded per warp,
cascaded pages that are constant on a tile, with few runs, without RLE, with
delta, and ragged last blocks."""
import numpy as np
import pytest

from golap_public_b200 import api, datagen, queries
from golap_public_b200._lib import GxError
from oracle import oracle as O

pytestmark = pytest.mark.gpu
FORMS = ["warp", "pipe", "shared", "queue"]


@pytest.fixture(autouse=True)
def _auto_form():
    yield
    api.set_scan_form("auto")


def _q1(f, dd, ok, dlo, dhi, qlo, qhi):
    return O.q1(f["date_key"], f["discount"], f["quantity"], f["extended_price"], dd["d_key"], ok, dlo, dhi, qlo, qhi)


@pytest.fixture(scope="module")
def q1_tables():
    dd = datagen.date_dim()
    n = 3_300_123  # ragged last chunk and block
    sorted_f = datagen.fact_q1(n, True)
    rand_f = datagen.fact_q1(n, False)
    tabs = {
        "literal_s32": (sorted_f, queries.encode_fact(sorted_f, {"date_key": "cascaded"}, lz4_segments=32)),
        "matches_s128": (sorted_f, queries.encode_fact(sorted_f, {"date_key": "cascaded"}, lz4_segments=128,
                                                       lz4_min_match=4)),
        "unsorted_casc": (rand_f, queries.encode_fact(rand_f, {k: "cascaded" for k in rand_f}, lz4_segments=32)),
        "raw": (sorted_f, queries.encode_fact(sorted_f, {k: "none" for k in sorted_f})),
        "casc_all": (sorted_f, queries.encode_fact(sorted_f, {k: "cascaded" for k in sorted_f})),
    }
    return dd, tabs


@pytest.mark.parametrize("form", FORMS)
@pytest.mark.parametrize("tab", ["literal_s32", "matches_s128", "unsorted_casc", "raw", "casc_all"])
def test_q1_every_form(cuda, q1_tables, form, tab):
    dd, tabs = q1_tables
    f, fact = tabs[tab]
    api.set_scan_form(form)
    for ym, lo, hi, prune in ((199402, 19940201, 19940228, True), (None, 19920101, 19981231, False)):
        ok = dd["d_yearmonthnum"] == ym if ym else np.ones(len(dd["d_key"]), bool)
        q = queries.Q1Query(fact, dd, ok, lo, hi, 4, 6, 26, 35, prune=prune)
        assert q.run() == _q1(f, dd, ok, 4, 6, 26, 35), (form, tab, ym)
        if prune:
            mins, maxs = fact.cols["date_key"].minmax()
            assert q.keep.cpu().numpy().tolist() == O.minmax_keep(mins, maxs, lo, hi).tolist()


@pytest.fixture(scope="module")
def star():
    n = 2_500_000
    f = datagen.fact_q3(n, True, n_customer=300_000, n_supplier=20_000, n_part=200_000, supplycost=True)
    cust = datagen.dim_geo(300_000, datagen.SEED, 21)
    supp = datagen.dim_geo(20_000, datagen.SEED, 22)
    part = datagen.dim_part(200_000)
    dd = datagen.date_dim()
    return f, cust, supp, part, dd


@pytest.mark.parametrize("form", FORMS)
@pytest.mark.parametrize("layout", ["linear", "bucket", "dense"])
def test_q3_every_form(cuda, star, form, layout):
    f, cust, supp, part, dd = star
    fact = queries.encode_fact(f, {"date_key": "cascaded"}, lz4_segments=32)
    api.set_scan_form(form)
    q = queries.Q3Query(fact, cust, supp, dd, 3, 1993, 1996, ht_layout=layout)
    sums, counts = O.q3(f["cust_key"], f["supp_key"], f["date_key"], f["revenue"], cust["key"], cust["nation"],
                        cust["region"] == 3, supp["key"], supp["nation"], supp["region"] == 3, dd["d_key"],
                        dd["d_year"], (dd["d_year"] >= 1993) & (dd["d_year"] <= 1996), 0, 25, 0, 25, 1993, 4)
    assert q.run() == {(c, s, 1993 + y): int(sums[c, s, y]) for c, s, y in zip(*np.nonzero(counts))}


@pytest.mark.parametrize("form", ["warp", "pipe", "shared"])
def test_q4_sum_diff_every_fused_form(cuda, star, form):
    f, cust, supp, part, dd = star
    fact = queries.encode_fact(f, {"date_key": "cascaded"}, lz4_segments=32, lz4_min_match=4)
    api.set_scan_form(form)
    got = queries.Q4Query(fact, cust, supp, part, dd, 1, 0, 1).run()
    sums, counts = O.q4(f["cust_key"], f["supp_key"], f["part_key"], f["date_key"], f["revenue"], f["supplycost"],
                        cust["key"], cust["nation"], cust["region"] == 1, supp["key"], supp["region"] == 1,
                        part["key"], (part["mfgr"] >= 0) & (part["mfgr"] <= 1), dd["d_key"], dd["d_year"],
                        np.ones(len(dd["d_key"]), bool), 1992, 7)
    assert got == {(c, 1992 + y): int(sums[y, c]) for y, c in zip(*np.nonzero(counts))}


def test_count_and_forced_form_errors(cuda):
    import torch

    from golap_public_b200 import _lib as L

    f = datagen.fact_q1(1_000_000, True)
    fact = queries.encode_fact(f, {"date_key": "cascaded"}, lz4_segments=32)
    res = torch.zeros(1, dtype=torch.int64, device="cuda")
    for form in FORMS:
        api.set_scan_form(form)
        res.zero_()
        p = api.ScanPlan(agg=L.GX_AGG_COUNT, result=res)
        p.filter(fact.cols["quantity"], 10, 20).value(fact.cols["discount"], 2, 7)
        p.run_sync()
        want = int(((f["quantity"] >= 10) & (f["quantity"] <= 20) & (f["discount"] >= 2) & (f["discount"] <= 7)).sum())
        assert int(res.item()) == want, form
    # plain LZ4 blocks (no side index) are not a warp-tile shape: forcing it fails, auto falls back
    plain = queries.encode_fact(f, {"date_key": "cascaded"}, lz4_segments=1)
    dd = datagen.date_dim()
    ok = dd["d_yearmonthnum"] == 199301
    api.set_scan_form("warp")
    with pytest.raises(GxError):
        queries.Q1Query(plain, dd, ok, 19930101, 19930131, 4, 6, 26, 35).run()
    api.set_scan_form("auto")
    assert queries.Q1Query(plain, dd, ok, 19930101, 19930131, 4, 6, 26, 35).run() == _q1(f, dd, ok, 4, 6, 26, 35)


@pytest.mark.parametrize("form", FORMS)
def test_cascaded_page_kinds_every_form(cuda, form):
    # cascaded pages of every kind: increasing with varied steps (delta, no
    # RLE), a staircase (RLE + delta), runs of about six rows (RLE with
    # hundreds of runs per page), runs longer than a tile (one- and two-run
    # tiles), random (bit-packed); SUM of a filtered column must equal numpy's
    import torch

    from golap_public_b200 import _lib as L

    rng = np.random.default_rng(5)
    n = 1_234_567
    cols = {
        "inc": np.cumsum(rng.integers(1, 60, n)).astype(np.int32),
        "stairs": np.repeat(np.cumsum(rng.integers(1, 9, n // 700 + 2)), 700)[:n].astype(np.int32),
        "runs6": np.repeat(rng.integers(-5000, 5000, n // 6 + 2), 6)[:n].astype(np.int32),
        # runs longer than a warp tile: tiles of one run and of two runs, with
        # and without delta between the runs' values
        "runs1500": np.repeat(rng.integers(-(1 << 30), 1 << 30, n // 1500 + 2), 1500)[:n].astype(np.int32),
        "stairs3000": np.repeat(np.cumsum(rng.integers(1, 4, n // 3000 + 2)), 3000)[:n].astype(np.int32),
        "rand": rng.integers(-(1 << 20), 1 << 20, n).astype(np.int32),
    }
    fact = queries.encode_fact(cols, {k: "cascaded" for k in cols})
    api.set_scan_form(form)
    res = torch.zeros(1, dtype=torch.int64, device="cuda")
    for name, v in cols.items():
        lo, hi = int(np.percentile(v, 20)), int(np.percentile(v, 70))
        res.zero_()
        p = api.ScanPlan(agg=L.GX_AGG_SUM, result=res)
        p.value(fact.cols[name], lo, hi)
        p.run_sync()
        m = (v >= lo) & (v <= hi)
        assert int(res.item()) == int(v[m].astype(np.int64).sum()), (form, name)
