"""gx_scan_static: the allocation-free scan entry point (its work list lives
in a file-scope device array).  Called through the C ABI, it must give the
same results as gx_scan on two calls in a row, and reject plans whose chunk
count exceeds GX_SCAN_STATIC_MAX_CHUNKS.  Collected last so it also runs
after every other GPU test in the same process."""
import ctypes as C

import numpy as np
import pytest

from golap_public_b200 import _lib as L
from golap_public_b200 import api, datagen, queries
from golap_public_b200._lib import GxError, check
from oracle import oracle as O

pytestmark = pytest.mark.gpu
MAX_CHUNKS = 16384  # GX_SCAN_STATIC_MAX_CHUNKS in include/gx.h


def _run(entry, plan, result, keep=None):
    result.zero_()
    if keep is not None:
        keep.fill_(7)
    check(getattr(L.lib(), entry)(C.byref(plan.to_c()), None))
    api.scan_check()
    return int(result.item()), (keep.cpu().numpy().tolist() if keep is not None else None)


def test_static_equals_scan_q1_pruned(cuda):
    # 12M rows sorted by date; cascaded date, LZ4 others; March 1995 (pruned)
    f = datagen.fact_q1(12_000_000, True)
    dd = datagen.date_dim()
    fact = queries.encode_fact(f, {"date_key": "cascaded"})
    ok = dd["d_yearmonthnum"] == 199503
    q = queries.Q1Query(fact, dd, ok, 19950301, 19950331, 4, 6, 26, 35, prune=True)
    want = O.q1(f["date_key"], f["discount"], f["quantity"], f["extended_price"], dd["d_key"], ok, 4, 6, 26, 35)
    got = []
    for _ in range(2):  # alternate the two entry points, two calls of each in a row
        got.append(_run("gx_scan", q.plan, q.result, q.keep))
        got.append(_run("gx_scan_static", q.plan, q.result, q.keep))
    got.append(_run("gx_scan_static", q.plan, q.result, q.keep))
    assert all(g == got[0] for g in got)
    assert got[0][0] == want
    mins, maxs = fact.cols["date_key"].minmax()
    assert got[0][1] == O.minmax_keep(mins, maxs, 19950301, 19950331).tolist()
    assert 1 <= sum(got[0][1]) < len(got[0][1])


def test_static_leaves_device_memory_unchanged(cuda):
    # the property the entry point exists for: after a first call (which loads
    # the kernels' code and looks up the array's address), further calls take
    # no device memory -- no pool allocation, no cudaMalloc
    f = datagen.fact_q1(6_000_000, True)
    dd = datagen.date_dim()
    fact = queries.encode_fact(f, {"date_key": "cascaded"})
    ok = dd["d_year"] == 1996
    q = queries.Q1Query(fact, dd, ok, 19960101, 19961231, 1, 3, 0, 24, prune=True)
    first = _run("gx_scan_static", q.plan, q.result, q.keep)
    cuda.cuda.synchronize()
    free0 = cuda.cuda.mem_get_info()[0]
    for _ in range(5):
        assert _run("gx_scan_static", q.plan, q.result, q.keep) == first
    cuda.cuda.synchronize()
    assert cuda.cuda.mem_get_info()[0] == free0


def test_static_equals_scan_grouped(cuda):
    f = datagen.fact_q3(5_000_000, True, n_customer=300_000, n_supplier=20_000)
    cust = datagen.dim_geo(300_000, datagen.SEED, 21)
    supp = datagen.dim_geo(20_000, datagen.SEED, 22)
    dd = datagen.date_dim()
    fact = queries.encode_fact(f, {"date_key": "cascaded"})
    q = queries.Q3Query(fact, cust, supp, dd, 2, 1993, 1996)
    results = []
    for entry in ("gx_scan", "gx_scan_static", "gx_scan_static", "gx_scan"):
        q.agg.reset()
        check(getattr(L.lib(), entry)(C.byref(q.plan.to_c()), None))
        api.scan_check()
        results.append(q.agg.read())
    assert results[0] and all(r == results[0] for r in results)


def _count_plan(col, res):
    return api.ScanPlan(agg=L.GX_AGG_COUNT, result=res).value(col, 100, 900)


def test_static_chunk_limit(cuda):
    rng = np.random.default_rng(17)
    res = cuda.zeros(1, dtype=cuda.int64, device="cuda")
    # exactly the limit: accepted, equal to gx_scan and to the host count
    v = rng.integers(0, 1000, MAX_CHUNKS * 64, dtype=np.int32)
    col = api.Column(v, "none", rows_per_chunk=64, rows_per_block=64)
    col.to_device("hbm")
    assert col.info.n_chunks == MAX_CHUNKS
    p = _count_plan(col, res)
    want = int(((v >= 100) & (v <= 900)).sum())
    assert _run("gx_scan_static", p, res)[0] == want
    assert _run("gx_scan", p, res)[0] == want
    assert _run("gx_scan_static", p, res)[0] == want
    # one chunk more: rejected before anything is launched
    v2 = rng.integers(0, 1000, MAX_CHUNKS * 64 + 1, dtype=np.int32)
    col2 = api.Column(v2, "none", rows_per_chunk=64, rows_per_block=64)
    col2.to_device("hbm")
    assert col2.info.n_chunks == MAX_CHUNKS + 1
    res.fill_(-5)
    with pytest.raises(GxError) as e:
        check(L.lib().gx_scan_static(C.byref(_count_plan(col2, res).to_c()), None))
    assert e.value.status == L.GX_ERR_INVALID
    assert "exceed" in str(e.value)
    assert int(res.item()) == -5
    # gx_scan still takes it
    assert _run("gx_scan", _count_plan(col2, res), res)[0] == int(((v2 >= 100) & (v2 <= 900)).sum())
