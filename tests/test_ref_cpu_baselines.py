"""The reference CPU baselines that bench.py times, on the compressed bytes the
GPU path scans: LZ4 blocks decoded by the reference's LZ4CPUManager
(core/comp_cpu.hpp:22-32), cascaded blocks by the harness's decoder of this
build's format, then the reference's query1inmem / query3_inmem loop bodies
(usecases/ssb/queries/01inmem.hpp:109-130, 03inmem.hpp:120-200) with its
HostHashMap / HostHashAggregate.  Their results must equal the oracle's."""
import ctypes as C

import numpy as np
import pytest

from golap_public_b200 import api, datagen
from oracle import oracle as O

pytestmark = pytest.mark.skipif(not O.ref_available(), reason="reference harness not built")

RPC, RPB = 250_000, 16384


def _cols(data, names, codecs):
    cols = [api.Column(data[k], codecs.get(k, "lz4"), rows_per_chunk=RPC, rows_per_block=RPB) for k in names]
    keep = [(c.payload(), c.blocks(), 1 if c.codec == "lz4" else 2) for c in cols]
    return cols, keep


@pytest.mark.parametrize("min_match", [0, 4])
def test_ref_cpu_q1_on_compressed_columns(min_match):
    n = 2_000_000
    f = datagen.fact_q1(n, True)
    dd = datagen.date_dim()
    names = ["date_key", "discount", "quantity", "extended_price"]
    cols = [api.Column(f[k], "cascaded" if k == "date_key" else "lz4", rows_per_chunk=RPC, rows_per_block=RPB,
                       lz4_min_match=min_match) for k in names]
    keep = [(c.payload(), c.blocks(), 1 if c.codec == "lz4" else 2) for c in cols]
    arr = O.comp_cols(keep)
    mins, maxs = cols[0].minmax()
    for ok, lo, hi in ((dd["d_yearmonthnum"] == 199401, 19940101, 19940131), (np.ones(len(dd["d_key"]), bool),
                                                                            19920101, 19981231)):
        el, ch, rows = C.c_double(), C.c_uint64(), C.c_uint64()
        got = O.ref().ref_cpu_q1_comp(4, n, RPC, RPB, arr, O._ptr(mins), O._ptr(maxs), O._ptr(dd["d_key"]),
                                      O._ptr(ok.astype(np.uint8)), len(ok), lo, hi, 4, 6, 26, 35, C.byref(el),
                                      C.byref(ch), C.byref(rows))
        want = O.q1(f["date_key"], f["discount"], f["quantity"], f["extended_price"], dd["d_key"], ok, 4, 6, 26, 35)
        assert got == want
        assert rows.value <= n and ch.value >= 1


def test_ref_cpu_q3_on_compressed_columns():
    n = 1_500_000
    g = datagen.fact_q3(n, True, n_customer=30_000, n_supplier=2_000)
    cust = datagen.dim_geo(30_000, datagen.SEED, 21)
    supp = datagen.dim_geo(2_000, datagen.SEED, 22)
    dd = datagen.date_dim()
    names = ["date_key", "cust_key", "supp_key", "revenue"]
    cols, keep = _cols(g, names, {"date_key": "cascaded"})
    arr = O.comp_cols(keep)
    mins, maxs = cols[0].minmax()
    region, ylo, yhi = 2, 1992, 1997
    gk = np.zeros(1024, np.int64)
    gs = np.zeros(1024, np.int64)
    ng, el, ch, rows = C.c_uint64(), C.c_double(), C.c_uint64(), C.c_uint64()
    tot = O.ref().ref_cpu_q3_comp(4, n, RPC, RPB, arr, O._ptr(mins), O._ptr(maxs), O._ptr(cust["key"]),
                                  O._ptr(cust["nation"]), O._ptr(cust["region"]), len(cust["key"]),
                                  O._ptr(supp["key"]), O._ptr(supp["nation"]), O._ptr(supp["region"]),
                                  len(supp["key"]), O._ptr(dd["d_key"]), O._ptr(dd["d_year"]), len(dd["d_key"]),
                                  region, ylo, yhi, O._ptr(gk), O._ptr(gs), len(gk), C.byref(ng), C.byref(el),
                                  C.byref(ch), C.byref(rows))
    sums, counts = O.q3(g["cust_key"], g["supp_key"], g["date_key"], g["revenue"], cust["key"], cust["nation"],
                        cust["region"] == region, supp["key"], supp["nation"], supp["region"] == region,
                        dd["d_key"], dd["d_year"], (dd["d_year"] >= ylo) & (dd["d_year"] <= yhi), 0, 25, 0, 25,
                        ylo, yhi - ylo + 1)
    ny = yhi - ylo + 1
    want = {(c * 25 + s) * ny + y: int(sums[c, s, y]) for c, s, y in zip(*np.nonzero(counts))}
    got = {int(gk[i]): int(gs[i]) for i in range(ng.value)}
    assert got == want
    assert tot == sum(want.values())
