"""The remaining SSB flights as plans on the fused scan: the Q2 shape
(pipeline_q2, usecases/ssb/queries/02.cuh:103; query2, 02inmem.hpp:100-180)
and the Q4 shape (pipeline_q4, 04.cuh:100; query4inmem, 04inmem.hpp:80-160,
profit = revenue - supplycost through GX_AGG_SUM_DIFF).  On the reference's
SF1 data the results must equal the reference's own Q2.1 / Q4.1 (group count
and total in tests/golden/ssb_sf1_reference.json) and the oracle per group;
on the synthetic star schema they must equal the oracle."""
import json
from pathlib import Path

import numpy as np
import pytest

from golap_public_b200 import datagen, queries
from oracle import oracle as O

pytestmark = pytest.mark.gpu
GOLDEN = json.loads((Path(__file__).parent / "golden" / "ssb_sf1_reference.json").read_text())


@pytest.fixture(scope="module")
def sf1():
    return O.ssb_generate(1)


def _fact_sf1(t, S=32):
    data = {"date_key": t["lo_orderdate"], "cust_key": t["lo_custkey"], "supp_key": t["lo_suppkey"],
            "part_key": t["lo_partkey"], "revenue": t["lo_revenue"], "supplycost": t["lo_supplycost"]}
    return queries.encode_fact(data, {"date_key": "cascaded"}, lz4_segments=S)


def _dims_sf1(t):
    part = {"key": t["p_key"], "category": t["p_category"], "brand": t["p_brand1"], "mfgr": t["p_mfgr"]}
    cust = {"key": t["c_key"], "nation": t["c_nation"], "region": t["c_region"]}
    supp = {"key": t["s_key"], "nation": t["s_nation"], "region": t["s_region"]}
    date = {"d_key": t["d_key"], "d_year": t["d_year"]}
    return part, cust, supp, date


@pytest.mark.parametrize("layout", ["linear", "dense"])
def test_ssb_sf1_q2_q4_match_reference(cuda, sf1, layout):
    fact = _fact_sf1(sf1)
    part, cust, supp, date = _dims_sf1(sf1)
    ref = O.ssb_queries(sf1)
    # Q2.1: p_category MFGR#12 (code 1), s_region AMERICA (1)
    q2 = queries.Q2Query(fact, part, supp, date, 1, 1, ht_layout=layout)
    got = q2.run()
    assert len(got) == GOLDEN["q2_1_groups"] and sum(got.values()) == GOLDEN["q2_1_sum"]
    sums, counts = ref["q2_1_cells"]
    assert got == {(b, 1992 + y): int(sums[b, y]) for b, y in zip(*np.nonzero(counts))}
    # Q4.1: c_region, s_region AMERICA, p_mfgr MFGR#1 or MFGR#2 (codes 0, 1)
    q4 = queries.Q4Query(fact, cust, supp, part, date, 1, 0, 1, ht_layout=layout)
    got = q4.run()
    assert len(got) == GOLDEN["q4_1_groups"] and sum(got.values()) == GOLDEN["q4_1_sum"]
    sums, counts = ref["q4_1_cells"]
    assert got == {(c, 1992 + y): int(sums[y, c]) for y, c in zip(*np.nonzero(counts))}


def test_synthetic_q2_q4_vs_oracle(cuda):
    n = 8_000_000
    f = datagen.fact_q3(n, True, supplycost=True)
    cust = datagen.dim_geo(3_000_000, datagen.SEED, 21)
    supp = datagen.dim_geo(200_000, datagen.SEED, 22)
    part = datagen.dim_part(1_400_000)
    dd = datagen.date_dim()
    fact = queries.encode_fact(f, {"date_key": "cascaded"})
    for category, region in ((7, 3), (22, 0)):
        got = queries.Q2Query(fact, part, supp, dd, category, region).run()
        sums, counts = O.q2(f["part_key"], f["supp_key"], f["date_key"], f["revenue"], part["key"], part["brand"],
                            part["category"] == category, supp["key"], supp["region"] == region, dd["d_key"],
                            dd["d_year"], 1000, 1992, 7)
        assert got == {(b, 1992 + y): int(sums[b, y]) for b, y in zip(*np.nonzero(counts))}
    for region, m0, m1 in ((0, 2, 3), (4, 0, 4)):
        got = queries.Q4Query(fact, cust, supp, part, dd, region, m0, m1).run()
        sums, counts = O.q4(f["cust_key"], f["supp_key"], f["part_key"], f["date_key"], f["revenue"],
                            f["supplycost"], cust["key"], cust["nation"], cust["region"] == region, supp["key"],
                            supp["region"] == region, part["key"], (part["mfgr"] >= m0) & (part["mfgr"] <= m1),
                            dd["d_key"], dd["d_year"], np.ones(len(dd["d_key"]), bool), 1992, 7)
        want = {(c, 1992 + y): int(sums[y, c]) for y, c in zip(*np.nonzero(counts))}
        assert got == want


def test_carry_with_digits_needs_the_fused_forms(cuda):
    # a plan that carries a value and builds a group key runs in the shared and
    # pipelined forms; the queue form (plain LZ4 blocks) refuses it
    from golap_public_b200._lib import GxError

    n = 300_000
    f = datagen.fact_q3(n, True, n_customer=3000, n_supplier=200, n_part=1400, supplycost=True)
    cust = datagen.dim_geo(3000, datagen.SEED, 21)
    supp = datagen.dim_geo(200, datagen.SEED, 22)
    part = datagen.dim_part(1400)
    dd = datagen.date_dim()
    plain = queries.encode_fact(f, {"date_key": "cascaded"}, lz4_segments=1)
    with pytest.raises(GxError):
        queries.Q4Query(plain, cust, supp, part, dd, 1, 0, 1).run()
