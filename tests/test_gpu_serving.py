"""Serving loop: requests submitted while others run are admitted as slots
and memory free up, overlap on the device, and each result equals the same
request run alone (and the oracle).  Admission keeps the admitted bytes
within the budget; a request larger than the budget is rejected."""
import numpy as np
import pytest

from golap_public_b200 import _lib as L
from golap_public_b200 import api, workload
from golap_public_b200._lib import GxError
from oracle import workload_oracle as WO

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def table(cuda):
    return workload.build_table(4_000_000, n_customer=300_000, n_supplier=20_000)


def _hbm(spec):
    return 8 if spec.groups is None else 16 * (2 * spec.groups.max_groups)


def test_mixed_requests_match_alone_and_oracle(table):
    rng = np.random.default_rng(21)
    specs = workload.random_queries(table, 64, rng, min_rows=50_000, max_rows=4_000_000)
    sv = api.Server(max_inflight=4, max_batch=16)
    tickets = [sv.submit(s.plan, s.row_lo, s.row_hi, _hbm(s)) for s in specs]
    lat = [sv.wait(t, 120.0) for t in tickets]
    api.scan_check()
    st = sv.stats()
    sv.close()
    assert st["completed"] == 64 and st["rejected"] == 0
    assert st["batches"] < 64  # requests were batched
    assert all(x > 0 for x in lat)
    in_mix = [workload.read_result(s) for s in specs]
    for s, got in zip(specs, in_mix):
        assert got == WO.expected(table, s)
    for s, got in list(zip(specs, in_mix))[:16]:
        b = api.Batch([(s.plan, s.row_lo, s.row_hi)])
        b.run()
        api.scan_check()
        assert workload.read_result(s) == got


def test_admission_budget_and_rejection(table):
    rng = np.random.default_rng(4)
    specs = workload.random_queries(table, 12, rng, min_rows=100_000, max_rows=1_000_000,
                                    mix=(("star", 1.0),))
    need = max(_hbm(s) for s in specs)
    # budget fits one request at a time: all still complete, peak stays within budget
    sv = api.Server(max_inflight=4, max_batch=8, hbm_budget=need)
    tickets = [sv.submit(s.plan, s.row_lo, s.row_hi, _hbm(s)) for s in specs]
    for t in tickets:
        sv.wait(t, 120.0)
    st = sv.stats()
    assert st["completed"] == 12 and st["hbm_peak"] <= need and st["hbm_in_use"] == 0
    for s in specs:
        assert workload.read_result(s) == WO.expected(table, s)
    with pytest.raises(GxError) as e:
        sv.submit(specs[0].plan, 0, 10, need + 1)
    assert e.value.status == L.GX_ERR_NOMEM
    assert sv.stats()["rejected"] == 1
    sv.close()


def test_wait_timeout_and_unknown_ticket(table):
    sv = api.Server(max_inflight=1, max_batch=1)
    with pytest.raises(GxError) as e:
        sv.wait(12345, 0.1)
    assert e.value.status == L.GX_ERR_INVALID
    sv.close()
