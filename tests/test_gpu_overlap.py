"""The single-plan scan may start while the kernel just before it on the
stream still runs (programmatic dependent launch).  Whatever that kernel
writes -- the join table, the result word, the chunk keep flags -- the scan
must see, and the flags it writes must not be overwritten by it: the Q1
shape (pipeline_q1_lineorder, usecases/ssb/queries/01.cuh:27-54) run right
after the writes, against the oracle."""
import numpy as np
import pytest

from golap_public_b200 import _lib as L
from golap_public_b200 import api, datagen, queries
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def test_scan_sees_the_kernel_just_before(cuda):
    torch = cuda
    f = datagen.fact_q1(3_000_000, True)
    dd = datagen.date_dim()
    fact = queries.encode_fact(f, {"date_key": "cascaded"})
    c = fact.cols
    n_chunks = c["date_key"].info.n_chunks
    dk = torch.from_numpy(dd["d_key"]).cuda()
    ok_dev = torch.zeros(len(dd["d_key"]), dtype=torch.int32, device="cuda")
    ht = api.HashMap(len(dd["d_key"]))
    res = torch.zeros(1, dtype=torch.int64, device="cuda")
    keep = torch.ones(n_chunks, dtype=torch.uint16, device="cuda")
    keep_out = torch.zeros(n_chunks, dtype=torch.uint16, device="cuda")

    def plan(keep_in):
        p = api.ScanPlan(agg=L.GX_AGG_SUM_PRODUCT, result=res, keep_chunks=keep_in, keep_out=keep_out)
        p.probe(c["date_key"], ht).filter(c["discount"], 4, 6, carry=True).filter(c["quantity"], 26, 35)
        return p.value(c["extended_price"])

    def want(ok):
        return O.q1(f["date_key"], f["discount"], f["quantity"], f["extended_price"], dd["d_key"], ok, 4, 6, 26, 35)

    for p in (plan(None), plan(keep)):
        for ok in (dd["d_yearmonthnum"] == 199401, dd["d_year"] == 1993, dd["d_year"] >= 1992):
            ok_dev.copy_(torch.from_numpy(ok.astype(np.int32)))
            for _ in range(3):
                res.fill_(777)
                keep.fill_(1)
                keep_out.fill_(7)
                res.zero_()
                ht.build(dk, None, preds=[(ok_dev, 1, 1)])  # the kernel just before the scan
                p.launch()
                api.scan_check()
                assert int(res.item()) == want(ok)
                assert int(keep_out.sum().item()) == n_chunks
    # keep flags cleared by the kernel just before the scan: nothing is scanned
    p = plan(keep)
    res.zero_()
    keep.zero_()
    p.launch()
    api.scan_check()
    assert int(res.item()) == 0
    assert int(keep_out.sum().item()) == 0
