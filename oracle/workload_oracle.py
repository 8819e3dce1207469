"""Expected results of the batched/serving query mix (test infrastructure).

Restates, on the CPU, the three query templates of
golap_public_b200/workload.py over a query's fact slice, with the oracle's
Q1 (usecases/ssb/queries/01inmem.hpp:83-130) and Q3
(usecases/ssb/queries/03inmem.hpp:120-200) restatements and a dense group-by
sum for the part_key template.  Used only by tests/ as the checker.
"""
import numpy as np

from . import oracle as O

N_NATIONS = 25
PART_KEYS = 1_400_000


def expected(t, spec):
    """Oracle result of a query on its fact slice [row_lo, row_hi)."""
    d = {k: v[spec.row_lo:spec.row_hi] for k, v in t.data.items()}
    dd = t.dims["date"]
    if spec.template == "scan":
        dlo, dhi = spec.params["date"]
        ok = (dd["d_key"] >= dlo) & (dd["d_key"] <= dhi)
        return O.q1(d["date_key"], d["discount"], d["quantity"], d["extended_price"], dd["d_key"], ok,
                    *spec.params["disc"], *spec.params["qty"])
    if spec.template == "star":
        r = spec.params["region"]
        y1, y2 = spec.params["years"]
        cu, su = t.dims["customer"], t.dims["supplier"]
        sums, counts = O.q3(d["cust_key"], d["supp_key"], d["date_key"], d["revenue"], cu["key"], cu["nation"],
                            cu["region"] == r, su["key"], su["nation"], su["region"] == r, dd["d_key"], dd["d_year"],
                            (dd["d_year"] >= y1) & (dd["d_year"] <= y2), 0, N_NATIONS, 0, N_NATIONS, y1, y2 - y1 + 1)
        yc = y2 - y1 + 1
        return {(cn * N_NATIONS + sn) * yc + y: int(sums[cn, sn, y]) for cn, sn, y in zip(*np.nonzero(counts))}
    y1, y2 = spec.params["years"]
    m = (d["date_key"] >= y1 * 10000 + 101) & (d["date_key"] <= y2 * 10000 + 1231)
    keys = (d["part_key"][m].astype(np.int64) - 1)
    vals = d["revenue"][m].astype(np.int64)
    sums = np.zeros(PART_KEYS, np.int64)
    assert O.lib().or_group_sum_dense(O._ptr(keys), O._ptr(vals), len(keys), O._ptr(sums), PART_KEYS) == 0
    present = np.bincount(keys, minlength=PART_KEYS) > 0
    return {int(k): int(sums[k]) for k in np.nonzero(present)[0]}
