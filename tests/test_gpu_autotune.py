"""Autotuner on the device: every grid point gives the same results (the
tuner checks that itself), the best point is the fastest, the choice
persists, and a tuned launch shape leaves batch and server results equal to
the oracle."""
import numpy as np
import pytest

from golap_public_b200 import api, autotune, workload
from oracle import workload_oracle as WO

pytestmark = pytest.mark.gpu


def test_tune_small_grid(cuda, tmp_path):
    space = {"rows_per_chunk": (262_144, 1_048_576), "threads": (128, 1024), "ht_layout": ("linear", "bucket")}
    res = autotune.tune(n_rows=3_000_000, queries_per_template=3, space=space, reps=2, n_customer=100_000,
                        n_supplier=10_000, min_rows=100_000)
    assert set(res["templates"]) == set(autotune.TEMPLATES)
    for tpl, v in res["templates"].items():
        assert len(v["points"]) == 8
        assert v["best"]["ms"] == min(p["ms"] for p in v["points"])
    f = autotune.save(res, tmp_path / "t.json")
    ch = autotune.load(f)
    assert set(ch) == set(autotune.TEMPLATES)


@pytest.mark.parametrize("threads", [0, 128, 512, 1024])
def test_launch_shapes_match_oracle(cuda, threads):
    t = workload.build_table(3_000_000, n_customer=100_000, n_supplier=10_000, rows_per_chunk=262_144,
                             ht_layouts=("bucket",))
    rng = np.random.default_rng(threads)
    specs = workload.random_queries(t, 12, rng, min_rows=100_000, max_rows=3_000_000,
                                    ht_layout={"scan": "bucket", "star": "bucket"})
    b = api.Batch([(s.plan, s.row_lo, s.row_hi) for s in specs], "shared").set_launch(threads)
    assert b.threads in (128, 256, 512, 1024) and (threads == 0 or b.threads == threads)
    b.graph()
    api.scan_check()
    for s in specs:
        assert workload.read_result(s) == WO.expected(t, s)
    if threads == 0:  # the per-batch launch tuner keeps results and picks a timed shape
        got = autotune.tune_launch(b, reps=1)
        assert got["threads"] == b.threads and got["ms"] == min(got["times_ms"].values())
        b.graph()
        api.scan_check()
        for s in specs:
            assert workload.read_result(s) == WO.expected(t, s)
    sv = api.Server(max_inflight=2, max_batch=8, batch_threads=threads)
    tickets = [sv.submit(s.plan, s.row_lo, s.row_hi, 64) for s in specs]
    for tk in tickets:
        sv.wait(tk, 120.0)
    sv.close()
    for s in specs:
        assert workload.read_result(s) == WO.expected(t, s)
