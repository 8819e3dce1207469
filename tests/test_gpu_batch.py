"""Batched form: many plans on row slices of one resident table in one
persistent launch (and as a replayed CUDA graph), in both execution forms
(per-query work items, and the shared scan that decodes each tile once for
all queries).  Every query's result must equal the oracle on its slice,
alone and in the mix."""
import numpy as np
import pytest

from golap_public_b200 import _lib as L
from golap_public_b200 import api, workload
from golap_public_b200._lib import GxError
from oracle import workload_oracle as WO

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def table(cuda):
    return workload.build_table(6_000_000, n_customer=300_000, n_supplier=20_000, ht_layouts=("linear", "dense"))


def _check(t, specs):
    for s in specs:
        assert workload.read_result(s) == WO.expected(t, s), (s.template, s.row_lo, s.row_hi, s.params)


MODES = ["queue", "shared"]


@pytest.mark.parametrize("mode", MODES)
def test_batch_mixed_queries(table, mode):
    rng = np.random.default_rng(5)
    specs = workload.random_queries(table, 48, rng, min_rows=100_000, max_rows=6_000_000)
    assert {s.template for s in specs} >= {"scan", "star"}
    b = api.Batch([(s.plan, s.row_lo, s.row_hi) for s in specs], mode)
    assert b.mode == mode
    b.run()
    api.scan_check()
    _check(table, specs)
    # replayed graph: results are cleared and recomputed identically
    for _ in range(2):
        b.graph()
        api.scan_check()
    _check(table, specs)


@pytest.mark.parametrize("mode", MODES)
def test_batch_dense_join_tables(table, mode):
    # the same templates probing dense join tables (date, customer and
    # supplier keys fill their ranges)
    rng = np.random.default_rng(15)
    specs = workload.random_queries(table, 40, rng, min_rows=100_000, max_rows=6_000_000, ht_layout="dense")
    assert {s.template for s in specs} >= {"scan", "star"}
    b = api.Batch([(s.plan, s.row_lo, s.row_hi) for s in specs], mode)
    b.run()
    api.scan_check()
    _check(table, specs)


@pytest.mark.parametrize("mode", MODES)
def test_each_query_alone_equals_in_mix(table, mode):
    rng = np.random.default_rng(11)
    specs = workload.random_queries(table, 12, rng, min_rows=50_000, max_rows=3_000_000,
                                    mix=(("scan", 0.4), ("star", 0.4), ("highcard", 0.2)))
    mixed = api.Batch([(s.plan, s.row_lo, s.row_hi) for s in specs], mode)
    mixed.run()
    api.scan_check()
    in_mix = [workload.read_result(s) for s in specs]
    for s, want in zip(specs, in_mix):
        alone = api.Batch([(s.plan, s.row_lo, s.row_hi)], mode)
        alone.run()
        api.scan_check()
        assert workload.read_result(s) == want == WO.expected(table, s)


@pytest.mark.parametrize("mode", MODES)
def test_highcard_group_by_part_key(table, mode):
    rng = np.random.default_rng(2)
    s = workload.make_query(table, "highcard", rng, 0, table.n_rows)
    b = api.Batch([(s.plan, 0, table.n_rows)], mode)
    b.run()
    api.scan_check()
    got = workload.read_result(s)
    assert len(got) > 100_000  # Zipf(1.1) over 1.4M keys: many distinct groups
    assert got == WO.expected(table, s)


@pytest.mark.parametrize("mode", MODES)
def test_empty_and_edge_slices(table, mode):
    rng = np.random.default_rng(3)
    specs = [workload.make_query(table, "scan", rng, 0, 0), workload.make_query(table, "scan", rng, 5, 6),
             workload.make_query(table, "star", rng, table.n_rows - 1, table.n_rows),
             workload.make_query(table, "scan", rng, 999_999, 1_000_001)]
    b = api.Batch([(s.plan, s.row_lo, s.row_hi) for s in specs], mode)
    b.run()
    api.scan_check()
    _check(table, specs)


def test_shared_rows_equal_queue_rows(table):
    # both forms count, per query, the slice rows of every tile they evaluate
    rng = np.random.default_rng(8)
    specs = workload.random_queries(table, 16, rng, min_rows=100_000, max_rows=6_000_000,
                                    mix=(("star", 0.5), ("highcard", 0.5)))
    got = {}
    for mode in MODES:
        b = api.Batch([(s.plan, s.row_lo, s.row_hi) for s in specs], mode)
        b.run()
        api.scan_check()
        got[mode] = (b.rows(), [workload.read_result(s) for s in specs])
    assert got["queue"] == got["shared"]


def test_shared_form_eligibility(table, cuda):
    rng = np.random.default_rng(4)
    s = workload.make_query(table, "scan", rng, 0, table.n_rows)
    assert api.Batch([(s.plan, 0, table.n_rows)]).mode == "shared"  # auto picks the shared form
    # a plan with a VALUE step before its last step does not qualify
    res = cuda.zeros(1, dtype=cuda.int64, device="cuda")
    p = api.ScanPlan(agg=L.GX_AGG_SUM, result=res).value(table.cols["quantity"]).filter(table.cols["discount"], 0, 5)
    assert api.Batch([(p, 0, 1000)]).mode == "queue"
    with pytest.raises(GxError) as e:
        api.Batch([(p, 0, 1000)], "shared")
    assert e.value.status == L.GX_ERR_INVALID and "VALUE" in str(e.value)


@pytest.mark.parametrize("threads", [256, 512, 1024])
def test_shared_small_blocks_many_segments(cuda, threads):
    # 4096-row blocks of 128 segments (32 rows each) with fixed 4-byte matches:
    # many short, match-heavy segments per tile on every CTA size
    rng = np.random.default_rng(threads)
    n = 1_000_000
    a = rng.integers(0, 4, n, dtype=np.int32)
    v = rng.integers(0, 6, n, dtype=np.int32)
    ca = api.Column(a, "lz4", rows_per_chunk=65_536, rows_per_block=4096, lz4_segments=128, lz4_min_match=4)
    cv = api.Column(v, "lz4", rows_per_chunk=65_536, rows_per_block=4096, lz4_segments=128, lz4_min_match=4)
    for c in (ca, cv):
        c.to_device("hbm")
    res = [cuda.zeros(1, dtype=cuda.int64, device="cuda") for _ in range(3)]
    slices = [(0, n), (12_345, 700_001), (500_000, 500_100)]
    plans = [api.ScanPlan(agg=L.GX_AGG_SUM, result=r).filter(ca, 1, 2).value(cv) for r in res]
    b = api.Batch([(p, lo, hi) for p, (lo, hi) in zip(plans, slices)], "shared").set_launch(threads)
    b.run()
    api.scan_check()
    for r, (lo, hi) in zip(res, slices):
        m = (a[lo:hi] >= 1) & (a[lo:hi] <= 2)
        assert int(r.item()) == int(v[lo:hi][m].astype(np.int64).sum())


class _FixedDraws:
    """Stands in for the generator of workload.make_query: fixed draws, so
    that many queries share their first steps."""

    def __init__(self, ints, u=0.9):
        self.ints = iter(ints)
        self.u = u

    def random(self):
        return self.u

    def integers(self, lo, hi=None):
        return next(self.ints)


def test_shared_prefix_groups(table):
    # 40 scans with one date range and one discount filter (two shared steps,
    # the second carries the discount), 40 star joins over one region (two
    # shared probes with group-key digits), then random queries; more than
    # two mask words of queries, so some groups are split at a word boundary.
    # Slices include short ones inside one tile with gaps between them.
    rng = np.random.default_rng(21)
    n = table.n_rows
    specs = []
    for i in range(40):
        lo = int(rng.integers(0, n - 1))
        hi = lo + (int(rng.integers(1, 3000)) if i % 3 == 0 else int(rng.integers(1, n - lo + 1)))
        specs.append(workload.make_query(table, "scan", _FixedDraws([1994, 3, int(rng.integers(1, 42))]), lo, min(hi, n)))
    for i in range(40):
        if i % 4 == 1:  # 200-row slices at a few places: several per tile, with gaps
            lo = 4096 * (10, 500, 1200)[i % 3] + 1000 + 300 * (i % 5)
            hi = lo + 200
        else:
            lo = 4096 * int(rng.integers(0, n // 4096)) + (0 if i % 2 else 1000 + 300 * (i % 5))
            hi = lo + int(rng.integers(1, n - lo + 1))
        y1 = int(rng.integers(1992, 1999))
        specs.append(workload.make_query(table, "star", _FixedDraws([1, y1, int(rng.integers(y1, 1999))]), lo, min(hi, n)))
    specs += workload.random_queries(table, 20, rng, min_rows=1000, max_rows=n)
    order = rng.permutation(len(specs))
    specs = [specs[i] for i in order]
    got = {}
    for mode in MODES:
        b = api.Batch([(s.plan, s.row_lo, s.row_hi) for s in specs], mode)
        assert b.mode == mode
        b.run()
        api.scan_check()
        first = [workload.read_result(s) for s in specs]
        b.graph()
        b.graph()
        api.scan_check()
        got[mode] = (b.rows(), [workload.read_result(s) for s in specs])
        assert got[mode][1] == first
    assert got["queue"] == got["shared"]
    _check(table, specs)
