"""The two query shapes of the hot path, built on the operator API.

Q1 shape -- usecases/ssb/queries/01.hpp:54-449 (query1) with the kernel
pipeline_q1_lineorder (01.cuh:27-54):
    SUM(extended_price * discount) over fact JOIN date
    WHERE <date predicate> AND discount in [dlo,dhi] AND quantity in [qlo,qhi]
  pruning: min/max of date_key against the date range of the predicate
  (the reference prunes with MetaChecker on its date metadata, 01.hpp:263-281)

Q3 shape -- usecases/ssb/queries/03.hpp:80-592 (query3) with pipeline_q3
(03.cuh:119-170):
    SUM(revenue) GROUP BY (customer.nation, supplier.nation, year)
    WHERE customer.region = r AND supplier.region = r AND year in [ylo,yhi]
  probes in customer -> supplier -> date order, like the reference.

Q2 shape -- usecases/ssb/queries/02.cuh:103 (pipeline_q2, part -> supplier
-> date) and 02inmem.hpp:100-180:
    SUM(revenue) GROUP BY (part.brand, year)
    WHERE part.category = c AND supplier.region = r

Q4 shape -- usecases/ssb/queries/04.cuh:100 (pipeline_q4) and
04inmem.hpp:120-160 (customer -> supplier -> date -> part):
    SUM(revenue - supplycost) GROUP BY (customer.nation, year)
    WHERE customer.region = r AND supplier.region = r AND part.mfgr in [m0,m1]
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from . import _lib as L
from .api import Column, HashAggregate, HashMap, ScanPlan


def _dev(a):
    import torch

    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


@dataclass
class FactTable:
    cols: dict  # name -> Column (device resident)
    n_rows: int


def encode_fact(data: dict, codecs: dict, rows_per_chunk=1_000_000, rows_per_block=16384, lz4_segments=128,
                residency="hbm", threads=0, **kw) -> FactTable:
    cols = {}
    for name, v in data.items():
        c = Column(v, codecs.get(name, "lz4"), rows_per_chunk, rows_per_block, lz4_segments, threads=threads,
                   name=name, **kw)
        if residency:
            c.to_device(residency)
        cols[name] = c
    return FactTable(cols, len(next(iter(data.values()))))


def _launch(plan: ScanPlan, stream_group: int, stream):
    if stream_group:
        plan.launch_streamed(stream_group, stream)
    else:
        plan.launch(stream)


class Q1Query:
    """Q1-shaped fused scan over a FactTable with columns date_key, discount, quantity, extended_price."""

    def __init__(self, fact: FactTable, date: dict, date_ok: np.ndarray, date_lo: int, date_hi: int,
                 dlo: int, dhi: int, qlo: int, qhi: int, prune: bool = True, join_prune: bool = False):
        import torch

        self.fact = fact
        self.ht = HashMap(max(1, int(date_ok.sum())))
        self._dk = _dev(date["d_key"])
        self._ok = _dev(date_ok.astype(np.int32))
        self.ht.build(self._dk, None, preds=[(self._ok, 1, 1)])
        self.prune = prune
        n_chunks = fact.cols["date_key"].info.n_chunks
        self.keep = torch.zeros(n_chunks, dtype=torch.uint16, device="cuda") if prune else None
        self.result = torch.zeros(1, dtype=torch.int64, device="cuda")
        c = fact.cols
        # join pruning (usecases/ssb/queries/01.hpp:246-270): chunks whose
        # date_key min/max holds none of the date table's keys are skipped
        self.join_prune = join_prune
        self.join_keep = None
        if join_prune:
            self._jkeys = torch.empty(max(1, len(date["d_key"])), dtype=torch.int32, device="cuda")
            self._jn = torch.zeros(1, dtype=torch.int64, device="cuda")
            self.join_keep = torch.zeros(n_chunks, dtype=torch.uint16, device="cuda")
            self.refresh_join_keep()
        self.plan = ScanPlan(agg=L.GX_AGG_SUM_PRODUCT, result=self.result, keep_out=self.keep,
                             keep_chunks=self.join_keep)
        if prune:  # MetaChecker::add_minmax on the date column, evaluated by the scan launch
            self.plan.prune_minmax(c["date_key"], date_lo, date_hi)
        self.plan.probe(c["date_key"], self.ht)
        self.plan.filter(c["discount"], dlo, dhi, carry=True)
        self.plan.filter(c["quantity"], qlo, qhi)
        self.plan.value(c["extended_price"])
        self.plan.to_c()

    def refresh_join_keep(self, stream=None):
        """Join-pruning flags from the date table's current keys (no host synchronisation)."""
        from .api import MetaChecker

        self.ht.keys(self._jkeys, self._jn, stream)
        self.join_keep.zero_()
        MetaChecker(self.join_keep.numel()).add_points(self.fact.cols["date_key"], self._jkeys, self._jn,
                                                       self.join_keep, stream)

    # >0: columns in pinned host memory are streamed to HBM in groups of this
    # many chunks (gx_scan_streamed); only chunks that survive pruning cross PCIe
    stream_group = 0

    def launch(self, stream=None):
        """Enqueue: clear result, prune + fused scan (no host synchronisation)."""
        self.result.zero_()
        _launch(self.plan, self.stream_group, stream)

    def run(self, stream=None) -> int:
        self.launch(stream)
        from .api import scan_check

        scan_check(stream)
        return int(self.result.item())


def build_from_compressed(ht: HashMap, key: Column, payload: Column | None, preds=(), stream=None):
    """Fill join table `ht` from compressed dimension columns in one fused
    launch (GX_AGG_BUILD): rows passing the range predicates [(Column, lo, hi)]
    are inserted with key from `key` and payload from `payload` (or the row
    number).  Replaces pipeline_customer_q3 and its per-chunk loop
    (usecases/ssb/queries/03.cuh:94-116, 03.hpp:408-476)."""
    ht.clear(stream)
    p = ScanPlan(agg=L.GX_AGG_BUILD, build_ht=ht)
    for col, lo, hi in preds:
        p.filter(col, lo, hi)
    if payload is not None:
        p.carry(payload)
    p.value(key)
    p.launch(stream)
    return p


class Q3Query:
    """Q3-shaped star join + group-by over a FactTable with cust_key, supp_key, date_key, revenue.

    `customer` is a dict of host arrays (key, nation, region), built from
    device copies of them, or a FactTable of compressed customer columns,
    built from the compressed chunks in one fused launch (build_from_compressed)."""

    def __init__(self, fact: FactTable, customer, supplier: dict, date: dict, region: int, ylo: int, yhi: int,
                 prune: bool = True, n_nations: int = 25, ht_layout: str = "linear"):
        import torch

        self.fact = fact
        self.n_nations = n_nations
        self.ylo, self.yhi = ylo, yhi
        self.region = region
        self.cust_comp = customer if isinstance(customer, FactTable) else None
        cust_host = None if self.cust_comp else customer
        # tables sized for the rows that pass the dimension filters (a table
        # built from compressed columns is sized for every customer)
        n_c = self.cust_comp.n_rows if self.cust_comp else int((customer["region"] == region).sum())
        self.hc = HashMap(max(1, n_c), "linear" if self.cust_comp and ht_layout == "dense" else ht_layout)
        self.hs = HashMap(max(1, int((supplier["region"] == region).sum())), ht_layout)
        self.hd = HashMap(max(1, int(((date["d_year"] >= ylo) & (date["d_year"] <= yhi)).sum())), ht_layout)
        empty = np.zeros(1, np.int32)
        self._keep_alive = [_dev(cust_host["key"] if cust_host else empty),
                            _dev(cust_host["nation"] if cust_host else empty),
                            _dev(cust_host["region"] if cust_host else empty),
                            _dev(supplier["key"]), _dev(supplier["nation"]), _dev(supplier["region"]),
                            _dev(date["d_key"]), _dev(date["d_year"])]
        ck, cn, cr, sk, sn, sr, dk, dy = self._keep_alive
        self.build_customer()
        self.hs.build(sk, sn, preds=[(sr, region, region)])
        self.hd.build(dk, dy, preds=[(dy, ylo, yhi)])
        n_chunks = fact.cols["date_key"].info.n_chunks
        self.prune = prune
        self.keep = torch.zeros(n_chunks, dtype=torch.uint16, device="cuda") if prune else None
        self.ycard = yhi - ylo + 1
        self.agg = HashAggregate(n_nations * n_nations * self.ycard)
        c = fact.cols
        self.plan = ScanPlan(agg=L.GX_AGG_SUM, groupby=self.agg, keep_out=self.keep)
        if prune:
            self.plan.prune_minmax(c["date_key"], ylo * 10000 + 101, yhi * 10000 + 1231)
        self.plan.probe(c["cust_key"], self.hc, 0, n_nations)
        self.plan.probe(c["supp_key"], self.hs, 0, n_nations)
        self.plan.probe(c["date_key"], self.hd, ylo, self.ycard)
        self.plan.value(c["revenue"])
        self.plan.to_c()

    def build_customer(self, stream=None):
        """The customer join table: filtered build from device arrays, or from the
        compressed customer columns in one fused launch."""
        if self.cust_comp:
            c = self.cust_comp.cols
            build_from_compressed(self.hc, c["key"], c["nation"], [(c["region"], self.region, self.region)], stream)
        else:
            ck, cn, cr = self._keep_alive[:3]
            self.hc.build(ck, cn, preds=[(cr, self.region, self.region)], stream=stream)

    stream_group = 0  # as Q1Query.stream_group

    def launch(self, stream=None):
        self.agg.reset(stream)
        self.scan(stream)

    def scan(self, stream=None):
        """The fused scan alone (group table already reset): launched right after
        the last join-table build, its table-free work overlaps that build."""
        _launch(self.plan, self.stream_group, stream)

    def decode_key(self, k: int):
        y = k % self.ycard
        s = (k // self.ycard) % self.n_nations
        c = k // (self.ycard * self.n_nations)
        return c, s, self.ylo + y

    def run(self, stream=None) -> dict:
        """{(c_nation, s_nation, year): sum} after synchronising."""
        self.launch(stream)
        from .api import scan_check

        scan_check(stream)
        raw = self.agg.read(stream=stream)
        return {self.decode_key(k): v for k, v in raw.items()}


class _StarQuery:
    """Common part of the star-join shapes: join tables, group table, plan."""

    stream_group = 0  # as Q1Query.stream_group

    def launch(self, stream=None):
        self.agg.reset(stream)
        _launch(self.plan, self.stream_group, stream)

    def run(self, stream=None) -> dict:
        self.launch(stream)
        from .api import scan_check

        scan_check(stream)
        return {self.decode_key(k): v for k, v in self.agg.read(stream=stream).items()}

    def _tables(self, dims, ht_layout):
        """dims: name -> (keys, payload or None, filter column or None, lo, hi); builds one table each."""
        self.ht = {}
        self._keep_alive = []
        for name, (keys, pay, fcol, lo, hi) in dims.items():
            ok = np.ones(len(keys), bool) if fcol is None else (fcol >= lo) & (fcol <= hi)
            ht = HashMap(max(1, int(ok.sum())), ht_layout)
            kd = _dev(keys)
            pd = _dev(pay) if pay is not None else None
            preds = []
            if fcol is not None:
                fd = _dev(fcol)
                preds = [(fd, lo, hi)]
                self._keep_alive.append(fd)
            ht.build(kd, pd, preds=preds)
            self._keep_alive += [kd, pd]
            self.ht[name] = ht


class Q2Query(_StarQuery):
    """Q2-shaped star join over a FactTable with part_key, supp_key, date_key, revenue."""

    def __init__(self, fact: FactTable, part: dict, supplier: dict, date: dict, category: int, region: int,
                 year0: int = 1992, n_years: int = 7, n_brands: int = 1000, ht_layout: str = "linear"):
        self.year0, self.n_years = year0, n_years
        self._tables({"part": (part["key"], part["brand"], part["category"], category, category),
                      "supp": (supplier["key"], None, supplier["region"], region, region),
                      "date": (date["d_key"], date["d_year"], None, 0, 0)}, ht_layout)
        self.agg = HashAggregate(n_brands * n_years)
        c = fact.cols
        self.plan = ScanPlan(agg=L.GX_AGG_SUM, groupby=self.agg)
        self.plan.probe(c["part_key"], self.ht["part"], 0, n_brands)
        self.plan.probe(c["supp_key"], self.ht["supp"])
        self.plan.probe(c["date_key"], self.ht["date"], year0, n_years)
        self.plan.value(c["revenue"])
        self.plan.to_c()

    def decode_key(self, k: int):
        """(brand, year)"""
        return k // self.n_years, self.year0 + k % self.n_years


class Q4Query(_StarQuery):
    """Q4-shaped star join over a FactTable with cust_key, supp_key, part_key, date_key, revenue, supplycost."""

    def __init__(self, fact: FactTable, customer: dict, supplier: dict, part: dict, date: dict, region: int,
                 mfgr_lo: int, mfgr_hi: int, year0: int = 1992, n_years: int = 7, ht_layout: str = "linear"):
        self.year0, self.n_years = year0, n_years
        self._tables({"cust": (customer["key"], customer["nation"], customer["region"], region, region),
                      "supp": (supplier["key"], None, supplier["region"], region, region),
                      "date": (date["d_key"], date["d_year"], None, 0, 0),
                      "part": (part["key"], None, part["mfgr"], mfgr_lo, mfgr_hi)}, ht_layout)
        self.agg = HashAggregate(25 * n_years)
        c = fact.cols
        self.plan = ScanPlan(agg=L.GX_AGG_SUM_DIFF, groupby=self.agg)
        self.plan.probe(c["cust_key"], self.ht["cust"], 0, 25)
        self.plan.probe(c["supp_key"], self.ht["supp"])
        self.plan.probe(c["date_key"], self.ht["date"], year0, n_years)
        self.plan.probe(c["part_key"], self.ht["part"])
        self.plan.carry(c["supplycost"])
        self.plan.value(c["revenue"])
        self.plan.to_c()

    def decode_key(self, k: int):
        """(c_nation, year)"""
        return k // self.n_years, self.year0 + k % self.n_years
