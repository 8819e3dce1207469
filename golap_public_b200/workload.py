"""Query mix of the batched and serving forms over one resident table.

The table is one wide fact table (date-sorted, compressed per 1M-row chunk)
with every column the three templates need, plus the dimension tables whose
join tables are built once and stay resident:

  scan      (Q1 shape, usecases/ssb/queries/01.hpp:54): a random month or
            year, discount band of 3, quantity band of 10;
            SUM(extended_price * discount); min/max pruning on date_key
  star      (Q3 shape, usecases/ssb/queries/03.hpp:80): random region, year
            range; SUM(revenue) GROUP BY (c_nation, s_nation, year)
  highcard  SUM(revenue) GROUP BY part_key over a year range, part_key drawn
            Zipf(1.1) over 1.4M keys (~1.4M groups at full size)

Each query covers a fact slice [row_lo, row_hi).  Date predicates are a
FILTER on date_key folded into the PROBE of the full date table (whose
payload is the year), so no per-query table build is needed; customer and
supplier tables exist per region (5 each).
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

from . import _lib as L
from . import datagen
from .api import Column, HashAggregate, HashMap, ScanPlan

N_NATIONS = 25
YEARS = (1992, 1998)  # date dimension spans 1992-01-01 .. 1998-12-31 (2,556 days)
PART_KEYS = 1_400_000


def _dev(a):
    import torch

    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


@dataclass
class WideTable:
    n_rows: int
    data: dict                      # host columns (kept for checking)
    cols: dict                      # name -> Column (device)
    dims: dict                      # customer / supplier / date dicts
    rows_per_chunk: int = 1_000_000
    ht: dict = field(default_factory=dict)  # layout -> {"date": HashMap, "cust": [5], "supp": [5]}
    _keep: list = field(default_factory=list)

    @property
    def ht_date(self) -> HashMap:
        return self.ht["linear"]["date"]

    @property
    def ht_cust(self) -> list:
        return self.ht["linear"]["cust"]

    @property
    def ht_supp(self) -> list:
        return self.ht["linear"]["supp"]


def generate(n_rows: int, seed: int = datagen.SEED, n_customer: int = 3_000_000, n_supplier: int = 200_000) -> dict:
    """Host columns of the wide fact table (seeded)."""
    f1 = datagen.fact_q1(n_rows, True, seed=seed)
    f3 = datagen.fact_q3(n_rows, True, seed=seed, n_customer=n_customer, n_supplier=n_supplier)
    return {"date_key": f1["date_key"], "discount": f1["discount"], "quantity": f1["quantity"],
            "extended_price": f1["extended_price"], "cust_key": f3["cust_key"], "supp_key": f3["supp_key"],
            "revenue": f3["revenue"],
            "part_key": datagen.zipf_keys(n_rows, PART_KEYS, 1.1, seed=seed)}


def build_table(n_rows: int, seed: int = datagen.SEED, n_customer: int = 3_000_000, n_supplier: int = 200_000,
                lz4_segments: int = 128, residency: str = "hbm", threads: int = 0, rows_per_chunk: int = 1_000_000,
                ht_layouts=("linear",), data: dict | None = None) -> WideTable:
    """Encode and load the wide table; join tables are built once per layout
    in ht_layouts ("linear" is always built).  `data` reuses host columns
    from generate() (same n_rows, seed and dimension sizes)."""
    if data is None:
        data = generate(n_rows, seed, n_customer, n_supplier)
    cols = {}
    for name, v in data.items():
        c = Column(v, "cascaded" if name == "date_key" else "lz4", rows_per_chunk, lz4_segments=lz4_segments,
                   threads=threads, name=name)
        if residency:
            c.to_device(residency)
        cols[name] = c
    dims = {"customer": datagen.dim_geo(n_customer, seed, 21), "supplier": datagen.dim_geo(n_supplier, seed, 22),
            "date": datagen.date_dim()}
    t = WideTable(n_rows, data, cols, dims, rows_per_chunk)
    dd = dims["date"]
    dk, dy = _dev(dd["d_key"]), _dev(dd["d_year"])
    t._keep += [dk, dy]
    dev = {}
    for name in ("customer", "supplier"):
        d = dims[name]
        dev[name] = (_dev(d["key"]), _dev(d["nation"]), _dev(d["region"]))
        t._keep += list(dev[name])
    for layout in dict.fromkeys(("linear",) + tuple(ht_layouts)):
        hts = {"date": HashMap(len(dd["d_key"]), layout).build(dk, dy), "cust": [], "supp": []}
        for name, key in (("customer", "cust"), ("supplier", "supp")):
            k, nat, reg = dev[name]
            for r in range(5):
                n_r = max(1, int((dims[name]["region"] == r).sum()))
                hts[key].append(HashMap(n_r, layout).build(k, nat, preds=[(reg, r, r)]))
        t.ht[layout] = hts
    return t


@dataclass
class QuerySpec:
    template: str
    row_lo: int
    row_hi: int
    params: dict
    plan: ScanPlan = None
    result: object = None    # device int64 (scalar)
    groups: HashAggregate = None


def _month_range(rng):
    y = int(rng.integers(YEARS[0], YEARS[1] + 1))
    m = int(rng.integers(1, 13))
    return y * 10000 + m * 100 + 1, y * 10000 + m * 100 + 31


def make_query(t: WideTable, template: str, rng, row_lo: int, row_hi: int, ht_layout: str = "linear") -> QuerySpec:
    import torch

    c = t.cols
    hts = t.ht[ht_layout]
    if template == "scan":
        if rng.random() < 0.5:
            dlo, dhi = _month_range(rng)
        else:
            y = int(rng.integers(YEARS[0], YEARS[1] + 1))
            dlo, dhi = y * 10000 + 101, y * 10000 + 1231
        d0 = int(rng.integers(0, 9))
        q0 = int(rng.integers(1, 42))
        spec = QuerySpec("scan", row_lo, row_hi, {"date": (dlo, dhi), "disc": (d0, d0 + 2), "qty": (q0, q0 + 9)})
        spec.result = torch.zeros(1, dtype=torch.int64, device="cuda")
        p = ScanPlan(agg=L.GX_AGG_SUM_PRODUCT, result=spec.result)
        p.prune_minmax(c["date_key"], dlo, dhi)
        p.steps.append(_step(c["date_key"], L.GX_STEP_FILTER | L.GX_STEP_PROBE, dlo, dhi, hts["date"]))
        p.filter(c["discount"], d0, d0 + 2, carry=True).filter(c["quantity"], q0, q0 + 9).value(c["extended_price"])
    elif template == "star":
        r = int(rng.integers(0, 5))
        y1 = int(rng.integers(YEARS[0], YEARS[1] + 1))
        y2 = int(rng.integers(y1, YEARS[1] + 1))
        spec = QuerySpec("star", row_lo, row_hi, {"region": r, "years": (y1, y2)})
        spec.groups = HashAggregate(N_NATIONS * N_NATIONS * (y2 - y1 + 1))
        p = ScanPlan(agg=L.GX_AGG_SUM, groupby=spec.groups)
        p.prune_minmax(c["date_key"], y1 * 10000 + 101, y2 * 10000 + 1231)
        p.probe(c["cust_key"], hts["cust"][r], 0, N_NATIONS).probe(c["supp_key"], hts["supp"][r], 0, N_NATIONS)
        p.steps.append(_step(c["date_key"], L.GX_STEP_FILTER | L.GX_STEP_PROBE, y1 * 10000 + 101, y2 * 10000 + 1231,
                             hts["date"], y1, y2 - y1 + 1))
        p.value(c["revenue"])
    elif template == "highcard":
        y1 = int(rng.integers(YEARS[0], YEARS[1] + 1))
        y2 = min(YEARS[1], y1 + int(rng.integers(0, 3)))
        spec = QuerySpec("highcard", row_lo, row_hi, {"years": (y1, y2)})
        spec.groups = HashAggregate(min(PART_KEYS, max(1, row_hi - row_lo)))
        p = ScanPlan(agg=L.GX_AGG_SUM, groupby=spec.groups)
        p.prune_minmax(c["date_key"], y1 * 10000 + 101, y2 * 10000 + 1231)
        p.filter(c["date_key"], y1 * 10000 + 101, y2 * 10000 + 1231)
        p.group(c["part_key"], 1, PART_KEYS).value(c["revenue"])
    else:
        raise ValueError(template)
    spec.plan = p
    return spec


def _step(col, flags, lo, hi, ht, digit_base=0, digit_card=0):
    from .api import Step

    return Step(col, flags, lo, hi, ht, digit_base, digit_card)


def random_queries(t: WideTable, n: int, rng, min_rows: int = 1_000_000, max_rows: int = 100_000_000,
                   mix=(("scan", 0.6), ("star", 0.3), ("highcard", 0.1)), ht_layout=None) -> list:
    """ht_layout: None (linear), a layout name, or {template: layout}."""
    """n queries; slice sizes log-uniform in [min_rows, max_rows] (clamped to the table)."""
    names = [m[0] for m in mix]
    probs = np.array([m[1] for m in mix], dtype=np.float64)
    probs /= probs.sum()
    hi_cap = min(max_rows, t.n_rows)
    lo_cap = min(min_rows, hi_cap)
    out = []
    for _ in range(n):
        size = int(round(math.exp(rng.uniform(math.log(lo_cap), math.log(hi_cap)))))
        start = int(rng.integers(0, t.n_rows - size + 1))
        tpl = str(rng.choice(names, p=probs))
        lay = (ht_layout.get(tpl, "linear") if isinstance(ht_layout, dict) else ht_layout) or "linear"
        out.append(make_query(t, tpl, rng, start, start + size, lay))
    return out


def read_result(spec: QuerySpec):
    """Scalar int for scan queries, {group key: sum} for grouped ones."""
    if spec.groups is None:
        return int(spec.result.item())
    return spec.groups.read()
