"""Seeded synthetic star-schema data with the shapes of the measured workloads.

The reference measures on SSB data from its own simplified generator
(usecases/ssb/data/SSB_def.hpp); this module draws int32 columns with the
distributions of the benchmark configurations instead (numpy PCG64, one
independent stream per column, default seed 0xBEE5BEE5):

  fact (Q1 shape): date_key (yyyymmdd of a day uniform over 2,556 days from
                   1992-01-01), quantity U[1,50], discount U[0,10],
                   extended_price U[90000,10494950]
  fact (Q3 shape): cust_key U[1,3M], supp_key U[1,200k], part_key U[1,1.4M],
                   date_key, revenue U[100,1000000]
  customer / supplier: key 1..N, nation U[0,25), region = region of nation
                   (5 nations per region, the SSB nation->region map)
  part:            key 1..N, category U[0,25), mfgr = category // 5,
                   brand = 40 * category + U[0,40)
  date:            2,556 rows: key, year, yearmonthnum
Sorted facts are produced directly in date order (multinomial day counts),
which is the same distribution as sorting the unsorted table by date_key.
"""
from __future__ import annotations

import datetime as _dt

import numpy as np

SEED = 0xBEE5BEE5
N_DAYS = 2556
# region index of each nation (alphabetical SSB nation order)
NATION_REGION = np.array([0, 1, 1, 1, 2, 4, 0, 3, 3, 2, 2, 4, 4, 2, 4, 0, 0, 0, 1, 3, 3, 4, 3, 1, 2], np.int32)


def _rng(seed: int, stream: int) -> np.random.Generator:
    return np.random.Generator(np.random.PCG64(np.random.SeedSequence([seed, stream])))


def date_dim(n_days: int = N_DAYS) -> dict:
    d0 = _dt.date(1992, 1, 1)
    days = [d0 + _dt.timedelta(days=i) for i in range(n_days)]
    key = np.array([d.year * 10000 + d.month * 100 + d.day for d in days], np.int32)
    year = np.array([d.year for d in days], np.int32)
    ym = np.array([d.year * 100 + d.month for d in days], np.int32)
    return {"d_key": key, "d_year": year, "d_yearmonthnum": ym}


def _date_column(n: int, sorted_: bool, rng) -> np.ndarray:
    keys = date_dim()["d_key"]
    if sorted_:
        counts = rng.multinomial(n, np.full(N_DAYS, 1.0 / N_DAYS))
        return np.repeat(keys, counts).astype(np.int32)
    return keys[rng.integers(0, N_DAYS, n)]


def fact_q1(n: int, sorted_by_date: bool, seed: int = SEED) -> dict:
    return {
        "date_key": _date_column(n, sorted_by_date, _rng(seed, 1)),
        "quantity": _rng(seed, 2).integers(1, 51, n, dtype=np.int32),
        "discount": _rng(seed, 3).integers(0, 11, n, dtype=np.int32),
        "extended_price": _rng(seed, 4).integers(90_000, 10_494_951, n, dtype=np.int32),
    }


def fact_q3(n: int, sorted_by_date: bool = True, seed: int = SEED, n_customer: int = 3_000_000,
            n_supplier: int = 200_000, n_part: int = 1_400_000, supplycost: bool = False) -> dict:
    """Star-schema fact table; with supplycost=True also supplycost U[100, 600,000]
    (the profit column of the Q4 shape)."""
    t = {
        "date_key": _date_column(n, sorted_by_date, _rng(seed, 11)),
        "cust_key": _rng(seed, 12).integers(1, n_customer + 1, n, dtype=np.int32),
        "supp_key": _rng(seed, 13).integers(1, n_supplier + 1, n, dtype=np.int32),
        "part_key": _rng(seed, 14).integers(1, n_part + 1, n, dtype=np.int32),
        "revenue": _rng(seed, 15).integers(100, 1_000_001, n, dtype=np.int32),
    }
    if supplycost:
        t["supplycost"] = _rng(seed, 16).integers(100, 600_001, n, dtype=np.int32)
    return t


def dim_geo(n: int, seed: int, stream: int) -> dict:
    nation = _rng(seed, stream).integers(0, 25, n, dtype=np.int32)
    return {"key": np.arange(1, n + 1, dtype=np.int32), "nation": nation, "region": NATION_REGION[nation]}


def dim_part(n: int, seed: int = SEED) -> dict:
    """key 1..n, category U[0,25), mfgr = category // 5 (the SSB MFGR#m of
    category MFGR#mn), brand = 40 * category + U[0,40) (the SSB MFGR#mnbb)."""
    r = _rng(seed, 23)
    cat = r.integers(0, 25, n, dtype=np.int32)
    return {"key": np.arange(1, n + 1, dtype=np.int32), "category": cat, "mfgr": (cat // 5).astype(np.int32),
            "brand": (40 * cat + r.integers(0, 40, n, dtype=np.int32)).astype(np.int32)}


def zipf_keys(n: int, n_keys: int, s: float = 1.1, seed: int = SEED, stream: int = 31) -> np.ndarray:
    """Keys 1..n_keys with P(k) proportional to k^-s (bounded Zipf)."""
    r = _rng(seed, stream)
    w = np.arange(1, n_keys + 1, dtype=np.float64) ** (-s)
    cdf = np.cumsum(w)
    cdf /= cdf[-1]
    return (np.searchsorted(cdf, r.random(n)) + 1).astype(np.int32)
