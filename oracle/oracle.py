"""ctypes bindings of the CPU checkers (test infrastructure only).

liboracle.so   -- restatement of the reference algorithms (oracle.c)
_ref/libgolapref.so -- the reference's own CPU code built from its sources
                       (ref_harness.cu); present where it was built.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import
this module, and only to check or time; the product never does.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
_LIB = HERE / "liboracle.so"
_REF = HERE / "_ref" / "libgolapref.so"

_P = C.c_void_p
_u64, _i64, _i32, _u32 = C.c_uint64, C.c_int64, C.c_int32, C.c_uint32


# The reference source tree of this checkout's build container (absent on
# machines that only run the prebuilt libraries); GX_REFERENCE_TREE overrides.
_REF_TREE = os.environ.get("GX_REFERENCE_TREE", "/root/reference")


def build() -> None:
    """Compile liboracle.so, and the reference harness where the reference tree exists."""
    cmd = ["make", "-s", "-C", str(HERE), "-f", "Makefile", "all"]
    if Path(_REF_TREE, "core").is_dir():
        cmd.append(f"REF={_REF_TREE}")
    subprocess.run(cmd, check=True)


def _ptr(a):
    return None if a is None else a.ctypes.data_as(_P)


_lib = None
_ref = None


def lib():
    global _lib
    if _lib is None:
        if not _LIB.exists():
            build()
        L = C.CDLL(str(_LIB))
        L.or_lz4_decode.restype = _i64
        L.or_lz4_decode.argtypes = [_P, _u64, _P, _u64]
        L.or_lz4_check_segments.restype = C.c_int
        L.or_lz4_check_segments.argtypes = [_P, _u64, _P, _u32, _u32, _u32, _P]
        L.or_casc_decode.restype = _i64
        L.or_casc_decode.argtypes = [_P, _u64, _P, _u64]
        L.or_minmax_keep.restype = None
        L.or_minmax_keep.argtypes = [_P, _P, _u64, _i32, _i32, _P, C.c_int]
        L.or_chunk_minmax.restype = None
        L.or_chunk_minmax.argtypes = [_P, _u64, _u64, _P, _P]
        L.or_join_probe.restype = C.c_int
        L.or_join_probe.argtypes = [_P, _P, _u64, _P, _u64, _P]
        L.or_q1.restype = _i64
        L.or_q1.argtypes = [_P, _P, _P, _P, _u64, _P, _P, _u64, _i32, _i32, _i32, _i32, _i32, _i32, _P, _u64]
        L.or_q3.restype = C.c_int
        L.or_q3.argtypes = [_P, _P, _P, _P, _u64, _P, _P, _P, _u64, _P, _P, _P, _u64, _P, _P, _P, _u64,
                            _i32, _u32, _i32, _u32, _i32, _u32, _P, _P, _P, _u64]
        L.or_minmax_points_keep.restype = None
        L.or_minmax_points_keep.argtypes = [_P, _P, _u64, _P, _u64, _P]
        L.or_hist_counts.restype = None
        L.or_hist_counts.argtypes = [_P, _u64, _u64, _u32, _P, _P, _P]
        L.or_hist_keep.restype = None
        L.or_hist_keep.argtypes = [_P, _P, _P, _u64, _u32, _i32, _i32, _P]
        L.or_bloom_k.restype = _u32
        L.or_bloom_k.argtypes = [_u64, C.c_double]
        L.or_bloom_words.restype = None
        L.or_bloom_words.argtypes = [_P, _u64, _u64, _u64, _u32, _P]
        L.or_bloom_keep.restype = None
        L.or_bloom_keep.argtypes = [_P, _u64, _u64, _u32, _i32, _P]
        L.or_group_sum_dense.restype = C.c_int
        L.or_group_sum_dense.argtypes = [_P, _P, _u64, _P, _u64]
        L.or_ssb_sizes_for.restype = None
        L.or_ssb_sizes_for.argtypes = [_u32] + [C.POINTER(_u64)] * 5
        L.or_ssb_generate.restype = _i64
        L.or_ssb_generate.argtypes = [_u32, _u64] + [_P] * 20
        L.or_q2.restype = C.c_int
        L.or_q2.argtypes = [_P, _P, _P, _P, _u64, _P, _P, _u64, _P, _u64, _P, _P, _u64, _i32, _i32, _i32, _P, _P]
        L.or_q4.restype = C.c_int
        L.or_q4.argtypes = [_P, _P, _P, _P, _P, _P, _u64, _P, _P, _u64, _P, _u64, _P, _u64, _P, _P, _P, _u64,
                            _i32, _i32, _P, _P]
        _lib = L
    return _lib


def ref_available() -> bool:
    return _REF.exists()


def ref():
    global _ref
    if _ref is None:
        if not _REF.exists():
            raise FileNotFoundError(f"{_REF} not built (reference tree absent when building)")
        R = C.CDLL(str(_REF))
        R.ref_ssb_golden.restype = C.c_int
        R.ref_ssb_golden.argtypes = [_u32, _u32, _P]
        R.ref_ssb_columns.restype = _i64
        R.ref_ssb_columns.argtypes = [_u32] + [_P] * 11
        R.ref_ssb_golden_flights.restype = C.c_int
        R.ref_ssb_golden_flights.argtypes = [_u32, _u32, _P]
        R.ref_ssb_part_columns.restype = _i64
        R.ref_ssb_part_columns.argtypes = [_u32] + [_P] * 5
        R.ref_lz4_compress_blocks.restype = C.c_int
        R.ref_lz4_compress_blocks.argtypes = [_P, _u64, _u64, _P, _u64, _P]
        R.ref_lz4_decompress.restype = C.c_int
        R.ref_lz4_decompress.argtypes = [_P, C.c_int, _P, C.c_int]
        R.ref_cpu_q1_comp.restype = _i64
        R.ref_cpu_q1_comp.argtypes = [_u32, _u64, _u64, _u64, _P, _P, _P, _P, _P, _u64,
                                      _i32, _i32, _i32, _i32, _i32, _i32, C.POINTER(C.c_double), C.POINTER(_u64),
                                      C.POINTER(_u64)]
        R.ref_cpu_q3_comp.restype = _i64
        R.ref_cpu_q3_comp.argtypes = [_u32, _u64, _u64, _u64, _P, _P, _P, _P, _P, _P, _u64, _P, _P, _P, _u64,
                                      _P, _P, _u64, _i32, _i32, _i32, _P, _P, _u64, C.POINTER(_u64),
                                      C.POINTER(C.c_double), C.POINTER(_u64), C.POINTER(_u64)]
        _ref = R
    return _ref


# ------------------------------------------------------------- wrappers

def lz4_decode(comp: np.ndarray, out_size: int) -> np.ndarray | None:
    out = np.zeros(out_size + 16, np.uint8)
    n = lib().or_lz4_decode(_ptr(comp), comp.nbytes, _ptr(out), out_size)
    return None if n < 0 else out[:n]


def casc_decode(blk: np.ndarray, max_rows: int) -> np.ndarray | None:
    out = np.zeros(max(max_rows, 1), np.int32)
    n = lib().or_casc_decode(_ptr(blk), blk.nbytes, _ptr(out), max_rows)
    return None if n < 0 else out[:n]


def minmax_keep(mins, maxs, lo, hi, keep=None):
    n = len(mins)
    if keep is None:
        keep = np.zeros(n, np.uint16)
        lib().or_minmax_keep(_ptr(mins), _ptr(maxs), n, lo, hi, _ptr(keep), 0)
    else:
        lib().or_minmax_keep(_ptr(mins), _ptr(maxs), n, lo, hi, _ptr(keep), 1)
    return keep


def minmax_points_keep(mins, maxs, keys) -> np.ndarray:
    """Join-pruning flags (check_mmmeta_multiple_pts)."""
    keep = np.zeros(len(mins), np.uint16)
    k = np.ascontiguousarray(keys, np.int32)
    mn = np.ascontiguousarray(mins, np.int32)
    mx = np.ascontiguousarray(maxs, np.int32)
    lib().or_minmax_points_keep(_ptr(mn), _ptr(mx), len(mn), _ptr(k), len(k), _ptr(keep))
    return keep


def hist_counts(v, rows_per_chunk, n_buckets):
    """EqHistogram counts per chunk (n_chunks, n_buckets)."""
    v = np.ascontiguousarray(v, np.int32)
    mins, maxs = chunk_minmax(v, rows_per_chunk)
    counts = np.zeros(len(mins) * n_buckets, np.uint64)
    lib().or_hist_counts(_ptr(v), len(v), rows_per_chunk, n_buckets, _ptr(mins), _ptr(maxs), _ptr(counts))
    return counts.reshape(len(mins), n_buckets)


def hist_keep(mins, maxs, counts, lo, hi):
    keep = np.zeros(len(mins), np.uint16)
    c = np.ascontiguousarray(counts, np.uint64)
    mn, mx = np.ascontiguousarray(mins, np.int32), np.ascontiguousarray(maxs, np.int32)
    lib().or_hist_keep(_ptr(mn), _ptr(mx), _ptr(c), len(mn), c.shape[1], lo, hi, _ptr(keep))
    return keep


def bloom_words(v, rows_per_chunk, m_bytes, p):
    """BloomMeta filters (n_chunks, m_bytes / 4 words) and k."""
    v = np.ascontiguousarray(v, np.int32)
    k = lib().or_bloom_k(m_bytes, p)
    nc = -(-len(v) // rows_per_chunk)
    words = np.zeros(nc * (m_bytes // 4), np.uint32)
    lib().or_bloom_words(_ptr(v), len(v), rows_per_chunk, m_bytes, k, _ptr(words))
    return words.reshape(nc, m_bytes // 4), k


def bloom_keep(words, m_bytes, k, val):
    w = np.ascontiguousarray(words, np.uint32)
    keep = np.zeros(w.shape[0], np.uint16)
    lib().or_bloom_keep(_ptr(w), w.shape[0], m_bytes, k, val, _ptr(keep))
    return keep


def chunk_minmax(v: np.ndarray, rows_per_chunk: int):
    nc = (len(v) + rows_per_chunk - 1) // rows_per_chunk
    mins = np.zeros(nc, np.int32)
    maxs = np.zeros(nc, np.int32)
    lib().or_chunk_minmax(_ptr(v), len(v), rows_per_chunk, _ptr(mins), _ptr(maxs))
    return mins, maxs


def join_probe(build_keys, build_ok, probe_keys) -> np.ndarray:
    bk = np.ascontiguousarray(build_keys, np.int64)
    pk = np.ascontiguousarray(probe_keys, np.int64)
    ok = None if build_ok is None else np.ascontiguousarray(build_ok, np.uint8)
    out = np.zeros(len(pk), np.int64)
    assert lib().or_join_probe(_ptr(bk), _ptr(ok), len(bk), _ptr(pk), len(pk), _ptr(out)) == 0
    return out


def q1(orderdate, discount, quantity, extprice, d_key, date_ok, dlo, dhi, qlo, qhi,
       plo=-(2**31), phi=2**31 - 1, keep_chunk=None, rows_per_chunk=1) -> int:
    a = [np.ascontiguousarray(x, np.int32) for x in (orderdate, discount, quantity, extprice, d_key)]
    ok = np.ascontiguousarray(date_ok, np.uint8)
    kc = None if keep_chunk is None else np.ascontiguousarray(keep_chunk, np.uint16)
    return int(lib().or_q1(_ptr(a[0]), _ptr(a[1]), _ptr(a[2]), _ptr(a[3]), len(a[0]), _ptr(a[4]), _ptr(ok),
                           len(a[4]), dlo, dhi, qlo, qhi, plo, phi, _ptr(kc), rows_per_chunk))


def q3(custkey, suppkey, orderdate, revenue, c_key, c_attr, c_ok, s_key, s_attr, s_ok, d_key, d_attr, d_ok,
       c_base, c_card, s_base, s_card, d_base, d_card, keep_chunk=None, rows_per_chunk=1):
    """Returns (sums, counts) as dense arrays of shape (c_card, s_card, d_card)."""
    f = [np.ascontiguousarray(x, np.int32) for x in (custkey, suppkey, orderdate, revenue)]
    c = [np.ascontiguousarray(x, np.int32) for x in (c_key, c_attr)]
    s = [np.ascontiguousarray(x, np.int32) for x in (s_key, s_attr)]
    d = [np.ascontiguousarray(x, np.int32) for x in (d_key, d_attr)]
    oks = [np.ascontiguousarray(x, np.uint8) for x in (c_ok, s_ok, d_ok)]
    cells = c_card * s_card * d_card
    sums = np.zeros(cells, np.int64)
    counts = np.zeros(cells, np.int64)
    kc = None if keep_chunk is None else np.ascontiguousarray(keep_chunk, np.uint16)
    rc = lib().or_q3(_ptr(f[0]), _ptr(f[1]), _ptr(f[2]), _ptr(f[3]), len(f[0]),
                     _ptr(c[0]), _ptr(c[1]), _ptr(oks[0]), len(c[0]),
                     _ptr(s[0]), _ptr(s[1]), _ptr(oks[1]), len(s[0]),
                     _ptr(d[0]), _ptr(d[1]), _ptr(oks[2]), len(d[0]),
                     c_base, c_card, s_base, s_card, d_base, d_card, _ptr(sums), _ptr(counts), _ptr(kc),
                     rows_per_chunk)
    if rc != 0:
        raise ValueError(f"or_q3 failed: {rc}")
    return sums.reshape(c_card, s_card, d_card), counts.reshape(c_card, s_card, d_card)


def _keyed(keys, attr, ok, n):
    """Dimension arrays indexed by key (0..n-1): attribute and pass flag; keys outside stay unset."""
    a = np.zeros(n, np.int32)
    f = np.zeros(n, np.uint8)
    k = np.asarray(keys, np.int64)
    a[k] = attr
    f[k] = np.asarray(ok, np.uint8)
    return a, f


def q2(partkey, suppkey, orderdate, revenue, p_key, p_brand, p_ok, s_key, s_ok, d_key, d_year, brand_card, year0,
       n_years):
    """Q2 shape (02inmem.hpp:100-180): (sums, counts) of shape (brand_card, n_years)."""
    f = [np.ascontiguousarray(x, np.int32) for x in (partkey, suppkey, orderdate, revenue)]
    npk = int(max(np.max(p_key), np.max(f[0]))) + 1
    nsk = int(max(np.max(s_key), np.max(f[1]))) + 1
    pb, pok = _keyed(p_key, p_brand, p_ok, npk)
    _, sok = _keyed(s_key, np.zeros(len(s_key), np.int32), s_ok, nsk)
    d = [np.ascontiguousarray(x, np.int32) for x in (d_key, d_year)]
    sums = np.zeros(brand_card * n_years, np.int64)
    counts = np.zeros_like(sums)
    rc = lib().or_q2(_ptr(f[0]), _ptr(f[1]), _ptr(f[2]), _ptr(f[3]), len(f[0]), _ptr(pok), _ptr(pb), npk, _ptr(sok),
                     nsk, _ptr(d[0]), _ptr(d[1]), len(d[0]), brand_card, year0, n_years, _ptr(sums), _ptr(counts))
    if rc != 0:
        raise ValueError(f"or_q2 failed: {rc}")
    return sums.reshape(brand_card, n_years), counts.reshape(brand_card, n_years)


def q4(custkey, suppkey, partkey, orderdate, revenue, supplycost, c_key, c_nation, c_ok, s_key, s_ok, p_key, p_ok,
       d_key, d_year, d_ok, year0, n_years):
    """Q4 shape (04inmem.hpp:120-160): (sums, counts) of SUM(revenue - supplycost), shape (n_years, 25)."""
    f = [np.ascontiguousarray(x, np.int32) for x in (custkey, suppkey, partkey, orderdate, revenue, supplycost)]
    nck = int(max(np.max(c_key), np.max(f[0]))) + 1
    nsk = int(max(np.max(s_key), np.max(f[1]))) + 1
    npk = int(max(np.max(p_key), np.max(f[2]))) + 1
    cn, cok = _keyed(c_key, c_nation, c_ok, nck)
    _, sok = _keyed(s_key, np.zeros(len(s_key), np.int32), s_ok, nsk)
    _, pok = _keyed(p_key, np.zeros(len(p_key), np.int32), p_ok, npk)
    d = [np.ascontiguousarray(x, np.int32) for x in (d_key, d_year)]
    dok = np.ascontiguousarray(d_ok, np.uint8)
    sums = np.zeros(n_years * 25, np.int64)
    counts = np.zeros_like(sums)
    rc = lib().or_q4(_ptr(f[0]), _ptr(f[1]), _ptr(f[2]), _ptr(f[3]), _ptr(f[4]), _ptr(f[5]), len(f[0]), _ptr(cok),
                     _ptr(cn), nck, _ptr(sok), nsk, _ptr(pok), npk, _ptr(d[0]), _ptr(d[1]), _ptr(dok), len(d[0]),
                     year0, n_years, _ptr(sums), _ptr(counts))
    if rc != 0:
        raise ValueError(f"or_q4 failed: {rc}")
    return sums.reshape(n_years, 25), counts.reshape(n_years, 25)


def ssb_generate(sf: int, seed: int = 0xBEE5BEE5) -> dict:
    """Oracle restatement of the reference SSB generator (int32 columns; part
    strings as integer codes: p_mfgr 0..4, p_category 0..24, p_brand1 0..999)."""
    L = lib()
    vals = [_u64() for _ in range(5)]
    L.or_ssb_sizes_for(sf, *[C.byref(v) for v in vals])
    n_orders, n_c, n_s, n_p, n_d = (v.value for v in vals)
    cap = n_orders * 7
    t = {k: np.zeros(n_d, np.int32) for k in ("d_key", "d_year", "d_yearmonthnum", "d_weeknuminyear")}
    t.update({k: np.zeros(n_c, np.int32) for k in ("c_nation", "c_region")})
    t.update({k: np.zeros(n_s, np.int32) for k in ("s_nation", "s_region")})
    t.update({k: np.zeros(n_p, np.int32) for k in ("p_mfgr", "p_category", "p_brand1")})
    lo = ("lo_orderdate", "lo_custkey", "lo_suppkey", "lo_quantity", "lo_discount", "lo_extendedprice", "lo_revenue",
          "lo_partkey", "lo_supplycost")
    t.update({k: np.zeros(cap, np.int32) for k in lo})
    n = L.or_ssb_generate(sf, seed, *[_ptr(t[k]) for k in ("d_key", "d_year", "d_yearmonthnum", "d_weeknuminyear",
                                                          "c_nation", "c_region", "s_nation", "s_region",
                                                          "p_mfgr", "p_category", "p_brand1") + lo])
    for k in lo:
        t[k] = t[k][:n]
    t["c_key"] = np.arange(n_c, dtype=np.int32)
    t["s_key"] = np.arange(n_s, dtype=np.int32)
    t["p_key"] = np.arange(n_p, dtype=np.int32)
    return t


def ssb_queries(t: dict) -> dict:
    """Q1.1/Q1.2/Q1.3/Q3.1 of the SSB flight on oracle tables (01inmem.hpp:143-152, 03inmem.hpp:229-236)."""
    r = {}
    base = (t["lo_orderdate"], t["lo_discount"], t["lo_quantity"], t["lo_extendedprice"], t["d_key"])
    r["q1_1"] = q1(*base, t["d_year"] == 1993, 1, 3, 0, 24)
    r["q1_2"] = q1(*base, t["d_yearmonthnum"] == 199401, 4, 6, 26, 35)
    r["q1_3"] = q1(*base, (t["d_weeknuminyear"] == 6) & (t["d_year"] == 1994), 5, 7, 26, 35)
    asia = 2
    sums, counts = q3(t["lo_custkey"], t["lo_suppkey"], t["lo_orderdate"], t["lo_revenue"],
                      t["c_key"], t["c_nation"], t["c_region"] == asia,
                      t["s_key"], t["s_nation"], t["s_region"] == asia,
                      t["d_key"], t["d_year"], (t["d_year"] >= 1992) & (t["d_year"] <= 1997),
                      0, 25, 0, 25, 1992, 7)
    r["q3_1_groups"] = int((counts > 0).sum())
    r["q3_1_sum"] = int(sums.sum())
    r["q3_1_cells"] = (sums, counts)
    # Q2.1 (02inmem.hpp:208-210): p_category = MFGR#12 (code 1), s_region AMERICA (1)
    sums, counts = q2(t["lo_partkey"], t["lo_suppkey"], t["lo_orderdate"], t["lo_revenue"], t["p_key"],
                      t["p_brand1"], t["p_category"] == 1, t["s_key"], t["s_region"] == 1, t["d_key"], t["d_year"],
                      1000, 1992, 7)
    r["q2_1_groups"] = int((counts > 0).sum())
    r["q2_1_sum"] = int(sums.sum())
    r["q2_1_cells"] = (sums, counts)
    # Q4.1 (04inmem.hpp:204-210): c_region, s_region AMERICA, p_mfgr MFGR#1 or MFGR#2 (codes 0, 1)
    sums, counts = q4(t["lo_custkey"], t["lo_suppkey"], t["lo_partkey"], t["lo_orderdate"], t["lo_revenue"],
                      t["lo_supplycost"], t["c_key"], t["c_nation"], t["c_region"] == 1, t["s_key"],
                      t["s_region"] == 1, t["p_key"], t["p_mfgr"] <= 1, t["d_key"], t["d_year"],
                      np.ones(len(t["d_key"]), bool), 1992, 7)
    r["q4_1_groups"] = int((counts > 0).sum())
    r["q4_1_sum"] = int(sums.sum())
    r["q4_1_cells"] = (sums, counts)
    return r


# --------------------------------------------- reference CPU baselines over compressed columns

class CompCol(C.Structure):
    """{payload, blocks, codec} as ref_cpu_*_comp take it (blocks: 4 uint64 per present block)."""
    _fields_ = [("payload", C.c_void_p), ("blocks", C.c_void_p), ("codec", C.c_uint32)]


def comp_cols(cols):
    """CompCol array over (payload uint8 array, blocks uint64 (n,4) array, codec) triples; the
    arrays must stay alive while the result is used."""
    arr = (CompCol * len(cols))()
    for i, (pl, blocks, codec) in enumerate(cols):
        arr[i].payload = pl.ctypes.data
        assert blocks.dtype == np.uint64 and blocks.flags.c_contiguous and pl.flags.c_contiguous
        arr[i].blocks = blocks.ctypes.data
        arr[i].codec = codec
    return arr
