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


def build() -> None:
    """Compile liboracle.so (and the reference harness where the tree exists)."""
    subprocess.run(["make", "-s", "-C", str(HERE), "-f", "Makefile", "all"], check=True)


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
        L.or_group_sum_dense.restype = C.c_int
        L.or_group_sum_dense.argtypes = [_P, _P, _u64, _P, _u64]
        L.or_ssb_sizes_for.restype = None
        L.or_ssb_sizes_for.argtypes = [_u32] + [C.POINTER(_u64)] * 5
        L.or_ssb_generate.restype = _i64
        L.or_ssb_generate.argtypes = [_u32, _u64] + [_P] * 15
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


def ssb_generate(sf: int, seed: int = 0xBEE5BEE5) -> dict:
    """Oracle restatement of the reference SSB generator (int32 columns)."""
    L = lib()
    vals = [_u64() for _ in range(5)]
    L.or_ssb_sizes_for(sf, *[C.byref(v) for v in vals])
    n_orders, n_c, n_s, n_p, n_d = (v.value for v in vals)
    cap = n_orders * 7
    t = {k: np.zeros(n_d, np.int32) for k in ("d_key", "d_year", "d_yearmonthnum", "d_weeknuminyear")}
    t.update({k: np.zeros(n_c, np.int32) for k in ("c_nation", "c_region")})
    t.update({k: np.zeros(n_s, np.int32) for k in ("s_nation", "s_region")})
    lo = ("lo_orderdate", "lo_custkey", "lo_suppkey", "lo_quantity", "lo_discount", "lo_extendedprice", "lo_revenue")
    t.update({k: np.zeros(cap, np.int32) for k in lo})
    n = L.or_ssb_generate(sf, seed, *[_ptr(t[k]) for k in ("d_key", "d_year", "d_yearmonthnum", "d_weeknuminyear",
                                                          "c_nation", "c_region", "s_nation", "s_region") + lo])
    for k in lo:
        t[k] = t[k][:n]
    t["c_key"] = np.arange(n_c, dtype=np.int32)
    t["s_key"] = np.arange(n_s, dtype=np.int32)
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
