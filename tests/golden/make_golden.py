"""Regenerates tests/golden/ssb_sf1_reference.json from the reference's own CPU
code (oracle/_ref/libgolapref.so, compiled from the GOLAP sources by
oracle/Makefile): the SSB tables from the reference generator
(usecases/ssb/data/SSB_def.hpp, seed 0xBEE5BEE5, scale factor 1) and the
Q1.1/Q1.2/Q1.3/Q3.1/Q2.1/Q4.1 results of the query loops over the
reference's HostHashMap/HostHashAggregate.  Also records per-column
checksums of the generated table (part strings as integer codes) so the
oracle's generator restatement can be compared without the reference tree.

Run: python tests/golden/make_golden.py
"""
import hashlib
import json
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))
from oracle import oracle as O  # noqa: E402

COLS = ["d_key", "d_year", "c_nation", "s_nation", "lo_orderdate", "lo_custkey", "lo_suppkey", "lo_quantity",
        "lo_discount", "lo_extendedprice", "lo_revenue"]


def main():
    O.build()
    R = O.ref()
    out = np.zeros(6, np.int64)
    R.ref_ssb_golden(1, 8, O._ptr(out))
    sizes = {"d_key": 2555, "d_year": 2555, "c_nation": 30000, "s_nation": 2000}
    arrs = {k: np.zeros(sizes.get(k, 1_500_000 * 7), np.int32) for k in COLS}
    n = R.ref_ssb_columns(1, *[O._ptr(arrs[k]) for k in COLS])
    digests = {}
    for k in COLS:
        a = arrs[k][:n] if k.startswith("lo_") else arrs[k]
        digests[k] = hashlib.sha256(a.tobytes()).hexdigest()
    fl = np.zeros(4, np.int64)
    R.ref_ssb_golden_flights(1, 8, O._ptr(fl))
    n_part = 200_000
    parts = {k: np.zeros(n_part, np.int32) for k in ("p_mfgr", "p_category", "p_brand1")}
    lo2 = {k: np.zeros(1_500_000 * 7, np.int32) for k in ("lo_partkey", "lo_supplycost")}
    n2 = R.ref_ssb_part_columns(1, *[O._ptr(parts[k]) for k in parts], *[O._ptr(lo2[k]) for k in lo2])
    assert n2 == n
    for k, a in parts.items():
        digests[k] = hashlib.sha256(a.tobytes()).hexdigest()
    for k, a in lo2.items():
        digests[k] = hashlib.sha256(a[:n].tobytes()).hexdigest()
    doc = {
        "source": "reference CPU code compiled from the GOLAP sources (oracle/ref_harness.cu)",
        "scale_factor": 1,
        "seed": 0xBEE5BEE5,
        "lineorder_rows": int(out[5]),
        "q1_1": int(out[0]),
        "q1_2": int(out[1]),
        "q1_3": int(out[2]),
        "q3_1_groups": int(out[3]),
        "q3_1_sum": int(out[4]),
        "q2_1_groups": int(fl[0]),
        "q2_1_sum": int(fl[1]),
        "q4_1_groups": int(fl[2]),
        "q4_1_sum": int(fl[3]),
        "column_sha256": digests,
    }
    (Path(__file__).parent / "ssb_sf1_reference.json").write_text(json.dumps(doc, indent=1) + "\n")
    print(json.dumps({k: v for k, v in doc.items() if k != "column_sha256"}))
    lz4_fixtures(R)


def lz4_fixtures(R):
    """LZ4 blocks made by the reference's LZ4CPUManager::compress (liblz4):
    the byte pattern (uint8)(size - i) of core/test/comp_tests.cu:33-37 at
    4 KiB / 32 KiB / 64 KiB, plus two int32 blocks (low-cardinality and
    random) of 16,384 values."""
    rng = np.random.default_rng(7)
    inputs = {f"pattern_{n}": np.array([(n - i) & 255 for i in range(n)], np.uint8) for n in (4096, 32768, 65536)}
    inputs["int32_lowcard"] = rng.integers(0, 11, 16384, dtype=np.int32).view(np.uint8)
    inputs["int32_random"] = rng.integers(-2**31, 2**31 - 1, 16384, dtype=np.int32).view(np.uint8)
    out = {}
    for k, v in inputs.items():
        cap = v.nbytes + v.nbytes // 255 + 64
        comp = np.zeros(cap, np.uint8)
        sizes = np.zeros(1, np.int32)
        assert R.ref_lz4_compress_blocks(O._ptr(v), v.nbytes, v.nbytes, O._ptr(comp), cap, O._ptr(sizes)) == 0
        out[k + "_raw"] = v
        out[k + "_lz4"] = comp[: sizes[0]]
    np.savez_compressed(Path(__file__).parent / "lz4_reference_blocks.npz", **out)
    print("lz4 fixtures:", {k: len(v) for k, v in out.items()})


if __name__ == "__main__":
    main()
