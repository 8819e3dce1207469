"""Pins the CPU oracle to the reference before anything is checked against it.

* SSB generator restatement vs the reference generator: per-column sha256 of
  the scale-factor-1 tables recorded from the reference's own code
  (tests/golden/ssb_sf1_reference.json, made by tests/golden/make_golden.py).
* Q1.1 / Q1.2 / Q1.3 / Q3.1 / Q2.1 / Q4.1 restatements vs the reference
  results on the same data (same fixture; the Q1/Q3 values agree with the
  published survey run).
* LZ4 decoder restatement vs blocks produced by the reference's
  LZ4CPUManager::compress (liblz4), tests/golden/lz4_reference_blocks.npz.
* Where the reference harness is built in this checkout, it is also run
  live and must reproduce the fixture.
"""
import hashlib
import json
from pathlib import Path

import numpy as np
import pytest

from oracle import oracle as O

GOLDEN = Path(__file__).parent / "golden"


@pytest.fixture(scope="module")
def sf1():
    return O.ssb_generate(1)


@pytest.fixture(scope="module")
def golden():
    return json.loads((GOLDEN / "ssb_sf1_reference.json").read_text())


def test_generator_matches_reference_columns(sf1, golden):
    assert len(sf1["lo_orderdate"]) == golden["lineorder_rows"]
    for k, digest in golden["column_sha256"].items():
        assert hashlib.sha256(sf1[k].tobytes()).hexdigest() == digest, k


def test_queries_match_reference(sf1, golden):
    r = O.ssb_queries(sf1)
    assert r["q1_1"] == golden["q1_1"] == 418218118998
    assert r["q1_2"] == golden["q1_2"] == 91465357047
    assert r["q1_3"] == golden["q1_3"] == 25077436727
    assert r["q3_1_groups"] == golden["q3_1_groups"] == 150
    assert r["q3_1_sum"] == golden["q3_1_sum"] == 772685826017
    assert r["q2_1_groups"] == golden["q2_1_groups"] == 280
    assert r["q2_1_sum"] == golden["q2_1_sum"] == 173123930382
    assert r["q4_1_groups"] == golden["q4_1_groups"] == 35
    assert r["q4_1_sum"] == golden["q4_1_sum"] == 330407033455


def test_lz4_decoder_on_reference_blocks():
    z = np.load(GOLDEN / "lz4_reference_blocks.npz")
    names = sorted({k[: -4] for k in z.files})
    assert len(names) == 5
    for n in names:
        raw, comp = z[n + "_raw"], z[n + "_lz4"]
        out = O.lz4_decode(comp, raw.nbytes)
        assert out is not None and np.array_equal(out, raw), n


def test_lz4_decoder_rejects_malformed():
    z = np.load(GOLDEN / "lz4_reference_blocks.npz")
    comp = z["pattern_4096_lz4"]
    raw = z["pattern_4096_raw"]
    assert O.lz4_decode(comp[:-3], raw.nbytes) is None or not np.array_equal(O.lz4_decode(comp[:-3], raw.nbytes), raw)
    assert O.lz4_decode(comp, raw.nbytes - 1) is None  # output overflow
    bad = comp.copy()
    bad[0] = 0x0F  # zero literals then a match at offset taken from literal bytes -> offset beyond output
    assert O.lz4_decode(bad, raw.nbytes) is None


def test_minmax_keep_known_answers():
    # MinMaxMeta::check_pred semantics (core/metadata.cuh:203-211): inclusive overlap.
    # Mirrors the known answers of core/test/metadata_tests.cu:210-272 with
    # integer chunks {0..15 as two chunks, and a constant chunk}.
    mins = np.array([0, 8, 1993], np.int32)
    maxs = np.array([7, 15, 1993], np.int32)
    assert O.minmax_keep(mins, maxs, 5, 5).tolist() == [1, 0, 0]
    assert O.minmax_keep(mins, maxs, 7, 8).tolist() == [1, 1, 0]
    assert O.minmax_keep(mins, maxs, 1993, 1993).tolist() == [0, 0, 1]
    assert O.minmax_keep(mins, maxs, 1994, 1994).tolist() == [0, 0, 0]
    assert O.minmax_keep(mins, maxs, -5, -1).tolist() == [0, 0, 0]
    k = O.minmax_keep(mins, maxs, 0, 10)
    assert O.minmax_keep(mins, maxs, 9, 2000, keep=k).tolist() == [0, 1, 0]


def test_join_probe_first_match_semantics():
    # HashMap::probe returns the matching build rid; a filtered-out row is a miss.
    bk = np.array([10, 20, 30, 40], np.int64)
    ok = np.array([1, 0, 1, 1], np.uint8)
    r = O.join_probe(bk, ok, np.array([20, 30, 5, 40, 10], np.int64))
    assert r.tolist() == [-1, 2, -1, 3, 0]


@pytest.mark.skipif(not O.ref_available(), reason="reference harness not built here")
def test_reference_harness_live(golden):
    out = np.zeros(6, np.int64)
    O.ref().ref_ssb_golden(1, 4, O._ptr(out))
    assert out.tolist() == [golden["q1_1"], golden["q1_2"], golden["q1_3"], golden["q3_1_groups"],
                            golden["q3_1_sum"], golden["lineorder_rows"]]


@pytest.mark.skipif(not O.ref_available(), reason="reference harness not built here")
def test_reference_harness_flights_live(golden):
    out = np.zeros(4, np.int64)
    O.ref().ref_ssb_golden_flights(1, 4, O._ptr(out))
    assert out.tolist() == [golden["q2_1_groups"], golden["q2_1_sum"], golden["q4_1_groups"], golden["q4_1_sum"]]
