"""Autotuner host logic (no GPU): choice persistence keyed by device, the
table configuration for a query mix and the launch shape of a mixed batch."""
from golap_public_b200 import autotune as AT


def _result(device="dev0"):
    pts = {
        "scan": {"rows_per_chunk": 262144, "threads": 512, "ht_layout": "bucket", "ms": 2.0},
        "star": {"rows_per_chunk": 1048576, "threads": 256, "ht_layout": "linear", "ms": 9.0},
        "highcard": {"rows_per_chunk": 4194304, "threads": 1024, "ht_layout": "linear", "ms": 4.0},
    }
    return {"device": device, "templates": {t: {"best": p, "points": [p]} for t, p in pts.items()}}


def test_save_load_roundtrip(tmp_path):
    f = tmp_path / "tuning.json"
    AT.save(_result("dev0"), f)
    AT.save(_result("dev1"), f)
    got = AT.load(f, device="dev0")
    assert got["scan"]["threads"] == 512 and got["star"]["ht_layout"] == "linear"
    assert AT.load(f, device="unknown") == {}
    assert AT.load(tmp_path / "missing.json", device="dev0") == {}


def test_table_config_and_choose():
    ch = {t: v["best"] for t, v in _result()["templates"].items()}
    # weighted time: scan 0.6*2=1.2, star 0.3*9=2.7, highcard 0.1*4=0.4 -> star's chunk size
    cfg = AT.table_config(ch)
    assert cfg["rows_per_chunk"] == 1048576
    assert set(cfg["ht_layouts"]) == {"linear", "bucket"} and cfg["ht_layouts"][0] == "linear"
    # time-weighted: 2 scans x 2 ms < 1 star x 9 ms -> star's launch shape
    assert AT.choose(ch, ["scan", "scan", "star"]) == {"threads": 256}
    assert AT.choose(ch, ["scan"] * 5 + ["star"]) == {"threads": 512}
    assert AT.choose(ch, ["highcard"]) == {"threads": 1024}
    assert AT.layouts(ch) == {"scan": "bucket", "star": "linear", "highcard": "linear"}
    assert AT.table_config({}) == {"rows_per_chunk": AT.DEFAULT["rows_per_chunk"], "ht_layouts": ("linear",)}
    assert AT.choose({}, ["scan"]) == {"threads": AT.DEFAULT["threads"]}


def test_search_space_covers_the_stated_ranges():
    assert min(AT.SPACE["rows_per_chunk"]) == 256 * 1024 and max(AT.SPACE["rows_per_chunk"]) == 4 * 1024 * 1024
    assert min(AT.SPACE["threads"]) == 128 and max(AT.SPACE["threads"]) == 1024
    assert set(AT.SPACE["ht_layout"]) == {"linear", "bucket", "dense"}
