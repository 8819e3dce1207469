"""Autotuner of the batched (shared-scan) form.

No reference counterpart: the reference fixes chunk size, block size and
table layout by command-line flags per run.  Here, per query template
(scan, star, highcard of workload.py), the tuner times a batch of that
template's queries in every point of a grid

    rows_per_chunk  256K .. 4M rows   (the table is re-encoded per value)
    threads         128 .. 1024       (CTA size of the shared-scan kernel)
    ht_layout       linear | bucket | dense   (join-table layout)

on a sample table, replays each batch from a CUDA graph, takes the median of
`reps` device-timed replays, checks that every point gives the same results
(bit-exact), and keeps the fastest point per template.  Choices persist as
JSON keyed by device name and template; `choose()` resolves the launch
shape for a mixed batch and `table_config()` the chunk size and join-table
layouts a table should be built with.
"""
from __future__ import annotations

import json
import os
import time
from dataclasses import asdict, dataclass
from pathlib import Path

import numpy as np

from . import api, workload

TEMPLATES = ("scan", "star", "highcard")
SPACE = {
    "rows_per_chunk": (262_144, 1_048_576, 4_194_304),
    "threads": (128, 256, 512, 1024),
    "ht_layout": ("linear", "bucket", "dense"),
}
DEFAULT = {"rows_per_chunk": 1_048_576, "threads": 256, "ht_layout": "linear"}


@dataclass
class Point:
    rows_per_chunk: int
    threads: int
    ht_layout: str
    ms: float


def default_path() -> Path:
    return Path(os.environ.get("GX_TUNING_FILE", Path.home() / ".cache" / "golap_public_b200" / "tuning.json"))


def device_key() -> str:
    import torch

    p = torch.cuda.get_device_properties(torch.cuda.current_device())
    return f"{p.name} sm{p.major}{p.minor} x{p.multi_processor_count}"


def _time_graph(batch: api.Batch, reps: int) -> float:
    import torch

    stream = torch.cuda.current_stream()
    batch.graph()
    torch.cuda.synchronize()
    ts = []
    for _ in range(reps):
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(stream)
        batch.graph()
        b.record(stream)
        b.synchronize()
        ts.append(a.elapsed_time(b))
    return float(np.median(ts))


def tune(n_rows: int = 20_000_000, queries_per_template: int = 16, space: dict | None = None, reps: int = 5,
         seed: int = 13, templates=TEMPLATES, n_customer: int = 300_000, n_supplier: int = 20_000,
         min_rows: int = 200_000, log=None) -> dict:
    """Grid search per template on a sample table of n_rows rows.  Returns
    {"device", "n_rows", "templates": {t: {"best": Point, "points": [Point]}}}."""
    import torch

    space = {**SPACE, **(space or {})}
    data = workload.generate(n_rows, n_customer=n_customer, n_supplier=n_supplier)
    pts = {t: [] for t in templates}
    ref = {}
    t0 = time.perf_counter()
    for rpc in space["rows_per_chunk"]:
        table = workload.build_table(n_rows, n_customer=n_customer, n_supplier=n_supplier, rows_per_chunk=rpc,
                                     ht_layouts=space["ht_layout"], data=data)
        for tpl in templates:
            for lay in space["ht_layout"]:
                rng = np.random.default_rng(seed + TEMPLATES.index(tpl))  # the same queries at every point
                specs = workload.random_queries(table, queries_per_template, rng, min_rows=min_rows,
                                                max_rows=n_rows, mix=((tpl, 1.0),), ht_layout=lay)
                batch = api.Batch([(s.plan, s.row_lo, s.row_hi) for s in specs], "shared")
                for nt in space["threads"]:
                    batch.set_launch(nt)
                    ms = _time_graph(batch, reps)
                    api.scan_check()
                    got = [workload.read_result(s) for s in specs]
                    if tpl not in ref:
                        ref[tpl] = got
                    elif got != ref[tpl]:
                        raise RuntimeError(f"tuning point {tpl} rpc={rpc} threads={nt} {lay} changed the results")
                    pts[tpl].append(Point(rpc, nt, lay, ms))
                    if log:
                        log(f"{tpl} rpc={rpc} threads={nt} {lay}: {ms:.3f} ms")
                batch.free()
                del specs
        for c in table.cols.values():
            c.free()
        del table
        torch.cuda.empty_cache()
    out = {"device": device_key(), "n_rows": n_rows, "queries_per_template": queries_per_template,
           "tune_s": time.perf_counter() - t0, "templates": {}}
    for tpl in templates:
        best = min(pts[tpl], key=lambda p: p.ms)
        out["templates"][tpl] = {"best": asdict(best), "points": [asdict(p) for p in pts[tpl]]}
    return out


def save(result: dict, path: Path | None = None) -> Path:
    path = Path(path or default_path())
    path.parent.mkdir(parents=True, exist_ok=True)
    store = json.loads(path.read_text()) if path.exists() else {}
    store[result["device"]] = {t: v["best"] for t, v in result["templates"].items()}
    path.write_text(json.dumps(store, indent=1))
    return path


def load(path: Path | None = None, device: str | None = None) -> dict:
    """{template: {"rows_per_chunk", "threads", "ht_layout", "ms"}} for this device ({} if never tuned)."""
    path = Path(path or default_path())
    if not path.exists():
        return {}
    return json.loads(path.read_text()).get(device or device_key(), {})


def table_config(choices: dict, mix=(("scan", 0.6), ("star", 0.3), ("highcard", 0.1))) -> dict:
    """Chunk size for a table serving `mix` (the choice of the template with
    the largest weighted tuned time) and the join-table layouts to build."""
    if not choices:
        return {"rows_per_chunk": DEFAULT["rows_per_chunk"], "ht_layouts": ("linear",)}
    weighted = [(w * choices[t]["ms"], t) for t, w in mix if t in choices]
    heavy = max(weighted)[1] if weighted else None
    rpc = choices[heavy]["rows_per_chunk"] if heavy else DEFAULT["rows_per_chunk"]
    layouts = tuple(dict.fromkeys(["linear"] + [c["ht_layout"] for c in choices.values()]))
    return {"rows_per_chunk": rpc, "ht_layouts": layouts}


def choose(choices: dict, templates) -> dict:
    """Launch shape for a batch holding queries of `templates`: the tuned
    thread count of the template that dominates the batch's tuned time
    (query count x the template's tuned batch time)."""
    if not choices:
        return {"threads": DEFAULT["threads"]}
    weight = {}
    for t in templates:
        weight[t] = weight.get(t, 0.0) + float(choices.get(t, {}).get("ms", 1.0))
    top = max(weight, key=weight.get)
    return {"threads": choices.get(top, DEFAULT)["threads"]}


def tune_launch(batch: api.Batch, candidates=(0, 256, 512, 1024), reps: int = 3) -> dict:
    """Launch shape for one concrete batch: times a graph replay of the batch
    at each candidate CTA size (0 = the library's automatic choice) and keeps
    the fastest.  Per-template tuning picks chunk size and table layout; the
    launch shape of a mixed batch depends on its own shared-memory footprint
    (columns, queries), so it is measured on the batch itself."""
    best = None
    times = {}
    for nt in candidates:
        batch.set_launch(nt)
        ms = _time_graph(batch, reps)
        times[nt if nt else f"auto({batch.threads})"] = ms
        if best is None or ms < best[1]:
            best = (nt, ms)
    batch.set_launch(best[0])
    return {"threads": batch.threads, "requested": best[0], "ms": best[1], "times_ms": times}


def layouts(choices: dict) -> dict:
    """{template: ht_layout} for workload.random_queries."""
    return {t: c["ht_layout"] for t, c in choices.items()}
