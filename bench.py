"""Benchmark of the fused compressed-scan hot path on B200.

Workload (one step = one query): a 60,000,000-row fact table sorted by
date_key, compressed per 1,000,000-row chunk (date_key cascaded, discount /
quantity / extended_price LZ4 on 64 KiB blocks), per-chunk min/max; the
query is SUM(extended_price * discount) over fact JOIN date WHERE the date
is in January 1994 AND discount BETWEEN 4 AND 6 AND quantity BETWEEN 26 AND
35.  A step builds the filtered date hash table, prunes chunks on min/max
and runs the fused scan; the int64 result stays on the device (value) or
comes back to the host (e2e).  Data is seeded synthetic data with the
workload's shapes and distributions.

  value     rows/s over the whole table (pruned chunks count, as in the
            reference's uncompressed-bytes / time definition), compressed
            columns resident in HBM, device time (CUDA events) per step,
            the step captured once as a CUDA graph and replayed, L2
            flushed between steps.
  e2e       the same query with the compressed columns in pinned host
            memory, read by the kernels over PCIe, timed through the public
            API with the date dimension copied in and the result read back.
  roofline  the fused scan kernel: algorithmic bytes (compressed bytes of
            the surviving tiles + their directory/segment index) per launch
            / launch time, against the measured HBM copy bandwidth.
  cpu_baseline  the reference's CPU path on the same data: LZ4CPUManager
            decompression + the query loop over HostHashMap, all host cores.

--impl reference runs only the CPU path (rank 0) and prints its line.
--gpus N runs N independent replicas (one per GPU; the query does not need
a collective); value is the total over ranks, time is the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import re
import subprocess
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

N_ROWS = 60_000_000
ROWS_PER_CHUNK = 1_000_000
ROWS_PER_BLOCK = 16384
DATE_LO, DATE_HI = 19940101, 19940131
DISC = (4, 6)
QTY = (26, 35)
WORKLOAD = ("Q1 shape on 60M rows sorted by date_key: date_key cascaded, discount/quantity/extended_price "
            "LZ4 on 64 KiB blocks, 1M-row chunks with min/max; month Jan 1994, discount 4..6, quantity 26..35")


def peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def profile_traffic():
    """dram bytes per launch of the fused scan kernel from the committed ncu summary (or None)."""
    p = ROOT / "profiles" / "shared_scan_kernel_q1_pruned_60M.md"
    if not p.exists():
        return None
    m = re.search(r"traffic_bytes_per_launch:\s*([0-9]+)", p.read_text())
    return int(m.group(1)) if m else None


class Clocks:
    """Samples SM clocks and clock-event (throttle) reasons through NVML in a
    background thread (every 2 ms) while the timed region runs; the samples
    are also written to gpurun_out/clocks_bench_<pid>.csv."""

    NAMES = (("hw_slowdown", 0x8), ("hw_thermal_slowdown", 0x40), ("sw_thermal_slowdown", 0x20),
             ("sw_power_cap", 0x4), ("hw_power_brake_slowdown", 0x80))

    def __init__(self, gpu: int):
        self.gpu = gpu
        self.samples = []
        self.max_mhz = None
        self.err = None
        self.path = ROOT / "gpurun_out" / f"clocks_bench_{os.getpid()}.csv"

    def _handle(self):
        import pynvml
        import torch

        pynvml.nvmlInit()
        try:
            p = torch.cuda.get_device_properties(self.gpu)
            return pynvml.nvmlDeviceGetHandleByPciBusId(f"{p.pci_domain_id:08x}:{p.pci_bus_id:02x}:{p.pci_device_id:02x}.0")
        except Exception:
            return pynvml.nvmlDeviceGetHandleByIndex(self.gpu)

    def _run(self):
        import pynvml

        while not self.stop.is_set():
            try:
                mhz = pynvml.nvmlDeviceGetClockInfo(self.h, pynvml.NVML_CLOCK_SM)
                rs = pynvml.nvmlDeviceGetCurrentClocksEventReasons(self.h)
                self.samples.append((time.perf_counter(), mhz, rs))
            except Exception as e:  # keep the bench running; report the gap
                self.err = str(e)
                return
            self.stop.wait(0.002)

    def __enter__(self):
        import threading

        self.stop = threading.Event()
        self.thread = None
        try:
            import pynvml

            self.h = self._handle()
            self.max_mhz = pynvml.nvmlDeviceGetMaxClockInfo(self.h, pynvml.NVML_CLOCK_SM)
            self.thread = threading.Thread(target=self._run, daemon=True)
            self.thread.start()
            t0 = time.perf_counter()
            while not self.samples and time.perf_counter() - t0 < 2.0 and self.err is None:
                time.sleep(0.001)
        except Exception as e:
            self.err = str(e)
        return self

    def __exit__(self, *a):
        self.stop.set()
        if self.thread:
            self.thread.join(2.0)
        try:
            self.path.parent.mkdir(exist_ok=True)
            with open(self.path, "w") as fh:
                fh.write("t_s,sm_mhz,reasons_hex\n")
                for t, m, r in self.samples:
                    fh.write(f"{t:.6f},{m},{r:#x}\n")
        except Exception:
            pass

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": self.max_mhz, "reasons": ["unsampled"],
                    **({"error": self.err} if self.err else {})}
        sm = [m for _, m, _ in self.samples]
        reasons = sorted({n for _, _, r in self.samples for n, bit in self.NAMES if r & bit})
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": self.max_mhz, "reasons": reasons,
                "samples": len(sm), "source": "nvml"}


def max_over_ranks(value: float, world: int, device=None) -> float:
    """Max of a per-rank time over all ranks (replicas: no data-path collective,
    only this timing reduction); identity for a single process."""
    if world <= 1:
        return value
    import torch
    import torch.distributed as dist

    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def make_data(seed):
    from golap_public_b200 import datagen

    return datagen.fact_q1(N_ROWS, True, seed=seed), datagen.date_dim()


# ----------------------------------------------------------------- GPU arm

def gpu_arm(args, rank, world):
    import torch
    import torch.distributed as dist

    from golap_public_b200 import api, queries
    from golap_public_b200.build import build

    build()
    dev = int(os.environ.get("LOCAL_RANK", 0))
    torch.cuda.set_device(dev)
    f, dd = make_data(args.seed)
    ok = dd["d_yearmonthnum"] == 199401
    fact = queries.encode_fact(f, {"date_key": "cascaded"}, ROWS_PER_CHUNK, ROWS_PER_BLOCK, args.segments)
    comp = {k: c.info.comp_bytes for k, c in fact.cols.items()}

    q = queries.Q1Query(fact, dd, ok, DATE_LO, DATE_HI, *DISC, *QTY, prune=True)
    dk_h = torch.from_numpy(dd["d_key"]).pin_memory()
    ok_h = torch.from_numpy(ok.astype(np.int32)).pin_memory()
    dk_d = torch.empty_like(dk_h, device="cuda")
    ok_d = torch.empty_like(ok_h, device="cuda")
    stream = torch.cuda.current_stream()

    def step():
        # the per-query work of the reference's query1 timed region
        # (01.hpp:235-430): date table build, pruning, fused scan
        q.ht.build(q._dk, None, preds=[(q._ok, 1, 1)])
        q.launch()

    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    got = q.run()
    want = got  # checked against the CPU baseline's result below
    kept = int(q.keep.sum().item())
    kept_chunks = np.nonzero(q.keep.cpu().numpy())[0].tolist()

    # algorithmic bytes of the scan per launch: compressed bytes of the
    # blocks the query needs (surviving chunks, and within them the blocks
    # whose date_key zone map meets the predicate) in the 4 columns + their
    # block directory and segment index entries + the date_key chunk min/max
    # and block zone maps read by pruning
    bpc = fact.cols["date_key"].info.blocks_per_chunk

    def slots_of(chunks, zone=True):
        out = []
        dk = f["date_key"]
        for ch in chunks:
            for j in range(bpc):
                r0 = ch * ROWS_PER_CHUNK + j * ROWS_PER_BLOCK
                r1 = min(N_ROWS, ch * ROWS_PER_CHUNK + min(ROWS_PER_CHUNK, (j + 1) * ROWS_PER_BLOCK))
                if r0 >= r1:
                    continue
                if zone and (dk[r0:r1].max() < DATE_LO or dk[r0:r1].min() > DATE_HI):
                    continue
                out.append(ch * bpc + j)
        return out

    def alg_bytes(chunks, zone=True):
        slots = slots_of(chunks, zone)
        tot = 0
        for name, c in fact.cols.items():
            info = c.info
            sel = c.blocks()[slots]
            tot += int(sel[:, 2].sum()) + 16 * len(sel) + (8 * info.lz4_segments * len(sel) if info.lz4_segments > 1 else 0)
        return tot + 8 * fact.cols["date_key"].info.n_chunks + (8 * bpc * len(chunks) if zone else 0)

    # the step (date table build, result clear, pruning + fused scan: one
    # library call) captured once as a CUDA graph and replayed per step, so
    # the host's launch calls do not pace the device
    def step_body():
        q.ht.build(q._dk, None, preds=[(q._ok, 1, 1)])
        q.result.zero_()
        q.plan.launch()

    side = torch.cuda.Stream()
    side.wait_stream(stream)
    with torch.cuda.stream(side):
        step_body()
    stream.wait_stream(side)
    torch.cuda.synchronize()
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph):
        step_body()
    torch.cuda.synchronize()
    for _ in range(args.warmup):
        graph.replay()
    torch.cuda.synchronize()
    if int(q.result.item()) != got:
        raise SystemExit("graph-replayed step differs from the direct call")

    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    with Clocks(dev) as clk:
        t_wall = time.perf_counter()
        for i in range(args.steps):
            flush.zero_()  # evict the previous step's tiles from L2 (untimed)
            a, c = ev[i]
            a.record(stream)
            graph.replay()
            c.record(stream)
        torch.cuda.synchronize()
        t_wall = time.perf_counter() - t_wall
    if world > 1:
        dist.barrier()
    step_ms = [a.elapsed_time(c) for a, c in ev]
    ms = max_over_ranks(float(np.mean(step_ms)), world, "cuda")
    if int(q.result.item()) != got:
        raise SystemExit("timed steps changed the result")
    # the fused scan alone (pruning + scan, one library call), launched directly
    scan_ms = []
    for _ in range(args.steps):
        flush.zero_()
        q.ht.build(q._dk, None, preds=[(q._ok, 1, 1)])
        q.result.zero_()
        b = torch.cuda.Event(enable_timing=True)
        c = torch.cuda.Event(enable_timing=True)
        b.record(stream)
        q.plan.launch()
        c.record(stream)
        c.synchronize()
        scan_ms.append(b.elapsed_time(c))
    scan_avg = float(np.mean(scan_ms))

    # full-table scan: the same Q1 plan over every date (pruning off), so every
    # tile needs all four columns -- the decode-bound throughput of the kernel
    ok_all = np.ones(len(dd["d_key"]), dtype=bool)
    q_all = queries.Q1Query(fact, dd, ok_all, int(dd["d_key"].min()), int(dd["d_key"].max()), *DISC, *QTY,
                            prune=False)
    m_all = (f["discount"] >= DISC[0]) & (f["discount"] <= DISC[1]) & (f["quantity"] >= QTY[0]) & \
            (f["quantity"] <= QTY[1])
    want_all = int((f["extended_price"][m_all].astype(np.int64) * f["discount"][m_all].astype(np.int64)).sum())
    if q_all.run() != want_all:
        raise SystemExit("full scan result differs from the numpy sum")
    for _ in range(3):
        q_all.launch()
    all_ms = []
    for _ in range(max(3, min(args.steps, 10))):
        flush.zero_()
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        q_all.result.zero_()
        a.record(stream)
        q_all.plan.launch()
        b.record(stream)
        torch.cuda.synchronize()
        all_ms.append(a.elapsed_time(b))
    all_ms_avg = float(np.mean(all_ms))
    all_bytes = alg_bytes(range(fact.cols["date_key"].info.n_chunks), zone=False)

    # e2e: pinned-host residency, date dimension in, result out
    fact_h = queries.encode_fact(f, {"date_key": "cascaded"}, ROWS_PER_CHUNK, ROWS_PER_BLOCK, args.segments,
                                 residency="pinned")
    qh = queries.Q1Query(fact_h, dd, ok, DATE_LO, DATE_HI, *DISC, *QTY, prune=True)
    res_h = torch.zeros(1, dtype=torch.int64).pin_memory()
    h2d_scan = alg_bytes(kept_chunks) - 8 * fact.cols["date_key"].info.n_chunks - 8 * bpc * len(kept_chunks)

    def e2e_step():
        dk_d.copy_(dk_h, non_blocking=True)
        ok_d.copy_(ok_h, non_blocking=True)
        qh.ht.build(dk_d, None, preds=[(ok_d, 1, 1)])
        qh.launch()
        res_h.copy_(qh.result, non_blocking=True)

    for _ in range(args.warmup):
        e2e_step()
    torch.cuda.synchronize()
    if int(res_h.item()) != want:
        raise SystemExit("e2e result mismatch")
    e_ms = []
    for _ in range(args.steps):
        flush.zero_()
        torch.cuda.synchronize()
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(stream)
        e2e_step()
        b.record(stream)
        b.synchronize()
        e_ms.append(a.elapsed_time(b))
    e2e_ms = max_over_ranks(float(np.mean(e_ms)), world, "cuda")

    pk, pk_kind = peaks()
    scan_bytes = alg_bytes(kept_chunks)
    achieved = scan_bytes / (scan_avg * 1e-3) / 1e9
    line = {
        "metric": "rows/s & GB/s vs HBM roofline; p50/p99 latency batched vs one-query-at-a-time",
        "value": N_ROWS * world / (ms * 1e-3),
        "unit": "rows/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": ms,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "int32",
        "data": "synthetic (seeded, configs[1] shapes and distributions)",
        "config": {"workload": WORKLOAD, "rows": N_ROWS, "chunks": N_ROWS // ROWS_PER_CHUNK, "chunks_scanned": kept,
                   "lz4_segments": args.segments, "residency": "hbm", "l2": "flushed between steps (256 MiB write)", "launch": "step replayed from a CUDA graph",
                   "parallelism": f"replicas x{world}", "comp_bytes": comp},
        "result": got,
        "latency_ms": {"p50": float(np.percentile(step_ms, 50)), "p99": float(np.percentile(step_ms, 99))},
        "scan_kernel_ms": scan_avg,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": pk, "unit": "GB/s", "frac": achieved / pk,
                     "traffic": profile_traffic(), "peak_kind": pk_kind,
                     "algorithmic_bytes_per_launch": scan_bytes},
        "full_scan": {"ms": all_ms_avg, "rows_per_s": N_ROWS / (all_ms_avg * 1e-3),
                      "comp_gbs": all_bytes / (all_ms_avg * 1e-3) / 1e9,
                      "roofline_frac": all_bytes / (all_ms_avg * 1e-3) / 1e9 / pk,
                      "uncomp_gbs": N_ROWS * 16 / (all_ms_avg * 1e-3) / 1e9},
        "e2e": {"value": N_ROWS * world / (e2e_ms * 1e-3), "unit": "rows/s",
                "h2d_bytes_per_step": int(h2d_scan + dd["d_key"].nbytes + ok.astype(np.int32).nbytes),
                "d2h_bytes_per_step": 8, "ms_per_step": e2e_ms, "residency": "pinned host (zero-copy reads)"},
        "gpu_launches": 2 * args.steps,  # date-table build (one launch for a small table) + fused scan (prunes its own work)
        "clocks": clk.summary(),
        "wall_s_timed": t_wall,
    }
    return line, f, dd


# --------------------------------------------------- batched and serving forms

def _hbm_bytes(spec):
    """Device bytes a request holds while it runs: its group table or result."""
    return 8 if spec.groups is None else 16 * (2 * spec.groups.max_groups) + 8


def batched_section(t, n_queries=256, seed=7, choices=None):
    """configs[3]-style batch: n queries on log-uniform slices (1M..100M rows)
    mixing the scan, star-join and high-cardinality templates.  One query at
    a time (its own launch sequence, back to back on one stream) vs all
    queries in one persistent launch replayed from a CUDA graph."""
    import torch

    from golap_public_b200 import api, autotune, workload

    choices = choices or {}
    rng = np.random.default_rng(seed)
    specs = workload.random_queries(t, n_queries, rng, ht_layout=autotune.layouts(choices))
    singles = {m: [api.Batch([(s.plan, s.row_lo, s.row_hi)], m) for s in specs] for m in ("queue", "shared")}
    for s, b in zip(specs, singles["shared"]):
        b.set_launch(**autotune.choose(choices, [s.template]))
    batch = api.Batch([(s.plan, s.row_lo, s.row_hi) for s in specs])
    launch = autotune.tune_launch(batch)  # the launch shape measured on this batch
    stream = torch.cuda.current_stream()
    single_mode = "queue"

    def one_at_a_time():
        for b in singles[single_mode]:
            b.run()

    def timed(fn, reps):
        ts = []
        for _ in range(reps):
            torch.cuda.synchronize()
            a = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            a.record(stream)
            fn()
            b.record(stream)
            b.synchronize()
            ts.append(a.elapsed_time(b))
        return float(np.median(ts))

    t_single = {}
    ref = None
    for m in ("queue", "shared"):
        single_mode = m
        one_at_a_time()
        torch.cuda.synchronize()
        got = [workload.read_result(s) for s in specs]
        if ref is not None and got != ref:
            raise SystemExit("one-at-a-time results differ between execution forms")
        ref = got
        t_single[m] = timed(one_at_a_time, 3)
    single_mode = min(t_single, key=t_single.get)  # the faster single-query form is the baseline
    batch.graph()
    torch.cuda.synchronize()
    if [workload.read_result(s) for s in specs] != ref:
        raise SystemExit("batched results differ from one-at-a-time results")
    t_one = t_single[single_mode]
    t_batch = timed(batch.graph, 5)
    rows = sum(s.row_hi - s.row_lo for s in specs)
    mix = {k: sum(1 for s in specs if s.template == k) for k in ("scan", "star", "highcard")}
    return {"queries": n_queries, "mix": mix, "slice_rows_total": rows, "batch_form": batch.mode,
            "batch_launch": launch,
            "one_at_a_time_ms": t_one, "one_at_a_time_form": single_mode,
            "one_at_a_time_ms_by_form": t_single, "batched_graph_ms": t_batch,
            "one_at_a_time_qps": n_queries / (t_one * 1e-3), "batched_qps": n_queries / (t_batch * 1e-3),
            "speedup": t_one / t_batch, "results_identical": True}


def serving_section(t, rates=(200, 1000, 2000), seconds=2.0, seed=9, max_backlog=300, choices=None):
    """configs[4]-style open loop: Poisson arrivals at each rate for `seconds`,
    60% pruned scans / 30% star joins / 10% Zipf group-bys over the whole
    resident table, served by the continuous-batching server and by a
    one-at-a-time server (one request per launch, one in flight).  A server
    that falls more than `max_backlog` requests behind is saturated: the
    arrivals stop there (counted as `shed`) so that the drain stays bounded."""
    import threading

    from golap_public_b200 import api, autotune, workload

    choices = choices or {}
    rng = np.random.default_rng(seed)
    pool = workload.random_queries(t, 384, rng, min_rows=t.n_rows, max_rows=t.n_rows,
                                   ht_layout=autotune.layouts(choices))
    threads = 0  # automatic launch shape per served batch (most resident warps for its footprint)
    out = {"batch_threads": "automatic"}
    for mode, (inflight, maxb) in (("batched", (4, 128)), ("one_at_a_time", (1, 1))):
        res = {}
        for rate in rates:
            sv = api.Server(max_inflight=inflight, max_batch=maxb, hbm_budget=120 << 30, batch_threads=threads)
            arr = np.cumsum(rng.exponential(1.0 / rate, int(rate * seconds)))
            busy = {}
            lats = []
            lock = threading.Lock()
            t0 = time.perf_counter()
            shed = 0
            for i, at in enumerate(arr):
                if sv.stats()["queued"] >= max_backlog:
                    shed = len(arr) - i
                    break
                spec_i = i % len(pool)
                if spec_i in busy:  # a pooled request's buffers are reused only after it finished
                    lats.append(sv.wait(busy.pop(spec_i), 300.0))
                while time.perf_counter() - t0 < at:
                    pass
                s = pool[spec_i]
                tk = sv.submit(s.plan, s.row_lo, s.row_hi, _hbm_bytes(s))
                busy[spec_i] = tk
            for tk in busy.values():
                lats.append(sv.wait(tk, 300.0))
            elapsed = time.perf_counter() - t0
            st = sv.stats()
            sv.close()
            lats = np.array(lats)
            res[str(rate)] = {"offered_qps": rate, "completed": int(st["completed"]), "shed": shed,
                              "sustained_qps": float(st["completed"] / elapsed),
                              "p50_ms": float(np.percentile(lats, 50)), "p99_ms": float(np.percentile(lats, 99)),
                              "mean_batch": float(st["queries_in_batches"] / max(1, st["batches"]))}
        out[mode] = res
    return out


# ----------------------------------------------------------------- CPU arm

def cpu_baseline(f, dd, steps=3, warmup=1, threads=None):
    """The reference's CPU path on the same data (see ref_cpu_q1 in oracle/ref_harness.cu)."""
    from oracle import oracle as O

    threads = threads or os.cpu_count() or 1
    ok = (dd["d_yearmonthnum"] == 199401).astype(np.uint8)
    n_chunks = N_ROWS // ROWS_PER_CHUNK
    bpc = -(-ROWS_PER_CHUNK // ROWS_PER_BLOCK)
    mins, maxs = O.chunk_minmax(f["date_key"], ROWS_PER_CHUNK)
    kind = "reference" if O.ref_available() else "port"
    if kind == "port":
        t = []
        for _ in range(steps):
            t0 = time.perf_counter()
            keep = O.minmax_keep(mins, maxs, DATE_LO, DATE_HI)
            r = O.q1(f["date_key"], f["discount"], f["quantity"], f["extended_price"], dd["d_key"], ok, *DISC, *QTY,
                     keep_chunk=keep, rows_per_chunk=ROWS_PER_CHUNK)
            t.append(time.perf_counter() - t0)
        ms = 1e3 * float(np.mean(t))
        return {"value": N_ROWS / (ms * 1e-3), "unit": "rows/s", "cores": 1, "kind": "port",
                "sample": "full query (oracle restatement, 1 thread)", "ms": ms, "result": r}
    R = O.ref()
    stride = ROWS_PER_BLOCK * 4 + ROWS_PER_BLOCK * 4 // 255 + 64
    comp, sizes = [], []
    for name in ("discount", "quantity", "extended_price"):
        v = f[name]
        buf = np.zeros(n_chunks * bpc * stride, np.uint8)
        sz = np.zeros(n_chunks * bpc, np.int32)
        for c in range(n_chunks):
            part = np.ascontiguousarray(v[c * ROWS_PER_CHUNK:(c + 1) * ROWS_PER_CHUNK])
            assert R.ref_lz4_compress_blocks(O._ptr(part), part.nbytes, ROWS_PER_BLOCK * 4,
                                             O._ptr(buf[c * bpc * stride:]), stride, O._ptr(sz[c * bpc:])) == 0
        comp.append(buf)
        sizes.append(sz)
    import ctypes as C

    comp_ptrs = (C.c_void_p * 3)(*[b.ctypes.data for b in comp])
    size_ptrs = (C.c_void_p * 3)(*[s.ctypes.data for s in sizes])
    res = None
    times = []
    for i in range(warmup + steps):
        el = C.c_double()
        scanned = C.c_uint64()
        r = R.ref_cpu_q1(threads, N_ROWS, ROWS_PER_CHUNK, ROWS_PER_BLOCK, O._ptr(f["date_key"]), O._ptr(mins),
                         O._ptr(maxs), comp_ptrs, stride, size_ptrs, O._ptr(dd["d_key"]), O._ptr(ok), len(ok),
                         DATE_LO, DATE_HI, *DISC, *QTY, C.byref(el), C.byref(scanned))
        res = r
        if i >= warmup:
            times.append(el.value)
    ms = float(np.mean(times))
    return {"value": N_ROWS / (ms * 1e-3), "unit": "rows/s", "cores": threads, "kind": "reference",
            "sample": f"full query: min/max pruning to {scanned.value} of {n_chunks} chunks, LZ4CPUManager decode of "
                      "discount/quantity/extended_price (liblz4 blocks of 64 KiB), HostHashMap date join; "
                      "date_key uncompressed (no reference CPU cascaded decoder)",
            "ms": ms, "result": int(res)}


def profile_batch(rows):
    """The batched section's 256-query batch (same seed and mix) with dense
    join tables, run three times in the shared form; prints its device time."""
    import torch

    from golap_public_b200 import api, workload

    t = workload.build_table(rows, ht_layouts=("dense",))
    specs = workload.random_queries(t, 256, np.random.default_rng(7), ht_layout="dense")
    batch = api.Batch([(s.plan, s.row_lo, s.row_hi) for s in specs], "shared")
    stream = torch.cuda.current_stream()
    for i in range(3):
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(stream)
        batch.run()
        b.record(stream)
        b.synchronize()
        api.scan_check()
        print(json.dumps({"profile_batch": i, "rows": rows, "threads": batch.threads, "ms": a.elapsed_time(b)}))


def main():
    global N_ROWS
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="gx", choices=["gx", "reference"])
    ap.add_argument("--segments", type=int, default=128)
    ap.add_argument("--seed", type=int, default=0xBEE5BEE5)
    ap.add_argument("--no-check", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-batch", action="store_true", help="skip the batched and serving sections")
    ap.add_argument("--batch-rows", type=int, default=100_000_000)
    ap.add_argument("--no-tune", action="store_true", help="batched/serving with the default launch shape")
    ap.add_argument("--rows", type=int, default=N_ROWS,
                    help="fact rows of the Q1 workload (default: the measured 60M-row configuration; smaller "
                         "values are for profiler captures)")
    ap.add_argument("--tune-rows", type=int, default=20_000_000)
    ap.add_argument("--profile-batch", action="store_true",
                    help="only build the batch table and run the 256-query mixed batch (shared form, dense join "
                         "tables, automatic launch shape) three times: the command profiler captures use")
    args = ap.parse_args()
    args.warmup = max(3, args.warmup)
    N_ROWS = args.rows
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))

    if args.profile_batch:
        profile_batch(args.batch_rows)
        return

    if args.impl == "reference":
        if rank != 0:
            return
        f, dd = make_data(args.seed)
        cb = cpu_baseline(f, dd, steps=args.steps, warmup=args.warmup)
        line = {
            "impl": "reference",
            "metric": "rows/s & GB/s vs HBM roofline; p50/p99 latency batched vs one-query-at-a-time",
            "value": cb["value"], "unit": "rows/s", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": cb["ms"], "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "int32", "data": "synthetic (seeded, configs[1] shapes and distributions)",
            "config": {"workload": WORKLOAD, "rows": N_ROWS, "chunks": N_ROWS // ROWS_PER_CHUNK},
            "result": cb["result"],
            "cpu_baseline": {k: cb[k] for k in ("value", "unit", "cores", "kind", "sample")},
            "e2e": {"value": cb["value"], "unit": "rows/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        }
        print(json.dumps(line))
        return

    if world > 1:
        import torch
        import torch.distributed as dist
        from datetime import timedelta

        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", 0)))
        dist.init_process_group("nccl", timeout=timedelta(seconds=300))
    line, f, dd = gpu_arm(args, rank, world)
    if not args.no_batch:
        from golap_public_b200 import autotune, workload

        choices = {}
        if not args.no_tune:
            tr = autotune.tune(n_rows=args.tune_rows, queries_per_template=16, reps=3)
            choices = {t: v["best"] for t, v in tr["templates"].items()}
            line["autotune"] = {"sample_rows": args.tune_rows, "queries_per_template": 16, "tune_s": tr["tune_s"],
                                "grid": {k: list(v) for k, v in autotune.SPACE.items()}, "best": choices,
                                "default_ms": {t: next(p["ms"] for p in v["points"]
                                                       if all(p[k] == autotune.DEFAULT[k] for k in autotune.DEFAULT))
                                               for t, v in tr["templates"].items()}}
        cfg = autotune.table_config(choices)
        t_build = time.perf_counter()
        wt = workload.build_table(args.batch_rows, rows_per_chunk=cfg["rows_per_chunk"], ht_layouts=cfg["ht_layouts"])
        build_s = time.perf_counter() - t_build
        line["batched"] = batched_section(wt, choices=choices)
        line["serving"] = serving_section(wt, choices=choices)
        line["batched"]["table_rows"] = args.batch_rows
        line["batched"]["table_rows_per_chunk"] = cfg["rows_per_chunk"]
        line["batched"]["table_build_s"] = build_s
        del wt
    if rank == 0 and not args.no_cpu:
        cb = cpu_baseline(f, dd, steps=3, warmup=1)
        line["cpu_baseline"] = {k: cb[k] for k in ("value", "unit", "cores", "kind", "sample")}
        line["cpu_baseline"]["ms"] = cb["ms"]
        if cb["result"] != line["result"]:
            raise SystemExit(f"cpu baseline result {cb['result']} != gpu {line['result']}")
    if world > 1:
        import torch.distributed as dist

        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line))


if __name__ == "__main__":
    main()
