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
            flushed between steps; surviving_rows_per_s counts only the
            rows of the tiles the scan reads.
  latency   p50/p99 of the same step over at least one second of replays.
  e2e       the same query with the compressed columns in pinned host
            memory, read by the kernels over PCIe, timed through the public
            API with the date dimension copied in and the result read back.
  roofline  the fused scan kernel of the step: algorithmic bytes
            (compressed bytes of the surviving tiles + their directory /
            side-index entries + min/max metadata) per launch / launch
            time, against the measured HBM copy bandwidth.
  full_scan the same plan over every date (no pruning, every tile needs
            all four columns): the bandwidth-bound case, with its own
            roofline; full_scan_lz4_matches repeats it with the LZ4 columns
            encoded with 4-byte matches (token-heavy streams).
  star_join the 600,000,000-row star join + group-by: three filtered
            dimension-table builds (customer 3M, supplier 200k, date) and
            the fused probe/aggregate scan; rows/s, roofline, e2e from
            pinned host memory, the reference CPU arm on the same bytes.
  cpu_baseline  the reference's CPU path on the same compressed bytes:
            LZ4CPUManager decompression (cascaded date_key: the harness's
            decoder of this build's format) + the query loop over
            HostHashMap, all host cores.

--impl reference runs only the CPU path (rank 0) and prints its line.
--gpus N runs N independent replicas (one per GPU; the query does not need
a collective); value is the total over ranks, time is the max over ranks.
Clock samples are written as CSV into the directory named by
GX_BENCH_CLOCKS_DIR when it is set.
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
STREAM_GROUP = 8  # chunks per staged group of the streamed (PCIe) scan
WORKLOAD = ("Q1 shape on 60M rows sorted by date_key: date_key cascaded, discount/quantity/extended_price "
            "LZ4 on 64 KiB blocks, 1M-row chunks with min/max; month Jan 1994, discount 4..6, quantity 26..35")


def pinned_h2d_gbs(nbytes=1 << 30, reps=3):
    """Host->HBM copy bandwidth from pinned memory: one large cudaMemcpyAsync, best of `reps`."""
    import torch

    h = torch.empty(nbytes, dtype=torch.uint8).pin_memory()
    d = torch.empty(nbytes, dtype=torch.uint8, device="cuda")
    best = float("inf")
    for _ in range(reps + 1):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        d.copy_(h, non_blocking=True)
        b.record()
        b.synchronize()
        best = min(best, a.elapsed_time(b))
    del h, d
    return nbytes / (best * 1e-3) / 1e9


def peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def profile_traffic(name="warp_scan_kernel_q1_pruned_60M.md", rows=None):
    """DRAM bytes (read + write) per launch of the fused scan kernel from a committed ncu summary, or
    None.  With `rows`, a capture of a smaller case (its `captured_rows`) is scaled to `rows`: used
    only for the full scan, whose traffic grows in proportion to the rows."""
    p = ROOT / "profiles" / name
    if not p.exists():
        return None
    text = p.read_text()
    m = re.search(r"traffic_bytes_per_launch:\s*([0-9]+)", text)
    if not m:
        return None
    t = int(m.group(1))
    if rows is not None:
        r = re.search(r"captured_rows:\s*([0-9]+)", text)
        if not r:
            return None
        t = int(round(t * rows / int(r.group(1))))
    return t


class Clocks:
    """Samples SM clocks and clock-event (throttle) reasons through NVML in a
    background thread (every 2 ms) while the timed region runs; the samples
    are also written as CSV into $GX_BENCH_CLOCKS_DIR when it is set."""

    NAMES = (("hw_slowdown", 0x8), ("hw_thermal_slowdown", 0x40), ("sw_thermal_slowdown", 0x20),
             ("sw_power_cap", 0x4), ("hw_power_brake_slowdown", 0x80))

    def __init__(self, gpu: int, tag: str = "step"):
        self.gpu = gpu
        self.samples = []
        self.max_mhz = None
        self.err = None
        d = os.environ.get("GX_BENCH_CLOCKS_DIR")
        self.path = Path(d) / f"clocks_bench_{tag}_{os.getpid()}.csv" if d else None

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
        if self.path is None:
            return
        try:
            self.path.parent.mkdir(parents=True, exist_ok=True)
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


Q1_COLS = ("date_key", "discount", "quantity", "extended_price")
Q3_COLS = ("date_key", "cust_key", "supp_key", "revenue")


def comp_columns(fact, names):
    """(payload, blocks, codec) of each column: the compressed bytes the GPU scans, for the CPU arm."""
    return [(fact.cols[n].payload_view(), fact.cols[n].blocks(), 1 if fact.cols[n].codec == "lz4" else 2)
            for n in names]


def present_index(info, n_rows):
    """Index into the present-block list (gx_column_blocks order) of every block slot, -1 if absent."""
    bpc = info.blocks_per_chunk
    idx = np.full(info.n_chunks * bpc, -1, np.int64)
    k = 0
    for ch in range(info.n_chunks):
        rows = min(info.rows_per_chunk, n_rows - ch * info.rows_per_chunk)
        nb = -(-rows // info.rows_per_block)
        idx[ch * bpc: ch * bpc + nb] = np.arange(k, k + nb)
        k += nb
    return idx


def alg_bytes(fact, names, slots, n_chunks_meta, zone_blocks):
    """Algorithmic bytes of one scan: compressed bytes of the given block slots in the
    named columns + 16 B of directory per block + 8 B per side-index entry, + 8 B of
    chunk min/max per chunk and 8 B of zone map per block checked."""
    tot = 0
    for name in names:
        c = fact.cols[name]
        info = c.info
        pidx = present_index(info, fact.n_rows)[np.asarray(slots, np.int64)] if len(slots) else []
        sel = c.blocks()[pidx] if len(slots) else np.zeros((0, 4), np.uint64)
        per = info.lz4_segments if (c.codec == "lz4" and info.lz4_segments > 1) else (
            -(-info.rows_per_block // 2048) if c.codec == "cascaded" else 0)
        tot += int(sel[:, 2].sum()) + 16 * len(sel) + 8 * per * len(sel)
    return tot + 8 * n_chunks_meta + 8 * zone_blocks


def time_launches(fn, reps, stream, flush=None, pre=None):
    """Device time (ms, CUDA events on `stream`) of fn() per rep, L2 flushed before each."""
    import torch

    out = []
    for _ in range(reps):
        if flush is not None:
            flush.zero_()
        if pre is not None:
            pre()
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(stream)
        fn()
        b.record(stream)
        b.synchronize()
        out.append(a.elapsed_time(b))
    return out


REF_GPU = ROOT / "baseline" / "_ref" / "libgolaprefgpu.so"


def ref_gpu_lib():
    """The same-box GPU reference point (baseline/refgpu/ref_gpu.cu), or None when not built."""
    import ctypes as C

    if not REF_GPU.exists():
        return None
    R = C.CDLL(str(REF_GPU))
    P, u64, i32 = C.c_void_p, C.c_uint64, C.c_int32
    R.ref_gpu_q1.restype = C.c_int64
    R.ref_gpu_q1.argtypes = [P, P, P, P, u64, P, P, u64, P, C.c_uint32, C.c_int, C.POINTER(C.c_double)]
    R.ref_gpu_q3.restype = C.c_int64
    R.ref_gpu_q3.argtypes = [P, P, P, P, u64, P, P, P, u64, P, P, P, u64, P, P, u64, i32, i32, i32, P, C.c_uint32,
                             C.c_int, P, P, u64, C.POINTER(u64), C.POINTER(C.c_double)]
    return R


def decompressed(fact, names):
    """The named columns decoded into int32 device tensors (one library call each)."""
    import torch

    from golap_public_b200 import api

    out = {}
    for k in names:
        t = torch.empty(fact.n_rows, dtype=torch.int32, device="cuda")
        api.ChunkDecompressor(fact.cols[k]).chunks(0, fact.cols[k].info.n_chunks, t)
        out[k] = t
    api.scan_check()
    return out


def roofline(bytes_, ms, pk, pk_kind, traffic=None):
    a = bytes_ / (ms * 1e-3) / 1e9
    return {"bound": "hbm", "achieved": a, "peak": pk, "unit": "GB/s", "frac": a / pk, "traffic": traffic,
            "peak_kind": pk_kind, "algorithmic_bytes_per_launch": int(bytes_)}


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
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    pk, pk_kind = peaks()

    for _ in range(args.warmup):
        q.ht.build(q._dk, None, preds=[(q._ok, 1, 1)])
        q.launch()
    torch.cuda.synchronize()
    got = q.run()
    kept = int(q.keep.sum().item())
    kept_chunks = np.nonzero(q.keep.cpu().numpy())[0].tolist()

    # block slots the pruned scan reads: surviving chunks, and within them the
    # blocks whose date_key zone map meets the predicate
    bpc = fact.cols["date_key"].info.blocks_per_chunk
    n_chunks = fact.cols["date_key"].info.n_chunks

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

    pruned_slots = slots_of(kept_chunks)
    scan_bytes = alg_bytes(fact, Q1_COLS, pruned_slots, n_chunks, bpc * len(kept_chunks))
    bi = fact.cols["date_key"].blocks()
    surviving_rows = int(bi[present_index(fact.cols["date_key"].info, N_ROWS)[pruned_slots], 3].sum())

    # the step (result clear, date table build, pruning + fused scan: one
    # library call) captured once as a CUDA graph and replayed per step, so
    # the host's launch calls do not pace the device; the scan follows the
    # build directly, so that its table-free work overlaps the build
    def step_body():
        q.result.zero_()
        q.ht.build(q._dk, None, preds=[(q._ok, 1, 1)])
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

    # latency distribution: the same graph replayed for at least one second
    lat_ms, lat_wall = [], time.perf_counter()
    with Clocks(dev, "latency") as clk_lat:
        while time.perf_counter() - lat_wall < args.latency_s or len(lat_ms) < 100:
            lat_ms += time_launches(graph.replay, 200, stream, flush)
        lat_wall = time.perf_counter() - lat_wall

    # the fused scan alone (pruning + scan, one library call), launched directly
    scan_ms = time_launches(q.plan.launch, max(args.steps, 20), stream, flush,
                            pre=lambda: (q.ht.build(q._dk, None, preds=[(q._ok, 1, 1)]), q.result.zero_()))
    scan_avg = float(np.mean(scan_ms))

    # full-table scan: the same Q1 plan over every date (pruning off), so every
    # tile needs all four columns -- the bandwidth-bound throughput of the kernel
    ok_all = np.ones(len(dd["d_key"]), dtype=bool)
    m_all = (f["discount"] >= DISC[0]) & (f["discount"] <= DISC[1]) & (f["quantity"] >= QTY[0]) & \
            (f["quantity"] <= QTY[1])
    want_all = int((f["extended_price"][m_all].astype(np.int64) * f["discount"][m_all].astype(np.int64)).sum())
    all_slots = slots_of(range(n_chunks), zone=False)

    def full_scan(fct, label, traffic=None):
        qa = queries.Q1Query(fct, dd, ok_all, int(dd["d_key"].min()), int(dd["d_key"].max()), *DISC, *QTY,
                             prune=False)
        if qa.run() != want_all:
            raise SystemExit(f"{label}: full scan result differs from the numpy sum")
        for _ in range(3):
            qa.launch()
        t = time_launches(qa.launch, max(5, min(args.steps, 20)), stream, flush)
        avg = float(np.mean(t))
        nbytes = alg_bytes(fct, Q1_COLS, all_slots, 0, 0)
        return {"ms": avg, "rows_per_s": N_ROWS / (avg * 1e-3), "comp_gbs": nbytes / (avg * 1e-3) / 1e9,
                "roofline_frac": nbytes / (avg * 1e-3) / 1e9 / pk, "uncomp_gbs": N_ROWS * 16 / (avg * 1e-3) / 1e9,
                "roofline": roofline(nbytes, avg, pk, pk_kind, traffic),
                "comp_bytes": {k: c.info.comp_bytes for k, c in fct.cols.items()}}

    full = full_scan(fact, "literal policy", profile_traffic("warp_scan_kernel_q1_fullscan_16M.md", N_ROWS))
    full["lz4_policy"] = "decode-cost-aware (lz4_min_match=0): random-valued columns stored as literal runs"
    # the same data with the LZ4 columns encoded with 4-byte matches
    fact_m = queries.encode_fact({k: f[k] for k in Q1_COLS if k != "date_key"}, {}, ROWS_PER_CHUNK, ROWS_PER_BLOCK,
                                 args.segments, lz4_min_match=4)
    fact_m.cols["date_key"] = fact.cols["date_key"]
    full_m = full_scan(fact_m, "4-byte matches")
    full_m["lz4_policy"] = "lz4_min_match=4 (every 4-byte repeat inside a segment becomes a match)"

    # same-box GPU reference point: the reference's own pipeline_q1_lineorder and
    # hash_map_build_pred_other compiled for sm_100a, on the decompressed columns
    ref_gpu = None
    R = ref_gpu_lib()
    if R is not None:
        import ctypes as C

        cols = decompressed(fact, Q1_COLS)
        ptrs = [C.c_void_p(cols[k].data_ptr()) for k in Q1_COLS]
        dkd = torch.from_numpy(dd["d_key"]).cuda()
        ref_gpu = {"what": "the reference's hash_map_build_pred_other + pipeline_q1_lineorder (one launch per "
                           "surviving 1M-row chunk, 512-thread CTAs) compiled for sm_100a, on columns already "
                           "decompressed into the reference's types (decompression not counted: a lower bound)"}
        for label, okv, chunks in (("pruned", ok, kept_chunks), ("full_scan", ok_all, list(range(n_chunks)))):
            ch = np.ascontiguousarray(chunks, np.uint32)
            okb = np.ascontiguousarray(okv.astype(np.uint8))
            rms = C.c_double()
            r = R.ref_gpu_q1(*ptrs, N_ROWS, C.c_void_p(dkd.data_ptr()), okb.ctypes.data_as(C.c_void_p), len(okb),
                             ch.ctypes.data_as(C.c_void_p), len(ch), 5, C.byref(rms))
            want_r = got if label == "pruned" else want_all
            ref_gpu[label] = {"ms": rms.value, "rows_per_s": N_ROWS / (rms.value * 1e-3), "result_equal": r == want_r,
                              "gx_ms": ms if label == "pruned" else full["ms"]}
            if r != want_r:
                raise SystemExit(f"reference GPU kernels gave {r}, the fused scan {want_r}")
        del cols

    # e2e: pinned-host residency, date dimension in, result out
    fact_h = queries.encode_fact(f, {"date_key": "cascaded"}, ROWS_PER_CHUNK, ROWS_PER_BLOCK, args.segments,
                                 residency="pinned")
    qh = queries.Q1Query(fact_h, dd, ok, DATE_LO, DATE_HI, *DISC, *QTY, prune=True)
    res_h = torch.zeros(1, dtype=torch.int64).pin_memory()
    h2d_scan = alg_bytes(fact, Q1_COLS, pruned_slots, 0, 0)

    def e2e_step():
        dk_d.copy_(dk_h, non_blocking=True)
        ok_d.copy_(ok_h, non_blocking=True)
        qh.ht.build(dk_d, None, preds=[(ok_d, 1, 1)])
        qh.launch()
        res_h.copy_(qh.result, non_blocking=True)

    for _ in range(args.warmup):
        e2e_step()
    torch.cuda.synchronize()
    if int(res_h.item()) != got:
        raise SystemExit("e2e result mismatch")
    e_ms = time_launches(e2e_step, args.steps, stream, flush, pre=torch.cuda.synchronize)
    e2e_zc_ms = max_over_ranks(float(np.mean(e_ms)), world, "cuda")
    # the same step with the surviving chunks staged into HBM by bulk copies
    # (gx_scan_streamed) instead of zero-copy reads
    qh.stream_group = STREAM_GROUP
    e2e_step()
    torch.cuda.synchronize()
    if int(res_h.item()) != got:
        raise SystemExit("streamed e2e result mismatch")
    e_ms = time_launches(e2e_step, args.steps, stream, flush, pre=torch.cuda.synchronize)
    e2e_st_ms = max_over_ranks(float(np.mean(e_ms)), world, "cuda")
    # full scan through PCIe: every chunk's compressed bytes cross the link
    qf = queries.Q1Query(fact_h, dd, ok_all, int(dd["d_key"].min()), int(dd["d_key"].max()), *DISC, *QTY,
                         prune=False)
    qf.stream_group = STREAM_GROUP
    qf.launch()
    torch.cuda.synchronize()
    if int(qf.result.item()) != want_all:
        raise SystemExit("streamed full-scan result mismatch")
    e_ms = time_launches(qf.launch, args.steps, stream, flush, pre=torch.cuda.synchronize)
    full_st_ms = max_over_ranks(float(np.mean(e_ms)), world, "cuda")
    h2d_full = alg_bytes(fact, Q1_COLS, all_slots, 0, 0)
    h2d_peak = pinned_h2d_gbs()
    e2e_ms, e2e_mode = min((e2e_zc_ms, "pinned host, zero-copy reads"),
                           (e2e_st_ms, f"pinned host, surviving chunks staged to HBM ({STREAM_GROUP}-chunk groups)"))
    del fact_h, qh, qf

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
        "config": {"workload": WORKLOAD, "rows": N_ROWS, "chunks": n_chunks, "chunks_scanned": kept,
                   "lz4_segments": args.segments, "residency": "hbm", "l2": "flushed between steps (256 MiB write)",
                   "launch": "step replayed from a CUDA graph", "parallelism": f"replicas x{world}",
                   "comp_bytes": comp},
        "result": got,
        "surviving_rows": surviving_rows,
        "surviving_rows_per_s": surviving_rows * world / (ms * 1e-3),
        "latency_ms": {"p50": float(np.percentile(lat_ms, 50)), "p99": float(np.percentile(lat_ms, 99)),
                       "mean": float(np.mean(lat_ms)), "samples": len(lat_ms), "timed_s": lat_wall,
                       "clocks": clk_lat.summary()},
        "scan_kernel_ms": scan_avg,
        "roofline": roofline(scan_bytes, scan_avg, pk, pk_kind, profile_traffic()),
        "roofline_full_scan": full["roofline"],
        "full_scan": full,
        "full_scan_lz4_matches": full_m,
        "reference_gpu": ref_gpu,
        "e2e": {"value": N_ROWS * world / (e2e_ms * 1e-3), "unit": "rows/s",
                "h2d_bytes_per_step": int(h2d_scan + dd["d_key"].nbytes + ok.astype(np.int32).nbytes),
                "d2h_bytes_per_step": 8, "ms_per_step": e2e_ms, "residency": e2e_mode,
                "zero_copy_ms": e2e_zc_ms, "streamed_ms": e2e_st_ms,
                "full_scan_streamed": {"ms": full_st_ms, "rows_per_s": N_ROWS * world / (full_st_ms * 1e-3),
                                       "h2d_bytes": h2d_full,
                                       "roofline": {"bound": "pcie", "achieved": h2d_full / (full_st_ms * 1e-3) / 1e9,
                                                    "peak": h2d_peak, "unit": "GB/s",
                                                    "frac": h2d_full / (full_st_ms * 1e-3) / 1e9 / h2d_peak,
                                                    "peak_kind": "measured here: one 1 GiB pinned host->HBM copy"}}},
        "gpu_launches": 2 * args.steps,  # date-table build (one launch for a small table) + fused scan (prunes its own work)
        "clocks": clk.summary(),
        "wall_s_timed": t_wall,
    }
    ctx = {"f": f, "dd": dd, "fact": fact, "fact_m": fact_m, "want_all": want_all}
    return line, ctx


def star_join_section(args, pk, pk_kind, world=1):
    """the 600M-row star join + group-by, one query per step:
    filtered builds of the customer (3M), supplier (200k) and date tables,
    then the fused scan probing customer -> supplier -> date and summing
    revenue per (c_nation, s_nation, year); min/max pruning on date_key."""
    import torch

    from golap_public_b200 import datagen, queries

    stream = torch.cuda.current_stream()
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    n = args.star_rows
    t0 = time.perf_counter()
    g = datagen.fact_q3(n, True, seed=args.seed)
    cust = datagen.dim_geo(3_000_000, args.seed, 21)
    supp = datagen.dim_geo(200_000, args.seed, 22)
    dd = datagen.date_dim()
    fact = queries.encode_fact({k: g[k] for k in Q3_COLS}, {"date_key": "cascaded"}, ROWS_PER_CHUNK,
                               ROWS_PER_BLOCK, args.segments)
    # the customer dimension compressed like the fact table; its join table is
    # built from the compressed chunks inside every step
    cust_c = queries.encode_fact(cust, {"key": "cascaded", "nation": "cascaded", "region": "cascaded"},
                                 ROWS_PER_CHUNK, ROWS_PER_BLOCK, args.segments)
    build_s = time.perf_counter() - t0
    region, ylo, yhi = 2, 1992, 1997
    q = queries.Q3Query(fact, cust_c, supp, dd, region, ylo, yhi, ht_layout=args.star_layout)
    got = q.run()

    def step():
        q.agg.reset()
        q.build_customer()
        q.hs.build(q._keep_alive[3], q._keep_alive[4], preds=[(q._keep_alive[5], region, region)])
        q.hd.build(q._keep_alive[6], q._keep_alive[7], preds=[(q._keep_alive[7], ylo, yhi)])
        q.scan()

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    step_ms = time_launches(step, max(5, min(args.steps, 20)), stream, flush)
    if q.run() != got:
        raise SystemExit("star join: repeated steps changed the result")
    scan_ms = time_launches(q.launch, max(5, min(args.steps, 20)), stream, flush)
    ms, sms = float(np.mean(step_ms)), float(np.mean(scan_ms))
    kept = np.nonzero(q.keep.cpu().numpy())[0]
    info = fact.cols["date_key"].info
    bpc = info.blocks_per_chunk
    pidx = present_index(info, n)
    # blocks of the surviving chunks whose date_key zone map meets the year range
    bi = fact.cols["date_key"].blocks()
    lo_key, hi_key = ylo * 10000 + 101, yhi * 10000 + 1231
    slots = []
    for c in kept:
        for j in range(bpc):
            k = pidx[c * bpc + j]
            if k < 0:
                continue
            r0 = c * ROWS_PER_CHUNK + j * ROWS_PER_BLOCK
            blk = g["date_key"][r0:r0 + int(bi[k, 3])]
            if blk.max() >= lo_key and blk.min() <= hi_key:
                slots.append(c * bpc + j)
    nbytes = alg_bytes(fact, Q3_COLS, slots, info.n_chunks, bpc * len(kept))
    rows_scanned = int(bi[pidx[np.asarray(slots)], 3].sum())
    # dimension side of a step: the compressed customer columns and the supplier /
    # date key + payload + filter columns read, 8 B per inserted entry written
    dim_bytes = sum(c.info.comp_bytes for c in cust_c.cols.values()) + 200_000 * 12 + len(dd["d_key"]) * 8 + \
        8 * (int((cust["region"] == region).sum()) + int((supp["region"] == region).sum()) + 2192)
    # the customer build alone (one fused decode + filter + insert launch over 3M compressed rows)
    cust_ms = float(np.mean(time_launches(q.build_customer, 10, stream, flush)))
    out = {"rows": n, "chunks": fact.cols["date_key"].info.n_chunks, "chunks_scanned": int(len(kept)),
           "rows_scanned": rows_scanned, "ht_layout": args.star_layout,
           "workload": "star join + group-by: 600M-row fact (cust_key U[1,3M], supp_key U[1,200k], date_key sorted, "
                       "revenue U[100,1M]; date_key cascaded, others LZ4), customer 3M / supplier 200k / date 2,556; "
                       f"c.region == s.region == {region}, year {ylo}..{yhi}; SUM(revenue) GROUP BY "
                       "(c_nation, s_nation, year)",
           "table_build_s": build_s, "groups": len(got), "result_total": int(sum(got.values())),
           "ms_per_step": ms, "rows_per_s": n * world / (ms * 1e-3),
           "surviving_rows_per_s": rows_scanned * world / (ms * 1e-3),
           "scan_kernel_ms": sms, "roofline": roofline(nbytes, sms, pk, pk_kind),
           "step_bytes_incl_dims": nbytes + dim_bytes,
           "customer_build_ms": cust_ms,
           "customer_build": "3M-row customer join table built from compressed customer columns (key, nation, "
                             "region cascaded) in one fused decode + filter + insert launch",
           "comp_bytes": {k: c.info.comp_bytes for k, c in fact.cols.items()}}
    # same-box GPU reference point (the reference's HashMap / HashAggregate /
    # hash_map_build_pred_other and pipeline_q3's loop body, sm_100a)
    R = ref_gpu_lib()
    if R is not None:
        import ctypes as C

        cols = decompressed(fact, Q3_COLS)
        dev = {k: torch.from_numpy(np.ascontiguousarray(v)).cuda() for k, v in
               (("ck", cust["key"]), ("cn", cust["nation"]), ("cr", cust["region"]), ("sk", supp["key"]),
                ("sn", supp["nation"]), ("sr", supp["region"]), ("dk", dd["d_key"]), ("dy", dd["d_year"]))}
        ch = np.ascontiguousarray(kept, np.uint32)
        gk = np.zeros(4096, np.int64)
        gs = np.zeros(4096, np.int64)
        ng, rms = C.c_uint64(), C.c_double()
        vp = lambda t: C.c_void_p(t.data_ptr())  # noqa: E731
        R.ref_gpu_q3(vp(cols["date_key"]), vp(cols["cust_key"]), vp(cols["supp_key"]), vp(cols["revenue"]), n,
                     vp(dev["ck"]), vp(dev["cn"]), vp(dev["cr"]), len(cust["key"]), vp(dev["sk"]), vp(dev["sn"]),
                     vp(dev["sr"]), len(supp["key"]), vp(dev["dk"]), vp(dev["dy"]), len(dd["d_key"]), region, ylo, yhi,
                     ch.ctypes.data_as(C.c_void_p), len(ch), 3, gk.ctypes.data_as(C.c_void_p),
                     gs.ctypes.data_as(C.c_void_p), len(gk), C.byref(ng), C.byref(rms))
        ny = yhi - ylo + 1
        rg = {}
        for i in range(ng.value):
            cs_, y = divmod(int(gk[i]), ny)
            c, s_ = divmod(cs_, 25)
            rg[(c, s_, ylo + y)] = int(gs[i])
        out["reference_gpu"] = {
            "what": "the reference's hash_map_build_pred_other (customer/supplier/date), HashMap probes and "
                    "HashAggregate::add in pipeline_q3's loop body (one launch per surviving 1M-row chunk) compiled "
                    "for sm_100a, on columns already decompressed into the reference's types (decompression not "
                    "counted: a lower bound)",
            "ms": rms.value, "rows_per_s": n / (rms.value * 1e-3), "groups_equal": rg == got, "gx_ms": ms}
        if rg != got:
            raise SystemExit("star join: reference GPU kernels' groups differ from the fused scan's")
        del cols, dev

    # e2e: the fact columns in pinned host memory, dimension columns copied in, groups read back
    fact_h = queries.encode_fact({k: g[k] for k in Q3_COLS}, {"date_key": "cascaded"}, ROWS_PER_CHUNK,
                                 ROWS_PER_BLOCK, args.segments, residency="pinned")
    qh = queries.Q3Query(fact_h, cust, supp, dd, region, ylo, yhi, ht_layout=args.star_layout)
    host_dims = [torch.from_numpy(np.ascontiguousarray(a)).pin_memory() for a in
                 (cust["key"], cust["nation"], cust["region"], supp["key"], supp["nation"], supp["region"],
                  dd["d_key"], dd["d_year"])]

    def e2e_step():
        for hsrc, ddst in zip(host_dims, qh._keep_alive):
            ddst.copy_(hsrc, non_blocking=True)
        ck, cn, cr, sk, sn, sr, dk, dy = qh._keep_alive
        qh.hc.build(ck, cn, preds=[(cr, region, region)])
        qh.hs.build(sk, sn, preds=[(sr, region, region)])
        qh.hd.build(dk, dy, preds=[(dy, ylo, yhi)])
        return qh.run()

    if e2e_step() != got:
        raise SystemExit("star join e2e result mismatch")
    e_ms = []
    for _ in range(3):
        flush.zero_()
        torch.cuda.synchronize()
        t = time.perf_counter()
        e2e_step()
        e_ms.append((time.perf_counter() - t) * 1e3)
    e = float(np.mean(e_ms))
    out["e2e"] = {"value": n / (e * 1e-3), "unit": "rows/s", "ms_per_step": e,
                  "h2d_bytes_per_step": int(nbytes + sum(h.numel() * 4 for h in host_dims)),
                  "d2h_bytes_per_step": 16 * len(got),
                  "residency": "pinned host (zero-copy reads); host wall clock around each call, groups read back"}
    del fact_h, qh
    return out, {"g": g, "cust": cust, "supp": supp, "dd": dd, "fact": fact, "got": got, "region": region,
                 "ylo": ylo, "yhi": yhi}


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

def cpu_q1(cols, mins, maxs, dd, ok, lo, hi, steps=3, warmup=1, threads=None):
    """The reference's CPU path on the Q1 workload's compressed bytes (ref_cpu_q1_comp in
    oracle/ref_harness.cu): LZ4CPUManager decode + query1inmem's loop over HostHashMap."""
    import ctypes as C

    from oracle import oracle as O

    threads = threads or os.cpu_count() or 1
    arr = O.comp_cols(cols)
    okb = ok.astype(np.uint8)
    times, res = [], None
    ch, rows = C.c_uint64(), C.c_uint64()
    for i in range(warmup + steps):
        el = C.c_double()
        res = O.ref().ref_cpu_q1_comp(threads, N_ROWS, ROWS_PER_CHUNK, ROWS_PER_BLOCK, arr, O._ptr(mins),
                                      O._ptr(maxs), O._ptr(dd["d_key"]), O._ptr(okb), len(okb), lo, hi, *DISC, *QTY,
                                      C.byref(el), C.byref(ch), C.byref(rows))
        if i >= warmup:
            times.append(el.value)
    return float(np.mean(times)), int(res), ch.value, rows.value, threads


def cpu_baseline(fact, dd, steps=3, warmup=1, threads=None):
    """The headline query (January 1994, pruned) on the reference CPU path, same compressed bytes."""
    from oracle import oracle as O

    ok = dd["d_yearmonthnum"] == 199401
    mins, maxs = fact.cols["date_key"].minmax()
    if not O.ref_available():
        raise SystemExit("reference harness not built: __graft_entry__.build() compiles it where the reference "
                         "tree is present")
    ms, res, ch, rows, thr = cpu_q1(comp_columns(fact, Q1_COLS), mins, maxs, dd, ok, DATE_LO, DATE_HI, steps,
                                    warmup, threads)
    return {"value": N_ROWS / (ms * 1e-3), "unit": "rows/s", "cores": thr, "kind": "reference",
            "sample": f"full query: min/max pruning to {ch} of {N_ROWS // ROWS_PER_CHUNK} chunks ({rows} rows), "
                      "LZ4CPUManager decode of the GPU path's own discount/quantity/extended_price LZ4 blocks, "
                      "date_key pages decoded by the harness's decoder of this build's cascaded format (the "
                      "reference has no CPU decoder for its cascaded codec), HostHashMap date join; surviving "
                      "blocks split over all threads",
            "ms": ms, "result": res, "surviving_rows_per_s": rows / (ms * 1e-3)}


def cpu_full_scan(fact, dd, want, steps=2, warmup=1, threads=None):
    """The unpruned full scan (every date) on the reference CPU path, same compressed bytes."""
    ok_all = np.ones(len(dd["d_key"]), dtype=bool)
    mins, maxs = fact.cols["date_key"].minmax()
    ms, res, ch, rows, thr = cpu_q1(comp_columns(fact, Q1_COLS), mins, maxs, dd, ok_all, int(dd["d_key"].min()),
                                    int(dd["d_key"].max()), steps, warmup, threads)
    if res != want:
        raise SystemExit(f"cpu full scan result {res} != {want}")
    return {"value": N_ROWS / (ms * 1e-3), "unit": "rows/s", "cores": thr, "kind": "reference", "ms": ms,
            "sample": f"all {N_ROWS} rows, every date (no pruning), same compressed bytes as the GPU full scan"}


def cpu_star_join(ctx, steps=2, warmup=1, threads=None):
    """The 600M-row star join on the reference CPU path (ref_cpu_q3_comp in oracle/ref_harness.cu):
    filtered HostHashMap builds, probes customer -> supplier -> date, thread-local group maps
    merged through HostHashAggregate, over the GPU path's compressed bytes."""
    import ctypes as C

    from oracle import oracle as O

    threads = threads or os.cpu_count() or 1
    fact, cust, supp, dd = ctx["fact"], ctx["cust"], ctx["supp"], ctx["dd"]
    region, ylo, yhi = ctx["region"], ctx["ylo"], ctx["yhi"]
    keep = comp_columns(fact, Q3_COLS)  # the arrays stay alive while the harness reads them
    arr = O.comp_cols(keep)
    mins, maxs = fact.cols["date_key"].minmax()
    gk = np.zeros(4096, np.int64)
    gs = np.zeros(4096, np.int64)
    ng, ch, rows = C.c_uint64(), C.c_uint64(), C.c_uint64()
    n = fact.n_rows
    times = []
    for i in range(warmup + steps):
        el = C.c_double()
        O.ref().ref_cpu_q3_comp(threads, n, ROWS_PER_CHUNK, ROWS_PER_BLOCK, arr, O._ptr(mins), O._ptr(maxs),
                                O._ptr(cust["key"]), O._ptr(cust["nation"]), O._ptr(cust["region"]), len(cust["key"]),
                                O._ptr(supp["key"]), O._ptr(supp["nation"]), O._ptr(supp["region"]),
                                len(supp["key"]), O._ptr(dd["d_key"]), O._ptr(dd["d_year"]), len(dd["d_key"]),
                                region, ylo, yhi, O._ptr(gk), O._ptr(gs), len(gk), C.byref(ng), C.byref(el),
                                C.byref(ch), C.byref(rows))
        if i >= warmup:
            times.append(el.value)
    ny = yhi - ylo + 1
    cpu_groups = {}
    for i in range(ng.value):
        k = int(gk[i])
        cs, y = divmod(k, ny)
        c, s_ = divmod(cs, 25)
        cpu_groups[(c, s_, ylo + y)] = int(gs[i])
    ms = float(np.mean(times))
    return {"value": n / (ms * 1e-3), "unit": "rows/s", "cores": threads, "kind": "reference", "ms": ms,
            "sample": f"full query over all {n} rows ({ch.value} chunks survive min/max pruning): filtered builds "
                      "of customer/supplier/date, LZ4CPUManager decode of the GPU path's LZ4 blocks, the harness's "
                      "decoder for the cascaded date_key pages, HostHashMap probes, HostHashAggregate",
            "groups_equal_gpu": cpu_groups == ctx["got"]}


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


def profile_scan(kind, rows, segments):
    """One single-plan scan of the Q1 workload's shape on `rows` rows, for a
    profiler: "q1full" (every date, no pruning: every tile needs all four
    columns), "q1full_matches" (the same with the LZ4 columns encoded with
    4-byte matches), "q1pruned" (the headline month) or "q3" (the star join
    with dense join tables); three untimed launches, then three timed ones."""
    import torch

    from golap_public_b200 import api, datagen, queries

    dd = datagen.date_dim()
    if kind == "q3":
        g = datagen.fact_q3(rows, True)
        fact = queries.encode_fact({k: g[k] for k in Q3_COLS}, {"date_key": "cascaded"}, ROWS_PER_CHUNK,
                                   ROWS_PER_BLOCK, segments)
        q = queries.Q3Query(fact, datagen.dim_geo(3_000_000, datagen.SEED, 21),
                            datagen.dim_geo(200_000, datagen.SEED, 22), dd, 2, 1992, 1997, ht_layout="dense")
    else:
        f = datagen.fact_q1(rows, True)
        fact = queries.encode_fact(f, {"date_key": "cascaded"}, ROWS_PER_CHUNK, ROWS_PER_BLOCK, segments,
                                   **({"lz4_min_match": 4} if kind == "q1full_matches" else {}))
        if kind in ("q1full", "q1full_matches"):
            ok = np.ones(len(dd["d_key"]), dtype=bool)
            q = queries.Q1Query(fact, dd, ok, int(dd["d_key"].min()), int(dd["d_key"].max()), *DISC, *QTY,
                                prune=False)
        else:
            q = queries.Q1Query(fact, dd, dd["d_yearmonthnum"] == 199401, DATE_LO, DATE_HI, *DISC, *QTY)
    stream = torch.cuda.current_stream()
    for i in range(6):
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(stream)
        q.launch()
        b.record(stream)
        b.synchronize()
        api.scan_check()
        if i >= 3:
            print(json.dumps({"profile_scan": kind, "rows": rows, "launch": i, "ms": a.elapsed_time(b)}))


def ingest(rows, segments, steps):
    """Column ingest of the Q1 workload's four columns: the GPU encoder from HBM
    (gx_column_encode_device: zone maps, plan pass, host layout, write pass and
    the device metadata, wall time of the call) and, apart, the first read of its
    host payload copy, against the host encoder (gx_column_encode, all host
    threads) with the same options; one JSON line per column.  GB/s are of the
    uncompressed int32 input."""
    import ctypes as C

    import torch

    from golap_public_b200 import _lib as L
    from golap_public_b200 import api, datagen

    f = datagen.fact_q1(rows, True)
    codecs = {"date_key": "cascaded"}
    for name, v in f.items():
        codec = codecs.get(name, "lz4")
        dev = torch.from_numpy(v).cuda()
        times, copy_times = [], []
        for i in range(max(3, steps) + 1):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            col = api.Column.from_device(dev, codec, ROWS_PER_CHUNK, ROWS_PER_BLOCK, segments)
            t1 = time.perf_counter()
            col.payload_view()
            t2 = time.perf_counter()
            times.append(t1 - t0)
            copy_times.append(t2 - t1)
            comp = col.info.comp_bytes
            col.free()
        t_dev = float(np.median(times[1:]))
        t_copy = float(np.median(copy_times[1:]))
        o = api.Column._opts(codec, ROWS_PER_CHUNK, ROWS_PER_BLOCK, segments, L.GX_LZ4_LITERAL, 16, 0)
        h = C.c_void_p()
        t0 = time.perf_counter()
        L.check(L.lib().gx_column_encode(v.ctypes.data_as(C.c_void_p), len(v), C.byref(o), C.byref(h)))
        t_host = time.perf_counter() - t0
        L.lib().gx_column_free(h)
        print(json.dumps({"ingest": name, "codec": codec, "rows": rows, "comp_bytes": comp,
                          "device_ms": round(t_dev * 1e3, 3), "device_gbs": round(4 * rows / t_dev / 1e9, 1),
                          "host_copy_read_ms": round(t_copy * 1e3, 3),
                          "host_ms": round(t_host * 1e3, 1), "host_gbs": round(4 * rows / t_host / 1e9, 2),
                          "host_threads": os.cpu_count()}))


def main():
    global N_ROWS
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="gx", choices=["gx", "reference"])
    ap.add_argument("--segments", type=int, default=128)
    ap.add_argument("--seed", type=int, default=0xBEE5BEE5)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-batch", action="store_true", help="skip the batched and serving sections")
    ap.add_argument("--no-star", action="store_true", help="skip the 600M-row star join section")
    ap.add_argument("--batch-rows", type=int, default=100_000_000)
    ap.add_argument("--star-rows", type=int, default=600_000_000)
    ap.add_argument("--star-layout", default="dense", choices=["linear", "bucket", "dense"])
    ap.add_argument("--latency-s", type=float, default=1.0, help="seconds of replays behind p50/p99")
    ap.add_argument("--no-tune", action="store_true", help="batched/serving with the default launch shape")
    ap.add_argument("--rows", type=int, default=N_ROWS,
                    help="fact rows of the Q1 workload (default: the measured 60M-row configuration; smaller "
                         "values are for profiler captures)")
    ap.add_argument("--tune-rows", type=int, default=20_000_000)
    ap.add_argument("--profile-scan", choices=["q1full", "q1full_matches", "q1pruned", "q3"],
                    help="run one single-plan scan six times on --rows rows (for a profiler) and exit")
    ap.add_argument("--profile-batch", action="store_true",
                    help="only build the batch table and run the 256-query mixed batch (shared form, dense join "
                         "tables, automatic launch shape) three times: the command profiler captures use")
    ap.add_argument("--ingest", action="store_true",
                    help="time the GPU column encoder against the host encoder on --rows rows and exit")
    args = ap.parse_args()
    args.warmup = max(3, args.warmup)
    N_ROWS = args.rows
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))

    if args.profile_scan:
        profile_scan(args.profile_scan, args.rows, args.segments)
        return
    if args.profile_batch:
        profile_batch(args.batch_rows)
        return
    if args.ingest:
        ingest(args.rows, args.segments, args.steps)
        return

    if args.impl == "reference":
        if rank != 0:
            return
        from golap_public_b200 import queries

        f, dd = make_data(args.seed)
        fact = queries.encode_fact(f, {"date_key": "cascaded"}, ROWS_PER_CHUNK, ROWS_PER_BLOCK, args.segments,
                                   residency=None)
        cb = cpu_baseline(fact, dd, steps=args.steps, warmup=args.warmup)
        line = {
            "impl": "reference",
            "metric": "rows/s & GB/s vs HBM roofline; p50/p99 latency batched vs one-query-at-a-time",
            "value": cb["value"], "unit": "rows/s", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": cb["ms"], "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "int32", "data": "synthetic (seeded, configs[1] shapes and distributions)",
            "config": {"workload": WORKLOAD, "rows": N_ROWS, "chunks": N_ROWS // ROWS_PER_CHUNK,
                       "lz4_segments": args.segments},
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
    line, ctx = gpu_arm(args, rank, world)
    pk, pk_kind = peaks()
    if rank == 0 and not args.no_cpu:
        cb = cpu_baseline(ctx["fact"], ctx["dd"], steps=3, warmup=1)
        line["cpu_baseline"] = {k: cb[k] for k in ("value", "unit", "cores", "kind", "sample", "ms")}
        line["cpu_baseline"]["surviving_rows_per_s"] = cb["surviving_rows_per_s"]
        if cb["result"] != line["result"]:
            raise SystemExit(f"cpu baseline result {cb['result']} != gpu {line['result']}")
        line["full_scan"]["cpu_reference"] = cpu_full_scan(ctx["fact"], ctx["dd"], ctx["want_all"])
    del ctx
    if not args.no_star:
        star, sctx = star_join_section(args, pk, pk_kind, world)
        if rank == 0 and not args.no_cpu:
            star["cpu_baseline"] = cpu_star_join(sctx)
            if not star["cpu_baseline"]["groups_equal_gpu"]:
                raise SystemExit("star join: reference CPU groups differ from the GPU groups")
        line["star_join"] = star
        del sctx
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
    if world > 1:
        import torch.distributed as dist

        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line))


if __name__ == "__main__":
    main()
