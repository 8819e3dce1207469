"""Host-side mirror of the reference operator API for the hot path.

Names follow the GOLAP classes they stand in for:
  Column            CompInfo/BlockInfo + the compressed chunk store
                    (core/comp.cuh:23-78) with its MinMaxMeta
                    (core/metadata.cuh:110-221) collected at ingest
  ChunkDecompressor ChunkDecompressor::step (core/comp.cuh:151-227)
  MetaChecker       MetaChecker::add_minmax (core/metadata.cuh:638-658)
  HashMap           HashMap + hash_map_build_pred_other
                    (core/dev_structs.cuh:37-132, core/join.cuh:107-135)
  HashAggregate     HashAggregate with SumAgg (core/dev_structs.cuh:158-253)
  ScanPlan          the fused per-chunk pipelines pipeline_q1_lineorder /
                    pipeline_q3 (usecases/ssb/queries/01.cuh:27, 03.cuh:119)

Device buffers are torch CUDA tensors (plumbing only); all compute runs in
libgx.so.  Errors raise GxError carrying the library's status and message.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from . import _lib as L
from ._lib import check


def _stream_handle(stream=None):
    import torch

    if stream is None:
        stream = torch.cuda.current_stream()
    return C.c_void_p(stream.cuda_stream)


def _dptr(t):
    return C.c_void_p(t.data_ptr()) if t is not None else None


CODECS = {"none": L.GX_CODEC_NONE, "lz4": L.GX_CODEC_LZ4, "cascaded": L.GX_CODEC_CASCADED}


class Column:
    """One compressed int32 column: chunks of rows_per_chunk rows, blocks of rows_per_block rows."""

    def __init__(self, values: np.ndarray, codec: str = "lz4", rows_per_chunk: int = 1_000_000,
                 rows_per_block: int = 16384, lz4_segments: int = 128, lz4_min_match: int = 0,
                 lz4_search_depth: int = 16, threads: int = 0, name: str = ""):
        values = np.ascontiguousarray(values, dtype=np.int32)
        o = self._opts(codec, rows_per_chunk, rows_per_block, lz4_segments, lz4_min_match, lz4_search_depth, threads)
        h = C.c_void_p()
        check(L.lib().gx_column_encode(values.ctypes.data_as(C.c_void_p), len(values), C.byref(o), C.byref(h)))
        self.handle = h
        self.name = name
        self.codec = codec

    @staticmethod
    def _opts(codec, rows_per_chunk, rows_per_block, lz4_segments, lz4_min_match, lz4_search_depth, threads):
        o = L.EncodeOpts()
        check(L.lib().gx_encode_opts_default(C.byref(o)))
        o.codec = CODECS[codec]
        o.rows_per_chunk = rows_per_chunk
        o.rows_per_block = rows_per_block
        o.lz4_segments = lz4_segments
        o.lz4_min_match = lz4_min_match
        o.lz4_search_depth = lz4_search_depth
        o.threads = threads
        return o

    @classmethod
    def from_device(cls, values, codec: str = "lz4", rows_per_chunk: int = 1_000_000, rows_per_block: int = 16384,
                    lz4_segments: int = 128, name: str = "", stream=None) -> "Column":
        """Encodes an int32 CUDA tensor on the GPU (gx_column_encode_device): the column is in HBM on
        return, byte-identical to Column(values.cpu().numpy(), ...) with the same options.  LZ4 blocks
        are literal runs (lz4_min_match = GX_LZ4_LITERAL)."""
        import torch

        if not (isinstance(values, torch.Tensor) and values.is_cuda and values.dtype == torch.int32):
            raise TypeError("Column.from_device needs an int32 CUDA tensor")
        values = values.contiguous()
        o = cls._opts(codec, rows_per_chunk, rows_per_block, lz4_segments, L.GX_LZ4_LITERAL, 0, 0)
        h = C.c_void_p()
        check(L.lib().gx_column_encode_device(_dptr(values), values.numel(), C.byref(o), C.byref(h),
                                              _stream_handle(stream)))
        self = cls.__new__(cls)
        self.handle = h
        self.name = name
        self.codec = codec
        return self

    # --- inspection
    @property
    def info(self) -> L.ColumnInfo:
        i = L.ColumnInfo()
        check(L.lib().gx_column_info_get(self.handle, C.byref(i)))
        return i

    def minmax(self):
        n = self.info.n_chunks
        mins = np.zeros(n, np.int32)
        maxs = np.zeros(n, np.int32)
        check(L.lib().gx_column_chunk_minmax(self.handle, mins.ctypes.data_as(C.c_void_p),
                                             maxs.ctypes.data_as(C.c_void_p)))
        return mins, maxs

    def block_minmax(self):
        """Per-block-slot zone maps (n_chunks * blocks_per_chunk entries each)."""
        i = self.info
        n = i.n_chunks * i.blocks_per_chunk
        mins = np.zeros(n, np.int32)
        maxs = np.zeros(n, np.int32)
        check(L.lib().gx_column_block_minmax(self.handle, mins.ctypes.data_as(C.c_void_p),
                                             maxs.ctypes.data_as(C.c_void_p)))
        return mins, maxs

    def blocks(self) -> np.ndarray:
        n = self.info.n_blocks
        arr = (L.BlockInfo * max(n, 1))()
        check(L.lib().gx_column_blocks(self.handle, arr))
        return np.array([(b.offset, b.size, b.payload, b.tuples) for b in arr[:n]], dtype=np.uint64).reshape(-1, 4)

    def payload(self) -> np.ndarray:
        return self.payload_view().copy()

    def payload_view(self) -> np.ndarray:
        """The host copy of the compressed payload without copying (valid while the column lives)."""
        p = L.u8p()
        n = C.c_uint64()
        check(L.lib().gx_column_payload(self.handle, C.byref(p), C.byref(n)))
        return np.ctypeslib.as_array(p, shape=(n.value,))

    def seg_index(self) -> np.ndarray:
        p = C.POINTER(C.c_uint32)()
        n = C.c_uint64()
        check(L.lib().gx_column_seg_index(self.handle, C.byref(p), C.byref(n)))
        if n.value == 0:
            return np.zeros(0, np.uint32)
        return np.ctypeslib.as_array(p, shape=(n.value,)).copy()

    # --- richer pruning metadata (built on the device)
    def build_hist(self, n_buckets: int, stream=None) -> "Column":
        """Equal-width histograms of n_buckets per chunk (EqHistogram)."""
        check(L.lib().gx_column_build_hist(self.handle, n_buckets, _stream_handle(stream)))
        return self

    def build_bloom(self, m_bytes: int, p: float, stream=None) -> "Column":
        """A Bloom filter of m_bytes per chunk for false-positive rate p (BloomMeta)."""
        check(L.lib().gx_column_build_bloom(self.handle, m_bytes, p, _stream_handle(stream)))
        return self

    def meta(self, stream=None):
        """(histogram counts (n_chunks, n_buckets) or None, Bloom words (n_chunks, m/4) or None, k)."""
        nb, mb, k = C.c_uint32(), C.c_uint64(), C.c_uint32()
        check(L.lib().gx_column_meta_read(self.handle, None, None, C.byref(nb), C.byref(mb), C.byref(k),
                                          _stream_handle(stream)))
        nc = self.info.n_chunks
        h = np.zeros((nc, nb.value), np.uint64) if nb.value else None
        w = np.zeros((nc, mb.value // 4), np.uint32) if mb.value else None
        check(L.lib().gx_column_meta_read(self.handle, h.ctypes.data_as(C.c_void_p) if h is not None else None,
                                          w.ctypes.data_as(C.c_void_p) if w is not None else None, None, None, None,
                                          _stream_handle(stream)))
        return h, w, k.value

    # --- device residency
    def to_device(self, residency: str = "hbm", stream=None) -> "Column":
        check(L.lib().gx_column_to_device(self.handle, 1 if residency == "hbm" else 2, _stream_handle(stream)))
        return self

    def release_device(self):
        check(L.lib().gx_column_release_device(self.handle))

    def free(self):
        if self.handle:
            L.lib().gx_column_free(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


class ChunkDecompressor:
    """Decompresses chunks of a device-resident Column into a device buffer."""

    def __init__(self, col: Column):
        self.col = col

    def step(self, chunk_idx: int, out, stream=None):
        check(L.lib().gx_decompress_chunk(self.col.handle, chunk_idx, _dptr(out), _stream_handle(stream)))

    def chunks(self, first: int, n: int, out, stream=None):
        check(L.lib().gx_decompress_chunks(self.col.handle, first, n, _dptr(out), _stream_handle(stream)))


class MetaChecker:
    """Combines min/max predicates into per-chunk keep flags (uint16, 1 = keep)."""

    def __init__(self, n_chunks: int):
        self.preds: list[tuple[Column, int, int]] = []
        self.n_chunks = n_chunks

    def add_minmax(self, col: Column, lo: int, hi: int) -> "MetaChecker":
        self.preds.append((col, lo, hi))
        return self

    def add_points(self, col: Column, keys, count, keep_out, stream=None):
        """Join pruning (check_mmmeta_multiple_pts, core/metadata.cuh:550-560): sets
        keep_out[c] = 1 where one of the keys (device tensors from HashMap.keys)
        lies in chunk c's min/max of `col`; AND the result with other flags."""
        check(L.lib().gx_check_minmax_points(col.handle, _dptr(keys), _dptr(count), keys.numel(), _dptr(keep_out),
                                             _stream_handle(stream)))
        return keep_out

    def add_hist(self, col: Column, lo: int, hi: int, keep_out, stream=None):
        """check_hist (core/metadata.cuh:584-595): sets keep_out[c] = 1 where a
        non-empty bucket of chunk c overlaps [lo, hi] (col.build_hist first)."""
        check(L.lib().gx_check_hist(col.handle, lo, hi, _dptr(keep_out), _stream_handle(stream)))
        return keep_out

    def add_bloom(self, col: Column, value: int, keep_out, stream=None):
        """check_bloom (core/metadata.cuh:612-620): sets keep_out[c] = 1 where
        value may be in chunk c (col.build_bloom first)."""
        check(L.lib().gx_check_bloom(col.handle, value, _dptr(keep_out), _stream_handle(stream)))
        return keep_out

    def run(self, keep_out, stream=None):
        n = len(self.preds)
        cols = (C.c_void_p * n)(*[c.handle.value for c, _, _ in self.preds])
        lo = (C.c_int32 * n)(*[p[1] for p in self.preds])
        hi = (C.c_int32 * n)(*[p[2] for p in self.preds])
        check(L.lib().gx_prune_minmax(cols, lo, hi, n, _dptr(keep_out), _stream_handle(stream)))
        return keep_out


class HashMap:
    """Join table on the device: key -> payload (row id when no payload).
    layout: "linear" or "bucket" (open addressing), or "dense" (one slot per
    key of the build keys' range; for keys that fill most of their range)."""

    def __init__(self, max_entries: int, layout: str = "linear"):
        h = C.c_void_p()
        lay = {"linear": L.GX_HT_LINEAR, "bucket": L.GX_HT_BUCKET, "dense": L.GX_HT_DENSE}[layout]
        check(L.lib().gx_hashtable_create2(max_entries, lay, C.byref(h)))
        self.handle = h
        self.layout = layout

    def build(self, keys, payload=None, preds=(), stream=None) -> "HashMap":
        n = keys.numel()
        arr = (L.Pred * max(1, len(preds)))()
        for i, (col, lo, hi) in enumerate(preds):
            arr[i].col_dev = col.data_ptr()
            arr[i].lo = lo
            arr[i].hi = hi
        check(L.lib().gx_hashtable_build(self.handle, _dptr(keys), _dptr(payload), n, arr, len(preds),
                                         _stream_handle(stream)))
        return self

    def clear(self, stream=None) -> "HashMap":
        """Empty the table (before GX_AGG_BUILD scans fill it)."""
        check(L.lib().gx_hashtable_clear(self.handle, _stream_handle(stream)))
        return self

    def count(self, stream=None) -> int:
        n = C.c_uint64()
        check(L.lib().gx_hashtable_count(self.handle, C.byref(n), _stream_handle(stream)))
        return n.value

    def probe(self, keys, payload_out=None, hits=None, stream=None):
        check(L.lib().gx_hashtable_probe(self.handle, _dptr(keys), keys.numel(), _dptr(payload_out), _dptr(hits),
                                         _stream_handle(stream)))

    def keys(self, out, count, stream=None):
        """Keys of the table's entries into the int32 device tensor `out` (any order),
        their number into the int64 device tensor `count` (collect_hashmap_keys,
        core/dev_structs.cuh:136-150); no host synchronisation."""
        check(L.lib().gx_hashtable_keys(self.handle, _dptr(out), out.numel(), _dptr(count), _stream_handle(stream)))
        return out, count

    def free(self):
        if self.handle:
            L.lib().gx_hashtable_free(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


class HashAggregate:
    """Device group table: int64 key -> int64 sum."""

    def __init__(self, max_groups: int):
        h = C.c_void_p()
        check(L.lib().gx_groupby_create(max_groups, C.byref(h)))
        self.handle = h
        self.max_groups = max_groups

    def reset(self, stream=None):
        check(L.lib().gx_groupby_reset(self.handle, _stream_handle(stream)))

    def add(self, keys, vals, stream=None):
        check(L.lib().gx_groupby_add(self.handle, _dptr(keys), _dptr(vals), keys.numel(), _stream_handle(stream)))

    def read(self, cap: int | None = None, stream=None) -> dict:
        cap = cap or self.max_groups
        k = np.zeros(cap, np.int64)
        s = np.zeros(cap, np.int64)
        n = C.c_uint64()
        check(L.lib().gx_groupby_read(self.handle, k.ctypes.data_as(C.c_void_p), s.ctypes.data_as(C.c_void_p), cap,
                                      C.byref(n), _stream_handle(stream)))
        return dict(zip(k[: n.value].tolist(), s[: n.value].tolist()))

    def free(self):
        if self.handle:
            L.lib().gx_groupby_free(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


@dataclass
class Step:
    col: Column
    flags: int
    lo: int = 0
    hi: int = 0
    ht: HashMap | None = None
    digit_base: int = 0
    digit_card: int = 0


@dataclass
class ScanPlan:
    """Ordered column steps of one fused scan (see gx_scan_plan in include/gx.h)."""

    steps: list = field(default_factory=list)
    agg: int = L.GX_AGG_SUM
    keep_chunks: object = None      # device uint16 tensor or None
    groupby: HashAggregate | None = None
    result: object = None           # device int64 tensor (1 element)
    prune: list = field(default_factory=list)  # (Column, lo, hi) min/max predicates
    keep_out: object = None         # device uint16 tensor receiving the chunk flags
    build_ht: "HashMap | None" = None  # GX_AGG_BUILD: the join table the surviving rows go into

    def prune_minmax(self, col, lo, hi):
        self.prune.append((col, lo, hi))
        return self

    def filter(self, col, lo, hi, carry=False):
        self.steps.append(Step(col, L.GX_STEP_FILTER | (L.GX_STEP_CARRY if carry else 0), lo, hi))
        return self

    def probe(self, col, ht, digit_base=0, digit_card=0):
        self.steps.append(Step(col, L.GX_STEP_PROBE, ht=ht, digit_base=digit_base, digit_card=digit_card))
        return self

    def group(self, col, digit_base, digit_card):
        """GROUP BY the column's value (one digit of the group key)."""
        self.steps.append(Step(col, L.GX_STEP_GROUP, digit_base=digit_base, digit_card=digit_card))
        return self

    def carry(self, col):
        self.steps.append(Step(col, L.GX_STEP_CARRY))
        return self

    def value(self, col, lo=None, hi=None):
        flags = L.GX_STEP_VALUE
        if lo is not None:
            flags |= L.GX_STEP_FILTER
        self.steps.append(Step(col, flags, lo or 0, hi or 0))
        return self

    def to_c(self) -> L.ScanPlan:
        p = L.ScanPlan()
        p.n_steps = len(self.steps)
        for i, s in enumerate(self.steps):
            d = p.steps[i]
            d.col = s.col.handle.value
            d.flags = s.flags
            d.lo = s.lo
            d.hi = s.hi
            d.ht = s.ht.handle.value if s.ht is not None else None
            d.digit_base = s.digit_base
            d.digit_card = s.digit_card
        p.agg = self.agg
        p.keep_chunks_dev = self.keep_chunks.data_ptr() if self.keep_chunks is not None else None
        p.groupby = self.groupby.handle.value if self.groupby is not None else None
        p.result_dev = self.result.data_ptr() if self.result is not None else None
        p.n_prune = len(self.prune)
        for i, (col, lo, hi) in enumerate(self.prune):
            p.prune[i].col = col.handle.value
            p.prune[i].lo = lo
            p.prune[i].hi = hi
        p.keep_out_dev = self.keep_out.data_ptr() if self.keep_out is not None else None
        p.build_ht = self.build_ht.handle.value if self.build_ht is not None else None
        self._c = p  # keep alive
        return p

    def launch(self, stream=None):
        check(L.lib().gx_scan(C.byref(self.to_c()), _stream_handle(stream)))

    def launch_streamed(self, chunks_per_group: int = 16, stream=None):
        """Scan pinned-host columns through double-buffered HBM staging:
        only the chunks that survive the min/max predicates are copied."""
        check(L.lib().gx_scan_streamed(C.byref(self.to_c()), chunks_per_group, _stream_handle(stream)))

    def run_sync(self, stream=None) -> int:
        rows = C.c_uint64()
        check(L.lib().gx_scan_sync(C.byref(self.to_c()), _stream_handle(stream), C.byref(rows)))
        return rows.value


SCAN_FORMS = {"auto": L.GX_FORM_AUTO, "warp": L.GX_FORM_WARP, "pipe": L.GX_FORM_PIPE, "shared": L.GX_FORM_SHARED,
              "queue": L.GX_FORM_QUEUE}


def set_scan_form(form: str = "auto"):
    """Kernel form of single-plan scans (process-wide): "auto" or one forced
    form ("warp", "pipe", "shared", "queue"); a forced form that cannot run a
    plan makes the launch fail instead of falling back."""
    check(L.lib().gx_scan_set_form(SCAN_FORMS[form]))


def scan_check(stream=None):
    check(L.lib().gx_scan_check(_stream_handle(stream)))


class Batch:
    """Many scan plans over one table, each on a row slice, in one persistent launch."""

    MODES = {"auto": L.GX_BATCH_AUTO, "queue": L.GX_BATCH_QUEUE, "shared": L.GX_BATCH_SHARED}

    def __init__(self, queries, mode: str = "auto"):
        """queries: iterable of (ScanPlan, row_lo, row_hi).  mode: "auto",
        "queue" (per-query work items) or "shared" (each tile decoded once for
        all queries that need it)."""
        queries = list(queries)
        arr = (L.Query * len(queries))()
        for i, (plan, lo, hi) in enumerate(queries):
            arr[i].plan = plan.to_c()
            arr[i].row_lo = lo
            arr[i].row_hi = hi
        self.plans = [q[0] for q in queries]
        h = C.c_void_p()
        check(L.lib().gx_batch_create2(arr, len(queries), self.MODES[mode], C.byref(h)))
        self.handle = h

    def set_launch(self, threads: int = 0, ctas_per_sm: int = 0) -> "Batch":
        """threads 0 = automatic (of 256, 512 and 128 threads, the most resident warps
        for the batch's shared memory)."""
        check(L.lib().gx_batch_set_launch(self.handle, threads, ctas_per_sm))
        return self

    @property
    def threads(self) -> int:
        t = C.c_uint32()
        check(L.lib().gx_batch_launch_get(self.handle, C.byref(t)))
        return t.value

    @property
    def mode(self) -> str:
        m = C.c_uint32()
        check(L.lib().gx_batch_mode(self.handle, C.byref(m)))
        return {L.GX_BATCH_QUEUE: "queue", L.GX_BATCH_SHARED: "shared"}[m.value]

    def run(self, stream=None):
        check(L.lib().gx_batch_run(self.handle, _stream_handle(stream)))

    def graph(self, stream=None):
        check(L.lib().gx_batch_graph(self.handle, _stream_handle(stream)))

    def rows(self, stream=None) -> int:
        n = C.c_uint64()
        check(L.lib().gx_batch_rows(self.handle, C.byref(n), _stream_handle(stream)))
        return n.value

    def free(self):
        if self.handle:
            L.lib().gx_batch_free(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


class Server:
    """Continuous-batching serving loop (gx_server_* in include/gx.h)."""

    def __init__(self, max_inflight: int = 4, max_batch: int = 128, hbm_budget: int = 120 << 30,
                 batch_threads: int = 0, batch_mode: str = "auto"):
        o = L.ServerOpts()
        check(L.lib().gx_server_opts_default(C.byref(o)))
        o.max_inflight, o.max_batch, o.hbm_budget = max_inflight, max_batch, hbm_budget
        o.batch_threads, o.batch_mode = batch_threads, Batch.MODES[batch_mode]
        h = C.c_void_p()
        check(L.lib().gx_server_create(C.byref(o), C.byref(h)))
        self.handle = h
        self._keep = {}

    def submit(self, plan: "ScanPlan", row_lo: int, row_hi: int, hbm_bytes: int) -> int:
        q = L.Query()
        q.plan = plan.to_c()
        q.row_lo, q.row_hi = row_lo, row_hi
        t = C.c_uint64()
        check(L.lib().gx_server_submit(self.handle, C.byref(q), hbm_bytes, C.byref(t)))
        self._keep[t.value] = plan
        return t.value

    def wait(self, ticket: int, timeout_s: float = 60.0) -> float:
        """Blocks until the request is done; returns its latency in ms."""
        lat = C.c_double()
        try:
            check(L.lib().gx_server_wait(self.handle, ticket, timeout_s, C.byref(lat)))
        finally:
            self._keep.pop(ticket, None)
        return lat.value

    def stats(self) -> dict:
        st = L.ServerStats()
        check(L.lib().gx_server_stats_get(self.handle, C.byref(st)))
        return {n: getattr(st, n) for n, _ in L.ServerStats._fields_}

    def close(self):
        if self.handle:
            L.lib().gx_server_free(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
