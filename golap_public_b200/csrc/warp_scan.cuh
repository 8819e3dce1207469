// warp_scan.cuh -- the one-query fused scan with one warp per row tile
// (device side; included by kernels.cu inside its anonymous namespace after
// pipe_scan.cuh, whose descriptors and helpers it shares).
//
// Replaces, for one query: ChunkDecompressor::step (core/comp.cuh:171-195)
// feeding pipeline_q1_lineorder (usecases/ssb/queries/01.cuh:27-54),
// pipeline_q2 (02.cuh:103), pipeline_q3 (03.cuh:119-170) or pipeline_q4
// (04.cuh:100), with the chunk pruning of MetaChecker
// (core/metadata.cuh:638-658) and the per-chunk worker loop of
// usecases/ssb/queries/01.hpp:350-424 folded into the same launch.
//
// Every warp is an independent worker: after one block-wide barrier at the
// start (chunk keep bits of the launch and their prefix counts, computed by
// each CTA) no warp waits for another.  The 1024-row tiles of the surviving
// chunks form a dense rank space; warp w of the grid takes tiles w, w + W,
// w + 2W, ... (W warps), four at a time:
//   * one decision round per four tiles: lane 8q + c reads column c's
//     directory entry and side-index entries for tile q (a cascaded page's
//     header and up to 8 runs too) and picks how the column is read --
//     staged (raw rows or a 16-byte aligned LZ4 literal run: one bulk copy
//     of the tile's rows into the warp's stage area), constant (a cascaded
//     page or run that holds one value on the tile), or decoded by the warp
//     into its buffer (LZ4 ranges with matches: groups of lanes per
//     segment; other cascaded pages: run windows of 32 runs, one per lane);
//     the round's staged ranges are bulk-prefetched into L2 and the next
//     round's directory lines prefetched;
//   * per tile: the bulk copies on the warp's mbarrier, the decodes, then the
//     plan's steps over row groups of 128 rows (4 consecutive rows per lane,
//     one 16-byte shared load per column).  Plans of the SSB shapes run a
//     compile-time evaluator selected by their signature (all values of a
//     row group in registers, steps over a constant column decided once per
//     tile); other plans a run-time step-major evaluator.
// Scalar sums stay in registers; grouped sums go to the CTA's group table in
// shared memory (keys that find no slot go to the global table), flushed when
// the CTA is done.  Join-table reads carry an L2 evict-last policy and the
// streamed column bytes an evict-first one, so that the tables stay in L2
// while the fact columns pass through it.

constexpr uint32_t kWsLog2 = 10;
constexpr uint32_t kWsTile = 1u << kWsLog2;    // rows of one warp tile
constexpr uint32_t kWsNT = 128;                // threads per CTA (4 independent warps)
constexpr uint32_t kWsWarps = kWsNT / 32;
constexpr uint32_t kWsBatch = 128;             // rows of one row group (4 per lane)
constexpr uint32_t kWsGroups = kWsTile / kWsBatch;  // row groups of a tile (4 keep bits each)
constexpr uint32_t kWsEvalGroups = 2;               // row groups a scalar compile-time evaluator runs at once
static_assert(kWsGroups % kWsEvalGroups == 0, "the evaluator's row-group batches cover the tile");
static_assert(kWsGroups * 4 <= 32, "the keep bits of a tile fit one word");
constexpr uint32_t kWsMaxCols = kPipeMaxCols;
constexpr uint32_t kWsGroupLog2 = 9;           // the CTA's group table: 512 slots
constexpr uint32_t kWsGroupSlots = 1u << kWsGroupLog2;
constexpr uint32_t kWsGroupProbes = 16;
constexpr uint32_t kWsNone = 0xFFFFFFFFu;
constexpr uint32_t kWsMaxDynSmem = 220u << 10;  // dynamic shared memory of one CTA at most
constexpr uint32_t kWsMaxChunkWords = 1024;     // chunk keep bits of one launch: 32768 chunks
// per-warp words before the stage: 8 constant slots (32 words), the mbarrier
// (2 + 2 padding), the dense join tables' {base, span} headers per step (16)
constexpr uint32_t kWsHead = 52;
static_assert(4 * kWsMaxCols + 4 + 2 * GX_MAX_STEPS <= kWsHead && kWsHead % 4 == 0, "the warp head holds its parts");
static_assert(kWsTile <= kCascPageRows && kCascPageRows % kWsTile == 0, "a warp tile lies in one cascaded page");

struct WsParams {
    ShQuery q;                      // steps index into cols
    gx_dcol cols[kWsMaxCols];
    uint32_t n_cols;
    uint32_t blocks_per_chunk, rows_per_chunk, rows_per_block, tiles_per_block;
    uint64_t n_rows;                // rows of the table
    uint32_t chunk_lo, chunk_hi;    // chunks [chunk_lo, chunk_hi) are scanned
    uint32_t stage_of[kWsMaxCols];  // stage area column c is copied into (raw / aligned-literal LZ4), or kWsNone
    uint32_t buf_of[kWsMaxCols];    // decode buffer of column c (cascaded / LZ4 with matches), or kWsNone
    uint32_t n_areas;               // stage areas + decode buffers per warp (kWsTile words each)
    uint32_t warp_words;            // shared memory words per warp
    uint32_t chunk_words;           // words of the chunk keep bitmap (and of its prefix counts)
    uint32_t grouped_tab;           // 1: the warp has a group table
    unsigned long long* rows_scanned;
};

// Column read modes of one tile.
// kWmRuns2: a cascaded tile covered by two runs (value cval on tile rows
// [0, aux0), value aux1 from there), written out without the page decoder.
enum : uint32_t { kWmStage = 0, kWmConst = 1, kWmLz4 = 2, kWmCasc = 3, kWmBad = 4, kWmRuns2 = 5 };

__device__ __forceinline__ uint64_t ws_shfl64(uint64_t v, uint32_t src) {
    return ((uint64_t)__shfl_sync(0xFFFFFFFFu, (uint32_t)(v >> 32), src) << 32) |
           __shfl_sync(0xFFFFFFFFu, (uint32_t)v, src);
}

// Inclusive warp scan (wrapping uint32 sum).
__device__ __forceinline__ uint32_t ws_scan(uint32_t x, uint32_t lane) {
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, x, d);
        if (lane >= (uint32_t)d) x += y;
    }
    return x;
}

// One bulk copy (no multicast) completing on m, its lines read under policy pol.
__device__ __forceinline__ void ws_bulk_copy(void* dst, const void* src, uint32_t bytes, uint64_t* m, uint64_t pol) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes.L2::cache_hint [%0], [%1], %2, [%3], %4;" ::
            "r"(smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(smem_u32(m)), "l"(pol)
        : "memory");
}

// Rows [h0, h0 + n) of a cascaded page decoded by one warp into out[0..n),
// or, when one run covers them, *cv = that value and 1 is returned (out is
// not written).  RLE pages are walked in windows of 32 runs (run j of the
// window in lane j: its value, start and end from warp scans that carry over
// from the previous windows); the rows of a window are written 32 at a time
// by the runs overlapping them.  Pages without RLE unpack their values
// directly; with DELTA the prefix up to row h0 is a warp reduction and the
// tile's rows a running warp scan.  Returns 0, 1 (constant) or kErrCorrupt
// (uniform over the warp).
__device__ __noinline__ int ws_casc_rows(const uint8_t* __restrict__ pg, uint32_t pg_bytes, uint32_t page_rows,
                                         uint32_t h0, uint32_t n, int32_t* out, int32_t* cv, uint32_t lane) {
    const casc_hdr h = casc_load_header(pg);
    if (!casc_header_ok(h, pg_bytes, page_rows) || h0 + n > page_rows) return kErrCorrupt;
    const bool rle = (h.flags & CASC_RLE) != 0, delta = (h.flags & CASC_DELTA) != 0;
    const uint32_t* vw = (const uint32_t*)(pg + h.vals_off);
    const uint32_t vb = h.val_bits, base = (uint32_t)h.val_base;
    if (!rle) {
        if (!delta) {
            for (uint32_t i = lane; i < n; i += 32) out[i] = (int32_t)(unpack_bits(vw, h0 + i, vb) + base);
            __syncwarp();
            return 0;
        }
        uint32_t pre = 0;  // entries 1 .. h0-1 (entry 0 is 0)
        for (uint32_t k = 1 + lane; k < h0; k += 32) pre += unpack_bits(vw, k, vb) + base;
        pre = __reduce_add_sync(0xFFFFFFFFu, pre);
        uint32_t run = (uint32_t)h.first + pre;
        for (uint32_t g = 0; g < n; g += 32) {
            const uint32_t i = h0 + g + lane;
            const uint32_t e = (i == 0 || g + lane >= n) ? 0u : unpack_bits(vw, i, vb) + base;
            const uint32_t x = ws_scan(e, lane);
            if (g + lane < n) out[g + lane] = (int32_t)(run + x);
            run += __shfl_sync(0xFFFFFFFFu, x, 31);
        }
        __syncwarp();
        return 0;
    }
    const uint32_t nr = h.n_runs;
    const uint32_t* lw = (const uint32_t*)(pg + h.lens_off);
    const uint32_t t0 = h0, t1 = h0 + n;
    uint32_t c_end = 0, c_val = 0;  // carried over the windows: rows and value deltas so far
    bool is_const = false;
    for (uint32_t w0 = 0; w0 < nr; w0 += 32) {
        const uint32_t j = w0 + lane;
        const bool in = j < nr;
        const uint32_t le = in ? unpack_bits(lw, j, h.len_bits) + h.len_base : 0u;
        const uint32_t ve = in ? ((delta && j == 0) ? 0u : unpack_bits(vw, j, vb) + base) : 0u;
        const uint32_t end = c_end + ws_scan(le, lane), start = end - le;
        const uint32_t val = delta ? (uint32_t)h.first + c_val + ws_scan(ve, lane) : ve;
        const uint32_t w_end = __shfl_sync(0xFFFFFFFFu, end, 31), w_start = c_end;
        c_end = w_end;
        if (delta) c_val += __reduce_add_sync(0xFFFFFFFFu, ve);
        // (every window is walked: the run lengths must add up to the page)
        if (is_const || w_end <= t0 || w_start >= t1) continue;
        // one run covering the whole tile: its value, nothing written
        const uint32_t cover = __ballot_sync(0xFFFFFFFFu, in && start <= t0 && end >= t1);
        if (cover) {
            *cv = (int32_t)__shfl_sync(0xFFFFFFFFu, val, __ffs(cover) - 1);
            is_const = true;
            continue;
        }
        const uint32_t r_lo = max(w_start, t0), r_hi = min(w_end, t1);
        for (uint32_t g = r_lo & ~31u; g < r_hi; g += 32) {
            const uint32_t r = g + lane;
            // runs of this window that overlap rows [g, g + 32)
            uint32_t m = __ballot_sync(0xFFFFFFFFu, in && le > 0 && start < g + 32 && end > g);
            int32_t v = 0;
            bool got = false;
            while (m) {
                const uint32_t k = __ffs(m) - 1;
                m &= m - 1;
                const uint32_t s = __shfl_sync(0xFFFFFFFFu, start, k), e = __shfl_sync(0xFFFFFFFFu, end, k);
                const uint32_t x = __shfl_sync(0xFFFFFFFFu, val, k);
                if (r >= s && r < e) {
                    v = (int32_t)x;
                    got = true;
                }
            }
            if (got && r >= r_lo && r < r_hi) out[r - t0] = v;
        }
    }
    if (c_end != page_rows) return kErrCorrupt;
    __syncwarp();
    return is_const ? 1 : 0;
}

// The warp's per-segment LZ4 decode of a tile: segments j0 .. j0+nseg-1 of
// the block that starts at address blk (blk_bytes compressed bytes; side
// index entries e) into out (segment t at out + t * seg_rows), G lanes per
// segment.  Returns 0 or kErrCorrupt (uniform).
__device__ __noinline__ int ws_lz4_rows(const uint8_t* blk, uint32_t blk_bytes, const uint32_t* e, uint32_t seg_shift,
                                        uint32_t rows, uint32_t r0, uint32_t n, uint32_t lo, uint32_t hi,
                                        uint32_t* out, uint32_t lane) {
    const uint32_t seg_rows = 1u << seg_shift;
    const uint32_t j0 = r0 >> seg_shift, nseg = (n + seg_rows - 1) >> seg_shift;
    // payload addresses keep the payload offsets' alignment modulo 16
    const uintptr_t a_wb = ((uintptr_t)blk + lo) & ~(uintptr_t)15;
    const uint32_t* A = (const uint32_t*)a_wb;
    const uint32_t wbase = (uint32_t)(a_wb - (uintptr_t)blk);
    const uint32_t glog = seg_group_log2(nseg, 32);
    const uint32_t G = 1u << glog;
    const uint32_t gl = lane & (G - 1u);
    const uint32_t gmask = G >= 32 ? 0xFFFFFFFFu : (((1u << G) - 1u) << (lane & ~(G - 1u)));
    int err = 0;
    for (uint32_t t0 = 0; t0 < nseg; t0 += (32u >> glog)) {
        const uint32_t t = t0 + (lane >> glog);
        if (t < nseg) {
            const uint32_t j = j0 + t;
            const uint32_t K = min(seg_rows, rows - j * seg_rows);
            const uint32_t cp = __ldg(e + 2 * j), info = __ldg(e + 2 * j + 1);
            const int r = lz4_seg_group(A, wbase, lo, hi, blk_bytes, cp, info, K, out + t * seg_rows, gl, G, gmask);
            if (r) err = r;
        }
    }
    __syncwarp();
    return __any_sync(0xFFFFFFFFu, err != 0) ? kErrCorrupt : 0;
}

// Add of (gk, val) to the warp's group table; keys that find no slot within
// kWsGroupProbes go to the global table.
__device__ __forceinline__ void ws_group_add(uint32_t gk, int64_t val, uint32_t* tkey, unsigned long long* tsum,
                                          int64_t* keys, int64_t* sums, uint32_t log2cap) {
    if (gk != kEmptyGKey) {
        uint32_t s = hash_key32((int32_t)gk, kWsGroupLog2);
        for (uint32_t i = 0; i < kWsGroupProbes; ++i) {
            uint32_t cur = ((volatile uint32_t*)tkey)[s];
            if (cur == kEmptyGKey) cur = atomicCAS(&tkey[s], kEmptyGKey, gk);
            if (cur == kEmptyGKey || cur == gk) {
                atomicAdd(&tsum[s], (unsigned long long)val);
                return;
            }
            s = (s + 1) & (kWsGroupSlots - 1);
        }
    }
    if (!group_add_global(keys, sums, log2cap, (int64_t)gk, val)) raise_error(kErrCapacity);
}

// Position of the k-th set bit of m (k < popc(m)).
__device__ __forceinline__ uint32_t ws_select(uint32_t m, uint32_t k) {
    uint32_t pos = 0;
#pragma unroll
    for (uint32_t width = 16; width >= 1; width >>= 1) {
        const uint32_t low = __popc(m & ((1u << width) - 1u));
        if (k >= low) {
            k -= low;
            m >>= width;
            pos += width;
        }
    }
    return pos;
}

// One row tile: block slot, first row in the block, rows, block rows, and
// the rows [a, b) of the tile inside the query's row slice.
struct WsTile {
    uint32_t slot, r0, n, rows, a, b;
};

// How one column of one tile is read.
struct WsCol {
    uint32_t mode;        // kWm*
    const uint8_t* src;   // stage: the rows; LZ4: the block; cascaded: the page
    uint32_t aux0, aux1;  // LZ4: [lo, hi) in the block; cascaded: page bytes, page rows
    uint32_t bytes;       // stage: bytes copied; LZ4: the block's compressed bytes
    int32_t cval;         // kWmConst: the value
};

// Rank-space tile t (t-th tile of the surviving chunks, chunk-major) ->
// its tile; false when t is past the end or the tile has no rows of the
// query's slice.
__device__ __forceinline__ bool ws_locate(const WsParams& P, const uint32_t* s_kbits, const uint32_t* s_kpre,
                                          uint32_t t, uint32_t t_end, WsTile& T) {
    if (t >= t_end) return false;
    const uint32_t tpb = P.tiles_per_block, bpc = P.blocks_per_chunk;
    const uint32_t PC = bpc * tpb;  // the launch keeps tile indices below 2^31
    const uint32_t k = t / PC, loc = t - k * PC;
    uint32_t lo = 0, hi = P.chunk_words - 1;  // the bitmap word holding the k-th surviving chunk
    while (lo < hi) {
        const uint32_t mid = (lo + hi + 1) >> 1;
        if (s_kpre[mid] <= k) lo = mid; else hi = mid - 1;
    }
    const uint32_t chunk = P.chunk_lo + lo * 32 + ws_select(s_kbits[lo], k - s_kpre[lo]);
    const uint32_t jb = loc / tpb, tile = loc % tpb;
    const uint64_t c_r0 = (uint64_t)chunk * P.rows_per_chunk;
    const uint64_t c_rows = min((uint64_t)P.rows_per_chunk, P.n_rows - c_r0);
    const uint64_t jrow = (uint64_t)jb * P.rows_per_block;
    T.rows = jrow < c_rows ? (uint32_t)min((uint64_t)P.rows_per_block, c_rows - jrow) : 0u;
    T.r0 = tile * kWsTile;
    T.slot = chunk * bpc + jb;
    if (T.r0 >= T.rows) return false;
    T.n = min(kWsTile, T.rows - T.r0);
    const uint64_t g0 = c_r0 + jrow + T.r0;
    const ShQuery& Q = P.q;
    T.a = Q.row_lo > g0 ? (uint32_t)min((uint64_t)T.n, Q.row_lo - g0) : 0u;
    T.b = Q.row_hi > g0 ? (uint32_t)min((uint64_t)T.n, Q.row_hi - g0) : 0u;
    return T.a < T.b;
}

// Column c's read decision for tile T (directory entry, side-index
// entries, a cascaded page's header: a single-run page needs no decode).
__device__ __forceinline__ WsCol ws_column(const WsParams& P, const gx_dcol& col, uint32_t c, const WsTile& T) {
    WsCol C;
    C.mode = kWmBad;
    C.src = nullptr;
    C.aux0 = C.aux1 = C.bytes = 0;
    C.cval = 0;
    const uint32_t slot = T.slot, r0 = T.r0, n = T.n, rows = T.rows;
    const uint4 dw = __ldg((const uint4*)(col.blocks + slot));
    const uint64_t d_off = ((uint64_t)dw.y << 32) | dw.x;
    const uint32_t d_bytes = dw.z, d_rows = dw.w;
    const bool dir_ok =
        d_rows == rows && d_off <= col.payload_bytes && (uint64_t)d_bytes + 32 <= col.payload_bytes - d_off;
    const uint8_t* blk = col.payload + d_off;
    if (col.codec == GX_CODEC_NONE) {
        if (dir_ok && d_bytes == rows * 4 && (d_off & 15u) == 0 && P.stage_of[c] != kWsNone) {
            C.mode = kWmStage;
            C.src = blk + 4ull * r0;
            C.bytes = (4 * n + 15u) & ~15u;
        }
    } else if (col.codec == GX_CODEC_LZ4) {
        const uint32_t sr = 1u << col.seg_shift;
        const uint32_t j0 = r0 >> col.seg_shift, nseg = (n + sr - 1) >> col.seg_shift;
        if ((r0 & (sr - 1u)) == 0 && j0 + nseg <= col.S) {
            const uint32_t* e = col.seg + (size_t)2 * col.S * slot;
            const uint32_t e0 = __ldg(e + 2 * j0), e1 = __ldg(e + 2 * j0 + 1);
            const uint32_t e2 = j0 + nseg < col.S ? __ldg(e + 2 * (j0 + nseg)) : 0u;
            const uint32_t hi = j0 + nseg < col.S ? e2 : d_bytes;
            if (dir_ok && e0 <= hi && hi <= d_bytes) {
                const bool lit = (e1 & 16u) && (e1 >> 5) >= 4 * n && hi - e0 == 4 * n;
                if (lit && ((d_off + e0) & 15u) == 0 && P.stage_of[c] != kWsNone) {
                    C.mode = kWmStage;
                    C.src = blk + e0;
                    C.bytes = (4 * n + 15u) & ~15u;
                } else if (P.buf_of[c] != kWsNone) {
                    C.mode = kWmLz4;
                    C.src = blk;
                    C.aux0 = e0;
                    C.aux1 = hi;
                    C.bytes = d_bytes;
                }
            }
        }
    } else if (col.codec == GX_CODEC_CASCADED) {
        const uint32_t page = r0 >> kCascPageLog2;
        if (page < col.S && P.buf_of[c] != kWsNone) {
            const uint32_t* e = col.seg + (size_t)2 * col.S * slot + 2 * page;
            const uint32_t po = __ldg(e), pb = __ldg(e + 1);
            if (dir_ok && (d_off & 15u) == 0 && (po & 15u) == 0 && (uint64_t)po + pb <= d_bytes && pb >= 32) {
                const uint8_t* pg = blk + po;
                C.mode = kWmCasc;
                C.src = pg;
                C.aux0 = pb;
                C.aux1 = min(kCascPageRows, rows - page * kCascPageRows);
                // pages that hold one value need no decode: zero-width values
                // without RLE (with DELTA: zero steps), or one run of the whole page
                const casc_hdr h = casc_load_header(pg);
                const bool rle = (h.flags & CASC_RLE) != 0, delta = (h.flags & CASC_DELTA) != 0;
                if (casc_header_ok(h, pb, C.aux1)) {
                    if (!rle && h.val_bits == 0 && (!delta || h.val_base == 0)) {
                        C.mode = kWmConst;
                        C.cval = delta ? h.first : h.val_base;
                    } else if (rle && h.n_runs <= 8) {
                        // a few runs (sorted columns): the run holding the tile's first
                        // row, and whether it also holds the last
                        const uint32_t* vw = (const uint32_t*)(pg + h.vals_off);
                        const uint32_t* lw = (const uint32_t*)(pg + h.lens_off);
                        const uint32_t h0 = r0 & (kCascPageRows - 1u), h1 = h0 + n;
                        uint32_t end = 0, val = 0;
                        for (uint32_t k = 0; k < h.n_runs; ++k) {
                            const uint32_t start = end;
                            end += unpack_bits(lw, k, h.len_bits) + h.len_base;
                            const uint32_t e =
                                (delta && k == 0) ? 0u : unpack_bits(vw, k, h.val_bits) + (uint32_t)h.val_base;
                            val = delta ? val + e : e;
                            if (start <= h0 && h0 < end) {
                                const uint32_t v0 = delta ? val + (uint32_t)h.first : val;
                                if (h1 <= end) {
                                    C.mode = kWmConst;
                                    C.cval = (int32_t)v0;
                                } else if (k + 1 < h.n_runs) {
                                    // the next run: when it covers the rest of the tile,
                                    // the tile is two runs
                                    const uint32_t end2 = end + unpack_bits(lw, k + 1, h.len_bits) + h.len_base;
                                    const uint32_t e2 = unpack_bits(vw, k + 1, h.val_bits) + (uint32_t)h.val_base;
                                    const uint32_t v1 = delta ? v0 + e2 : e2;
                                    if (h1 <= end2) {
                                        C.mode = kWmRuns2;
                                        C.cval = (int32_t)v0;
                                        C.aux0 = end - h0;
                                        C.aux1 = v1;
                                    }
                                }
                                break;
                            }
                        }
                    }
                }
            }
        }
    }
    return C;
}

// Decisions for the four tiles t0 + q*W (q = 0..3) at once: lane 8q + c
// decides column c of tile q (and checks prune predicate c's zone map), so
// the four tiles cost one round of dependent loads.  Returns the mask of
// the tiles to scan; every lane of group q holds tile q in T.
__device__ __forceinline__ uint32_t ws_decide(const WsParams& P, const gx_dcol* s_cols, const uint32_t* s_kbits,
                                              const uint32_t* s_kpre, uint32_t t0, uint32_t W, uint32_t t_end,
                                              uint32_t lane, WsTile& T, WsCol& C) {
    const ShQuery& Q = P.q;
    const uint32_t q = lane >> 3, c = lane & 7;
    const bool ok = ws_locate(P, s_kbits, s_kpre, t0 + q * W, t_end, T);
    bool zfail = false;
    if (ok && c < Q.n_prune) {
        const PrunePred& pr = Q.prune[c];
        if (pr.bmins) zfail = !(pr.lo <= __ldg(pr.bmaxs + T.slot) && pr.hi >= __ldg(pr.bmins + T.slot));
    }
    C.mode = kWmBad;
    if (ok && c < P.n_cols) C = ws_column(P, s_cols[c], c, T);
    const uint32_t oks = __ballot_sync(0xFFFFFFFFu, ok), fails = __ballot_sync(0xFFFFFFFFu, zfail);
    uint32_t vm = 0;
#pragma unroll
    for (uint32_t g = 0; g < 4; ++g)
        if (((oks >> (8 * g)) & 1u) && ((fails >> (8 * g)) & 0xFFu) == 0) vm |= 1u << g;
    return vm;
}

// L2 prefetch of the directory and side-index lines of the four tiles
// t0 + q*W (lane 8q + c: column c), so that their decisions read L2.
__device__ __forceinline__ void ws_prefetch_meta(const WsParams& P, const gx_dcol* s_cols, const uint32_t* s_kbits,
                                                 const uint32_t* s_kpre, uint32_t t0, uint32_t W, uint32_t t_end,
                                                 uint32_t lane) {
    const uint32_t q = lane >> 3, c = lane & 7;
    WsTile T;
    if (c >= P.n_cols || !ws_locate(P, s_kbits, s_kpre, t0 + q * W, t_end, T)) return;
    const gx_dcol& col = s_cols[c];
    asm volatile("prefetch.global.L2 [%0];" ::"l"(col.blocks + T.slot));
    if (col.codec == GX_CODEC_LZ4)
        asm volatile("prefetch.global.L2 [%0];" ::"l"(col.seg + (size_t)2 * col.S * T.slot + 2 * (T.r0 >> col.seg_shift)));
    else if (col.codec == GX_CODEC_CASCADED)
        asm volatile("prefetch.global.L2 [%0];" ::"l"(col.seg + (size_t)2 * col.S * T.slot + 2 * (T.r0 >> kCascPageLog2)));
}

__device__ __forceinline__ void ws_bulk_prefetch_l2(const void* src, uint32_t bytes, uint64_t pol) {
    asm volatile("cp.async.bulk.prefetch.L2.global.L2::cache_hint [%0], %1, %2;" ::"l"(src), "r"(bytes), "l"(pol)
                 : "memory");
}

// A step over a column that holds one value v on the whole tile: decided
// once.  Returns true when the tile's rows are all dropped; else multiplies
// in the group-key digit of every kept row.
__device__ __forceinline__ bool ws_step_const(const ShStep& stp, int32_t v, uint32_t keep, uint32_t* gkb, bool grouped,
                                           uint32_t lane) {
    const uint32_t flags = stp.flags, dcard = stp.digit_card;
    bool f = !(flags & GX_STEP_FILTER) || (v >= stp.lo && v <= stp.hi);
    int32_t pp = v;
    if (f && (flags & GX_STEP_PROBE)) f = ht_probe_any(stp.ht, stp.ht_log2, stp.ht_layout, v, &pp);
    if (!f) return true;
    if (dcard && grouped) {
        const uint32_t dgt = (uint32_t)(pp - stp.digit_base);
        if (dgt >= dcard) {
            if (lane == 0) raise_error(kErrInvalid);
            return true;
        }
#pragma unroll 1
        for (uint32_t j = 0; j < kWsGroups; ++j) {
            if (!((keep >> (4 * j)) & 15u)) continue;
            uint4* g = (uint4*)(gkb + 128 * j + 4 * lane);
            uint4 x = *g;
            x.x = x.x * dcard + dgt;
            x.y = x.y * dcard + dgt;
            x.z = x.z * dcard + dgt;
            x.w = x.w * dcard + dgt;
            *g = x;
        }
    }
    return false;
}

// A filter / probe / digit step over the tile's rows of a column at `col`
// (shared memory, kWsTile rows).  Probes issue the first-slot reads of a
// row group's distinct keys together and reuse the lane's last result for a
// repeated key.  Returns the new keep bits.
__device__ __forceinline__ uint32_t ws_step_rows(const ShStep& stp, const uint8_t* col, uint32_t keep, uint32_t* gkb,
                                              bool grouped, uint64_t pol_keep, uint32_t lane) {
    const uint32_t flags = stp.flags, dcard = stp.digit_card;
    const int32_t lo = stp.lo, hi = stp.hi, dbase = stp.digit_base;
    const bool filt = (flags & GX_STEP_FILTER) != 0, probe = (flags & GX_STEP_PROBE) != 0;
    const uint64_t* const ht = stp.ht;
    const uint32_t htlog = stp.ht_log2, htlay = stp.ht_layout;
    const bool dense = htlay == GX_HT_DENSE, bucket = htlay == GX_HT_BUCKET;
    uint32_t hbase = 0, hspan = 0;
    if (probe && dense) {
        const uint64_t hdr = __ldg((const unsigned long long*)ht);
        hbase = (uint32_t)hdr;
        hspan = (uint32_t)(hdr >> 32);
    }
    int32_t mv = 0, mp = 0;  // the lane's last probed key and its result
    bool mhave = false, mf = false;
#pragma unroll 1
    for (uint32_t j = 0; j < kWsGroups; ++j) {
        uint32_t kk = (keep >> (4 * j)) & 15u;
        if (!kk) continue;
        const uint4 w4 = *(const uint4*)(col + (128 * j + 4 * lane) * 4);
        const int32_t v[4] = {(int32_t)w4.x, (int32_t)w4.y, (int32_t)w4.z, (int32_t)w4.w};
        if (filt) {
#pragma unroll
            for (uint32_t i = 0; i < 4; ++i)
                if (!(v[i] >= lo && v[i] <= hi)) kk &= ~(1u << i);
        }
        int32_t pp[4] = {v[0], v[1], v[2], v[3]};
        if (probe && kk) {
            uint64_t ee[4];
            uint32_t rd = 0;
#pragma unroll
            for (uint32_t i = 0; i < 4; ++i) {
                const bool again =
                    (i > 0 && v[i] == v[i - 1] && ((kk >> (i - 1)) & 1u)) || (mhave && v[i] == mv);
                const uint32_t u = (uint32_t)v[i] - hbase;
                const bool r = ((kk >> i) & 1u) && !again && !bucket && v[i] != kEmptyKey && (!dense || u < hspan);
                const unsigned long long* sl = (const unsigned long long*)ht + (dense ? 1 + u : hash_key32(v[i], htlog));
                ee[i] = r ? ws_ld_slot(sl, pol_keep) : (unsigned long long)kEmptySlot;
                rd |= r ? 1u << i : 0u;
            }
#pragma unroll
            for (uint32_t i = 0; i < 4; ++i) {
                if (!((kk >> i) & 1u)) continue;
                bool f;
                int32_t p = v[i];
                if (mhave && v[i] == mv) {
                    f = mf;
                    p = mp;
                } else if ((rd >> i) & 1u) {
                    const int32_t ek = (int32_t)(uint32_t)ee[i];
                    if (ek == v[i]) {
                        f = true;
                        p = (int32_t)(uint32_t)(ee[i] >> 32);
                    } else if (dense || ek == kEmptyKey) {
                        f = false;
                    } else {
                        f = sh_probe(ht, htlog, htlay, v[i], &p);
                    }
                } else {
                    // bucket tables, keys the memo held when the reads were issued,
                    // the reserved key, keys outside a dense range
                    f = sh_probe(ht, htlog, htlay, v[i], &p);
                }
                mhave = true;
                mv = v[i];
                mf = f;
                mp = p;
                pp[i] = p;
                if (!f) kk &= ~(1u << i);
            }
        }
        if (dcard && grouped && kk) {
            uint4* g = (uint4*)(gkb + 128 * j + 4 * lane);
            const uint4 x = *g;
            uint32_t xg[4] = {x.x, x.y, x.z, x.w};
#pragma unroll
            for (uint32_t i = 0; i < 4; ++i) {
                if (!((kk >> i) & 1u)) continue;
                const uint32_t dgt = (uint32_t)(pp[i] - dbase);
                if (dgt >= dcard) {
                    raise_error(kErrInvalid);
                    kk &= ~(1u << i);
                } else {
                    xg[i] = xg[i] * dcard + dgt;
                }
            }
            *g = make_uint4(xg[0], xg[1], xg[2], xg[3]);
        }
        keep = (keep & ~(15u << (4 * j))) | (kk << (4 * j));
    }
    return keep;
}

// The aggregate over the kept rows of the tile: the value column at `col`
// (mask 0: one value), the carried column at `ccol`.  Returns the scalar
// part; grouped sums go to the warp's group table.
__device__ __forceinline__ int64_t ws_aggregate(uint32_t agg, bool grouped, bool carried, const uint8_t* col, uint32_t msk,
                                             const uint8_t* ccol, uint32_t cmask, uint32_t keep, const uint32_t* gkb,
                                             uint32_t* tkey, unsigned long long* tsum, int64_t* g_keys,
                                             int64_t* g_sums, uint32_t g_log2, uint32_t lane) {
    if (!grouped && agg == GX_AGG_COUNT) return __popc(keep);
    if (!grouped && agg == GX_AGG_SUM && msk == 0) return (int64_t)__popc(keep) * *(const int32_t*)col;
    int64_t acc = 0;
#pragma unroll 1
    for (uint32_t j = 0; j < kWsGroups; ++j) {
        const uint32_t kk = (keep >> (4 * j)) & 15u;
        if (!kk) continue;
        const uint32_t ro = (128 * j + 4 * lane) * 4;
        const uint4 w4 = *(const uint4*)(col + (ro & msk));
        const uint4 cw = carried ? *(const uint4*)(ccol + (ro & cmask)) : make_uint4(0, 0, 0, 0);
        const int32_t v[4] = {(int32_t)w4.x, (int32_t)w4.y, (int32_t)w4.z, (int32_t)w4.w};
        const int32_t cv[4] = {(int32_t)cw.x, (int32_t)cw.y, (int32_t)cw.z, (int32_t)cw.w};
        if (!grouped) {
            if (agg == GX_AGG_SUM_PRODUCT) {
#pragma unroll
                for (uint32_t i = 0; i < 4; ++i) acc += ((kk >> i) & 1u) ? (int64_t)v[i] * cv[i] : 0;
            } else if (agg == GX_AGG_SUM_DIFF) {
#pragma unroll
                for (uint32_t i = 0; i < 4; ++i) acc += ((kk >> i) & 1u) ? (int64_t)v[i] - cv[i] : 0;
            } else {
#pragma unroll
                for (uint32_t i = 0; i < 4; ++i) acc += ((kk >> i) & 1u) ? (int64_t)v[i] : 0;
            }
        } else {
            const uint4 gw = *(const uint4*)(gkb + 128 * j + 4 * lane);
            const uint32_t g[4] = {gw.x, gw.y, gw.z, gw.w};
#pragma unroll
            for (uint32_t i = 0; i < 4; ++i) {
                if (!((kk >> i) & 1u)) continue;
                const int64_t val = agg == GX_AGG_SUM_PRODUCT ? (int64_t)v[i] * cv[i]
                                    : agg == GX_AGG_SUM_DIFF  ? (int64_t)v[i] - cv[i]
                                    : agg == GX_AGG_COUNT      ? 1
                                                               : (int64_t)v[i];
                ws_group_add(g[i], val, tkey, tsum, g_keys, g_sums, g_log2);
            }
        }
    }
    return acc;
}

// ---- plan signatures: compile-time evaluators for the known query shapes
// A signature packs the step count (bits 0-2), the aggregate (3-5), grouped
// (6) and per step s a kind nibble at bit 7 + 4 s: 1 FILTER, 2 PROBE,
// 4 CARRY, 8 group-key digit.  Signature 0 is the run-time evaluator.
constexpr uint32_t kWkF = 1, kWkP = 2, kWkC = 4, kWkD = 8;
constexpr uint32_t ws_sig(uint32_t ns, uint32_t agg, bool grouped, uint32_t k0, uint32_t k1 = 0, uint32_t k2 = 0,
                          uint32_t k3 = 0, uint32_t k4 = 0, uint32_t k5 = 0) {
    return ns | (agg << 3) | ((grouped ? 1u : 0u) << 6) | (k0 << 7) | (k1 << 11) | (k2 << 15) | (k3 << 19) |
           (k4 << 23) | (k5 << 27);
}
// pipeline_q1_lineorder: date probe, discount filter carried, quantity filter, price x discount
constexpr uint32_t kSigQ1 = ws_sig(4, GX_AGG_SUM_PRODUCT, false, kWkP, kWkF | kWkC, kWkF, 0);
// pipeline_q3: customer / supplier / date probes with digits, revenue grouped
constexpr uint32_t kSigQ3 = ws_sig(4, GX_AGG_SUM, true, kWkP | kWkD, kWkP | kWkD, kWkP | kWkD, 0);
// pipeline_q2: part probe (brand digit), supplier probe, date probe (year digit), revenue grouped
constexpr uint32_t kSigQ2 = ws_sig(4, GX_AGG_SUM, true, kWkP | kWkD, kWkP, kWkP | kWkD, 0);
// pipeline_q4: customer (nation digit), supplier, date (year digit), part probes, supplycost carried, profit grouped
constexpr uint32_t kSigQ4 = ws_sig(6, GX_AGG_SUM_DIFF, true, kWkP | kWkD, kWkP, kWkP | kWkD, kWkP, kWkC, 0);

// The tile's rows evaluated through all steps of a compile-time signature,
// one 128-row group at a time: every column's 4 values of the lane are
// loaded first, then the steps run on registers (carried values and group
// keys included).  Steps over a column that holds one value on the tile
// (other than the last) are decided once for the tile.  Returns the scalar
// part; grouped sums go to the warp's group table.
template <uint32_t SIG>
__device__ __forceinline__ int64_t ws_eval_sig(const ShQuery& Q, const uint8_t* sbase, const uint32_t* off,
                                               const uint32_t* msk, uint32_t keep, uint32_t* tkey,
                                               unsigned long long* tsum, uint64_t pol_keep, const uint64_t* s_hdr,
                                               uint32_t lane) {
    constexpr uint32_t NS = SIG & 7, AGG = (SIG >> 3) & 7;
    constexpr bool GR = ((SIG >> 6) & 1) != 0;
    int64_t acc = 0;
    uint32_t cd[NS];  // constant steps: the group-key digit
    int32_t cv[NS];   // constant steps: the value
#pragma unroll
    for (uint32_t s = 0; s < NS; ++s) {
        cd[s] = 0;
        cv[s] = 0;
        if (s + 1 < NS && msk[s] == 0) {
            const uint32_t K = (SIG >> (7 + 4 * s)) & 15u;
            const ShStep& stp = Q.steps[s];
            const int32_t v = *(const int32_t*)(sbase + off[s]);
            cv[s] = v;
            bool f = !(K & kWkF) || (v >= stp.lo && v <= stp.hi);
            int32_t pp = v;
            if ((K & kWkP) && f) {
                if (stp.ht_layout == GX_HT_DENSE) {  // one read: the table header is cached
                    const uint64_t hdr = s_hdr[s];
                    const uint32_t u = (uint32_t)v - (uint32_t)hdr;
                    f = false;
                    if (v != kEmptyKey && u < (uint32_t)(hdr >> 32)) {
                        const unsigned long long e = ws_ld_slot((const unsigned long long*)stp.ht + 1 + u, pol_keep);
                        f = (int32_t)(uint32_t)e == v;
                        pp = (int32_t)(uint32_t)(e >> 32);
                    }
                } else {
                    f = ht_probe_any(stp.ht, stp.ht_log2, stp.ht_layout, v, &pp);
                }
            }
            if ((K & kWkD) && f) {
                cd[s] = (uint32_t)(pp - stp.digit_base);
                if (cd[s] >= stp.digit_card) {
                    if (lane == 0) raise_error(kErrInvalid);
                    f = false;
                }
            }
            if (!f) return 0;  // no row of the tile passes
        }
    }
    // kWsEvalGroups row groups at a time for scalar plans: their column loads
    // and first-slot probes are all in flight before any is used (grouped
    // plans, whose group-table inserts are long inlined loops, run one)
    constexpr uint32_t H = GR ? 1u : kWsEvalGroups;
#pragma unroll 1
    for (uint32_t j0 = 0; j0 < kWsGroups; j0 += H) {
        uint32_t kk[H];
        uint32_t live = 0;
#pragma unroll
        for (uint32_t h = 0; h < H; ++h) {
            kk[h] = (keep >> (4 * (j0 + h))) & 15u;
            live |= kk[h];
        }
        if (!live) continue;
        uint4 w[H][NS];
#pragma unroll
        for (uint32_t h = 0; h < H; ++h) {
            const uint32_t ro = (128 * (j0 + h) + 4 * lane) * 4;
            // (a column constant on the tile reads its broadcast slot: mask 0)
#pragma unroll
            for (uint32_t s = 0; s < NS; ++s) w[h][s] = *(const uint4*)(sbase + off[s] + (ro & msk[s]));
        }
        int32_t carry[H][4];
        uint32_t g[H][4];
#pragma unroll
        for (uint32_t h = 0; h < H; ++h)
#pragma unroll
            for (uint32_t i = 0; i < 4; ++i) {
                carry[h][i] = 0;
                g[h][i] = 0;
            }
#pragma unroll
        for (uint32_t s = 0; s < NS; ++s) {
            const uint32_t K = (SIG >> (7 + 4 * s)) & 15u;
            const ShStep& stp = Q.steps[s];
            if (s + 1 < NS && msk[s] == 0) {  // decided for the tile
                if (K & kWkD) {
                    const uint32_t dcard = stp.digit_card;
#pragma unroll
                    for (uint32_t h = 0; h < H; ++h)
#pragma unroll
                        for (uint32_t i = 0; i < 4; ++i) g[h][i] = g[h][i] * dcard + cd[s];
                }
                if (K & kWkC) {
#pragma unroll
                    for (uint32_t h = 0; h < H; ++h)
#pragma unroll
                        for (uint32_t i = 0; i < 4; ++i) carry[h][i] = cv[s];
                }
                continue;
            }
            int32_t v[H][4];
#pragma unroll
            for (uint32_t h = 0; h < H; ++h) {
                v[h][0] = (int32_t)w[h][s].x;
                v[h][1] = (int32_t)w[h][s].y;
                v[h][2] = (int32_t)w[h][s].z;
                v[h][3] = (int32_t)w[h][s].w;
            }
            if (K & kWkF) {
                // lo <= v <= hi as one unsigned comparison of v - lo with hi - lo
                // (an empty range, hi < lo, keeps nothing)
                const uint32_t lo = (uint32_t)stp.lo, span = (uint32_t)stp.hi - lo;
                const uint32_t none = stp.hi < stp.lo ? 0u : 15u;
#pragma unroll
                for (uint32_t h = 0; h < H; ++h) {
                    uint32_t pass = 0;
#pragma unroll
                    for (uint32_t i = 0; i < 4; ++i) pass |= ((uint32_t)v[h][i] - lo <= span) ? 1u << i : 0u;
                    kk[h] &= pass & none;
                }
            }
            int32_t pp[H][4];
#pragma unroll
            for (uint32_t h = 0; h < H; ++h)
#pragma unroll
                for (uint32_t i = 0; i < 4; ++i) pp[h][i] = v[h][i];
            if (K & kWkP) {
                const uint64_t* const ht = stp.ht;
                const uint32_t htlog = stp.ht_log2, htlay = stp.ht_layout;
                const bool dense = htlay == GX_HT_DENSE, bucket = htlay == GX_HT_BUCKET;
                uint32_t hbase = 0, hspan = 0;
                if (dense) {
                    const uint64_t hdr = s_hdr[s];
                    hbase = (uint32_t)hdr;
                    hspan = (uint32_t)(hdr >> 32);
                }
                // the first slot of every kept row's key, all read before any is used
                uint64_t ee[H][4];
#pragma unroll
                for (uint32_t h = 0; h < H; ++h)
#pragma unroll
                    for (uint32_t i = 0; i < 4; ++i) {
                        const uint32_t u = (uint32_t)v[h][i] - hbase;
                        const bool r =
                            ((kk[h] >> i) & 1u) && !bucket && v[h][i] != kEmptyKey && (!dense || u < hspan);
                        const unsigned long long* sl =
                            (const unsigned long long*)ht + (dense ? 1 + u : hash_key32(v[h][i], htlog));
                        ee[h][i] = r ? ws_ld_slot(sl, pol_keep) : (unsigned long long)kEmptySlot;
                    }
#pragma unroll
                for (uint32_t h = 0; h < H; ++h)
#pragma unroll
                    for (uint32_t i = 0; i < 4; ++i) {
                        if (!((kk[h] >> i) & 1u)) continue;
                        const int32_t ek = (int32_t)(uint32_t)ee[h][i];
                        bool f;
                        int32_t p = v[h][i];
                        if (ek == v[h][i] && v[h][i] != kEmptyKey) {
                            f = true;
                            p = (int32_t)(uint32_t)(ee[h][i] >> 32);
                        } else if (!bucket && (dense || ek == kEmptyKey)) {
                            f = false;  // an empty first slot, or a dense table's slot of another key
                        } else {
                            f = sh_probe(ht, htlog, htlay, v[h][i], &p);  // a linear chain, or a bucket table
                        }
                        pp[h][i] = p;
                        if (!f) kk[h] &= ~(1u << i);
                    }
            }
            if (K & kWkD) {
                const uint32_t dcard = stp.digit_card;
                const int32_t dbase = stp.digit_base;
#pragma unroll
                for (uint32_t h = 0; h < H; ++h)
#pragma unroll
                    for (uint32_t i = 0; i < 4; ++i) {
                        if (!((kk[h] >> i) & 1u)) continue;
                        const uint32_t dgt = (uint32_t)(pp[h][i] - dbase);
                        if (dgt >= dcard) {
                            raise_error(kErrInvalid);
                            kk[h] &= ~(1u << i);
                        } else {
                            g[h][i] = g[h][i] * dcard + dgt;
                        }
                    }
            }
            if (K & kWkC) {
#pragma unroll
                for (uint32_t h = 0; h < H; ++h)
#pragma unroll
                    for (uint32_t i = 0; i < 4; ++i) carry[h][i] = v[h][i];
            }
            live = 0;
#pragma unroll
            for (uint32_t h = 0; h < H; ++h) live |= kk[h];
            if (!live) break;
            if (s + 1 == NS) {
#pragma unroll
                for (uint32_t h = 0; h < H; ++h) {
                    if (GR) {
#pragma unroll
                        for (uint32_t i = 0; i < 4; ++i) {
                            if (!((kk[h] >> i) & 1u)) continue;
                            const int64_t val = AGG == GX_AGG_SUM_PRODUCT ? (int64_t)v[h][i] * carry[h][i]
                                                : AGG == GX_AGG_SUM_DIFF  ? (int64_t)v[h][i] - carry[h][i]
                                                : AGG == GX_AGG_COUNT      ? 1
                                                                           : (int64_t)v[h][i];
                            ws_group_add(g[h][i], val, tkey, tsum, Q.g_keys, Q.g_sums, Q.g_log2);
                        }
                    } else {
                        // kept rows as multiply-adds by 0 or 1 (one wide multiply-add per row)
#pragma unroll
                        for (uint32_t i = 0; i < 4; ++i) {
                            const int32_t on = (int32_t)((kk[h] >> i) & 1u);
                            if (AGG == GX_AGG_SUM_PRODUCT) {
                                acc += (int64_t)v[h][i] * (int64_t)(on ? carry[h][i] : 0);
                            } else if (AGG == GX_AGG_SUM_DIFF) {
                                acc += (int64_t)v[h][i] * on;
                                acc -= (int64_t)carry[h][i] * on;
                            } else if (AGG == GX_AGG_COUNT) {
                                acc += on;
                            } else {
                                acc += (int64_t)v[h][i] * on;
                            }
                        }
                    }
                }
            }
        }
    }
    return acc;
}

template <uint32_t SIG>
__global__ void __launch_bounds__(kWsNT, (SIG == 0 || ((SIG >> 6) & 1)) ? 4 : 3) warp_scan_kernel(const __grid_constant__ WsParams P) {
    extern __shared__ __align__(16) uint8_t smem[];
    __shared__ gx_dcol s_cols[kWsMaxCols];
    __shared__ uint32_t s_nsurv;
    const uint32_t tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const uint32_t ncols = P.n_cols;
    const ShQuery& Q = P.q;
    uint32_t* const s_kbits = (uint32_t*)smem;               // chunk keep bits of [chunk_lo, chunk_hi)
    uint32_t* const s_kpre = s_kbits + P.chunk_words;        // surviving chunks before each word
    uint32_t* const wmem = s_kpre + P.chunk_words + (size_t)warp * P.warp_words;
    uint4* const cslot = (uint4*)wmem;                       // constant columns (4 copies of the value)
    uint64_t* const bar = (uint64_t*)(wmem + 4 * kWsMaxCols);  // the warp's stage mbarrier
    uint64_t* const whdr = (uint64_t*)(wmem + 4 * kWsMaxCols + 4);  // dense join tables' headers, per step
    uint32_t* const areas = wmem + kWsHead;                  // n_areas x kWsTile words
    // grouped plans: the run-time evaluator's group key of each row of the tile
    // (compile-time evaluators keep keys in registers), then the group table
    uint32_t* const gkb = areas + (size_t)P.n_areas * kWsTile;
    // grouped: the CTA's group table (keys, then sums) after the warps' regions
    uint32_t* const tkey = s_kpre + P.chunk_words + (size_t)kWsWarps * P.warp_words;
    unsigned long long* const tsum = (unsigned long long*)(tkey + kWsGroupSlots);
    const uint64_t pol_keep = ws_policy_keep(), pol_stream = ws_policy_stream();

    // The launch may overlap the kernel before it on the stream (programmatic
    // dependent launch): until a thread has passed griddep_wait it reads only
    // the columns (payload, directory, side index, min/max, zone maps: never
    // written by kernels), and every read of join tables, keep_in, and every
    // global write (results, keep_out, group tables) comes after its wait.
    bool waited = false;
    if (Q.keep_in) {  // keep flags may come from the kernel before
        griddep_wait();
        waited = true;
    }
    // a warp's first evaluation: the wait, then the dense join tables' headers
    auto await_tables = [&]() {
        if (!waited) griddep_wait();
        waited = true;
        if (lane < GX_MAX_STEPS) {
            const ShStep& st = Q.steps[lane];
            whdr[lane] = (lane < Q.n_steps && (st.flags & GX_STEP_PROBE) && st.ht_layout == GX_HT_DENSE)
                             ? __ldcg((const unsigned long long*)st.ht)
                             : 0ull;
        }
        __syncwarp();
    };
    bool tables = false;  // whdr loaded
    for (uint32_t i = tid; i < ncols * (uint32_t)(sizeof(gx_dcol) / 4); i += kWsNT)
        ((uint32_t*)s_cols)[i] = ((const uint32_t*)P.cols)[i];
    // chunk keep (keep_in and the prune predicates' chunk min/max, the
    // reference's granularity), one ballot word per 32 chunks; CTA 0 writes
    // keep_out from them at the end
    const uint32_t n_range = P.chunk_hi - P.chunk_lo;
    for (uint32_t wb = warp * 32; wb < P.chunk_words * 32; wb += kWsNT) {
        const uint32_t i = wb + lane, chunk = P.chunk_lo + i;
        bool ck = i < n_range;
        if (ck) {
            if (Q.keep_in) ck = __ldg(Q.keep_in + chunk) != 0;
            for (uint32_t p = 0; p < Q.n_prune; ++p) {
                const PrunePred& pr = Q.prune[p];
                ck = ck && pr.lo <= __ldg(pr.maxs + chunk) && pr.hi >= __ldg(pr.mins + chunk);
            }
        }
        const uint32_t word = __ballot_sync(0xFFFFFFFFu, ck);
        if (lane == 0) s_kbits[wb / 32] = word;
    }
    if (lane == 0) mbar_init(bar, 1);
    if (P.grouped_tab) {
        for (uint32_t i = tid; i < kWsGroupSlots; i += kWsNT) {
            tkey[i] = kEmptyGKey;
            tsum[i] = 0;
        }
    }
    __syncthreads();
    if (warp == 0) {  // exclusive prefix of the popcounts: per lane a run of words, then a warp scan
        const uint32_t per = (P.chunk_words + 31) / 32, w0 = min(P.chunk_words, lane * per),
                       w1 = min(P.chunk_words, w0 + per);
        uint32_t cnt = 0;
        for (uint32_t i = w0; i < w1; ++i) cnt += __popc(s_kbits[i]);
        uint32_t run = ws_scan(cnt, lane) - cnt;
        for (uint32_t i = w0; i < w1; ++i) {
            s_kpre[i] = run;
            run += __popc(s_kbits[i]);
        }
        if (lane == 31) s_nsurv = run;
    }
    __syncthreads();  // the last block-wide barrier: warps are independent from here on

    const uint32_t PC = P.blocks_per_chunk * P.tiles_per_block;
    const uint32_t t_end = s_nsurv * PC;
    const uint32_t ns = Q.n_steps, agg = Q.agg;
    const bool grouped = Q.grouped != 0;
    const uint32_t W = gridDim.x * kWsWarps;
    int64_t local = 0;
    unsigned long long local_rows = 0;
    uint32_t ph = 0;
    bool stop = false;
    for (uint32_t t0 = blockIdx.x * kWsWarps + warp; t0 < t_end && !stop; t0 += 4 * W) {
        WsTile T;
        WsCol C;
        const uint32_t vm = ws_decide(P, s_cols, s_kbits, s_kpre, t0, W, t_end, lane, T, C);
        ws_prefetch_meta(P, s_cols, s_kbits, s_kpre, t0 + 4 * W, W, t_end, lane);
        // the staged ranges of every tile of the four go to L2 now
        if (((vm >> (lane >> 3)) & 1u) && (lane & 7) < ncols && C.mode == kWmStage) ws_bulk_prefetch_l2(C.src, C.bytes, pol_stream);
        for (uint32_t q = 0; q < 4 && !stop; ++q) {
            if (!((vm >> q) & 1u)) continue;
            const uint32_t L0 = 8 * q, Lc = 8 * q + (lane & 7);
            const uint32_t slot = __shfl_sync(0xFFFFFFFFu, T.slot, L0), r0 = __shfl_sync(0xFFFFFFFFu, T.r0, L0);
            const uint32_t n = __shfl_sync(0xFFFFFFFFu, T.n, L0), rows = __shfl_sync(0xFFFFFFFFu, T.rows, L0);
            const uint32_t a = __shfl_sync(0xFFFFFFFFu, T.a, L0), b = __shfl_sync(0xFFFFFFFFu, T.b, L0);
            // lane c (< ncols): column c of this tile
            const uint32_t mode = __shfl_sync(0xFFFFFFFFu, C.mode, Lc);
            const uint8_t* src = (const uint8_t*)ws_shfl64((uint64_t)C.src, Lc);
            const uint32_t aux0 = __shfl_sync(0xFFFFFFFFu, C.aux0, Lc), aux1 = __shfl_sync(0xFFFFFFFFu, C.aux1, Lc);
            const uint32_t cbytes = __shfl_sync(0xFFFFFFFFu, C.bytes, Lc);
            const int32_t cval = (int32_t)__shfl_sync(0xFFFFFFFFu, (uint32_t)C.cval, Lc);
            const bool mine = lane < ncols;
            // ---- stage copies (one bulk copy per in-place column)
            const uint32_t my = (mine && mode == kWmStage) ? cbytes : 0u;
            const uint32_t total = __reduce_add_sync(0xFFFFFFFFu, my);
            if (total) {
                if (lane == 0) mbar_expect_tx_arrive(bar, total);
                __syncwarp();
                if (my) ws_bulk_copy(areas + (size_t)P.stage_of[lane] * kWsTile, src, my, bar, pol_stream);
            }
            // ---- decodes, one column at a time by the whole warp
            int terr = __any_sync(0xFFFFFFFFu, mine && mode == kWmBad) ? kErrCorrupt : 0;
            uint32_t roff = 0, rmask = 0xFFFFFFFFu;  // lane c: shared-memory byte offset of column c's rows
            if (mine) {
                if (mode == kWmStage) {
                    roff = (uint32_t)((uint8_t*)(areas + (size_t)P.stage_of[lane] * kWsTile) - smem);
                } else if (mode == kWmConst) {
                    cslot[lane] = make_uint4((uint32_t)cval, (uint32_t)cval, (uint32_t)cval, (uint32_t)cval);
                    roff = (uint32_t)((uint8_t*)&cslot[lane] - smem);
                    rmask = 0;
                }
            }
            for (uint32_t c = 0; c < ncols && !terr; ++c) {
                const uint32_t m = __shfl_sync(0xFFFFFFFFu, mode, c);
                if (m != kWmLz4 && m != kWmCasc && m != kWmRuns2) continue;
                uint32_t* buf = areas + (size_t)P.buf_of[c] * kWsTile;
                if (m == kWmRuns2) {  // two runs: the rows written out directly
                    const uint32_t v0 = (uint32_t)__shfl_sync(0xFFFFFFFFu, (uint32_t)cval, c);
                    const uint32_t split = __shfl_sync(0xFFFFFFFFu, aux0, c), v1 = __shfl_sync(0xFFFFFFFFu, aux1, c);
#pragma unroll 1
                    for (uint32_t j = 0; j < kWsTile / 128; ++j) {
                        const uint32_t r = 128 * j + 4 * lane;
                        *(uint4*)(buf + r) = make_uint4(r < split ? v0 : v1, r + 1 < split ? v0 : v1,
                                                        r + 2 < split ? v0 : v1, r + 3 < split ? v0 : v1);
                    }
                    __syncwarp();
                    if (lane == c) roff = (uint32_t)((uint8_t*)buf - smem);
                    continue;
                }
                const uint8_t* cs = (const uint8_t*)ws_shfl64((uint64_t)src, c);
                const uint32_t x0 = __shfl_sync(0xFFFFFFFFu, aux0, c), x1 = __shfl_sync(0xFFFFFFFFu, aux1, c);
                int r;
                int32_t cv = 0;
                if (m == kWmCasc) {
                    r = ws_casc_rows(cs, x0, x1, r0 & (kCascPageRows - 1u), n, (int32_t*)buf, &cv, lane);
                } else {
                    const uint32_t bb = __shfl_sync(0xFFFFFFFFu, cbytes, c);
                    const gx_dcol& col = s_cols[c];
                    r = ws_lz4_rows(cs, bb, col.seg + (size_t)2 * col.S * slot, col.seg_shift, rows, r0, n, x0, x1,
                                    buf, lane);
                }
                if (r == 1) {  // one value for the whole tile
                    if (lane == c) {
                        cslot[c] = make_uint4((uint32_t)cv, (uint32_t)cv, (uint32_t)cv, (uint32_t)cv);
                        roff = (uint32_t)((uint8_t*)&cslot[c] - smem);
                        rmask = 0;
                    }
                } else if (r) {
                    terr = r;
                } else if (lane == c) {
                    roff = (uint32_t)((uint8_t*)buf - smem);
                }
            }
            // ---- the staged bytes
            if (total) {
                const bool ok = __all_sync(0xFFFFFFFFu, mbar_wait_bounded(bar, ph));
                ph ^= 1u;
                if (!ok) {
                    // the copies did not land: stop this warp (after one more bounded
                    // wait, so that no copy is left in flight into its shared memory)
                    if (lane == 0) raise_error(kErrTimeout);
                    mbar_wait_bounded(bar, ph ^ 1u);
                    stop = true;
                    break;
                }
            }
            __syncwarp();
            if (terr) {
                if (lane == 0) raise_error(terr);
            } else {
                local_rows += b - a;  // lane-uniform; lane 0's count is the warp's
                // ---- evaluation, step-major over the tile: the lane's rows are
                // 128 j + 4 lane + i (j < kWsGroups, i < 4), keep bit 4 j + i
                uint32_t keep = kWsGroups == 8 ? 0xFFFFFFFFu : (1u << (4 * kWsGroups)) - 1u;
                if (a != 0 || b != kWsTile) {
                    keep = 0;
#pragma unroll 1
                    for (uint32_t j = 0; j < kWsGroups; ++j) {
                        const int32_t base = (int32_t)(128 * j + 4 * lane);
                        const int32_t l = min(4, max(0, (int32_t)a - base)), h = min(4, max(0, (int32_t)b - base));
                        keep |= (h > l ? ((1u << h) - 1u) & ~((1u << l) - 1u) : 0u) << (4 * j);
                    }
                }
                if (SIG == 0 && grouped) {
#pragma unroll 1
                    for (uint32_t j = 0; j < kWsGroups; ++j) *(uint4*)(gkb + 128 * j + 4 * lane) = make_uint4(0, 0, 0, 0);
                }
                if (!tables) {
                    await_tables();
                    tables = true;
                }
                if constexpr (SIG != 0) {
                    constexpr uint32_t NS = SIG & 7;
                    uint32_t off[NS], msk[NS];
#pragma unroll
                    for (uint32_t s = 0; s < NS; ++s) {
                        const uint32_t c = Q.steps[s].col;
                        off[s] = __shfl_sync(0xFFFFFFFFu, roff, c);
                        msk[s] = __shfl_sync(0xFFFFFFFFu, rmask, c);
                    }
                    local += ws_eval_sig<SIG>(Q, smem, off, msk, keep, tkey, tsum, pol_keep, whdr, lane);
                }
                uint32_t coff = 0, cmask = 0;  // the carried column (none: carried values are 0)
                bool carried = false;
                for (uint32_t s = 0; SIG == 0 && s < ns; ++s) {
                    if (!__any_sync(0xFFFFFFFFu, keep)) break;
                    const ShStep& stp = Q.steps[s];
                    const uint32_t flags = stp.flags;
                    const uint32_t c = stp.col;
                    const uint32_t off = __shfl_sync(0xFFFFFFFFu, roff, c), msk = __shfl_sync(0xFFFFFFFFu, rmask, c);
                    if (flags & GX_STEP_CARRY) {
                        coff = off;
                        cmask = msk;
                        carried = true;
                    }
                    if (msk == 0) {
                        if (ws_step_const(stp, *(const int32_t*)(smem + off), keep, gkb, grouped, lane)) keep = 0;
                    } else if ((flags & (GX_STEP_FILTER | GX_STEP_PROBE)) || stp.digit_card) {
                        keep = ws_step_rows(stp, smem + off, keep, gkb, grouped, pol_keep, lane);
                    }
                    if (s + 1 == ns && keep)
                        local += ws_aggregate(agg, grouped, carried, smem + off, msk, smem + coff, cmask, keep, gkb,
                                              tkey, tsum, Q.g_keys, Q.g_sums, Q.g_log2, lane);
                }
            }
            // every lane is done with the tile's areas before the next copies overwrite them
            __syncwarp();
            if (lane == 0) fence_proxy_async_smem();
        }
    }
    // ---- results: the CTA's group table once every warp is done, else the warp's sum
    __syncwarp();
    if (!waited) griddep_wait();
    if (blockIdx.x == 0 && Q.keep_out)
        for (uint32_t i = tid; i < n_range; i += kWsNT) Q.keep_out[P.chunk_lo + i] = (s_kbits[i / 32] >> (i % 32)) & 1u;
    if (grouped && P.grouped_tab) {
        __syncthreads();
        for (uint32_t i = tid; i < kWsGroupSlots; i += kWsNT) {
            const uint32_t key = tkey[i];
            if (key != kEmptyGKey && !group_add_global(Q.g_keys, Q.g_sums, Q.g_log2, (int64_t)key, (int64_t)tsum[i]))
                raise_error(kErrCapacity);
        }
    } else if (!grouped) {
        const uint64_t u = warp_sum_u64((uint64_t)local);
        if (lane == 0 && u && Q.result) atomicAdd((unsigned long long*)Q.result, (unsigned long long)u);
    }
    if (lane == 0 && P.rows_scanned && local_rows) atomicAdd(P.rows_scanned, local_rows);
}
