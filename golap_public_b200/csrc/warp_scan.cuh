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
// Every warp is an independent worker: there is no block-wide barrier and no
// producer.  Warp w of the grid takes the row tiles w, w + W, w + 2W, ... of
// the table (kWsTile rows of one block each; W warps in the grid).  Per tile:
//   * lane c loads column c's directory entry and the tile's side-index
//     entries, and decides how the column's rows are read: in place from
//     HBM (raw rows, or an LZ4 literal run whose first byte is 16-byte
//     aligned), as one value for the whole tile (a cascaded run covering the
//     tile), or decoded by the warp into the warp's buffer in shared memory
//     (an LZ4 range with matches: groups of lanes per segment; a cascaded
//     page: run windows of 32 runs, one run per lane);
//   * the in-place ranges are prefetched into L2 (one line per lane);
//   * the plan's steps run over batches of 128 rows, 4 consecutive rows per
//     lane read with one 16-byte load per column (every column's load of a
//     batch is issued before the first step runs), filters, join probes
//     (each lane probes a repeated key once), group-key digits, carried
//     value, and the aggregate.
// Scalar sums stay in registers; grouped sums go to the warp's own group
// table in shared memory (keys that find no slot go to the global table) and
// are flushed when the warp is done.  Nothing waits on another warp.

constexpr uint32_t kWsLog2 = 10;
constexpr uint32_t kWsTile = 1u << kWsLog2;    // rows of one warp tile
constexpr uint32_t kWsNT = 256;                // threads per CTA (8 independent warps)
constexpr uint32_t kWsWarps = kWsNT / 32;
constexpr uint32_t kWsBatch = 128;             // rows per evaluation batch (4 per lane)
constexpr uint32_t kWsMaxCols = kPipeMaxCols;
constexpr uint32_t kWsGroupLog2 = 7;           // warp group table: 128 slots
constexpr uint32_t kWsGroupSlots = 1u << kWsGroupLog2;
constexpr uint32_t kWsGroupProbes = 16;
constexpr uint32_t kWsNoBuf = 0xFFFFFFFFu;
constexpr uint32_t kWsMaxDynSmem = 200u << 10;  // dynamic shared memory of one CTA at most
static_assert(kWsTile <= kCascPageRows && kCascPageRows % kWsTile == 0, "a warp tile lies in one cascaded page");

struct WsParams {
    ShQuery q;                      // steps index into cols
    gx_dcol cols[kWsMaxCols];
    uint32_t n_cols;
    uint32_t blocks_per_chunk, rows_per_chunk, rows_per_block, tiles_per_block;
    uint64_t n_rows;                // rows of the table
    uint32_t chunk_lo, chunk_hi;    // chunks [chunk_lo, chunk_hi) are scanned
    uint32_t buf_of[kWsMaxCols];    // the warp buffer column c decodes into, or kWsNoBuf (always read in place)
    uint32_t n_bufs;                // decode buffers per warp (kWsTile words each)
    uint32_t warp_words;            // shared memory words per warp
    uint32_t grouped_tab;           // 1: the warp has a group table
    unsigned long long* rows_scanned;
};

// Column read modes of one tile.
enum : uint32_t { kWmDirect = 0, kWmConst = 1, kWmLz4 = 2, kWmCasc = 3, kWmBad = 4 };

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
// the block into out (segment t at out + t * seg_rows), G lanes per segment.
// Returns 0 or kErrCorrupt (uniform).
__device__ __noinline__ int ws_lz4_rows(const gx_dcol& c, uint32_t slot, uint64_t blk_off, uint32_t blk_bytes,
                                        uint32_t rows, uint32_t r0, uint32_t n, uint32_t lo, uint32_t hi,
                                        uint32_t* out, uint32_t lane) {
    const uint32_t seg_rows = 1u << c.seg_shift;
    const uint32_t j0 = r0 >> c.seg_shift, nseg = (n + seg_rows - 1) >> c.seg_shift;
    const uint64_t abs_wb = (blk_off + lo) & ~15ull;
    const uint32_t* A = (const uint32_t*)(c.payload + abs_wb);
    const uint32_t wbase = (uint32_t)(abs_wb - blk_off);
    const uint32_t* e = c.seg + (size_t)2 * c.S * slot;
    uint32_t glog = seg_group_log2(nseg, 32);
    const uint32_t G = 1u << glog;
    const uint32_t gl = lane & (G - 1u);
    const uint32_t gmask = G >= 32 ? 0xFFFFFFFFu : (((1u << G) - 1u) << (lane & ~(G - 1u)));
    int err = 0;
    // all groups run the same number of rounds (the shuffles inside stay converged per group)
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
__device__ __noinline__ void ws_group_add(uint32_t gk, int64_t val, uint32_t* tkey, unsigned long long* tsum,
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

__global__ void __launch_bounds__(kWsNT, 2) warp_scan_kernel(const __grid_constant__ WsParams P) {
    extern __shared__ __align__(16) uint8_t smem[];
    __shared__ gx_dcol s_cols[kWsMaxCols];
    const uint32_t tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const uint32_t ncols = P.n_cols;
    if (tid < ncols * (sizeof(gx_dcol) / 4))
        ((uint32_t*)s_cols)[tid] = ((const uint32_t*)P.cols)[tid];
    __syncthreads();  // the only block-wide barrier: the column table is read-only from here on

    uint32_t* const wmem = (uint32_t*)smem + (size_t)warp * P.warp_words;
    uint4* const cslot = (uint4*)wmem;                       // kWsMaxCols broadcast slots (constant columns)
    uint32_t* const bufs = wmem + 4 * kWsMaxCols;            // n_bufs x kWsTile words
    uint32_t* const tkey = bufs + (size_t)P.n_bufs * kWsTile;  // group table: keys, then sums (8-byte aligned)
    unsigned long long* const tsum = (unsigned long long*)(tkey + kWsGroupSlots);
    if (P.grouped_tab) {
        for (uint32_t i = lane; i < kWsGroupSlots; i += 32) {
            tkey[i] = kEmptyGKey;
            tsum[i] = 0;
        }
    }
    __syncwarp();

    const ShQuery& Q = P.q;
    const uint32_t ns = Q.n_steps, agg = Q.agg;
    const bool grouped = Q.grouped != 0;
    const uint32_t tpb = P.tiles_per_block, bpc = P.blocks_per_chunk;
    const uint64_t PC = (uint64_t)bpc * tpb;  // tiles per chunk
    const uint64_t t_begin = (uint64_t)P.chunk_lo * PC, t_end = (uint64_t)P.chunk_hi * PC;
    const uint64_t W = (uint64_t)gridDim.x * kWsWarps;
    int64_t local = 0;
    unsigned long long local_rows = 0;

    for (uint64_t w = t_begin + (uint64_t)blockIdx.x * kWsWarps + warp; w < t_end; w += W) {
        const uint32_t chunk = (uint32_t)(w / PC), loc = (uint32_t)(w % PC);
        const uint32_t jb = loc / tpb, tile = loc % tpb;
        const uint32_t slot = chunk * bpc + jb;
        const uint64_t c_r0 = (uint64_t)chunk * P.rows_per_chunk;
        const uint64_t c_rows = min((uint64_t)P.rows_per_chunk, P.n_rows - c_r0);
        const uint64_t jrow = (uint64_t)jb * P.rows_per_block;
        const uint32_t rows = jrow < c_rows ? (uint32_t)min((uint64_t)P.rows_per_block, c_rows - jrow) : 0u;
        const uint32_t r0 = tile * kWsTile;
        // chunk keep (keep_in and the prune predicates' chunk min/max); the
        // warp of the chunk's first tile publishes it
        bool ck = Q.keep_in ? __ldg(Q.keep_in + chunk) != 0 : true;
        for (uint32_t p = 0; p < Q.n_prune; ++p) {
            const PrunePred& pr = Q.prune[p];
            ck = ck && pr.lo <= __ldg(pr.maxs + chunk) && pr.hi >= __ldg(pr.mins + chunk);
        }
        if (loc == 0 && lane == 0 && Q.keep_out) Q.keep_out[chunk] = ck ? 1 : 0;
        if (!ck || r0 >= rows) continue;
        const uint32_t n = min(kWsTile, rows - r0);
        const uint64_t g0 = c_r0 + jrow + r0;
        const uint32_t a = Q.row_lo > g0 ? (uint32_t)min((uint64_t)n, Q.row_lo - g0) : 0u;
        const uint32_t b = Q.row_hi > g0 ? (uint32_t)min((uint64_t)n, Q.row_hi - g0) : 0u;
        if (a >= b) continue;
        bool zk = true;
        for (uint32_t p = 0; p < Q.n_prune; ++p) {
            const PrunePred& pr = Q.prune[p];
            if (pr.bmins) zk = zk && pr.lo <= __ldg(pr.bmaxs + slot) && pr.hi >= __ldg(pr.bmins + slot);
        }
        if (!zk) continue;

        // ---- columns: lane c decides how column c is read
        uint32_t mode = kWmBad;
        const uint8_t* cptr = nullptr;   // direct: the tile's first row; casc: the page
        uint32_t aux0 = 0, aux1 = 0;     // LZ4: [lo, hi); casc: page bytes, page rows
        uint64_t blk_off = 0;
        uint32_t blk_bytes = 0;
        if (lane < ncols) {
            const gx_dcol& col = s_cols[lane];
            const uint4 dw = __ldg((const uint4*)(col.blocks + slot));
            const uint64_t d_off = ((uint64_t)dw.y << 32) | dw.x;
            const uint32_t d_bytes = dw.z, d_rows = dw.w;
            blk_off = d_off;
            blk_bytes = d_bytes;
            const bool dir_ok = d_rows == rows && d_off <= col.payload_bytes &&
                                (uint64_t)d_bytes + 32 <= col.payload_bytes - d_off;
            if (dir_ok && col.codec == GX_CODEC_NONE) {
                if (d_bytes == rows * 4 && (d_off & 15u) == 0) {
                    mode = kWmDirect;
                    cptr = col.payload + d_off + 4ull * r0;
                }
            } else if (dir_ok && col.codec == GX_CODEC_LZ4) {
                const uint32_t sr = 1u << col.seg_shift;
                const uint32_t j0 = r0 >> col.seg_shift, nseg = (n + sr - 1) >> col.seg_shift;
                if ((r0 & (sr - 1u)) == 0 && j0 + nseg <= col.S) {
                    const uint32_t* e = col.seg + (size_t)2 * col.S * slot;
                    const uint32_t e0 = __ldg(e + 2 * j0), e1 = __ldg(e + 2 * j0 + 1);
                    const uint32_t hi = j0 + nseg < col.S ? __ldg(e + 2 * (j0 + nseg)) : d_bytes;
                    if (e0 <= hi && hi <= d_bytes) {
                        const bool lit = (e1 & 16u) && (e1 >> 5) >= 4 * n && hi - e0 == 4 * n;
                        if (lit && ((d_off + e0) & 15u) == 0) {
                            mode = kWmDirect;
                            cptr = col.payload + d_off + e0;
                        } else if (P.buf_of[lane] != kWsNoBuf) {
                            mode = kWmLz4;
                            aux0 = e0;
                            aux1 = hi;
                        }
                    }
                }
            } else if (dir_ok && col.codec == GX_CODEC_CASCADED) {
                const uint32_t page = r0 >> kCascPageLog2;
                const uint32_t* e = col.seg + (size_t)2 * col.S * slot + 2 * page;
                const uint32_t po = __ldg(e), pb = __ldg(e + 1);
                if ((po & 15u) == 0 && (uint64_t)po + pb <= d_bytes && (d_off & 15u) == 0 &&
                    P.buf_of[lane] != kWsNoBuf && page < col.S) {
                    mode = kWmCasc;
                    cptr = col.payload + d_off + po;
                    aux0 = pb;
                    aux1 = min(kCascPageRows, rows - page * kCascPageRows);
                }
            }
            // in-place rows go to L2 now; the batches read them from there
        }
        if (__any_sync(0xFFFFFFFFu, lane < ncols && mode == kWmBad)) {
            if (lane == 0) raise_error(kErrCorrupt);
            continue;
        }
        for (uint32_t c = 0; c < ncols; ++c) {
            const uint32_t m = __shfl_sync(0xFFFFFFFFu, mode, c);
            if (m != kWmDirect) continue;
            const uint8_t* p = (const uint8_t*)ws_shfl64((uint64_t)cptr, c);
            if (lane * 128 < 4 * n) asm volatile("prefetch.global.L2 [%0];" ::"l"(p + lane * 128));
        }
        // decodes (one column at a time, the whole warp)
        int terr = 0;
        const uint8_t* rptr = cptr;  // lane c: where column c's rows are read
        uint32_t rmask = 0xFFFFFFFFu;
        for (uint32_t c = 0; c < ncols && !terr; ++c) {
            const uint32_t m = __shfl_sync(0xFFFFFFFFu, mode, c);
            if (m == kWmDirect) continue;
            uint32_t* buf = bufs + (size_t)P.buf_of[c] * kWsTile;
            const uint32_t x0 = __shfl_sync(0xFFFFFFFFu, aux0, c), x1 = __shfl_sync(0xFFFFFFFFu, aux1, c);
            int r;
            int32_t cv = 0;
            if (m == kWmCasc) {
                const uint8_t* pg = (const uint8_t*)ws_shfl64((uint64_t)cptr, c);
                r = ws_casc_rows(pg, x0, x1, r0 & (kCascPageRows - 1u), n, (int32_t*)buf, &cv, lane);
            } else {
                const uint64_t bo = ws_shfl64(blk_off, c);
                const uint32_t bb = __shfl_sync(0xFFFFFFFFu, blk_bytes, c);
                r = ws_lz4_rows(s_cols[c], slot, bo, bb, rows, r0, n, x0, x1, buf, lane);
            }
            if (r == 1) {  // one value for the whole tile
                if (lane == 0) cslot[c] = make_uint4((uint32_t)cv, (uint32_t)cv, (uint32_t)cv, (uint32_t)cv);
                if (lane == c) {
                    rptr = (const uint8_t*)&cslot[c];
                    rmask = 0;
                }
            } else if (r) {
                terr = r;
            } else if (lane == c) {
                rptr = (const uint8_t*)buf;
            }
        }
        __syncwarp();
        if (terr) {
            if (lane == 0) raise_error(terr);
            continue;
        }
        local_rows += b - a;  // lane-uniform; counted once per warp below

        // ---- evaluation
        const uint8_t* sp[GX_MAX_STEPS];
        uint32_t sm[GX_MAX_STEPS];
#pragma unroll
        for (uint32_t s = 0; s < GX_MAX_STEPS; ++s) {
            if (s < ns) {
                const uint32_t c = Q.steps[s].col;
                sp[s] = (const uint8_t*)ws_shfl64((uint64_t)rptr, c);
                sm[s] = __shfl_sync(0xFFFFFFFFu, rmask, c);
            }
        }
        for (uint32_t rb = 0; rb < n; rb += kWsBatch) {
            const uint32_t r_first = rb + lane * 4;
            uint4 vals[GX_MAX_STEPS];
#pragma unroll
            for (uint32_t s = 0; s < GX_MAX_STEPS; ++s)
                if (s < ns)
                    vals[s] = r_first < n ? *(const uint4*)(sp[s] + ((r_first * 4) & sm[s])) : make_uint4(0, 0, 0, 0);
            uint32_t keep = 0;
#pragma unroll
            for (uint32_t i = 0; i < 4; ++i) keep |= (r_first + i >= a && r_first + i < b) ? 1u << i : 0u;
            uint32_t gk[4] = {0, 0, 0, 0};
            int32_t carry[4] = {0, 0, 0, 0};
#pragma unroll
            for (uint32_t s = 0; s < GX_MAX_STEPS; ++s) {
                if (s >= ns || !__any_sync(0xFFFFFFFFu, keep)) break;
                const ShStep& stp = Q.steps[s];
                const uint32_t flags = stp.flags, dcard = stp.digit_card;
                const int32_t lo = stp.lo, hi = stp.hi, dbase = stp.digit_base;
                const bool last = s + 1 == ns;
                const bool filt = (flags & GX_STEP_FILTER) != 0, carry_step = (flags & GX_STEP_CARRY) != 0;
                const bool probe = (flags & GX_STEP_PROBE) != 0;
                const int32_t v[4] = {(int32_t)vals[s].x, (int32_t)vals[s].y, (int32_t)vals[s].z, (int32_t)vals[s].w};
                uint32_t kk = keep;
                if (filt) {
#pragma unroll
                    for (uint32_t i = 0; i < 4; ++i)
                        if (!(v[i] >= lo && v[i] <= hi)) kk &= ~(1u << i);
                }
                int32_t pp[4] = {v[0], v[1], v[2], v[3]};
                if (probe) {
                    const uint64_t* const ht = stp.ht;
                    const uint32_t htlog = stp.ht_log2, htlay = stp.ht_layout;
                    if (htlay == GX_HT_BUCKET) {
                        int32_t mv = kEmptyKey, mp = 0;
                        bool mk = false;
#pragma unroll
                        for (uint32_t i = 0; i < 4; ++i) {
                            if (!((kk >> i) & 1u)) continue;
                            if (v[i] != mv || i == 0) {
                                mp = v[i];
                                mk = sh_probe(ht, htlog, htlay, v[i], &mp);
                                mv = v[i];
                            }
                            pp[i] = mp;
                            if (!mk) kk &= ~(1u << i);
                        }
                    } else {
                        // first-slot reads of the lane's distinct keys, all issued before use
                        const bool dense = htlay == GX_HT_DENSE;
                        uint32_t hbase = 0, hspan = 0;
                        if (dense) {
                            const uint64_t hdr = __ldg((const unsigned long long*)ht);
                            hbase = (uint32_t)hdr;
                            hspan = (uint32_t)(hdr >> 32);
                        }
                        uint64_t ee[4];
                        uint32_t rd = 0;
                        const uint32_t kf = kk;  // rows kept up to the probe
#pragma unroll
                        for (uint32_t i = 0; i < 4; ++i) {
                            const bool again = i > 0 && v[i] == v[i - 1] && ((kf >> (i - 1)) & 1u);
                            const uint32_t u = (uint32_t)v[i] - hbase;
                            const bool r = ((kk >> i) & 1u) && !again && v[i] != kEmptyKey && (!dense || u < hspan);
                            const unsigned long long* slotp =
                                (const unsigned long long*)ht + (dense ? 1 + u : hash_key32(v[i], htlog));
                            ee[i] = r ? __ldg(slotp) : (unsigned long long)kEmptySlot;
                            rd |= r ? 1u << i : 0u;
                        }
                        bool pf = false;  // the previous kept row's key was found
                        int32_t pv = 0;
#pragma unroll
                        for (uint32_t i = 0; i < 4; ++i) {
                            if (!((kk >> i) & 1u)) continue;
                            const bool again = i > 0 && v[i] == v[i - 1] && ((kf >> (i - 1)) & 1u);
                            bool f;
                            int32_t p = v[i];
                            if (again) {
                                f = pf;
                                p = pv;
                            } else if (!((rd >> i) & 1u)) {
                                f = false;
                            } else {
                                const int32_t ek = (int32_t)(uint32_t)ee[i];
                                if (ek == v[i]) {
                                    f = true;
                                    p = (int32_t)(uint32_t)(ee[i] >> 32);
                                } else if (dense || ek == kEmptyKey) {
                                    f = false;
                                } else {
                                    f = sh_probe(ht, htlog, htlay, v[i], &p);
                                }
                            }
                            pf = f;
                            pv = p;
                            pp[i] = p;
                            if (!f) kk &= ~(1u << i);
                        }
                    }
                }
                if (dcard) {
#pragma unroll
                    for (uint32_t i = 0; i < 4; ++i) {
                        if (!((kk >> i) & 1u)) continue;
                        const uint32_t dgt = (uint32_t)(pp[i] - dbase);
                        if (dgt >= dcard) {
                            raise_error(kErrInvalid);
                            kk &= ~(1u << i);
                        } else {
                            gk[i] = gk[i] * dcard + dgt;
                        }
                    }
                }
                if (carry_step) {
#pragma unroll
                    for (uint32_t i = 0; i < 4; ++i) carry[i] = v[i];
                }
                keep = kk;
                if (last) {
#pragma unroll
                    for (uint32_t i = 0; i < 4; ++i) {
                        const bool k = (kk >> i) & 1u;
                        const int64_t val = agg == GX_AGG_SUM_PRODUCT ? (int64_t)v[i] * carry[i]
                                            : agg == GX_AGG_SUM_DIFF  ? (int64_t)v[i] - carry[i]
                                            : agg == GX_AGG_COUNT      ? 1
                                                                       : (int64_t)v[i];
                        if (!grouped) {
                            local += k ? val : 0;
                        } else if (k) {
                            if (P.grouped_tab)
                                ws_group_add(gk[i], val, tkey, tsum, Q.g_keys, Q.g_sums, Q.g_log2);
                            else if (!group_add_global(Q.g_keys, Q.g_sums, Q.g_log2, (int64_t)gk[i], val))
                                raise_error(kErrCapacity);
                        }
                    }
                }
            }
        }
        __syncwarp();
    }
    // ---- the warp's results
    if (grouped && P.grouped_tab) {
        __syncwarp();
        for (uint32_t i = lane; i < kWsGroupSlots; i += 32) {
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
