// pipe_scan.cuh -- the one-query fused scan as a warp-specialised pipeline
// (device side; included by kernels.cu inside its anonymous namespace after
// shared_scan.cuh, whose query descriptor and evaluation helpers it uses).
//
// Replaces, for one query: ChunkDecompressor::step (core/comp.cuh:171-195)
// feeding pipeline_q1_lineorder (usecases/ssb/queries/01.cuh:27-54) or
// pipeline_q3 (usecases/ssb/queries/03.cuh:119-170), with the chunk pruning of
// MetaChecker (core/metadata.cuh:638-658) and the per-chunk worker loop of
// usecases/ssb/queries/01.hpp:350-424 folded into the same launch.
//
// One CTA per SM: kPipeNC consumer threads (warps 0..15) and one producer
// warp (warp 16).
//
// Producer.  Walks this CTA's share of the row tiles (tile w of the table
// goes to CTA w mod grid): per group of 32 chunks one round of loads decides
// which chunks survive min/max pruning (keep_in and every prune predicate;
// CTA 0 writes keep_out), then the CTA's candidate tiles of the surviving
// chunks are checked 32 at a time, one per lane, with every load the check
// and the staging need (directory entries of all columns, the tile's segment
// or page entries, zone maps) issued together.  For every live tile it waits
// until a ring slot is free, writes the tile's descriptor into the slot and
// issues one cp.async.bulk per column (no multicast) of the tile's bytes --
// a literal run, a compressed LZ4 range, a cascaded page or raw rows -- all
// completing on the slot's "full" mbarrier.  Tiles are issued in order; an
// end marker follows the last one.
//
// Consumers.  Per tile: wait for the slot's full barrier (thread 0, bounded,
// then a barrier of the consumer warps so the decision is uniform); decode
// what is not already rows -- a cascaded page, an LZ4 range with matches, a
// literal run that is not 4-byte aligned -- into the column's decode buffer;
// literal and raw tiles are read in place from the ring; then the plan's
// steps run step-major over the thread's 4 rows (the evaluation of
// shared_scan_kernel for one query); the slot is released (the "empty"
// mbarrier) once every consumer is past the tile.  Scalar sums stay in
// registers until the end of the launch; grouped sums go to a CTA group table
// in shared memory that persists across tiles and is flushed into the global
// table at the end, or earlier when it is half full.
//
// No wait is unbounded: mbarrier waits give up after kMbarWaitCap tries of at
// most 1 us, raise GX_ERR_TIMEOUT and stop the CTA (the producer then waits,
// again bounded, for the copies it issued before it leaves).

constexpr uint32_t kPipeNC = 512;                  // consumer threads
constexpr uint32_t kPipeNW = kPipeNC / 32;         // consumer warps
constexpr uint32_t kPipeNT = kPipeNC + 32;         // + the producer warp
constexpr uint32_t kPipeTile = kShTile;            // 2048 rows
constexpr uint32_t kPipeRPT = kPipeTile / kPipeNC; // rows per consumer thread
constexpr uint32_t kPipeColBytes = 8512;           // one column of one tile: 8 KiB of rows + LZ4 overhead + alignment
constexpr uint32_t kPipeMaxStages = 6;
constexpr uint32_t kPipeMaxCols = GX_MAX_STEPS;
constexpr uint32_t kPipeBar = 1;                   // named barrier of the consumer warps
constexpr uint32_t kPipeMaxDynSmem = 216u << 10;   // dynamic shared memory (the static part is ~10.5 KiB)
static_assert(kPipeColBytes % 16 == 0, "ring areas stay 16-byte aligned");
static_assert(32 + 4 * (kCascPageRows + 4) <= kPipeColBytes, "a cascaded page of 32-bit values fits one area");
static_assert(4 * kPipeTile + 4 * kPipeTile / 255 + 64 <= kPipeColBytes, "a tile's LZ4 range fits one area");

enum : uint8_t { kPcPlain = 0, kPcLz4 = 1, kPcCasc = 2, kPcShift = 3, kPcBad = 4 };

// One column of a staged tile (16 bytes).
struct PipeCol {
    uint8_t kind;   // kPc*
    uint8_t pad_;
    uint16_t off;   // byte offset in the column's ring area of the tile's first byte (plain: first row; LZ4: byte lo)
    uint32_t lo;    // LZ4: the tile's first compressed byte in the block
    uint32_t hi;    // LZ4: one past its last byte; cascaded: page bytes
    uint32_t end;   // LZ4: the block's compressed size
};
static_assert(sizeof(PipeCol) == 16, "PipeCol layout");

// Descriptor of one staged tile (written by the producer, read by consumers
// after the slot's full barrier).
struct PipeTile {
    uint32_t slot, r0, n, rows;  // block slot, first row in the block, tile rows, block rows
    uint32_t a, b;               // rows [a, b) of the tile lie in the query's slice
    uint32_t end;                // 1: end of this CTA's work
    uint32_t pad_;
    PipeCol col[kPipeMaxCols];
};
static_assert(sizeof(PipeTile) % 16 == 0, "PipeTile layout");

struct PipeParams {
    ShQuery q;                      // steps index into cols
    gx_dcol cols[kPipeMaxCols];
    uint32_t n_cols;
    uint32_t stages;
    uint32_t n_chunks, blocks_per_chunk, rows_per_chunk, rows_per_block;
    uint32_t tile_rows, tiles_per_block;
    uint64_t n_rows;                // rows of the table
    uint32_t dec_mask;              // columns with a decode buffer (LZ4, cascaded)
    uint32_t gt_slots;              // CTA group-table slots (grouped queries) or 0
    unsigned long long* rows_scanned;
    // GX_AGG_BUILD: the join table the surviving rows are inserted into
    uint64_t* build_slots;
    unsigned long long* build_counters;  // inserted, duplicates, dropped
    uint32_t build_log2, build_layout;
    uint32_t build_rowid;           // 1: the payload is the table row (no CARRY step)
    uint32_t chunk_lo, chunk_hi;    // chunks [chunk_lo, chunk_hi) are scanned (a streamed group, or all)
};

// One insert of a GX_AGG_BUILD plan into a linear or bucket join table
// (layouts of include/gx_hash.h): 0 inserted, 1 duplicate key (the first
// insert wins), 2 no slot or the reserved key.
__device__ __forceinline__ uint32_t pipe_ht_insert(uint64_t* slots, uint32_t log2cap, uint32_t layout, int32_t key,
                                                   int32_t pay) {
    if (key == kEmptyKey) return 2;
    const unsigned long long e = ((unsigned long long)(uint32_t)pay << 32) | (uint32_t)key;
    if (layout == GX_HT_BUCKET) {
        const uint32_t lb = log2cap - 3, bmask = (1u << lb) - 1;
        uint32_t bkt = hash_key32(key, lb);
        for (uint32_t t = 0; t <= bmask; ++t) {
            unsigned long long* bp = (unsigned long long*)slots + (size_t)bkt * kBucketSlots;
            for (uint32_t j = 0; j < kBucketSlots; ++j) {
                const unsigned long long old = atomicCAS(bp + j, (unsigned long long)kEmptySlot, e);
                if (old == (unsigned long long)kEmptySlot) return 0;
                if ((int32_t)(uint32_t)old == key) return 1;
            }
            bkt = (bkt + 1) & bmask;
        }
        return 2;
    }
    const uint32_t mask = (1u << log2cap) - 1;
    uint32_t sl = hash_key32(key, log2cap);
    for (uint32_t t = 0; t <= mask; ++t) {
        const unsigned long long old = atomicCAS((unsigned long long*)slots + sl, (unsigned long long)kEmptySlot, e);
        if (old == (unsigned long long)kEmptySlot) return 0;
        if ((int32_t)(uint32_t)old == key) return 1;
        sl = (sl + 1) & mask;
    }
    return 2;
}

__device__ __forceinline__ void mbar_arrive(uint64_t* m) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(m)) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx_arrive(uint64_t* m, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(m)), "r"(bytes) : "memory");
}
// One bulk copy completing on m (its bytes are announced by the slot's single
// expect_tx arrival).
__device__ __forceinline__ void bulk_copy_1d(void* dst, const void* src, uint32_t bytes, uint64_t* m) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                 ::"r"(smem_u32(dst)), "l"(src), "r"(bytes), "r"(smem_u32(m))
                 : "memory");
}

__device__ __forceinline__ void pipe_sync() { grp_sync<kPipeNC, kPipeBar>(); }

// Bounded wait for a phase that also gives up as soon as the other side of
// the pipeline has stopped (*abort set).
__device__ __forceinline__ bool mbar_wait_or_abort(uint64_t* m, uint32_t phase, const volatile int* abort) {
    for (uint32_t i = 0; i < kMbarWaitCap; ++i) {
        if (mbar_try_wait_sleep(m, phase, 1000u)) return true;
        if (*abort) return false;
    }
    return false;
}

// Named-barrier OR-vote of the consumer warps.
__device__ __forceinline__ bool pipe_any(bool p) {
    uint32_t r;
    asm volatile(
        "{\n .reg .pred a, b;\n setp.ne.u32 a, %1, 0;\n bar.red.or.pred b, %2, %3, a;\n selp.u32 %0, 1, 0, b;\n}"
        : "=r"(r)
        : "r"((uint32_t)p), "n"(kPipeBar), "n"(kPipeNC)
        : "memory");
    return r != 0;
}

// Chunk-level keep of the query (keep_in and every prune predicate's chunk
// min/max: the reference's pruning granularity).
__device__ __forceinline__ bool pipe_chunk_keep(const ShQuery& Q, uint32_t chunk) {
    bool ck = Q.keep_in ? __ldg(Q.keep_in + chunk) != 0 : true;
    for (uint32_t p = 0; p < Q.n_prune; ++p) {
        const PrunePred& pr = Q.prune[p];
        const int32_t mx = __ldg(pr.maxs + chunk), mn = __ldg(pr.mins + chunk);
        ck = ck && pr.lo <= mx && pr.hi >= mn;
    }
    return ck;
}

// Add of (gk, val) to the CTA's persistent group table (one query: the table
// is flushed only at the end of the launch or when half full); a key that
// finds no slot within kShGroupProbes goes to the global table directly.
// *fill counts claimed slots.
__device__ __noinline__ void pipe_group_add(uint32_t gk, int64_t val, unsigned long long* tsum, uint32_t* tkey,
                                            uint32_t* fill, int64_t* keys, int64_t* sums, uint32_t log2cap) {
    if (gk != kEmptyGKey) {
        uint32_t s = hash_key32((int32_t)gk, kShGroupLog2);
        for (uint32_t i = 0; i < kShGroupProbes; ++i) {
            uint32_t cur = ((volatile uint32_t*)tkey)[s];
            if (cur == kEmptyGKey) {
                cur = atomicCAS(&tkey[s], kEmptyGKey, gk);
                if (cur == kEmptyGKey) atomicAdd(fill, 1u);
            }
            if (cur == kEmptyGKey || cur == gk) {
                atomicAdd(&tsum[s], (unsigned long long)val);
                return;
            }
            s = (s + 1) & (kShGroupSlots - 1);
        }
    }
    if (!group_add_global(keys, sums, log2cap, (int64_t)gk, val)) raise_error(kErrCapacity);
}

// Flush of the CTA group table into the global one (consumer warps, between
// named barriers); leaves it empty.
__device__ __forceinline__ void pipe_group_flush(unsigned long long* tsum, uint32_t* tkey, uint32_t* fill,
                                                 int64_t* keys, int64_t* sums, uint32_t log2cap, uint32_t tid) {
    pipe_sync();
    for (uint32_t j = tid; j < kShGroupSlots; j += kPipeNC) {
        const uint32_t key = tkey[j];
        if (key != kEmptyGKey) {
            if (!group_add_global(keys, sums, log2cap, (int64_t)key, (int64_t)tsum[j])) raise_error(kErrCapacity);
            tkey[j] = kEmptyGKey;
            tsum[j] = 0;
        }
    }
    if (tid == 0) *fill = 0;
    pipe_sync();
}

// LZ4 range with matches of column c of a staged tile, decoded segment by
// segment into buf (groups of G lanes per segment, as in decode_tile); the
// tile's segment entries are read from the side index.  Returns the
// per-segment pad (log2 words) or -1 after recording kErrCorrupt in *s_err.
__device__ __forceinline__ int pipe_lz4_tile(const gx_dcol& c, const PipeTile& T, const PipeCol& pc,
                                             const uint8_t* area, uint32_t* buf, uint32_t* s_seg, int* s_err,
                                             uint32_t tid) {
    const uint32_t seg_rows = 1u << c.seg_shift;
    const uint32_t j0 = T.r0 >> c.seg_shift, nseg = (T.n + seg_rows - 1) >> c.seg_shift;
    const uint32_t* e = c.seg + (size_t)2 * c.S * T.slot;
    for (uint32_t t = tid; t <= nseg && t <= kMaxSegments; t += kPipeNC) {
        const uint32_t j = j0 + t;
        s_seg[2 * t] = j < c.S ? __ldg(e + 2 * j) : pc.end;
        s_seg[2 * t + 1] = j < c.S ? __ldg(e + 2 * j + 1) : 0u;
    }
    pipe_sync();
    if (nseg > kMaxSegments || s_seg[0] != pc.lo || s_seg[2 * nseg] != pc.hi) {
        if (tid == 0) *s_err = kErrCorrupt;
        return -1;
    }
    const uint32_t wbase = pc.lo - pc.off;  // block-relative position of the area's first byte (wrapping)
    const bool literal_tile = (uint64_t)(pc.hi - pc.lo) * 8 >= (uint64_t)T.n * 4 * 7;
    uint32_t glog = literal_tile ? 5u : seg_group_log2(nseg, kPipeNC);
    while (glog > 0 && glog < 5 && (nseg << glog) > 256u) --glog;
    const uint32_t G = 1u << glog;
    const uint32_t pl = glog == 5 ? 0u : glog;
    const uint32_t gl = tid & (G - 1u), lane = tid & 31u;
    const uint32_t gmask = G >= 32 ? 0xFFFFFFFFu : (((1u << G) - 1u) << (lane & ~(G - 1u)));
    for (uint32_t t = tid >> glog; t < nseg; t += (kPipeNC >> glog)) {
        const uint32_t j = j0 + t;
        const uint32_t K = min(seg_rows, T.rows - j * seg_rows);
        const int r2 = lz4_seg_group((const uint32_t*)area, wbase, pc.lo, pc.hi, pc.end, s_seg[2 * t],
                                     s_seg[2 * t + 1], K, buf + t * (seg_rows + (1u << pl)), gl, G, gmask);
        if (r2 && gl == 0) *s_err = r2;
    }
    return (int)pl;
}

__global__ void __launch_bounds__(kPipeNT, 1) pipe_scan_kernel(const __grid_constant__ PipeParams P) {
    constexpr uint32_t NW = kPipeNW, RPT = kPipeRPT;
    extern __shared__ __align__(16) uint8_t smem[];
    __shared__ __align__(8) uint64_t s_full[kPipeMaxStages], s_empty[kPipeMaxStages];
    __shared__ __align__(16) PipeTile s_desc[kPipeMaxStages];
    __shared__ __align__(16) PipeTile s_cand[32];      // producer: the round's candidate descriptors
    __shared__ const uint8_t* s_csrc[32][kPipeMaxCols];  // producer: their copy sources
    __shared__ uint32_t s_cbytes[32][kPipeMaxCols];      // producer: their copy sizes
    __shared__ uint32_t s_tmp[NW + 1];
    __shared__ uint32_t s_seg[2 * (kMaxSegments + 1)];
    __shared__ const uint32_t* s_cptr[kPipeMaxCols];
    __shared__ uint32_t s_csh[kPipeMaxCols], s_cpd[kPipeMaxCols];
    __shared__ int s_err, s_ok, s_abort;
    __shared__ uint32_t s_gfill;

    const uint32_t tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const uint32_t S = P.stages, ncols = P.n_cols;
    uint8_t* const ring = smem;
    uint32_t* const decbuf = (uint32_t*)(smem + (size_t)S * ncols * kPipeColBytes);
    const uint32_t n_dec = __popc(P.dec_mask);
    int32_t* const run_val = (int32_t*)(decbuf + (size_t)n_dec * kShColWords);
    uint32_t* const run_end = (uint32_t*)(run_val + kCascPageMaxRuns);
    unsigned long long* const s_gsum = (unsigned long long*)(run_end + kCascPageMaxRuns);
    uint32_t* const s_gkey = (uint32_t*)(s_gsum + P.gt_slots);

    if (tid == 0) {
        for (uint32_t i = 0; i < S; ++i) {
            mbar_init(&s_full[i], 1);
            mbar_init(&s_empty[i], 1);
        }
        s_err = 0;
        s_ok = 1;
        s_abort = 0;
        s_gfill = 0;
    }
    for (uint32_t i = tid; i < P.gt_slots; i += kPipeNT) {
        s_gsum[i] = 0;
        s_gkey[i] = kEmptyGKey;
    }
    __syncthreads();

    if (warp == NW) {
        // ------------------------------------------------------------ producer
        const ShQuery& Q = P.q;
        const uint32_t G = gridDim.x, b = blockIdx.x;
        const uint32_t tpb = P.tiles_per_block, bpc = P.blocks_per_chunk, tile_rows = P.tile_rows;
        const uint32_t PC = bpc * tpb;                // candidates per chunk
        const uint32_t K = (PC + G - 1) / G;          // most candidates of one CTA in one chunk
        uint32_t k = 0;                               // tiles issued
        bool abort = false;
        for (uint32_t cb = P.chunk_lo; cb < P.chunk_hi && !abort; cb += 32) {
            const uint32_t cc = cb + lane;
            bool ck = false;
            if (cc < P.chunk_hi) {
                ck = pipe_chunk_keep(Q, cc);
                if (b == 0 && Q.keep_out) Q.keep_out[cc] = ck ? 1 : 0;
            }
            const uint32_t live = __ballot_sync(0xFFFFFFFFu, ck);
            const uint32_t npairs = __popc(live) * K;
            for (uint32_t p0 = 0; p0 < npairs && !abort; p0 += 32) {
                // candidate p = (i-th surviving chunk of the group, j-th tile of this CTA in it)
                const uint32_t p = p0 + lane;
                bool have = false;
                uint32_t slot = 0, tile = 0, chunk = 0;
                if (p < npairs) {
                    const uint32_t i = p / K, j = p % K;
                    uint32_t m = live;
                    for (uint32_t t = 0; t < i; ++t) m &= m - 1;
                    chunk = cb + (__ffs(m) - 1);
                    const uint64_t base = (uint64_t)chunk * PC;
                    const uint32_t j0 = (uint32_t)((b + G - (uint32_t)(base % G)) % G);
                    const uint32_t loc = j0 + j * G;
                    if (loc < PC) {
                        slot = chunk * bpc + loc / tpb;
                        tile = loc % tpb;
                        have = true;
                    }
                }
                // rows of the block from the layout (no dependent load)
                uint32_t rows = 0, r0 = tile * tile_rows, n = 0;
                if (have) {
                    const uint64_t c_r0 = (uint64_t)chunk * P.rows_per_chunk;
                    const uint64_t c_rows = min((uint64_t)P.rows_per_chunk, P.n_rows - c_r0);
                    const uint64_t jb = (uint64_t)(slot - chunk * bpc) * P.rows_per_block;
                    rows = jb < c_rows ? (uint32_t)min((uint64_t)P.rows_per_block, c_rows - jb) : 0u;
                    have = r0 < rows;
                    n = have ? min(tile_rows, rows - r0) : 0u;
                }
                // the query's slice and the block zone maps
                uint32_t a = 0, bb = n;
                if (have) {
                    const uint64_t g0 = (uint64_t)chunk * P.rows_per_chunk +
                                        (uint64_t)(slot - chunk * bpc) * P.rows_per_block + r0;
                    a = Q.row_lo > g0 ? (uint32_t)min((uint64_t)n, Q.row_lo - g0) : 0u;
                    bb = Q.row_hi > g0 ? (uint32_t)min((uint64_t)n, Q.row_hi - g0) : 0u;
                    have = a < bb;
                    for (uint32_t q = 0; have && q < Q.n_prune; ++q) {
                        const PrunePred& pr = Q.prune[q];
                        if (pr.bmins) have = pr.lo <= __ldg(pr.bmaxs + slot) && pr.hi >= __ldg(pr.bmins + slot);
                    }
                }
                // staging of every column: directory entry, then the tile's byte range
                if (have) {
                    PipeTile& T = s_cand[lane];
                    T.slot = slot;
                    T.r0 = r0;
                    T.n = n;
                    T.rows = rows;
                    T.a = a;
                    T.b = bb;
                    T.end = 0;
                    T.pad_ = 0;
#pragma unroll
                    for (uint32_t c = 0; c < kPipeMaxCols; ++c) {
                        if (c >= ncols) break;
                        const gx_dcol& col = P.cols[c];
                        const gx_dblock d = col.blocks[slot];
                        uint32_t e0 = 0, e1 = 0, e2 = 0;
                        const bool lz = col.codec == GX_CODEC_LZ4, cs = col.codec == GX_CODEC_CASCADED;
                        uint32_t j0 = 0, nseg = 0;
                        if (lz) {
                            j0 = r0 >> col.seg_shift;
                            nseg = (n + (1u << col.seg_shift) - 1) >> col.seg_shift;
                            const uint32_t* e = col.seg + (size_t)2 * col.S * slot;
                            e0 = __ldg(e + 2 * j0);
                            e1 = __ldg(e + 2 * j0 + 1);
                            e2 = j0 + nseg < col.S ? __ldg(e + 2 * (j0 + nseg)) : 0u;
                        } else if (cs) {
                            const uint32_t* e = col.seg + (size_t)2 * col.S * slot + 2 * (r0 >> kCascPageLog2);
                            e0 = __ldg(e);
                            e1 = __ldg(e + 1);
                        }
                        PipeCol pc{kPcBad, 0, 0, 0, 0, 0};
                        const uint8_t* src = nullptr;
                        uint32_t bytes = 0;
                        const bool dir_ok = d.n_rows == rows && d.offset <= col.payload_bytes &&
                                            (uint64_t)d.comp_bytes + 32 <= col.payload_bytes - d.offset;
                        if (dir_ok && col.codec == GX_CODEC_NONE) {
                            if (d.comp_bytes == rows * 4 && (d.offset & 15u) == 0) {
                                src = col.payload + d.offset + 4ull * r0;
                                bytes = (4 * n + 15u) & ~15u;
                                pc.kind = kPcPlain;
                            }
                        } else if (dir_ok && lz) {
                            const uint32_t lo = e0, hi = j0 + nseg < col.S ? e2 : d.comp_bytes;
                            const uint64_t abs_lo = d.offset + lo, abs_wb = abs_lo & ~15ull;
                            const uint64_t nb = ((d.offset + hi + 15u) & ~15ull) - abs_wb + 16u;
                            if (lo <= hi && hi <= d.comp_bytes && nb <= kPipeColBytes &&
                                (r0 & ((1u << col.seg_shift) - 1u)) == 0 && j0 + nseg <= col.S) {
                                src = col.payload + abs_wb;
                                bytes = (uint32_t)nb;
                                pc.off = (uint16_t)(abs_lo - abs_wb);
                                pc.lo = lo;
                                pc.hi = hi;
                                pc.end = d.comp_bytes;
                                const bool lit = (e1 & 16u) && (e1 >> 5) >= 4 * n && hi - lo == 4 * n;
                                pc.kind = lit ? ((pc.off & 3u) ? kPcShift : kPcPlain) : kPcLz4;
                            }
                        } else if (dir_ok && cs) {
                            if ((e0 & 15u) == 0 && (uint64_t)e0 + e1 <= d.comp_bytes && e1 <= kPipeColBytes &&
                                (d.offset & 15u) == 0 && (r0 & (kCascPageRows - 1)) == 0) {
                                src = col.payload + d.offset + e0;
                                bytes = (e1 + 15u) & ~15u;
                                pc.kind = kPcCasc;
                                pc.hi = e1;
                            }
                        }
                        T.col[c] = pc;
                        s_csrc[lane][c] = src;
                        s_cbytes[lane][c] = bytes;
                    }
                }
                __syncwarp();
                // issue the live candidates in lane order
                uint32_t lm = __ballot_sync(0xFFFFFFFFu, have);
                while (lm && !abort) {
                    const uint32_t L = __ffs(lm) - 1;
                    lm &= lm - 1;
                    const uint32_t st = k % S;
                    int ok = 1;
                    if (lane == 0) {
                        if (k >= S) ok = mbar_wait_or_abort(&s_empty[st], ((k / S) - 1) & 1u, &s_abort);
                    }
                    ok = __shfl_sync(0xFFFFFFFFu, ok, 0);
                    if (!ok) {
                        abort = true;
                        break;
                    }
                    // the warp copies the descriptor into the slot (a word per lane) and
                    // lane c issues column c's copy, after lane 0 announced the bytes
                    {
                        const uint32_t* from = (const uint32_t*)&s_cand[L];
                        uint32_t* to = (uint32_t*)&s_desc[st];
                        for (uint32_t w = lane; w < sizeof(PipeTile) / 4; w += 32) to[w] = from[w];
                    }
                    const uint32_t cbytes = lane < ncols ? s_cbytes[L][lane] : 0u;
                    const uint32_t total = __reduce_add_sync(0xFFFFFFFFu, cbytes);
                    __syncwarp();
                    if (lane == 0) {
                        fence_proxy_async_smem();
                        mbar_expect_tx_arrive(&s_full[st], total);
                    }
                    __syncwarp();
                    if (cbytes)
                        bulk_copy_1d(ring + ((size_t)st * ncols + lane) * kPipeColBytes, s_csrc[L][lane], cbytes,
                                     &s_full[st]);
                    __syncwarp();
                    ++k;
                }
            }
        }
        // end marker
        if (!abort) {
            const uint32_t st = k % S;
            int ok = 1;
            if (k >= S && lane == 0) ok = mbar_wait_or_abort(&s_empty[st], ((k / S) - 1) & 1u, &s_abort);
            ok = __shfl_sync(0xFFFFFFFFu, ok, 0);
            if (ok) {
                if (lane == 0) {
                    s_desc[st].end = 1;
                    mbar_arrive(&s_full[st]);
                }
            } else {
                abort = true;
            }
        }
        if (abort) {
            // the consumers stopped (or will): tell them, then wait (bounded) for
            // the copies this warp issued before leaving the shared memory
            if (lane == 0) {
                raise_error(kErrTimeout);
                s_abort = 1;
                const uint32_t first = k > S ? k - S : 0;
                for (uint32_t t = first; t < k; ++t) mbar_wait_bounded(&s_full[t % S], (t / S) & 1u);
            }
        }
        return;
    }

    // ------------------------------------------------------------- consumers
    const ShQuery& Q = P.q;
    int64_t local = 0;
    unsigned long long local_rows = 0;
    const bool grouped = Q.grouped != 0;
    const uint32_t agg = Q.agg;
    uint32_t b_ins = 0, b_dup = 0, b_bad = 0;  // GX_AGG_BUILD counters of this thread
    for (uint32_t k = 0;; ++k) {
        const uint32_t st = k % S, ph = (k / S) & 1u;
        if (tid == 0) s_ok = mbar_wait_or_abort(&s_full[st], ph, &s_abort);
        pipe_sync();
        if (!s_ok) {
            if (tid == 0) {
                raise_error(kErrTimeout);
                s_abort = 1;
            }
            break;
        }
        mbar_try_wait(&s_full[st], ph);  // completes at once: this thread's acquire of the staged bytes
        const PipeTile& T = s_desc[st];
        if (T.end) break;
        const uint32_t n = T.n;
        // columns: plain rows in place, else decoded into the column's buffer
        if (tid < ncols) {
            const PipeCol pc = T.col[tid];
            if (pc.kind == kPcPlain || pc.kind == kPcBad) {  // decoded columns: set below by thread 0
                s_cptr[tid] = (const uint32_t*)(ring + ((size_t)st * ncols + tid) * kPipeColBytes + pc.off);
                s_csh[tid] = 31u;
                s_cpd[tid] = 0u;
            }
            if (pc.kind == kPcBad) atomicCAS(&s_err, 0, kErrCorrupt);
        }
        uint32_t dslot = 0;
        bool decoded = false;  // a decode ran since the last barrier (its scratch must not be reused yet)
        for (uint32_t c = 0; c < ncols; ++c) {
            const bool has_buf = (P.dec_mask >> c) & 1u;
            uint32_t* buf = decbuf + (size_t)dslot * kShColWords;
            dslot += has_buf ? 1u : 0u;
            const PipeCol pc = T.col[c];
            if (pc.kind == kPcPlain || pc.kind == kPcBad) continue;
            const uint8_t* area = ring + ((size_t)st * ncols + c) * kPipeColBytes;
            if (!has_buf) {
                if (tid == 0) s_err = kErrCorrupt;
                continue;
            }
            if (decoded) pipe_sync();  // the previous decode's run tables / segment entries are free again
            decoded = true;
            if (pc.kind == kPcCasc) {
                const int rc = casc_decode_page<kPipeNC, kPipeBar, false>(area, pc.hi, n, (int32_t*)buf, run_val,
                                                                          run_end, s_tmp, tid);
                if (tid == 0) {
                    if (rc) s_err = rc;
                    s_cptr[c] = buf;
                    s_csh[c] = 31u;
                    s_cpd[c] = 0u;
                }
            } else if (pc.kind == kPcShift) {
                const uint32_t* A = (const uint32_t*)area;
                const uint32_t w0 = pc.off >> 2, sh = (pc.off & 3u) * 8;
                for (uint32_t r = tid; r < n; r += kPipeNC) buf[r] = __funnelshift_r(A[w0 + r], A[w0 + r + 1], sh);
                if (tid == 0) {
                    s_cptr[c] = buf;
                    s_csh[c] = 31u;
                    s_cpd[c] = 0u;
                }
            } else {  // kPcLz4
                const int pl = pipe_lz4_tile(P.cols[c], T, pc, area, buf, s_seg, &s_err, tid);
                if (tid == 0) {
                    s_cptr[c] = buf;
                    s_csh[c] = P.cols[c].seg_shift;
                    s_cpd[c] = pl < 0 ? 0u : (uint32_t)pl;
                }
            }
        }
        pipe_sync();  // decoded buffers and column pointers complete
        const int terr = s_err;
        if (terr) {  // corrupt tile: dropped, the error kept (s_err is cleared past the tile's last barrier)
            if (tid == 0) raise_error(terr);
        } else {
            // ---- evaluation: the plan's steps, step-major over this thread's rows
            const uint32_t a = T.a, b = T.b;
            if (tid == 0) local_rows += b - a;
            uint32_t keep = 0;
            uint32_t gk[RPT];
            int32_t carry[RPT];
#pragma unroll
            for (uint32_t i = 0; i < RPT; ++i) {
                const uint32_t r = (i * NW + warp) * 32 + lane;
                if (r >= a && r < b) keep |= 1u << i;
                gk[i] = 0;
                carry[i] = 0;
            }
            const uint32_t ns = Q.n_steps;
            for (uint32_t s = 0; s < ns; ++s) {
                const ShStep& stp = Q.steps[s];
                const uint32_t c = stp.col, flags = stp.flags, dcard = stp.digit_card;
                const int32_t lo = stp.lo, hi = stp.hi, dbase = stp.digit_base;
                const uint64_t* const ht = stp.ht;
                const uint32_t htlog = stp.ht_log2, htlay = stp.ht_layout;
                const uint32_t* const col = s_cptr[c];
                const uint32_t sh = s_csh[c], pd = s_cpd[c];
                const bool last = s + 1 == ns;
                const bool simple = !(flags & GX_STEP_PROBE) && dcard == 0;
                const bool filt = (flags & GX_STEP_FILTER) != 0, carry_step = (flags & GX_STEP_CARRY) != 0;
                if (simple && !last) {
#pragma unroll
                    for (uint32_t i = 0; i < RPT; ++i) {
                        const uint32_t r = (i * NW + warp) * 32 + lane;
                        const int32_t v = (int32_t)col[sh_col_index(r, sh, pd)];
                        const bool kk = ((keep >> i) & 1u) && (!filt || (v >= lo && v <= hi));
                        if (carry_step) carry[i] = v;
                        keep = kk ? keep : (keep & ~(1u << i));
                    }
                } else if (simple && last && !grouped && agg != GX_AGG_COUNT && agg != GX_AGG_BUILD) {
                    const bool prod = agg == GX_AGG_SUM_PRODUCT, diff = agg == GX_AGG_SUM_DIFF;
#pragma unroll
                    for (uint32_t i = 0; i < RPT; ++i) {
                        const uint32_t r = (i * NW + warp) * 32 + lane;
                        const int32_t v = (int32_t)col[sh_col_index(r, sh, pd)];
                        const bool kk = ((keep >> i) & 1u) && (!filt || (v >= lo && v <= hi));
                        const int32_t c2 = carry_step ? v : carry[i];
                        const int64_t val = prod ? (int64_t)v * c2 : diff ? (int64_t)v - c2 : (int64_t)v;
                        local += kk ? val : 0;
                    }
                } else if ((flags & GX_STEP_PROBE) && htlay != GX_HT_BUCKET && !last) {
                    // dense or linear join table: the first slot reads of all rows are
                    // issued before any is used; a linear probe that the first slot does
                    // not settle walks its chain
                    const bool dense = htlay == GX_HT_DENSE;
                    uint32_t hbase = 0, hspan = 0;
                    if (dense) {
                        const uint64_t hdr = __ldg((const unsigned long long*)ht);
                        hbase = (uint32_t)hdr;
                        hspan = (uint32_t)(hdr >> 32);
                    }
                    int32_t vv[RPT];
                    uint64_t ee[RPT];
                    uint32_t fk = 0;
#pragma unroll
                    for (uint32_t i = 0; i < RPT; ++i) {
                        const uint32_t r = (i * NW + warp) * 32 + lane;
                        bool kk = (keep >> i) & 1u;
                        const int32_t v = (int32_t)col[sh_col_index(r, sh, pd)];
                        if (filt) kk = kk && v >= lo && v <= hi;
                        const uint32_t u = (uint32_t)v - hbase;
                        const bool rd = kk && v != kEmptyKey && (!dense || u < hspan);
                        const unsigned long long* sp =
                            (const unsigned long long*)ht + (dense ? 1 + u : hash_key32(v, htlog));
                        vv[i] = v;
                        ee[i] = rd ? __ldg(sp) : (unsigned long long)kEmptySlot;
                        fk |= rd ? 1u << i : 0u;
                    }
#pragma unroll
                    for (uint32_t i = 0; i < RPT; ++i) {
                        if (!((keep >> i) & 1u)) continue;
                        const int32_t v = vv[i];
                        bool kk = (fk >> i) & 1u;
                        int32_t pp = 0;
                        if (kk) {
                            const int32_t ek = (int32_t)(uint32_t)ee[i];
                            if (ek == v) {
                                pp = (int32_t)(uint32_t)(ee[i] >> 32);
                            } else if (dense || ek == kEmptyKey) {
                                kk = false;
                            } else {
                                pp = v;
                                kk = sh_probe(ht, htlog, htlay, v, &pp);
                            }
                        }
                        if (dcard && kk) {
                            const uint32_t dgt = (uint32_t)(pp - dbase);
                            if (dgt >= dcard) {
                                raise_error(kErrInvalid);
                                kk = false;
                            } else {
                                gk[i] = gk[i] * dcard + dgt;
                            }
                        }
                        if (carry_step && kk) carry[i] = v;
                        if (!kk) keep &= ~(1u << i);
                    }
                } else {
                    // general step: bucket-table probes (one-entry memo), group-key
                    // digits, COUNT, grouped aggregation
                    int32_t mv = kEmptyKey, mp = 0;
                    bool mk = false;
#pragma unroll
                    for (uint32_t i = 0; i < RPT; ++i) {
                        const uint32_t r = (i * NW + warp) * 32 + lane;
                        bool kk = (keep >> i) & 1u;
                        const int32_t v = (int32_t)col[sh_col_index(r, sh, pd)];
                        if (filt) kk = kk && v >= lo && v <= hi;
                        int32_t pp = v;
                        if ((flags & GX_STEP_PROBE) && kk) {
                            if (v != mv) {
                                mp = v;
                                mk = sh_probe(ht, htlog, htlay, v, &mp);
                                mv = v;
                            }
                            kk = mk;
                            pp = mp;
                        }
                        if ((keep >> i) & 1u) {
                            if (dcard && kk) {
                                const uint32_t dgt = (uint32_t)(pp - dbase);
                                if (dgt >= dcard) {
                                    raise_error(kErrInvalid);
                                    kk = false;
                                } else {
                                    gk[i] = gk[i] * dcard + dgt;
                                }
                            }
                            if (carry_step && kk) carry[i] = v;
                            if (!kk) keep &= ~(1u << i);
                        }
                        if (last && agg == GX_AGG_BUILD) {
                            if (kk) {
                                const uint32_t sl = T.slot, ch = sl / P.blocks_per_chunk;
                                const int32_t pay =
                                    P.build_rowid
                                        ? (int32_t)((uint64_t)ch * P.rows_per_chunk +
                                                    (uint64_t)(sl - ch * P.blocks_per_chunk) * P.rows_per_block +
                                                    T.r0 + (i * NW + warp) * 32 + lane)
                                        : carry[i];
                                const uint32_t o = pipe_ht_insert(P.build_slots, P.build_log2, P.build_layout, v, pay);
                                b_ins += o == 0;
                                b_dup += o == 1;
                                b_bad += o == 2;
                            }
                        } else if (last) {
                            const int64_t val = !kk                          ? 0
                                                : agg == GX_AGG_SUM_PRODUCT ? (int64_t)v * carry[i]
                                                : agg == GX_AGG_SUM_DIFF    ? (int64_t)v - carry[i]
                                                : agg == GX_AGG_COUNT        ? 1
                                                                             : (int64_t)v;
                            if (!grouped) local += val;
                            else if (kk)
                                pipe_group_add(gk[i], val, s_gsum, s_gkey, &s_gfill, Q.g_keys, Q.g_sums, Q.g_log2);
                        }
                    }
                }
            }
        }
        // every consumer is past the tile: release its slot
        pipe_sync();
        if (tid == 0) {
            mbar_arrive(&s_empty[st]);
            if (terr) s_err = 0;
        }
        if (grouped && s_gfill > kShGroupSlots / 2)
            pipe_group_flush(s_gsum, s_gkey, &s_gfill, Q.g_keys, Q.g_sums, Q.g_log2, tid);
    }
    // ---- end of the launch: scalar sum, group table, build counters, rows
    if (agg == GX_AGG_BUILD) {
        const uint32_t ins = __reduce_add_sync(0xFFFFFFFFu, b_ins), dup = __reduce_add_sync(0xFFFFFFFFu, b_dup),
                       bad = __reduce_add_sync(0xFFFFFFFFu, b_bad);
        if (lane == 0) {
            if (ins) atomicAdd(P.build_counters, (unsigned long long)ins);
            if (dup) atomicAdd(P.build_counters + 1, (unsigned long long)dup);
            if (bad) atomicAdd(P.build_counters + 2, (unsigned long long)bad);
        }
    } else if (grouped) {
        pipe_group_flush(s_gsum, s_gkey, &s_gfill, Q.g_keys, Q.g_sums, Q.g_log2, tid);
    } else {
        unsigned long long u = (unsigned long long)local;
#pragma unroll
        for (int d = 16; d > 0; d >>= 1) u += __shfl_down_sync(0xFFFFFFFFu, u, d);
        if (lane == 0 && u && Q.result) atomicAdd((unsigned long long*)Q.result, u);
    }
    if (tid == 0 && P.rows_scanned && local_rows) atomicAdd(P.rows_scanned, local_rows);
}
