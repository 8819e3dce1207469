// shared_scan.cuh -- the shared-scan form of a batch (device side; included
// by kernels.cu inside its anonymous namespace).  No reference counterpart:
// the reference runs one query per pipeline.
//
// Many queries over one fact table: every (block, tile) that at least one
// query needs is decoded ONCE -- each column any of its active queries reads,
// into its own shared-memory buffer -- and then every active query is
// evaluated on the tile row by row from shared memory.  A query's steps keep
// their meaning (FILTER, PROBE with group-key digits, CARRY, then the final
// VALUE step), so each query's result equals the result of running it alone.
//
// Work list: for every block slot, a bit mask of the queries that need it
// (slice overlap, chunk min/max of the prune predicates -- the reference's
// pruning granularity -- and the block zone map); slots with a non-empty
// mask are compacted (order does not matter: all sums are integer).

constexpr uint32_t kShTile = 2048;        // rows per shared tile
constexpr uint32_t kShMaxCols = 16;       // distinct columns in one shared batch
constexpr uint32_t kShMaxQueries = 1024;  // queries in one shared batch
constexpr uint32_t kShNT = 256;           // default threads per CTA of a batch (128, 256, 512, 1024 are built)
constexpr uint32_t kShSingleNT = 128;     // one-query launches: 4 CTAs (4 tiles in flight) per SM
constexpr uint32_t kShColWords = kShTile + 256;  // one column buffer (with segment padding)
constexpr uint32_t kShMaxQcBytes = 96u << 10;     // compact descriptors of a batch held in shared memory
constexpr uint32_t kShMaxDynSmem = 220u << 10;    // dynamic shared memory of one CTA (static use is ~1.3 KiB)
constexpr uint32_t kShGroupLog2 = 10;             // CTA group table of grouped queries: 1024 slots (12 KiB)
constexpr uint32_t kShGroupSlots = 1u << kShGroupLog2;
constexpr uint32_t kShGroupProbes = 32;

struct ShStep {
    uint32_t flags;
    int32_t lo, hi;
    uint32_t col;  // index into the batch's column table
    const uint64_t* ht;
    uint32_t ht_log2, ht_layout;
    int32_t digit_base;
    uint32_t digit_card;
};

struct ShQuery {
    ShStep steps[GX_MAX_STEPS];  // the last step is the (only) VALUE step
    uint32_t n_steps;
    uint32_t agg;
    uint32_t grouped;
    uint32_t col_mask;  // columns the query reads
    uint64_t row_lo, row_hi;
    int64_t* result;
    int64_t* g_keys;
    int64_t* g_sums;
    uint32_t g_log2;
    uint32_t n_prune;
    PrunePred prune[GX_MAX_STEPS];
    const uint16_t* keep_in;  // per-chunk keep flags or null
    uint16_t* keep_out;       // per-chunk keep flags written by the work-list pass, or null
};

// Compact copies of a batch's query descriptors, held in shared memory for
// the whole launch (the evaluation reads them for every (query, tile, step)).
struct ShStepC {
    int32_t lo, hi;
    const uint64_t* ht;
    int32_t dbase;
    uint32_t dcard;
    uint8_t col, flags, htlog, htlay;
};
struct ShQueryC {
    uint64_t row_lo, row_hi;
    int64_t* g_keys;
    int64_t* g_sums;
    uint32_t step0;  // index of the query's first step in the step array
    uint8_t n_steps, agg, grouped, g_log2;
    uint32_t gbits;  // mask-word bits of the query's prefix group (0: no group)
    uint8_t pfx;     // steps the group shares (fewer than any member's step count)
    uint8_t psave;   // what the shared prefix hands on: bit 0 group-key digits, bit 1 carried value
    uint16_t col_mask;  // columns the query reads
};
static_assert(sizeof(ShStepC) == 32 && sizeof(ShQueryC) == 48, "compact descriptor sizes");

struct ShParams {
    const gx_dcol* cols;        // the batch's column table (global memory)
    uint32_t n_cols;
    const ShQuery* qs;
    uint32_t n_queries;
    uint32_t mask_words;        // ceil(n_queries / 32)
    // batches: the work list of shared_items_kernel (one-query launches prune
    // their own work and leave these null)
    const uint32_t* slot_mask;  // n_slots * mask_words
    const uint32_t* items;      // compacted slots
    const uint32_t* n_items;
    uint32_t* work_counter;
    uint32_t blocks_per_chunk, rows_per_chunk, rows_per_block;
    uint32_t tile_rows, tiles_per_block;
    unsigned long long* rows_scanned;  // optional: sum over (query, tile) of the query's rows in the tile
    const uint4* qc;            // batches: [ShQueryC x n_queries | ShStepC x steps], copied to shared memory
    uint32_t qc_bytes;          // size of that image (a multiple of 16)
    const gx_dblock* dir;       // directory of the table (any of its columns)
    uint32_t n_slots;
    uint32_t pst_carry;         // offset of the carried values in the prefix-state buffer (words)
    uint32_t pst_words;         // size of the prefix-state buffer (words)
    uint32_t gt_slots;          // CTA group-table slots (kShGroupSlots with grouped queries, else 0)
    // one query carried in the parameters themselves (qs and cols null)
    ShQuery q1;
    gx_dcol cols1[kShMaxCols];
};

__device__ __forceinline__ const ShQuery* sh_queries(const ShParams& P) { return P.qs ? P.qs : &P.q1; }

// The fields the evaluation reads, from the parameters (one-query launch) or
// from the compact copies in shared memory (batch).
struct QView {
    uint64_t row_lo, row_hi;
    int64_t* g_keys;
    int64_t* g_sums;
    uint32_t n_steps, agg, g_log2, step0;
    uint32_t gbits, pfx, psave;
    bool grouped;
};
struct SView {
    int32_t lo, hi, dbase;
    const uint64_t* ht;
    uint32_t dcard, col, flags, htlog, htlay;
};
template <bool SINGLE>
__device__ __forceinline__ QView sh_qv(const ShParams& P, const uint8_t* s_qc, uint32_t q) {
    QView v;
    if constexpr (SINGLE) {
        v.row_lo = P.q1.row_lo;
        v.row_hi = P.q1.row_hi;
        v.g_keys = P.q1.g_keys;
        v.g_sums = P.q1.g_sums;
        v.n_steps = P.q1.n_steps;
        v.agg = P.q1.agg;
        v.g_log2 = P.q1.g_log2;
        v.step0 = 0;
        v.gbits = 0;
        v.pfx = 0;
        v.psave = 0;
        v.grouped = P.q1.grouped != 0;
    } else {
        const ShQueryC& c = ((const ShQueryC*)s_qc)[q];
        v.row_lo = c.row_lo;
        v.row_hi = c.row_hi;
        v.g_keys = c.g_keys;
        v.g_sums = c.g_sums;
        v.n_steps = c.n_steps;
        v.agg = c.agg;
        v.g_log2 = c.g_log2;
        v.step0 = c.step0;
        v.gbits = c.gbits;
        v.pfx = c.pfx;
        v.psave = c.psave;
        v.grouped = c.grouped != 0;
    }
    return v;
}
template <bool SINGLE>
__device__ __forceinline__ SView sh_sv(const ShParams& P, const uint8_t* s_qc, const QView& Q, uint32_t s) {
    SView v;
    if constexpr (SINGLE) {
        const ShStep& t = P.q1.steps[s];
        v.lo = t.lo;
        v.hi = t.hi;
        v.dbase = t.digit_base;
        v.ht = t.ht;
        v.dcard = t.digit_card;
        v.col = t.col;
        v.flags = t.flags;
        v.htlog = t.ht_log2;
        v.htlay = t.ht_layout;
    } else {
        const ShStepC& t = ((const ShStepC*)(s_qc + sizeof(ShQueryC) * P.n_queries))[Q.step0 + s];
        v.lo = t.lo;
        v.hi = t.hi;
        v.dbase = t.dbase;
        v.ht = t.ht;
        v.dcard = t.dcard;
        v.col = t.col;
        v.flags = t.flags;
        v.htlog = t.htlog;
        v.htlay = t.htlay;
    }
    return v;
}

// Query q and column c: in the parameters themselves for a one-query launch
// (SINGLE: constant-bank reads), else in global memory.
template <bool SINGLE>
__device__ __forceinline__ const ShQuery& sh_q(const ShParams& P, uint32_t q) {
    if constexpr (SINGLE) return P.q1;
    else return P.qs[q];
}
template <bool SINGLE>
__device__ __forceinline__ const gx_dcol& sh_c(const ShParams& P, uint32_t c) {
    if constexpr (SINGLE) return P.cols1[c];
    else return P.cols[c];
}

// One warp per block slot: lane l tests query 32*w + l of mask word w; the
// word is the warp ballot.  Slots with any query set are appended to items.
// Queries with keep_out get their per-chunk flags (chunk min/max and keep_in,
// the reference's granularity) from the warp of the chunk's first block.
__global__ void shared_items_kernel(const __grid_constant__ ShParams P, uint32_t* slot_mask, uint32_t* items,
                                    uint32_t* n_items) {
    const ShQuery* qs = sh_queries(P);
    const uint32_t lane = threadIdx.x & 31;
    const uint32_t warps = gridDim.x * (blockDim.x / 32);
    const uint32_t mask_words = P.mask_words, n_queries = P.n_queries;
    for (uint32_t s = blockIdx.x * (blockDim.x / 32) + threadIdx.x / 32; s < P.n_slots; s += warps) {
        const uint32_t rows = P.dir[s].n_rows;
        const uint32_t chunk = s / P.blocks_per_chunk, j = s % P.blocks_per_chunk;
        const uint64_t g0 = (uint64_t)chunk * P.rows_per_chunk + (uint64_t)j * P.rows_per_block, g1 = g0 + rows;
        bool any = false;
        for (uint32_t w = 0; w < mask_words; ++w) {
            const uint32_t q = w * 32 + lane;
            bool keep = false;
            if (q < n_queries) {
                const ShQuery& Q = qs[q];
                bool ck = Q.keep_in ? Q.keep_in[chunk] != 0 : true;
                for (uint32_t p = 0; ck && p < Q.n_prune; ++p) {
                    const PrunePred& pr = Q.prune[p];
                    ck = pr.lo <= pr.maxs[chunk] && pr.hi >= pr.mins[chunk];
                }
                if (Q.keep_out && j == 0) Q.keep_out[chunk] = ck ? 1 : 0;
                keep = ck && rows && Q.row_lo < g1 && Q.row_hi > g0;
                for (uint32_t p = 0; keep && p < Q.n_prune; ++p) {
                    const PrunePred& pr = Q.prune[p];
                    if (pr.bmins) keep = pr.lo <= pr.bmaxs[s] && pr.hi >= pr.bmins[s];
                }
            }
            const uint32_t m = __ballot_sync(0xFFFFFFFFu, keep);
            if (lane == 0) slot_mask[(size_t)s * mask_words + w] = m;
            any = any || m;
        }
        if (any && lane == 0) items[atomicAdd(n_items, 1u)] = s;
    }
}

// Out-of-line pieces of the evaluation: the row loop is unrolled RPT times,
// so large bodies inside it are called rather than inlined to keep the hot
// code small (instruction-fetch stalls).
__device__ __noinline__ bool sh_probe(const uint64_t* ht, uint32_t htlog, uint32_t htlay, int32_t v, int32_t* p) {
    return ht_probe_any(ht, htlog, htlay, v, p);
}

// Add of (gk, val) to the CTA's group table in shared memory (the partial
// sums of one query over one tile; flushed to the query's global table when
// its tile is done), so that keys repeated within a tile -- skewed group-bys
// -- cost one global update per tile.  A key that finds no slot within
// kShGroupProbes goes to the global table directly.
__device__ __noinline__ void sh_group_add(uint32_t gk, int64_t val, unsigned long long* tsum, int64_t* keys,
                                          int64_t* sums, uint32_t log2cap) {
    uint32_t* const tkey = (uint32_t*)(tsum + kShGroupSlots);
    if (gk != kEmptyGKey) {
        uint32_t s = hash_key32((int32_t)gk, kShGroupLog2);
        for (uint32_t i = 0; i < kShGroupProbes; ++i) {
            uint32_t cur = ((volatile uint32_t*)tkey)[s];
            if (cur == kEmptyGKey) cur = atomicCAS(&tkey[s], kEmptyGKey, gk);
            if (cur == kEmptyGKey || cur == gk) {
                atomicAdd(&tsum[s], (unsigned long long)val);
                return;
            }
            s = (s + 1) & (kShGroupSlots - 1);
        }
    }
    if (!group_add_global(keys, sums, log2cap, (int64_t)gk, val)) raise_error(kErrCapacity);
}

// Flush of the CTA's group table into the query's global table (all NT
// threads, between barriers); leaves the table empty.
template <int NT>
__device__ __forceinline__ void sh_group_flush(unsigned long long* tsum, uint32_t* tkey, int64_t* keys, int64_t* sums,
                                               uint32_t log2cap) {
    __syncthreads();
    for (uint32_t j = threadIdx.x; j < kShGroupSlots; j += NT) {
        const uint32_t key = tkey[j];
        if (key != kEmptyGKey) {
            if (!group_add_global(keys, sums, log2cap, (int64_t)key, (int64_t)tsum[j])) raise_error(kErrCapacity);
            tkey[j] = kEmptyGKey;
            tsum[j] = 0;
        }
    }
    __syncthreads();
}

__device__ __forceinline__ uint32_t sh_col_index(uint32_t r, uint32_t sh, uint32_t pd) {
    return r + ((r >> sh) << pd);
}

// Decode column c of the tile into its buffer (all NT threads).  Records the
// column's layout in s_sh/s_pd (every thread writes the same value).
// Returns 0, or the device error after which the tile is dropped.
template <int NT>
__device__ __forceinline__ int shared_decode(const gx_dcol& col, uint32_t c, uint32_t slot, uint32_t rows,
                                             uint32_t r0, uint32_t n, uint32_t* colbuf, uint8_t* stage,
                                             uint64_t* mbar, uint32_t& phase, uint32_t* s_tmp, int* s_err,
                                             int* s_fatal, uint32_t* s_sh, uint32_t* s_pd, uint32_t* s_seg) {
    uint32_t* buf = colbuf + c * kShColWords;
    uint32_t pad_log2 = 0;
    const int layout = decode_tile<NT, kTileRows>(col, slot, rows, r0, n, buf, stage, mbar, phase, s_tmp, s_err,
                                                  pad_log2, s_seg);
    const int derr = *s_err;
    __syncthreads();
    if (derr) {
        if (threadIdx.x == 0) {
            raise_error(derr);
            *s_err = 0;
            if (derr == kErrTimeout) *s_fatal = 1;  // the stage may still be written: stop this CTA
        }
        __syncthreads();
        return derr;
    }
    s_sh[c] = layout == kSegRows ? col.seg_shift : 31u;
    s_pd[c] = layout == kSegRows ? pad_log2 : 0u;
    __syncthreads();
    return 0;
}

// Literal columns of a tile, copied at once (a batch: every column its
// active queries read, before they run; one query: its remaining columns
// once its first step leaves rows alive).  A column of segmented LZ4 whose
// tile lies inside one literal run (random-valued columns; the encoder
// stores them as literals) is a plain byte range of the block; the columns
// in that form are copied straight from global memory into their buffers
// with all their loads in flight together, instead of one staged decode per
// column as a step first needs it.  shared_literal_locate: thread c checks
// column c (directory entry and the tile's segment entries) and records the
// tile's first byte, or null, in s_lit[c]; a one-query launch locates its
// later columns at the tile's start and prefetches their bytes into L2, so
// that the copy after the first step reads L2.  All NT threads call both
// functions (rows land in plain order).
template <int NT, bool SINGLE>
__device__ __forceinline__ void shared_literal_locate(const ShParams& P, uint32_t cols, uint32_t slot, uint32_t rows,
                                                      uint32_t r0, uint32_t n, const uint8_t** s_lit, uint32_t* s_sh,
                                                      uint32_t* s_pd, bool prefetch) {
    const uint32_t tid = threadIdx.x;
    if (tid < kShMaxCols) {
        const uint8_t* src = nullptr;
        if ((cols >> tid) & 1u) {
            const gx_dcol& c = sh_c<SINGLE>(P, tid);
            if (c.codec == GX_CODEC_LZ4 && c.S > 1 && !c.host_mapped && (n & 3u) == 0 &&
                (r0 & ((1u << c.seg_shift) - 1u)) == 0) {
                const gx_dblock d = c.blocks[slot];
                const uint32_t j0 = r0 >> c.seg_shift;
                const uint32_t nseg = (n + (1u << c.seg_shift) - 1) >> c.seg_shift;
                const uint32_t* e = c.seg + (size_t)2 * c.S * slot;
                if (d.n_rows == rows && d.offset <= c.payload_bytes &&
                    (uint64_t)d.comp_bytes + 32 <= c.payload_bytes - d.offset && j0 + nseg <= c.S) {
                    const uint32_t lo = __ldg(e + 2 * j0), info0 = __ldg(e + 2 * j0 + 1);
                    const uint32_t hi = j0 + nseg < c.S ? __ldg(e + 2 * (j0 + nseg)) : d.comp_bytes;
                    if ((info0 & 16u) && (info0 >> 5) >= 4 * n && hi >= lo && hi - lo == 4 * n &&
                        hi <= d.comp_bytes) {
                        src = c.payload + d.offset + lo;
                        if (prefetch) {
                            // the bytes (16-byte aligned cover, inside the payload's slack) into L2
                            const uint64_t a0 = (d.offset + lo) & ~15ull;
                            const uint8_t* a = c.payload + a0;
                            const uint32_t bytes = (uint32_t)(((d.offset + hi + 15u) & ~15ull) - a0);
                            asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(a), "r"(bytes)
                                         : "memory");
                        }
                    }
                }
            }
        }
        s_lit[tid] = src;
        if (src) {
            s_sh[tid] = 31u;
            s_pd[tid] = 0u;
        }
    }
}

// Copy of the located literal columns in `cols` (after a barrier that made
// shared_literal_locate's results visible); returns the columns copied.
template <int NT>
__device__ __forceinline__ uint32_t shared_literal_copy(uint32_t cols, uint32_t n, uint32_t* colbuf,
                                                        const uint8_t* const* s_lit) {
    const uint32_t tid = threadIdx.x;
    uint32_t done = 0;
    for (uint32_t cm = cols; cm; cm &= cm - 1)
        if (s_lit[__ffs(cm) - 1]) done |= 1u << (__ffs(cm) - 1);
    // items (column, 4-row group): five aligned words give the four rows
    const uint32_t per = n / 4, nlit = __popc(done);
    uint32_t cm = done;
    for (uint32_t k = 0; k < nlit; ++k, cm &= cm - 1) {
        const uint32_t c = __ffs(cm) - 1;
        const uint8_t* src = s_lit[c];
        const uint32_t* A = (const uint32_t*)((uintptr_t)src & ~(uintptr_t)3);
        const uint32_t sh = ((uint32_t)(uintptr_t)src & 3u) * 8;
        uint4* dst = (uint4*)(colbuf + c * kShColWords);
#pragma unroll 4
        for (uint32_t q4 = tid; q4 < per; q4 += NT) {
            const uint32_t* w = A + 4 * q4;
            const uint32_t a0 = __ldg(w), a1 = __ldg(w + 1), a2 = __ldg(w + 2), a3 = __ldg(w + 3), a4 = __ldg(w + 4);
            dst[q4] = make_uint4(__funnelshift_r(a0, a1, sh), __funnelshift_r(a1, a2, sh),
                                 __funnelshift_r(a2, a3, sh), __funnelshift_r(a3, a4, sh));
        }
    }
    if (done) __syncthreads();
    return done;
}

// One-query launches: whether tile `tile` of block slot `slot` is work --
// the pruning of shared_items_kernel (chunk min/max and keep_in, the slice,
// the block zone maps) applied per tile; writes the chunk's keep_out flag
// for the chunk's first tile.
__device__ __forceinline__ bool sh_single_live(const ShParams& P, uint32_t slot, uint32_t tile) {
    const ShQuery& Q = P.q1;
    const uint32_t chunk = slot / P.blocks_per_chunk, j = slot % P.blocks_per_chunk;
    bool ck = Q.keep_in ? Q.keep_in[chunk] != 0 : true;
    for (uint32_t p = 0; ck && p < Q.n_prune; ++p) {
        const PrunePred& pr = Q.prune[p];
        ck = pr.lo <= pr.maxs[chunk] && pr.hi >= pr.mins[chunk];
    }
    if (Q.keep_out && j == 0 && tile == 0) Q.keep_out[chunk] = ck ? 1 : 0;
    const uint32_t rows = P.dir[slot].n_rows, r0 = tile * P.tile_rows;
    if (!ck || r0 >= rows) return false;
    const uint64_t g0 = (uint64_t)chunk * P.rows_per_chunk + (uint64_t)j * P.rows_per_block + r0;
    const uint32_t n = min(P.tile_rows, rows - r0);
    if (!(Q.row_lo < g0 + n && Q.row_hi > g0)) return false;
    for (uint32_t p = 0; p < Q.n_prune; ++p) {
        const PrunePred& pr = Q.prune[p];
        if (pr.bmins && !(pr.lo <= pr.bmaxs[slot] && pr.hi >= pr.bmins[slot])) return false;
    }
    return true;
}

// Persistent shared-scan kernel: NT threads, tiles of up to kShTile rows.
// Per tile, the active queries are evaluated one after another, step-major:
// a step's fields go to registers, then the step runs over the RPT row
// groups this thread owns (group i*NW + warp, row lane), whose state (alive
// bit, group key, carried value) stays in registers; the last step
// aggregates.  A column is decoded when a step first needs it and then
// serves every later query of the tile; before decoding for a query whose
// rows are all dead, the query stops (a block-wide vote), so dead tiles cost
// only the columns their first steps read.
// Queries whose first steps are identical (star joins over one dimension
// selection, say) form prefix groups: per tile, those steps run once over
// the union of the active members' rows and each member starts after them.
// Dynamic shared memory: n_cols column buffers | stage | per-query partial
// sums | per-tile active-query mask | descriptors | prefix state (group-key
// digits and carried values of the shared steps, one word per tile row) |
// CTA group table (sums, then keys).
template <int NT, int MINB, bool SINGLE = false>
__global__ void __launch_bounds__(NT, MINB) shared_scan_kernel(const __grid_constant__ ShParams P) {
    constexpr int NW = NT / 32;
    constexpr int RPT = (kShTile + NT - 1) / NT;  // row groups per warp
    using C = Cfg<kTileRows>;  // stage sized for 4096-row tiles (holds the cascaded run tables)
    extern __shared__ __align__(16) uint8_t smem[];
    uint32_t* colbuf = (uint32_t*)smem;
    uint8_t* stage = (uint8_t*)(colbuf + (size_t)P.n_cols * kShColWords);
    unsigned long long* s_part = (unsigned long long*)(stage + C::kStage);
    uint32_t* s_qmask = (uint32_t*)(s_part + P.n_queries);
    uint8_t* s_qc = (uint8_t*)(((uintptr_t)(s_qmask + P.mask_words) + 15) & ~(uintptr_t)15);

    __shared__ __align__(8) uint64_t s_mbar;
    __shared__ uint32_t s_item;
    __shared__ int s_err;
    __shared__ int s_fatal;
    __shared__ uint32_t s_sh[kShMaxCols], s_pd[kShMaxCols];
    __shared__ uint32_t s_tmp[NW + 1];
    __shared__ uint32_t s_seg[2 * (kMaxSegments + 1)];
    __shared__ uint32_t s_cols;                    // batches: columns the tile's active queries read
    __shared__ uint32_t s_list[SINGLE ? NT : 1];   // one query: this CTA's live items of the round
    __shared__ uint32_t s_ln, s_li, s_w0;          // their count, the next one, the next round's start
    __shared__ const uint8_t* s_lit[kShMaxCols];   // batches: a literal tile's first byte, or null

    const uint32_t tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    for (uint32_t i = tid; i < P.n_queries; i += NT) s_part[i] = 0;
    // CTA group table (present when the launch has grouped queries)
    unsigned long long* const s_gsum = (unsigned long long*)(s_qc + P.qc_bytes + 4ull * P.pst_words);
    uint32_t* const s_gkey = (uint32_t*)(s_gsum + P.gt_slots);
    for (uint32_t i = tid; i < P.gt_slots; i += NT) {
        s_gsum[i] = 0;
        s_gkey[i] = kEmptyGKey;
    }
    const uint64_t pol_keep = ws_policy_keep();  // join tables stay in L2 while the columns stream through
    if (!SINGLE)
        for (uint32_t i = tid; i < P.qc_bytes / 16; i += NT) ((uint4*)s_qc)[i] = __ldg(P.qc + i);
    if (tid == 0) {
        s_err = 0;
        s_fatal = 0;
        if (!SINGLE) s_cols = 0;
        mbar_init(&s_mbar, 1);
    }
    uint32_t phase = 0;
    unsigned long long local_rows = 0;
    const uint32_t tpb = P.tiles_per_block, tile_rows = P.tile_rows;
    // one query: every (slot, tile) item is a candidate, checked by the CTA it
    // falls to (item w goes to CTA w mod grid); batches: the compacted work
    // list of shared_items_kernel, taken from a counter
    const uint32_t total = SINGLE ? P.n_slots * tpb : *P.n_items * tpb;
    const uint32_t MW = P.mask_words;
    if (tid == 0) {
        if (SINGLE) {
            s_ln = 0;
            s_li = 0;
            s_w0 = 0;
        } else {
            s_item = atomicAdd(P.work_counter, 1u);
        }
    }
    __syncthreads();

    while (true) {
        uint32_t it;
        if constexpr (SINGLE) {
            // the round's list used up: check the next round of candidates, one per thread
            while (s_li >= s_ln && s_w0 < total) {
                const uint32_t w = s_w0 + blockIdx.x + tid * gridDim.x;
                const bool live = w < total && sh_single_live(P, w / tpb, w % tpb);
                const uint32_t bal = __ballot_sync(0xFFFFFFFFu, live);
                if (lane == 0) s_tmp[warp] = __popc(bal);
                __syncthreads();
                uint32_t off = 0, cnt = 0;
                for (uint32_t k = 0; k < (uint32_t)NW; ++k) {
                    off += k < warp ? s_tmp[k] : 0u;
                    cnt += s_tmp[k];
                }
                if (live) s_list[off + __popc(bal & ((1u << lane) - 1u))] = w;
                __syncthreads();
                if (tid == 0) {
                    s_ln = cnt;
                    s_li = 0;
                    s_w0 += gridDim.x * NT;
                }
                __syncthreads();
            }
            if (s_li >= s_ln) break;
            it = s_list[s_li];
        } else {
            it = s_item;
            if (it >= total) break;
        }
        // batches: thread 0 takes the next work item now; its result is needed only at the tile's end
        uint32_t next_it = 0xFFFFFFFFu;
        if (!SINGLE && tid == 0) next_it = atomicAdd(P.work_counter, 1u);
        const uint32_t slot = SINGLE ? it / tpb : P.items[it / tpb];
        const uint32_t r0 = (it % tpb) * tile_rows;
        const uint32_t rows = P.dir[slot].n_rows;
        if (r0 < rows) {
        const uint32_t n = min(tile_rows, rows - r0);
        const uint32_t chunk = slot / P.blocks_per_chunk, j = slot % P.blocks_per_chunk;
        const uint64_t g0 = (uint64_t)chunk * P.rows_per_chunk + (uint64_t)j * P.rows_per_block + r0;
        // active queries of this tile: the block's mask restricted to slices that reach the tile
        for (uint32_t w = tid; w < MW; w += NT) {
            uint32_t m = SINGLE ? 1u : P.slot_mask[(size_t)slot * MW + w], keepm = m;
            while (m) {
                const uint32_t bit = __ffs(m) - 1;
                m &= m - 1;
                const QView Q = sh_qv<SINGLE>(P, s_qc, w * 32 + bit);
                if (!(Q.row_lo < g0 + n && Q.row_hi > g0)) keepm &= ~(1u << bit);
            }
            s_qmask[w] = keepm;
            if constexpr (!SINGLE) {
                uint32_t cm = 0;
                for (uint32_t mm = keepm; mm; mm &= mm - 1) cm |= ((const ShQueryC*)s_qc)[w * 32 + __ffs(mm) - 1].col_mask;
                if (cm) atomicOr(&s_cols, cm);
            }
        }
        __syncthreads();
        uint32_t lit = 0;  // batches: literal columns already copied
        if constexpr (!SINGLE) {
            shared_literal_locate<NT, SINGLE>(P, s_cols, slot, rows, r0, n, s_lit, s_sh, s_pd, false);
            __syncthreads();
            lit = shared_literal_copy<NT>(s_cols, n, colbuf, s_lit);
        } else {
            // one query: its columns after the first step's, located and prefetched now
            const uint32_t first = P.q1.steps[0].col;
            shared_literal_locate<NT, SINGLE>(P, P.q1.col_mask & ~(1u << first), slot, rows, r0, n, s_lit, s_sh,
                                              s_pd, true);
        }
        uint32_t* const s_pst = (uint32_t*)(s_qc + P.qc_bytes);  // prefix-state buffer (batches)
        uint32_t decoded = lit;  // columns of this tile already in their buffers
        bool dropped = false;
        bool lit_tried = false;  // one-query launches: literal columns copied past the first step
        for (uint32_t w = 0; w < MW && !dropped; ++w) {
            uint32_t m = s_qmask[w];
            while (m && !dropped) {
                const uint32_t q = w * 32 + (__ffs(m) - 1);
                m &= m - 1;
                // The other members of q's prefix group that are active in this tile
                // (the host orders a batch so that a group sits in one mask word).  With
                // any, a first pass runs the shared steps once over the union of the
                // members' rows, and each member then starts from its result.
                const QView Qg = sh_qv<SINGLE>(P, s_qc, q);
                const uint32_t gm = m & Qg.gbits, pfx = Qg.pfx, psave = Qg.psave;
                m &= ~gm;
                uint32_t ua = Qg.row_lo > g0 ? (uint32_t)(Qg.row_lo - g0) : 0u;
                uint32_t ub = Qg.row_hi < g0 + n ? (uint32_t)(Qg.row_hi - g0) : n;
                if (gm) {
                    uint32_t rows_g = ub - ua;
                    for (uint32_t r2 = gm; r2; r2 &= r2 - 1) {
                        const QView Qm = sh_qv<SINGLE>(P, s_qc, w * 32 + (__ffs(r2) - 1));
                        const uint32_t a2 = Qm.row_lo > g0 ? (uint32_t)(Qm.row_lo - g0) : 0u;
                        const uint32_t b2 = Qm.row_hi < g0 + n ? (uint32_t)(Qm.row_hi - g0) : n;
                        rows_g += b2 - a2;
                        ua = min(ua, a2);
                        ub = max(ub, b2);
                    }
                    if (tid == 0) local_rows += rows_g;
                }
                bool pre = gm != 0;      // the pass over the shared steps
                uint32_t keep_pre = 0;   // its surviving rows
                uint32_t rest = gm, cq = q;
                while (true) {
                const QView Q = sh_qv<SINGLE>(P, s_qc, cq);
                uint32_t a = ua, b = ub;
                if (!pre) {
                    a = Q.row_lo > g0 ? (uint32_t)(Q.row_lo - g0) : 0u;
                    b = Q.row_hi < g0 + n ? (uint32_t)(Q.row_hi - g0) : n;
                    if (tid == 0 && !gm) local_rows += b - a;
                }
                const uint32_t s_begin = gm && !pre ? pfx : 0u, ns = pre ? pfx : Q.n_steps, agg = Q.agg;
                const bool from_pre = gm && !pre;
                const bool grouped = Q.grouped != 0;
                uint32_t keep = 0;  // bit i: row of group i alive
                uint32_t gk[RPT];
                int32_t carry[RPT];
#pragma unroll
                for (int i = 0; i < RPT; ++i) {
                    const uint32_t r = (i * NW + warp) * 32 + lane;
                    if (r >= a && r < b && (!from_pre || ((keep_pre >> i) & 1u))) keep |= 1u << i;
                    gk[i] = from_pre && (psave & 1u) ? s_pst[r] : 0u;
                    carry[i] = from_pre && (psave & 2u) ? (int32_t)s_pst[P.pst_carry + r] : 0;
                }
                int64_t local = 0;
                for (uint32_t s = s_begin; s < ns; ++s) {
                    const SView st = sh_sv<SINGLE>(P, s_qc, Q, s);
                    const uint32_t c = st.col, flags = st.flags, dcard = st.dcard;
                    if (!((decoded >> c) & 1u)) {
                        // the query's rows are all dead: skip its remaining steps (and this decode)
                        if (s > 0 && !__syncthreads_or(keep != 0)) break;
                        if constexpr (SINGLE) {
                            // past the first step with rows alive: the query's remaining
                            // literal columns are copied together (their loads in flight at once)
                            if (s > 0 && !lit_tried) {
                                lit_tried = true;
                                decoded |= shared_literal_copy<NT>(P.q1.col_mask & ~decoded, n, colbuf, s_lit);
                            }
                        }
                    }
                    if (!((decoded >> c) & 1u)) {
                        if (shared_decode<NT>(sh_c<SINGLE>(P, c), c, slot, rows, r0, n, colbuf, stage, &s_mbar,
                                              phase, s_tmp, &s_err, &s_fatal, s_sh, s_pd, s_seg)) {
                            dropped = true;
                            break;
                        }
                        decoded |= 1u << c;
                    }
                    const int32_t lo = st.lo, hi = st.hi, dbase = st.dbase;
                    const uint64_t* const ht = st.ht;
                    const uint32_t htlog = st.htlog, htlay = st.htlay;
                    const uint32_t* const col = colbuf + c * kShColWords;
                    const uint32_t sh = s_sh[c], pd = s_pd[c];
                    const bool last = s + 1 == Q.n_steps;  // never within the shared steps
                    const bool simple = !(flags & GX_STEP_PROBE) && dcard == 0;  // no probe, no digit
                    const bool filt = (flags & GX_STEP_FILTER) != 0, carry_step = (flags & GX_STEP_CARRY) != 0;
                    if (simple && !last) {
                        // FILTER and/or CARRY: branch-free over the thread's rows (dead
                        // rows read their in-bounds slot and stay dead)
#pragma unroll
                        for (int i = 0; i < RPT; ++i) {
                            const uint32_t r = (i * NW + warp) * 32 + lane;
                            const int32_t v = (int32_t)col[sh_col_index(r, sh, pd)];
                            const bool k = ((keep >> i) & 1u) && (!filt || (v >= lo && v <= hi));
                            if (carry_step) carry[i] = v;
                            keep = k ? keep : (keep & ~(1u << i));
                        }
                    } else if (simple && last && !grouped && agg != GX_AGG_COUNT) {
                        // the VALUE step of a scalar SUM / SUM_PRODUCT
                        const bool prod = agg == GX_AGG_SUM_PRODUCT, diff = agg == GX_AGG_SUM_DIFF;
#pragma unroll
                        for (int i = 0; i < RPT; ++i) {
                            const uint32_t r = (i * NW + warp) * 32 + lane;
                            const int32_t v = (int32_t)col[sh_col_index(r, sh, pd)];
                            const bool k = ((keep >> i) & 1u) && (!filt || (v >= lo && v <= hi));
                            const int32_t c2 = carry_step ? v : carry[i];
                            const int64_t val = prod ? (int64_t)v * c2 : diff ? (int64_t)v - c2 : (int64_t)v;
                            local += k ? val : 0;
                        }
                    } else if (RPT <= 8 && (flags & GX_STEP_PROBE) && htlay != GX_HT_BUCKET && !last) {
                        // probe of a dense or linear join table: the first slot reads of all
                        // RPT rows are issued before any is used; a linear probe that the
                        // first slot does not settle (another key there) walks its chain
                        // (up to 8 rows per thread, where the registers allow)
                        const bool dense = htlay == GX_HT_DENSE;
                        uint32_t hbase = 0, hspan = 0;
                        if (dense) {
                            const uint64_t hdr = __ldg((const unsigned long long*)ht);
                            hbase = (uint32_t)hdr;
                            hspan = (uint32_t)(hdr >> 32);
                        }
                        int32_t vv[RPT];
                        uint64_t ee[RPT];
                        uint32_t fk = 0;  // rows whose slot was read
#pragma unroll
                        for (int i = 0; i < RPT; ++i) {
                            const uint32_t r = (i * NW + warp) * 32 + lane;
                            bool k = (keep >> i) & 1u;
                            const int32_t v = k ? (int32_t)col[sh_col_index(r, sh, pd)] : 0;
                            if (filt) k = k && v >= lo && v <= hi;
                            const uint32_t u = (uint32_t)v - hbase;
                            const bool rd = k && v != kEmptyKey && (!dense || u < hspan);
                            const unsigned long long* sp =
                                (const unsigned long long*)ht + (dense ? 1 + u : hash_key32(v, htlog));
                            vv[i] = v;
                            ee[i] = rd ? ws_ld_slot(sp, pol_keep) : (unsigned long long)kEmptySlot;
                            fk |= rd ? 1u << i : 0u;
                        }
#pragma unroll
                        for (int i = 0; i < RPT; ++i) {
                            if (!((keep >> i) & 1u)) continue;
                            const int32_t v = vv[i];
                            bool k = (fk >> i) & 1u;
                            int32_t p = 0;
                            if (k) {
                                const int32_t ek = (int32_t)(uint32_t)ee[i];
                                if (ek == v) {
                                    p = (int32_t)(uint32_t)(ee[i] >> 32);
                                } else if (dense || ek == kEmptyKey) {
                                    k = false;
                                } else {
                                    p = v;
                                    k = sh_probe(ht, htlog, htlay, v, &p);
                                }
                            }
                            if (dcard && k) {
                                const uint32_t dgt = (uint32_t)(p - dbase);
                                if (dgt >= dcard) {
                                    raise_error(kErrInvalid);
                                    k = false;
                                } else {
                                    gk[i] = gk[i] * dcard + dgt;
                                }
                            }
                            if (carry_step && k) carry[i] = v;
                            if (!k) keep &= ~(1u << i);
                        }
                    } else if ((flags & GX_STEP_PROBE) && dcard == 0 && !carry_step && !last) {
                        // a probe that only filters (a date or dimension membership test): a
                        // rolled loop with a one-entry memo -- small code, which matters on the
                        // first tiles of a launch, when every CTA runs it cold
                        int32_t mv = kEmptyKey;
                        bool mk = false;
#pragma unroll 1
                        for (int i = 0; i < RPT; ++i) {
                            if (!((keep >> i) & 1u)) continue;
                            const uint32_t r = (i * NW + warp) * 32 + lane;
                            const int32_t v = (int32_t)col[sh_col_index(r, sh, pd)];
                            bool k = !filt || (v >= lo && v <= hi);
                            if (k) {
                                if (v != mv) {
                                    int32_t pp = v;
                                    mk = sh_probe(ht, htlog, htlay, v, &pp);
                                    mv = v;
                                }
                                k = mk;
                            }
                            if (!k) keep &= ~(1u << i);
                        }
                    } else {
                        // general step: probes (one-entry memo: a thread's rows are NT apart,
                        // so on sorted or run-length columns they mostly repeat the key),
                        // group-key digits, COUNT, grouped aggregation
                        int32_t mv = kEmptyKey, mp = 0;
                        bool mk = false;
#pragma unroll
                        for (int i = 0; i < RPT; ++i) {
                            const uint32_t r = (i * NW + warp) * 32 + lane;
                            bool k = (keep >> i) & 1u;
                            int32_t v = k ? (int32_t)col[sh_col_index(r, sh, pd)] : 0;
                            if (filt) k = k && v >= lo && v <= hi;
                            int32_t p = v;
                            if ((flags & GX_STEP_PROBE) && k) {
                                if (v != mv) {
                                    mp = v;
                                    mk = sh_probe(ht, htlog, htlay, v, &mp);
                                    mv = v;
                                }
                                k = mk;
                                p = mp;
                            }
                            if ((keep >> i) & 1u) {  // alive on entry: digits, carry, and the new alive bit
                                if (dcard && k) {
                                    const uint32_t dgt = (uint32_t)(p - dbase);
                                    if (dgt >= dcard) {
                                        raise_error(kErrInvalid);
                                        k = false;
                                    } else {
                                        gk[i] = gk[i] * dcard + dgt;
                                    }
                                }
                                if (carry_step && k) carry[i] = v;
                                if (!k) keep &= ~(1u << i);
                            }
                            if (last) {  // the VALUE step: aggregate the row
                                const int64_t val = !k ? 0
                                                  : agg == GX_AGG_SUM_PRODUCT ? (int64_t)v * carry[i]
                                                  : agg == GX_AGG_SUM_DIFF    ? (int64_t)v - carry[i]
                                                  : agg == GX_AGG_COUNT        ? 1
                                                                               : (int64_t)v;
                                if (!grouped) local += val;
                                else if (k) {
                                    const QView Qa = sh_qv<SINGLE>(P, s_qc, cq);  // re-read: not kept live
                                    sh_group_add(gk[i], val, s_gsum, Qa.g_keys, Qa.g_sums, Qa.g_log2);
                                }
                            }
                        }
                    }
                }
                if (pre) {
                    // hand the shared steps' result to the members (each thread keeps its own rows)
#pragma unroll
                    for (int i = 0; i < RPT; ++i) {
                        const uint32_t r = (i * NW + warp) * 32 + lane;
                        if (psave & 1u) s_pst[r] = gk[i];
                        if (psave & 2u) s_pst[P.pst_carry + r] = (uint32_t)carry[i];
                    }
                    keep_pre = keep;
                    if (dropped || !__syncthreads_or(keep != 0)) break;  // no member has a live row
                    pre = false;
                    continue;
                }
                if (grouped) {
                    const QView Qa = sh_qv<SINGLE>(P, s_qc, cq);
                    sh_group_flush<NT>(s_gsum, s_gkey, Qa.g_keys, Qa.g_sums, Qa.g_log2);
                }
                if (!grouped && !dropped) {
                    unsigned long long u = (unsigned long long)local;
#pragma unroll
                    for (int d = 16; d > 0; d >>= 1) u += __shfl_down_sync(0xFFFFFFFFu, u, d);
                    if (lane == 0 && u) atomicAdd(&s_part[cq], u);
                }
                if (dropped || !rest) break;
                cq = w * 32 + (__ffs(rest) - 1);
                rest &= rest - 1;
                }  // jobs of the group
            }
        }
        }  // r0 < rows
        __syncthreads();
        if (tid == 0) {
            if (SINGLE) {
                ++s_li;
                if (s_fatal) {  // stop this CTA: nothing left in the list or in later rounds
                    s_li = s_ln;
                    s_w0 = total;
                }
            } else {
                s_item = s_fatal ? 0xFFFFFFFFu : next_it;
                s_cols = 0;
            }
        }
        __syncthreads();
    }
    __syncthreads();
    for (uint32_t q = tid; q < P.n_queries; q += NT) {
        const unsigned long long v = s_part[q];
        const ShQuery& Q = sh_q<SINGLE>(P, q);
        if (v && Q.result) atomicAdd((unsigned long long*)Q.result, v);
    }
    if (tid == 0 && P.rows_scanned && local_rows) atomicAdd(P.rows_scanned, local_rows);
}
