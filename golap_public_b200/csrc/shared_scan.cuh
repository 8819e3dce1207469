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
constexpr uint32_t kShNT = 256;           // threads per CTA
constexpr uint32_t kShColWords = kShTile + 256;  // one column buffer (with segment padding)

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
};

struct ShParams {
    const gx_dcol* cols;        // the batch's column table (global memory)
    uint32_t n_cols;
    const ShQuery* qs;
    uint32_t n_queries;
    uint32_t mask_words;        // ceil(n_queries / 32)
    const uint32_t* slot_mask;  // n_slots * mask_words
    const uint32_t* items;      // compacted slots
    const uint32_t* n_items;
    uint32_t* work_counter;
    uint32_t blocks_per_chunk, rows_per_chunk, rows_per_block;
    uint32_t tile_rows, tiles_per_block;
    unsigned long long* rows_scanned;  // optional: sum over (query, tile) of the query's rows in the tile
};

// One warp per block slot: lane l tests query 32*w + l of mask word w; the
// word is the warp ballot.  Slots with any query set are appended to items.
__global__ void shared_items_kernel(const gx_dblock* __restrict__ dir, uint32_t n_slots, const ShQuery* __restrict__ qs,
                                    uint32_t n_queries, uint32_t mask_words, uint32_t blocks_per_chunk,
                                    uint32_t rows_per_chunk, uint32_t rows_per_block, uint32_t* slot_mask,
                                    uint32_t* items, uint32_t* n_items) {
    const uint32_t lane = threadIdx.x & 31;
    const uint32_t warps = gridDim.x * (blockDim.x / 32);
    for (uint32_t s = blockIdx.x * (blockDim.x / 32) + threadIdx.x / 32; s < n_slots; s += warps) {
        const uint32_t rows = dir[s].n_rows;
        const uint32_t chunk = s / blocks_per_chunk, j = s % blocks_per_chunk;
        const uint64_t g0 = (uint64_t)chunk * rows_per_chunk + (uint64_t)j * rows_per_block, g1 = g0 + rows;
        bool any = false;
        for (uint32_t w = 0; w < mask_words; ++w) {
            const uint32_t q = w * 32 + lane;
            bool keep = false;
            if (q < n_queries && rows) {
                const ShQuery& Q = qs[q];
                keep = Q.row_lo < g1 && Q.row_hi > g0;
                if (keep && Q.keep_in) keep = Q.keep_in[chunk] != 0;
                for (uint32_t p = 0; keep && p < Q.n_prune; ++p) {
                    const PrunePred& pr = Q.prune[p];
                    keep = pr.lo <= pr.maxs[chunk] && pr.hi >= pr.mins[chunk];
                    if (keep && pr.bmins) keep = pr.lo <= pr.bmaxs[s] && pr.hi >= pr.bmins[s];
                }
            }
            const uint32_t m = __ballot_sync(0xFFFFFFFFu, keep);
            if (lane == 0) slot_mask[(size_t)s * mask_words + w] = m;
            any = any || m;
        }
        if (any && lane == 0) items[atomicAdd(n_items, 1u)] = s;
    }
}

__device__ __forceinline__ uint32_t sh_col_index(uint32_t r, uint32_t sh, uint32_t pd) {
    return r + ((r >> sh) << pd);
}

// Evaluate query Q on rows [a, b) of the decoded tile.  Called by all NT
// threads; every warp runs the same number of row-group iterations.
template <int NT>
__device__ __forceinline__ void shared_eval_query(const ShQuery& Q, uint32_t q, uint32_t a, uint32_t b,
                                                  const uint32_t* __restrict__ colbuf, const uint32_t* s_sh,
                                                  const uint32_t* s_pd, unsigned long long* s_part) {
    const uint32_t tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const uint32_t ns = Q.n_steps;
    const uint32_t agg = Q.agg;
    const bool grouped = Q.grouped != 0;
    int64_t local = 0;
    for (uint32_t base = (a & ~31u) + warp * 32; base < b; base += NT) {
        const uint32_t r = base + lane;
        bool keep = r >= a && r < b;
        int64_t carry = 0, val = 0;
        uint32_t gk = 0;
        for (uint32_t s = 0; s < ns && keep; ++s) {
            const ShStep& st = Q.steps[s];
            const uint32_t c = st.col;
            const int32_t v = (int32_t)colbuf[c * kShColWords + sh_col_index(r, s_sh[c], s_pd[c])];
            const uint32_t flags = st.flags;
            if (flags & GX_STEP_FILTER) keep = v >= st.lo && v <= st.hi;
            int32_t p = v;
            if ((flags & GX_STEP_PROBE) && keep) keep = ht_probe_any(st.ht, st.ht_log2, st.ht_layout, v, &p);
            if (st.digit_card && keep) {
                const uint32_t dgt = (uint32_t)(p - st.digit_base);
                if (dgt >= st.digit_card) {
                    raise_error(kErrInvalid);
                    keep = false;
                } else {
                    gk = gk * st.digit_card + dgt;
                }
            }
            if ((flags & GX_STEP_CARRY) && keep) carry = v;
            if ((flags & GX_STEP_VALUE) && keep)
                val = agg == GX_AGG_SUM_PRODUCT ? (int64_t)v * carry : (agg == GX_AGG_COUNT ? 1 : (int64_t)v);
        }
        if (!grouped) {
            local += keep ? val : 0;
        } else {
            uint32_t active = __ballot_sync(0xFFFFFFFFu, keep);
            while (active) {
                const int leader = __ffs(active) - 1;
                const uint32_t lk = __shfl_sync(0xFFFFFFFFu, gk, leader);
                const bool peer = keep && gk == lk && ((active >> lane) & 1u);
                const uint32_t peers = __ballot_sync(0xFFFFFFFFu, peer);
                const uint64_t tot = warp_sum_u64(peer ? (uint64_t)val : 0ull);
                if ((int)lane == leader && !group_add_global(Q.g_keys, Q.g_sums, Q.g_log2, (int64_t)lk, (int64_t)tot))
                    raise_error(kErrCapacity);
                active &= ~peers;
            }
        }
    }
    if (!grouped) {
        unsigned long long u = (unsigned long long)local;
#pragma unroll
        for (int d = 16; d > 0; d >>= 1) u += __shfl_down_sync(0xFFFFFFFFu, u, d);
        if (lane == 0 && u) atomicAdd(&s_part[q], u);
    }
}

// Persistent shared-scan kernel: kShNT threads, tiles of up to kShTile rows.
// Dynamic shared memory: n_cols column buffers | stage | per-query partial
// sums | per-tile active-query mask.
__global__ void __launch_bounds__(kShNT, 2) shared_scan_kernel(const __grid_constant__ ShParams P) {
    constexpr int NT = kShNT;
    constexpr int NW = NT / 32;
    using C = Cfg<kTileRows>;  // stage sized for 4096-row tiles (holds the cascaded run tables)
    extern __shared__ __align__(16) uint8_t smem[];
    uint32_t* colbuf = (uint32_t*)smem;
    uint8_t* stage = (uint8_t*)(colbuf + (size_t)P.n_cols * kShColWords);
    unsigned long long* s_part = (unsigned long long*)(stage + C::kStage);
    uint32_t* s_qmask = (uint32_t*)(s_part + P.n_queries);

    __shared__ __align__(8) uint64_t s_mbar;
    __shared__ uint32_t s_item;
    __shared__ int s_err;
    __shared__ int s_fatal;
    __shared__ uint32_t s_colmask;
    __shared__ uint32_t s_sh[kShMaxCols], s_pd[kShMaxCols];
    __shared__ uint32_t s_tmp[NW + 1];
    __shared__ CascTile s_ct;

    const uint32_t tid = threadIdx.x;
    for (uint32_t i = tid; i < P.n_queries; i += NT) s_part[i] = 0;
    if (tid == 0) {
        s_err = 0;
        s_fatal = 0;
        mbar_init(&s_mbar, 1);
    }
    uint32_t phase = 0;
    unsigned long long local_rows = 0;
    const uint32_t tpb = P.tiles_per_block, tile_rows = P.tile_rows;
    const uint32_t total = *P.n_items * tpb;
    const uint32_t MW = P.mask_words;
    __syncthreads();

    while (true) {
        if (tid == 0) {
            s_item = s_fatal ? 0xFFFFFFFFu : atomicAdd(P.work_counter, 1u);
            s_colmask = 0;
        }
        __syncthreads();
        const uint32_t it = s_item;
        if (it >= total) break;
        const uint32_t slot = P.items[it / tpb];
        const uint32_t r0 = (it % tpb) * tile_rows;
        const uint32_t rows = P.cols[0].blocks[slot].n_rows;
        if (r0 >= rows) {
            __syncthreads();
            continue;
        }
        const uint32_t n = min(tile_rows, rows - r0);
        const uint32_t chunk = slot / P.blocks_per_chunk, j = slot % P.blocks_per_chunk;
        const uint64_t g0 = (uint64_t)chunk * P.rows_per_chunk + (uint64_t)j * P.rows_per_block + r0;
        // active queries of this tile (slice overlap within the block) and the columns they read
        uint32_t cm = 0;
        for (uint32_t w = tid; w < MW; w += NT) {
            uint32_t m = P.slot_mask[(size_t)slot * MW + w], keepm = m;
            while (m) {
                const uint32_t bit = __ffs(m) - 1;
                m &= m - 1;
                const ShQuery& Q = P.qs[w * 32 + bit];
                if (Q.row_lo < g0 + n && Q.row_hi > g0) cm |= Q.col_mask;
                else keepm &= ~(1u << bit);
            }
            s_qmask[w] = keepm;
        }
        if (cm) atomicOr(&s_colmask, cm);
        __syncthreads();
        uint32_t cols = s_colmask;
        bool dropped = false;
        while (cols) {
            const uint32_t c = __ffs(cols) - 1;
            cols &= cols - 1;
            const gx_dcol& col = P.cols[c];
            uint32_t* buf = colbuf + c * kShColWords;
            uint32_t pad_log2 = 0;
            int layout = decode_tile<NT, kTileRows>(col, slot, rows, r0, n, buf, stage, &s_mbar, phase, s_tmp, &s_ct,
                                                    &s_err, pad_log2);
            const int derr = s_err;
            __syncthreads();
            if (derr) {
                if (tid == 0) {
                    raise_error(derr);
                    s_err = 0;
                    if (derr == kErrTimeout) s_fatal = 1;
                }
                __syncthreads();
                dropped = true;
                break;
            }
            if (layout == kRuns) {
                casc_runs_to_rows<NT>(s_ct, (const int32_t*)stage, (const uint32_t*)(stage + 4 * kCascMaxRuns), r0, n,
                                      (int32_t*)buf);
                layout = kRows;
            }
            if (tid == 0) {
                s_sh[c] = layout == kSegRows ? col.seg_shift : 31u;
                s_pd[c] = layout == kSegRows ? pad_log2 : 0u;
            }
            __syncthreads();
        }
        if (!dropped) {
            for (uint32_t w = 0; w < MW; ++w) {
                uint32_t m = s_qmask[w];
                while (m) {
                    const uint32_t q = w * 32 + (__ffs(m) - 1);
                    m &= m - 1;
                    const ShQuery& Q = P.qs[q];
                    const uint32_t a = Q.row_lo > g0 ? (uint32_t)(Q.row_lo - g0) : 0u;
                    const uint32_t b = Q.row_hi < g0 + n ? (uint32_t)(Q.row_hi - g0) : n;
                    if (tid == 0) local_rows += b - a;
                    shared_eval_query<NT>(Q, q, a, b, colbuf, s_sh, s_pd, s_part);
                }
            }
        }
        __syncthreads();
    }
    __syncthreads();
    for (uint32_t q = tid; q < P.n_queries; q += NT) {
        const unsigned long long v = s_part[q];
        if (v && P.qs[q].result) atomicAdd((unsigned long long*)P.qs[q].result, v);
    }
    if (tid == 0 && P.rows_scanned && local_rows) atomicAdd(P.rows_scanned, local_rows);
}
