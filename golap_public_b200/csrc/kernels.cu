// kernels.cu -- sm_100a kernels of the hot path and the C-ABI entry points
// that launch them.
//
//   shared_scan_kernel (shared_scan.cuh) the fused scan: per 2048-row tile,
//                      decode into shared memory -> filter -> probe ->
//                      aggregate, one query (which prunes its own work) or a
//                      batch (work list from shared_items_kernel)
//                      (replaces ChunkDecompressor + pipeline_q1_lineorder,
//                      usecases/ssb/queries/01.cuh:27-54, and pipeline_q3,
//                      usecases/ssb/queries/03.cuh:119-170)
//   scan_kernel        the per-query (queue) form of the same fused scan
//   items_kernel       min/max pruning + compaction of surviving chunks
//                      (check_mmmeta/combine_and, core/metadata.cuh:540-547,632-636)
//   decompress_kernel  chunk decompression to global memory
//                      (ChunkDecompressor::step, core/comp.cuh:171-195)
//   ht_build_kernel / ht_build_small_kernel / ht_build_dense_kernel / ht_probe_kernel
//                      (hash_map_build_pred_other core/join.cuh:107-135,
//                       hash_join_count core/join.cuh:46-59)
//   groupby_add_kernel (group_by_agg_2col core/group.cuh:15-24 with SumAgg)
//
// A work unit is a row tile: one (chunk, block, tile) triple covering up to
// kTileRows rows of every column of the table.  Segmented LZ4 blocks are
// decoded tile by tile (a tile holds whole segments), so four CTAs fit on
// an SM; plans with plain LZ4 or segments longer than a tile fall back to
// whole-block tiles.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cstring>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "../../include/gx.h"
#include "gx_device.cuh"
#include "gx_internal.h"

using namespace gx;

// First error raised by any kernel of this library on the current device.
__device__ int g_gx_error;

__device__ __forceinline__ void raise_error(int code) { atomicCAS(&g_gx_error, 0, code); }

#define GX_CK(call)                                                                       \
    do {                                                                                  \
        cudaError_t e_ = (call);                                                          \
        if (e_ != cudaSuccess)                                                            \
            return gx::set_error(GX_ERR_CUDA, "%s failed: %s", #call, cudaGetErrorString(e_)); \
    } while (0)

// Scratch memory of the library's launches comes from a per-device memory
// pool that keeps up to 256 MiB cached across synchronisations: the default
// pool returns its memory at every synchronisation, so every call after one
// would map fresh memory (hundreds of microseconds).
// Per-device caches (memory pools, kernel attributes, occupancies, the
// static scratch address) hold kMaxDevices entries; every one of them
// refuses a device index outside that range in the same way.
constexpr int kMaxDevices = 64;
static inline bool device_index_ok(int dev) { return dev >= 0 && dev < kMaxDevices; }

static cudaError_t scratch_alloc(void** p, size_t bytes, cudaStream_t s) {
    static std::mutex mu;
    static cudaMemPool_t pools[kMaxDevices] = {};
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (!device_index_ok(dev)) return cudaErrorInvalidDevice;
    cudaMemPool_t pool;
    {
        std::lock_guard<std::mutex> lk(mu);
        if (!pools[dev]) {
            cudaMemPoolProps props{};
            props.allocType = cudaMemAllocationTypePinned;
            props.location.type = cudaMemLocationTypeDevice;
            props.location.id = dev;
            e = cudaMemPoolCreate(&pools[dev], &props);
            if (e != cudaSuccess) return e;
            uint64_t keep = 256ull << 20;
            cudaMemPoolSetAttribute(pools[dev], cudaMemPoolAttrReleaseThreshold, &keep);
        }
        pool = pools[dev];
    }
    return cudaMallocFromPoolAsync(p, bytes, pool, s);
}

namespace {

constexpr uint32_t kTileRows = 4096;      // tile of the small configuration
constexpr uint32_t kSmemGroupLog2 = 10;   // 1024-slot shared partial group table

// Shared-memory budget of one CTA for tiles of up to MAXT rows.
template <int MAXT>
struct Cfg {
    static constexpr uint32_t kBufWords = MAXT + 256;  // segment padding: nseg * lanes per segment <= 256
    static constexpr uint32_t kMaskWords = MAXT / 32;
    static constexpr uint32_t kStage = MAXT * 4 + MAXT * 4 / 128 + 256;      // compressed window + slack
    static_assert(4 * kCascMaxRuns + 4 * (kCascMaxRuns + 4) <= kStage, "run tables fit the stage");
    static_assert(MAXT * 4 <= kStage, "raw tile fits the stage");
};
static_assert(Cfg<kMaxRowsPerBlock>::kStage >= kStageBytes, "a whole block fits the large stage");

struct ScanStep {
    gx_dcol col;
    uint32_t flags;
    int32_t lo, hi;
    const uint64_t* ht;
    uint32_t ht_log2;
    uint32_t ht_layout;
    int32_t digit_base;
    uint32_t digit_card;
    uint32_t first_digit;
};

struct PrunePred {
    const int32_t* mins;   // per chunk (the reference's MinMaxMeta granularity)
    const int32_t* maxs;
    int32_t lo, hi;
    const int32_t* bmins;  // per block slot (zone map), or null
    const int32_t* bmaxs;
};

// One query: its steps, the row slice it covers, where its aggregate goes.
struct QueryDesc {
    ScanStep steps[GX_MAX_STEPS];
    uint32_t n_steps;
    uint32_t agg;
    uint32_t grouped;       // sums per group key
    uint32_t need_aux;      // aux array (carry or group key) in shared memory
    uint32_t carry_digits;  // a carried value and group-key digits (not in the queue form's one aux array)
    uint64_t row_lo, row_hi;
    int64_t* result;
    int64_t* g_keys;
    int64_t* g_sums;
    uint32_t g_log2;
    uint32_t n_prune;
    PrunePred prune[GX_MAX_STEPS];
};

struct ScanParams {
    QueryDesc q;             // the query (single mode)
    const QueryDesc* qs;     // the queries (batch mode)
    const uint32_t* item_q;  // batch mode: query of each work item
    uint32_t blocks_per_chunk;
    uint32_t rows_per_chunk;
    uint32_t rows_per_block;
    uint32_t tile_rows;
    uint32_t tiles_per_block;
    uint32_t smem_aux;       // shared-memory layout: aux array present
    uint32_t smem_groups;    // shared-memory layout: partial group table present
    const uint32_t* items;   // surviving chunk ids
    const uint32_t* n_items;
    uint32_t* work_counter;
    unsigned long long* rows_scanned;
};

struct ItemsParams {
    const uint16_t* keep_in;
    uint16_t* keep_out;
    PrunePred preds[GX_MAX_STEPS];
    uint32_t n_preds;
    uint32_t n_chunks;
    uint32_t* items;
    uint32_t* n_items;
    uint32_t* work_counter;
};

// Layout of a decoded tile in shared memory.
enum : int { kRows = 0, kSegRows = 1 };

// Stage `bytes` bytes from `src` (16-byte aligned, bytes a multiple of 16
// and within the stage) into shared memory.  HBM-resident columns: thread 0
// issues one cp.async.bulk and every thread waits on the mbarrier (bounded);
// host-mapped columns: cooperative 16-byte loads.  All NT threads call it.
// Returns 0 or kErrTimeout.
template <int NT>
__device__ __forceinline__ int stage_bytes(const gx_dcol& c, const uint8_t* src, uint32_t bytes, uint8_t* stage,
                                           uint64_t* mbar, uint32_t& phase) {
    const uint32_t tid = threadIdx.x;
    int rc = 0;
    if (!c.host_mapped) {
        // earlier generic-proxy reads of `stage` by any thread are ordered
        // before the bulk copy that overwrites it
        fence_proxy_async_smem();
        __syncthreads();
        if (tid == 0) tma_load_1d(stage, src, bytes, mbar);
        if (!mbar_wait_bounded(mbar, phase)) {
            // give the copy one more bounded chance to land before the buffer is abandoned
            mbar_wait_bounded(mbar, phase);
            rc = kErrTimeout;
        }
        phase ^= 1u;
    } else {
        __syncthreads();
        const uint4* s = (const uint4*)src;
        uint4* d = (uint4*)stage;
        for (uint32_t i = tid; i < bytes / 16; i += NT) d[i] = s[i];
    }
    return rc;
}

// Decode rows [r0, r0+n) of block `slot` of column `c` into shared memory.
// Returns the layout (kRows: buf[r]; kSegRows: buf[r + ((r >> seg_shift) <<
// pad_log2)], each segment followed by 2^pad_log2 pad words) or -1 with
// *s_err set.  All NT threads call it.
template <int NT, int MAXT>
__device__ __forceinline__ int decode_tile(const gx_dcol& c, uint32_t slot, uint32_t rows, uint32_t r0, uint32_t n,
                                           uint32_t* buf, uint8_t* stage, uint64_t* mbar, uint32_t& phase,
                                           uint32_t* tmp, int* s_err, uint32_t& pad_log2, uint32_t* seg_smem) {
    using C = Cfg<MAXT>;
    const uint32_t tid = threadIdx.x;
    // segmented LZ4: this thread's entry of the tile's segment index, loaded
    // together with the directory entry (the two reads do not depend on each
    // other, so their latencies overlap)
    const bool segd = c.codec == GX_CODEC_LZ4 && c.S > 1;
    uint32_t se0 = 0, se1 = 0;
    bool se_in = false;
    if (segd && tid <= kMaxSegments) {
        const uint32_t j = (r0 >> c.seg_shift) + tid;
        const uint32_t nseg_t = (n + (1u << c.seg_shift) - 1) >> c.seg_shift;
        if (tid <= nseg_t && j < c.S) {
            const uint32_t* e = c.seg + (size_t)2 * c.S * slot + 2 * j;
            se0 = __ldg(e);
            se1 = __ldg(e + 1);
            se_in = true;
        }
    }
    const gx_dblock d = c.blocks[slot];
    const uint8_t* blk = c.payload + d.offset;
    // directory sanity: the stream lies inside the payload (whose slack
    // covers the decoders' over-read) and the tile fits the buffers
    if (d.n_rows != rows || rows > kMaxRowsPerBlock || n > MAXT || d.offset > c.payload_bytes ||
        (uint64_t)d.comp_bytes + 32 > c.payload_bytes - d.offset) {
        if (tid == 0) *s_err = kErrCorrupt;
        __syncthreads();
        return -1;
    }
    if (c.codec == GX_CODEC_NONE) {
        if (d.comp_bytes != rows * 4) {
            if (tid == 0) *s_err = kErrCorrupt;
        } else {
            const uint32_t* src = (const uint32_t*)blk + r0;
            if ((r0 & 3u) == 0) {
                const uint32_t nv = n / 4;
                for (uint32_t i = tid; i < nv; i += NT) ((uint4*)buf)[i] = __ldg((const uint4*)src + i);
                for (uint32_t i = nv * 4 + tid; i < n; i += NT) buf[i] = __ldg(src + i);
            } else {
                for (uint32_t i = tid; i < n; i += NT) buf[i] = __ldg(src + i);
            }
        }
        __syncthreads();
        return kRows;
    }
    if (c.codec == GX_CODEC_LZ4) {
        uint32_t lo = 0, hi = d.comp_bytes, j0 = 0, nseg = 0, seg_rows = 0;
        if (c.S > 1) {
            seg_rows = 1u << c.seg_shift;
            j0 = r0 >> c.seg_shift;
            nseg = (n + seg_rows - 1) >> c.seg_shift;
            // the tile's nseg + 1 segment entries into shared memory (entries past
            // the block's last segment stand for its end); threads beyond the first
            // NT entries fetch theirs here
            const uint32_t* e = c.seg + (size_t)2 * c.S * slot;
            for (uint32_t t = tid; t <= nseg && t <= kMaxSegments; t += NT) {
                const uint32_t j = j0 + t;
                const bool mine = t == tid && se_in;
                seg_smem[2 * t] = mine ? se0 : (j < c.S ? __ldg(e + 2 * j) : d.comp_bytes);
                seg_smem[2 * t + 1] = mine ? se1 : (j < c.S ? __ldg(e + 2 * j + 1) : 0u);
            }
            __syncthreads();
            lo = seg_smem[0];
            hi = nseg <= kMaxSegments ? seg_smem[2 * nseg] : 0u;
            if ((r0 & (seg_rows - 1)) || j0 + nseg > c.S || nseg > kMaxSegments || lo > hi || hi > d.comp_bytes) {
                if (tid == 0) *s_err = kErrCorrupt;
                __syncthreads();
                return -1;
            }
        } else if (r0 != 0 || n != rows) {  // plain LZ4 decodes whole blocks only
            if (tid == 0) *s_err = kErrInvalid;
            __syncthreads();
            return -1;
        }
        // the staged window starts on the 16-byte boundary at or below the tile's
        // first byte (LZ4 blocks need not start on one); wbase is that boundary
        // relative to the block start, in wrapping arithmetic (the decoders only
        // form differences pos - wbase)
        const uint64_t abs_lo = d.offset + lo;
        const uint64_t abs_wb = abs_lo & ~15ull;
        const uint32_t wbase = (uint32_t)(abs_wb - d.offset);
        const uint32_t bytes = (uint32_t)(((d.offset + hi + 15u) & ~15ull) - abs_wb) + 16u;
        if (bytes > C::kStage) {
            if (tid == 0) *s_err = kErrCorrupt;
            __syncthreads();
            return -1;
        }
        const int rc = stage_bytes<NT>(c, c.payload + abs_wb, bytes, stage, mbar, phase);
        if (rc && tid == 0) *s_err = rc;
        __syncthreads();
        if (rc) return -1;
        if (c.S > 1) {
            // one literal run covers the whole tile (the first entry resumes inside a
            // run long enough, and the tile's bytes are exactly its rows): a flat,
            // vectorised copy of n words from byte lo, rows in plain order
            const uint32_t info0 = seg_smem[1];
            if ((info0 & 16u) && (info0 >> 5) >= 4 * n && hi - lo == 4 * n && (n & 3u) == 0 && lo == seg_smem[0]) {
                const uint32_t* A = (const uint32_t*)stage;
                const uint32_t rb = (uint32_t)(abs_lo - abs_wb), w0 = rb >> 2, sh = (rb & 3u) * 8;
                for (uint32_t q4 = tid; q4 < n / 4; q4 += NT) {
                    const uint32_t w = w0 + 4 * q4;
                    const uint32_t a0 = A[w], a1 = A[w + 1], a2 = A[w + 2], a3 = A[w + 3], a4 = A[w + 4];
                    ((uint4*)buf)[q4] = make_uint4(__funnelshift_r(a0, a1, sh), __funnelshift_r(a1, a2, sh),
                                                   __funnelshift_r(a2, a3, sh), __funnelshift_r(a3, a4, sh));
                }
                __syncthreads();
                return kRows;
            }
            // a group of G adjacent lanes per segment; segment t at buf + t * (seg_rows + G)
            // lanes per segment: a whole warp when the tile is mostly literals
            // (few sequences; conflict-free 32-word copies), else spread the
            // segments over all NT threads
            const bool literal_tile = (uint64_t)(hi - lo) * 8 >= (uint64_t)n * 4 * 7;
            // padding (nseg << glog words, or nseg for whole-warp groups) must fit the
            // 256 words every decode buffer reserves beyond its rows
            uint32_t glog = literal_tile ? 5u : seg_group_log2(nseg, NT);
            while (glog > 0 && glog < 5 && (nseg << glog) > 256u) --glog;
            const uint32_t G = 1u << glog;
            // pad words after each segment: G (groups of a warp on distinct
            // banks), 1 for a whole-warp group (its stores are contiguous)
            const uint32_t pl = glog == 5 ? 0u : glog;
            const uint32_t gl = tid & (G - 1u), lane = tid & 31u;
            const uint32_t gmask = G >= 32 ? 0xFFFFFFFFu : (((1u << G) - 1u) << (lane & ~(G - 1u)));
            for (uint32_t t = tid >> glog; t < nseg; t += (NT >> glog)) {
                const uint32_t j = j0 + t;
                const uint32_t K = min(seg_rows, rows - j * seg_rows);
                const int r2 = lz4_seg_group((const uint32_t*)stage, wbase, lo, hi, d.comp_bytes, seg_smem[2 * t],
                                             seg_smem[2 * t + 1], K, buf + t * (seg_rows + (1u << pl)), gl, G, gmask);
                if (r2 && gl == 0) *s_err = r2;
            }
            pad_log2 = pl;
            __syncthreads();
            return kSegRows;
        }
        if (tid < 32) {
            const int r2 = lz4_warp_block(SharedSrc{stage + (uint32_t)(d.offset - abs_wb)}, d.comp_bytes,
                                          (uint8_t*)buf, rows * 4, tid);
            if (r2 && tid == 0) *s_err = r2;
        }
        __syncthreads();
        return kRows;
    }
    // cascaded: the tile's pages one after another (tiles start on page
    // boundaries); run tables live in the (idle) stage area
    int32_t* run_val = (int32_t*)stage;
    uint32_t* run_end = (uint32_t*)(stage + 4 * kCascMaxRuns);
    const uint32_t p0 = r0 >> kCascPageLog2, p1 = (r0 + n + kCascPageRows - 1) >> kCascPageLog2;
    if ((r0 & (kCascPageRows - 1)) || !c.seg || p1 > c.S) {
        if (tid == 0) *s_err = kErrCorrupt;
        __syncthreads();
        return -1;
    }
    for (uint32_t p = p0; p < p1; ++p) {
        const uint32_t* e = c.seg + (size_t)2 * c.S * slot + 2 * p;
        const uint32_t off = __ldg(e), pb = __ldg(e + 1);
        const uint32_t pr = min(kCascPageRows, rows - p * kCascPageRows);
        int rc = kErrCorrupt;
        if ((off & 15u) == 0 && (uint64_t)off + pb <= d.comp_bytes)
            rc = casc_decode_page<NT>(blk + off, pb, pr, (int32_t*)buf + (p * kCascPageRows - r0), run_val, run_end,
                                      tmp);
        if (rc) {
            if (tid == 0) *s_err = rc;
            __syncthreads();
            return -1;
        }
    }
    return kRows;
}

// Flush a CTA's partial aggregate of query Q: the scalar sum (one global
// atomic) or the shared partial group table (merged into Q's global table,
// then cleared).  All NT threads call it.
template <int NT>
__device__ __forceinline__ void flush_query(const QueryDesc& Q, int64_t& local_sum, uint32_t* gkeys,
                                            unsigned long long* gsums, unsigned long long* s_red) {
    constexpr int NW = NT / 32;
    const uint32_t tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if (!Q.grouped) {
        unsigned long long u = (unsigned long long)local_sum;
#pragma unroll
        for (int d = 16; d > 0; d >>= 1) u += __shfl_down_sync(0xFFFFFFFFu, u, d);
        if (lane == 0) s_red[warp] = u;
        __syncthreads();
        if (tid == 0 && Q.result) {
            unsigned long long t = 0;
            for (int w = 0; w < NW; ++w) t += s_red[w];
            if (t) atomicAdd((unsigned long long*)Q.result, t);
        }
        local_sum = 0;
        __syncthreads();
    } else {
        __syncthreads();
        for (uint32_t i = tid; i < (1u << kSmemGroupLog2); i += NT) {
            if (gkeys[i] != kEmptyGKey) {
                if (!group_add_global(Q.g_keys, Q.g_sums, Q.g_log2, (int64_t)gkeys[i], (int64_t)gsums[i]))
                    raise_error(kErrCapacity);
                gkeys[i] = kEmptyGKey;
                gsums[i] = 0;
            }
        }
        __syncthreads();
    }
}

// The fused scan.  Persistent CTAs take row tiles from a work list (one
// entry per surviving chunk of a query); per tile, every step of the query
// decodes its column into shared memory and updates the selection mask;
// the VALUE step aggregates.  BATCH: the tile's query comes from the work
// list and query descriptors live in global memory.
template <int NT, int MAXT, bool BATCH>
__global__ void __launch_bounds__(NT, (MAXT < 16384 ? 4 : 1)) scan_kernel(const __grid_constant__ ScanParams P) {
    using C = Cfg<MAXT>;
    constexpr int NW = NT / 32;
    extern __shared__ __align__(16) uint8_t smem[];
    uint32_t* buf = (uint32_t*)smem;
    uint32_t* aux = buf + C::kBufWords;
    uint32_t* mask = aux + (P.smem_aux ? MAXT : 0);
    uint8_t* stage = (uint8_t*)(mask + C::kMaskWords);
    uint32_t* gkeys = (uint32_t*)(stage + C::kStage);
    unsigned long long* gsums = (unsigned long long*)(gkeys + (P.smem_groups ? (1u << kSmemGroupLog2) : 0));

    __shared__ __align__(8) uint64_t s_mbar;
    __shared__ uint32_t s_item;
    __shared__ int s_err;
    __shared__ int s_fatal;
    __shared__ uint32_t s_alive;
    __shared__ uint32_t s_tmp[NW + 1];
    __shared__ unsigned long long s_red[NW];
    __shared__ uint32_t s_seg[2 * (kMaxSegments + 1)];

    const uint32_t tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if (P.smem_groups) {
        for (uint32_t i = tid; i < (1u << kSmemGroupLog2); i += NT) {
            gkeys[i] = kEmptyGKey;
            gsums[i] = 0;
        }
    }
    if (tid == 0) {
        s_err = 0;
        s_fatal = 0;
        mbar_init(&s_mbar, 1);
    }
    uint32_t phase = 0;
    int64_t local_sum = 0;
    unsigned long long local_rows = 0;
    const uint32_t tpb = P.tiles_per_block, tile_rows = P.tile_rows;
    const uint32_t per_chunk = P.blocks_per_chunk * tpb;
    const uint32_t total = *P.n_items * per_chunk;
    int cur_q = -1;
    __syncthreads();

    while (true) {
        if (tid == 0) s_item = s_fatal ? 0xFFFFFFFFu : atomicAdd(P.work_counter, 1u);
        __syncthreads();
        const uint32_t it = s_item;
        __syncthreads();
        if (it >= total) break;
        const uint32_t k = it / per_chunk, rem = it % per_chunk;
        const int q = BATCH ? (int)P.item_q[k] : 0;
        if (q != cur_q) {  // uniform across the CTA
            if (cur_q >= 0) flush_query<NT>(BATCH ? P.qs[cur_q] : P.q, local_sum, gkeys, gsums, s_red);
            cur_q = q;
        }
        const QueryDesc& Q = BATCH ? P.qs[q] : P.q;
        const uint32_t chunk = P.items[k];
        const uint32_t j = rem / tpb;
        const uint32_t slot = chunk * P.blocks_per_chunk + j;
        const uint32_t r0 = (rem % tpb) * tile_rows;
        const uint32_t rows = Q.steps[0].col.blocks[slot].n_rows;
        if (r0 >= rows) continue;
        const uint32_t n = min(tile_rows, rows - r0);
        // rows of the tile inside the query's slice [row_lo, row_hi)
        const uint64_t g0 = (uint64_t)chunk * P.rows_per_chunk + (uint64_t)j * P.rows_per_block + r0;
        const uint32_t a = Q.row_lo > g0 ? (Q.row_lo - g0 < n ? (uint32_t)(Q.row_lo - g0) : n) : 0u;
        const uint32_t b = Q.row_hi > g0 ? (Q.row_hi - g0 < n ? (uint32_t)(Q.row_hi - g0) : n) : 0u;
        if (a >= b) continue;
        // block zone maps: a block outside a prune predicate's range holds no
        // row the plan keeps (prune predicates are implied by its filters)
        bool zone_out = false;
        for (uint32_t p = 0; p < Q.n_prune; ++p) {
            const PrunePred& pr = Q.prune[p];
            if (pr.bmins && (pr.lo > __ldg(pr.bmaxs + slot) || pr.hi < __ldg(pr.bmins + slot))) zone_out = true;
        }
        if (zone_out) continue;
        const uint32_t ngroups = (n + 31) / 32;
        for (uint32_t g = tid; g < ngroups; g += NT) {
            const uint32_t lo = max(a, g * 32), hi = min(b, g * 32 + 32);
            mask[g] = lo >= hi ? 0u : ((hi - lo == 32) ? 0xFFFFFFFFu : (((1u << (hi - lo)) - 1u) << (lo & 31)));
        }
        if (tid == 0) local_rows += b - a;
        __syncthreads();

        for (uint32_t si = 0; si < Q.n_steps; ++si) {
            const ScanStep& st = Q.steps[si];
            uint32_t pad_log2 = 0;
            const int layout = decode_tile<NT, MAXT>(st.col, slot, rows, r0, n, buf, stage, &s_mbar, phase, s_tmp,
                                                     &s_err, pad_log2, s_seg);
            const int derr = s_err;
            __syncthreads();  // every thread has read s_err before it is reset
            if (derr) {       // corrupt block: drop the tile, remember the error
                if (tid == 0) {
                    raise_error(derr);
                    s_err = 0;
                    if (derr == kErrTimeout) s_fatal = 1;  // the stage may still be written: stop this CTA
                }
                __syncthreads();
                break;
            }
            const uint32_t flags = st.flags;
            const uint32_t dcard = st.digit_card;
            if (tid == 0) s_alive = 0;
            __syncthreads();
            uint32_t alive_w = 0;
            {
                const uint32_t shift = st.col.seg_shift;
                for (uint32_t g = warp; g < ngroups; g += NW) {
                    const uint32_t m = mask[g];
                    if (m == 0) continue;
                    const uint32_t r = g * 32 + lane;
                    bool keep = (m >> lane) & 1u;
                    int32_t v = 0;
                    if (keep) v = (int32_t)buf[layout == kSegRows ? r + ((r >> shift) << pad_log2) : r];
                    if ((flags & GX_STEP_FILTER) && keep) keep = v >= st.lo && v <= st.hi;
                    int32_t p = v;
                    if ((flags & GX_STEP_PROBE) && keep) keep = ht_probe_any(st.ht, st.ht_log2, st.ht_layout, v, &p);
                    if (dcard && keep) {
                        const uint32_t dgt = (uint32_t)(p - st.digit_base);
                        if (dgt >= dcard) {
                            raise_error(kErrInvalid);
                            keep = false;
                        } else {
                            aux[r] = st.first_digit ? dgt : aux[r] * dcard + dgt;
                        }
                    }
                    if ((flags & GX_STEP_CARRY) && keep) aux[r] = (uint32_t)v;
                    if (flags & GX_STEP_VALUE) {
                        int64_t val = 0;
                        if (keep) {
                            if (Q.agg == GX_AGG_SUM_PRODUCT) val = (int64_t)v * (int64_t)(int32_t)aux[r];
                            else if (Q.agg == GX_AGG_SUM_DIFF) val = (int64_t)v - (int64_t)(int32_t)aux[r];
                            else if (Q.agg == GX_AGG_COUNT) val = 1;
                            else val = v;
                        }
                        if (!Q.grouped) {
                            local_sum += val;
                        } else {
                            // warp-aggregated update of the shared partial group table
                            const uint32_t gk = keep ? aux[r] : 0;
                            uint32_t active = __ballot_sync(0xFFFFFFFFu, keep);
                            while (active) {
                                const int leader = __ffs(active) - 1;
                                const uint32_t lk = __shfl_sync(0xFFFFFFFFu, gk, leader);
                                const bool peer = keep && gk == lk && ((active >> lane) & 1u);
                                const uint32_t peers = __ballot_sync(0xFFFFFFFFu, peer);
                                const uint64_t tot = warp_sum_u64(peer ? (uint64_t)val : 0ull);
                                if ((int)lane == leader) {
                                    if (!group_add_smem(gkeys, gsums, kSmemGroupLog2, lk, tot))
                                        if (!group_add_global(Q.g_keys, Q.g_sums, Q.g_log2, (int64_t)lk, (int64_t)tot))
                                            raise_error(kErrCapacity);
                                }
                                active &= ~peers;
                            }
                        }
                    }
                    const uint32_t nm = __ballot_sync(0xFFFFFFFFu, keep);
                    if (lane == 0) mask[g] = nm;
                    alive_w += __popc(nm);
                }
            }
            if (lane == 0 && alive_w) atomicAdd(&s_alive, alive_w);
            __syncthreads();
            if (s_alive == 0) break;  // nothing left in this tile
        }
        __syncthreads();
    }
    if (cur_q >= 0) flush_query<NT>(BATCH ? P.qs[cur_q] : P.q, local_sum, gkeys, gsums, s_red);
    if (tid == 0 && P.rows_scanned && local_rows) atomicAdd(P.rows_scanned, local_rows);
}

// One CTA: per-chunk keep flags (AND over min/max predicates and the
// optional input flags), order-preserving compaction of the surviving chunk
// ids, reset of the work counter.
__global__ void __launch_bounds__(1024) items_kernel(const __grid_constant__ ItemsParams P) {
    __shared__ uint32_t s_count;
    __shared__ uint32_t s_warp[32];
    if (threadIdx.x == 0) s_count = 0;
    __syncthreads();
    for (uint32_t base = 0; base < P.n_chunks; base += blockDim.x) {
        const uint32_t c = base + threadIdx.x;
        bool keep = false;
        if (c < P.n_chunks) {
            keep = P.keep_in ? P.keep_in[c] != 0 : true;
            for (uint32_t p = 0; p < P.n_preds; ++p) {
                const PrunePred& q = P.preds[p];
                keep = keep && (q.lo <= q.maxs[c]) && (q.hi >= q.mins[c]);
            }
            if (P.keep_out) P.keep_out[c] = keep ? 1 : 0;
        }
        const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
        const uint32_t b = __ballot_sync(0xFFFFFFFFu, keep);
        if (lane == 0) s_warp[warp] = __popc(b);
        __syncthreads();
        if (threadIdx.x == 0) {
            uint32_t run = s_count;
            for (uint32_t w = 0; w < blockDim.x / 32; ++w) {
                const uint32_t x = s_warp[w];
                s_warp[w] = run;
                run += x;
            }
            s_count = run;
        }
        __syncthreads();
        if (keep) P.items[s_warp[warp] + __popc(b & ((1u << lane) - 1u))] = c;
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        *P.n_items = s_count;
        *P.work_counter = 0;
    }
}

// Batch: per-query reset of the aggregate targets (scalar result = 0, group
// table emptied).  blockIdx.y = query; blocks along x stride the table.
__global__ void batch_reset_kernel(const QueryDesc* __restrict__ qs, unsigned long long* rows) {
    const QueryDesc& Q = qs[blockIdx.y];
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        if (Q.result) *Q.result = 0;
        if (blockIdx.y == 0 && rows) *rows = 0;
    }
    if (Q.grouped) {
        const uint64_t cap = 1ull << Q.g_log2;
        for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < cap; i += (uint64_t)gridDim.x * blockDim.x) {
            Q.g_keys[i] = kEmptyGroup;
            Q.g_sums[i] = 0;
        }
    }
}

// Batch: min/max pruning of every (query, chunk) candidate (the chunks that
// overlap the query's slice) and order-preserving compaction of the
// survivors into the work list; resets the work counter.  One CTA.
__global__ void __launch_bounds__(1024) batch_items_kernel(const QueryDesc* __restrict__ qs,
                                                           const uint32_t* __restrict__ cand_q,
                                                           const uint32_t* __restrict__ cand_chunk, uint32_t n_cand,
                                                           uint32_t* items_q, uint32_t* items_chunk, uint32_t* n_items,
                                                           uint32_t* work_counter) {
    __shared__ uint32_t s_count;
    __shared__ uint32_t s_warp[32];
    if (threadIdx.x == 0) s_count = 0;
    __syncthreads();
    for (uint32_t base = 0; base < n_cand; base += blockDim.x) {
        const uint32_t i = base + threadIdx.x;
        bool keep = false;
        uint32_t q = 0, c = 0;
        if (i < n_cand) {
            q = cand_q[i];
            c = cand_chunk[i];
            const QueryDesc& Q = qs[q];
            keep = true;
            for (uint32_t p = 0; p < Q.n_prune; ++p) {
                const PrunePred& pr = Q.prune[p];
                keep = keep && (pr.lo <= pr.maxs[c]) && (pr.hi >= pr.mins[c]);
            }
        }
        const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
        const uint32_t b = __ballot_sync(0xFFFFFFFFu, keep);
        if (lane == 0) s_warp[warp] = __popc(b);
        __syncthreads();
        if (threadIdx.x == 0) {
            uint32_t run = s_count;
            for (uint32_t w = 0; w < blockDim.x / 32; ++w) {
                const uint32_t x = s_warp[w];
                s_warp[w] = run;
                run += x;
            }
            s_count = run;
        }
        __syncthreads();
        if (keep) {
            const uint32_t o = s_warp[warp] + __popc(b & ((1u << lane) - 1u));
            items_q[o] = q;
            items_chunk[o] = c;
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        *n_items = s_count;
        *work_counter = 0;
    }
}

// Decompress tiles of slots [slot0, slot0 + gridDim.x / tpb) into dst, rows
// laid out contiguously from the first row of chunk row0.  One CTA per tile.
template <int NT, int MAXT>
__global__ void __launch_bounds__(NT) decompress_kernel(const __grid_constant__ gx_dcol c, uint32_t slot0, uint32_t tile_rows,
                                                        uint32_t tpb, uint64_t row0, int32_t* dst) {
    using C = Cfg<MAXT>;
    extern __shared__ __align__(16) uint8_t smem[];
    uint32_t* buf = (uint32_t*)smem;
    uint8_t* stage = (uint8_t*)(buf + C::kBufWords);
    __shared__ __align__(8) uint64_t s_mbar;
    __shared__ int s_err;
    __shared__ uint32_t s_tmp[NT / 32 + 1];
    __shared__ uint32_t s_seg[2 * (kMaxSegments + 1)];
    const uint32_t slot = slot0 + blockIdx.x / tpb;
    const uint32_t r0 = (blockIdx.x % tpb) * tile_rows;
    const gx_dblock d = c.blocks[slot];
    if (r0 >= d.n_rows) return;
    const uint32_t n = min(tile_rows, d.n_rows - r0);
    if (threadIdx.x == 0) {
        s_err = 0;
        mbar_init(&s_mbar, 1);
    }
    __syncthreads();
    uint32_t phase = 0, pad_log2 = 0;
    const int layout = decode_tile<NT, MAXT>(c, slot, d.n_rows, r0, n, buf, stage, &s_mbar, phase, s_tmp, &s_err,
                                             pad_log2, s_seg);
    if (s_err) {
        if (threadIdx.x == 0) raise_error(s_err);
        return;
    }
    const uint32_t chunk = slot / c.blocks_per_chunk, j = slot % c.blocks_per_chunk;
    const uint64_t first = (uint64_t)chunk * c.rows_per_chunk + (uint64_t)j * c.rows_per_block + r0 - row0;
    int32_t* out = dst + first;
    for (uint32_t r = threadIdx.x; r < n; r += NT)
        out[r] = (int32_t)buf[layout == kSegRows ? r + ((r >> c.seg_shift) << pad_log2) : r];
}

__global__ void raw_lz4_kernel(const uint8_t* comp, const uint64_t* coff, uint8_t* out, const uint64_t* ooff,
                               uint64_t n_blocks, int32_t* status) {
    const uint64_t b = (uint64_t)blockIdx.x * (blockDim.x / 32) + threadIdx.x / 32;
    if (b >= n_blocks) return;
    const uint64_t c0 = coff[b], c1 = coff[b + 1], o0 = ooff[b], o1 = ooff[b + 1];
    int rc = kErrCorrupt;
    if (c1 >= c0 && o1 >= o0 && c1 - c0 < (1ull << 31) && o1 - o0 < (1ull << 31))
        rc = lz4_warp_block(GlobalSrc{comp + c0}, (uint32_t)(c1 - c0), out + o0, (uint32_t)(o1 - o0),
                            threadIdx.x & 31);
    if ((threadIdx.x & 31) == 0) status[b] = rc;
}

// Min and max of data[0..n) into range[0] / range[1], which start at
// INT32_MAX / INT32_MIN (warp reductions, one atomic pair per warp).
__global__ void minmax_reduce_kernel(const int32_t* data, uint64_t n, int32_t* range) {
    int32_t lo = INT32_MAX, hi = INT32_MIN;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    const bool vec = ((uintptr_t)data & 15u) == 0;
    if (vec) {
        const uint64_t n4 = n / 4;
        for (uint64_t j = i; j < n4; j += stride) {
            const int4 v = __ldg((const int4*)data + j);
            lo = min(lo, min(min(v.x, v.y), min(v.z, v.w)));
            hi = max(hi, max(max(v.x, v.y), max(v.z, v.w)));
        }
        i += n4 * 4;
    }
    for (; i < n; i += stride) {
        const int32_t v = __ldg(data + i);
        lo = min(lo, v);
        hi = max(hi, v);
    }
    lo = __reduce_min_sync(0xFFFFFFFFu, lo);
    hi = __reduce_max_sync(0xFFFFFFFFu, hi);
    if ((threadIdx.x & 31) == 0) {
        atomicMin(&range[0], lo);
        atomicMax(&range[1], hi);
    }
}

// Keys of the occupied slots of a join table, compacted in any order
// (warp-aggregated counter); a dense table's header slot is skipped.
__global__ void ht_keys_kernel(const uint64_t* slots, uint64_t n_slots, uint32_t first, int32_t* out, uint64_t cap,
                               unsigned long long* count) {
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    const uint32_t lane = threadIdx.x & 31;
    const uint64_t n_iter = (n_slots + stride - 1) / stride;  // uniform trip count: every lane reaches the ballot
    for (uint64_t it = 0; it < n_iter; ++it) {
        const uint64_t i = it * stride + blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
        int32_t k = kEmptyKey;
        if (i < n_slots && i >= first) k = (int32_t)(uint32_t)slots[i];
        const bool has = k != kEmptyKey;
        const uint32_t m = __ballot_sync(0xFFFFFFFFu, has);
        unsigned long long base = 0;
        if (lane == 0 && m) base = atomicAdd(count, (unsigned long long)__popc(m));
        base = __shfl_sync(0xFFFFFFFFu, base, 0);
        if (has) {
            const unsigned long long o = base + __popc(m & ((1u << lane) - 1u));
            if (o < cap) out[o] = k;
        }
    }
}

// Join pruning: out[c] = 1 where chunk c's [min, max] holds one of the keys
// (the first min(*n_keys, cap) of them, staged through shared memory).
__global__ void prune_points_kernel(const int32_t* mins, const int32_t* maxs, uint32_t n_chunks, const int32_t* keys,
                                    const unsigned long long* n_keys, uint64_t cap, uint16_t* out) {
    __shared__ int32_t s_keys[2048];
    const uint64_t nk = min((uint64_t)*n_keys, cap);
    const uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    const int32_t lo = c < n_chunks ? mins[c] : 1, hi = c < n_chunks ? maxs[c] : 0;
    bool hit = false;
    for (uint64_t k0 = 0; k0 < nk; k0 += 2048) {
        const uint32_t m = (uint32_t)min((uint64_t)2048, nk - k0);
        __syncthreads();
        for (uint32_t i = threadIdx.x; i < m; i += blockDim.x) s_keys[i] = keys[k0 + i];
        __syncthreads();
        if (!hit)
            for (uint32_t i = 0; i < m; ++i) hit |= s_keys[i] >= lo && s_keys[i] <= hi;
    }
    if (c < n_chunks && hit) out[c] = 1;
}

// Slots emptied, counters zeroed (one launch).
__global__ void ht_clear_kernel(uint64_t* slots, uint64_t n, unsigned long long* counters) {
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += stride) slots[i] = kEmptySlot;
    if (blockIdx.x == 0 && threadIdx.x < 4) counters[threadIdx.x] = 0;
}

__global__ void check_minmax_kernel(const int32_t* mins, const int32_t* maxs, uint32_t n, int32_t lo, int32_t hi,
                                    uint16_t* out) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        if (lo <= maxs[i] && hi >= mins[i]) out[i] = 1;
}

__global__ void combine_and_kernel(uint16_t* out, const uint16_t* a, const uint16_t* b, uint64_t n) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        out[i] = a[i] & b[i];
}

__global__ void fill_u64_kernel(uint64_t* p, uint64_t n, uint64_t v) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        p[i] = v;
}

struct BuildPreds {
    gx_pred p[4];
    uint32_t n;
};

// Linear-probing inserts of rows i0, i0 + stride, ... (< n) that pass the
// predicates; counts inserted / duplicate / dropped rows into counters.
__device__ __forceinline__ void ht_insert_rows(uint64_t* slots, uint32_t log2cap, const int32_t* keys,
                                               const int32_t* payload, uint64_t i0, uint64_t stride, uint64_t n,
                                               const BuildPreds& preds, unsigned long long* counters) {
    const uint32_t mask = (1u << log2cap) - 1;
    unsigned long long ins = 0, dup = 0, bad = 0;
    for (uint64_t i = i0; i < n; i += stride) {
        bool pass = true;
        for (uint32_t k = 0; k < preds.n; ++k) {
            int32_t x = preds.p[k].col_dev[i];
            pass = pass && x >= preds.p[k].lo && x <= preds.p[k].hi;
        }
        if (!pass) continue;
        const int32_t key = keys[i];
        if (key == kEmptyKey) {
            ++bad;
            continue;
        }
        const int32_t pay = payload ? payload[i] : (int32_t)i;
        const unsigned long long e = ((unsigned long long)(uint32_t)pay << 32) | (uint32_t)key;
        uint32_t s = hash_key32(key, log2cap);
        bool done = false;
        for (uint32_t t = 0; t <= mask; ++t) {
            unsigned long long old = atomicCAS((unsigned long long*)slots + s, (unsigned long long)kEmptySlot, e);
            if (old == (unsigned long long)kEmptySlot) {
                ++ins;
                done = true;
                break;
            }
            if ((int32_t)(uint32_t)old == key) {
                ++dup;
                done = true;
                break;
            }
            s = (s + 1) & mask;
        }
        if (!done) ++bad;
    }
    if (ins) atomicAdd(&counters[0], ins);
    if (dup) atomicAdd(&counters[1], dup);
    if (bad) atomicAdd(&counters[2], bad);
}

__global__ void ht_build_kernel(uint64_t* slots, uint32_t log2cap, const int32_t* keys, const int32_t* payload,
                                uint64_t n, const __grid_constant__ BuildPreds preds, unsigned long long* counters) {
    griddep_launch();
    ht_insert_rows(slots, log2cap, keys, payload, blockIdx.x * (uint64_t)blockDim.x + threadIdx.x,
                   (uint64_t)gridDim.x * blockDim.x, n, preds, counters);
}

// A small linear table in one launch: one CTA clears the slots and the
// counters, then inserts (dimension tables such as the date table).
constexpr uint64_t kSmallHtSlots = 1u << 16, kSmallHtRows = 1u << 16;
__global__ void ht_build_small_kernel(uint64_t* slots, uint32_t log2cap, const int32_t* keys, const int32_t* payload,
                                      uint64_t n, const __grid_constant__ BuildPreds preds,
                                      unsigned long long* counters) {
    griddep_launch();  // a scan launched after the build may start its table-free work now
    const uint64_t cap = 1ull << log2cap;
    for (uint64_t i = threadIdx.x; i < cap; i += blockDim.x) slots[i] = kEmptySlot;
    if (threadIdx.x < 4) counters[threadIdx.x] = 0;
    __syncthreads();
    ht_insert_rows(slots, log2cap, keys, payload, threadIdx.x, blockDim.x, n, preds, counters);
}

// Smallest and largest key of the rows that pass the predicates (range[0],
// range[1]; start at INT32_MAX, INT32_MIN).  The reserved empty key is skipped.
__global__ void ht_range_kernel(const int32_t* keys, uint64_t n, const __grid_constant__ BuildPreds preds,
                                int32_t* range) {
    int32_t lo = INT32_MAX, hi = INT32_MIN;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        bool pass = true;
        for (uint32_t k = 0; k < preds.n; ++k) {
            int32_t x = preds.p[k].col_dev[i];
            pass = pass && x >= preds.p[k].lo && x <= preds.p[k].hi;
        }
        const int32_t key = keys[i];
        if (!pass || key == kEmptyKey) continue;
        lo = min(lo, key);
        hi = max(hi, key);
    }
    lo = __reduce_min_sync(0xFFFFFFFFu, lo);
    hi = __reduce_max_sync(0xFFFFFFFFu, hi);
    if ((threadIdx.x & 31) == 0 && lo <= hi) {
        atomicMin(&range[0], lo);
        atomicMax(&range[1], hi);
    }
}

// Dense build: slots[0] holds {base, span}; row i's entry goes to slot
// 1 + (key - base); the first insert of a key wins, later ones count as
// duplicates (as in the hashed layouts).
__global__ void ht_build_dense_kernel(uint64_t* slots, int32_t base, uint32_t span, const int32_t* keys,
                                      const int32_t* payload, uint64_t n, const __grid_constant__ BuildPreds preds,
                                      unsigned long long* counters) {
    griddep_launch();
    unsigned long long ins = 0, dup = 0, bad = 0;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        bool pass = true;
        for (uint32_t k = 0; k < preds.n; ++k) {
            int32_t x = preds.p[k].col_dev[i];
            pass = pass && x >= preds.p[k].lo && x <= preds.p[k].hi;
        }
        if (!pass) continue;
        const int32_t key = keys[i];
        const uint32_t u = (uint32_t)key - (uint32_t)base;
        if (key == kEmptyKey || u >= span) {
            ++bad;
            continue;
        }
        const int32_t pay = payload ? payload[i] : (int32_t)i;
        const unsigned long long e = ((unsigned long long)(uint32_t)pay << 32) | (uint32_t)key;
        const unsigned long long old = atomicCAS((unsigned long long*)slots + 1 + u, (unsigned long long)kEmptySlot, e);
        if (old == (unsigned long long)kEmptySlot)
            ++ins;
        else
            ++dup;
    }
    if (ins) atomicAdd(&counters[0], ins);
    if (dup) atomicAdd(&counters[1], dup);
    if (bad) atomicAdd(&counters[2], bad);
}

__global__ void ht_build_bucket_kernel(uint64_t* slots, uint32_t log2cap, const int32_t* keys, const int32_t* payload,
                                       uint64_t n, const __grid_constant__ BuildPreds preds,
                                       unsigned long long* counters) {
    griddep_launch();
    const uint32_t lb = log2cap - 3, bmask = (1u << lb) - 1;
    unsigned long long ins = 0, dup = 0, bad = 0;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        bool pass = true;
        for (uint32_t k = 0; k < preds.n; ++k) {
            int32_t x = preds.p[k].col_dev[i];
            pass = pass && x >= preds.p[k].lo && x <= preds.p[k].hi;
        }
        if (!pass) continue;
        const int32_t key = keys[i];
        if (key == kEmptyKey) {
            ++bad;
            continue;
        }
        const int32_t pay = payload ? payload[i] : (int32_t)i;
        const unsigned long long e = ((unsigned long long)(uint32_t)pay << 32) | (uint32_t)key;
        uint32_t bkt = hash_key32(key, lb);
        bool done = false;
        for (uint32_t t = 0; t <= bmask && !done; ++t) {
            unsigned long long* bp = (unsigned long long*)slots + (size_t)bkt * kBucketSlots;
            for (uint32_t j = 0; j < kBucketSlots; ++j) {
                unsigned long long old = atomicCAS(bp + j, (unsigned long long)kEmptySlot, e);
                if (old == (unsigned long long)kEmptySlot) {
                    ++ins;
                    done = true;
                    break;
                }
                if ((int32_t)(uint32_t)old == key) {
                    ++dup;
                    done = true;
                    break;
                }
            }
            bkt = (bkt + 1) & bmask;
        }
        if (!done) ++bad;
    }
    if (ins) atomicAdd(&counters[0], ins);
    if (dup) atomicAdd(&counters[1], dup);
    if (bad) atomicAdd(&counters[2], bad);
}

__global__ void ht_probe_kernel(const uint64_t* slots, uint32_t log2cap, uint32_t layout, const int32_t* keys,
                                uint64_t n, int32_t* out, unsigned long long* hits) {
    unsigned long long h = 0;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        int32_t p = 0;
        bool hit = ht_probe_any(slots, log2cap, layout, keys[i], &p);
        if (out) out[i] = hit ? p : INT32_MIN;
        h += hit;
    }
    if (hits) {
        for (int d = 16; d > 0; d >>= 1) h += __shfl_down_sync(0xFFFFFFFFu, h, d);
        if ((threadIdx.x & 31) == 0 && h) atomicAdd(hits, h);
    }
}

__global__ void groupby_add_kernel(int64_t* gk, int64_t* gs, uint32_t log2cap, const int64_t* keys,
                                   const int64_t* vals, uint64_t n) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const int64_t k = keys[i];
        if (k == kEmptyGroup || !group_add_global(gk, gs, log2cap, k, vals[i])) raise_error(kErrCapacity);
    }
}

__global__ void groupby_compact_kernel(const int64_t* gk, const int64_t* gs, uint64_t cap, int64_t* ok, int64_t* os,
                                       unsigned long long* count, uint64_t out_cap) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < cap; i += (uint64_t)gridDim.x * blockDim.x) {
        if (gk[i] == kEmptyGroup) continue;
        unsigned long long j = atomicAdd(count, 1ull);
        if (j < out_cap) {
            ok[j] = gk[i];
            os[j] = gs[i];
        }
    }
}

// ------------------------------------------------------------ host helpers

int sm_count() {
    static int cached[kMaxDevices] = {0};
    int dev = 0;
    cudaGetDevice(&dev);
    if (!device_index_ok(dev)) {  // callers reject such devices; answer without caching
        int n = 0;
        cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
        return n > 0 ? n : 1;
    }
    if (!cached[dev]) {
        int n = 0;
        cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
        cached[dev] = n > 0 ? n : 1;
    }
    return cached[dev];
}

uint32_t log2_ceil(uint64_t x) {
    uint32_t l = 0;
    while ((1ull << l) < x) ++l;
    return l;
}

template <int MAXT>
size_t scan_smem_bytes(bool need_aux, bool grouped) {
    using C = Cfg<MAXT>;
    size_t b = 4ull * C::kBufWords;
    if (need_aux) b += 4ull * MAXT;
    b += 4ull * C::kMaskWords;
    b += C::kStage;  // also holds the cascaded run tables
    if (grouped) b += (4ull + 8ull) * (1u << kSmemGroupLog2);
    return b;
}

template <int MAXT>
size_t dec_smem_bytes() {
    return 4ull * Cfg<MAXT>::kBufWords + Cfg<MAXT>::kStage;
}

gx_status wait_stream(cudaStream_t s, double timeout_s) {
    auto t0 = std::chrono::steady_clock::now();
    while (true) {
        cudaError_t e = cudaStreamQuery(s);
        if (e == cudaSuccess) return GX_OK;
        if (e != cudaErrorNotReady) return set_error(GX_ERR_CUDA, "stream failed: %s", cudaGetErrorString(e));
        double el = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        if (el > timeout_s) return set_error(GX_ERR_TIMEOUT, "stream did not finish within %.0f s", timeout_s);
        std::this_thread::sleep_for(std::chrono::microseconds(el < 0.01 ? 5 : 200));
    }
}

// Tile size usable for a set of columns: kTileRows when every LZ4 column is
// segmented with segments no longer than a tile, else whole blocks.
uint32_t pick_tile_rows(const gx_column* const* cols, uint32_t n) {
    const uint32_t rb = cols[0]->rows_per_block;
    if (rb <= kTileRows) return rb;
    for (uint32_t i = 0; i < n; ++i) {
        const gx_column* c = cols[i];
        if (c->codec == GX_CODEC_LZ4 && (c->S <= 1 || (1u << c->seg_shift) > kTileRows)) return rb;
    }
    return kTileRows;
}

// Per-device setup of a kernel's dynamic shared-memory limit.
template <class K>
gx_status allow_smem(K kernel, size_t bytes) {
    cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    if (e != cudaSuccess) return set_error(GX_ERR_CUDA, "cudaFuncSetAttribute: %s", cudaGetErrorString(e));
    return GX_OK;
}

#include "shared_scan.cuh"
#include "pipe_scan.cuh"
#include "warp_scan.cuh"

}  // namespace

// ---------------------------------------------------------------- objects

struct gx_hashtable {
    uint64_t* slots = nullptr;
    uint32_t log2cap = 0;
    uint32_t layout = GX_HT_LINEAR;
    uint64_t max_entries = 0;
    unsigned long long* counters = nullptr;  // inserted, duplicates, dropped
    int32_t* range = nullptr;                // dense layout: key range of the last build (device)
};

struct gx_groupby {
    int64_t* keys = nullptr;
    int64_t* sums = nullptr;
    uint32_t log2cap = 0;
    uint64_t max_groups = 0;
};

struct gx_batch {
    uint32_t n = 0;
    QueryDesc* d_qs = nullptr;
    uint32_t* d_buf = nullptr;  // cand_q | cand_chunk | items_q | items_chunk | n_items | counter
    uint32_t n_cand = 0;
    uint32_t cap_q = 0, cap_cand = 0;   // device buffer capacities
    QueryDesc* h_qs = nullptr;          // pinned host staging (async assignment)
    uint32_t* h_cand = nullptr;
    unsigned long long* d_rows = nullptr;
    ScanParams P{};
    uint32_t grid = 1, threads = 128;
    size_t smem = 0;
    uint32_t reset_x = 1;
    int device = -1;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    // execution form
    uint32_t mode_pref = GX_BATCH_AUTO;
    uint32_t mode = GX_BATCH_QUEUE;
    // shared form
    ShQuery* d_sq = nullptr;
    ShQuery* h_sq = nullptr;      // pinned staging
    uint32_t cap_sq = 0;
    gx_dcol* d_cols = nullptr;
    gx_dcol* h_cols = nullptr;    // pinned staging (kShMaxCols entries)
    uint32_t* d_slot_mask = nullptr;
    size_t cap_mask = 0;          // words
    uint32_t* d_sh_items = nullptr;  // n_items | work_counter | items[n_slots]
    uint32_t cap_slots = 0;
    ShParams SP{};
    uint32_t n_slots = 0;
    const gx_dblock* dir0 = nullptr;
    uint32_t sh_grid = 1, sh_items_grid = 1;
    size_t sh_smem = 0;
    uint8_t* d_qc = nullptr;       // compact descriptors (device) and pinned staging
    uint8_t* h_qc = nullptr;
    size_t cap_qc = 0;
    uint32_t sh_threads = kShNT;   // launch shape of the shared form in use
    uint32_t sh_threads_req = 0;   // requested threads per CTA (0 = automatic)
    uint32_t sh_ctas_per_sm = 0;   // 0 = as many as fit
};

static int shared_occupancy(uint32_t threads, size_t smem) {
    int per_sm = 0;
    switch (threads) {
        case 128: cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, shared_scan_kernel<128, 4>, 128, smem); break;
        case 512: cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, shared_scan_kernel<512, 1>, 512, smem); break;
        case 1024: cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, shared_scan_kernel<1024, 1>, 1024, smem); break;
        default: cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, shared_scan_kernel<256, 2>, 256, smem); break;
    }
    return per_sm;
}

// Persistent grid of the shared form for the batch's thread count.  An
// automatic shape (sh_threads_req 0) takes, of 256, 512 and 128 threads, the
// CTA size with the most resident warps per SM for the batch's shared memory
// (the earlier one on ties).  1024-thread CTAs are left to explicit
// requests: with 2 rows per thread per tile, a query's per-tile work is
// spread too thin and its probes have too few reads in flight per thread.
static void shared_geometry(gx_batch* b) {
    if (b->sh_threads_req == 0) {
        uint32_t best = 256;
        int best_warps = -1;
        for (uint32_t nt : {256u, 512u, 128u}) {
            const int w = shared_occupancy(nt, b->sh_smem) * (int)(nt / 32);
            if (w > best_warps) {
                best_warps = w;
                best = nt;
            }
        }
        b->sh_threads = best;
    } else {
        b->sh_threads = b->sh_threads_req;
    }
    int per_sm = 1;
    switch (b->sh_threads) {
        case 128: cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, shared_scan_kernel<128, 4>, 128, b->sh_smem); break;
        case 512: cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, shared_scan_kernel<512, 1>, 512, b->sh_smem); break;
        case 1024: cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, shared_scan_kernel<1024, 1>, 1024, b->sh_smem); break;
        default: cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, shared_scan_kernel<256, 2>, 256, b->sh_smem); break;
    }
    per_sm = std::max(1, per_sm);
    if (b->sh_ctas_per_sm) per_sm = std::min<int>(per_sm, (int)b->sh_ctas_per_sm);
    const uint64_t tiles = (uint64_t)b->n_slots * b->SP.tiles_per_block;
    b->sh_grid = (uint32_t)std::max<uint64_t>(1, std::min<uint64_t>((uint64_t)sm_count() * per_sm, tiles));
}

static void launch_shared_kernel(const gx_batch* b, cudaStream_t s) {
    switch (b->sh_threads) {
        case 128: shared_scan_kernel<128, 4><<<b->sh_grid, 128, b->sh_smem, s>>>(b->SP); break;
        case 512: shared_scan_kernel<512, 1><<<b->sh_grid, 512, b->sh_smem, s>>>(b->SP); break;
        case 1024: shared_scan_kernel<1024, 1><<<b->sh_grid, 1024, b->sh_smem, s>>>(b->SP); break;
        default: shared_scan_kernel<256, 2><<<b->sh_grid, 256, b->sh_smem, s>>>(b->SP); break;
    }
}

extern "C" {

gx_status gx_column_to_device(gx_column* col, int residency, void* stream) {
    if (!col || (residency != 1 && residency != 2)) return set_error(GX_ERR_INVALID, "gx_column_to_device: bad args");
    if (const int st = host_payload(col)) return st;  // a device-encoded column: its host copy first
    gx_column_release_device(col);
    cudaStream_t s = (cudaStream_t)stream;
    const size_t pb = col->payload.size();
    if (residency == 1) {
        GX_CK(cudaMalloc(&col->d_payload, pb));
        GX_CK(cudaMemcpyAsync(col->d_payload, col->payload.data(), pb, cudaMemcpyHostToDevice, s));
    } else {
        GX_CK(cudaHostAlloc(&col->h_pinned, pb, cudaHostAllocMapped | cudaHostAllocPortable));
        std::memcpy(col->h_pinned, col->payload.data(), pb);
        GX_CK(cudaHostGetDevicePointer(&col->d_payload, col->h_pinned, 0));
    }
    GX_CK(cudaMalloc(&col->d_blocks, sizeof(gx_dblock) * col->blocks.size()));
    GX_CK(cudaMemcpyAsync(col->d_blocks, col->blocks.data(), sizeof(gx_dblock) * col->blocks.size(),
                          cudaMemcpyHostToDevice, s));
    if (!col->seg.empty()) {
        GX_CK(cudaMalloc(&col->d_seg, 4 * col->seg.size()));
        GX_CK(cudaMemcpyAsync(col->d_seg, col->seg.data(), 4 * col->seg.size(), cudaMemcpyHostToDevice, s));
    }
    GX_CK(cudaMalloc(&col->d_mins, 4 * col->n_chunks));
    GX_CK(cudaMalloc(&col->d_maxs, 4 * col->n_chunks));
    GX_CK(cudaMemcpyAsync(col->d_mins, col->mins.data(), 4 * col->n_chunks, cudaMemcpyHostToDevice, s));
    GX_CK(cudaMemcpyAsync(col->d_maxs, col->maxs.data(), 4 * col->n_chunks, cudaMemcpyHostToDevice, s));
    if (col->bmins.size() == col->n_slots && col->n_slots) {
        GX_CK(cudaMalloc(&col->d_bmins, 4ull * col->n_slots));
        GX_CK(cudaMalloc(&col->d_bmaxs, 4ull * col->n_slots));
        GX_CK(cudaMemcpyAsync(col->d_bmins, col->bmins.data(), 4ull * col->n_slots, cudaMemcpyHostToDevice, s));
        GX_CK(cudaMemcpyAsync(col->d_bmaxs, col->bmaxs.data(), 4ull * col->n_slots, cudaMemcpyHostToDevice, s));
    }
    GX_CK(cudaStreamSynchronize(s));
    cudaGetDevice(&col->device);
    col->residency = residency;
    return GX_OK;
}

gx_status gx_column_release_device(gx_column* col) {
    if (!col) return set_error(GX_ERR_INVALID, "null column");
    if (const int st = host_payload(col)) return st;  // keep the payload of a device-encoded column
    if (col->residency == 1 && col->d_payload) cudaFree(col->d_payload);
    if (col->h_pinned) cudaFreeHost(col->h_pinned);
    if (col->d_blocks) cudaFree(col->d_blocks);
    if (col->d_seg) cudaFree(col->d_seg);
    if (col->d_mins) cudaFree(col->d_mins);
    if (col->d_maxs) cudaFree(col->d_maxs);
    if (col->d_bmins) cudaFree(col->d_bmins);
    if (col->d_bmaxs) cudaFree(col->d_bmaxs);
    if (col->d_hist) cudaFree(col->d_hist);
    if (col->d_bloom) cudaFree(col->d_bloom);
    col->d_hist = nullptr;
    col->d_bloom = nullptr;
    col->hist_buckets = 0;
    col->bloom_bytes = 0;
    col->bloom_k = 0;
    col->d_bmins = col->d_bmaxs = nullptr;
    col->d_payload = nullptr;
    col->h_pinned = nullptr;
    col->d_blocks = nullptr;
    col->d_seg = nullptr;
    col->d_mins = col->d_maxs = nullptr;
    col->residency = 0;
    return GX_OK;
}

gx_status gx_decompress_chunks(const gx_column* col, uint64_t first_chunk, uint64_t n_chunks, void* dst_dev,
                               void* stream) {
    if (!col || !dst_dev) return set_error(GX_ERR_INVALID, "gx_decompress_chunks: null argument");
    if (!col->residency) return set_error(GX_ERR_INVALID, "column is not on the device");
    if (first_chunk + n_chunks > col->n_chunks) return set_error(GX_ERR_INVALID, "chunk range out of bounds");
    if (n_chunks == 0) return GX_OK;
    static bool attr_set[kMaxDevices] = {false};
    int dev = 0;
    cudaGetDevice(&dev);
    if (!device_index_ok(dev)) return set_error(GX_ERR_INVALID, "device %d out of range", dev);
    if (!attr_set[dev]) {
        gx_status st = allow_smem(decompress_kernel<128, kTileRows>, dec_smem_bytes<kTileRows>());
        if (!st) st = allow_smem(decompress_kernel<256, kMaxRowsPerBlock>, dec_smem_bytes<kMaxRowsPerBlock>());
        if (st) return st;
        attr_set[dev] = true;
    }
    const uint32_t slot0 = (uint32_t)(first_chunk * col->blocks_per_chunk);
    const uint32_t nslots = (uint32_t)(n_chunks * col->blocks_per_chunk);
    const uint64_t row0 = first_chunk * (uint64_t)col->rows_per_chunk;
    const uint32_t tile = pick_tile_rows(&col, 1);
    const uint32_t tpb = (col->rows_per_block + tile - 1) / tile;
    cudaStream_t s = (cudaStream_t)stream;
    if (tile <= kTileRows)
        decompress_kernel<128, kTileRows><<<nslots * tpb, 128, dec_smem_bytes<kTileRows>(), s>>>(
            col->view(), slot0, tile, tpb, row0, (int32_t*)dst_dev);
    else
        decompress_kernel<256, kMaxRowsPerBlock><<<nslots * tpb, 256, dec_smem_bytes<kMaxRowsPerBlock>(), s>>>(
            col->view(), slot0, tile, tpb, row0, (int32_t*)dst_dev);
    GX_CK(cudaGetLastError());
    return GX_OK;
}

gx_status gx_decompress_chunk(const gx_column* col, uint64_t chunk_idx, void* dst_dev, void* stream) {
    return gx_decompress_chunks(col, chunk_idx, 1, dst_dev, stream);
}

gx_status gx_lz4_decompress_raw(const uint8_t* comp_dev, const uint64_t* comp_offsets_dev, uint8_t* out_dev,
                                const uint64_t* out_offsets_dev, uint64_t n_blocks, int32_t* status_dev,
                                void* stream) {
    if (!comp_dev || !comp_offsets_dev || !out_dev || !out_offsets_dev || !status_dev)
        return set_error(GX_ERR_INVALID, "gx_lz4_decompress_raw: null argument");
    if (n_blocks == 0) return GX_OK;
    const uint32_t wpb = 4;
    raw_lz4_kernel<<<(unsigned)((n_blocks + wpb - 1) / wpb), 32 * wpb, 0, (cudaStream_t)stream>>>(
        comp_dev, comp_offsets_dev, out_dev, out_offsets_dev, n_blocks, status_dev);
    GX_CK(cudaGetLastError());
    return GX_OK;
}

gx_status gx_check_minmax(const gx_column* col, int32_t lo, int32_t hi, uint16_t* out_dev, void* stream) {
    if (!col || !out_dev || !col->residency) return set_error(GX_ERR_INVALID, "gx_check_minmax: bad args");
    uint32_t n = col->n_chunks;
    check_minmax_kernel<<<std::max(1u, std::min(64u, (n + 511) / 512)), 512, 0, (cudaStream_t)stream>>>(
        col->d_mins, col->d_maxs, n, lo, hi, out_dev);
    GX_CK(cudaGetLastError());
    return GX_OK;
}

gx_status gx_combine_and(uint16_t* out_dev, const uint16_t* a_dev, const uint16_t* b_dev, uint64_t n, void* stream) {
    if (!out_dev || !a_dev || !b_dev) return set_error(GX_ERR_INVALID, "gx_combine_and: null argument");
    if (n == 0) return GX_OK;
    combine_and_kernel<<<(unsigned)std::min<uint64_t>(64, (n + 511) / 512), 512, 0, (cudaStream_t)stream>>>(
        out_dev, a_dev, b_dev, n);
    GX_CK(cudaGetLastError());
    return GX_OK;
}

static gx_status fill_prune(ItemsParams* ip, const gx_column* const* cols, const int32_t* lo, const int32_t* hi,
                            uint32_t n_preds, uint32_t n_chunks) {
    if (n_preds > GX_MAX_STEPS) return set_error(GX_ERR_INVALID, "too many prune predicates");
    for (uint32_t p = 0; p < n_preds; ++p) {
        if (!cols[p] || !cols[p]->residency) return set_error(GX_ERR_INVALID, "prune column %u not on device", p);
        if (cols[p]->n_chunks != n_chunks) return set_error(GX_ERR_INVALID, "prune columns disagree on chunk count");
        ip->preds[p] = PrunePred{cols[p]->d_mins, cols[p]->d_maxs, lo[p], hi[p], nullptr, nullptr};
    }
    ip->n_preds = n_preds;
    ip->n_chunks = n_chunks;
    return GX_OK;
}

gx_status gx_prune_minmax(const gx_column* const* cols, const int32_t* lo, const int32_t* hi, uint32_t n_preds,
                          uint16_t* keep_dev, void* stream) {
    if (!cols || !lo || !hi || !keep_dev || n_preds == 0) return set_error(GX_ERR_INVALID, "gx_prune_minmax: bad args");
    cudaStream_t s = (cudaStream_t)stream;
    const uint32_t n_chunks = cols[0]->n_chunks;
    ItemsParams ip{};
    gx_status st = fill_prune(&ip, cols, lo, hi, n_preds, n_chunks);
    if (st) return st;
    uint32_t* scratch = nullptr;
    GX_CK(scratch_alloc((void**)&scratch, 4ull * (n_chunks + 2), s));
    ip.keep_out = keep_dev;
    ip.items = scratch + 2;
    ip.n_items = scratch;
    ip.work_counter = scratch + 1;
    items_kernel<<<1, 1024, 0, s>>>(ip);
    cudaError_t e = cudaGetLastError();
    cudaFreeAsync(scratch, s);
    if (e != cudaSuccess) return set_error(GX_ERR_CUDA, "items_kernel: %s", cudaGetErrorString(e));
    return GX_OK;
}

// ------------------------------------------------------------ hash tables

gx_status gx_hashtable_create(uint64_t max_entries, gx_hashtable** out) {
    if (!out || max_entries == 0 || max_entries > (1ull << 30)) return set_error(GX_ERR_INVALID, "gx_hashtable_create: bad args");
    gx_hashtable* h = new gx_hashtable();
    h->max_entries = max_entries;
    h->log2cap = std::max<uint32_t>(4, log2_ceil(2 * max_entries));
    cudaError_t e = cudaMalloc(&h->slots, 8ull << h->log2cap);
    if (e == cudaSuccess) e = cudaMalloc(&h->counters, 4 * sizeof(unsigned long long));
    if (e != cudaSuccess) {
        cudaFree(h->slots);
        delete h;
        return set_error(GX_ERR_NOMEM, "gx_hashtable_create: %s", cudaGetErrorString(e));
    }
    *out = h;
    return GX_OK;
}

gx_status gx_hashtable_create2(uint64_t max_entries, uint32_t layout, gx_hashtable** out) {
    if (layout > GX_HT_DENSE) return set_error(GX_ERR_INVALID, "unknown hash table layout %u", layout);
    gx_status st = gx_hashtable_create(max_entries, out);
    if (st) return st;
    (*out)->layout = layout;
    if (layout == GX_HT_DENSE) {
        cudaError_t e = cudaMalloc(&(*out)->range, 2 * sizeof(int32_t));
        if (e != cudaSuccess) {
            gx_hashtable_free(*out);
            *out = nullptr;
            return set_error(GX_ERR_NOMEM, "gx_hashtable_create2: %s", cudaGetErrorString(e));
        }
    }
    return GX_OK;
}

gx_status gx_hashtable_free(gx_hashtable* ht) {
    if (!ht) return GX_OK;
    cudaFree(ht->slots);
    cudaFree(ht->counters);
    cudaFree(ht->range);
    delete ht;
    return GX_OK;
}

}  // extern "C"

// Dense build: the key range of the rows that pass (one device reduction,
// read back), the table sized to it (reallocated when it grows), slot 0 the
// {base, span} header, then one slot per key of the range.
static gx_status hashtable_build_dense(gx_hashtable* ht, const int32_t* keys_dev, const int32_t* payload_dev,
                                       uint64_t n, const BuildPreds& bp, unsigned grid, cudaStream_t s) {
    int32_t range[2] = {INT32_MAX, INT32_MIN};
    if (n) {
        fill_u64_kernel<<<1, 32, 0, s>>>((uint64_t*)ht->range, 1,
                                         ((uint64_t)(uint32_t)INT32_MIN << 32) | (uint32_t)INT32_MAX);
        ht_range_kernel<<<grid, 256, 0, s>>>(keys_dev, n, bp, ht->range);
        GX_CK(cudaGetLastError());
        GX_CK(cudaMemcpyAsync(range, ht->range, sizeof(range), cudaMemcpyDeviceToHost, s));
        gx_status st = wait_stream(s, 120.0);
        if (st) return st;
    }
    const uint64_t span = range[0] <= range[1] ? (uint64_t)((int64_t)range[1] - range[0] + 1) : 0;
    const uint64_t limit = std::min<uint64_t>(1ull << 30, std::max<uint64_t>(64 * ht->max_entries, 1ull << 20));
    if (span > limit)
        return set_error(GX_ERR_INVALID, "dense hash table: keys span %llu values, above the limit %llu",
                         (unsigned long long)span, (unsigned long long)limit);
    const uint32_t need = std::max<uint32_t>(4, log2_ceil(span + 1));
    if (need > ht->log2cap) {
        GX_CK(cudaStreamSynchronize(s));
        cudaFree(ht->slots);
        ht->slots = nullptr;
        ht->log2cap = 0;
        GX_CK(cudaMalloc(&ht->slots, 8ull << need));
        ht->log2cap = need;
    }
    const uint64_t cap = 1ull << ht->log2cap;
    fill_u64_kernel<<<(unsigned)std::min<uint64_t>(1024, (cap + 255) / 256), 256, 0, s>>>(ht->slots, cap, kEmptySlot);
    fill_u64_kernel<<<1, 32, 0, s>>>(ht->slots, 1, (span << 32) | (uint32_t)(span ? range[0] : 0));
    GX_CK(cudaMemsetAsync(ht->counters, 0, 4 * sizeof(unsigned long long), s));
    if (span)
        ht_build_dense_kernel<<<grid, 256, 0, s>>>(ht->slots, range[0], (uint32_t)span, keys_dev, payload_dev, n, bp,
                                                   ht->counters);
    GX_CK(cudaGetLastError());
    return GX_OK;
}

extern "C" {

gx_status gx_hashtable_build(gx_hashtable* ht, const int32_t* keys_dev, const int32_t* payload_dev, uint64_t n,
                             const gx_pred* preds, uint32_t n_preds, void* stream) {
    if (!ht || (!keys_dev && n) || n_preds > 4 || (n_preds && !preds)) return set_error(GX_ERR_INVALID, "gx_hashtable_build: bad args");
    cudaStream_t s = (cudaStream_t)stream;
    BuildPreds bp{};
    for (uint32_t i = 0; i < n_preds; ++i) bp.p[i] = preds[i];
    bp.n = n_preds;
    const unsigned grid = (unsigned)std::min<uint64_t>(4 * sm_count(), (n + 255) / 256);
    if (ht->layout == GX_HT_DENSE) return hashtable_build_dense(ht, keys_dev, payload_dev, n, bp, grid, s);
    const uint64_t cap = 1ull << ht->log2cap;
    if (ht->layout == GX_HT_LINEAR && cap <= kSmallHtSlots && n <= kSmallHtRows) {
        ht_build_small_kernel<<<1, 1024, 0, s>>>(ht->slots, ht->log2cap, keys_dev, payload_dev, n, bp, ht->counters);
        GX_CK(cudaGetLastError());
        return GX_OK;
    }
    fill_u64_kernel<<<(unsigned)std::min<uint64_t>(1024, (cap + 255) / 256), 256, 0, s>>>(ht->slots, cap, kEmptySlot);
    GX_CK(cudaMemsetAsync(ht->counters, 0, 4 * sizeof(unsigned long long), s));
    if (n == 0) return GX_OK;
    if (ht->layout == GX_HT_BUCKET)
        ht_build_bucket_kernel<<<grid, 256, 0, s>>>(ht->slots, ht->log2cap, keys_dev, payload_dev, n, bp, ht->counters);
    else
        ht_build_kernel<<<grid, 256, 0, s>>>(ht->slots, ht->log2cap, keys_dev, payload_dev, n, bp, ht->counters);
    GX_CK(cudaGetLastError());
    return GX_OK;
}

gx_status gx_hashtable_count(const gx_hashtable* ht, uint64_t* n_entries, void* stream) {
    if (!ht || !n_entries) return set_error(GX_ERR_INVALID, "gx_hashtable_count: bad args");
    unsigned long long c[4];
    GX_CK(cudaMemcpyAsync(c, ht->counters, sizeof(c), cudaMemcpyDeviceToHost, (cudaStream_t)stream));
    gx_status st = wait_stream((cudaStream_t)stream, 120.0);
    if (st) return st;
    *n_entries = c[0];
    if (c[2]) return set_error(GX_ERR_CAPACITY, "hash table: %llu rows not inserted (full or reserved key)", c[2]);
    if (c[0] > ht->max_entries) return set_error(GX_ERR_CAPACITY, "hash table holds %llu > max_entries %llu", c[0],
                                                 (unsigned long long)ht->max_entries);
    return GX_OK;
}

gx_status gx_hashtable_view(const gx_hashtable* ht, const uint64_t** slots_dev, uint32_t* log2cap) {
    if (!ht || !slots_dev || !log2cap) return set_error(GX_ERR_INVALID, "gx_hashtable_view: null argument");
    *slots_dev = ht->slots;
    *log2cap = ht->log2cap;
    return GX_OK;
}

gx_status gx_hashtable_view2(gx_hashtable* ht, uint64_t** slots_dev, uint32_t* log2cap, uint64_t** counters_dev) {
    if (!ht || !slots_dev || !log2cap || !counters_dev)
        return set_error(GX_ERR_INVALID, "gx_hashtable_view2: null argument");
    if (ht->layout != GX_HT_LINEAR) return set_error(GX_ERR_INVALID, "gx_hashtable_view2: linear tables only");
    *slots_dev = ht->slots;
    *log2cap = ht->log2cap;
    *counters_dev = (uint64_t*)ht->counters;
    return GX_OK;
}

gx_status gx_hashtable_clear(gx_hashtable* ht, void* stream) {
    if (!ht) return set_error(GX_ERR_INVALID, "gx_hashtable_clear: null table");
    const uint64_t cap = 1ull << ht->log2cap;
    const unsigned grid = (unsigned)std::max<uint64_t>(1, std::min<uint64_t>(4ull * sm_count(), (cap + 255) / 256));
    ht_clear_kernel<<<grid, 256, 0, (cudaStream_t)stream>>>(ht->slots, cap, ht->counters);
    GX_CK(cudaGetLastError());
    return GX_OK;
}

gx_status gx_hashtable_keys(const gx_hashtable* ht, int32_t* keys_dev, uint64_t cap, uint64_t* n_keys_dev,
                            void* stream) {
    if (!ht || !n_keys_dev || (cap && !keys_dev)) return set_error(GX_ERR_INVALID, "gx_hashtable_keys: null argument");
    cudaStream_t s = (cudaStream_t)stream;
    GX_CK(cudaMemsetAsync(n_keys_dev, 0, sizeof(uint64_t), s));
    const uint64_t n = 1ull << ht->log2cap;
    const unsigned grid = (unsigned)std::max<uint64_t>(1, std::min<uint64_t>(4ull * sm_count(), (n + 255) / 256));
    ht_keys_kernel<<<grid, 256, 0, s>>>(ht->slots, n, ht->layout == GX_HT_DENSE ? 1u : 0u, keys_dev, cap,
                                        (unsigned long long*)n_keys_dev);
    GX_CK(cudaGetLastError());
    return GX_OK;
}

gx_status gx_check_minmax_points(const gx_column* col, const int32_t* keys_dev, const uint64_t* n_keys_dev,
                                 uint64_t cap, uint16_t* out_dev, void* stream) {
    if (!col || !col->residency || !n_keys_dev || !out_dev || (cap && !keys_dev))
        return set_error(GX_ERR_INVALID, "gx_check_minmax_points: bad args");
    const uint32_t n = col->n_chunks;
    prune_points_kernel<<<(n + 255) / 256, 256, 0, (cudaStream_t)stream>>>(
        col->d_mins, col->d_maxs, n, keys_dev, (const unsigned long long*)n_keys_dev, cap, out_dev);
    GX_CK(cudaGetLastError());
    return GX_OK;
}

gx_status gx_minmax_reduce(const int32_t* data_dev, uint64_t n, int32_t* range_dev, void* stream) {
    if (!range_dev || (n && !data_dev)) return set_error(GX_ERR_INVALID, "gx_minmax_reduce: null argument");
    cudaStream_t s = (cudaStream_t)stream;
    const int32_t init[2] = {INT32_MAX, INT32_MIN};
    GX_CK(cudaMemcpyAsync(range_dev, init, sizeof(init), cudaMemcpyHostToDevice, s));
    if (n == 0) return GX_OK;
    const unsigned grid = (unsigned)std::max<uint64_t>(1, std::min<uint64_t>(2ull * sm_count(), (n + 4095) / 4096));
    minmax_reduce_kernel<<<grid, 512, 0, s>>>(data_dev, n, range_dev);
    GX_CK(cudaGetLastError());
    return GX_OK;
}

gx_status gx_groupby_view(gx_groupby* gb, int64_t** keys_dev, int64_t** sums_dev, uint32_t* log2cap) {
    if (!gb || !keys_dev || !sums_dev || !log2cap) return set_error(GX_ERR_INVALID, "gx_groupby_view: null argument");
    *keys_dev = gb->keys;
    *sums_dev = gb->sums;
    *log2cap = gb->log2cap;
    return GX_OK;
}

gx_status gx_hashtable_probe(const gx_hashtable* ht, const int32_t* keys_dev, uint64_t n, int32_t* payload_out_dev,
                             uint64_t* hits_dev, void* stream) {
    if (!ht || (!keys_dev && n)) return set_error(GX_ERR_INVALID, "gx_hashtable_probe: bad args");
    if (n == 0) return GX_OK;
    ht_probe_kernel<<<(unsigned)std::min<uint64_t>(8 * sm_count(), (n + 255) / 256), 256, 0, (cudaStream_t)stream>>>(
        ht->slots, ht->log2cap, ht->layout, keys_dev, n, payload_out_dev, (unsigned long long*)hits_dev);
    GX_CK(cudaGetLastError());
    return GX_OK;
}

// ---------------------------------------------------------------- groupby

gx_status gx_groupby_create(uint64_t max_groups, gx_groupby** out) {
    if (!out || max_groups == 0 || max_groups > (1ull << 30)) return set_error(GX_ERR_INVALID, "gx_groupby_create: bad args");
    gx_groupby* g = new gx_groupby();
    g->max_groups = max_groups;
    g->log2cap = std::max<uint32_t>(4, log2_ceil(2 * max_groups));
    cudaError_t e = cudaMalloc(&g->keys, 8ull << g->log2cap);
    if (e == cudaSuccess) e = cudaMalloc(&g->sums, 8ull << g->log2cap);
    if (e != cudaSuccess) {
        cudaFree(g->keys);
        delete g;
        return set_error(GX_ERR_NOMEM, "gx_groupby_create: %s", cudaGetErrorString(e));
    }
    *out = g;
    gx_status st = gx_groupby_reset(g, nullptr);
    if (st) return st;
    GX_CK(cudaDeviceSynchronize());
    return GX_OK;
}

gx_status gx_groupby_free(gx_groupby* gb) {
    if (!gb) return GX_OK;
    cudaFree(gb->keys);
    cudaFree(gb->sums);
    delete gb;
    return GX_OK;
}

gx_status gx_groupby_reset(gx_groupby* gb, void* stream) {
    if (!gb) return set_error(GX_ERR_INVALID, "null groupby");
    const uint64_t cap = 1ull << gb->log2cap;
    fill_u64_kernel<<<(unsigned)std::min<uint64_t>(1024, (cap + 255) / 256), 256, 0, (cudaStream_t)stream>>>(
        (uint64_t*)gb->keys, cap, (uint64_t)kEmptyGroup);
    GX_CK(cudaMemsetAsync(gb->sums, 0, 8 * cap, (cudaStream_t)stream));
    GX_CK(cudaGetLastError());
    return GX_OK;
}

gx_status gx_groupby_add(gx_groupby* gb, const int64_t* keys_dev, const int64_t* vals_dev, uint64_t n, void* stream) {
    if (!gb || (n && (!keys_dev || !vals_dev))) return set_error(GX_ERR_INVALID, "gx_groupby_add: bad args");
    if (n == 0) return GX_OK;
    groupby_add_kernel<<<(unsigned)std::min<uint64_t>(8 * sm_count(), (n + 255) / 256), 256, 0, (cudaStream_t)stream>>>(
        gb->keys, gb->sums, gb->log2cap, keys_dev, vals_dev, n);
    GX_CK(cudaGetLastError());
    return GX_OK;
}

gx_status gx_groupby_read(gx_groupby* gb, int64_t* keys_host, int64_t* sums_host, uint64_t cap, uint64_t* n_groups,
                          void* stream) {
    if (!gb || !n_groups || (cap && (!keys_host || !sums_host))) return set_error(GX_ERR_INVALID, "gx_groupby_read: bad args");
    cudaStream_t s = (cudaStream_t)stream;
    const uint64_t tcap = 1ull << gb->log2cap;
    const uint64_t ocap = std::max<uint64_t>(cap, 1);
    char* scratch = nullptr;
    GX_CK(scratch_alloc((void**)&scratch, 16 * ocap + 16, s));
    int64_t* ok = (int64_t*)scratch;
    int64_t* os = ok + ocap;
    unsigned long long* cnt = (unsigned long long*)(os + ocap);
    GX_CK(cudaMemsetAsync(cnt, 0, 8, s));
    groupby_compact_kernel<<<(unsigned)std::min<uint64_t>(1024, (tcap + 255) / 256), 256, 0, s>>>(
        gb->keys, gb->sums, tcap, ok, os, cnt, cap);
    unsigned long long c = 0;
    GX_CK(cudaMemcpyAsync(&c, cnt, 8, cudaMemcpyDeviceToHost, s));
    gx_status st = wait_stream(s, 120.0);
    if (st) {
        cudaFreeAsync(scratch, s);
        return st;
    }
    *n_groups = c;
    if (c > cap) {
        cudaFreeAsync(scratch, s);
        return set_error(GX_ERR_CAPACITY, "gx_groupby_read: %llu groups > cap %llu", c, (unsigned long long)cap);
    }
    if (c) {
        GX_CK(cudaMemcpyAsync(keys_host, ok, 8 * c, cudaMemcpyDeviceToHost, s));
        GX_CK(cudaMemcpyAsync(sums_host, os, 8 * c, cudaMemcpyDeviceToHost, s));
    }
    cudaFreeAsync(scratch, s);
    return wait_stream(s, 120.0);
}

// ------------------------------------------------------------------- scan

}  // extern "C"

// Validates a plan and fills the query descriptor (steps, aggregate target,
// prune predicates).  *tile_rows receives the tile size its columns allow.
static gx_status build_query(const gx_scan_plan* plan, QueryDesc* Q, uint32_t* tile_rows, const gx_column** ref_col) {
    if (!plan || plan->n_steps == 0 || plan->n_steps > GX_MAX_STEPS)
        return set_error(GX_ERR_INVALID, "scan plan needs 1..%d steps", GX_MAX_STEPS);
    std::memset(Q, 0, sizeof(*Q));
    const gx_column* c0 = plan->steps[0].col;
    if (!c0 || !c0->residency) return set_error(GX_ERR_INVALID, "step 0 column is not on the device");
    bool any_value = false, any_digit = false, any_carry = false;
    uint64_t card_prod = 1;
    const gx_column* cols[GX_MAX_STEPS];
    const uint32_t known = GX_STEP_FILTER | GX_STEP_PROBE | GX_STEP_CARRY | GX_STEP_VALUE | GX_STEP_GROUP;
    for (uint32_t i = 0; i < plan->n_steps; ++i) {
        const gx_scan_step& s = plan->steps[i];
        const gx_column* c = s.col;
        if (!c || !c->residency) return set_error(GX_ERR_INVALID, "step %u column is not on the device", i);
        if (c->n_rows != c0->n_rows || c->rows_per_chunk != c0->rows_per_chunk ||
            c->rows_per_block != c0->rows_per_block)
            return set_error(GX_ERR_INVALID, "step %u column layout differs from step 0", i);
        if (s.flags == 0 || (s.flags & ~known)) return set_error(GX_ERR_INVALID, "step %u has invalid flags", i);
        if ((s.flags & GX_STEP_PROBE) && (s.flags & GX_STEP_GROUP))
            return set_error(GX_ERR_INVALID, "step %u: PROBE and GROUP are exclusive", i);
        cols[i] = c;
        ScanStep& d = Q->steps[i];
        d.col = c->view();
        d.flags = s.flags;
        d.lo = s.lo;
        d.hi = s.hi;
        if (s.flags & GX_STEP_PROBE) {
            if (!s.ht) return set_error(GX_ERR_INVALID, "step %u probes a null hash table", i);
            d.ht = s.ht->slots;
            d.ht_log2 = s.ht->log2cap;
            d.ht_layout = s.ht->layout;
        }
        if ((s.flags & GX_STEP_GROUP) && s.digit_card == 0)
            return set_error(GX_ERR_INVALID, "step %u: GROUP needs digit_card > 0", i);
        if ((s.flags & (GX_STEP_PROBE | GX_STEP_GROUP)) && s.digit_card) {
            d.digit_base = s.digit_base;
            d.digit_card = s.digit_card;
            d.first_digit = any_digit ? 0 : 1;
            any_digit = true;
            card_prod *= s.digit_card;
            if (card_prod >= 0xFFFFFFFFull) return set_error(GX_ERR_INVALID, "group key space exceeds 2^32-1");
        }
        if (s.flags & GX_STEP_CARRY) any_carry = true;
        if (s.flags & GX_STEP_VALUE) any_value = true;
    }
    if (!any_value) return set_error(GX_ERR_INVALID, "scan plan has no VALUE step");
    if (plan->agg > GX_AGG_SUM_DIFF) return set_error(GX_ERR_INVALID, "unknown aggregate");
    if (plan->agg == GX_AGG_BUILD) {
        if (!plan->build_ht) return set_error(GX_ERR_INVALID, "a BUILD plan needs build_ht");
        if (plan->build_ht->layout == GX_HT_DENSE)
            return set_error(GX_ERR_INVALID, "a BUILD plan fills linear or bucket tables (dense tables size "
                                             "themselves from the key range in gx_hashtable_build)");
        if (plan->groupby || any_digit) return set_error(GX_ERR_INVALID, "a BUILD plan has no group key");
    }
    if ((plan->agg == GX_AGG_SUM_PRODUCT || plan->agg == GX_AGG_SUM_DIFF) && !any_carry)
        return set_error(GX_ERR_INVALID, "SUM_PRODUCT / SUM_DIFF need a CARRY step");
    Q->carry_digits = any_carry && any_digit ? 1 : 0;  // only the shared and pipelined forms keep both
    if (plan->groupby && !any_digit) return set_error(GX_ERR_INVALID, "grouped scan needs PROBE/GROUP steps with digits");
    if (!plan->groupby && !plan->result_dev && plan->agg != GX_AGG_BUILD)
        return set_error(GX_ERR_INVALID, "scan plan needs result_dev or groupby");
    if (!plan->groupby && any_digit) return set_error(GX_ERR_INVALID, "group-key digits need a groupby table");
    Q->n_steps = plan->n_steps;
    Q->agg = plan->agg;
    Q->grouped = plan->groupby ? 1 : 0;
    Q->need_aux = (any_carry || any_digit) ? 1 : 0;
    Q->row_lo = 0;
    Q->row_hi = ~0ull;
    Q->result = plan->result_dev;
    if (plan->groupby) {
        Q->g_keys = plan->groupby->keys;
        Q->g_sums = plan->groupby->sums;
        Q->g_log2 = plan->groupby->log2cap;
    }
    if (plan->n_prune > GX_MAX_STEPS) return set_error(GX_ERR_INVALID, "too many prune predicates");
    for (uint32_t i = 0; i < plan->n_prune; ++i) {
        const gx_column* pc = plan->prune[i].col;
        if (!pc || !pc->residency) return set_error(GX_ERR_INVALID, "prune column %u not on device", i);
        if (pc->n_chunks != c0->n_chunks) return set_error(GX_ERR_INVALID, "prune column %u has another chunking", i);
        Q->prune[i] = PrunePred{pc->d_mins, pc->d_maxs, plan->prune[i].lo, plan->prune[i].hi, pc->d_bmins, pc->d_bmaxs};
    }
    Q->n_prune = plan->n_prune;
    *tile_rows = pick_tile_rows(cols, plan->n_steps);
    *ref_col = c0;
    return GX_OK;
}

static gx_status ensure_kernel_attrs() {
    static bool attr_set[kMaxDevices] = {false};
    int dev = 0;
    cudaGetDevice(&dev);
    if (!device_index_ok(dev)) return set_error(GX_ERR_INVALID, "device %d out of range", dev);
    if (attr_set[dev]) return GX_OK;
    gx_status st = allow_smem(scan_kernel<128, kTileRows, false>, scan_smem_bytes<kTileRows>(true, true));
    if (!st) st = allow_smem(scan_kernel<128, kTileRows, true>, scan_smem_bytes<kTileRows>(true, true));
    if (!st) st = allow_smem(scan_kernel<256, kMaxRowsPerBlock, false>, scan_smem_bytes<kMaxRowsPerBlock>(true, true));
    if (!st) st = allow_smem(scan_kernel<256, kMaxRowsPerBlock, true>, scan_smem_bytes<kMaxRowsPerBlock>(true, true));
    const size_t sh_max = kShMaxDynSmem;
    if (!st) st = allow_smem(shared_scan_kernel<128, 4>, sh_max);
    if (!st) st = allow_smem(shared_scan_kernel<256, 2>, sh_max);
    if (!st) st = allow_smem(shared_scan_kernel<512, 1>, sh_max);
    if (!st) st = allow_smem(shared_scan_kernel<1024, 1>, sh_max);
    if (!st) st = allow_smem(shared_scan_kernel<kShSingleNT, 4, true>, sh_max);
    if (!st) st = allow_smem(pipe_scan_kernel, kPipeMaxDynSmem);
    if (!st) st = allow_smem(warp_scan_kernel<0>, kWsMaxDynSmem);
    if (!st) st = allow_smem(warp_scan_kernel<kSigQ1>, kWsMaxDynSmem);
    if (!st) st = allow_smem(warp_scan_kernel<kSigQ2>, kWsMaxDynSmem);
    if (!st) st = allow_smem(warp_scan_kernel<kSigQ3>, kWsMaxDynSmem);
    if (!st) st = allow_smem(warp_scan_kernel<kSigQ4>, kWsMaxDynSmem);
    if (st) return st;
    attr_set[dev] = true;
    return GX_OK;
}

// Grid and shared memory of a scan launch (persistent: CTAs per SM x SMs).
template <bool BATCH>
static void scan_geometry(uint32_t tile_rows, bool aux, bool groups, uint64_t tiles, uint32_t* grid, uint32_t* threads,
                          size_t* smem) {
    if (tile_rows <= kTileRows) {
        *smem = scan_smem_bytes<kTileRows>(aux, groups);
        // resident CTAs per SM, per device and shared-memory layout (queried once)
        static int occ[kMaxDevices][2][2] = {};  // ensure_kernel_attrs has checked the device
        int dev = 0;
        cudaGetDevice(&dev);
        int& per_sm = occ[dev][aux][groups];
        if (per_sm == 0) {
            int v = 1;
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&v, scan_kernel<128, kTileRows, BATCH>, 128, *smem);
            per_sm = std::max(1, v);
        }
        *grid = (uint32_t)std::max<uint64_t>(1, std::min<uint64_t>((uint64_t)sm_count() * per_sm, tiles));
        *threads = 128;
    } else {
        *smem = scan_smem_bytes<kMaxRowsPerBlock>(aux, groups);
        *grid = (uint32_t)std::max<uint64_t>(1, std::min<uint64_t>(sm_count(), tiles));
        *threads = 256;
    }
}

template <bool BATCH>
static void launch_scan_kernel(const ScanParams& P, uint32_t grid, uint32_t threads, size_t smem, cudaStream_t s) {
    if (threads == 128)
        scan_kernel<128, kTileRows, BATCH><<<grid, 128, smem, s>>>(P);
    else
        scan_kernel<256, kMaxRowsPerBlock, BATCH><<<grid, 256, smem, s>>>(P);
}

// One query of the shared form: fills `out` from the plan and its validated
// descriptor, adding the plan's columns to `cols`.  Returns false (why = the
// reason) when the plan does not qualify.
static bool shared_query(const gx_scan_plan& pl, const QueryDesc& qd, std::vector<const gx_column*>& cols,
                         ShQuery& out, std::string* why) {
    std::memset(&out, 0, sizeof(ShQuery));
    for (uint32_t k = 0; k < pl.n_steps; ++k) {
        const bool is_value = (pl.steps[k].flags & GX_STEP_VALUE) != 0;
        if (is_value != (k + 1 == pl.n_steps)) {
            *why = "a plan whose only VALUE step is not its last step";
            return false;
        }
        const gx_column* c = pl.steps[k].col;
        if (c->codec == GX_CODEC_LZ4 && (c->S <= 1 || (1u << c->seg_shift) > kShTile)) {
            *why = "an LZ4 column without segments of at most 2048 rows";
            return false;
        }
        uint32_t ci = 0;
        while (ci < cols.size() && cols[ci] != c) ++ci;
        if (ci == cols.size()) {
            if (cols.size() == kShMaxCols) {
                *why = "more than 16 distinct columns";
                return false;
            }
            cols.push_back(c);
        }
        const ScanStep& d = qd.steps[k];
        ShStep& e = out.steps[k];
        e.flags = d.flags;
        e.lo = d.lo;
        e.hi = d.hi;
        e.col = ci;
        e.ht = d.ht;
        e.ht_log2 = d.ht_log2;
        e.ht_layout = d.ht_layout;
        e.digit_base = d.digit_base;
        e.digit_card = d.digit_card;
        out.col_mask |= 1u << ci;
    }
    out.n_steps = pl.n_steps;
    out.agg = qd.agg;
    out.grouped = qd.grouped;
    out.row_lo = qd.row_lo;
    out.row_hi = qd.row_hi;
    out.result = qd.result;
    out.g_keys = qd.g_keys;
    out.g_sums = qd.g_sums;
    out.g_log2 = qd.g_log2;
    out.n_prune = qd.n_prune;
    for (uint32_t p = 0; p < out.n_prune; ++p) out.prune[p] = qd.prune[p];
    return true;
}

// Layout fields of the shared-form parameters for a table whose first column is c0.
static void shared_layout(ShParams& P, const gx_column* c0) {
    P.blocks_per_chunk = c0->blocks_per_chunk;
    P.rows_per_chunk = c0->rows_per_chunk;
    P.rows_per_block = c0->rows_per_block;
    P.tile_rows = std::min<uint32_t>(kShTile, c0->rows_per_block);
    P.tiles_per_block = (c0->rows_per_block + P.tile_rows - 1) / P.tile_rows;
    P.dir = c0->d_blocks;
    P.n_slots = c0->n_slots;
}

static size_t shared_smem_bytes(uint32_t n_cols, uint32_t n_queries, uint32_t qc_bytes = 0, uint32_t pst_words = 0,
                                uint32_t gt_slots = 0) {
    const bool tail = qc_bytes || pst_words || gt_slots;  // 16-byte aligned region after the query mask
    return 4ull * kShColWords * n_cols + Cfg<kTileRows>::kStage + 8ull * n_queries + 4ull * ((n_queries + 31) / 32) +
           (tail ? 16ull : 0ull) + qc_bytes + 4ull * pst_words + 12ull * gt_slots;
}

// Prefix groups of a batch.  Queries whose first steps (any but the VALUE
// step) are identical -- same column, flags, bounds, join table and digits --
// evaluate those steps once per tile in the shared scan.  shared_group sorts
// the queries so that equal step sequences sit next to each other (stable:
// equal ones keep their order; results do not depend on the order, every
// query carries its own outputs) and marks each run of two or more adjacent
// queries inside one 32-query mask word; the run shares the shortest common
// prefix of its neighbours.
struct ShGroup {
    uint32_t gbits = 0;
    uint8_t pfx = 0, psave = 0;
};

static int sh_step_cmp(const ShStep& x, const ShStep& y) {
    const uint64_t a[9] = {x.col, x.flags, (uint64_t)(uint32_t)x.lo, (uint64_t)(uint32_t)x.hi, (uint64_t)(uintptr_t)x.ht,
                           x.ht_log2, x.ht_layout, (uint64_t)(uint32_t)x.digit_base, x.digit_card};
    const uint64_t b[9] = {y.col, y.flags, (uint64_t)(uint32_t)y.lo, (uint64_t)(uint32_t)y.hi, (uint64_t)(uintptr_t)y.ht,
                           y.ht_log2, y.ht_layout, (uint64_t)(uint32_t)y.digit_base, y.digit_card};
    for (int i = 0; i < 9; ++i)
        if (a[i] != b[i]) return a[i] < b[i] ? -1 : 1;
    return 0;
}

static uint32_t sh_common_prefix(const ShQuery& x, const ShQuery& y) {
    const uint32_t lim = std::min(x.n_steps, y.n_steps) - 1;  // the VALUE step is never shared
    uint32_t k = 0;
    while (k < lim && sh_step_cmp(x.steps[k], y.steps[k]) == 0) ++k;
    return k;
}

static std::vector<ShGroup> shared_group(std::vector<ShQuery>& sq) {
    std::stable_sort(sq.begin(), sq.end(), [](const ShQuery& x, const ShQuery& y) {
        const uint32_t lim = std::min(x.n_steps, y.n_steps) - 1;
        for (uint32_t k = 0; k < lim; ++k)
            if (const int c = sh_step_cmp(x.steps[k], y.steps[k])) return c < 0;
        return x.n_steps < y.n_steps;
    });
    std::vector<ShGroup> g(sq.size());
    size_t i = 0;
    while (i < sq.size()) {
        size_t j = i + 1;
        uint32_t p = ~0u;
        for (; j < sq.size() && j % 32 != 0; ++j) {
            const uint32_t l = sh_common_prefix(sq[j - 1], sq[j]);
            if (l == 0) break;
            p = std::min(p, l);
        }
        if (j - i >= 2) {
            ShGroup e;
            e.gbits = (uint32_t)((((1ull << (j - i)) - 1ull) << (i % 32)) & 0xFFFFFFFFull);
            e.pfx = (uint8_t)p;
            for (uint32_t k = 0; k < p; ++k) {
                if (sq[i].steps[k].digit_card) e.psave |= 1;
                if (sq[i].steps[k].flags & GX_STEP_CARRY) e.psave |= 2;
            }
            for (size_t k = i; k < j; ++k) g[k] = e;
        }
        i = j;
    }
    return g;
}

// Words of prefix state the batch's groups need (group-key digits, carried
// values: one word per tile row each) and the offset of the carried values.
static uint32_t shared_pst_words(const std::vector<ShGroup>& g, uint32_t* carry_off) {
    bool gk = false, cv = false;
    for (const ShGroup& e : g) {
        gk = gk || (e.psave & 1);
        cv = cv || (e.psave & 2);
    }
    *carry_off = gk ? kShTile : 0u;
    return kShTile * ((gk ? 1u : 0u) + (cv ? 1u : 0u));
}

// The compact descriptor image of a batch: ShQueryC per query, then ShStepC
// per step, padded to 16 bytes.
static std::vector<uint8_t> shared_compact(const std::vector<ShQuery>& sq, const std::vector<ShGroup>& groups) {
    size_t steps = 0;
    for (const ShQuery& q : sq) steps += q.n_steps;
    const size_t bytes = (sizeof(ShQueryC) * sq.size() + sizeof(ShStepC) * steps + 15) & ~(size_t)15;
    std::vector<uint8_t> img(bytes, 0);
    ShQueryC* qc = (ShQueryC*)img.data();
    ShStepC* sc = (ShStepC*)(img.data() + sizeof(ShQueryC) * sq.size());
    uint32_t k = 0;
    for (size_t i = 0; i < sq.size(); ++i) {
        const ShQuery& q = sq[i];
        qc[i].row_lo = q.row_lo;
        qc[i].row_hi = q.row_hi;
        qc[i].g_keys = q.g_keys;
        qc[i].g_sums = q.g_sums;
        qc[i].step0 = k;
        qc[i].n_steps = (uint8_t)q.n_steps;
        qc[i].agg = (uint8_t)q.agg;
        qc[i].grouped = (uint8_t)q.grouped;
        qc[i].g_log2 = (uint8_t)q.g_log2;
        qc[i].gbits = groups[i].gbits;
        qc[i].pfx = groups[i].pfx;
        qc[i].psave = groups[i].psave;
        qc[i].col_mask = (uint16_t)q.col_mask;
        for (uint32_t t = 0; t < q.n_steps; ++t, ++k) {
            const ShStep& st = q.steps[t];
            sc[k].lo = st.lo;
            sc[k].hi = st.hi;
            sc[k].ht = st.ht;
            sc[k].dbase = st.digit_base;
            sc[k].dcard = st.digit_card;
            sc[k].col = (uint8_t)st.col;
            sc[k].flags = (uint8_t)st.flags;
            sc[k].htlog = (uint8_t)st.ht_log2;
            sc[k].htlay = (uint8_t)st.ht_layout;
        }
    }
    return img;
}

// A plan that qualifies for the shared form (its only VALUE step last, LZ4
// columns segmented) runs as a one-query shared scan: the query rides in the
// kernel parameters, columns are decoded per 2048-row tile only when a step
// needs them.  *done = false when the plan does not qualify.
static gx_status scan_launch_shared(const gx_scan_plan* plan, const QueryDesc& qd, const gx_column* c0,
                                    cudaStream_t s, unsigned long long* rows_dev, bool* done) {
    *done = false;
    std::vector<const gx_column*> cols;
    std::string why;
    ShParams P;
    std::memset(&P, 0, sizeof(P));
    if (!shared_query(*plan, qd, cols, P.q1, &why)) return GX_OK;
    P.q1.keep_in = plan->keep_chunks_dev;
    P.q1.keep_out = plan->keep_out_dev;
    for (size_t i = 0; i < cols.size(); ++i) P.cols1[i] = cols[i]->view();
    P.n_cols = (uint32_t)cols.size();
    P.n_queries = 1;
    P.mask_words = 1;
    shared_layout(P, c0);
    P.rows_scanned = rows_dev;
    const uint32_t n_slots = c0->n_slots;
    // no work list: the kernel's CTAs check their share of the (slot, tile)
    // items themselves (see sh_single_live), so the launch is one kernel
    P.gt_slots = P.q1.grouped ? kShGroupSlots : 0u;
    const size_t smem = shared_smem_bytes(P.n_cols, 1, 0, 0, P.gt_slots);
    static int occ[kMaxDevices][kShMaxCols + 1][2] = {};  // ensure_kernel_attrs has checked the device
    int dev = 0;
    cudaGetDevice(&dev);
    int& per_sm = occ[dev][P.n_cols][P.gt_slots ? 1 : 0];
    if (per_sm == 0) {
        int v = 1;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&v, shared_scan_kernel<kShSingleNT, 4, true>, kShSingleNT, smem);
        per_sm = std::max(1, v);
    }
    const uint64_t tiles = (uint64_t)n_slots * P.tiles_per_block;
    const unsigned grid = (unsigned)std::max<uint64_t>(1, std::min<uint64_t>((uint64_t)sm_count() * per_sm, tiles));
    shared_scan_kernel<kShSingleNT, 4, true><<<grid, kShSingleNT, smem, s>>>(P);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return set_error(GX_ERR_CUDA, "shared scan launch: %s", cudaGetErrorString(e));
    *done = true;
    return GX_OK;
}

// A plan that qualifies for the shared form and reads only HBM-resident
// columns runs as the warp-specialised pipeline (pipe_scan_kernel): one CTA
// per SM, a ring of stages sized to the shared memory.  *done = false when the
// plan does not qualify.
// A streamed scan's chunk group: chunks [chunk_lo, chunk_hi) of the table,
// with the payloads of the listed (pinned-host) columns staged in HBM; a
// staged view's payload pointer stands for payload offset 0.
struct PipeGroup {
    uint32_t chunk_lo, chunk_hi;
    uint32_t n;
    const gx_column* col[kPipeMaxCols];
    const uint8_t* payload[kPipeMaxCols];
};

static gx_status scan_launch_pipe(const gx_scan_plan* plan, const QueryDesc& qd, const gx_column* c0,
                                  cudaStream_t s, unsigned long long* rows_dev, bool* done,
                                  const PipeGroup* grp = nullptr) {
    *done = false;
    std::vector<const gx_column*> cols;
    std::string why;
    PipeParams P;
    std::memset(&P, 0, sizeof(P));
    if (!shared_query(*plan, qd, cols, P.q, &why)) return GX_OK;
    if (cols.size() > kPipeMaxCols) return GX_OK;
    uint32_t dec = 0, n_dec = 0;
    for (size_t i = 0; i < cols.size(); ++i) {
        const gx_column* c = cols[i];
        const uint8_t* staged = nullptr;
        for (uint32_t k = 0; grp && k < grp->n; ++k)
            if (grp->col[k] == c) staged = grp->payload[k];
        if (c->residency != 1 && !staged) return GX_OK;  // pinned-host columns: zero-copy reads in the shared form
        if (c->codec != GX_CODEC_NONE) {
            dec |= 1u << i;
            ++n_dec;
        }
        P.cols[i] = c->view();
        if (staged) {
            P.cols[i].payload = staged;
            P.cols[i].host_mapped = 0;
        }
    }
    P.q.keep_in = plan->keep_chunks_dev;
    P.q.keep_out = plan->keep_out_dev;
    P.n_cols = (uint32_t)cols.size();
    P.n_chunks = c0->n_chunks;
    P.chunk_lo = grp ? grp->chunk_lo : 0u;
    P.chunk_hi = grp ? grp->chunk_hi : c0->n_chunks;
    P.blocks_per_chunk = c0->blocks_per_chunk;
    P.rows_per_chunk = c0->rows_per_chunk;
    P.rows_per_block = c0->rows_per_block;
    P.tile_rows = std::min<uint32_t>(kPipeTile, c0->rows_per_block);
    P.tiles_per_block = (c0->rows_per_block + P.tile_rows - 1) / P.tile_rows;
    P.n_rows = c0->n_rows;
    P.dec_mask = dec;
    P.gt_slots = P.q.grouped ? kShGroupSlots : 0u;
    P.rows_scanned = rows_dev;
    if (plan->agg == GX_AGG_BUILD) {
        P.build_rowid = 1;
        for (uint32_t k = 0; k < plan->n_steps; ++k)
            if (plan->steps[k].flags & GX_STEP_CARRY) P.build_rowid = 0;
        P.build_slots = plan->build_ht->slots;
        P.build_log2 = plan->build_ht->log2cap;
        P.build_layout = plan->build_ht->layout;
        P.build_counters = plan->build_ht->counters;
    }
    const size_t fixed = 4ull * kShColWords * n_dec + 8ull * kCascPageMaxRuns + 12ull * P.gt_slots;
    const size_t per_stage = (size_t)kPipeColBytes * P.n_cols;
    if (fixed + 2 * per_stage > kPipeMaxDynSmem) return GX_OK;
    P.stages = (uint32_t)std::min<size_t>(kPipeMaxStages, (kPipeMaxDynSmem - fixed) / per_stage);
    const size_t smem = fixed + P.stages * per_stage;
    const uint64_t tiles = (uint64_t)(P.chunk_hi - P.chunk_lo) * c0->blocks_per_chunk * P.tiles_per_block;
    const unsigned grid = (unsigned)std::max<uint64_t>(1, std::min<uint64_t>((uint64_t)sm_count(), tiles));
    pipe_scan_kernel<<<grid, kPipeNT, smem, s>>>(P);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return set_error(GX_ERR_CUDA, "pipelined scan launch: %s", cudaGetErrorString(e));
    *done = true;
    return GX_OK;
}

// Form selection of gx_scan (gx_scan_set_form): process-wide.
static std::atomic<uint32_t> g_scan_form{GX_FORM_AUTO};

// 1 when every block of an LZ4 column is one literal run whose first byte is
// 16-byte aligned in the payload (the warp-tile scan then reads the column in
// place and gives it no decode buffer).  Computed once from the host copy.
static bool lz4_all_direct(const gx_column* c) {
    if (c->lz4_direct >= 0) return c->lz4_direct != 0;
    bool ok = c->codec == GX_CODEC_LZ4;
    for (uint32_t sl = 0; ok && sl < c->n_slots; ++sl) {
        const gx::gx_dblock& d = c->blocks[sl];
        if (!d.n_rows) continue;
        if (d.offset + d.comp_bytes > c->payload.size() || d.comp_bytes == 0) {
            ok = false;
            break;
        }
        const uint8_t* p = c->payload.data() + d.offset;
        uint64_t pos = 1, lit = p[0] >> 4;
        if ((p[0] & 15u) != 0 && lit != 15) {
            ok = false;
            break;
        }
        if (lit == 15) {
            uint8_t x;
            do {
                if (pos >= d.comp_bytes) break;
                x = p[pos++];
                lit += x;
            } while (x == 255);
        }
        ok = lit == 4ull * d.n_rows && pos + lit == d.comp_bytes && ((d.offset + pos) & 15u) == 0;
    }
    c->lz4_direct = ok ? 1 : 0;
    return ok;
}

// The warp-tile scan (warp_scan_kernel) for a plan, or *done = false when
// the plan is not of its shape: HBM-resident (or staged) columns sharing the
// table layout, LZ4 ones segmented with segments of at most kWsTile rows, no
// BUILD, at most 32768 chunks.  Shared memory per warp: one kWsTile-row area
// per column (a stage area for raw and all-literal LZ4 columns, a decode
// buffer for cascaded and other LZ4 columns) and a group table for grouped
// plans.
static gx_status scan_launch_warp(const gx_scan_plan* plan, const QueryDesc& qd, const gx_column* c0, cudaStream_t s,
                                  unsigned long long* rows_dev, bool* done, const PipeGroup* grp = nullptr) {
    *done = false;
    if (plan->agg == GX_AGG_BUILD) return GX_OK;
    std::vector<const gx_column*> cols;
    std::string why;
    WsParams P;
    std::memset(&P, 0, sizeof(P));
    if (!shared_query(*plan, qd, cols, P.q, &why)) return GX_OK;
    if (cols.size() > kWsMaxCols) return GX_OK;
    uint32_t areas = 0;
    for (size_t i = 0; i < kWsMaxCols; ++i) P.stage_of[i] = P.buf_of[i] = kWsNone;
    for (size_t i = 0; i < cols.size(); ++i) {
        const gx_column* c = cols[i];
        const uint8_t* staged = nullptr;
        for (uint32_t k = 0; grp && k < grp->n; ++k)
            if (grp->col[k] == c) staged = grp->payload[k];
        if (c->residency != 1 && !staged) return GX_OK;
        if (c->rows_per_block != c0->rows_per_block || c->rows_per_chunk != c0->rows_per_chunk) return GX_OK;
        if (c->codec == GX_CODEC_LZ4 && (c->S <= 1 || c->seg_shift > kWsLog2)) return GX_OK;
        P.cols[i] = c->view();
        if (staged) {
            P.cols[i].payload = staged;
            P.cols[i].host_mapped = 0;
        }
        if (c->codec == GX_CODEC_NONE || (c->codec == GX_CODEC_LZ4 && lz4_all_direct(c)))
            P.stage_of[i] = areas++;
        else
            P.buf_of[i] = areas++;
    }
    P.q.keep_in = plan->keep_chunks_dev;
    P.q.keep_out = plan->keep_out_dev;
    P.n_cols = (uint32_t)cols.size();
    P.blocks_per_chunk = c0->blocks_per_chunk;
    P.rows_per_chunk = c0->rows_per_chunk;
    P.rows_per_block = c0->rows_per_block;
    P.tiles_per_block = (c0->rows_per_block + kWsTile - 1) / kWsTile;
    P.n_rows = c0->n_rows;
    P.chunk_lo = grp ? grp->chunk_lo : 0u;
    P.chunk_hi = grp ? grp->chunk_hi : c0->n_chunks;
    const uint32_t n_range = P.chunk_hi - P.chunk_lo;
    P.chunk_words = ((n_range + 31) / 32 + 3) & ~3u;
    if (P.chunk_words > kWsMaxChunkWords) return GX_OK;
    // the kernel indexes tiles in 32 bits (with room for its stride)
    if ((uint64_t)n_range * P.blocks_per_chunk * P.tiles_per_block >= (1ull << 31)) return GX_OK;
    P.n_areas = areas;
    P.grouped_tab = P.q.grouped ? 1u : 0u;
    P.rows_scanned = rows_dev;
    // the plan's signature: a compile-time evaluator when one matches
    uint32_t kinds[GX_MAX_STEPS] = {};
    for (uint32_t k = 0; k < plan->n_steps; ++k) {
        const uint32_t f = plan->steps[k].flags;
        kinds[k] = ((f & GX_STEP_FILTER) ? kWkF : 0u) | ((f & GX_STEP_PROBE) ? kWkP : 0u) |
                   ((f & GX_STEP_CARRY) ? kWkC : 0u) | (P.q.steps[k].digit_card ? kWkD : 0u);
    }
    const uint32_t sig = plan->n_steps <= 6 ? ws_sig(plan->n_steps, P.q.agg, P.q.grouped != 0, kinds[0], kinds[1],
                                                     kinds[2], kinds[3], kinds[4], kinds[5])
                                            : 0u;
    void (*kern)(WsParams) = warp_scan_kernel<0>;
    if (sig == kSigQ1) kern = warp_scan_kernel<kSigQ1>;
    else if (sig == kSigQ2) kern = warp_scan_kernel<kSigQ2>;
    else if (sig == kSigQ3) kern = warp_scan_kernel<kSigQ3>;
    else if (sig == kSigQ4) kern = warp_scan_kernel<kSigQ4>;
    // shared memory per warp: the areas, then (grouped) the run-time
    // evaluator's per-row group keys and the group table
    const bool rt_eval = kern == warp_scan_kernel<0>;
    P.warp_words = kWsHead + areas * kWsTile + (P.grouped_tab && rt_eval ? kWsTile : 0u);
    const size_t smem = 4ull * (2ull * P.chunk_words + (size_t)P.warp_words * kWsWarps +
                                (P.grouped_tab ? 3ull * kWsGroupSlots : 0ull));
    if (smem > kWsMaxDynSmem) return GX_OK;
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kWsNT, smem) != cudaSuccess || per_sm < 1)
        return set_error(GX_ERR_CUDA, "warp scan occupancy query failed");
    const uint64_t tiles = (uint64_t)n_range * c0->blocks_per_chunk * P.tiles_per_block;
    const uint64_t want = (tiles + kWsWarps - 1) / kWsWarps;
    const unsigned grid = (unsigned)std::max<uint64_t>(1, std::min<uint64_t>((uint64_t)sm_count() * per_sm, want));
    // programmatic dependent launch: the scan's chunk pruning, tile decisions
    // and first copies overlap the kernel before it on the stream (typically
    // the join-table build); the kernel waits for it before it reads a join
    // table or writes a result.  Not for streamed groups, whose staging copies
    // arrive on another stream.
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(kWsNT);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = grp ? 0u : 1u;
    cudaError_t e = cudaLaunchKernelEx(&cfg, kern, P);
    if (e == cudaSuccess) e = cudaGetLastError();
    if (e != cudaSuccess) return set_error(GX_ERR_CUDA, "warp scan launch: %s", cudaGetErrorString(e));
    *done = true;
    return GX_OK;
}

static gx_status scan_launch(const gx_scan_plan* plan, cudaStream_t s, unsigned long long* rows_dev) {
    ScanParams P;
    std::memset(&P, 0, sizeof(P));
    const gx_column* c0 = nullptr;
    uint32_t tile_rows = 0;
    gx_status st = build_query(plan, &P.q, &tile_rows, &c0);
    if (st) return st;
    st = ensure_kernel_attrs();
    if (st) return st;
    bool done = false;
    const uint32_t form = g_scan_form.load(std::memory_order_relaxed);
    if (form == GX_FORM_AUTO || form == GX_FORM_WARP) {
        st = scan_launch_warp(plan, P.q, c0, s, rows_dev, &done);
        if (st || done) return st;
        if (form == GX_FORM_WARP) return set_error(GX_ERR_INVALID, "the plan is not of the warp-tile form's shape");
    }
    if (form == GX_FORM_AUTO || form == GX_FORM_PIPE) {
        st = scan_launch_pipe(plan, P.q, c0, s, rows_dev, &done);
        if (st || done) return st;
        if (form == GX_FORM_PIPE) return set_error(GX_ERR_INVALID, "the plan is not of the pipelined form's shape");
    }
    if (plan->agg == GX_AGG_BUILD)
        return set_error(GX_ERR_INVALID, "a BUILD plan needs HBM-resident columns (LZ4 ones segmented, segments of "
                                         "at most 2048 rows) and its VALUE step last");
    if (form == GX_FORM_AUTO || form == GX_FORM_SHARED) {
        st = scan_launch_shared(plan, P.q, c0, s, rows_dev, &done);
        if (st || done) return st;
        if (form == GX_FORM_SHARED) return set_error(GX_ERR_INVALID, "the plan is not of the shared form's shape");
    }
    if (P.q.carry_digits)
        return set_error(GX_ERR_INVALID, "a plan with a carried value and group-key digits needs the shared or "
                                         "pipelined form (segmented LZ4 columns, its only VALUE step last)");
    ItemsParams ip{};
    for (uint32_t i = 0; i < P.q.n_prune; ++i) ip.preds[i] = P.q.prune[i];
    ip.n_preds = P.q.n_prune;
    ip.n_chunks = c0->n_chunks;
    ip.keep_in = plan->keep_chunks_dev;
    ip.keep_out = plan->keep_out_dev;
    const uint32_t n_chunks = c0->n_chunks;
    uint32_t* scratch = nullptr;
    GX_CK(scratch_alloc((void**)&scratch, 4ull * (n_chunks + 4), s));
    ip.n_items = scratch;
    ip.work_counter = scratch + 1;
    ip.items = scratch + 4;
    items_kernel<<<1, 1024, 0, s>>>(ip);
    P.blocks_per_chunk = c0->blocks_per_chunk;
    P.rows_per_chunk = c0->rows_per_chunk;
    P.rows_per_block = c0->rows_per_block;
    P.tile_rows = tile_rows;
    P.tiles_per_block = (c0->rows_per_block + tile_rows - 1) / tile_rows;
    P.smem_aux = P.q.need_aux;
    P.smem_groups = P.q.grouped;
    P.items = ip.items;
    P.n_items = ip.n_items;
    P.work_counter = ip.work_counter;
    P.rows_scanned = rows_dev;
    const uint64_t tiles = (uint64_t)n_chunks * c0->blocks_per_chunk * P.tiles_per_block;
    uint32_t grid = 1, threads = 128;
    size_t smem = 0;
    scan_geometry<false>(tile_rows, P.smem_aux, P.smem_groups, tiles, &grid, &threads, &smem);
    launch_scan_kernel<false>(P, grid, threads, smem, s);
    cudaError_t e = cudaGetLastError();
    cudaFreeAsync(scratch, s);
    if (e != cudaSuccess) return set_error(GX_ERR_CUDA, "scan launch: %s", cudaGetErrorString(e));
    return GX_OK;
}

// Streamed scan of pinned-host columns (gx_scan_streamed): chunk groups
// whose surviving chunks' compressed bytes are copied to HBM on a copy
// stream (double-buffered), each group scanned by the pipelined kernel while
// the next one is copied.
static gx_status scan_streamed(const gx_scan_plan* plan, uint32_t per_group, cudaStream_t s) {
    QueryDesc qd;
    uint32_t tile_rows = 0;
    const gx_column* c0 = nullptr;
    gx_status st = build_query(plan, &qd, &tile_rows, &c0);
    if (st) return st;
    st = ensure_kernel_attrs();
    if (st) return st;
    if (per_group == 0) return set_error(GX_ERR_INVALID, "gx_scan_streamed: chunks_per_group must be > 0");
    // the plan's distinct pinned-host columns
    std::vector<gx_column*> staged;
    for (uint32_t i = 0; i < plan->n_steps; ++i) {
        gx_column* c = const_cast<gx_column*>(plan->steps[i].col);
        if (c->residency == 2 && std::find(staged.begin(), staged.end(), c) == staged.end()) staged.push_back(c);
    }
    const uint32_t n_chunks = c0->n_chunks, bpc = c0->blocks_per_chunk;
    // chunk keep on the host: the plan's min/max predicates (the kernel applies
    // them again together with keep_chunks_dev)
    std::vector<uint8_t> keep(n_chunks, 1);
    for (uint32_t p = 0; p < plan->n_prune; ++p) {
        const gx_column* pc = plan->prune[p].col;
        for (uint32_t c = 0; c < n_chunks; ++c)
            if (!(plan->prune[p].lo <= pc->maxs[c] && plan->prune[p].hi >= pc->mins[c])) keep[c] = 0;
    }
    // byte range of chunk c of column col: [first block offset, last block end)
    auto chunk_range = [&](const gx_column* col, uint32_t c, uint64_t* a, uint64_t* b) {
        *a = col->blocks[(size_t)c * bpc].offset;
        *b = *a;
        for (uint32_t j = 0; j < bpc; ++j) {
            const gx_dblock& d = col->blocks[(size_t)c * bpc + j];
            if (d.n_rows) *b = std::max<uint64_t>(*b, d.offset + d.comp_bytes);
        }
    };
    // groups with a surviving chunk, and the staging bytes each column needs
    struct Group {
        uint32_t lo, hi;
    };
    std::vector<Group> groups;
    std::vector<uint64_t> cap(staged.size(), 0);
    for (uint32_t g0 = 0; g0 < n_chunks; g0 += per_group) {
        const uint32_t g1 = std::min(n_chunks, g0 + per_group);
        uint32_t first = g1, last = g0;
        for (uint32_t c = g0; c < g1; ++c)
            if (keep[c]) {
                first = std::min(first, c);
                last = c;
            }
        if (first == g1) continue;
        groups.push_back({first, last + 1});
        for (size_t k = 0; k < staged.size(); ++k) {
            uint64_t a0, b0, a1, b1;
            chunk_range(staged[k], first, &a0, &b0);
            chunk_range(staged[k], last, &a1, &b1);
            cap[k] = std::max<uint64_t>(cap[k], b1 - (a0 & ~15ull) + kPayloadSlack);
        }
    }
    if (plan->agg == GX_AGG_BUILD) return set_error(GX_ERR_INVALID, "gx_scan_streamed: BUILD plans are not streamed");
    // chunks outside every group's [first, last] range are pruned; the
    // launches write the flags of the chunks inside the ranges
    if (plan->keep_out_dev) GX_CK(cudaMemsetAsync(plan->keep_out_dev, 0, 2ull * n_chunks, s));
    if (groups.empty()) return GX_OK;
    std::vector<uint8_t*> buf(2 * staged.size(), nullptr);
    for (size_t k = 0; k < staged.size(); ++k)
        for (int b = 0; b < 2; ++b) GX_CK(scratch_alloc((void**)&buf[2 * k + b], cap[k], s));
    cudaStream_t cs = nullptr;
    cudaEvent_t ready, copied[2], consumed[2];
    GX_CK(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
    GX_CK(cudaEventCreateWithFlags(&ready, cudaEventDisableTiming));
    for (int b = 0; b < 2; ++b) {
        GX_CK(cudaEventCreateWithFlags(&copied[b], cudaEventDisableTiming));
        GX_CK(cudaEventCreateWithFlags(&consumed[b], cudaEventDisableTiming));
    }
    GX_CK(cudaEventRecord(ready, s));  // staging allocated (stream-ordered) before the first copy
    GX_CK(cudaStreamWaitEvent(cs, ready, 0));
    for (size_t gi = 0; gi < groups.size() && !st; ++gi) {
        const int b = (int)(gi & 1);
        const Group& G = groups[gi];
        if (gi >= 2) GX_CK(cudaStreamWaitEvent(cs, consumed[b], 0));
        PipeGroup pg{};
        pg.chunk_lo = G.lo;
        pg.chunk_hi = G.hi;
        for (size_t k = 0; k < staged.size(); ++k) {
            const gx_column* col = staged[k];
            uint64_t a0, b0;
            chunk_range(col, G.lo, &a0, &b0);
            const uint64_t base = a0 & ~15ull;
            // runs of surviving chunks, each copied at its offset in the group's range
            for (uint32_t c = G.lo; c < G.hi;) {
                if (!keep[c]) {
                    ++c;
                    continue;
                }
                uint32_t e = c;
                while (e + 1 < G.hi && keep[e + 1]) ++e;
                uint64_t ra, rb, ea, eb;
                chunk_range(col, c, &ra, &rb);
                chunk_range(col, e, &ea, &eb);
                ra &= ~15ull;
                const uint64_t end = std::min<uint64_t>(col->payload.size(), eb + kPayloadSlack);
                GX_CK(cudaMemcpyAsync(buf[2 * k + b] + (ra - base), (const uint8_t*)col->h_pinned + ra, end - ra,
                                      cudaMemcpyHostToDevice, cs));
                c = e + 1;
            }
            pg.col[pg.n] = col;
            pg.payload[pg.n++] = buf[2 * k + b] - base;
        }
        GX_CK(cudaEventRecord(copied[b], cs));
        GX_CK(cudaStreamWaitEvent(s, copied[b], 0));
        bool done = false;
        const uint32_t form = g_scan_form.load(std::memory_order_relaxed);
        if (form != GX_FORM_PIPE) st = scan_launch_warp(plan, qd, c0, s, nullptr, &done, &pg);
        if (!st && !done && form != GX_FORM_WARP) st = scan_launch_pipe(plan, qd, c0, s, nullptr, &done, &pg);
        if (!st && !done) st = set_error(GX_ERR_INVALID, "gx_scan_streamed: the plan needs the pipelined form");
        if (!st) GX_CK(cudaEventRecord(consumed[b], s));
    }
    for (uint8_t* p : buf) cudaFreeAsync(p, s);  // after the last kernel on s
    cudaEventDestroy(ready);
    for (int b = 0; b < 2; ++b) {
        cudaEventDestroy(copied[b]);
        cudaEventDestroy(consumed[b]);
    }
    cudaStreamDestroy(cs);
    return st;
}

// Work-list scratch of gx_scan_static, one per device: word 0 = surviving
// chunk count, word 1 = work counter, words 4.. = surviving chunk ids.
// items_kernel writes both counters before scan_kernel reads them (same
// stream), so no word needs to be zero beforehand.
constexpr uint32_t kStaticMaxChunks = GX_SCAN_STATIC_MAX_CHUNKS;
static __device__ __align__(256) uint32_t g_scan_static_scratch[4 + kStaticMaxChunks];

// Device address of g_scan_static_scratch on the current device, looked up
// once per device (with that device current) and cached.
static gx_status static_scratch(uint32_t** out) {
    static std::mutex mu;
    static uint32_t* addr[kMaxDevices] = {nullptr};
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return set_error(GX_ERR_CUDA, "gx_scan_static: cudaGetDevice: %s", cudaGetErrorString(e));
    if (!device_index_ok(dev)) return set_error(GX_ERR_INVALID, "gx_scan_static: device %d out of range", dev);
    std::lock_guard<std::mutex> lk(mu);
    if (!addr[dev]) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_scan_static_scratch);
        if (e != cudaSuccess || !p)
            return set_error(GX_ERR_CUDA, "gx_scan_static: cudaGetSymbolAddress: %s", cudaGetErrorString(e));
        addr[dev] = (uint32_t*)p;
    }
    *out = addr[dev];
    return GX_OK;
}

// scan_launch with the work list in g_scan_static_scratch: no allocation.
static gx_status scan_launch_static(const gx_scan_plan* plan, cudaStream_t s) {
    ScanParams P;
    std::memset(&P, 0, sizeof(P));
    const gx_column* c0 = nullptr;
    uint32_t tile_rows = 0;
    gx_status st = build_query(plan, &P.q, &tile_rows, &c0);
    if (st) return st;
    if (plan->agg == GX_AGG_BUILD) return set_error(GX_ERR_INVALID, "gx_scan_static: BUILD plans run through gx_scan");
    if (P.q.carry_digits)
        return set_error(GX_ERR_INVALID, "gx_scan_static: a carried value with group-key digits runs through gx_scan");
    const uint32_t n_chunks = c0->n_chunks;
    if (n_chunks > kStaticMaxChunks)
        return set_error(GX_ERR_INVALID, "gx_scan_static: %u chunks exceed the static work list of %u chunks", n_chunks,
                         kStaticMaxChunks);
    st = ensure_kernel_attrs();
    if (st) return st;
    uint32_t* scratch = nullptr;
    st = static_scratch(&scratch);
    if (st) return st;
    ItemsParams ip{};
    for (uint32_t i = 0; i < P.q.n_prune; ++i) ip.preds[i] = P.q.prune[i];
    ip.n_preds = P.q.n_prune;
    ip.n_chunks = n_chunks;
    ip.keep_in = plan->keep_chunks_dev;
    ip.keep_out = plan->keep_out_dev;
    ip.n_items = scratch;
    ip.work_counter = scratch + 1;
    ip.items = scratch + 4;
    items_kernel<<<1, 1024, 0, s>>>(ip);
    P.blocks_per_chunk = c0->blocks_per_chunk;
    P.rows_per_chunk = c0->rows_per_chunk;
    P.rows_per_block = c0->rows_per_block;
    P.tile_rows = tile_rows;
    P.tiles_per_block = (c0->rows_per_block + tile_rows - 1) / tile_rows;
    P.smem_aux = P.q.need_aux;
    P.smem_groups = P.q.grouped;
    P.items = ip.items;
    P.n_items = ip.n_items;
    P.work_counter = ip.work_counter;
    P.rows_scanned = nullptr;
    const uint64_t tiles = (uint64_t)n_chunks * c0->blocks_per_chunk * P.tiles_per_block;
    uint32_t grid = 1, threads = 128;
    size_t smem = 0;
    scan_geometry<false>(tile_rows, P.smem_aux, P.smem_groups, tiles, &grid, &threads, &smem);
    launch_scan_kernel<false>(P, grid, threads, smem, s);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return set_error(GX_ERR_CUDA, "gx_scan_static launch: %s", cudaGetErrorString(e));
    return GX_OK;
}

extern "C" {

gx_status gx_scan_static(const gx_scan_plan* plan, void* stream) {
    return scan_launch_static(plan, (cudaStream_t)stream);
}

gx_status gx_scan(const gx_scan_plan* plan, void* stream) {
    return scan_launch(plan, (cudaStream_t)stream, nullptr);
}

gx_status gx_scan_set_form(uint32_t form) {
    if (form > GX_FORM_QUEUE) return set_error(GX_ERR_INVALID, "unknown scan form %u", form);
    g_scan_form.store(form, std::memory_order_relaxed);
    return GX_OK;
}

gx_status gx_scan_streamed(const gx_scan_plan* plan, uint32_t chunks_per_group, void* stream) {
    return scan_streamed(plan, chunks_per_group, (cudaStream_t)stream);
}

gx_status gx_scan_check(void* stream) {
    cudaStream_t s = (cudaStream_t)stream;
    int err = 0, zero = 0;
    GX_CK(cudaMemcpyFromSymbolAsync(&err, g_gx_error, sizeof(int), 0, cudaMemcpyDeviceToHost, s));
    gx_status st = wait_stream(s, 120.0);
    if (st) return st;
    if (err) {
        GX_CK(cudaMemcpyToSymbolAsync(g_gx_error, &zero, sizeof(int), 0, cudaMemcpyHostToDevice, s));
        GX_CK(cudaStreamSynchronize(s));
        return set_error(err, "device reported %s", gx_status_str(err));
    }
    return GX_OK;
}

gx_status gx_scan_sync(const gx_scan_plan* plan, void* stream, uint64_t* rows_scanned) {
    cudaStream_t s = (cudaStream_t)stream;
    unsigned long long* rows = nullptr;
    if (rows_scanned) {
        GX_CK(scratch_alloc((void**)&rows, 8, s));
        GX_CK(cudaMemsetAsync(rows, 0, 8, s));
    }
    gx_status st = scan_launch(plan, s, rows);
    if (!st && rows_scanned) {
        unsigned long long r = 0;
        cudaMemcpyAsync(&r, rows, 8, cudaMemcpyDeviceToHost, s);
        st = wait_stream(s, 300.0);
        *rows_scanned = r;
    }
    if (rows) cudaFreeAsync(rows, s);
    if (st) return st;
    return gx_scan_check(stream);
}


}  // extern "C"

// Shared form: checks that the batch qualifies (why = the first reason it
// does not) and fills the shared descriptors; uploads on stream s.
static gx_status shared_prepare(gx_batch* b, const gx_query* queries, uint32_t n, const std::vector<QueryDesc>& qs,
                                const gx_column* c0, cudaStream_t s, bool* ok, std::string* why) {
    *ok = false;
    if (n > kShMaxQueries) {
        *why = "more than 1024 queries";
        return GX_OK;
    }
    std::vector<const gx_column*> cols;
    std::vector<ShQuery> sq(n);
    for (uint32_t i = 0; i < n; ++i)
        if (!shared_query(queries[i].plan, qs[i], cols, sq[i], why)) return GX_OK;
    const std::vector<ShGroup> groups = shared_group(sq);
    uint32_t pst_carry = 0;
    const uint32_t pst_words = shared_pst_words(groups, &pst_carry);
    const std::vector<uint8_t> img = shared_compact(sq, groups);
    if (img.size() > kShMaxQcBytes) {
        *why = "query descriptors above 96 KiB";
        return GX_OK;
    }
    bool any_grouped = false;
    for (const ShQuery& q : sq) any_grouped = any_grouped || q.grouped;
    const uint32_t gt_slots = any_grouped ? kShGroupSlots : 0u;
    if (shared_smem_bytes((uint32_t)cols.size(), n, (uint32_t)img.size(), pst_words, gt_slots) > kShMaxDynSmem) {
        *why = "columns, queries and descriptors above 220 KiB of shared memory";
        return GX_OK;
    }
    if (img.size() > b->cap_qc) {
        cudaFree(b->d_qc);
        cudaFreeHost(b->h_qc);
        b->d_qc = nullptr;
        b->h_qc = nullptr;
        b->cap_qc = 0;
        GX_CK(cudaMalloc(&b->d_qc, img.size()));
        GX_CK(cudaMallocHost(&b->h_qc, img.size()));
        b->cap_qc = img.size();
    }
    std::memcpy(b->h_qc, img.data(), img.size());
    GX_CK(cudaMemcpyAsync(b->d_qc, b->h_qc, img.size(), cudaMemcpyHostToDevice, s));
    const uint32_t mw = (n + 31) / 32;
    const uint32_t n_slots = c0->n_slots;
    // grow buffers (the stream's earlier work is finished by the caller)
    if (n > b->cap_sq) {
        cudaFree(b->d_sq);
        cudaFreeHost(b->h_sq);
        b->d_sq = nullptr;
        b->h_sq = nullptr;
        b->cap_sq = 0;
        GX_CK(cudaMalloc(&b->d_sq, sizeof(ShQuery) * n));
        GX_CK(cudaMallocHost(&b->h_sq, sizeof(ShQuery) * n));
        b->cap_sq = n;
    }
    if (!b->d_cols) {
        GX_CK(cudaMalloc(&b->d_cols, sizeof(gx_dcol) * kShMaxCols));
        GX_CK(cudaMallocHost(&b->h_cols, sizeof(gx_dcol) * kShMaxCols));
    }
    if ((size_t)n_slots * mw > b->cap_mask) {
        cudaFree(b->d_slot_mask);
        b->d_slot_mask = nullptr;
        b->cap_mask = 0;
        GX_CK(cudaMalloc(&b->d_slot_mask, 4ull * n_slots * mw));
        b->cap_mask = (size_t)n_slots * mw;
    }
    if (n_slots > b->cap_slots) {
        cudaFree(b->d_sh_items);
        b->d_sh_items = nullptr;
        b->cap_slots = 0;
        GX_CK(cudaMalloc(&b->d_sh_items, 4ull * (n_slots + 2)));
        b->cap_slots = n_slots;
    }
    std::memcpy(b->h_sq, sq.data(), sizeof(ShQuery) * n);
    for (size_t i = 0; i < cols.size(); ++i) b->h_cols[i] = cols[i]->view();
    GX_CK(cudaMemcpyAsync(b->d_sq, b->h_sq, sizeof(ShQuery) * n, cudaMemcpyHostToDevice, s));
    GX_CK(cudaMemcpyAsync(b->d_cols, b->h_cols, sizeof(gx_dcol) * cols.size(), cudaMemcpyHostToDevice, s));
    ShParams& P = b->SP;
    std::memset(&P, 0, sizeof(P));
    P.cols = b->d_cols;
    P.n_cols = (uint32_t)cols.size();
    P.qs = b->d_sq;
    P.n_queries = n;
    P.mask_words = mw;
    P.slot_mask = b->d_slot_mask;
    P.n_items = b->d_sh_items;
    P.work_counter = b->d_sh_items + 1;
    P.items = b->d_sh_items + 2;
    shared_layout(P, c0);
    P.rows_scanned = b->d_rows;
    P.qc = (const uint4*)b->d_qc;
    P.qc_bytes = (uint32_t)img.size();
    P.pst_carry = pst_carry;
    P.pst_words = pst_words;
    P.gt_slots = gt_slots;
    b->n_slots = n_slots;
    b->dir0 = c0->d_blocks;
    b->sh_smem = shared_smem_bytes(P.n_cols, n, P.qc_bytes, pst_words, gt_slots);
    shared_geometry(b);
    b->sh_items_grid = (uint32_t)std::max<uint64_t>(1, std::min<uint64_t>(8ull * sm_count(), (n_slots + 7) / 8));
    *ok = true;
    return GX_OK;
}

extern "C" {

gx_status gx_batch_assign(gx_batch* b, const gx_query* queries, uint32_t n_queries, void* stream) {
    if (!b || !queries || n_queries == 0) return set_error(GX_ERR_INVALID, "gx_batch_assign: bad args");
    cudaStream_t s = (cudaStream_t)stream;
    std::vector<QueryDesc> qs(n_queries);
    const gx_column* c0 = nullptr;
    uint32_t tile_rows = ~0u;
    bool aux = false, groups = false;
    uint64_t max_table = 0;
    std::vector<uint32_t> cq, cc;
    for (uint32_t i = 0; i < n_queries; ++i) {
        const gx_column* ci = nullptr;
        uint32_t tr = 0;
        gx_status st = build_query(&queries[i].plan, &qs[i], &tr, &ci);
        if (st) return st;
        if (queries[i].plan.agg == GX_AGG_BUILD)
            return set_error(GX_ERR_INVALID, "query %u: BUILD plans run through gx_scan, not in a batch", i);
        if (c0 && (ci->n_rows != c0->n_rows || ci->rows_per_chunk != c0->rows_per_chunk ||
                   ci->rows_per_block != c0->rows_per_block))
            return set_error(GX_ERR_INVALID, "query %u scans a table with another layout", i);
        c0 = c0 ? c0 : ci;
        tile_rows = std::min(tile_rows, tr);
        aux = aux || qs[i].need_aux;
        groups = groups || qs[i].grouped;
        if (qs[i].grouped) max_table = std::max<uint64_t>(max_table, 1ull << qs[i].g_log2);
        const uint64_t lo = queries[i].row_lo, hi = std::min<uint64_t>(queries[i].row_hi, c0->n_rows);
        if (lo > hi) return set_error(GX_ERR_INVALID, "query %u has row_lo > row_hi", i);
        qs[i].row_lo = lo;
        qs[i].row_hi = hi;
        if (lo < hi)
            for (uint64_t c = lo / c0->rows_per_chunk; c <= (hi - 1) / c0->rows_per_chunk; ++c) {
                cq.push_back(i);
                cc.push_back((uint32_t)c);
            }
    }
    gx_status st = ensure_kernel_attrs();
    if (st) return st;
    const uint32_t nc = (uint32_t)std::max<size_t>(1, cq.size());
    // grow buffers when needed (the stream's earlier work is finished first)
    if (n_queries > b->cap_q || nc > b->cap_cand) {
        GX_CK(cudaStreamSynchronize(s));
        const uint32_t cq_new = std::max(n_queries, b->cap_q), cc_new = std::max(nc, b->cap_cand);
        cudaFree(b->d_qs);
        cudaFree(b->d_buf);
        cudaFreeHost(b->h_qs);
        cudaFreeHost(b->h_cand);
        b->d_qs = nullptr;
        b->d_buf = nullptr;
        b->h_qs = nullptr;
        b->h_cand = nullptr;
        cudaError_t e = cudaMalloc(&b->d_qs, sizeof(QueryDesc) * cq_new);
        if (e == cudaSuccess) e = cudaMalloc(&b->d_buf, 4ull * (4ull * cc_new + 4));
        if (e == cudaSuccess) e = cudaMallocHost(&b->h_qs, sizeof(QueryDesc) * cq_new);
        if (e == cudaSuccess) e = cudaMallocHost(&b->h_cand, 8ull * cc_new);
        if (e != cudaSuccess) {
            b->cap_q = b->cap_cand = 0;
            return set_error(GX_ERR_NOMEM, "gx_batch_assign: %s", cudaGetErrorString(e));
        }
        b->cap_q = cq_new;
        b->cap_cand = cc_new;
    } else {
        // the pinned staging may still feed an earlier copy on this stream
        GX_CK(cudaStreamSynchronize(s));
    }
    if (b->exec) {
        cudaGraphExecDestroy(b->exec);
        b->exec = nullptr;
    }
    if (b->graph) {
        cudaGraphDestroy(b->graph);
        b->graph = nullptr;
    }
    const uint32_t cap = b->cap_cand;
    std::memcpy(b->h_qs, qs.data(), sizeof(QueryDesc) * n_queries);
    std::memcpy(b->h_cand, cq.data(), 4 * cq.size());
    std::memcpy(b->h_cand + cap, cc.data(), 4 * cc.size());
    GX_CK(cudaMemcpyAsync(b->d_qs, b->h_qs, sizeof(QueryDesc) * n_queries, cudaMemcpyHostToDevice, s));
    if (!cq.empty()) {
        GX_CK(cudaMemcpyAsync(b->d_buf, b->h_cand, 4 * cq.size(), cudaMemcpyHostToDevice, s));
        GX_CK(cudaMemcpyAsync(b->d_buf + cap, b->h_cand + cap, 4 * cc.size(), cudaMemcpyHostToDevice, s));
    }
    b->n = n_queries;
    b->n_cand = (uint32_t)cq.size();
    ScanParams& P = b->P;
    std::memset(&P, 0, sizeof(P));
    P.qs = b->d_qs;
    P.item_q = b->d_buf + 2 * cap;
    P.items = b->d_buf + 3 * cap;
    P.n_items = b->d_buf + 4 * cap;
    P.work_counter = b->d_buf + 4 * cap + 1;
    P.rows_scanned = b->d_rows;
    P.blocks_per_chunk = c0->blocks_per_chunk;
    P.rows_per_chunk = c0->rows_per_chunk;
    P.rows_per_block = c0->rows_per_block;
    P.tile_rows = tile_rows;
    P.tiles_per_block = (c0->rows_per_block + tile_rows - 1) / tile_rows;
    P.smem_aux = aux;
    P.smem_groups = groups;
    const uint64_t tiles = (uint64_t)nc * c0->blocks_per_chunk * P.tiles_per_block;
    scan_geometry<true>(tile_rows, aux, groups, tiles, &b->grid, &b->threads, &b->smem);
    b->reset_x = (uint32_t)std::min<uint64_t>(64, std::max<uint64_t>(1, max_table / 4096));
    b->mode = GX_BATCH_QUEUE;
    if (b->mode_pref != GX_BATCH_QUEUE) {
        bool ok = false;
        std::string why;
        st = shared_prepare(b, queries, n_queries, qs, c0, s, &ok, &why);
        if (st) return st;
        if (ok) b->mode = GX_BATCH_SHARED;
        else if (b->mode_pref == GX_BATCH_SHARED)
            return set_error(GX_ERR_INVALID, "batch cannot run in the shared form: %s", why.c_str());
    }
    if (b->mode == GX_BATCH_QUEUE)
        for (uint32_t i = 0; i < n_queries; ++i)
            if (qs[i].carry_digits)
                return set_error(GX_ERR_INVALID, "query %u carries a value and group-key digits: the queue form "
                                                 "keeps one of them per row",
                                 i);
    return GX_OK;
}

gx_status gx_batch_create(const gx_query* queries, uint32_t n_queries, gx_batch** out) {
    return gx_batch_create2(queries, n_queries, GX_BATCH_AUTO, out);
}

gx_status gx_batch_set_launch(gx_batch* b, uint32_t threads, uint32_t ctas_per_sm) {
    if (!b || (threads != 0 && threads != 128 && threads != 256 && threads != 512 && threads != 1024))
        return set_error(GX_ERR_INVALID, "gx_batch_set_launch: threads must be 0 (automatic), 128, 256, 512 or 1024");
    b->sh_threads_req = threads;
    b->sh_ctas_per_sm = ctas_per_sm;
    if (b->exec) {
        cudaGraphExecDestroy(b->exec);
        b->exec = nullptr;
    }
    if (b->graph) {
        cudaGraphDestroy(b->graph);
        b->graph = nullptr;
    }
    if (b->mode == GX_BATCH_SHARED) shared_geometry(b);
    return GX_OK;
}

gx_status gx_batch_launch_get(const gx_batch* b, uint32_t* threads) {
    if (!b || !threads) return set_error(GX_ERR_INVALID, "gx_batch_launch_get: bad args");
    *threads = b->mode == GX_BATCH_SHARED ? b->sh_threads : 0u;
    return GX_OK;
}

gx_status gx_batch_mode(const gx_batch* b, uint32_t* mode) {
    if (!b || !mode) return set_error(GX_ERR_INVALID, "gx_batch_mode: bad args");
    *mode = b->mode;
    return GX_OK;
}

gx_status gx_batch_create2(const gx_query* queries, uint32_t n_queries, uint32_t mode, gx_batch** out) {
    if (!queries || !out || n_queries == 0 || mode > GX_BATCH_SHARED)
        return set_error(GX_ERR_INVALID, "gx_batch_create: bad args");
    gx_batch* b = new gx_batch();
    b->mode_pref = mode;
    cudaGetDevice(&b->device);
    if (cudaMalloc(&b->d_rows, 8) != cudaSuccess) {
        delete b;
        return set_error(GX_ERR_NOMEM, "gx_batch_create: out of device memory");
    }
    gx_status st = gx_batch_assign(b, queries, n_queries, nullptr);
    if (st == GX_OK && cudaStreamSynchronize(nullptr) != cudaSuccess) st = set_error(GX_ERR_CUDA, "gx_batch_create: copy failed");
    if (st) {
        gx_batch_free(b);
        return st;
    }
    *out = b;
    return GX_OK;
}

gx_status gx_batch_free(gx_batch* b) {
    if (!b) return GX_OK;
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    cudaFree(b->d_qs);
    cudaFree(b->d_buf);
    cudaFree(b->d_rows);
    cudaFreeHost(b->h_qs);
    cudaFreeHost(b->h_cand);
    cudaFree(b->d_sq);
    cudaFreeHost(b->h_sq);
    cudaFree(b->d_cols);
    cudaFreeHost(b->h_cols);
    cudaFree(b->d_slot_mask);
    cudaFree(b->d_sh_items);
    cudaFree(b->d_qc);
    cudaFreeHost(b->h_qc);
    delete b;
    return GX_OK;
}

gx_status gx_batch_run(gx_batch* b, void* stream) {
    if (!b) return set_error(GX_ERR_INVALID, "null batch");
    cudaStream_t s = (cudaStream_t)stream;
    const size_t nc = b->cap_cand;
    batch_reset_kernel<<<dim3(b->reset_x, b->n), 256, 0, s>>>(b->d_qs, b->d_rows);
    if (b->mode == GX_BATCH_SHARED) {
        GX_CK(cudaMemsetAsync(b->d_sh_items, 0, 8, s));
        shared_items_kernel<<<b->sh_items_grid, 256, 0, s>>>(b->SP, b->d_slot_mask, b->d_sh_items + 2,
                                                               b->d_sh_items);
        launch_shared_kernel(b, s);
        GX_CK(cudaGetLastError());
        return GX_OK;
    }
    batch_items_kernel<<<1, 1024, 0, s>>>(b->d_qs, b->d_buf, b->d_buf + nc, b->n_cand, b->d_buf + 2 * nc,
                                          b->d_buf + 3 * nc, b->d_buf + 4 * nc, b->d_buf + 4 * nc + 1);
    launch_scan_kernel<true>(b->P, b->grid, b->threads, b->smem, s);
    GX_CK(cudaGetLastError());
    return GX_OK;
}

gx_status gx_batch_graph(gx_batch* b, void* stream) {
    if (!b) return set_error(GX_ERR_INVALID, "null batch");
    cudaStream_t s = (cudaStream_t)stream;
    if (!b->exec) {
        cudaStream_t cap;
        GX_CK(cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking));
        cudaError_t e = cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal);
        if (e == cudaSuccess) {
            gx_status st = gx_batch_run(b, cap);
            e = cudaStreamEndCapture(cap, &b->graph);
            if (st) {
                cudaStreamDestroy(cap);
                return st;
            }
        }
        if (e == cudaSuccess) e = cudaGraphInstantiate(&b->exec, b->graph, 0);
        cudaStreamDestroy(cap);
        if (e != cudaSuccess) return set_error(GX_ERR_CUDA, "batch graph capture: %s", cudaGetErrorString(e));
    }
    GX_CK(cudaGraphLaunch(b->exec, s));
    return GX_OK;
}

gx_status gx_batch_rows(gx_batch* b, uint64_t* rows, void* stream) {
    if (!b || !rows) return set_error(GX_ERR_INVALID, "gx_batch_rows: bad args");
    unsigned long long r = 0;
    GX_CK(cudaMemcpyAsync(&r, b->d_rows, 8, cudaMemcpyDeviceToHost, (cudaStream_t)stream));
    gx_status st = wait_stream((cudaStream_t)stream, 300.0);
    *rows = r;
    return st;
}

}  // extern "C"
