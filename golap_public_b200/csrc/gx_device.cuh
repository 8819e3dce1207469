// gx_device.cuh -- sm_100a device building blocks: block decoders (segmented
// LZ4, generic LZ4, cascaded), TMA bulk staging, join-table probing and
// group-table updates.  Included by kernels.cu only.
//
// Reference counterparts: the nvCOMP decompressors behind
// ChunkDecompressor::step (core/comp.cuh:186), HashMap::probe
// (core/dev_structs.cuh:105-113) and HashAggregate::add
// (core/dev_structs.cuh:210-244).  Unlike HashAggregate::add, no wait here
// is unbounded: every probe loop is capped by the table size and every
// mbarrier wait by an iteration count.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "gx_internal.h"

namespace gx {

constexpr int kErrCorrupt = 2;   // == GX_ERR_CORRUPT
constexpr int kErrCapacity = 3;  // == GX_ERR_CAPACITY
constexpr int kErrTimeout = 4;   // == GX_ERR_TIMEOUT
constexpr int kErrInvalid = 6;   // == GX_ERR_INVALID
constexpr uint64_t kEmptySlot = (uint64_t)(uint32_t)kEmptyKey;  // {key=INT32_MIN, payload=0}
constexpr uint32_t kEmptyGKey = 0xFFFFFFFFu;                    // shared-memory group table

// ---------------------------------------------------------- byte access
__device__ __forceinline__ uint32_t ldb(const uint8_t* p) { return (uint32_t)__ldg(p); }

// Global-memory byte source (read-only path) for the generic LZ4 decoder.
struct GlobalSrc {
    const uint8_t* p;
    __device__ __forceinline__ uint32_t b(uint32_t i) const { return ldb(p + i); }
};
// Byte source over a block staged in shared memory.
struct SharedSrc {
    const uint8_t* p;
    __device__ __forceinline__ uint32_t b(uint32_t i) const { return p[i]; }
};

// ------------------------------------------------ TMA bulk copy + mbarrier
// One-dimensional cp.async.bulk (no multicast) from global memory into this
// CTA's shared memory, completed on an mbarrier.  Source, destination and
// size must be 16-byte aligned / multiples of 16.
__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* m, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(m)), "r"(count) : "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
// Orders this thread's earlier generic-proxy accesses of shared memory
// before later async-proxy (TMA) writes to it.
__device__ __forceinline__ void fence_proxy_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ void tma_load_1d(void* dst, const void* src, uint32_t bytes, uint64_t* m) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(m)), "r"(bytes) : "memory");
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                 ::"r"(smem_u32(dst)), "l"(src), "r"(bytes), "r"(smem_u32(m))
                 : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* m, uint32_t phase) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
        : "=r"(ok)
        : "r"(smem_u32(m)), "r"(phase)
        : "memory");
    return ok != 0;
}

// try_wait that may suspend the thread until the phase completes or about
// `ns` nanoseconds pass: waiting threads sleep instead of spinning through
// issue slots while a bulk copy is in flight.
__device__ __forceinline__ bool mbar_try_wait_sleep(uint64_t* m, uint32_t phase, uint32_t ns) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n selp.u32 %0, 1, 0, p;\n}"
        : "=r"(ok)
        : "r"(smem_u32(m)), "r"(phase), "r"(ns)
        : "memory");
    return ok != 0;
}

// Bounded wait for the phase to complete (never waits forever: at most
// kMbarWaitCap tries of at most 1 us each).
constexpr uint32_t kMbarWaitCap = 1u << 21;
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* m, uint32_t phase) {
    for (uint32_t i = 0; i < kMbarWaitCap; ++i)
        if (mbar_try_wait_sleep(m, phase, 1000u)) return true;
    return false;
}

// Programmatic dependent launch: a kernel launched with programmatic stream
// serialization may start while the kernel before it on the stream still
// runs; griddep_wait blocks the calling thread until that kernel has
// completed and its writes are visible (at once when there is none), and
// griddep_launch lets the kernel that follows start early once every CTA of
// this one has issued it.
__device__ __forceinline__ void griddep_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void griddep_launch() { asm volatile("griddepcontrol.launch_dependents;" :::); }

// L2 cache policies: join tables stay (evict last), streamed bytes go first.
__device__ __forceinline__ uint64_t ws_policy_keep() {
    uint64_t p;
    asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(p));
    return p;
}
__device__ __forceinline__ uint64_t ws_policy_stream() {
    uint64_t p;
    asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p));
    return p;
}
// A join-table slot read under policy pol (read-only path).
__device__ __forceinline__ unsigned long long ws_ld_slot(const unsigned long long* a, uint64_t pol) {
    unsigned long long v;
    asm("ld.global.nc.L2::cache_hint.b64 %0, [%1], %2;" : "=l"(v) : "l"(a), "l"(pol));
    return v;
}
// ------------------------------------------------- segmented LZ4
// 4 bytes at byte offset r of a staged window (little endian, any alignment).
__device__ __forceinline__ uint32_t fetch4(const uint32_t* __restrict__ A, uint32_t r) {
    const uint32_t w = r >> 2;
    return __funnelshift_r(A[w], A[w + 1], (r & 3u) * 8);
}

// LZ4 length extension at stream position pos: adds bytes to len until one
// below 255 has been added, four bytes per step (per-byte equality with 255
// by __vcmpeq4).  Consumes no byte at or past hi (returns false then).
__device__ __forceinline__ bool lz4_len_ext(const uint32_t* __restrict__ A, uint32_t wbase, uint32_t& pos,
                                            uint32_t hi, uint32_t& len) {
    while (true) {
        if (pos >= hi) return false;
        const uint32_t x = fetch4(A, pos - wbase);
        const uint32_t ff = __vcmpeq4(x, 0xFFFFFFFFu);
        if (ff == 0xFFFFFFFFu) {
            len += 4 * 255;
            pos += 4;
            continue;
        }
        const uint32_t nfull = (uint32_t)(__ffs(~ff) - 1) >> 3;  // leading bytes equal to 255
        len += 255 * nfull + ((x >> (8 * nfull)) & 255u);
        pos += nfull + 1;
        return pos <= hi;
    }
}

// Decodes one segment of a segmented LZ4 block with a group of G lanes
// (G a power of two <= 32, the group's lanes adjacent in one warp; gmask =
// the group's lanes, gl = this lane's index in the group).  Every lane of the
// group parses the same sequence headers (broadcast shared loads), so the
// group stays converged; literal runs and matches are copied G words per
// step.  A match's words are all computed from output before the match:
// out[k + i] = out[k - offw + (i mod offw)] (LZ4 overlap semantics), so one
// __syncwarp before each match orders it after every earlier write of the
// group.  Same stream contract as the per-lane decoder: A = staged words
// from byte wbase, [lo, hi) the tile's compressed range, K output words.
// Returns 0 or kErrCorrupt (identical on every lane of the group).
__device__ __forceinline__ int lz4_seg_group(const uint32_t* __restrict__ A, uint32_t wbase, uint32_t lo,
                                             uint32_t hi, uint32_t block_end, uint32_t comp_pos, uint32_t info,
                                             uint32_t K, uint32_t* __restrict__ out, uint32_t gl, uint32_t G,
                                             uint32_t gmask) {
    if (comp_pos < lo || comp_pos > hi) return kErrCorrupt;
    uint32_t pos = comp_pos, k = 0, litw = 0, mnib = 0;
    bool tok_next = true;
    if (info & 16u) {  // the segment starts inside a sequence
        const uint32_t lit = info >> 5;
        if (lit & 3u) return kErrCorrupt;
        litw = lit >> 2;
        mnib = info & 15u;
        tok_next = false;
    }
    while (true) {
        if (tok_next) {
            if (k >= K) break;
            if (pos >= hi) return kErrCorrupt;
            const uint32_t x = fetch4(A, pos - wbase);
            uint32_t lit = (x >> 4) & 15u;
            mnib = x & 15u;
            ++pos;
            if (lit == 15 && !lz4_len_ext(A, wbase, pos, hi, lit)) return kErrCorrupt;
            if (lit & 3u) return kErrCorrupt;
            litw = lit >> 2;
        }
        const uint32_t n = min(litw, K - k);
        if ((uint64_t)pos + 4ull * n > hi) return kErrCorrupt;
        {
            const uint32_t r = pos - wbase, w = r >> 2, sh = (r & 3u) * 8;
            for (uint32_t i = gl; i < n; i += G) out[k + i] = __funnelshift_r(A[w + i], A[w + i + 1], sh);
        }
        k += n;
        pos += 4 * n;
        if (k >= K) break;  // the segment ends inside or right after the literals
        // literals done: the block may end here (then the segment is short)
        if (pos == block_end || (uint64_t)pos + 2 > hi) return kErrCorrupt;
        const uint32_t off = fetch4(A, pos - wbase) & 0xFFFFu;
        pos += 2;
        uint32_t ml = mnib + 4;
        if (mnib == 15 && !lz4_len_ext(A, wbase, pos, hi, ml)) return kErrCorrupt;
        if ((off & 3u) || (ml & 3u) || off == 0) return kErrCorrupt;
        const uint32_t offw = off >> 2, mw = ml >> 2;
        if (offw > k || mw > K - k) return kErrCorrupt;
        __syncwarp(gmask);
        const uint32_t* src = out + (k - offw);
        if (offw >= mw) {
            for (uint32_t i = gl; i < mw; i += G) out[k + i] = src[i];
        } else if (offw == 1) {
            const uint32_t v = src[0];
            for (uint32_t i = gl; i < mw; i += G) out[k + i] = v;
        } else {
            uint32_t r = gl % offw;
            const uint32_t step = G % offw;
            for (uint32_t i = gl; i < mw; i += G) {
                out[k + i] = src[r];
                r += step;
                if (r >= offw) r -= offw;
            }
        }
        k += mw;
        tok_next = true;
    }
    return 0;
}

// log2 of the lanes per segment for `nseg` segments on NT threads: the
// largest power of two G <= 32 with nseg * G <= NT (at least 1).
__device__ __forceinline__ uint32_t seg_group_log2(uint32_t nseg, uint32_t NT) {
    const uint32_t q = nseg ? NT / nseg : NT;
    return q <= 1 ? 0u : min(5u, 31u - (uint32_t)__clz(q));
}

// ------------------------------------------------ generic LZ4, one warp
// Decodes a complete LZ4 block (any conforming encoder, byte granular) into
// `out` (out_size bytes expected).  All 32 lanes call it; every lane sees the
// same control flow.  Returns 0 or kErrCorrupt (uniform across the warp).
template <class Src>
__device__ __noinline__ int lz4_warp_block(const Src in, uint32_t in_size, uint8_t* __restrict__ out,
                                           uint32_t out_size, uint32_t lane) {
    uint32_t pos = 0, o = 0;
    int err = 0;
    while (true) {
        if (pos >= in_size) { err = kErrCorrupt; break; }
        uint32_t tok = in.b(pos++);
        uint32_t lit = tok >> 4;
        if (lit == 15) {
            uint32_t b;
            do {
                if (pos >= in_size) { err = kErrCorrupt; break; }
                b = in.b(pos++);
                lit += b;
            } while (b == 255);
            if (err) break;
        }
        if ((uint64_t)pos + lit > in_size || (uint64_t)o + lit > out_size) { err = kErrCorrupt; break; }
        for (uint32_t i = lane; i < lit; i += 32) out[o + i] = (uint8_t)in.b(pos + i);
        o += lit;
        pos += lit;
        if (pos == in_size) break;  // last sequence: literals only
        if (pos + 2 > in_size) { err = kErrCorrupt; break; }
        uint32_t off = in.b(pos) | (in.b(pos + 1) << 8);
        pos += 2;
        uint32_t ml = (tok & 15u) + 4;
        if ((tok & 15u) == 15) {
            uint32_t b;
            do {
                if (pos >= in_size) { err = kErrCorrupt; break; }
                b = in.b(pos++);
                ml += b;
            } while (b == 255);
            if (err) break;
        }
        if (off == 0 || off > o || (uint64_t)o + ml > out_size) { err = kErrCorrupt; break; }
        __syncwarp();
        const uint32_t src = o - off;
        if (off >= ml) {
            for (uint32_t i = lane; i < ml; i += 32) out[o + i] = out[src + i];
        } else {
            for (uint32_t i = lane; i < ml; i += 32) out[o + i] = out[src + (i % off)];
        }
        __syncwarp();
        o += ml;
    }
    __syncwarp();
    if (!err && o != out_size) err = kErrCorrupt;
    return err;
}

// ------------------------------------------------------ block-wide scans
// Barrier of a group of NT threads: BAR == 0 is the whole CTA
// (__syncthreads), otherwise named barrier BAR of exactly NT threads (the
// consumer warps of a warp-specialised kernel).
template <int NT, int BAR>
__device__ __forceinline__ void grp_sync() {
    if constexpr (BAR == 0) {
        __syncthreads();
    } else {
        asm volatile("bar.sync %0, %1;" ::"n"(BAR), "n"(NT) : "memory");
    }
}

// Inclusive scan (wrapping uint32 addition) of a[0..n) in shared memory by
// the NT threads of a group (tid = index in the group); thread t owns the
// contiguous range [t*per, (t+1)*per).  `tmp` has >= NT/32 words.  Must be
// called by all NT threads.
template <int NT, int BAR = 0>
__device__ __forceinline__ void block_inclusive_scan(uint32_t* a, uint32_t n, uint32_t* tmp,
                                                     uint32_t tid = threadIdx.x) {
    const uint32_t lane = tid & 31, warp = tid >> 5;
    const uint32_t per = (n + NT - 1) / NT;
    const uint32_t b = min(n, tid * per), e = min(n, b + per);
    uint32_t s = 0;
    for (uint32_t i = b; i < e; ++i) s += a[i];
    uint32_t x = s;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        uint32_t y = __shfl_up_sync(0xFFFFFFFFu, x, d);
        if (lane >= (uint32_t)d) x += y;
    }
    if (lane == 31) tmp[warp] = x;
    grp_sync<NT, BAR>();
    if (warp == 0) {
        uint32_t w = lane < NT / 32 ? tmp[lane] : 0;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            uint32_t y = __shfl_up_sync(0xFFFFFFFFu, w, d);
            if (lane >= (uint32_t)d) w += y;
        }
        if (lane < NT / 32) tmp[lane] = w;
    }
    grp_sync<NT, BAR>();
    uint32_t run = (x - s) + (warp ? tmp[warp - 1] : 0);
    for (uint32_t i = b; i < e; ++i) {
        run += a[i];
        a[i] = run;
    }
    grp_sync<NT, BAR>();
}

// ------------------------------------------------------- cascaded pages
__device__ __forceinline__ bool casc_header_ok(const casc_hdr& h, uint32_t pg_bytes, uint32_t rows) {
    const bool rle = (h.flags & CASC_RLE) != 0;
    if (pg_bytes < 32 || h.n_rows != rows || h.val_bits > 32 || h.len_bits > 32) return false;
    if (rle ? (h.n_runs == 0 || h.n_runs > kCascPageMaxRuns) : h.n_runs != rows) return false;
    if (h.vals_off < 32 || (h.vals_off & 3) ||
        (uint64_t)h.vals_off + 4ull * (((uint64_t)h.n_runs * h.val_bits + 31) / 32 + 1) > pg_bytes)
        return false;
    if (rle && ((h.lens_off & 3) || h.lens_off < 32 ||
                (uint64_t)h.lens_off + 4ull * (((uint64_t)h.n_runs * h.len_bits + 31) / 32 + 1) > pg_bytes))
        return false;
    return true;
}

// Header of a page (16-byte aligned; global or shared memory).
__device__ __forceinline__ casc_hdr casc_load_header(const uint8_t* pg) {
    const uint4* hw = (const uint4*)pg;
    const uint4 a = hw[0], b = hw[1];
    casc_hdr h;
    h.n_rows = a.x;
    h.n_runs = a.y;
    h.flags = (uint8_t)(a.z & 255u);
    h.val_bits = (uint8_t)((a.z >> 8) & 255u);
    h.len_bits = (uint8_t)((a.z >> 16) & 255u);
    h.pad = (uint8_t)(a.z >> 24);
    h.first = (int32_t)a.w;
    h.val_base = (int32_t)b.x;
    h.len_base = b.y;
    h.vals_off = b.z;
    h.lens_off = b.w;
    return h;
}

// Decodes one cascaded page of `rows` rows (<= kCascPageRows; global or
// shared memory, 16-byte aligned) into out[0..rows) in shared memory, plain
// row order.  RLE pages go through run tables run_val / run_end (shared,
// kCascPageMaxRuns entries each): run values (with a delta scan), run ends
// (an inclusive scan of the lengths), then each thread expands a contiguous
// range of rows from the run that holds its first row (binary search).
// Called by the NT threads of a group (barrier BAR, tid = index in the
// group).  Returns 0 or kErrCorrupt (uniform over the group).
// With FINAL_SYNC false the values are complete only after the caller's
// next barrier of the group (callers that place one right after save one).
template <int NT, int BAR = 0, bool FINAL_SYNC = true>
__device__ __forceinline__ int casc_decode_page(const uint8_t* __restrict__ pg, uint32_t pg_bytes, uint32_t rows,
                                                int32_t* out, int32_t* run_val, uint32_t* run_end, uint32_t* tmp,
                                                uint32_t tid = threadIdx.x) {
    if (pg_bytes < 32) return kErrCorrupt;
    const casc_hdr h = casc_load_header(pg);
    if (!casc_header_ok(h, pg_bytes, rows)) return kErrCorrupt;
    const bool rle = (h.flags & CASC_RLE) != 0, delta = (h.flags & CASC_DELTA) != 0;
    const uint32_t* vw = (const uint32_t*)(pg + h.vals_off);
    if (!rle) {
        for (uint32_t i = tid; i < rows; i += NT)
            out[i] = (int32_t)((i == 0 && delta) ? 0u : unpack_bits(vw, i, h.val_bits) + (uint32_t)h.val_base);
        if (delta) {
            grp_sync<NT, BAR>();
            block_inclusive_scan<NT, BAR>((uint32_t*)out, rows, tmp, tid);
            for (uint32_t i = tid; i < rows; i += NT) out[i] = (int32_t)((uint32_t)out[i] + (uint32_t)h.first);
        }
        if (FINAL_SYNC) grp_sync<NT, BAR>();
        return 0;
    }
    const uint32_t nr = h.n_runs;
    const uint32_t* lw = (const uint32_t*)(pg + h.lens_off);
    if (nr <= 32) {
        // few runs (sorted or low-cardinality pages): one warp builds the run
        // table with shuffle scans, one barrier publishes it
        if (tid < 32) {
            const bool in = tid < nr;
            uint32_t v = in ? ((tid == 0 && delta) ? 0u : unpack_bits(vw, tid, h.val_bits) + (uint32_t)h.val_base) : 0u;
            uint32_t e = in ? unpack_bits(lw, tid, h.len_bits) + h.len_base : 0u;
#pragma unroll
            for (int d = 1; d < 32; d <<= 1) {
                const uint32_t pv = __shfl_up_sync(0xFFFFFFFFu, v, d), pe = __shfl_up_sync(0xFFFFFFFFu, e, d);
                if (tid >= (uint32_t)d) {
                    if (delta) v += pv;
                    e += pe;
                }
            }
            if (in) {
                run_val[tid] = (int32_t)(delta ? v + (uint32_t)h.first : v);
                run_end[tid] = e;
            }
        }
        grp_sync<NT, BAR>();
    } else {
        for (uint32_t i = tid; i < nr; i += NT) {
            run_val[i] = (int32_t)((i == 0 && delta) ? 0u : unpack_bits(vw, i, h.val_bits) + (uint32_t)h.val_base);
            run_end[i] = unpack_bits(lw, i, h.len_bits) + h.len_base;
        }
        grp_sync<NT, BAR>();
        if (delta) {
            block_inclusive_scan<NT, BAR>((uint32_t*)run_val, nr, tmp, tid);
            for (uint32_t i = tid; i < nr; i += NT) run_val[i] = (int32_t)((uint32_t)run_val[i] + (uint32_t)h.first);
        }
        block_inclusive_scan<NT, BAR>(run_end, nr, tmp, tid);
    }
    if (run_end[nr - 1] != rows) return kErrCorrupt;  // uniform: every thread reads the same word
    const uint32_t per = (rows + NT - 1) / NT;
    const uint32_t r_begin = min(rows, tid * per), r_stop = min(rows, r_begin + per);
    if (r_begin < r_stop) {
        uint32_t lo = 0, hi = nr - 1;  // first run ending after r_begin
        while (lo < hi) {
            const uint32_t mid = (lo + hi) >> 1;
            if (run_end[mid] <= r_begin) lo = mid + 1; else hi = mid;
        }
        uint32_t k = lo, e = run_end[k];
        int32_t v = run_val[k];
        for (uint32_t r = r_begin; r < r_stop; ++r) {
            while (r >= e && k + 1 < nr) {
                ++k;
                e = run_end[k];
                v = run_val[k];
            }
            out[r] = v;
        }
    }
    if (FINAL_SYNC) grp_sync<NT, BAR>();
    return 0;
}

// --------------------------------------------------------- join tables
__device__ __forceinline__ bool ht_probe(const uint64_t* __restrict__ slots, uint32_t log2cap, int32_t key,
                                         int32_t* payload) {
    if (key == kEmptyKey) return false;
    const uint32_t mask = (1u << log2cap) - 1;
    uint32_t s = hash_key32(key, log2cap);
    for (uint32_t i = 0; i <= mask; ++i) {
        uint64_t e = __ldg((const unsigned long long*)slots + s);
        int32_t k = (int32_t)(uint32_t)e;
        if (k == key) {
            *payload = (int32_t)(uint32_t)(e >> 32);
            return true;
        }
        if (k == kEmptyKey) return false;
        s = (s + 1) & mask;
    }
    return false;
}

// Bucketized layout: 2^log2cap slots grouped in buckets of 8 (64 bytes); a
// key hashes to a bucket, is placed in its first free slot, and spills to
// the next bucket when the bucket is full.
constexpr uint32_t kBucketSlots = 8;

__device__ __forceinline__ bool ht_probe_bucket(const uint64_t* __restrict__ slots, uint32_t log2cap, int32_t key,
                                                int32_t* payload) {
    if (key == kEmptyKey || log2cap < 3) return false;
    const uint32_t lb = log2cap - 3, bmask = (1u << lb) - 1;
    uint32_t bkt = hash_key32(key, lb);
    for (uint32_t i = 0; i <= bmask; ++i) {
        const ulonglong2* bp = (const ulonglong2*)(slots + (size_t)bkt * kBucketSlots);
        const ulonglong2 a = __ldg(bp), b = __ldg(bp + 1), c = __ldg(bp + 2), d = __ldg(bp + 3);
        const unsigned long long e[8] = {a.x, a.y, b.x, b.y, c.x, c.y, d.x, d.y};
        bool any_empty = false;
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            const int32_t k = (int32_t)(uint32_t)e[j];
            if (k == key) {
                *payload = (int32_t)(uint32_t)(e[j] >> 32);
                return true;
            }
            any_empty |= (k == kEmptyKey);
        }
        if (any_empty) return false;
        bkt = (bkt + 1) & bmask;
    }
    return false;
}

// Dense layout: slot 0 = {base, span}; the key's entry at slot 1 + (key - base).
__device__ __forceinline__ bool ht_probe_dense(const uint64_t* __restrict__ slots, int32_t key, int32_t* payload) {
    const uint64_t h = __ldg((const unsigned long long*)slots);
    const uint32_t u = (uint32_t)key - (uint32_t)h;
    if (key == kEmptyKey || u >= (uint32_t)(h >> 32)) return false;
    const uint64_t e = __ldg((const unsigned long long*)slots + 1 + u);
    if ((int32_t)(uint32_t)e != key) return false;
    *payload = (int32_t)(uint32_t)(e >> 32);
    return true;
}

__device__ __forceinline__ bool ht_probe_any(const uint64_t* __restrict__ slots, uint32_t log2cap, uint32_t layout,
                                             int32_t key, int32_t* payload) {
    if (layout == GX_HT_DENSE) return ht_probe_dense(slots, key, payload);
    return layout ? ht_probe_bucket(slots, log2cap, key, payload) : ht_probe(slots, log2cap, key, payload);
}

// --------------------------------------------------------- group tables
// Global open-addressing group table: keys int64 (kEmptyGroup = free), sums int64.
__device__ __forceinline__ bool group_add_global(int64_t* keys, int64_t* sums, uint32_t log2cap, int64_t key,
                                                 int64_t v) {
    const uint32_t mask = (1u << log2cap) - 1;
    uint32_t s = hash_key64(key, log2cap);
    for (uint32_t i = 0; i <= mask; ++i) {
        // A slot's key is written once (free -> key) and never changes, so a plain
        // (possibly cached, possibly stale) read that shows a key is final: the
        // common case -- the key already there -- costs a read and a fire-and-forget
        // add, and only a slot that reads free takes the compare-and-swap.
        long long cur;
        asm volatile("ld.global.ca.b64 %0, [%1];" : "=l"(cur) : "l"(keys + s));
        if (cur == (long long)key) {
            atomicAdd((unsigned long long*)&sums[s], (unsigned long long)v);
            return true;
        }
        if (cur == (long long)kEmptyGroup) {
            const unsigned long long old = atomicCAS((unsigned long long*)&keys[s], (unsigned long long)kEmptyGroup,
                                                     (unsigned long long)key);
            if (old == (unsigned long long)kEmptyGroup || old == (unsigned long long)key) {
                atomicAdd((unsigned long long*)&sums[s], (unsigned long long)v);
                return true;
            }
        }
        s = (s + 1) & mask;
    }
    return false;
}

// Shared-memory partial group table (uint32 keys).  Returns false when full.
__device__ __forceinline__ bool group_add_smem(uint32_t* keys, unsigned long long* sums, uint32_t log2cap,
                                               uint32_t key, uint64_t v) {
    const uint32_t mask = (1u << log2cap) - 1;
    uint32_t s = hash_key32((int32_t)key, log2cap);
    for (uint32_t i = 0; i <= mask; ++i) {
        uint32_t old = atomicCAS(&keys[s], kEmptyGKey, key);
        if (old == kEmptyGKey || old == key) {
            atomicAdd(&sums[s], (unsigned long long)v);
            return true;
        }
        s = (s + 1) & mask;
    }
    return false;
}

// Sum of a 64-bit value over all 32 lanes (non-members pass 0).  Exact:
// four 16-bit limbs are reduced separately and recombined modulo 2^64.
__device__ __forceinline__ uint64_t warp_sum_u64(uint64_t u) {
    uint32_t p0 = __reduce_add_sync(0xFFFFFFFFu, (uint32_t)(u & 0xFFFF));
    uint32_t p1 = __reduce_add_sync(0xFFFFFFFFu, (uint32_t)((u >> 16) & 0xFFFF));
    uint32_t p2 = __reduce_add_sync(0xFFFFFFFFu, (uint32_t)((u >> 32) & 0xFFFF));
    uint32_t p3 = __reduce_add_sync(0xFFFFFFFFu, (uint32_t)(u >> 48));
    return (uint64_t)p0 + ((uint64_t)p1 << 16) + ((uint64_t)p2 << 32) + ((uint64_t)p3 << 48);
}

}  // namespace gx
