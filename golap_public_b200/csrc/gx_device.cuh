// gx_device.cuh -- sm_100a device building blocks: block decoders (segmented
// LZ4, generic LZ4, cascaded, raw), join-table probing and group-table
// updates.  Included by kernels.cu only.
//
// Reference counterparts: the nvCOMP decompressors behind
// ChunkDecompressor::step (core/comp.cuh:186), HashMap::probe
// (core/dev_structs.cuh:105-113) and HashAggregate::add
// (core/dev_structs.cuh:210-244).  Unlike HashAggregate::add, no wait here
// is unbounded: every probe loop is capped by the table size.
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

// 32-bit load from an arbitrary byte address in global memory (two aligned
// loads + funnel shift).  The payload carries >= 16 bytes of slack so the
// second word is always inside the allocation.
__device__ __forceinline__ uint32_t ldu32(const uint8_t* p) {
    uintptr_t a = (uintptr_t)p;
    const uint32_t* w = (const uint32_t*)(a & ~(uintptr_t)3);
    uint32_t lo = __ldg(w), hi = __ldg(w + 1);
    return __funnelshift_r(lo, hi, (uint32_t)(a & 3) * 8);
}

// Byte sources for the decoders: global memory (read-only path) or a block
// staged in shared memory.  w(i) reads 4 bytes at an arbitrary offset i.
struct GlobalSrc {
    const uint8_t* p;
    __device__ __forceinline__ uint32_t b(uint32_t i) const { return ldb(p + i); }
    __device__ __forceinline__ uint32_t w(uint32_t i) const { return ldu32(p + i); }
};
struct SharedSrc {
    const uint8_t* p;  // 16-byte aligned, >= 4 readable bytes past the stream end
    __device__ __forceinline__ uint32_t b(uint32_t i) const { return p[i]; }
    __device__ __forceinline__ uint32_t w(uint32_t i) const {
        const uint32_t* a = (const uint32_t*)(p + (i & ~3u));
        return __funnelshift_r(a[0], a[1], (i & 3u) * 8);
    }
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

// Bounded wait for the phase to complete (never spins forever).
constexpr uint32_t kMbarWaitCap = 1u << 22;
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* m, uint32_t phase) {
    for (uint32_t i = 0; i < kMbarWaitCap; ++i)
        if (mbar_try_wait(m, phase)) return true;
    return false;
}

// ------------------------------------------------- segmented LZ4, one lane
// Decodes output bytes [ob, oe) of a segmented LZ4 block (format in
// gx_internal.h) into `out` (word array whose element 0 is output byte ob).
// Returns 0 or kErrCorrupt.
template <class Src>
__device__ __forceinline__ int lz4_seg_lane(const Src in, uint32_t in_size, uint32_t comp_pos, uint32_t info,
                                            uint32_t ob, uint32_t oe, uint32_t* __restrict__ out) {
    if (comp_pos > in_size) return kErrCorrupt;
    uint32_t pos = comp_pos;
    uint32_t k = 0;
    const uint32_t K = (oe - ob) >> 2;
    uint32_t lit = 0, mnib = 0;
    bool resume = (info & 16u) != 0;
    if (resume) {
        lit = info >> 5;
        mnib = info & 15u;
    }
    while (k < K) {
        if (!resume) {
            if (pos >= in_size) return kErrCorrupt;
            uint32_t tok = in.b(pos++);
            lit = tok >> 4;
            mnib = tok & 15u;
            if (lit == 15) {
                uint32_t b;
                do {
                    if (pos >= in_size) return kErrCorrupt;
                    b = in.b(pos++);
                    lit += b;
                } while (b == 255);
            }
        }
        resume = false;
        if (lit & 3u) return kErrCorrupt;
        const uint32_t litw = lit >> 2;
        const uint32_t n = min(litw, K - k);
        if ((uint64_t)pos + (uint64_t)n * 4 > (uint64_t)in_size) return kErrCorrupt;
        {
            uint32_t i = 0;
            for (; i + 4 <= n; i += 4) {
                uint32_t a0 = in.w(pos + 4 * i), a1 = in.w(pos + 4 * i + 4);
                uint32_t a2 = in.w(pos + 4 * i + 8), a3 = in.w(pos + 4 * i + 12);
                out[k + i] = a0;
                out[k + i + 1] = a1;
                out[k + i + 2] = a2;
                out[k + i + 3] = a3;
            }
            for (; i < n; ++i) out[k + i] = in.w(pos + 4 * i);
        }
        k += n;
        pos += n * 4;
        if (k >= K) break;                 // segment ends inside / at the end of this literal run
        if ((uint64_t)pos + 2 > (uint64_t)in_size) return kErrCorrupt;  // block ended before the segment did
        uint32_t off = in.b(pos) | (in.b(pos + 1) << 8);
        pos += 2;
        uint32_t ml = mnib + 4;
        if (mnib == 15) {
            uint32_t b;
            do {
                if (pos >= in_size) return kErrCorrupt;
                b = in.b(pos++);
                ml += b;
            } while (b == 255);
        }
        if ((off & 3u) || (ml & 3u) || off == 0) return kErrCorrupt;
        const uint32_t offw = off >> 2, mlw = ml >> 2;
        if (offw > k || mlw > K - k) return kErrCorrupt;
        uint32_t* dst = out + k;
        const uint32_t* s = out + (k - offw);
        if (offw >= mlw) {
            uint32_t i = 0;
            for (; i + 4 <= mlw; i += 4) {
                uint32_t a0 = s[i], a1 = s[i + 1], a2 = s[i + 2], a3 = s[i + 3];
                dst[i] = a0;
                dst[i + 1] = a1;
                dst[i + 2] = a2;
                dst[i + 3] = a3;
            }
            for (; i < mlw; ++i) dst[i] = s[i];
        } else {
            // overlapping match: output word i repeats source word i mod offw,
            // and all source words precede k, so the copies are independent
            uint32_t j = 0;
            for (uint32_t i = 0; i < mlw; ++i) {
                dst[i] = s[j];
                if (++j == offw) j = 0;
            }
        }
        k += mlw;
    }
    return 0;
}

// ------------------------------------------------ generic LZ4, one warp
// Decodes a complete LZ4 block (any conforming encoder, byte granular) into
// `out` (out_size bytes expected).  All 32 lanes call it; every lane sees the
// same control flow.  Returns 0 or kErrCorrupt (uniform across the warp).
template <class Src>
__device__ __forceinline__ int lz4_warp_block(const Src in, uint32_t in_size, uint8_t* __restrict__ out,
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
// Inclusive scan (wrapping uint32 addition) of a[0..n) in shared memory by
// NT threads; each thread owns a contiguous range.  `tmp` has >= NT/32 + 1
// words.  Must be called by all NT threads.
template <int NT>
__device__ __forceinline__ void block_inclusive_scan(uint32_t* a, uint32_t n, uint32_t* tmp) {
    const uint32_t tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
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
    __syncthreads();
    if (warp == 0) {
        uint32_t w = lane < NT / 32 ? tmp[lane] : 0;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            uint32_t y = __shfl_up_sync(0xFFFFFFFFu, w, d);
            if (lane >= (uint32_t)d) w += y;
        }
        if (lane < NT / 32) tmp[lane] = w;
    }
    __syncthreads();
    uint32_t run = (x - s) + (warp ? tmp[warp - 1] : 0);
    for (uint32_t i = b; i < e; ++i) {
        run += a[i];
        a[i] = run;
    }
    __syncthreads();
}

// ------------------------------------------------------- cascaded block
// Decodes one cascaded block (format in gx_internal.h) into out[0..rows)
// (shared memory).  run_val/run_start are shared scratch of kCascMaxRuns
// (+1) entries.  All NT threads call it.  Returns 0 or kErrCorrupt (uniform).
template <int NT>
__device__ __forceinline__ int casc_decode_block(const uint8_t* __restrict__ blk, uint32_t blk_bytes,
                                                 uint32_t rows, int32_t* out, int32_t* run_val,
                                                 uint32_t* run_start, uint32_t* tmp) {
    const uint32_t tid = threadIdx.x;
    casc_hdr h;
    {
        const uint32_t* hw = (const uint32_t*)blk;
        uint32_t w[8];
#pragma unroll
        for (int i = 0; i < 8; ++i) w[i] = __ldg(hw + i);
        memcpy(&h, w, sizeof(h));
    }
    const bool rle = (h.flags & CASC_RLE) != 0, delta = (h.flags & CASC_DELTA) != 0;
    if (blk_bytes < 32 || h.n_rows != rows || h.val_bits > 32 || h.len_bits > 32 ||
        (rle ? (h.n_runs == 0 || h.n_runs > kCascMaxRuns) : h.n_runs != rows) ||
        h.vals_off < 32 || (h.vals_off & 3) ||
        (uint64_t)h.vals_off + 4ull * (((uint64_t)h.n_runs * h.val_bits + 31) / 32 + 1) > blk_bytes ||
        (rle && ((h.lens_off & 3) || h.lens_off < 32 ||
                 (uint64_t)h.lens_off + 4ull * (((uint64_t)h.n_runs * h.len_bits + 31) / 32 + 1) > blk_bytes)))
        return kErrCorrupt;
    const uint32_t* vw = (const uint32_t*)(blk + h.vals_off);
    uint32_t* dst = rle ? (uint32_t*)run_val : (uint32_t*)out;
    const uint32_t n = h.n_runs;
    for (uint32_t i = tid; i < n; i += NT) dst[i] = unpack_bits(vw, i, h.val_bits) + (uint32_t)h.val_base;
    __syncthreads();
    if (delta) {
        block_inclusive_scan<NT>(dst, n, tmp);
        for (uint32_t i = tid; i < n; i += NT) dst[i] += (uint32_t)h.first;
        __syncthreads();
    }
    if (!rle) return 0;
    const uint32_t* lw = (const uint32_t*)(blk + h.lens_off);
    for (uint32_t i = tid; i < n; i += NT) run_start[i + 1] = unpack_bits(lw, i, h.len_bits) + h.len_base;
    if (tid == 0) run_start[0] = 0;
    __syncthreads();
    block_inclusive_scan<NT>(run_start + 1, n, tmp);
    if (run_start[n] != rows) return kErrCorrupt;  // uniform: all threads read the same word
    // fill: each thread owns a contiguous row range; binary search its first run
    const uint32_t per = (rows + NT - 1) / NT;
    const uint32_t r0 = min(rows, tid * per), r1 = min(rows, r0 + per);
    if (r0 < r1) {
        uint32_t lo = 0, hi = n;  // find last run with start <= r0
        while (hi - lo > 1) {
            uint32_t mid = (lo + hi) >> 1;
            if (run_start[mid] <= r0) lo = mid; else hi = mid;
        }
        uint32_t run = lo, end = run_start[run + 1];
        int32_t v = run_val[run];
        for (uint32_t r = r0; r < r1; ++r) {
            while (r >= end) {
                ++run;
                end = run_start[run + 1];
                v = run_val[run];
            }
            out[r] = v;
        }
    }
    __syncthreads();
    return 0;
}

// --------------------------------------------------------- join tables
__device__ __forceinline__ bool ht_probe(const uint64_t* __restrict__ slots, uint32_t log2cap,
                                         int32_t key, int32_t* payload) {
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

// --------------------------------------------------------- group tables
// Global open-addressing group table: keys int64 (kEmptyGroup = free), sums int64.
__device__ __forceinline__ bool group_add_global(int64_t* keys, int64_t* sums, uint32_t log2cap,
                                                 int64_t key, int64_t v) {
    const uint32_t mask = (1u << log2cap) - 1;
    uint32_t s = hash_key64(key, log2cap);
    for (uint32_t i = 0; i <= mask; ++i) {
        unsigned long long old = atomicCAS((unsigned long long*)&keys[s], (unsigned long long)kEmptyGroup,
                                           (unsigned long long)key);
        if (old == (unsigned long long)kEmptyGroup || old == (unsigned long long)key) {
            atomicAdd((unsigned long long*)&sums[s], (unsigned long long)v);
            return true;
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

// Sum of a 64-bit value over the lanes in `peers` (all 32 lanes call it,
// non-members contribute 0).  Exact: four 16-bit limbs reduced separately.
__device__ __forceinline__ uint64_t warp_sum_u64(uint64_t u) {
    uint32_t p0 = __reduce_add_sync(0xFFFFFFFFu, (uint32_t)(u & 0xFFFF));
    uint32_t p1 = __reduce_add_sync(0xFFFFFFFFu, (uint32_t)((u >> 16) & 0xFFFF));
    uint32_t p2 = __reduce_add_sync(0xFFFFFFFFu, (uint32_t)((u >> 32) & 0xFFFF));
    uint32_t p3 = __reduce_add_sync(0xFFFFFFFFu, (uint32_t)(u >> 48));
    return (uint64_t)p0 + ((uint64_t)p1 << 16) + ((uint64_t)p2 << 32) + ((uint64_t)p3 << 48);
}

}  // namespace gx
