// encode_gpu.cu -- column ingest on the GPU: values already in HBM encoded
// into the column format of gx_internal.h, with the per-chunk min/max and
// the per-block zone maps, in two passes (plan, then write).
//
// Replaces prepare_compressed's per-chunk compress + MinMaxMeta::init_chunk
// (core/apps.cuh:149-255, core/metadata.cuh:157-160) for columns whose
// values are already on the device.  The bytes equal those of the host
// encoder (encode.cpp) for the codecs built here: raw blocks, cascaded
// pages (the same choice among {plain, delta} x {no RLE, RLE} with the same
// tie order), and LZ4 blocks that are one literal run each (the host
// encoder's no-match candidate, lz4_min_match = GX_LZ4_LITERAL).
//
// Pass 1 (genc_plan_kernel, one CTA per block and cascaded page): zone maps
// by atomic min/max; for a cascaded page, the sizes of the four candidate
// encodings (run starts by comparing neighbours, run lengths from a block
// scan of the start flags) and the chosen one's parameters.  The host then
// lays the payload out (one small device-to-host copy of the plans: block
// sizes, page offsets, LZ4 alignment pads, one scan) exactly as the host
// encoder's concatenation does.  Pass 2 (genc_write_kernel) writes every
// block at its offset: raw rows, the LZ4 token + length extension + the
// literal bytes, or the cascaded block header and pages (bit-packed streams
// by atomic OR into the zeroed payload).
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <cstring>
#include <mutex>
#include <vector>

#include "../../include/gx.h"
#include "gx_device.cuh"
#include "gx_internal.h"

using namespace gx;

namespace {

constexpr uint32_t kGencNT = 256;

// The chosen encoding of one cascaded page (pass 1 -> host -> pass 2).
struct PagePlan {
    uint32_t bytes;   // page bytes (a multiple of 16)
    uint32_t n;       // values in the value stream (rows, or runs with RLE)
    uint32_t flags;   // CASC_RLE | CASC_DELTA
    uint32_t vbits, lbits;
    int32_t vbase;    // frame of reference of the value stream
    uint32_t lbase;   // frame of reference of the run lengths
    int32_t first;    // v[0]
};
static_assert(sizeof(PagePlan) == 32, "PagePlan layout");

struct GencParams {
    const int32_t* vals;
    uint64_t n_rows;
    uint32_t codec, rows_per_chunk, rows_per_block, blocks_per_chunk, n_slots, pages;
    uint32_t rle, delta, bp;
    int32_t* bmins;
    int32_t* bmaxs;
    PagePlan* plans;        // n_slots * pages (cascaded)
    // pass 2
    uint8_t* payload;
    const uint64_t* offset; // n_slots: where the block's stream starts
    const uint32_t* page_off;  // n_slots * (pages + 1): page offsets in the block (cascaded)
};

__device__ __forceinline__ uint32_t genc_block_rows(const GencParams& P, uint32_t s, uint64_t* r0) {
    const uint32_t c = s / P.blocks_per_chunk, j = s % P.blocks_per_chunk;
    const uint64_t c0 = (uint64_t)c * P.rows_per_chunk;
    const uint64_t c1 = min(P.n_rows, c0 + P.rows_per_chunk);
    *r0 = c0 + (uint64_t)j * P.rows_per_block;
    return *r0 < c1 ? (uint32_t)min((uint64_t)P.rows_per_block, c1 - *r0) : 0u;
}

__host__ __device__ __forceinline__ uint32_t genc_bits(uint64_t range) {
#ifdef __CUDA_ARCH__
    return range == 0 ? 0u : (uint32_t)(64 - __clzll((long long)range));
#else
    return range == 0 ? 0u : (uint32_t)(64 - __builtin_clzll(range));
#endif
}

__host__ __device__ __forceinline__ uint32_t genc_stream_bytes(uint64_t n, uint32_t w) {
    const uint64_t words = (n * w + 31) / 32 + 1;  // + one padding word
    return (uint32_t)((4 * words + 15) & ~15ull);
}

// Block-wide min and max of a pair of int64 values (NT threads).
__device__ __forceinline__ void genc_minmax(int64_t& mn, int64_t& mx, int64_t* red) {
    const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) {
        mn = min(mn, (int64_t)__shfl_xor_sync(0xFFFFFFFFu, (long long)mn, d));
        mx = max(mx, (int64_t)__shfl_xor_sync(0xFFFFFFFFu, (long long)mx, d));
    }
    __syncthreads();
    if (lane == 0) {
        red[2 * warp] = mn;
        red[2 * warp + 1] = mx;
    }
    __syncthreads();
    mn = red[0];
    mx = red[1];
    for (uint32_t w = 1; w < kGencNT / 32; ++w) {
        mn = min(mn, red[2 * w]);
        mx = max(mx, red[2 * w + 1]);
    }
}

// The runs of a page in shared memory: start[k] = first row of run k,
// start[nr] = rows (only when nr <= kCascPageMaxRuns).  Returns nr (or a
// value above kCascPageMaxRuns when there are more runs).
__device__ uint32_t genc_runs(const int32_t* v, uint32_t rows, uint32_t* flag, uint32_t* start, uint32_t* tmp) {
    for (uint32_t i = threadIdx.x; i < rows; i += kGencNT) flag[i] = (i == 0 || v[i] != v[i - 1]) ? 1u : 0u;
    __syncthreads();
    block_inclusive_scan<kGencNT>(flag, rows, tmp);  // ends with a barrier
    const uint32_t nr = rows ? flag[rows - 1] : 0u;
    if (nr <= kCascPageMaxRuns) {
        for (uint32_t i = threadIdx.x; i < rows; i += kGencNT) {
            const bool st = i == 0 || flag[i] != flag[i - 1];
            if (st) start[flag[i] - 1] = i;
        }
        if (threadIdx.x == 0) start[nr] = rows;
    }
    __syncthreads();
    return nr;
}

// Pass 1: zone maps (atomic min/max per block) and, for cascaded columns, the
// chosen encoding of page blockIdx.y of block blockIdx.x.
__global__ void __launch_bounds__(kGencNT) genc_plan_kernel(const GencParams P) {
    __shared__ int32_t sv[kCascPageRows];
    __shared__ uint32_t flag[kCascPageRows];
    __shared__ uint32_t start[kCascPageMaxRuns + 1];
    __shared__ uint32_t tmp[kGencNT / 32 + 1];
    __shared__ int64_t red[2 * (kGencNT / 32)];
    const uint32_t s = blockIdx.x, p = blockIdx.y, tid = threadIdx.x;
    uint64_t r0;
    const uint32_t rows = genc_block_rows(P, s, &r0);
    if (!rows) return;
    const bool casc = P.codec == GX_CODEC_CASCADED;
    const uint32_t lo = casc ? p * kCascPageRows : 0u;
    if (lo >= rows) return;
    const uint32_t hi = casc ? min(rows, lo + kCascPageRows) : rows, n = hi - lo;
    int64_t mn = INT64_MAX, mx = INT64_MIN;
    for (uint32_t i = tid; i < n; i += kGencNT) {
        const int32_t v = P.vals[r0 + lo + i];
        if (casc) sv[i] = v;
        mn = min(mn, (int64_t)v);
        mx = max(mx, (int64_t)v);
    }
    genc_minmax(mn, mx, red);  // its barriers also publish sv
    if (tid == 0) {
        atomicMin(&P.bmins[s], (int)mn);
        atomicMax(&P.bmaxs[s], (int)mx);
    }
    if (!casc) return;
    // delta entries: 0, then v[i] - v[i-1] (wrapping int32)
    int64_t dmn = INT64_MAX, dmx = INT64_MIN;
    for (uint32_t i = tid; i < n; i += kGencNT) {
        const int64_t e = i == 0 ? 0 : (int64_t)(int32_t)((uint32_t)sv[i] - (uint32_t)sv[i - 1]);
        dmn = min(dmn, e);
        dmx = max(dmx, e);
    }
    genc_minmax(dmn, dmx, red);
    // runs (at most kCascPageMaxRuns for RLE): value deltas between runs, lengths
    const uint32_t nr = P.rle ? genc_runs(sv, n, flag, start, tmp) : 0xFFFFFFFFu;
    const bool rle_ok = P.rle && nr <= kCascPageMaxRuns && n > 0;
    int64_t rmn = INT64_MAX, rmx = INT64_MIN, lmn = INT64_MAX, lmx = INT64_MIN;
    if (rle_ok) {
        for (uint32_t k = tid; k < nr; k += kGencNT) {
            const int64_t e = k == 0 ? 0 : (int64_t)(int32_t)((uint32_t)sv[start[k]] - (uint32_t)sv[start[k - 1]]);
            const int64_t len = (int64_t)(start[k + 1] - start[k]);
            rmn = min(rmn, e);
            rmx = max(rmx, e);
            lmn = min(lmn, len);
            lmx = max(lmx, len);
        }
        genc_minmax(rmn, rmx, red);
        genc_minmax(lmn, lmx, red);
    }
    if (tid != 0) return;
    // the four candidates in the host encoder's order, strict improvement only
    const bool bp = P.bp != 0;
    auto vbits = [&](int64_t a, int64_t b) { return bp ? genc_bits((uint64_t)(b - a)) : 32u; };
    PagePlan best;
    best.n = n;
    best.flags = 0;
    best.vbits = vbits(mn, mx);
    best.vbase = bp ? (int32_t)mn : 0;
    best.lbits = 0;
    best.lbase = 0;
    best.bytes = 32 + genc_stream_bytes(n, best.vbits);
    best.first = sv[0];
    if (P.delta) {
        const uint32_t vb = vbits(dmn, dmx), bytes = 32 + genc_stream_bytes(n, vb);
        if (bytes < best.bytes) {
            best.flags = CASC_DELTA;
            best.vbits = vb;
            best.vbase = bp ? (int32_t)dmn : 0;
            best.bytes = bytes;
        }
    }
    if (rle_ok) {
        const uint32_t lb = bp ? genc_bits((uint64_t)(lmx - lmn)) : 32u;
        const uint32_t lbase = bp ? (uint32_t)lmn : 0u;
        const uint32_t lbytes = genc_stream_bytes(nr, lb);
        const uint32_t vb = vbits(mn, mx), bytes = 32 + genc_stream_bytes(nr, vb) + lbytes;
        if (bytes < best.bytes) {
            best.flags = CASC_RLE;
            best.n = nr;
            best.vbits = vb;
            best.vbase = bp ? (int32_t)mn : 0;
            best.lbits = lb;
            best.lbase = lbase;
            best.bytes = bytes;
        }
        if (P.delta) {
            const uint32_t vbd = vbits(rmn, rmx), bytesd = 32 + genc_stream_bytes(nr, vbd) + lbytes;
            if (bytesd < best.bytes) {
                best.flags = CASC_RLE | CASC_DELTA;
                best.n = nr;
                best.vbits = vbd;
                best.vbase = bp ? (int32_t)rmn : 0;
                best.lbits = lb;
                best.lbase = lbase;
                best.bytes = bytesd;
            }
        }
    }
    P.plans[(size_t)s * P.pages + p] = best;
}

// Element i of width w at bit i * w of the zeroed word stream (atomic OR:
// neighbouring elements share words).
__device__ __forceinline__ void genc_pack(uint32_t* words, uint32_t i, uint32_t w, uint32_t u) {
    if (w == 0) return;
    const uint64_t bit = (uint64_t)i * w;
    const uint32_t wi = (uint32_t)(bit >> 5), sh = (uint32_t)(bit & 31);
    if (w < 32) u &= (1u << w) - 1u;
    atomicOr(&words[wi], u << sh);
    if (sh + w > 32) atomicOr(&words[wi + 1], (uint32_t)((uint64_t)u >> (32 - sh)));
}

// Pass 2: block blockIdx.x (page blockIdx.y of a cascaded block) written at
// its offset in the zeroed payload.
__global__ void __launch_bounds__(kGencNT) genc_write_kernel(const GencParams P) {
    __shared__ int32_t sv[kCascPageRows];
    __shared__ uint32_t flag[kCascPageRows];
    __shared__ uint32_t start[kCascPageMaxRuns + 1];
    __shared__ uint32_t tmp[kGencNT / 32 + 1];
    const uint32_t s = blockIdx.x, p = blockIdx.y, tid = threadIdx.x;
    uint64_t r0;
    const uint32_t rows = genc_block_rows(P, s, &r0);
    if (!rows) return;
    uint8_t* const blk = P.payload + P.offset[s];
    if (P.codec == GX_CODEC_NONE) {
        for (uint32_t i = tid; i < rows; i += kGencNT) ((int32_t*)blk)[i] = P.vals[r0 + i];
        return;
    }
    if (P.codec == GX_CODEC_LZ4) {
        // one sequence: token, literal-length extension, the rows as literal bytes
        const uint32_t Lb = 4 * rows, ext = Lb >= 15 ? (Lb - 15) / 255 + 1 : 0u, lit0 = 1 + ext;
        for (uint32_t k = tid; k < lit0; k += kGencNT) {
            uint8_t b;
            if (k == 0) b = (uint8_t)(min(Lb, 15u) << 4);
            else if (k < ext) b = 255;
            else b = (uint8_t)((Lb - 15) % 255);
            blk[k] = b;
        }
        for (uint32_t i = tid; i < rows; i += kGencNT) ((int32_t*)(blk + lit0))[i] = P.vals[r0 + i];
        return;
    }
    // cascaded: the block header (page 0's CTA), then page p
    const uint32_t n_pages = (rows + kCascPageRows - 1) / kCascPageRows;
    if (p >= n_pages) return;
    const uint32_t* po = P.page_off + (size_t)s * (P.pages + 1);
    if (p == 0)
        for (uint32_t k = tid; k < n_pages + 3; k += kGencNT)
            ((uint32_t*)blk)[k] = k == 0 ? n_pages : k == 1 ? kCascPageRows : po[k - 2];
    const PagePlan pl = P.plans[(size_t)s * P.pages + p];
    const uint32_t lo = p * kCascPageRows, n = min(rows, lo + kCascPageRows) - lo;
    for (uint32_t i = tid; i < n; i += kGencNT) sv[i] = P.vals[r0 + lo + i];
    __syncthreads();
    const bool rle = (pl.flags & CASC_RLE) != 0, delta = (pl.flags & CASC_DELTA) != 0;
    uint8_t* const pg = blk + po[p];
    const uint32_t vals_off = 32, lens_off = rle ? 32 + genc_stream_bytes(pl.n, pl.vbits) : 0u;
    if (tid == 0) {
        uint32_t* h = (uint32_t*)pg;
        h[0] = n;
        h[1] = pl.n;
        h[2] = pl.flags | (pl.vbits << 8) | ((rle ? pl.lbits : 0u) << 16);
        h[3] = (uint32_t)pl.first;
        h[4] = (uint32_t)pl.vbase;
        h[5] = rle ? pl.lbase : 0u;
        h[6] = vals_off;
        h[7] = lens_off;
    }
    uint32_t* const vw = (uint32_t*)(pg + vals_off);
    if (!rle) {
        for (uint32_t i = tid; i < n; i += kGencNT) {
            const int32_t e = delta ? (i == 0 ? 0 : (int32_t)((uint32_t)sv[i] - (uint32_t)sv[i - 1])) : sv[i];
            genc_pack(vw, i, pl.vbits, (uint32_t)e - (uint32_t)pl.vbase);
        }
        return;
    }
    const uint32_t nr = genc_runs(sv, n, flag, start, tmp);
    if (nr != pl.n) return;  // cannot happen: the same rows as in pass 1
    uint32_t* const lw = (uint32_t*)(pg + lens_off);
    for (uint32_t k = tid; k < nr; k += kGencNT) {
        const int32_t e =
            delta ? (k == 0 ? 0 : (int32_t)((uint32_t)sv[start[k]] - (uint32_t)sv[start[k - 1]])) : sv[start[k]];
        genc_pack(vw, k, pl.vbits, (uint32_t)e - (uint32_t)pl.vbase);
        genc_pack(lw, k, pl.lbits, (start[k + 1] - start[k]) - pl.lbase);
    }
}

__global__ void genc_fill_kernel(int32_t* a, int32_t* b, uint32_t n) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        a[i] = INT32_MAX;
        b[i] = INT32_MIN;
    }
}

}  // namespace

namespace gx {

int host_payload(const gx_column* col) {
    static std::mutex mu;
    std::lock_guard<std::mutex> lock(mu);
    if (!col->host_pending) return GX_OK;
    if (!col->d_payload) return set_error(GX_ERR_INVALID, "column payload is neither on the host nor on the device");
    int dev = 0;
    cudaGetDevice(&dev);
    if (col->device >= 0 && col->device != dev) cudaSetDevice(col->device);
    auto& host = const_cast<gx_column*>(col)->payload;
    host.resize(col->dev_payload_bytes);
    const cudaError_t e = cudaMemcpy(host.data(), col->d_payload, col->dev_payload_bytes, cudaMemcpyDeviceToHost);
    if (col->device >= 0 && col->device != dev) cudaSetDevice(dev);
    if (e != cudaSuccess) {
        host.clear();
        return set_error(GX_ERR_CUDA, "reading a column payload back: %s", cudaGetErrorString(e));
    }
    col->host_pending = false;
    return GX_OK;
}

}  // namespace gx

#define GENC_CK(call)                                                                       \
    do {                                                                                    \
        cudaError_t e_ = (call);                                                            \
        if (e_ != cudaSuccess) {                                                            \
            st = set_error(GX_ERR_CUDA, "%s: %s", #call, cudaGetErrorString(e_));           \
            goto done;                                                                      \
        }                                                                                   \
    } while (0)

extern "C" gx_status gx_column_encode_device(const int32_t* values_dev, uint64_t n_rows, const gx_encode_opts* opts,
                                             gx_column** out, void* stream) {
    if (!values_dev || !opts || !out) return set_error(GX_ERR_INVALID, "gx_column_encode_device: null argument");
    const uint32_t codec = opts->codec, rpc = opts->rows_per_chunk, rpb = opts->rows_per_block;
    uint32_t S = opts->lz4_segments;
    if (n_rows == 0) return set_error(GX_ERR_INVALID, "gx_column_encode_device: empty column");
    if (rpb == 0 || rpb > kMaxRowsPerBlock)
        return set_error(GX_ERR_INVALID, "rows_per_block must be in 1..%u", kMaxRowsPerBlock);
    if (rpc == 0) return set_error(GX_ERR_INVALID, "rows_per_chunk must be > 0");
    if (codec > GX_CODEC_CASCADED) return set_error(GX_ERR_INVALID, "unknown codec %u", codec);
    if (codec == GX_CODEC_LZ4) {
        if (S == 0 || S > kMaxSegments || (S & (S - 1)) != 0)
            return set_error(GX_ERR_INVALID, "lz4_segments must be a power of two in 1..%u", kMaxSegments);
        if (S > 1 && ((rpb & (rpb - 1)) != 0 || rpb < S))
            return set_error(GX_ERR_INVALID, "segmented LZ4 needs a power-of-two rows_per_block >= segments");
        if (opts->lz4_min_match != GX_LZ4_LITERAL)
            return set_error(GX_ERR_INVALID,
                             "gx_column_encode_device: LZ4 is encoded as literal runs only (lz4_min_match = "
                             "GX_LZ4_LITERAL); use gx_column_encode for match-finding policies");
    } else if (codec == GX_CODEC_CASCADED) {
        S = (rpb + kCascPageRows - 1) / kCascPageRows;
    } else {
        S = 1;
    }
    cudaStream_t s = (cudaStream_t)stream;
    gx_status st = GX_OK;
    gx_column* col = new (std::nothrow) gx_column();
    if (!col) return set_error(GX_ERR_NOMEM, "gx_column_encode_device: out of host memory");
    PagePlan* d_plans = nullptr;
    uint64_t* d_offset = nullptr;
    uint32_t* d_page_off = nullptr;
    {
        col->n_rows = n_rows;
        col->codec = codec;
        col->rows_per_chunk = rpc;
        col->rows_per_block = rpb;
        col->n_chunks = (uint32_t)((n_rows + rpc - 1) / rpc);
        col->blocks_per_chunk = (rpc + rpb - 1) / rpb;
        col->n_slots = col->n_chunks * col->blocks_per_chunk;
        col->S = S;
        col->seg_shift = 0;
        if (codec == GX_CODEC_CASCADED) {
            col->seg_shift = kCascPageLog2;
        } else if (S > 1) {
            const uint32_t sr = rpb / S;
            while ((1u << col->seg_shift) < sr) ++col->seg_shift;
        }
        const uint32_t n_slots = col->n_slots;
        const uint32_t pages = codec == GX_CODEC_CASCADED ? S : 1u;
        col->blocks.assign(n_slots, gx_dblock{0, 0, 0});
        if (S > 1 || codec == GX_CODEC_CASCADED) col->seg.assign((size_t)2 * S * n_slots, 0);
        col->mins.assign(col->n_chunks, 0);
        col->maxs.assign(col->n_chunks, 0);
        col->bmins.assign(n_slots, INT32_MAX);
        col->bmaxs.assign(n_slots, INT32_MIN);

        GencParams P{};
        P.vals = values_dev;
        P.n_rows = n_rows;
        P.codec = codec;
        P.rows_per_chunk = rpc;
        P.rows_per_block = rpb;
        P.blocks_per_chunk = col->blocks_per_chunk;
        P.n_slots = n_slots;
        P.pages = pages;
        P.rle = opts->casc_rle != 0;
        P.delta = opts->casc_delta != 0;
        P.bp = opts->casc_bitpack != 0;
        GENC_CK(cudaMalloc(&col->d_bmins, 4ull * n_slots));
        GENC_CK(cudaMalloc(&col->d_bmaxs, 4ull * n_slots));
        P.bmins = col->d_bmins;
        P.bmaxs = col->d_bmaxs;
        genc_fill_kernel<<<std::min<uint32_t>(1024, (n_slots + 255) / 256), 256, 0, s>>>(P.bmins, P.bmaxs, n_slots);
        if (codec == GX_CODEC_CASCADED) {
            GENC_CK(cudaMalloc(&d_plans, sizeof(PagePlan) * (size_t)n_slots * pages));
            P.plans = d_plans;
        }
        // pass 1: zone maps and the cascaded pages' encodings
        genc_plan_kernel<<<dim3(n_slots, pages), kGencNT, 0, s>>>(P);
        GENC_CK(cudaGetLastError());
        std::vector<PagePlan> plans(codec == GX_CODEC_CASCADED ? (size_t)n_slots * pages : 0);
        GENC_CK(cudaMemcpyAsync(col->bmins.data(), P.bmins, 4ull * n_slots, cudaMemcpyDeviceToHost, s));
        GENC_CK(cudaMemcpyAsync(col->bmaxs.data(), P.bmaxs, 4ull * n_slots, cudaMemcpyDeviceToHost, s));
        if (!plans.empty())
            GENC_CK(cudaMemcpyAsync(plans.data(), d_plans, sizeof(PagePlan) * plans.size(), cudaMemcpyDeviceToHost, s));
        GENC_CK(cudaStreamSynchronize(s));

        // the payload layout of the host encoder: blocks in slot order, each
        // starting on a 16-byte boundary (an LZ4 block padded so that its first
        // literal byte is), cascaded pages 16-byte aligned after the block header
        std::vector<uint64_t> offset(n_slots, 0);
        std::vector<uint32_t> page_off(codec == GX_CODEC_CASCADED ? (size_t)n_slots * (pages + 1) : 0, 0);
        uint64_t cursor = 0;
        for (uint32_t sl = 0; sl < n_slots; ++sl) {
            const uint32_t c = sl / col->blocks_per_chunk, j = sl % col->blocks_per_chunk;
            const uint64_t c0 = (uint64_t)c * rpc, c1 = std::min<uint64_t>(n_rows, c0 + rpc);
            const uint64_t r0 = c0 + (uint64_t)j * rpb;
            if (r0 >= c1) continue;
            const uint32_t rows = (uint32_t)std::min<uint64_t>(rpb, c1 - r0);
            uint64_t pad = 0, used = 0;
            if (codec == GX_CODEC_NONE) {
                used = 4ull * rows;
            } else if (codec == GX_CODEC_LZ4) {
                const uint32_t Lb = 4 * rows, ext = Lb >= 15 ? (Lb - 15) / 255 + 1 : 0u, lit0 = 1 + ext;
                used = (uint64_t)lit0 + Lb;
                pad = (16 - lit0 % 16) % 16;
                if (S > 1) {
                    uint32_t* e = &col->seg[(size_t)2 * S * sl];
                    const uint32_t seg_rows = rpb / S;
                    e[0] = lit0;
                    e[1] = (Lb << 5) | 16u;
                    for (uint32_t k = 1; k < S; ++k) {
                        const uint32_t N = (uint32_t)std::min<uint64_t>((uint64_t)k * seg_rows, rows);
                        if (N < rows) {
                            e[2 * k] = lit0 + 4 * N;
                            e[2 * k + 1] = (((rows - N) * 4) << 5) | 16u;
                        } else {
                            e[2 * k] = (uint32_t)used;
                            e[2 * k + 1] = 16u;
                        }
                    }
                }
            } else {
                const uint32_t n_pages = (rows + kCascPageRows - 1) / kCascPageRows;
                uint32_t* po = &page_off[(size_t)sl * (pages + 1)];
                uint32_t off = (8 + 4 * (n_pages + 1) + 15) & ~15u;
                for (uint32_t p = 0; p < n_pages; ++p) {
                    const uint32_t b = plans[(size_t)sl * pages + p].bytes;
                    po[p] = off;
                    col->seg[(size_t)2 * S * sl + 2 * p] = off;
                    col->seg[(size_t)2 * S * sl + 2 * p + 1] = b;
                    off += b;
                }
                po[n_pages] = off;
                used = off;
            }
            offset[sl] = cursor + pad;
            col->blocks[sl] = gx_dblock{cursor + pad, (uint32_t)used, rows};
            cursor += (pad + used + kPayloadAlign - 1) & ~(uint64_t)(kPayloadAlign - 1);
        }
        for (uint32_t c = 0; c < col->n_chunks; ++c) {
            int32_t mn = INT32_MAX, mx = INT32_MIN;
            for (uint32_t j = 0; j < col->blocks_per_chunk; ++j) {
                mn = std::min(mn, col->bmins[(size_t)c * col->blocks_per_chunk + j]);
                mx = std::max(mx, col->bmaxs[(size_t)c * col->blocks_per_chunk + j]);
            }
            col->mins[c] = mn;
            col->maxs[c] = mx;
        }
        col->n_blocks = 0;
        for (auto& b : col->blocks) col->n_blocks += b.n_rows ? 1 : 0;

        // pass 2: the bytes, into a zeroed payload with the host encoder's slack
        const uint64_t total = cursor + kPayloadSlack;
        GENC_CK(cudaMalloc(&col->d_payload, total));
        col->residency = 1;  // owns d_payload from here on
        GENC_CK(cudaMemsetAsync(col->d_payload, 0, total, s));
        GENC_CK(cudaMalloc(&d_offset, 8ull * n_slots));
        GENC_CK(cudaMemcpyAsync(d_offset, offset.data(), 8ull * n_slots, cudaMemcpyHostToDevice, s));
        if (!page_off.empty()) {
            GENC_CK(cudaMalloc(&d_page_off, 4 * page_off.size()));
            GENC_CK(cudaMemcpyAsync(d_page_off, page_off.data(), 4 * page_off.size(), cudaMemcpyHostToDevice, s));
        }
        P.payload = (uint8_t*)col->d_payload;
        P.offset = d_offset;
        P.page_off = d_page_off;
        genc_write_kernel<<<dim3(n_slots, pages), kGencNT, 0, s>>>(P);
        GENC_CK(cudaGetLastError());

        // the device metadata, and the host copy of the payload
        GENC_CK(cudaMalloc(&col->d_blocks, sizeof(gx_dblock) * n_slots));
        GENC_CK(cudaMemcpyAsync(col->d_blocks, col->blocks.data(), sizeof(gx_dblock) * n_slots, cudaMemcpyHostToDevice,
                                s));
        if (!col->seg.empty()) {
            GENC_CK(cudaMalloc(&col->d_seg, 4 * col->seg.size()));
            GENC_CK(cudaMemcpyAsync(col->d_seg, col->seg.data(), 4 * col->seg.size(), cudaMemcpyHostToDevice, s));
        }
        GENC_CK(cudaMalloc(&col->d_mins, 4ull * col->n_chunks));
        GENC_CK(cudaMalloc(&col->d_maxs, 4ull * col->n_chunks));
        GENC_CK(cudaMemcpyAsync(col->d_mins, col->mins.data(), 4ull * col->n_chunks, cudaMemcpyHostToDevice, s));
        GENC_CK(cudaMemcpyAsync(col->d_maxs, col->maxs.data(), 4ull * col->n_chunks, cudaMemcpyHostToDevice, s));
        GENC_CK(cudaStreamSynchronize(s));
        // the host copy of the payload is read back on first use (host_payload)
        col->dev_payload_bytes = total;
        col->host_pending = true;
        cudaGetDevice(&col->device);
        if (codec == GX_CODEC_LZ4) col->lz4_direct = 1;  // every block one literal run, placed aligned
    }
done:
    if (d_plans) cudaFree(d_plans);
    if (d_offset) cudaFree(d_offset);
    if (d_page_off) cudaFree(d_page_off);
    if (st != GX_OK) {
        gx_column_release_device(col);
        delete col;
        return st;
    }
    *out = col;
    return GX_OK;
}
