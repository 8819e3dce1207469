// meta.cu -- richer per-chunk pruning metadata, built on the device from a
// compressed column and checked by one launch per predicate.
//
// Reference counterparts (core/metadata.cuh):
//   EqHistogram<T> (:225-382) with fill_hist / check_hist (:573-595):
//     n_buckets equal-width buckets between the chunk's min and max; value v
//     goes to bucket (uint64)((v - min) * n_buckets / (double)(max - min)),
//     clamped to the last bucket (bucket 0 when min == max); a predicate
//     [lo, hi] keeps the chunk when a non-empty bucket lies in
//     [(lo - min) * inv, (hi - min) * inv] (first bucket = the last one when
//     lo == max; for min == max: lo <= min <= hi and bucket 0 non-empty).
//   BloomMeta<T> (:385-537) with fill_bloom / check_bloom (:602-620): an
//     m-byte filter per chunk, k = ceil(ln 2 * 8m / n) hash functions for
//     n = ceil(8m * ln(0.5^ln2) / ln p); bit (h(v + i) mod 8m) for i < k,
//     h the 64-bit finaliser of :464-472 on the value sign-extended to 64 bits.
// Bucket indexes follow the reference's double arithmetic exactly (the
// difference v - min is taken in 64-bit integers, which equals the
// reference's for every range of a 32-bit column).
// The column is decoded chunk range by chunk range into stream-ordered
// scratch (gx_decompress_chunks); per chunk, CTAs accumulate their rows'
// buckets / bits in shared memory and merge them with one atomic per
// non-empty bucket / non-zero word.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>

#include "../../include/gx.h"
#include "gx_internal.h"

using namespace gx;

#define GX_CK(call)                                                                       \
    do {                                                                                  \
        cudaError_t e_ = (call);                                                          \
        if (e_ != cudaSuccess)                                                            \
            return gx::set_error(GX_ERR_CUDA, "%s failed: %s", #call, cudaGetErrorString(e_)); \
    } while (0)

namespace {

constexpr uint32_t kMaxBuckets = 4096;          // shared-memory histogram of one CTA
constexpr uint64_t kMaxBloomBytes = 32u << 10;  // shared-memory filter of one CTA
constexpr uint64_t kPassRows = 64ull << 20;     // rows decoded per pass

__device__ __forceinline__ uint32_t hist_bucket(int32_t v, int32_t mn, int32_t mx, uint32_t nb) {
    if (mx == mn) return 0;
    const double inv = (double)nb / (double)((int64_t)mx - (int64_t)mn);
    const uint64_t b = (uint64_t)((double)((int64_t)v - (int64_t)mn) * inv);
    return (uint32_t)min((uint64_t)nb - 1, b);
}

__device__ __forceinline__ uint64_t bloom_hash(uint64_t v, uint64_t mbits) {
    v ^= v >> 33;
    v *= 0xff51afd7ed558ccdull;
    v ^= v >> 33;
    v *= 0xc4ceb9fe1a85ec53ull;
    v ^= v >> 33;
    return v % mbits;
}

// grid.x = chunks of the pass, grid.y = CTAs per chunk; rows of chunk c at
// vals[(c - c0) * rpc ...]
__global__ void hist_fill_kernel(const int32_t* vals, uint64_t c0, uint64_t rpc, uint64_t n_rows, const int32_t* mins,
                                 const int32_t* maxs, uint32_t nb, unsigned long long* hist) {
    extern __shared__ unsigned long long s_h[];
    const uint64_t c = c0 + blockIdx.x;
    for (uint32_t i = threadIdx.x; i < nb; i += blockDim.x) s_h[i] = 0;
    __syncthreads();
    const uint64_t r0 = c * rpc, rows = min(rpc, n_rows - r0);
    const int32_t mn = mins[c], mx = maxs[c];
    const int32_t* v = vals + (size_t)blockIdx.x * rpc;
    for (uint64_t r = blockIdx.y * (uint64_t)blockDim.x + threadIdx.x; r < rows; r += (uint64_t)gridDim.y * blockDim.x)
        atomicAdd(&s_h[hist_bucket(v[r], mn, mx, nb)], 1ull);
    __syncthreads();
    for (uint32_t i = threadIdx.x; i < nb; i += blockDim.x)
        if (s_h[i]) atomicAdd(&hist[c * nb + i], s_h[i]);
}

__global__ void bloom_fill_kernel(const int32_t* vals, uint64_t c0, uint64_t rpc, uint64_t n_rows, uint64_t m_bytes,
                                  uint32_t k, uint32_t* bloom) {
    extern __shared__ uint32_t s_b[];
    const uint64_t c = c0 + blockIdx.x;
    const uint32_t words = (uint32_t)(m_bytes / 4);
    for (uint32_t i = threadIdx.x; i < words; i += blockDim.x) s_b[i] = 0;
    __syncthreads();
    const uint64_t r0 = c * rpc, rows = min(rpc, n_rows - r0);
    const uint64_t mbits = m_bytes * 8;
    const int32_t* v = vals + (size_t)blockIdx.x * rpc;
    for (uint64_t r = blockIdx.y * (uint64_t)blockDim.x + threadIdx.x; r < rows; r += (uint64_t)gridDim.y * blockDim.x) {
        const uint64_t lv = (uint64_t)(int64_t)v[r];
        for (uint32_t i = 0; i < k; ++i) {
            const uint64_t bit = bloom_hash(lv + i, mbits);
            atomicOr(&s_b[bit >> 5], 1u << (bit & 31));
        }
    }
    __syncthreads();
    for (uint32_t i = threadIdx.x; i < words; i += blockDim.x)
        if (s_b[i]) atomicOr(&bloom[c * words + i], s_b[i]);
}

// one thread per (chunk, bucket), as check_hist walks them
__global__ void hist_check_kernel(const int32_t* mins, const int32_t* maxs, const unsigned long long* hist,
                                  uint64_t n_chunks, uint32_t nb, int32_t lo, int32_t hi, uint16_t* out) {
    for (uint64_t idx = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; idx < n_chunks * nb;
         idx += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t c = idx / nb;
        const int64_t b = (int64_t)(idx % nb);
        const int32_t mn = mins[c], mx = maxs[c];
        if (mn == mx) {
            if (b == 0 && lo <= mn && hi >= mx && hist[c * nb] != 0) out[c] = 1;
            continue;
        }
        const double inv = (double)nb / (double)((int64_t)mx - (int64_t)mn);
        int64_t first = (int64_t)(((double)lo - mn) * inv);
        const int64_t last = (int64_t)(((double)hi - mn) * inv);
        if (lo == mx) first = nb - 1;
        if (first <= b && last >= b && hist[c * nb + b] != 0) out[c] = 1;
    }
}

__global__ void bloom_check_kernel(const uint32_t* bloom, uint64_t n_chunks, uint64_t m_bytes, uint32_t k, int32_t val,
                                   uint16_t* out) {
    const uint64_t mbits = m_bytes * 8;
    const uint64_t lv = (uint64_t)(int64_t)val;
    for (uint64_t c = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; c < n_chunks; c += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t* f = bloom + c * (m_bytes / 4);
        bool res = true;
        for (uint32_t i = 0; i < k; ++i) {
            const uint64_t bit = bloom_hash(lv + i, mbits);
            if (!(f[bit >> 5] & (1u << (bit & 31)))) res = false;
        }
        if (res) out[c] = 1;
    }
}

// The column decoded pass by pass; fn(vals, first chunk, chunks in the pass).
template <class F>
gx_status for_each_pass(gx_column* col, cudaStream_t s, F fn) {
    const uint64_t per = std::max<uint64_t>(1, kPassRows / col->rows_per_chunk);
    const uint64_t cap_rows = std::min<uint64_t>(col->n_rows, per * col->rows_per_chunk);
    int32_t* buf = nullptr;
    GX_CK(cudaMallocAsync((void**)&buf, 4 * cap_rows, s));
    gx_status st = GX_OK;
    for (uint64_t c0 = 0; c0 < col->n_chunks && !st; c0 += per) {
        const uint64_t nc = std::min<uint64_t>(per, col->n_chunks - c0);
        st = gx_decompress_chunks(col, c0, nc, buf, s);
        if (!st) st = fn(buf, c0, nc);
    }
    cudaFreeAsync(buf, s);
    return st;
}

int sm_count_here() {
    int dev = 0, n = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    return n > 0 ? n : 1;
}

}  // namespace

extern "C" {

gx_status gx_column_build_hist(gx_column* col, uint32_t n_buckets, void* stream) {
    if (!col || !col->residency) return set_error(GX_ERR_INVALID, "gx_column_build_hist: column not on the device");
    if (n_buckets == 0 || n_buckets > kMaxBuckets)
        return set_error(GX_ERR_INVALID, "gx_column_build_hist: n_buckets must be in 1..%u", kMaxBuckets);
    cudaStream_t s = (cudaStream_t)stream;
    if (col->d_hist) cudaFree(col->d_hist);
    col->d_hist = nullptr;
    col->hist_buckets = 0;
    const uint64_t bytes = 8ull * col->n_chunks * n_buckets;
    GX_CK(cudaMalloc(&col->d_hist, bytes));
    GX_CK(cudaMemsetAsync(col->d_hist, 0, bytes, s));
    const uint32_t ctas = (uint32_t)std::max<uint64_t>(1, std::min<uint64_t>(64, (col->rows_per_chunk + 4095) / 4096));
    gx_status st = for_each_pass(col, s, [&](const int32_t* v, uint64_t c0, uint64_t nc) -> gx_status {
        hist_fill_kernel<<<dim3((unsigned)nc, ctas), 256, 8ull * n_buckets, s>>>(
            v, c0, col->rows_per_chunk, col->n_rows, col->d_mins, col->d_maxs, n_buckets,
            (unsigned long long*)col->d_hist);
        GX_CK(cudaGetLastError());
        return GX_OK;
    });
    if (!st) col->hist_buckets = n_buckets;
    return st;
}

gx_status gx_check_hist(const gx_column* col, int32_t lo, int32_t hi, uint16_t* out_dev, void* stream) {
    if (!col || !out_dev || !col->d_hist) return set_error(GX_ERR_INVALID, "gx_check_hist: no histograms built");
    const uint64_t n = (uint64_t)col->n_chunks * col->hist_buckets;
    const unsigned grid = (unsigned)std::max<uint64_t>(1, std::min<uint64_t>(4ull * sm_count_here(), (n + 255) / 256));
    hist_check_kernel<<<grid, 256, 0, (cudaStream_t)stream>>>(col->d_mins, col->d_maxs,
                                                               (const unsigned long long*)col->d_hist, col->n_chunks,
                                                               col->hist_buckets, lo, hi, out_dev);
    GX_CK(cudaGetLastError());
    return GX_OK;
}

gx_status gx_column_build_bloom(gx_column* col, uint64_t m_bytes, double p, void* stream) {
    if (!col || !col->residency) return set_error(GX_ERR_INVALID, "gx_column_build_bloom: column not on the device");
    if (m_bytes == 0 || (m_bytes & 3) || m_bytes > kMaxBloomBytes || !(p > 0.0 && p < 1.0))
        return set_error(GX_ERR_INVALID, "gx_column_build_bloom: m_bytes in 4..%llu (a multiple of 4), 0 < p < 1",
                         (unsigned long long)kMaxBloomBytes);
    // the reference's (p, m) parameterisation, core/metadata.cuh:395-400
    const uint64_t mbits = m_bytes << 3;
    const uint64_t nn = (uint64_t)std::ceil(((double)mbits * std::log(std::pow(0.5, std::log(2.0))) / std::log(p)));
    const uint64_t k = (uint64_t)std::ceil(std::log(2.0) * (double)mbits / (double)(nn ? nn : 1));
    if (k == 0 || k > 64)
        return set_error(GX_ERR_INVALID, "gx_column_build_bloom: %llu hash functions", (unsigned long long)k);
    cudaStream_t s = (cudaStream_t)stream;
    if (col->d_bloom) cudaFree(col->d_bloom);
    col->d_bloom = nullptr;
    col->bloom_bytes = 0;
    GX_CK(cudaMalloc(&col->d_bloom, m_bytes * col->n_chunks));
    GX_CK(cudaMemsetAsync(col->d_bloom, 0, m_bytes * col->n_chunks, s));
    const uint32_t ctas = (uint32_t)std::max<uint64_t>(1, std::min<uint64_t>(64, (col->rows_per_chunk + 4095) / 4096));
    gx_status st = for_each_pass(col, s, [&](const int32_t* v, uint64_t c0, uint64_t nc) -> gx_status {
        bloom_fill_kernel<<<dim3((unsigned)nc, ctas), 256, m_bytes, s>>>(v, c0, col->rows_per_chunk, col->n_rows,
                                                                       m_bytes, (uint32_t)k, col->d_bloom);
        GX_CK(cudaGetLastError());
        return GX_OK;
    });
    if (!st) {
        col->bloom_bytes = m_bytes;
        col->bloom_k = (uint32_t)k;
    }
    return st;
}

gx_status gx_check_bloom(const gx_column* col, int32_t value, uint16_t* out_dev, void* stream) {
    if (!col || !out_dev || !col->d_bloom) return set_error(GX_ERR_INVALID, "gx_check_bloom: no Bloom filters built");
    const unsigned grid = (unsigned)std::max<uint64_t>(1, (col->n_chunks + 255) / 256);
    bloom_check_kernel<<<grid, 256, 0, (cudaStream_t)stream>>>(col->d_bloom, col->n_chunks, col->bloom_bytes,
                                                                col->bloom_k, value, out_dev);
    GX_CK(cudaGetLastError());
    return GX_OK;
}

gx_status gx_column_meta_read(const gx_column* col, uint64_t* hist_host, uint32_t* bloom_host, uint32_t* n_buckets,
                              uint64_t* bloom_bytes, uint32_t* bloom_k, void* stream) {
    if (!col) return set_error(GX_ERR_INVALID, "gx_column_meta_read: null column");
    cudaStream_t s = (cudaStream_t)stream;
    if (n_buckets) *n_buckets = col->hist_buckets;
    if (bloom_bytes) *bloom_bytes = col->bloom_bytes;
    if (bloom_k) *bloom_k = col->bloom_k;
    if (hist_host && col->d_hist)
        GX_CK(cudaMemcpyAsync(hist_host, col->d_hist, 8ull * col->n_chunks * col->hist_buckets,
                              cudaMemcpyDeviceToHost, s));
    if (bloom_host && col->d_bloom)
        GX_CK(cudaMemcpyAsync(bloom_host, col->d_bloom, col->bloom_bytes * col->n_chunks, cudaMemcpyDeviceToHost, s));
    GX_CK(cudaStreamSynchronize(s));
    return GX_OK;
}

}  // extern "C"
