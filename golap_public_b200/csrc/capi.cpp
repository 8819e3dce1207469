// capi.cpp -- host-only part of the C-ABI: status strings, thread-local
// error messages, column encoding / inspection.
#include <cuda_runtime.h>

#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <new>

#include "../../include/gx.h"
#include "gx_internal.h"

namespace gx {
static thread_local char g_last_error[1024] = {0};

int set_error(int status, const char* fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_last_error, sizeof(g_last_error), fmt, ap);
    va_end(ap);
    return status;
}
}  // namespace gx

extern "C" {

const char* gx_status_str(gx_status s) {
    switch (s) {
        case GX_OK: return "GX_OK";
        case GX_ERR_CUDA: return "GX_ERR_CUDA";
        case GX_ERR_CORRUPT: return "GX_ERR_CORRUPT";
        case GX_ERR_CAPACITY: return "GX_ERR_CAPACITY";
        case GX_ERR_TIMEOUT: return "GX_ERR_TIMEOUT";
        case GX_ERR_NOMEM: return "GX_ERR_NOMEM";
        case GX_ERR_INVALID: return "GX_ERR_INVALID";
        default: return "GX_ERR_UNKNOWN";
    }
}

size_t gx_last_error(char* buf, size_t cap) {
    size_t n = strlen(gx::g_last_error);
    if (buf && cap) {
        size_t c = n < cap - 1 ? n : cap - 1;
        memcpy(buf, gx::g_last_error, c);
        buf[c] = 0;
    }
    return n;
}

const char* gx_version(void) { return "gx 0.1 (sm_100a)"; }

gx_status gx_device_count(int* count) {
    if (!count) return gx::set_error(GX_ERR_INVALID, "null count");
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess) {
        *count = 0;
        return gx::set_error(GX_ERR_CUDA, "cudaGetDeviceCount: %s", cudaGetErrorString(e));
    }
    *count = n;
    return GX_OK;
}

gx_status gx_encode_opts_default(gx_encode_opts* o) {
    if (!o) return gx::set_error(GX_ERR_INVALID, "null opts");
    o->codec = GX_CODEC_LZ4;
    o->rows_per_chunk = 1000000;
    o->rows_per_block = 16384;
    o->lz4_segments = 128;
    o->lz4_min_match = 0;  // decode-cost-aware
    o->lz4_search_depth = 16;
    o->casc_rle = 1;
    o->casc_delta = 1;
    o->casc_bitpack = 1;
    o->threads = 0;
    return GX_OK;
}

gx_status gx_column_encode(const int32_t* host_values, uint64_t n_rows, const gx_encode_opts* opts, gx_column** out) {
    if (!host_values || !opts || !out) return gx::set_error(GX_ERR_INVALID, "gx_column_encode: null argument");
    gx_column* c = new (std::nothrow) gx_column();
    if (!c) return gx::set_error(GX_ERR_NOMEM, "gx_column_encode: out of host memory");
    int st;
    try {
        st = gx::column_encode(host_values, n_rows, opts->codec, opts->rows_per_chunk, opts->rows_per_block,
                               opts->lz4_segments, opts->lz4_min_match, opts->lz4_search_depth, opts->casc_rle != 0,
                               opts->casc_delta != 0, opts->casc_bitpack != 0, opts->threads, c);
    } catch (const std::bad_alloc&) {
        st = gx::set_error(GX_ERR_NOMEM, "gx_column_encode: out of host memory");
    }
    if (st != GX_OK) {
        delete c;
        return st;
    }
    *out = c;
    return GX_OK;
}

gx_status gx_column_free(gx_column* col) {
    if (!col) return GX_OK;
    col->host_pending = false;  // going away: no host copy needed
    gx_column_release_device(col);
    delete col;
    return GX_OK;
}

gx_status gx_column_info_get(const gx_column* c, gx_column_info* o) {
    if (!c || !o) return gx::set_error(GX_ERR_INVALID, "gx_column_info_get: null argument");
    memset(o, 0, sizeof(*o));
    o->n_rows = c->n_rows;
    uint64_t comp = 0;
    for (const auto& b : c->blocks) comp += b.comp_bytes;
    o->comp_bytes = comp + 4ull * c->seg.size();
    o->uncomp_bytes = 4ull * c->n_rows;
    o->meta_bytes = sizeof(gx::gx_dblock) * c->blocks.size() + 8ull * c->n_chunks;
    o->codec = c->codec;
    o->rows_per_chunk = c->rows_per_chunk;
    o->rows_per_block = c->rows_per_block;
    o->n_chunks = c->n_chunks;
    o->blocks_per_chunk = c->blocks_per_chunk;
    o->n_blocks = c->n_blocks;
    o->lz4_segments = c->codec == GX_CODEC_LZ4 ? c->S : 1u;
    o->on_device = (uint32_t)c->residency;
    return GX_OK;
}

gx_status gx_column_chunk_minmax(const gx_column* c, int32_t* mins, int32_t* maxs) {
    if (!c || !mins || !maxs) return gx::set_error(GX_ERR_INVALID, "gx_column_chunk_minmax: null argument");
    memcpy(mins, c->mins.data(), 4 * c->mins.size());
    memcpy(maxs, c->maxs.data(), 4 * c->maxs.size());
    return GX_OK;
}

gx_status gx_column_block_minmax(const gx_column* c, int32_t* mins, int32_t* maxs) {
    if (!c || !mins || !maxs) return gx::set_error(GX_ERR_INVALID, "gx_column_block_minmax: null argument");
    memcpy(mins, c->bmins.data(), 4 * c->bmins.size());
    memcpy(maxs, c->bmaxs.data(), 4 * c->bmaxs.size());
    return GX_OK;
}

gx_status gx_column_blocks(const gx_column* c, gx_block_info* out) {
    if (!c || !out) return gx::set_error(GX_ERR_INVALID, "gx_column_blocks: null argument");
    uint64_t k = 0;
    for (size_t s = 0; s < c->blocks.size(); ++s) {
        const auto& b = c->blocks[s];
        if (!b.n_rows) continue;
        out[k].offset = b.offset;
        out[k].size = (b.comp_bytes + 15ull) & ~15ull;
        out[k].payload = b.comp_bytes;
        out[k].tuples = b.n_rows;
        ++k;
    }
    return GX_OK;
}

gx_status gx_column_payload(const gx_column* c, const uint8_t** payload, uint64_t* bytes) {
    if (!c || !payload || !bytes) return gx::set_error(GX_ERR_INVALID, "gx_column_payload: null argument");
    if (const int st = gx::host_payload(c)) return st;
    *payload = c->payload.data();
    *bytes = c->payload.size();
    return GX_OK;
}

gx_status gx_column_seg_index(const gx_column* c, const uint32_t** words, uint64_t* n_words) {
    if (!c || !words || !n_words) return gx::set_error(GX_ERR_INVALID, "gx_column_seg_index: null argument");
    *words = c->seg.empty() ? nullptr : c->seg.data();
    *n_words = c->seg.size();
    return GX_OK;
}

}  // extern "C"
