// gx_internal.h -- formats and structures shared by the host encoder, the
// C-ABI layer and the sm_100a kernels.
//
// Layout of a compressed column in memory (host and HBM alike):
//
//   payload   : concatenation of per-block byte streams (raw and cascaded
//               blocks start on a 16-byte boundary, LZ4 blocks see below),
//               followed by kPayloadSlack bytes of slack at the very end.
//   directory : one gx_dblock per (chunk, block-in-chunk) slot, padded to
//               n_chunks * blocks_per_chunk entries; absent blocks of a short
//               last chunk have n_rows == 0.
//   seg index : LZ4 columns with S > 1 segments: S pairs of uint32 per block
//               (see "segmented LZ4" below); cascaded columns: one pair
//               {page offset, page bytes} per page (see "cascaded block").
//   min/max   : int32 per chunk (inclusive), the MinMaxMeta of the reference
//               (core/metadata.cuh:110-221).
//
// Segmented LZ4 (own encoder policy on top of the standard LZ4 block format;
// any LZ4 decoder, e.g. liblz4, decodes these blocks unchanged):
//   * a block of R rows is divided into S segments of R/S rows; segment j
//     produces output bytes [N_j, N_j+1) with N_j = min(j*R/S, rows)*4;
//   * no match crosses a segment boundary, and every match source lies in
//     the same segment (so each segment decodes independently);
//   * all literal runs, match lengths and offsets are multiples of 4 bytes
//     (int32 granularity), so decoders copy whole words;
//   * entry j = {comp_pos, info}: the decoder state at output byte N_j.
//       info bit 4 == 0: comp_pos is a token position;
//       info bit 4 == 1: comp_pos is the position of the literal byte that
//       produces N_j (or of the 16-bit match offset when no literal remains);
//       info >> 5 = literal bytes remaining in that sequence, info & 15 = the
//       token's match-length nibble.  Entry 0 resumes inside the block's
//       first literal run when the block starts with literals.
//
//   LZ4 blocks start anywhere in the payload (not necessarily on a 16-byte
//   boundary): a block that opens with literals is placed so that its first
//   literal byte is 16-byte aligned, so the row tiles of a literal run are
//   16-byte aligned byte ranges that bulk copies move unshifted.
//
// Cascaded block (own format; the reference's nvCOMP Cascaded stream format
// is not available, so only decoded values are comparable).  The block is a
// sequence of independently decodable pages of kCascPageRows rows (the last
// one shorter), so one row tile never needs the rest of its block:
//   block header: uint32 n_pages, uint32 page_rows, uint32 page_off[n_pages+1]
//   (byte offsets from the block start; the last one is the stream end),
//   padded to 16 bytes; then the pages, each 16-byte aligned.  The column's
//   side index repeats {page_off, page_bytes} per page (S = pages per block,
//   seg_shift = log2(kCascPageRows)) so device code locates a page with
//   independent loads.
// Cascaded page: casc_hdr (32 bytes), then a bit-packed value stream and,
//   with RLE (at most kCascPageMaxRuns runs), a bit-packed run-length stream,
//   each 16-byte aligned, each with one padding word.  Values: with DELTA,
//   entry 0 is 0 and entry i = v[i]-v[i-1] (wrapping int32); the stored word
//   is entry - val_base (frame of reference) in val_bits bits.  Lengths:
//   stored length - len_base in len_bits bits.  v[i] = first +
//   sum_{k<=i} entry[k] with DELTA, else entry[i].  Element i of a stream
//   with width w sits at bits [i*w, i*w+w) of the little-endian uint32 word
//   sequence.
#pragma once
#include <stdint.h>

#include "../../include/gx_hash.h"

#ifndef GX_HOSTDEV
#if defined(__CUDACC__)
#define GX_HOSTDEV __host__ __device__
#else
#define GX_HOSTDEV
#endif
#endif

namespace gx {

constexpr uint32_t kMaxRowsPerBlock = 16384;   // 64 KiB of int32: one decode buffer
constexpr uint32_t kMaxSegments = 128;
constexpr uint32_t kCascMaxRuns = 2048;        // run tables of one decode (>= kCascPageMaxRuns)
constexpr uint32_t kCascPageLog2 = 11;
constexpr uint32_t kCascPageRows = 1u << kCascPageLog2;  // rows of one cascaded page
constexpr uint32_t kCascPageMaxRuns = 512;     // RLE pages hold at most this many runs
constexpr uint32_t kCascMaxPages = kMaxRowsPerBlock / kCascPageRows;
constexpr uint32_t kStageBytes = 66048;        // shared staging buffer for one compressed block
constexpr uint32_t kPayloadAlign = 16;
constexpr uint32_t kPayloadSlack = 64;
constexpr int32_t kEmptyKey = INT32_MIN;        // hash-table empty marker (reserved key)
constexpr int64_t kEmptyGroup = INT64_MIN;      // group-table empty marker (reserved key)

enum CascFlags : uint8_t { CASC_RLE = 1, CASC_DELTA = 2 };

struct casc_hdr {
    uint32_t n_rows;
    uint32_t n_runs;     // == n_rows without RLE
    uint8_t flags;       // CascFlags
    uint8_t val_bits;    // 0..32
    uint8_t len_bits;    // 0..16
    uint8_t pad;
    int32_t first;       // DELTA: v[0]
    int32_t val_base;    // frame of reference for the value stream
    uint32_t len_base;   // frame of reference for run lengths
    uint32_t vals_off;   // byte offset of the value stream from the block start
    uint32_t lens_off;   // byte offset of the length stream (0 without RLE)
};
static_assert(sizeof(casc_hdr) == 32, "casc_hdr layout");

// Device block descriptor (16 bytes).
struct gx_dblock {
    uint64_t offset;      // byte offset of the block stream in the payload
    uint32_t comp_bytes;  // bytes used by the stream
    uint32_t n_rows;      // rows in the block (0 = absent slot)
};
static_assert(sizeof(gx_dblock) == 16, "gx_dblock layout");

// POD view of a device-resident column, passed by value to kernels.
struct gx_dcol {
    const uint8_t* payload;
    const gx_dblock* blocks;
    const uint32_t* seg;        // 2*S words per block (LZ4 with S > 1, cascaded), else null
    const int32_t* mins;
    const int32_t* maxs;
    uint64_t n_rows;
    uint32_t codec;
    uint32_t S;                 // LZ4 segments per block (1 = plain LZ4); cascaded: pages per block
    uint32_t seg_shift;         // log2(rows per segment / page) when the side index exists
    uint32_t rows_per_chunk;
    uint32_t rows_per_block;
    uint32_t blocks_per_chunk;
    uint32_t n_chunks;
    uint32_t n_slots;           // n_chunks * blocks_per_chunk
    uint64_t payload_bytes;     // size of the payload allocation
    uint32_t host_mapped;       // payload lives in pinned host memory (no TMA staging)
    uint32_t pad_;
};

// Bit-packed stream reader: element i of width w (0..32).
GX_HOSTDEV inline uint32_t unpack_bits(const uint32_t* words, uint32_t i, uint32_t w) {
    if (w == 0) return 0;
    uint64_t bit = (uint64_t)i * w;
    uint32_t wi = (uint32_t)(bit >> 5), sh = (uint32_t)(bit & 31);
    uint64_t two = (uint64_t)words[wi] | ((uint64_t)words[wi + 1] << 32);
    uint64_t mask = (w == 32) ? 0xFFFFFFFFull : ((1ull << w) - 1);
    return (uint32_t)((two >> sh) & mask);
}

// Join/group table hashing: the public definitions in include/gx_hash.h.
GX_HOSTDEV inline uint32_t hash_key32(int32_t key, uint32_t log2cap) { return gx_hash32(key, log2cap); }
GX_HOSTDEV inline uint32_t hash_key64(int64_t key, uint32_t log2cap) { return gx_hash64(key, log2cap); }

}  // namespace gx

// ---------------------------------------------------------------- host side
#include <string>
#include <vector>

struct gx_column {
    // layout
    uint64_t n_rows = 0;
    uint32_t codec = 0;
    uint32_t rows_per_chunk = 0, rows_per_block = 0;
    uint32_t n_chunks = 0, blocks_per_chunk = 0, n_blocks = 0, n_slots = 0;
    uint32_t S = 1, seg_shift = 0;
    // host copy
    std::vector<uint8_t> payload;
    std::vector<gx::gx_dblock> blocks;   // n_slots entries
    std::vector<uint32_t> seg;           // 2*S*n_slots words (S > 1)
    std::vector<int32_t> mins, maxs;     // n_chunks
    std::vector<int32_t> bmins, bmaxs;   // n_slots: per-block zone map (absent slots: empty range)
    // device copy
    int residency = 0;                   // 0 none, 1 HBM, 2 pinned host (mapped)
    void* d_payload = nullptr;           // device address (HBM or mapped)
    void* h_pinned = nullptr;            // pinned host allocation (residency 2)
    gx::gx_dblock* d_blocks = nullptr;
    uint32_t* d_seg = nullptr;
    int32_t* d_mins = nullptr;
    int32_t* d_maxs = nullptr;
    // richer pruning metadata built on the device (meta.cu): equal-width
    // histograms (hist_buckets counts per chunk) and Bloom filters
    // (bloom_bytes per chunk, bloom_k hash functions)
    uint32_t hist_buckets = 0;
    uint64_t* d_hist = nullptr;
    uint64_t bloom_bytes = 0;
    uint32_t bloom_k = 0;
    uint32_t* d_bloom = nullptr;
    // LZ4: every block is one 16-byte aligned literal run (-1 = not known yet)
    mutable int lz4_direct = -1;
    int32_t* d_bmins = nullptr;
    int32_t* d_bmaxs = nullptr;
    int device = -1;
    // a column encoded on the device keeps its payload in HBM only until a
    // caller needs the host copy (gx::host_payload reads it back once)
    mutable bool host_pending = false;
    uint64_t dev_payload_bytes = 0;

    gx::gx_dcol view() const {
        gx::gx_dcol v{};
        v.payload = (const uint8_t*)d_payload;
        v.blocks = d_blocks;
        v.seg = d_seg;
        v.mins = d_mins;
        v.maxs = d_maxs;
        v.n_rows = n_rows;
        v.codec = codec;
        v.S = S;
        v.seg_shift = seg_shift;
        v.rows_per_chunk = rows_per_chunk;
        v.rows_per_block = rows_per_block;
        v.blocks_per_chunk = blocks_per_chunk;
        v.n_chunks = n_chunks;
        v.n_slots = n_slots;
        v.payload_bytes = host_pending ? dev_payload_bytes : payload.size();
        v.host_mapped = residency == 2 ? 1u : 0u;
        return v;
    }
};

namespace gx {
// Thread-local error message plumbing (implemented in capi.cpp).
int set_error(int status, const char* fmt, ...);
// Fills the host copy of a device-encoded column's payload (once; a no-op for
// columns encoded on the host).  Implemented in encode_gpu.cu.
int host_payload(const gx_column* col);

// Host encoders (encode.cpp).
// Encodes `rows` int32 values as a segmented (S > 1) or plain (S == 1) LZ4
// block; returns the compressed size, appends S {comp_pos, info} pairs to seg.
size_t lz4_encode_block(const int32_t* vals, uint32_t rows, uint32_t S, uint32_t seg_rows,
                        uint32_t min_match, uint32_t depth, std::vector<uint8_t>& out,
                        uint32_t* seg_entries, uint32_t* n_seq);
size_t lz4_encode_block_auto(const int32_t* vals, uint32_t rows, uint32_t S, uint32_t seg_rows, uint32_t depth,
                             std::vector<uint8_t>& out, uint32_t* seg_entries);
size_t casc_encode_page(const int32_t* vals, uint32_t rows, bool allow_rle, bool allow_delta,
                        bool allow_bp, std::vector<uint8_t>& out);
// A block of pages; page_entries receives {page_off, page_bytes} per page.
size_t casc_encode_block(const int32_t* vals, uint32_t rows, bool allow_rle, bool allow_delta,
                         bool allow_bp, std::vector<uint8_t>& out, uint32_t* page_entries);
// Column encoder (encode.cpp): fills layout, payload, directory, min/max.
int column_encode(const int32_t* vals, uint64_t n_rows, uint32_t codec, uint32_t rows_per_chunk,
                  uint32_t rows_per_block, uint32_t S, uint32_t min_match, uint32_t depth,
                  bool rle, bool delta, bool bp, uint32_t threads, gx_column* col);
}  // namespace gx
