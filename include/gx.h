/*
 * gx.h -- C-ABI of the B200-native GOLAP query hot path.
 *
 * Plain pointers and sizes only.  Every entry point returns a gx_status
 * (0 == GX_OK); on failure a thread-local message is available through
 * gx_last_error().  No entry point exits the process, and no device wait is
 * unbounded: kernels that spin carry an iteration cap and report
 * GX_ERR_TIMEOUT through a device error word that the host reads.
 *
 * Each declaration names the reference interface it replaces (paths are
 * relative to the GOLAP source tree).  The C++ drop-in layer in
 * include/golap_compat/ re-exposes those reference class names on top of
 * these calls.
 *
 * Streams are passed as `void*` (a cudaStream_t); NULL is the legacy default
 * stream.  "dev" pointers are device (or device-mapped) addresses.
 */
#ifndef GX_H
#define GX_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------------ status */

typedef int32_t gx_status;
enum {
    GX_OK = 0,
    GX_ERR_CUDA = 1,     /* a CUDA runtime call failed                         */
    GX_ERR_CORRUPT = 2,  /* a compressed block failed validation               */
    GX_ERR_CAPACITY = 3, /* a hash/group table or work list ran out of room    */
    GX_ERR_TIMEOUT = 4,  /* a bounded device or host wait gave up              */
    GX_ERR_NOMEM = 5,    /* allocation failed / admission budget exceeded      */
    GX_ERR_INVALID = 6   /* bad argument                                       */
};

/* Text for a status code (static storage). */
const char* gx_status_str(gx_status s);
/* Copy this thread's last error message into buf (NUL-terminated); returns its length. */
size_t gx_last_error(char* buf, size_t cap);
/* Library version string, and the CUDA device count the library sees. */
const char* gx_version(void);
gx_status gx_device_count(int* count);

/* ------------------------------------------------------- column encoding
 * Replaces: CompInfo / BlockInfo (core/comp.cuh:23-78), ChunkCompressor
 * (core/comp.cuh:81-148), prepare_compressed (core/apps.cuh:149-255) and the
 * per-chunk MinMaxMeta::init_chunk collection (core/metadata.cuh:157-160).
 *
 * A column is split into chunks of rows_per_chunk rows; each chunk into blocks
 * of rows_per_block rows (blocks never straddle chunks).  Every block of every
 * column of a table covers the same rows, so a (chunk, block) pair addresses
 * one row tile across all columns.
 */
enum {
    GX_CODEC_NONE = 0,     /* raw little-endian int32                            */
    GX_CODEC_LZ4 = 1,      /* LZ4 block format, one block per rows_per_block     */
    GX_CODEC_CASCADED = 2  /* RLE + delta + frame-of-reference bit-packing       */
};

typedef struct gx_encode_opts {
    uint32_t codec;            /* GX_CODEC_*                                             */
    uint32_t rows_per_chunk;   /* default 1,000,000                                      */
    uint32_t rows_per_block;   /* default 16,384 (64 KiB of int32)                       */
    uint32_t lz4_segments;     /* independent decode segments per LZ4 block (1..128);
                                  1 = plain LZ4 (one serial stream per block)             */
    uint32_t lz4_min_match;    /* minimum match bytes (multiple of 4, >= 4), or 0: per
                                  block the cheapest of 4/8/16 by bytes + 24 x sequences */
    uint32_t lz4_search_depth; /* hash-chain candidates examined per position            */
    uint32_t casc_rle;         /* cascaded: allow run-length encoding                    */
    uint32_t casc_delta;       /* cascaded: allow delta encoding                         */
    uint32_t casc_bitpack;     /* cascaded: allow bit-packing (else 32-bit words)        */
    uint32_t threads;          /* host encoder threads (0 = hardware concurrency)        */
} gx_encode_opts;

typedef struct gx_column gx_column;

typedef struct gx_column_info {
    uint64_t n_rows;
    uint64_t comp_bytes;       /* payload bytes incl. per-block headers/side indexes   */
    uint64_t uncomp_bytes;     /* n_rows * 4                                            */
    uint64_t meta_bytes;       /* block directory + min/max bytes                        */
    uint32_t codec;
    uint32_t rows_per_chunk;
    uint32_t rows_per_block;
    uint32_t n_chunks;
    uint32_t blocks_per_chunk;
    uint32_t n_blocks;
    uint32_t lz4_segments;
    uint32_t on_device;        /* 0 none, 1 HBM, 2 pinned host (device-mapped)          */
} gx_column_info;

/* One compressed block (the reference BlockInfo, core/comp.cuh:23-32). */
typedef struct gx_block_info {
    uint64_t offset;   /* byte offset of the block in the column payload */
    uint64_t size;     /* bytes reserved for the block (16-byte aligned)  */
    uint64_t payload;  /* bytes actually used by the compressed block     */
    uint64_t tuples;   /* rows in the block                               */
} gx_block_info;

gx_status gx_encode_opts_default(gx_encode_opts* opts);
/* Encode n_rows int32 values from host memory into a new column (host side). */
gx_status gx_column_encode(const int32_t* host_values, uint64_t n_rows,
                           const gx_encode_opts* opts, gx_column** out);
/* lz4_min_match value that admits no match: every LZ4 block is one literal run
 * (the decode-cost-aware policy's no-match candidate). */
#define GX_LZ4_LITERAL 0xFFFFFFF0u
/* Encode n_rows int32 values already in device memory into a new column that is
 * resident in HBM on return (as after gx_column_to_device(col, 1, stream)), with
 * its per-chunk min/max and per-block zone maps filled in.  The host copy of the
 * payload is read back from HBM on first use (gx_column_payload,
 * gx_column_to_device, gx_column_release_device).  The column is byte-identical
 * to gx_column_encode of the same values and options.  Codecs:
 * NONE, CASCADED, and LZ4 with lz4_min_match = GX_LZ4_LITERAL (other LZ4 match
 * policies are GX_ERR_INVALID: use gx_column_encode).  Synchronises `stream`.
 * Replaces: prepare_compressed's per-chunk compress + MinMaxMeta::init_chunk
 * (core/apps.cuh:149-255, core/metadata.cuh:157-160) for data already on the GPU. */
gx_status gx_column_encode_device(const int32_t* values_dev, uint64_t n_rows, const gx_encode_opts* opts,
                                  gx_column** out, void* stream);
gx_status gx_column_free(gx_column* col);
gx_status gx_column_info_get(const gx_column* col, gx_column_info* out);
/* Per-chunk min/max (host arrays of n_chunks entries; MinMaxMeta mins_hst/maxs_hst). */
gx_status gx_column_chunk_minmax(const gx_column* col, int32_t* mins, int32_t* maxs);
/* Per-block zone maps (host arrays of n_chunks * blocks_per_chunk entries, one per
 * block slot in chunk order; a slot past a short chunk's end holds the empty range
 * INT32_MAX / INT32_MIN).  The block-level refinement of MinMaxMeta. */
gx_status gx_column_block_minmax(const gx_column* col, int32_t* mins, int32_t* maxs);
/* Per-block descriptors (host array of n_blocks entries). */
gx_status gx_column_blocks(const gx_column* col, gx_block_info* out);
/* Raw access to the host copy of the compressed payload and the LZ4 segment
 * index (for CPU-side checkers).  Pointers stay valid until gx_column_free. */
gx_status gx_column_payload(const gx_column* col, const uint8_t** payload, uint64_t* bytes);
gx_status gx_column_seg_index(const gx_column* col, const uint32_t** words, uint64_t* n_words);
/* Copy the compressed column to the device.  residency 1 = HBM, 2 = pinned
 * host memory mapped into the device address space (zero-copy reads). */
gx_status gx_column_to_device(gx_column* col, int residency, void* stream);
gx_status gx_column_release_device(gx_column* col);

/* ------------------------------------------------------------ decompression
 * Replaces: ChunkDecompressor::step (core/comp.cuh:151-227, nvCOMP decompress
 * at :186).  Writes the decoded int32 rows of the given chunks to dst_dev. */
gx_status gx_decompress_chunk(const gx_column* col, uint64_t chunk_idx, void* dst_dev, void* stream);
gx_status gx_decompress_chunks(const gx_column* col, uint64_t first_chunk, uint64_t n_chunks,
                               void* dst_dev, void* stream);
/* Decode independent raw LZ4 blocks produced by any conforming LZ4 encoder
 * (e.g. liblz4's LZ4_compress_default, as LZ4CPUManager::compress does at
 * core/comp_cpu.hpp:28-31).  comp_offsets/out_offsets have n_blocks+1 entries
 * (device arrays).  status_dev (n_blocks int32, device) receives 0 or
 * GX_ERR_CORRUPT per block. */
gx_status gx_lz4_decompress_raw(const uint8_t* comp_dev, const uint64_t* comp_offsets_dev,
                                uint8_t* out_dev, const uint64_t* out_offsets_dev,
                                uint64_t n_blocks, int32_t* status_dev, void* stream);

/* ------------------------------------------------------------------ pruning
 * Replaces: MinMaxMeta::check_pred (core/metadata.cuh:203-211), check_mmmeta
 * (core/metadata.cuh:540-547), combine_and (:632-636) and
 * MetaChecker::add_minmax (:645-658).  Inclusive overlap test
 * lo <= chunk_max && hi >= chunk_min; flag 1 = keep. */

/* check_mmmeta semantics: sets out_dev[c] = 1 where the chunk overlaps [lo,hi],
 * leaves other entries untouched. */
gx_status gx_check_minmax(const gx_column* col, int32_t lo, int32_t hi,
                          uint16_t* out_dev, void* stream);
/* out = a & b over n entries (combine_and). */
gx_status gx_combine_and(uint16_t* out_dev, const uint16_t* a_dev, const uint16_t* b_dev,
                         uint64_t n, void* stream);
/* Whole MetaChecker pass in one launch: keep_dev[c] = AND over predicates. */
gx_status gx_prune_minmax(const gx_column* const* cols, const int32_t* lo, const int32_t* hi,
                          uint32_t n_preds, uint16_t* keep_dev, void* stream);
/* Join pruning, check_mmmeta_multiple_pts (core/metadata.cuh:550-560) as used
 * behind --join_prune (usecases/ssb/queries/01.hpp:246-270): sets out_dev[c] = 1
 * where some key lies in chunk c's [min, max] of col, leaves other entries
 * untouched.  The keys are keys_dev[0 .. min(*n_keys_dev, cap)) with the count
 * on the device, as gx_hashtable_keys leaves it (no host synchronisation). */
gx_status gx_check_minmax_points(const gx_column* col, const int32_t* keys_dev, const uint64_t* n_keys_dev,
                                 uint64_t cap, uint16_t* out_dev, void* stream);

/* Richer per-chunk metadata, built on the device from the (device-resident)
 * compressed column and checked with the same flag convention.
 * Replaces: EqHistogram (core/metadata.cuh:225-382) with fill_hist /
 * check_hist (:573-595), and BloomMeta (:385-537) with fill_bloom /
 * check_bloom (:602-620), as MetaChecker::add_hist / add_bloom use them. */
/* n_buckets (1..4096) equal-width buckets per chunk between its min and max. */
gx_status gx_column_build_hist(gx_column* col, uint32_t n_buckets, void* stream);
/* out_dev[c] = 1 where a non-empty bucket of chunk c overlaps [lo, hi]; other entries untouched. */
gx_status gx_check_hist(const gx_column* col, int32_t lo, int32_t hi, uint16_t* out_dev, void* stream);
/* A Bloom filter of m_bytes (a multiple of 4, at most 32 KiB) per chunk for
 * false-positive rate p (the reference's (p, m) parameters). */
gx_status gx_column_build_bloom(gx_column* col, uint64_t m_bytes, double p, void* stream);
/* out_dev[c] = 1 where value may be in chunk c; other entries untouched. */
gx_status gx_check_bloom(const gx_column* col, int32_t value, uint16_t* out_dev, void* stream);
/* Host copies of the built metadata (each pointer may be NULL): counts
 * (n_chunks x n_buckets), filter words (n_chunks x bloom_bytes / 4), sizes. */
gx_status gx_column_meta_read(const gx_column* col, uint64_t* hist_host, uint32_t* bloom_host, uint32_t* n_buckets,
                              uint64_t* bloom_bytes, uint32_t* bloom_k, void* stream);

/* --------------------------------------------------------------- hash join
 * Replaces: HashMap (core/dev_structs.cuh:37-132) with its filtered build
 * hash_map_build_pred_other (core/join.cuh:107-135) and the probe kernels
 * hash_join_count / hash_join_rids (core/join.cuh:46-97).  The table is
 * open addressing with linear probing over 64-bit slots {key, payload};
 * keys are unique on the build side (dimension keys), as in every reference
 * use.  Probing returns the payload of the matching key or "miss". */
typedef struct gx_hashtable gx_hashtable;

/* Conjunctive range predicate on a dimension column (PredInfo, core/dev_structs.cuh:22-26). */
typedef struct gx_pred {
    const int32_t* col_dev;
    int32_t lo;
    int32_t hi;
} gx_pred;

gx_status gx_hashtable_create(uint64_t max_entries, gx_hashtable** out);
/* Table layouts: linear probing over single slots, or buckets of 8 slots
 * (64 bytes, read with one 64-byte access per probe step), or a dense table
 * for build keys that fill most of an integer range (surrogate keys,
 * yyyymmdd dates): slot 1 + (key - base) holds the key's entry, so a probe
 * is one read.  A dense table is sized by gx_hashtable_build to the range of
 * the inserted keys (it synchronises the stream once to read the range); a
 * range wider than max(64 * max_entries, 2^20) keys fails with
 * GX_ERR_INVALID.  Formats in include/gx_hash.h. */
enum { GX_HT_LINEAR = 0, GX_HT_BUCKET = 1, GX_HT_DENSE = 2 };
gx_status gx_hashtable_create2(uint64_t max_entries, uint32_t layout, gx_hashtable** out);
gx_status gx_hashtable_free(gx_hashtable* ht);
/* Clear, then insert (keys[i], payload[i] or i when payload_dev == NULL) for
 * every row i < n that passes all predicates.  Duplicate keys: the first
 * inserted wins for probing, later ones are counted as dropped. */
gx_status gx_hashtable_build(gx_hashtable* ht, const int32_t* keys_dev, const int32_t* payload_dev,
                             uint64_t n, const gx_pred* preds, uint32_t n_preds, void* stream);
/* Number of inserted entries (host, synchronises the stream). */
gx_status gx_hashtable_count(const gx_hashtable* ht, uint64_t* n_entries, void* stream);
/* For each probe key: payload_out[i] = payload or INT32_MIN on a miss
 * (payload_out may be NULL); *hits_dev += number of hits (may be NULL). */
gx_status gx_hashtable_probe(const gx_hashtable* ht, const int32_t* keys_dev, uint64_t n,
                             int32_t* payload_out_dev, uint64_t* hits_dev, void* stream);

/* Device view of the table for probing from other kernels (slot format and
 * hash in include/gx_hash.h): *slots_dev = 2^log2cap 64-bit slots (for a
 * dense table, take the view after gx_hashtable_build, which sizes it).  Replaces
 * passing HashMap by value to a kernel (core/dev_structs.cuh:71-82). */
gx_status gx_hashtable_view(const gx_hashtable* ht, const uint64_t** slots_dev, uint32_t* log2cap);

/* Writable view for inserting from other kernels (linear tables only):
 * counters_dev[0] counts inserted keys, [1] duplicates, [2] rows that found
 * no slot or carried the reserved key (gx_hashtable_count reads them).
 * Replaces HashMap::insert from a kernel (core/dev_structs.cuh:89-98), used by
 * hash_map_build_pred_other (core/join.cuh:107-135) and
 * pipeline_customer_q3 (usecases/ssb/queries/03.cuh:94-116). */
gx_status gx_hashtable_view2(gx_hashtable* ht, uint64_t** slots_dev, uint32_t* log2cap, uint64_t** counters_dev);
/* Keys of the table's entries into keys_dev (any order; at most cap written),
 * their count into *n_keys_dev (device uint64, may exceed cap).  Replaces
 * collect_hashmap_keys (core/dev_structs.cuh:136-150). */
gx_status gx_hashtable_keys(const gx_hashtable* ht, int32_t* keys_dev, uint64_t cap, uint64_t* n_keys_dev,
                            void* stream);
/* Empty every slot and zero the counters (the cudaMemset of the HashMap
 * constructor, core/dev_structs.cuh:47-56); gx_hashtable_build clears by itself. */
gx_status gx_hashtable_clear(gx_hashtable* ht, void* stream);

/* ------------------------------------------------------------ min/max
 * Replaces: MinMaxMeta::init_chunk (core/metadata.cuh:157-160), the two CUB
 * reductions per chunk: range_dev[0] = min, range_dev[1] = max of data_dev[0..n)
 * (device arrays; for n == 0 they stay INT32_MAX / INT32_MIN). */
gx_status gx_minmax_reduce(const int32_t* data_dev, uint64_t n, int32_t* range_dev, void* stream);

/* ---------------------------------------------------------- hash aggregate
 * Replaces: HashAggregate (core/dev_structs.cuh:158-253) with SumAgg
 * (usecases/ssb/queries/query_common.cuh:24-29) and the group_by_agg kernels
 * (core/group.cuh:15-36).  Open addressing over int64 keys, int64 sums. */
typedef struct gx_groupby gx_groupby;

gx_status gx_groupby_create(uint64_t max_groups, gx_groupby** out);
gx_status gx_groupby_free(gx_groupby* gb);
gx_status gx_groupby_reset(gx_groupby* gb, void* stream);
/* sums[key] += vals[i] for i < n (device arrays). */
gx_status gx_groupby_add(gx_groupby* gb, const int64_t* keys_dev, const int64_t* vals_dev,
                         uint64_t n, void* stream);
/* Device view for aggregating from other kernels (format in include/gx_hash.h):
 * 2^log2cap int64 keys and sums.  Replaces passing HashAggregate by value
 * (core/dev_structs.cuh:196-207). */
gx_status gx_groupby_view(gx_groupby* gb, int64_t** keys_dev, int64_t** sums_dev, uint32_t* log2cap);
/* Copy the non-empty groups to host arrays (unordered); *n_groups = count.
 * Fails with GX_ERR_CAPACITY if cap is too small or the table overflowed. */
gx_status gx_groupby_read(gx_groupby* gb, int64_t* keys_host, int64_t* sums_host, uint64_t cap,
                          uint64_t* n_groups, void* stream);

/* -------------------------------------------------------------- fused scan
 * Replaces: ChunkDecompressor + pipeline_q1_lineorder
 * (usecases/ssb/queries/01.cuh:27-54) and ChunkDecompressor +
 * pipeline_q3 (usecases/ssb/queries/03.cuh:119-170), driven per chunk by the
 * worker loops of usecases/ssb/queries/01.hpp:350-424 and 03.hpp:487-547.
 *
 * A plan is an ordered list of column steps over one fact table.  For every
 * row tile that survives pruning, one kernel decodes each referenced column
 * into shared memory, applies the steps in order, and aggregates.
 *   FILTER  : keep rows with lo <= v <= hi
 *   PROBE   : keep rows whose value is a key of ht; if digit_card > 0 the
 *             payload p extends the group key: g = g*digit_card + (p-digit_base)
 *   CARRY   : remember v (for SUM_PRODUCT / SUM_DIFF, or as a BUILD payload)
 *   VALUE   : aggregate v (times the carried value when agg == SUM_PRODUCT,
 *             minus it when agg == SUM_DIFF)
 *   GROUP   : the value itself extends the group key like a PROBE payload
 *             (g = g*digit_card + (v-digit_base)); GROUP BY a fact column
 * Flags may be OR-ed (FILTER|CARRY).  The aggregate is int64:
 * a scalar sum (groupby == NULL) or sums per group key. */
enum {
    GX_STEP_FILTER = 1,
    GX_STEP_PROBE = 2,
    GX_STEP_CARRY = 4,
    GX_STEP_VALUE = 8,
    GX_STEP_GROUP = 16
};
enum { GX_AGG_SUM = 0, GX_AGG_SUM_PRODUCT = 1, GX_AGG_COUNT = 2, GX_AGG_BUILD = 3, GX_AGG_SUM_DIFF = 4 };
/* GX_AGG_SUM_DIFF sums v - carried (SUM(lo_revenue - lo_supplycost) of
 * usecases/ssb/queries/04inmem.hpp:146).  A plan may carry a value and build
 * a group key at once only where gx_scan runs it in the shared or pipelined
 * form (segmented LZ4, its only VALUE step last); gx_scan_static and queue-form
 * batches refuse such plans. */
/* GX_AGG_BUILD fills a join table instead of aggregating: every row that
 * passes the plan's FILTER / PROBE steps is inserted into plan.build_ht with
 * the VALUE step's column as the key and the carried value (a CARRY step) as
 * the payload, or the table row number when the plan carries nothing.  The
 * scan does not clear the table first (gx_hashtable_clear); duplicate keys
 * behave as in gx_hashtable_build and gx_hashtable_count reports the rows.
 * Linear and bucket tables; columns HBM-resident, LZ4 columns segmented.
 * Replaces: pipeline_customer_q3 (usecases/ssb/queries/03.cuh:94-116) with the
 * per-chunk loop that feeds it decompressed customer chunks
 * (usecases/ssb/queries/03.hpp:408-476): decode, filter, compact and insert
 * become one fused kernel over the compressed dimension columns. */

#define GX_MAX_STEPS 8

typedef struct gx_scan_step {
    const gx_column* col;
    uint32_t flags;              /* GX_STEP_*                                  */
    int32_t lo, hi;              /* FILTER bounds (inclusive)                  */
    const gx_hashtable* ht;      /* PROBE table                                */
    int32_t digit_base;          /* PROBE: payload offset for the group key    */
    uint32_t digit_card;         /* PROBE: payload cardinality (0 = no digit)  */
} gx_scan_step;

/* Min/max pruning predicate evaluated by the scan itself (the MetaChecker
 * pass of usecases/ssb/queries/01.hpp:263-281 folded into the launch). */
typedef struct gx_scan_prune {
    const gx_column* col;
    int32_t lo, hi;
} gx_scan_prune;

typedef struct gx_scan_plan {
    uint32_t n_steps;
    gx_scan_step steps[GX_MAX_STEPS];
    uint32_t agg;                     /* GX_AGG_*                                */
    const uint16_t* keep_chunks_dev;  /* per-chunk keep flags or NULL (scan all) */
    gx_groupby* groupby;              /* NULL = scalar result                    */
    int64_t* result_dev;              /* scalar result (int64, device)           */
    uint32_t n_prune;                 /* min/max predicates ANDed with keep_chunks */
    gx_scan_prune prune[GX_MAX_STEPS];
    uint16_t* keep_out_dev;           /* optional: resulting per-chunk flags     */
    gx_hashtable* build_ht;           /* GX_AGG_BUILD: the table rows go into    */
} gx_scan_plan;

/* Run the plan on `stream`.  Does not clear result_dev or the group table
 * (callers accumulate across calls, like the reference's atomics).  The
 * launch may overlap the kernel just before it on the stream (programmatic
 * dependent launch): until that kernel completes the scan only reads column
 * data; join tables, keep_chunks_dev, results, group tables and keep_out_dev
 * are read and written after it, so every write of earlier work is seen. */
gx_status gx_scan(const gx_scan_plan* plan, void* stream);
/* Same, then synchronise and report device-side errors (corrupt blocks,
 * table overflow).  *rows_scanned (optional) = rows in surviving tiles. */
gx_status gx_scan_sync(const gx_scan_plan* plan, void* stream, uint64_t* rows_scanned);
/* Read and clear the device error word of the scan engine. */
gx_status gx_scan_check(void* stream);

/* Which kernel form gx_scan / gx_scan_sync / gx_scan_streamed use.  No
 * reference counterpart (the reference has one kernel per query shape).
 * GX_FORM_AUTO (default) tries, in this order: the warp-tile scan (one warp
 * per 1024-row tile, no block-wide barriers; LZ4 columns segmented with
 * segments of at most 1024 rows, no GX_AGG_BUILD), the pipelined scan (a
 * producer warp staging tiles with bulk copies for 16 consumer warps), the
 * shared form (one CTA per 2048-row tile) and the queue form (any plan).
 * Any other value forces that form: plans it cannot run fail with
 * GX_ERR_INVALID (the queue form accepts what gx_scan accepts, except a
 * carried value combined with group-key digits).  Every form gives identical
 * results.  Process-wide setting, for tests and measurements. */
enum { GX_FORM_AUTO = 0, GX_FORM_WARP = 1, GX_FORM_PIPE = 2, GX_FORM_SHARED = 3, GX_FORM_QUEUE = 4 };
gx_status gx_scan_set_form(uint32_t form);

/* Streamed scan of a plan whose columns are in pinned host memory
 * (gx_column_to_device with residency 2).  Replaces the reference's load-then-decompress chain
 * for host-resident columns (DataCopy / VarLoader / BatchLoader feeding the
 * decompressor: core/access.hpp:17-60, 190-435, one chunk per pipeline step):
 * the table is cut into groups of `chunks_per_group` chunks; the compressed
 * bytes of each group's chunks that survive the plan's min/max predicates
 * are copied host->HBM with cudaMemcpyAsync on an internal copy stream into
 * one of two staging buffers, and the group is scanned from HBM by the
 * warp-tile kernel (else the pipelined one; see gx_scan_set_form) while the
 * next group's bytes are copied.  Pruned chunks are never copied.  Results
 * equal gx_scan's.  keep_chunks_dev is applied by the kernel (chunks it drops
 * are still copied).  HBM-resident columns of the plan are read in place.
 * Plans neither kernel runs (GX_AGG_BUILD, queue-only shapes) are rejected
 * with GX_ERR_INVALID.
 * Staging memory (two buffers per host column, each the largest group's
 * bytes) comes from the stream-ordered pool and is released on `stream`. */
gx_status gx_scan_streamed(const gx_scan_plan* plan, uint32_t chunks_per_group, void* stream);

/* Allocation-free form of gx_scan.  No reference counterpart: the reference
 * has no scan entry point whose scratch avoids the allocator.
 * Identical results to gx_scan, but always through the two-launch queue form
 * (a pruning/work-list kernel, then the per-query scan kernel), whose chunk
 * work list lives in one file-scope device array per device
 * (GX_SCAN_STATIC_MAX_CHUNKS chunk ids, 64 KiB) instead of stream-ordered
 * pool memory, so the call never allocates or frees device memory.  (Plans
 * that gx_scan runs as a single pipelined or shared-form launch take no
 * scratch there either; this entry point keeps them on the queue form.)  It is for callers that own every byte of device
 * memory through their own budget (tables carved out of HBM up front, with
 * the driver's pool kept empty) and for callers that cannot afford a pool
 * allocation that may fail or map new memory in the middle of a query.
 * Plans over more than GX_SCAN_STATIC_MAX_CHUNKS chunks are rejected with
 * GX_ERR_INVALID.  Nothing in the array has to start at zero: the launch
 * writes the chunk count and resets the work counter before the scan reads
 * them, in stream order.  The array is shared by all callers on a device, so
 * two calls that can overlap in time (different streams, or different host
 * threads without ordering between their streams) race and give wrong
 * results: serialise them on one stream. */
#define GX_SCAN_STATIC_MAX_CHUNKS 16384u
gx_status gx_scan_static(const gx_scan_plan* plan, void* stream);

/* ------------------------------------------------------------ batched scan
 * No reference counterpart (the reference runs one query per pipeline).
 * Many plans over the same fact table, each restricted to a row slice
 * [row_lo, row_hi), run as ONE persistent launch: a single work list of
 * (query, chunk) items is built on the device after per-query min/max
 * pruning, and every CTA switches between queries as it takes items.  Each
 * query's result_dev (scalar) or groupby (grouped) receives exactly what
 * gx_scan of that plan alone over the slice would produce; gx_batch_run
 * clears them first.  The launch sequence can be captured once into a CUDA
 * graph and replayed (gx_batch_graph). */
typedef struct gx_query {
    gx_scan_plan plan;   /* keep_chunks_dev / keep_out_dev are ignored */
    uint64_t row_lo, row_hi;
} gx_query;

typedef struct gx_batch gx_batch;

gx_status gx_batch_create(const gx_query* queries, uint32_t n_queries, gx_batch** out);
/* Execution form.  QUEUE: the work list above, every query decoding its own
 * columns.  SHARED: every (block, tile) that any query needs is decoded once
 * -- each column its active queries read, into shared memory -- and all of
 * those queries are evaluated on it; needs every plan to end with its only
 * VALUE step, LZ4 columns with segments of at most 2048 rows, at most 16
 * distinct columns and 1024 queries.  AUTO (gx_batch_create): SHARED when
 * the batch qualifies, else QUEUE; asking for SHARED when it does not
 * qualifies fails with GX_ERR_INVALID and the reason. */
enum { GX_BATCH_AUTO = 0, GX_BATCH_QUEUE = 1, GX_BATCH_SHARED = 2 };
gx_status gx_batch_create2(const gx_query* queries, uint32_t n_queries, uint32_t mode, gx_batch** out);
/* The form the batch currently runs in (GX_BATCH_QUEUE or GX_BATCH_SHARED). */
gx_status gx_batch_mode(const gx_batch* b, uint32_t* mode);
/* Launch shape of the shared form: threads per CTA (128, 256, 512 or 1024,
 * or 0 = automatic, the default: of 256, 512 and 128, the size with the most
 * resident warps for the batch's shared memory) and a cap on CTAs per SM
 * (0 = as many as fit).
 * Kept across gx_batch_assign; drops a captured graph.  The autotuner sets
 * it. */
gx_status gx_batch_set_launch(gx_batch* b, uint32_t threads, uint32_t ctas_per_sm);
/* Threads per CTA the shared form currently launches with (0 for QUEUE). */
gx_status gx_batch_launch_get(const gx_batch* b, uint32_t* threads);
/* Replace the batch's queries (buffers reused, grown when needed; the
 * descriptor upload is enqueued on `stream`).  Drops a captured graph. */
gx_status gx_batch_assign(gx_batch* b, const gx_query* queries, uint32_t n_queries, void* stream);
gx_status gx_batch_free(gx_batch* b);
/* Clear results, build the work list, run all queries (3 or 4 launches). */
gx_status gx_batch_run(gx_batch* b, void* stream);
/* Capture gx_batch_run into a CUDA graph on first use, then replay it. */
gx_status gx_batch_graph(gx_batch* b, void* stream);
/* Rows of surviving tiles counted by the last run (host, synchronises). */
gx_status gx_batch_rows(gx_batch* b, uint64_t* rows, void* stream);

/* ------------------------------------------------------------ serving loop
 * No reference counterpart.  A continuous-batching server over resident
 * tables: submit() queues a request (a gx_query plus the device bytes it
 * holds while running: its group table and result); a scheduler thread keeps
 * up to max_inflight batches on the device, each formed FIFO from the queue
 * as soon as a slot is free, admitting requests while the admitted bytes stay
 * within hbm_budget; under load (a queue of max_batch / 4 or more) a free
 * slot waits while another batch runs, so that batches grow (larger batches
 * share each decoded tile among more queries).  A request's results land in its own result_dev /
 * groupby.  wait() blocks (bounded) until the request is done and reports its
 * latency (submit -> completion). */
typedef struct gx_server gx_server;
typedef struct gx_server_opts {
    uint32_t max_inflight;  /* batches on the device at once (default 4)       */
    uint32_t max_batch;     /* requests per batch (default 128)                */
    uint64_t hbm_budget;    /* bytes admitted requests may hold (default 120 GiB) */
    uint32_t batch_threads; /* launch shape of shared-form batches (0 = default) */
    uint32_t batch_mode;    /* GX_BATCH_AUTO / QUEUE / SHARED (default AUTO)   */
} gx_server_opts;
typedef struct gx_server_stats {
    uint64_t submitted, completed, rejected, batches, queries_in_batches;
    uint64_t hbm_in_use, hbm_peak, queued;
} gx_server_stats;

gx_status gx_server_opts_default(gx_server_opts* opts);
gx_status gx_server_create(const gx_server_opts* opts, gx_server** out);
/* GX_ERR_NOMEM when hbm_bytes exceeds the whole budget (rejected). */
gx_status gx_server_submit(gx_server* sv, const gx_query* q, uint64_t hbm_bytes, uint64_t* ticket);
gx_status gx_server_wait(gx_server* sv, uint64_t ticket, double timeout_s, double* latency_ms);
gx_status gx_server_stats_get(gx_server* sv, gx_server_stats* out);
/* Drains the queue (waits for running batches), then stops the scheduler. */
gx_status gx_server_free(gx_server* sv);

#ifdef __cplusplus
}
#endif
#endif /* GX_H */
