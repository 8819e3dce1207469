// golap_compat.cuh -- the reference's operator names over the gx C-ABI.
//
// A pipeline written against GOLAP's core/comp.cuh, core/metadata.cuh,
// core/join.cuh, core/agg.cuh and core/dev_structs.cuh (e.g. the worker loop
// of usecases/ssb/queries/01.hpp:350-424) switches to the B200 build by
// including this header instead.  Differences that a caller sees:
//   * CompInfo owns a gx_column (the compressed chunk store, HBM or pinned
//     host); it is produced by prepare_compressed() from a host int32 column
//     instead of by an nvCOMP manager.
//   * ChunkDecompressor takes the CompInfo instead of an nvCOMP manager.
//   * MinMaxMeta<int32_t> is filled at ingest (no CUB pass per chunk).
//   * HashMap is open addressing: insert happens in bulk through build()
//     (hash_map_build_pred_other); probe(key) is a __device__ function like
//     the reference's and returns the build payload (row id by default) or
//     (uint64_t)-1.  Build keys must be unique and != INT32_MIN.
//   * HashAggregate keys are int64; add(key, val) sums int64 values.
//   * Errors throw std::runtime_error with the library's message instead of
//     calling exit().
// Objects own their device memory; copies passed by value into kernels are
// non-owning views (the reference's is_orig pattern).
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "../gx.h"
#include "../gx_hash.h"

namespace golap {

inline void gx_check(gx_status s) {
    if (s != GX_OK) {
        char buf[1024];
        gx_last_error(buf, sizeof buf);
        throw std::runtime_error(std::string(gx_status_str(s)) + ": " + buf);
    }
}

// ------------------------------------------------------------- comp.cuh
// core/comp.cuh:23-32
struct BlockInfo {
    uint64_t offset;
    uint64_t size;
    uint64_t payload;
    uint64_t tuples;
};

// core/comp.cuh:35-78.  chunk_bytes / uncomp_bytes are in bytes of int32 rows.
struct CompInfo {
    uint64_t chunk_bytes = 0;
    uint64_t uncomp_bytes = 0;
    std::string comp_algo;
    uint64_t nvchunk = 1 << 16;
    uint64_t comp_bytes = (uint64_t)-1;
    int num_RLEs = 2;
    int num_deltas = 1;
    int use_bp = 1;
    std::vector<uint64_t> chunk_size_vec;
    std::vector<BlockInfo> blocks;
    std::shared_ptr<gx_column> column;

    uint64_t max_uncomp_chunk() const { return chunk_bytes; }
    uint64_t start_offset() const { return blocks.empty() ? (uint64_t)-1 : blocks[0].offset; }
    uint64_t end_offset() { return blocks.empty() ? (uint64_t)-1 : blocks[0].offset + get_comp_bytes(); }
    uint64_t get_comp_bytes() {
        if (comp_bytes != (uint64_t)-1) return comp_bytes;
        comp_bytes = 0;
        for (auto& b : blocks) comp_bytes += b.size;
        return comp_bytes;
    }
    uint64_t chunk_num() const {
        gx_column_info i;
        gx_check(gx_column_info_get(column.get(), &i));
        return i.n_chunks;
    }
};

// Ingest of one int32 column (prepare_compressed, core/apps.cuh:149-255):
// chunk, compress ("LZ4", "Cascaded" or "Uncompressed"), collect min/max and
// place the compressed bytes on the device (residency 1 = HBM, 2 = pinned
// host memory read zero-copy).
inline CompInfo prepare_compressed(const int32_t* host_col, uint64_t n_rows, uint64_t chunk_bytes,
                                   const std::string& comp_algo, int residency = 1, cudaStream_t stream = 0,
                                   uint64_t nvchunk = 1 << 16, uint32_t lz4_segments = 32) {
    gx_encode_opts o;
    gx_check(gx_encode_opts_default(&o));
    o.codec = comp_algo == "LZ4" ? GX_CODEC_LZ4 : comp_algo == "Cascaded" ? GX_CODEC_CASCADED : GX_CODEC_NONE;
    o.rows_per_chunk = (uint32_t)(chunk_bytes / 4);
    o.rows_per_block = (uint32_t)(nvchunk / 4);
    o.lz4_segments = lz4_segments;
    gx_column* c = nullptr;
    gx_check(gx_column_encode(host_col, n_rows, &o, &c));
    CompInfo info;
    info.column = std::shared_ptr<gx_column>(c, [](gx_column* p) { gx_column_free(p); });
    gx_check(gx_column_to_device(c, residency, (void*)stream));
    gx_column_info ci;
    gx_check(gx_column_info_get(c, &ci));
    info.chunk_bytes = chunk_bytes;
    info.uncomp_bytes = ci.uncomp_bytes;
    info.comp_algo = comp_algo;
    info.nvchunk = nvchunk;
    std::vector<gx_block_info> b(ci.n_blocks);
    gx_check(gx_column_blocks(c, b.data()));
    for (auto& x : b) info.blocks.push_back(BlockInfo{x.offset, x.size, x.payload, x.tuples});
    return info;
}

// ChunkDecompressor::step (core/comp.cuh:151-227): each step decompresses
// the next chunk into out_ptr (advanced by chunk_bytes when advance_out);
// skip_step moves past a pruned chunk.
class ChunkDecompressor {
   public:
    ChunkDecompressor(CompInfo& info, char* out_ptr, bool advance_out)
        : info_(info), out_ptr_(out_ptr), advance_out_(advance_out), last_produced(info.chunk_bytes) {}
    bool step(cudaStream_t stream, cudaEvent_t event = nullptr) {
        if (cur_ >= info_.chunk_num()) return false;
        gx_check(gx_decompress_chunk(info_.column.get(), cur_, out_ptr_, (void*)stream));
        if (event) cudaEventRecord(event, stream);
        advance();
        return true;
    }
    bool skip_step(cudaStream_t, cudaEvent_t = nullptr) {
        if (cur_ >= info_.chunk_num()) return false;
        advance();
        return true;
    }
    uint64_t last_produced;

   private:
    void advance() {
        if (advance_out_) out_ptr_ += info_.chunk_bytes;
        ++cur_;
    }
    CompInfo& info_;
    char* out_ptr_;
    bool advance_out_;
    uint64_t cur_ = 0;
};

// ---------------------------------------------------------- metadata.cuh
// MinMaxMeta<T> (core/metadata.cuh:110-221) for int32 columns: device and
// host min/max per chunk, filled at ingest.
template <typename T>
struct MinMaxMeta {
    static_assert(sizeof(T) == 4, "the B200 build stores int32 columns");
    MinMaxMeta() = default;
    explicit MinMaxMeta(const CompInfo& info) : chunk_num(info.chunk_num()), column(info.column) {
        mins_hst_v.resize(chunk_num);
        maxs_hst_v.resize(chunk_num);
        gx_check(gx_column_chunk_minmax(column.get(), (int32_t*)mins_hst_v.data(), (int32_t*)maxs_hst_v.data()));
        mins_hst = mins_hst_v.data();
        maxs_hst = maxs_hst_v.data();
        gx_check(cudaMalloc(&mins, chunk_num * sizeof(T)) == cudaSuccess ? GX_OK : GX_ERR_NOMEM);
        gx_check(cudaMalloc(&maxs, chunk_num * sizeof(T)) == cudaSuccess ? GX_OK : GX_ERR_NOMEM);
        owner = std::shared_ptr<void>(nullptr, [m = mins, x = maxs](void*) {
            cudaFree(m);
            cudaFree(x);
        });
        to_device();
        cudaDeviceSynchronize();
    }
    void to_device(cudaStream_t s = 0) {
        cudaMemcpyAsync(mins, mins_hst, chunk_num * sizeof(T), cudaMemcpyHostToDevice, s);
        cudaMemcpyAsync(maxs, maxs_hst, chunk_num * sizeof(T), cudaMemcpyHostToDevice, s);
    }
    void to_host(cudaStream_t = 0) {}  // host mirror is authoritative (filled at ingest)
    bool check_pred_host(uint64_t chunk_idx, T low, T high) const {
        return low <= maxs_hst[chunk_idx] && high >= mins_hst[chunk_idx];
    }
    __device__ void check_pred(uint64_t chunk_idx, uint16_t* out, T low, T high) const {
        if (low <= maxs[chunk_idx] && high >= mins[chunk_idx]) out[chunk_idx] = 1;
    }
    T* mins = nullptr;
    T* maxs = nullptr;
    T* mins_hst = nullptr;
    T* maxs_hst = nullptr;
    uint64_t chunk_num = 0;
    std::shared_ptr<gx_column> column;

   private:
    std::vector<T> mins_hst_v, maxs_hst_v;
    std::shared_ptr<void> owner;
};

// check_mmmeta (core/metadata.cuh:540-547): out[c] = 1 where chunk c overlaps [lo,hi].
template <typename T>
inline void check_mmmeta(const MinMaxMeta<T>& m, uint16_t* out, T lo, T hi, cudaStream_t s = 0) {
    gx_check(gx_check_minmax(m.column.get(), (int32_t)lo, (int32_t)hi, out, (void*)s));
}
// combine_and (core/metadata.cuh:632-636)
inline void combine_and(uint16_t* out, uint16_t* a, uint16_t* b, uint64_t num, cudaStream_t s = 0) {
    gx_check(gx_combine_and(out, a, b, num, (void*)s));
}

// MetaChecker (core/metadata.cuh:638-658): ANDs min/max predicates into one
// uint16 flag per chunk (1 = keep).
struct MetaChecker {
    MetaChecker(uint64_t /*block_num*/, uint64_t chunk_num, uint16_t* combined_check_dev, uint16_t* tmp_dev,
                cudaStream_t& stream)
        : chunk_num(chunk_num), combined(combined_check_dev), tmp(tmp_dev), stream(stream) {}
    template <typename T>
    void add_minmax(MinMaxMeta<T>& meta, T lo, T hi) {
        cudaMemsetAsync(tmp, 0, chunk_num * sizeof(uint16_t), stream);
        check_mmmeta(meta, tmp, lo, hi, stream);
        combine_and(combined, added ? combined : tmp, tmp, chunk_num, stream);
        added = true;
    }

   private:
    uint64_t chunk_num;
    uint16_t *combined, *tmp;
    cudaStream_t stream;
    bool added = false;
};

// --------------------------------------------------------- dev_structs.cuh
template <typename T>
struct DirectKey {
    __host__ __device__ T operator()(T* t) const { return *t; }
};

// PredInfo-style range predicate on a device column (core/dev_structs.cuh:22-26).
struct RangePred {
    const int32_t* col;
    int32_t lo, hi;
};

// HashMap (core/dev_structs.cuh:37-132).  BUILD_TUPLE is kept for source
// compatibility; the table stores an int32 payload per key (the build row id
// unless build() is given a payload column).
template <typename BUILD_TUPLE = int32_t, typename KEY_TYPE = uint64_t>
class HashMap {
   public:
    HashMap(uint64_t ht_size, BUILD_TUPLE* table = nullptr) : table(table) {
        gx_hashtable* h = nullptr;
        gx_check(gx_hashtable_create(ht_size, &h));
        owner = std::shared_ptr<gx_hashtable>(h, [](gx_hashtable* p) { gx_hashtable_free(p); });
        gx_check(gx_hashtable_view(h, &slots, &log2cap));
    }
    // hash_map_build_pred_other (core/join.cuh:107-135): insert row i (key
    // keys[i], payload payload[i] or i) when every predicate holds.
    void build(const int32_t* keys_dev, uint64_t n, const std::vector<RangePred>& preds = {},
               const int32_t* payload_dev = nullptr, cudaStream_t s = 0) {
        std::vector<gx_pred> p;
        for (auto& r : preds) p.push_back(gx_pred{r.col, r.lo, r.hi});
        gx_check(gx_hashtable_build(owner.get(), keys_dev, payload_dev, n, p.data(), (uint32_t)p.size(), (void*)s));
    }
    uint64_t filled(cudaStream_t s = 0) const {
        uint64_t n = 0;
        gx_check(gx_hashtable_count(owner.get(), &n, (void*)s));
        return n;
    }
    // HashMap::probe (core/dev_structs.cuh:105-113): payload of the matching
    // key, or (uint64_t)-1.
    template <typename BUILD_TUPLE_KEY = DirectKey<BUILD_TUPLE>>
    __device__ __forceinline__ uint64_t probe(KEY_TYPE key, BUILD_TUPLE_KEY = BUILD_TUPLE_KEY()) const {
        const int32_t k = (int32_t)key;
        if ((KEY_TYPE)k != key || k == GX_EMPTY_KEY) return (uint64_t)-1;
        const uint32_t mask = (1u << log2cap) - 1;
        uint32_t s = gx_hash32(k, log2cap);
        for (uint32_t i = 0; i <= mask; ++i) {
            const uint64_t e = __ldg((const unsigned long long*)slots + s);
            const int32_t ek = (int32_t)(uint32_t)e;
            if (ek == k) return (uint64_t)(uint32_t)(e >> 32);
            if (ek == GX_EMPTY_KEY) return (uint64_t)-1;
            s = (s + 1) & mask;
        }
        return (uint64_t)-1;
    }
    gx_hashtable* handle() const { return owner.get(); }
    BUILD_TUPLE* table;

   private:
    const uint64_t* slots = nullptr;
    uint32_t log2cap = 0;
    std::shared_ptr<gx_hashtable> owner;  // shared: by-value copies in kernels do not own
};

// HashAggregate (core/dev_structs.cuh:158-253) with SumAgg
// (usecases/ssb/queries/query_common.cuh:24-29): int64 key -> int64 sum.
class HashAggregate {
   public:
    explicit HashAggregate(uint64_t num_groups) {
        gx_groupby* g = nullptr;
        gx_check(gx_groupby_create(num_groups, &g));
        owner = std::shared_ptr<gx_groupby>(g, [](gx_groupby* p) { gx_groupby_free(p); });
        gx_check(gx_groupby_view(g, &keys, &sums, &log2cap));
    }
    // Returns false when the table is full (the caller decides; nothing waits).
    __device__ __forceinline__ bool add(int64_t key, int64_t val) const {
        const uint32_t mask = (1u << log2cap) - 1;
        uint32_t s = gx_hash64(key, log2cap);
        for (uint32_t i = 0; i <= mask; ++i) {
            unsigned long long old = atomicCAS((unsigned long long*)&keys[s], (unsigned long long)GX_EMPTY_GROUP,
                                               (unsigned long long)key);
            if (old == (unsigned long long)GX_EMPTY_GROUP || old == (unsigned long long)key) {
                atomicAdd((unsigned long long*)&sums[s], (unsigned long long)val);
                return true;
            }
            s = (s + 1) & mask;
        }
        return false;
    }
    // Groups present after the kernels on `s` finished: {key, sum} pairs.
    std::vector<std::pair<int64_t, int64_t>> read(uint64_t cap, cudaStream_t s = 0) const {
        std::vector<int64_t> k(cap), v(cap);
        uint64_t n = 0;
        gx_check(gx_groupby_read(owner.get(), k.data(), v.data(), cap, &n, (void*)s));
        std::vector<std::pair<int64_t, int64_t>> out;
        for (uint64_t i = 0; i < n; ++i) out.emplace_back(k[i], v[i]);
        return out;
    }
    gx_groupby* handle() const { return owner.get(); }

   private:
    int64_t* keys = nullptr;
    int64_t* sums = nullptr;
    uint32_t log2cap = 0;
    std::shared_ptr<gx_groupby> owner;
};

}  // namespace golap
