// golap_compat.cuh -- the reference's operator names and call forms over the
// gx C-ABI.
//
// A pipeline written against GOLAP's core/comp.cuh, core/metadata.cuh,
// core/join.cuh, core/agg.cuh and core/dev_structs.cuh (the worker loops of
// usecases/ssb/queries/01.hpp:350-424 and 03.hpp:408-547) compiles against
// this header with the same class names, constructors and kernel launches:
//   HashMap<BUILD_TUPLE, KEY_TYPE>(ht_size, table), __device__ insert/probe
//   hash_map_build_pred_other<<<...>>>(hm, n, key_fn, PredInfo...)
//   HashAggregate<GROUP_ATTR, AGG_TYPE>(num_groups, group_attr, agg_res),
//     __device__ add(group, val, agg_func) -> slot, wrote_group
//   MinMaxMeta<T>(chunk_num, max_tuples), init_chunk, to_host/to_device,
//     check_pred(_host); check_mmmeta<<<...>>>, combine_and<<<...>>>,
//     MetaChecker::add_minmax(std::any& or MinMaxMeta&, lo, hi)
//   ChunkDecompressor(chunk_bytes, in, out, advance_in, advance_out,
//     manager, chunk_size_vec) with step / skip_step; build_gpucomp_manager
//   Aggregate(in, out, num, reduction, init).execute(stream)
// Differences a caller sees:
//   * Columns are int32 (the measured schema).  CompInfo owns a gx_column
//     (the compressed chunk store, HBM or pinned host) made by
//     prepare_compressed() from a host column; the "manager" of a
//     ChunkDecompressor is bound to that CompInfo and decodes its chunks in
//     order, so the compressed input pointer of the reference constructor is
//     not read.
//   * HashMap is open addressing over {int32 key, int32 payload} slots: build
//     keys must be unique and != INT32_MIN, row ids < 2^31; probe returns the
//     inserted row id or (uint64_t)-1, as the reference's does.
//   * HashAggregate::add never waits without bound: a slot whose group is not
//     written within kAddSpinCap polls, or a full table, records an error
//     (read by check()) and returns (uint64_t)-1.
//   * Errors throw std::runtime_error with the library's message instead of
//     calling exit().
// Objects own their device memory; copies passed by value into kernels are
// non-owning views (the reference's is_orig pattern, done with shared_ptr).
#pragma once
#include <cuda_runtime.h>

#include <any>
#include <cstdint>
#include <memory>
#include <stdexcept>
#include <string>
#include <type_traits>
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
inline void cuda_check(cudaError_t e, const char* what) {
    if (e != cudaSuccess) throw std::runtime_error(std::string(what) + ": " + cudaGetErrorString(e));
}
template <typename T>
inline std::shared_ptr<T> device_alloc(uint64_t n) {
    T* p = nullptr;
    cuda_check(cudaMalloc(&p, (n ? n : 1) * sizeof(T)), "cudaMalloc");
    return std::shared_ptr<T>(p, [](T* q) { cudaFree(q); });
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

namespace detail {
inline gx_encode_opts ingest_opts(uint64_t chunk_bytes, const std::string& comp_algo, uint64_t nvchunk,
                                  uint32_t lz4_segments) {
    gx_encode_opts o;
    gx_check(gx_encode_opts_default(&o));
    o.codec = comp_algo == "LZ4" ? GX_CODEC_LZ4 : comp_algo == "Cascaded" ? GX_CODEC_CASCADED : GX_CODEC_NONE;
    o.rows_per_chunk = (uint32_t)(chunk_bytes / 4);
    o.rows_per_block = (uint32_t)(nvchunk / 4);
    o.lz4_segments = lz4_segments;
    return o;
}

// The CompInfo of an encoded column (owns it from here on).
inline CompInfo comp_info_of(gx_column* c, uint64_t n_rows, uint64_t chunk_bytes, const std::string& comp_algo,
                             uint64_t nvchunk) {
    CompInfo info;
    info.column = std::shared_ptr<gx_column>(c, [](gx_column* p) { gx_column_free(p); });
    gx_column_info ci;
    gx_check(gx_column_info_get(c, &ci));
    info.chunk_bytes = chunk_bytes;
    info.uncomp_bytes = ci.uncomp_bytes;
    info.comp_algo = comp_algo;
    info.nvchunk = nvchunk;
    std::vector<gx_block_info> b(ci.n_blocks);
    gx_check(gx_column_blocks(c, b.data()));
    for (auto& x : b) info.blocks.push_back(BlockInfo{x.offset, x.size, x.payload, x.tuples});
    for (uint64_t r = 0; r < n_rows; r += chunk_bytes / 4)
        info.chunk_size_vec.push_back(4 * std::min<uint64_t>(chunk_bytes / 4, n_rows - r));
    return info;
}
}  // namespace detail

// Ingest of one int32 column (prepare_compressed, core/apps.cuh:149-255):
// chunk, compress ("LZ4", "Cascaded" or "Uncompressed"), collect min/max and
// place the compressed bytes on the device (residency 1 = HBM, 2 = pinned
// host memory read zero-copy).
inline CompInfo prepare_compressed(const int32_t* host_col, uint64_t n_rows, uint64_t chunk_bytes,
                                   const std::string& comp_algo, int residency = 1, cudaStream_t stream = 0,
                                   uint64_t nvchunk = 1 << 16, uint32_t lz4_segments = 32) {
    const gx_encode_opts o = detail::ingest_opts(chunk_bytes, comp_algo, nvchunk, lz4_segments);
    gx_column* c = nullptr;
    gx_check(gx_column_encode(host_col, n_rows, &o, &c));
    CompInfo info = detail::comp_info_of(c, n_rows, chunk_bytes, comp_algo, nvchunk);
    gx_check(gx_column_to_device(c, residency, (void*)stream));
    return info;
}

// The same for a column already in device memory (the reference's
// prepare_compressed over a device-resident golap::Column): encoded on the
// GPU, in HBM on return.  "LZ4" writes every block as one literal run.
inline CompInfo prepare_compressed_device(const int32_t* dev_col, uint64_t n_rows, uint64_t chunk_bytes,
                                          const std::string& comp_algo, cudaStream_t stream = 0,
                                          uint64_t nvchunk = 1 << 16, uint32_t lz4_segments = 32) {
    gx_encode_opts o = detail::ingest_opts(chunk_bytes, comp_algo, nvchunk, lz4_segments);
    o.lz4_min_match = GX_LZ4_LITERAL;
    gx_column* c = nullptr;
    gx_check(gx_column_encode_device(dev_col, n_rows, &o, &c, (void*)stream));
    return detail::comp_info_of(c, n_rows, chunk_bytes, comp_algo, nvchunk);
}

// The decoder of one compressed column: what build_gpucomp_manager returns
// (core/comp.cuh:230-256).  Bound to the CompInfo whose chunks it decodes.
struct CompManager {
    explicit CompManager(CompInfo& info) : info(&info) {}
    CompInfo* info;
};
inline std::shared_ptr<CompManager> build_gpucomp_manager(CompInfo& info) {
    return std::make_shared<CompManager>(info);
}

// ChunkDecompressor (core/comp.cuh:151-227): each step decodes the next chunk
// of the manager's column into out_ptr (advanced by the chunk's bytes when
// advance_out); skip_step moves past a pruned chunk.  chunk_bytes ==
// (uint64_t)-1 takes the chunk sizes from chunk_size_vec, as the reference.
class ChunkDecompressor {
   public:
    ChunkDecompressor(const ChunkDecompressor&) = delete;
    ChunkDecompressor(ChunkDecompressor&&) = default;
    ChunkDecompressor(uint64_t chunk_bytes, char* in_ptr, char* out_ptr, bool advance_in, bool advance_out,
                      CompManager& comp_manager, std::vector<uint64_t>& chunk_size_vec)
        : info_(comp_manager.info), sizes_(&chunk_size_vec), chunk_bytes_(chunk_bytes), in_ptr_(in_ptr),
          out_ptr_(out_ptr), advance_in_(advance_in), advance_out_(advance_out) {
        last_produced = chunk_bytes;
    }
    // The earlier short form: decode the CompInfo's chunks into out_ptr.
    ChunkDecompressor(CompInfo& info, char* out_ptr, bool advance_out)
        : info_(&info), sizes_(&info.chunk_size_vec), chunk_bytes_(info.chunk_bytes), out_ptr_(out_ptr),
          advance_out_(advance_out) {
        last_produced = info.chunk_bytes;
    }
    bool step(cudaStream_t stream, cudaEvent_t event = nullptr) {
        if (cur_ >= info_->chunk_num()) return false;
        if (chunk_bytes_ == (uint64_t)-1) last_produced = (*sizes_)[cur_];
        gx_check(gx_decompress_chunk(info_->column.get(), cur_, out_ptr_, (void*)stream));
        if (event) cuda_check(cudaEventRecord(event, stream), "cudaEventRecord");
        advance();
        return true;
    }
    bool skip_step(cudaStream_t, cudaEvent_t = nullptr) {
        if (cur_ >= info_->chunk_num()) return false;
        advance();
        return true;
    }
    uint64_t last_produced = 0;

   private:
    void advance() {
        if (advance_out_) out_ptr_ += chunk_bytes_ != (uint64_t)-1 ? chunk_bytes_ : (*sizes_)[cur_];
        ++cur_;
    }
    CompInfo* info_;
    std::vector<uint64_t>* sizes_;
    uint64_t chunk_bytes_;
    char* in_ptr_ = nullptr;
    char* out_ptr_;
    bool advance_in_ = false, advance_out_;
    uint64_t cur_ = 0;
};

// ---------------------------------------------------------- metadata.cuh
// MinMaxMeta<T> (core/metadata.cuh:110-221) for int32 columns: device and
// pinned host min/max per chunk.  Either filled at ingest (from a CompInfo)
// or, as in the reference, sized with (chunk_num, max_tuples) and filled
// chunk by chunk with init_chunk (gx_minmax_reduce on the device column).
template <typename T>
struct MinMaxMeta {
    static_assert(std::is_same<T, int32_t>::value, "the B200 build stores int32 columns");
    MinMaxMeta() = default;
    MinMaxMeta(uint64_t chunk_num, uint64_t /*max_tuples_in_chunk*/) : chunk_num(chunk_num) { alloc(); }
    explicit MinMaxMeta(const CompInfo& info) : chunk_num(info.chunk_num()), column(info.column) {
        alloc();
        gx_check(gx_column_chunk_minmax(column.get(), (int32_t*)mins_hst, (int32_t*)maxs_hst));
        to_device();
        cuda_check(cudaStreamSynchronize(0), "cudaStreamSynchronize");
    }
    // min/max of num_items rows at data (device) into chunk chunk_idx
    void init_chunk(uint64_t chunk_idx, T* data, uint64_t num_items, cudaStream_t stream = 0) {
        gx_check(gx_minmax_reduce((const int32_t*)data, num_items, range_ + 2 * chunk_idx, (void*)stream));
        cuda_check(cudaMemcpyAsync(mins + chunk_idx, range_ + 2 * chunk_idx, sizeof(T), cudaMemcpyDeviceToDevice,
                                   stream), "cudaMemcpyAsync");
        cuda_check(cudaMemcpyAsync(maxs + chunk_idx, range_ + 2 * chunk_idx + 1, sizeof(T), cudaMemcpyDeviceToDevice,
                                   stream), "cudaMemcpyAsync");
    }
    void to_device(cudaStream_t s = 0) {
        cuda_check(cudaMemcpyAsync(mins, mins_hst, chunk_num * sizeof(T), cudaMemcpyDefault, s), "cudaMemcpyAsync");
        cuda_check(cudaMemcpyAsync(maxs, maxs_hst, chunk_num * sizeof(T), cudaMemcpyDefault, s), "cudaMemcpyAsync");
    }
    void to_host(cudaStream_t s = 0) {
        cuda_check(cudaMemcpyAsync(mins_hst, mins, chunk_num * sizeof(T), cudaMemcpyDefault, s), "cudaMemcpyAsync");
        cuda_check(cudaMemcpyAsync(maxs_hst, maxs, chunk_num * sizeof(T), cudaMemcpyDefault, s), "cudaMemcpyAsync");
    }
    void free_temp() {}
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
    void alloc() {
        auto d = device_alloc<T>(4 * chunk_num);  // mins | maxs | per-chunk {min, max} of init_chunk
        mins = d.get();
        maxs = mins + chunk_num;
        range_ = (int32_t*)(maxs + chunk_num);
        T* h = nullptr;
        cuda_check(cudaMallocHost(&h, 2 * (chunk_num ? chunk_num : 1) * sizeof(T)), "cudaMallocHost");
        mins_hst = h;
        maxs_hst = h + chunk_num;
        std::shared_ptr<T> hh(h, [](T* p) { cudaFreeHost(p); });
        owner_ = std::make_shared<std::pair<std::shared_ptr<T>, std::shared_ptr<T>>>(d, hh);
    }
    int32_t* range_ = nullptr;
    std::shared_ptr<void> owner_;  // shared: by-value copies in kernels do not own
};

// check_mmmeta (core/metadata.cuh:540-547): out[c] = 1 where chunk c overlaps [low, high].
template <typename T>
__global__ void check_mmmeta(MinMaxMeta<T> mmmeta, uint16_t* out, T low, T high) {
    for (uint64_t idx = blockDim.x * (uint64_t)blockIdx.x + threadIdx.x; idx < mmmeta.chunk_num;
         idx += (uint64_t)blockDim.x * gridDim.x)
        mmmeta.check_pred(idx, out, low, high);
}
// combine_and / combine_or (core/metadata.cuh:627-636)
__global__ static void combine_and(uint16_t* out, uint16_t* out_a, uint16_t* out_b, uint64_t num) {
    for (uint64_t idx = blockDim.x * (uint64_t)blockIdx.x + threadIdx.x; idx < num; idx += (uint64_t)blockDim.x * gridDim.x)
        out[idx] = out_a[idx] & out_b[idx];
}
__global__ static void combine_or(uint16_t* out, uint16_t* out_a, uint16_t* out_b, uint64_t num) {
    for (uint64_t idx = blockDim.x * (uint64_t)blockIdx.x + threadIdx.x; idx < num; idx += (uint64_t)blockDim.x * gridDim.x)
        out[idx] = out_a[idx] | out_b[idx];
}
// The same through the library (one launch each; flags of a column's chunks).
template <typename T>
inline void check_mmmeta_async(const MinMaxMeta<T>& m, uint16_t* out, T lo, T hi, cudaStream_t s = 0) {
    gx_check(gx_check_minmax(m.column.get(), (int32_t)lo, (int32_t)hi, out, (void*)s));
}
inline void combine_and_async(uint16_t* out, uint16_t* a, uint16_t* b, uint64_t num, cudaStream_t s = 0) {
    gx_check(gx_combine_and(out, a, b, num, (void*)s));
}

// MetaChecker (core/metadata.cuh:638-658): ANDs min/max predicates into one
// uint16 flag per chunk (1 = keep); tmp is zeroed after every predicate.
struct MetaChecker {
    MetaChecker(uint64_t block_num, uint64_t chunk_num, uint16_t* combined_check_dev, uint16_t* tmp_dev,
                cudaStream_t& stream)
        : block_num(block_num ? block_num : 1), chunk_num(chunk_num), combined(combined_check_dev), tmp(tmp_dev),
          stream(stream) {
        cuda_check(cudaMemsetAsync(tmp, 0, chunk_num * sizeof(uint16_t), stream), "cudaMemsetAsync");
    }
    template <typename T>
    void add_minmax(MinMaxMeta<T>& meta, T lo, T hi) {
        check_mmmeta<<<(unsigned)block_num, 512, 0, stream>>>(meta, tmp, lo, hi);
        combine_and<<<(unsigned)block_num, 512, 0, stream>>>(combined, added ? combined : tmp, tmp, chunk_num);
        cuda_check(cudaMemsetAsync(tmp, 0, chunk_num * sizeof(uint16_t), stream), "cudaMemsetAsync");
        added = true;
    }
    template <typename T>
    void add_minmax(std::any& meta, T lo, T hi) {
        add_minmax(std::any_cast<MinMaxMeta<T>&>(meta), lo, hi);
    }

   private:
    uint64_t block_num, chunk_num;
    uint16_t *combined, *tmp;
    cudaStream_t stream;
    bool added = false;
};

// --------------------------------------------------------- dev_structs.cuh
template <typename T>
struct DirectKey {
    __host__ __device__ T operator()(T* t) const { return *t; }
};
// core/dev_structs.cuh:22-35
template <typename T, typename PREDICATE>
struct PredInfo {
    T* col;
    PREDICATE pred;
};
template <typename T, T C>
struct ConstPred {
    __host__ __device__ bool operator()(T* ptr) const { return *ptr == C; }
};
template <typename T>
struct RangePredFn {
    T lo, hi;
    __host__ __device__ bool operator()(T* ptr) const { return *ptr >= lo && *ptr <= hi; }
};

// Range predicate on a device column for the bulk build() below.
struct RangePred {
    const int32_t* col;
    int32_t lo, hi;
};

// HashMap (core/dev_structs.cuh:37-132).  Construction allocates an empty
// table sized for ht_size entries; insert (device) and probe (device) have
// the reference's signatures; build() is the library's bulk filtered build.
template <typename BUILD_TUPLE = int32_t, typename KEY_TYPE = uint64_t>
class HashMap {
   public:
    HashMap(uint64_t ht_size, BUILD_TUPLE* table = nullptr) : ht_size(ht_size), table(table) {
        gx_hashtable* h = nullptr;
        gx_check(gx_hashtable_create(ht_size, &h));
        owner = std::shared_ptr<gx_hashtable>(h, [](gx_hashtable* p) { gx_hashtable_free(p); });
        gx_check(gx_hashtable_view2(h, &slots, &log2cap, &filled));
        gx_check(gx_hashtable_clear(h, nullptr));
        cuda_check(cudaStreamSynchronize(0), "cudaStreamSynchronize");
    }
    // HashMap::insert (core/dev_structs.cuh:89-98): row rid of `table` under key.
    __device__ __forceinline__ void insert(uint64_t rid, KEY_TYPE key) const {
        const int32_t k = (int32_t)key;
        unsigned long long* cnt = (unsigned long long*)filled;
        if ((KEY_TYPE)k != key || k == GX_EMPTY_KEY || rid > 0x7FFFFFFFull) {
            atomicAdd(cnt + 2, 1ull);
            return;
        }
        const unsigned long long e = ((unsigned long long)rid << 32) | (uint32_t)k;
        const unsigned long long empty = (unsigned long long)(uint32_t)GX_EMPTY_KEY;
        const uint32_t mask = (1u << log2cap) - 1;
        uint32_t s = gx_hash32(k, log2cap);
        for (uint32_t i = 0; i <= mask; ++i) {
            const unsigned long long old = atomicCAS((unsigned long long*)slots + s, empty, e);
            if (old == empty) {
                atomicAdd(cnt, 1ull);
                return;
            }
            if ((int32_t)(uint32_t)old == k) {
                atomicAdd(cnt + 1, 1ull);
                return;
            }
            s = (s + 1) & mask;
        }
        atomicAdd(cnt + 2, 1ull);
    }
    // hash_map_build_pred_other through the library: insert row i (key
    // keys[i], payload payload[i] or i) when every predicate holds.
    void build(const int32_t* keys_dev, uint64_t n, const std::vector<RangePred>& preds = {},
               const int32_t* payload_dev = nullptr, cudaStream_t s = 0) {
        std::vector<gx_pred> p;
        for (auto& r : preds) p.push_back(gx_pred{r.col, r.lo, r.hi});
        gx_check(gx_hashtable_build(owner.get(), keys_dev, payload_dev, n, p.data(), (uint32_t)p.size(), (void*)s));
    }
    // Inserted entries (synchronises s; fails on rows that found no slot).
    uint64_t num_filled(cudaStream_t s = 0) const {
        uint64_t n = 0;
        gx_check(gx_hashtable_count(owner.get(), &n, (void*)s));
        return n;
    }
    // HashMap::probe (core/dev_structs.cuh:105-113): the inserted row id of
    // the matching key, or (uint64_t)-1.
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
    uint64_t ht_size;
    BUILD_TUPLE* table;
    uint64_t* filled = nullptr;  // device counters: inserted, duplicate keys, rows not inserted

   private:
    uint64_t* slots = nullptr;
    uint32_t log2cap = 0;
    std::shared_ptr<gx_hashtable> owner;  // shared: by-value copies in kernels do not own
};

// ---------------------------------------------------------------- join.cuh
// hash_map_build_pred_other (core/join.cuh:107-135): thread r inserts row r
// of hashmap.table under build_key(&table[r]) when every PredInfo holds.
template <typename BUILD_TUPLE, typename BUILD_KEY>
__device__ inline void hash_map_build_pred_dev(HashMap<BUILD_TUPLE, uint64_t>& hashmap, uint64_t num_tuples,
                                               BUILD_KEY build_key) {
    const uint64_t r_id = blockDim.x * (uint64_t)blockIdx.x + threadIdx.x;
    if (r_id >= num_tuples) return;
    hashmap.insert(r_id, build_key(&hashmap.table[r_id]));
}
template <typename BUILD_TUPLE, typename BUILD_KEY, typename FIRST, typename... REST>
__device__ inline void hash_map_build_pred_dev(HashMap<BUILD_TUPLE, uint64_t>& hashmap, uint64_t num_tuples,
                                               BUILD_KEY build_key, FIRST pred_info, REST... rest) {
    const uint64_t r_id = blockDim.x * (uint64_t)blockIdx.x + threadIdx.x;
    if (r_id >= num_tuples) return;
    if (!pred_info.pred(&pred_info.col[r_id])) return;
    hash_map_build_pred_dev(hashmap, num_tuples, build_key, rest...);
}
template <typename BUILD_TUPLE, typename BUILD_KEY, typename... ALL>
__global__ void hash_map_build_pred_other(HashMap<BUILD_TUPLE, uint64_t> hashmap, uint64_t num_tuples,
                                          BUILD_KEY build_key, ALL... all) {
    hash_map_build_pred_dev(hashmap, num_tuples, build_key, all...);
}

// HashAggregate (core/dev_structs.cuh:158-253): groups of type GROUP_ATTR
// (with hash() and operator==) in num_groups slots of the caller's
// group_attr / agg_res arrays (device); add() claims or finds the group's
// slot by linear probing and applies agg_func(&agg_res[slot], val).
template <typename GROUP_ATTR, typename AGG_TYPE>
class HashAggregate {
   public:
    static constexpr uint32_t kAddSpinCap = 1u << 22;
    HashAggregate(uint64_t num_groups, GROUP_ATTR* group_attr, AGG_TYPE* agg_res)
        : num_groups(num_groups), group_attr(group_attr), agg_res(agg_res) {
        auto mem = device_alloc<uint32_t>(2 * num_groups + 4);  // reserved | wrote_group | added (u64) | error
        reserved = mem.get();
        wrote_group = reserved + num_groups;
        added = (uint64_t*)(wrote_group + num_groups + (num_groups & 1));
        error = (int*)(added + 1);
        cuda_check(cudaMemset(reserved, 0, (2 * num_groups + 4) * sizeof(uint32_t)), "cudaMemset");
        owner = mem;
    }
    template <typename AGG_FUNC>
    __device__ inline uint64_t add(GROUP_ATTR group, AGG_TYPE agg_val, AGG_FUNC agg_func) const {
        uint64_t slot = group.hash() % num_groups;
        for (uint64_t probe = 0; probe < num_groups; ++probe) {
            const uint32_t old = atomicCAS(&reserved[slot], 0u, 1u);
            if (old == 0u) {  // the group's representative: write it, then publish
                group_attr[slot] = group;
                __threadfence();
                atomicExch(&wrote_group[slot], 1u);
                return apply(slot, agg_val, agg_func);
            }
            uint32_t spin = 0;
            while (((volatile uint32_t*)wrote_group)[slot] == 0u) {
                if (++spin > kAddSpinCap) {
                    atomicCAS(error, 0, (int)GX_ERR_TIMEOUT);
                    return (uint64_t)-1;
                }
            }
            __threadfence();
            if (group_attr[slot] == group) return apply(slot, agg_val, agg_func);
            slot = (slot + 1) % num_groups;
        }
        atomicCAS(error, 0, (int)GX_ERR_CAPACITY);
        return (uint64_t)-1;
    }
    // Status of the adds so far (synchronises the device).
    void check() const {
        int e = 0;
        cuda_check(cudaMemcpy(&e, error, sizeof(int), cudaMemcpyDeviceToHost), "cudaMemcpy");
        if (e) throw std::runtime_error(std::string("HashAggregate: ") + gx_status_str(e));
    }
    uint32_t* reserved = nullptr;
    uint32_t* wrote_group = nullptr;
    uint64_t* added = nullptr;
    uint64_t num_groups;
    GROUP_ATTR* group_attr;
    AGG_TYPE* agg_res;

   private:
    template <typename AGG_FUNC>
    __device__ inline uint64_t apply(uint64_t slot, AGG_TYPE v, AGG_FUNC f) const {
        atomicAdd((unsigned long long*)added, 1ull);
        f(&agg_res[slot], v);
        return slot;
    }
    int* error = nullptr;
    std::shared_ptr<uint32_t> owner;  // shared: by-value copies in kernels do not own
};

// ------------------------------------------------------------------ agg.cuh
// Aggregate (core/agg.cuh:16-36): reduction of num IN_TYPE values into *out
// with a binary functor and an init value, as two launches (per-CTA partials,
// then one CTA over the partials) over scratch allocated at construction.
template <typename IN_TYPE, typename RESULT_TYPE, typename REDUCTION, int NT>
__global__ void aggregate_partial(const IN_TYPE* in, uint64_t num, REDUCTION red, IN_TYPE init, IN_TYPE* part) {
    __shared__ IN_TYPE s[NT];
    IN_TYPE acc = init;
    for (uint64_t i = blockIdx.x * (uint64_t)NT + threadIdx.x; i < num; i += (uint64_t)gridDim.x * NT)
        acc = red(acc, in[i]);
    s[threadIdx.x] = acc;
    __syncthreads();
    for (int w = NT / 2; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w) s[threadIdx.x] = red(s[threadIdx.x], s[threadIdx.x + w]);
        __syncthreads();
    }
    if (threadIdx.x == 0) part[blockIdx.x] = s[0];
}
template <typename IN_TYPE, typename RESULT_TYPE, typename REDUCTION, int NT>
__global__ void aggregate_final(const IN_TYPE* part, uint32_t n, REDUCTION red, IN_TYPE init, RESULT_TYPE* out) {
    __shared__ IN_TYPE s[NT];
    IN_TYPE acc = init;
    for (uint32_t i = threadIdx.x; i < n; i += NT) acc = red(acc, part[i]);
    s[threadIdx.x] = acc;
    __syncthreads();
    for (int w = NT / 2; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w) s[threadIdx.x] = red(s[threadIdx.x], s[threadIdx.x + w]);
        __syncthreads();
    }
    if (threadIdx.x == 0) *out = (RESULT_TYPE)s[0];
}
template <typename IN_TYPE, typename RESULT_TYPE, typename REDUCTION>
class Aggregate {
   public:
    static constexpr int kNT = 256;
    static constexpr uint32_t kParts = 512;
    Aggregate(IN_TYPE* in, RESULT_TYPE* out, uint32_t num, REDUCTION reduction, IN_TYPE init)
        : in(in), out(out), num(num), reduction(reduction), init(init), part(device_alloc<IN_TYPE>(kParts)) {}
    void execute(cudaStream_t stream = 0) {
        const uint32_t blocks = (uint32_t)std::max<uint64_t>(1, std::min<uint64_t>(kParts, (num + kNT - 1) / kNT));
        aggregate_partial<IN_TYPE, RESULT_TYPE, REDUCTION, kNT><<<blocks, kNT, 0, stream>>>(in, num, reduction, init,
                                                                                          part.get());
        aggregate_final<IN_TYPE, RESULT_TYPE, REDUCTION, kNT><<<1, kNT, 0, stream>>>(part.get(), blocks, reduction,
                                                                                   init, out);
        cuda_check(cudaGetLastError(), "Aggregate::execute");
    }

   private:
    IN_TYPE* in;
    RESULT_TYPE* out;
    uint32_t num;
    REDUCTION reduction;
    IN_TYPE init;
    std::shared_ptr<IN_TYPE> part;
};

// Int64 group table of the library (gx_groupby: the fused scan's grouped
// aggregate) for kernels that add int64 keys directly.
class GroupTable {
   public:
    explicit GroupTable(uint64_t num_groups) {
        gx_groupby* g = nullptr;
        gx_check(gx_groupby_create(num_groups, &g));
        owner = std::shared_ptr<gx_groupby>(g, [](gx_groupby* p) { gx_groupby_free(p); });
        gx_check(gx_groupby_view(g, &keys, &sums, &log2cap));
        gx_check(gx_groupby_reset(g, nullptr));
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
