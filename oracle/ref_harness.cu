// ref_harness.cu -- the reference's own CPU code, compiled from its sources
// (GOLAP, header-only) into oracle/_ref/libgolapref.so.  Test
// infrastructure only: tests/ use it to pin the oracle restatement, and
// bench.py's reference arm times it.  Nothing in the product links it.
//
// Compiled from the reference tree (include paths set by oracle/Makefile):
//   core/util.hpp          uniform_int LCG, SliceSeq, Timer, Log
//   core/mem.hpp, table.hpp, types.hpp   column containers (MemBase)
//   usecases/ssb/data/SSB_def.hpp, SSB_helper.hpp   the seeded SSB generator
//   core/dev_structs.cuh   DirectKey
//   core/host_structs.hpp  HostHashMap, HostHashAggregate
//   core/core.hpp, comp_cpu.hpp   LZ4CPUManager (system liblz4 1.9.4)
// The query loop bodies of query1inmem (usecases/ssb/queries/01inmem.hpp:
// 83-130) and query3_inmem (usecases/ssb/queries/03inmem.hpp:120-200) are
// restated below on top of those reference structures: their headers include
// usecases/ssb/ssb.hpp, which pulls in every GPU query and therefore nvCOMP,
// which is not available here.  Group struct Q3NATION_GROUP
// (usecases/ssb/queries/03.cuh:29-59) is restated for the same reason.
#include <atomic>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <thread>
#include <unordered_map>
#include <vector>

#include "helper_cuda.h"
#include "util.hpp"
#include "mem.hpp"
#include "types.hpp"
#include "table.hpp"
#include "dev_structs.cuh"
#include "host_structs.hpp"
#include "core.hpp"
#include "comp_cpu.hpp"
#include "data/SSB_def.hpp"

// Plain heap memory with the golap::HostMem interface (core/mem.hpp:226-307)
// so the reference generator runs without a CUDA driver (HostMem allocates
// pinned memory through cudaMallocHost).
class HarnessMem : public golap::MemBase {
   public:
    HarnessMem(const HarnessMem&) = delete;
    HarnessMem() : golap::MemBase(0, 1, 0) {}
    template <typename T>
    HarnessMem(golap::Tag<T>, uint64_t num, uint64_t alloc_unit = 1, uint64_t alignment = 0)
        : golap::MemBase(0, alloc_unit ? alloc_unit : 1, alignment) {
        resize(sizeof(T), num, false);
    }
    ~HarnessMem() { std::free(real_data_); }
    void set(int val, cudaStream_t = 0) {
        if (bytes) std::memset(data, val, bytes);
    }

   protected:
    void resize(uint64_t type_size, uint64_t num, bool keep = false) {
        uint64_t nb = util::div_ceil(type_size * num, alloc_unit) * alloc_unit;
        void* p = nb ? std::calloc(1, nb + 64) : nullptr;
        if (keep && bytes && p) std::memcpy(p, data, bytes < nb ? bytes : nb);
        std::free(real_data_);
        real_data_ = p;
        data = p;
        bytes = nb;
    }
    void* real_data_ = nullptr;
};

using Tables = SSB_Tables_col<HarnessMem>;

// Restatement of Q3NATION_GROUP (usecases/ssb/queries/03.cuh:29-59).
struct HGroup {
    util::Padded<char[16]> c_nation;
    util::Padded<char[16]> s_nation;
    uint16_t d_year;
    uint64_t hash() const {
        uint64_t h = (*(uint32_t*)c_nation.d);
        h <<= 32;
        h |= (*(uint32_t*)s_nation.d);
        h ^= d_year;
        return h;
    }
    bool operator==(const HGroup& o) const {
        for (int i = 0; i < 16; ++i) {
            if (c_nation.d[i] != o.c_nation.d[i]) return false;
            if (c_nation.d[i] == '\0') break;
        }
        for (int i = 0; i < 16; ++i) {
            if (s_nation.d[i] != o.s_nation.d[i]) return false;
            if (s_nation.d[i] == '\0') break;
        }
        return d_year == o.d_year;
    }
};
struct HGroupHash {
    std::size_t operator()(const HGroup& g) const { return g.hash(); }
};
struct HostSumAtomic {
    void operator()(std::atomic<uint64_t>* agg, uint64_t v) { agg->fetch_add(v, std::memory_order_relaxed); }
};

static bool region_is(const util::Padded<char[13]>& r, const char* name) {
    return std::strncmp(r.d, name, 13) == 0;
}

enum class Q1V { Q11, Q12, Q13 };

// query1inmem body (01inmem.hpp:83-130) over the reference tables.
template <Q1V V>
static uint64_t run_q1(Tables& t, uint32_t workers, uint8_t dlo, uint8_t dhi, uint8_t qlo, uint8_t qhi) {
    golap::HostHashMap hash_map(t.date.num_tuples, t.date.col<Date::KEY>().data());
    std::atomic<uint64_t> agg{0};
    util::SliceSeq ds{t.date.num_tuples, workers}, ls{t.lineorder.num_tuples, workers};
    std::vector<std::tuple<uint64_t, uint64_t>> dsl(workers), lsl(workers);
    for (auto& [s, e] : dsl) ds.get(s, e);
    for (auto& [s, e] : lsl) ls.get(s, e);
    std::vector<std::thread> th;
    for (uint32_t w = 0; w < workers; ++w)
        th.emplace_back([&, w] {
            auto [s, e] = dsl[w];
            for (uint64_t i = s; i < e; ++i) {
                bool ok = true;
                if constexpr (V == Q1V::Q11) ok = t.date.col<Date::YEAR>().data()[i] == 1993;
                if constexpr (V == Q1V::Q12) ok = t.date.col<Date::YEARMONTHNUM>().data()[i] == 199401;
                if constexpr (V == Q1V::Q13)
                    ok = t.date.col<Date::WEEKNUMINYEAR>().data()[i] == 6 && t.date.col<Date::YEAR>().data()[i] == 1994;
                if (ok) hash_map.insert(i, t.date.col<Date::KEY>().data()[i]);
            }
        });
    for (auto& x : th) x.join();
    th.clear();
    for (uint32_t w = 0; w < workers; ++w)
        th.emplace_back([&, w] {
            auto [s, e] = lsl[w];
            uint64_t part = 0;
            auto* disc = t.lineorder.col<Lineorder::DISCOUNT>().data();
            auto* qty = t.lineorder.col<Lineorder::QUANTITY>().data();
            auto* ext = t.lineorder.col<Lineorder::EXTENDEDPRICE>().data();
            auto* od = t.lineorder.col<Lineorder::ORDERDATE>().data();
            for (uint64_t i = s; i < e; ++i) {
                if (disc[i] < dlo || disc[i] > dhi || qty[i] < qlo || qty[i] > qhi) continue;
                if (hash_map.probe(od[i]) == (uint64_t)-1) continue;
                part += ext[i] * disc[i];
            }
            agg.fetch_add(part, std::memory_order_relaxed);
        });
    for (auto& x : th) x.join();
    return agg.load();
}

// query3_inmem body for Q3.1 (03inmem.hpp:120-200; predicates of
// query3_1inmem :229-236: region ASIA on both sides, DATE_9297).
static void run_q31(Tables& t, uint32_t workers, uint64_t* n_groups, uint64_t* total) {
    golap::HostHashMap ch(t.customer.num_tuples, t.customer.col<Customer::KEY>().data());
    golap::HostHashMap sh(t.supplier.num_tuples, t.supplier.col<Supplier::KEY>().data());
    golap::HostHashMap dh(t.date.num_tuples, t.date.col<Date::KEY>().data());
    const uint64_t num_groups = 800;
    std::vector<HGroup> groups(num_groups);
    auto aggs = std::make_unique<std::atomic<uint64_t>[]>(num_groups);
    for (uint64_t i = 0; i < num_groups; ++i) aggs[i] = 0;
    golap::HostHashAggregate<HGroup, std::atomic<uint64_t>> ha(num_groups, groups.data(), aggs.get());
    util::SliceSeq cs{t.customer.num_tuples, workers}, ss{t.supplier.num_tuples, workers},
        dss{t.date.num_tuples, workers}, ls{t.lineorder.num_tuples, workers};
    std::vector<std::tuple<uint64_t, uint64_t>> csl(workers), ssl(workers), dsl(workers), lsl(workers);
    for (auto& [s, e] : csl) cs.get(s, e);
    for (auto& [s, e] : ssl) ss.get(s, e);
    for (auto& [s, e] : dsl) dss.get(s, e);
    for (auto& [s, e] : lsl) ls.get(s, e);
    std::vector<std::thread> th;
    for (uint32_t w = 0; w < workers; ++w)
        th.emplace_back([&, w] {
            auto [s, e] = csl[w];
            for (uint64_t i = s; i < e; ++i)
                if (region_is(t.customer.col<Customer::REGION>().data()[i], "ASIA"))
                    ch.insert(i, t.customer.col<Customer::KEY>().data()[i]);
            std::tie(s, e) = ssl[w];
            for (uint64_t i = s; i < e; ++i)
                if (region_is(t.supplier.col<Supplier::REGION>().data()[i], "ASIA"))
                    sh.insert(i, t.supplier.col<Supplier::KEY>().data()[i]);
            std::tie(s, e) = dsl[w];
            for (uint64_t i = s; i < e; ++i) {
                auto y = t.date.col<Date::YEAR>().data()[i];
                if (y >= 1992 && y <= 1997) dh.insert(i, t.date.col<Date::KEY>().data()[i]);
            }
        });
    for (auto& x : th) x.join();
    th.clear();
    for (uint32_t w = 0; w < workers; ++w)
        th.emplace_back([&, w] {
            auto [s, e] = lsl[w];
            std::unordered_map<HGroup, uint64_t, HGroupHash> local;
            for (uint64_t i = s; i < e; ++i) {
                uint64_t cm = ch.probe(t.lineorder.col<Lineorder::CUSTKEY>().data()[i]);
                if (cm == (uint64_t)-1) continue;
                uint64_t sm = sh.probe(t.lineorder.col<Lineorder::SUPPKEY>().data()[i]);
                if (sm == (uint64_t)-1) continue;
                uint64_t dm = dh.probe(t.lineorder.col<Lineorder::ORDERDATE>().data()[i]);
                if (dm == (uint64_t)-1) continue;
                HGroup g{t.supplier.col<Supplier::NATION>().data()[sm], t.customer.col<Customer::NATION>().data()[cm],
                         t.date.col<Date::YEAR>().data()[dm]};
                local[g] += t.lineorder.col<Lineorder::REVENUE>().data()[i];
            }
            for (auto& [k, v] : local) ha.add(k, v, HostSumAtomic());
        });
    for (auto& x : th) x.join();
    uint64_t ng = 0, sum = 0;
    for (uint64_t i = 0; i < num_groups; ++i) {
        if (ha.wrote_group[i] == 0) continue;
        ++ng;
        sum += aggs[i];
    }
    *n_groups = ng;
    *total = sum;
}

static int nation_index(const util::Padded<char[16]>& n) {
    int i = 0;
    for (auto& kv : NATION) {
        if (std::strncmp(kv.first.c_str(), n.d, 16) == 0) return i;
        ++i;
    }
    return -1;
}

extern "C" {

// Generates the SSB tables with the reference generator (scale factor sf,
// seed 0xBEE5BEE5) and runs Q1.1, Q1.2, Q1.3 and Q3.1.
// out = {q11, q12, q13, q31_groups, q31_sum, lineorder_rows}.
__attribute__((visibility("default"))) int ref_ssb_golden(uint32_t sf, uint32_t workers, int64_t* out) {
    Tables t(sf, 1);
    t.init();
    t.populate();
    out[0] = (int64_t)run_q1<Q1V::Q11>(t, workers, 1, 3, 0, 24);
    out[1] = (int64_t)run_q1<Q1V::Q12>(t, workers, 4, 6, 26, 35);
    out[2] = (int64_t)run_q1<Q1V::Q13>(t, workers, 5, 7, 26, 35);
    uint64_t ng = 0, tot = 0;
    run_q31(t, workers, &ng, &tot);
    out[3] = (int64_t)ng;
    out[4] = (int64_t)tot;
    out[5] = (int64_t)t.lineorder.num_tuples;
    return 0;
}

// Copies reference-generated columns (as int32) for cross-checking the
// oracle's generator.  Arrays sized by the caller (lineorder: >= 7*orders).
__attribute__((visibility("default"))) int64_t ref_ssb_columns(uint32_t sf, int32_t* d_key, int32_t* d_year,
                                                               int32_t* c_nation, int32_t* s_nation,
                                                               int32_t* lo_orderdate, int32_t* lo_custkey,
                                                               int32_t* lo_suppkey, int32_t* lo_quantity,
                                                               int32_t* lo_discount, int32_t* lo_extendedprice,
                                                               int32_t* lo_revenue) {
    Tables t(sf, 1);
    t.init();
    t.populate();
    for (uint64_t i = 0; i < t.date.num_tuples; ++i) {
        d_key[i] = (int32_t)t.date.col<Date::KEY>().data()[i];
        d_year[i] = t.date.col<Date::YEAR>().data()[i];
    }
    for (uint64_t i = 0; i < t.customer.num_tuples; ++i) c_nation[i] = nation_index(t.customer.col<Customer::NATION>().data()[i]);
    for (uint64_t i = 0; i < t.supplier.num_tuples; ++i) s_nation[i] = nation_index(t.supplier.col<Supplier::NATION>().data()[i]);
    for (uint64_t i = 0; i < t.lineorder.num_tuples; ++i) {
        lo_orderdate[i] = (int32_t)t.lineorder.col<Lineorder::ORDERDATE>().data()[i];
        lo_custkey[i] = (int32_t)t.lineorder.col<Lineorder::CUSTKEY>().data()[i];
        lo_suppkey[i] = (int32_t)t.lineorder.col<Lineorder::SUPPKEY>().data()[i];
        lo_quantity[i] = t.lineorder.col<Lineorder::QUANTITY>().data()[i];
        lo_discount[i] = t.lineorder.col<Lineorder::DISCOUNT>().data()[i];
        lo_extendedprice[i] = (int32_t)t.lineorder.col<Lineorder::EXTENDEDPRICE>().data()[i];
        lo_revenue[i] = (int32_t)t.lineorder.col<Lineorder::REVENUE>().data()[i];
    }
    return (int64_t)t.lineorder.num_tuples;
}

// LZ4CPUManager::compress on each block of `block_bytes` (core/comp_cpu.hpp:28-31).
// comp_out must hold LZ4_compressBound per block; comp_sizes receives sizes.
__attribute__((visibility("default"))) int ref_lz4_compress_blocks(const char* in, uint64_t n_bytes, uint64_t block_bytes,
                                                                   char* comp_out, uint64_t stride, int32_t* comp_sizes) {
    golap::LZ4CPUManager m;
    uint64_t nb = (n_bytes + block_bytes - 1) / block_bytes;
    for (uint64_t b = 0; b < nb; ++b) {
        uint64_t len = std::min(block_bytes, n_bytes - b * block_bytes);
        int r = m.compress(in + b * block_bytes, comp_out + b * stride, (int)len);
        if (r <= 0) return -1;
        comp_sizes[b] = r;
    }
    return 0;
}

// LZ4CPUManager::decompress of one block (core/comp_cpu.hpp:24-27).
__attribute__((visibility("default"))) int ref_lz4_decompress(const char* in, int comp_size, char* out, int decomp_size) {
    golap::LZ4CPUManager m;
    return m.decompress(out, in, comp_size, decomp_size);
}

// CPU baseline for a Q1-shaped query over LZ4-compressed chunks, composed of
// the reference's CPU pieces the way its GPU driver composes its GPU pieces
// (usecases/ssb/queries/01.hpp:350-424): min/max host pruning
// (MinMaxMeta::check_pred_host, core/metadata.cuh:195-200) over the
// per-chunk min/max arrays, then per surviving chunk LZ4CPUManager
// decompression of the discount / quantity / extended-price blocks and the
// query1inmem probe loop (01inmem.hpp:109-130) with a HostHashMap date table.
// date_key is handed over uncompressed: the reference has no CPU cascaded
// decoder.  Chunks are split over `workers` threads with SliceSeq.
// Returns the sum; *elapsed_ms receives the wall time of the timed part.
__attribute__((visibility("default"))) int64_t ref_cpu_q1(
    uint32_t workers, uint64_t n_rows, uint64_t rows_per_chunk, uint64_t rows_per_block,
    const int32_t* date_key, const int32_t* date_mins, const int32_t* date_maxs,
    const char* const* comp_cols /* 3: discount, quantity, extendedprice */, uint64_t comp_stride,
    const int32_t* const* comp_sizes, const int32_t* d_key, const uint8_t* d_ok, uint64_t n_date, int32_t date_lo,
    int32_t date_hi, int32_t dlo, int32_t dhi, int32_t qlo, int32_t qhi, double* elapsed_ms, uint64_t* chunks_scanned) {
    std::vector<uint64_t> dkeys(n_date);
    for (uint64_t i = 0; i < n_date; ++i) dkeys[i] = (uint64_t)d_key[i];
    util::Timer timer;
    golap::HostHashMap<uint64_t> hm(n_date, dkeys.data());
    for (uint64_t i = 0; i < n_date; ++i)
        if (d_ok[i]) hm.insert(i, dkeys[i]);
    const uint64_t n_chunks = (n_rows + rows_per_chunk - 1) / rows_per_chunk;
    const uint64_t bpc = (rows_per_chunk + rows_per_block - 1) / rows_per_block;
    std::vector<uint64_t> keep;
    for (uint64_t c = 0; c < n_chunks; ++c)
        if (date_lo <= date_maxs[c] && date_hi >= date_mins[c]) keep.push_back(c);
    std::atomic<uint64_t> agg{0};
    util::SliceSeq sl{keep.size(), workers};
    std::vector<std::tuple<uint64_t, uint64_t>> sls(workers);
    for (auto& [s, e] : sls) sl.get(s, e);
    std::vector<std::thread> th;
    for (uint32_t w = 0; w < workers; ++w)
        th.emplace_back([&, w] {
            golap::LZ4CPUManager m;
            std::vector<int32_t> buf[3];
            for (auto& b : buf) b.resize(rows_per_block);
            uint64_t part = 0;
            auto [s, e] = sls[w];
            for (uint64_t k = s; k < e; ++k) {
                const uint64_t c = keep[k];
                const uint64_t r0 = c * rows_per_chunk, r1 = std::min(n_rows, r0 + rows_per_chunk);
                for (uint64_t j = 0; j < bpc; ++j) {
                    const uint64_t b0 = r0 + j * rows_per_block;
                    if (b0 >= r1) break;
                    const uint64_t rows = std::min(rows_per_block, r1 - b0);
                    const uint64_t slot = c * bpc + j;
                    for (int col = 0; col < 3; ++col)
                        m.decompress((char*)buf[col].data(), comp_cols[col] + slot * comp_stride,
                                     comp_sizes[col][slot], (int)(rows * 4));
                    for (uint64_t i = 0; i < rows; ++i) {
                        int32_t disc = buf[0][i], qty = buf[1][i];
                        if (disc < dlo || disc > dhi || qty < qlo || qty > qhi) continue;
                        if (hm.probe((uint64_t)date_key[b0 + i]) == (uint64_t)-1) continue;
                        part += (uint64_t)((int64_t)buf[2][i] * disc);
                    }
                }
            }
            agg.fetch_add(part, std::memory_order_relaxed);
        });
    for (auto& x : th) x.join();
    *elapsed_ms = timer.elapsed();
    *chunks_scanned = keep.size();
    return (int64_t)agg.load();
}

}  // extern "C"

// libnuma and snappy are declared by shims but never called; definitions
// keep the shared object self-contained if the linker asks for them.
extern "C" long get_mempolicy(int*, unsigned long*, unsigned long, void*, unsigned) { return -1; }
namespace snappy {
bool RawUncompress(const char*, size_t, char*) { return false; }
void RawCompress(const char*, size_t, char*, size_t* n) { *n = 0; }
}  // namespace snappy
