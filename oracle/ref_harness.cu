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

// Restatement of YEARBRAND_GROUP (usecases/ssb/queries/02.cuh:45-62) and
// Q41_GROUP (usecases/ssb/queries/04.cuh:12-31).
struct HYearBrand {
    uint16_t d_year;
    util::Padded<char[10]> p_brand1;
    uint64_t hash() const {
        uint64_t h = 0;
        std::memcpy(&h, p_brand1.d, 8);
        return h ^ d_year;
    }
    bool operator==(const HYearBrand& o) const {  // brands are 9 characters, never shorter
        for (int i = 0; i < 9; ++i)
            if (p_brand1.d[i] == '\0' || p_brand1.d[i] != o.p_brand1.d[i]) return false;
        return d_year == o.d_year;
    }
};
struct HYearBrandHash {
    std::size_t operator()(const HYearBrand& g) const { return g.hash(); }
};
struct HQ41 {
    uint16_t d_year;
    util::Padded<char[16]> c_nation;
    uint64_t hash() const {
        uint64_t h = (*(uint32_t*)c_nation.d);
        h <<= 32;
        h ^= d_year;
        return h;
    }
    bool operator==(const HQ41& o) const {
        for (int i = 0; i < 16; ++i) {
            if (c_nation.d[i] != o.c_nation.d[i]) return false;
            if (c_nation.d[i] == '\0') break;
        }
        return d_year == o.d_year;
    }
};
struct HQ41Hash {
    std::size_t operator()(const HQ41& g) const { return g.hash(); }
};

static bool str_is(const char* d, const char* s, int n) { return std::strncmp(d, s, n) == 0; }

// query2 body for Q2.1 (usecases/ssb/queries/02inmem.hpp:100-180, predicates
// of query2_1inmem :208-210: p_category MFGR#12, s_region AMERICA; every date).
static void run_q21(Tables& t, uint32_t workers, uint64_t* n_groups, uint64_t* total) {
    golap::HostHashMap ph(t.part.num_tuples, t.part.col<Part::KEY>().data());
    golap::HostHashMap sh(t.supplier.num_tuples, t.supplier.col<Supplier::KEY>().data());
    golap::HostHashMap dh(t.date.num_tuples, t.date.col<Date::KEY>().data());
    const uint64_t num_groups = 500;
    std::vector<HYearBrand> groups(num_groups);
    auto aggs = std::make_unique<std::atomic<uint64_t>[]>(num_groups);
    for (uint64_t i = 0; i < num_groups; ++i) aggs[i] = 0;
    golap::HostHashAggregate<HYearBrand, std::atomic<uint64_t>> ha(num_groups, groups.data(), aggs.get());
    util::SliceSeq ps{t.part.num_tuples, workers}, ss{t.supplier.num_tuples, workers}, dss{t.date.num_tuples, workers},
        ls{t.lineorder.num_tuples, workers};
    std::vector<std::tuple<uint64_t, uint64_t>> psl(workers), ssl(workers), dsl(workers), lsl(workers);
    for (auto& [s, e] : psl) ps.get(s, e);
    for (auto& [s, e] : ssl) ss.get(s, e);
    for (auto& [s, e] : dsl) dss.get(s, e);
    for (auto& [s, e] : lsl) ls.get(s, e);
    std::vector<std::thread> th;
    for (uint32_t w = 0; w < workers; ++w)
        th.emplace_back([&, w] {
            auto [s, e] = psl[w];
            for (uint64_t i = s; i < e; ++i)
                if (str_is(t.part.col<Part::CATEGORY>().data()[i].d, "MFGR#12", 8))
                    ph.insert(i, t.part.col<Part::KEY>().data()[i]);
            std::tie(s, e) = ssl[w];
            for (uint64_t i = s; i < e; ++i)
                if (region_is(t.supplier.col<Supplier::REGION>().data()[i], "AMERICA"))
                    sh.insert(i, t.supplier.col<Supplier::KEY>().data()[i]);
            std::tie(s, e) = dsl[w];
            for (uint64_t i = s; i < e; ++i) dh.insert(i, t.date.col<Date::KEY>().data()[i]);
        });
    for (auto& x : th) x.join();
    th.clear();
    for (uint32_t w = 0; w < workers; ++w)
        th.emplace_back([&, w] {
            auto [s, e] = lsl[w];
            std::unordered_map<HYearBrand, uint64_t, HYearBrandHash> local;
            for (uint64_t i = s; i < e; ++i) {
                const uint64_t pm = ph.probe(t.lineorder.col<Lineorder::PARTKEY>().data()[i]);
                if (pm == (uint64_t)-1) continue;
                const uint64_t sm = sh.probe(t.lineorder.col<Lineorder::SUPPKEY>().data()[i]);
                if (sm == (uint64_t)-1) continue;
                const uint64_t dm = dh.probe(t.lineorder.col<Lineorder::ORDERDATE>().data()[i]);
                local[HYearBrand{t.date.col<Date::YEAR>().data()[dm], t.part.col<Part::BRAND1>().data()[pm]}] +=
                    t.lineorder.col<Lineorder::REVENUE>().data()[i];
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

// query4inmem body for Q4.1 (usecases/ssb/queries/04inmem.hpp:80-160,
// predicates of query4_1inmem :204-210: c_region and s_region AMERICA,
// p_mfgr MFGR#1 or MFGR#2, every date); profit = revenue - supplycost.
static void run_q41(Tables& t, uint32_t workers, uint64_t* n_groups, uint64_t* total) {
    golap::HostHashMap ch(t.customer.num_tuples, t.customer.col<Customer::KEY>().data());
    golap::HostHashMap sh(t.supplier.num_tuples, t.supplier.col<Supplier::KEY>().data());
    golap::HostHashMap dh(t.date.num_tuples, t.date.col<Date::KEY>().data());
    golap::HostHashMap ph(t.part.num_tuples, t.part.col<Part::KEY>().data());
    const uint64_t num_groups = 800;
    std::vector<HQ41> groups(num_groups);
    auto aggs = std::make_unique<std::atomic<uint64_t>[]>(num_groups);
    for (uint64_t i = 0; i < num_groups; ++i) aggs[i] = 0;
    golap::HostHashAggregate<HQ41, std::atomic<uint64_t>> ha(num_groups, groups.data(), aggs.get());
    util::SliceSeq cs{t.customer.num_tuples, workers}, ss{t.supplier.num_tuples, workers},
        dss{t.date.num_tuples, workers}, ps{t.part.num_tuples, workers}, ls{t.lineorder.num_tuples, workers};
    std::vector<std::tuple<uint64_t, uint64_t>> csl(workers), ssl(workers), dsl(workers), psl(workers), lsl(workers);
    for (auto& [s, e] : csl) cs.get(s, e);
    for (auto& [s, e] : ssl) ss.get(s, e);
    for (auto& [s, e] : dsl) dss.get(s, e);
    for (auto& [s, e] : psl) ps.get(s, e);
    for (auto& [s, e] : lsl) ls.get(s, e);
    std::vector<std::thread> th;
    for (uint32_t w = 0; w < workers; ++w)
        th.emplace_back([&, w] {
            auto [s, e] = csl[w];
            for (uint64_t i = s; i < e; ++i)
                if (region_is(t.customer.col<Customer::REGION>().data()[i], "AMERICA"))
                    ch.insert(i, t.customer.col<Customer::KEY>().data()[i]);
            std::tie(s, e) = ssl[w];
            for (uint64_t i = s; i < e; ++i)
                if (region_is(t.supplier.col<Supplier::REGION>().data()[i], "AMERICA"))
                    sh.insert(i, t.supplier.col<Supplier::KEY>().data()[i]);
            std::tie(s, e) = dsl[w];
            for (uint64_t i = s; i < e; ++i) dh.insert(i, t.date.col<Date::KEY>().data()[i]);
            std::tie(s, e) = psl[w];
            for (uint64_t i = s; i < e; ++i) {
                const char* m = t.part.col<Part::MFGR>().data()[i].d;
                if (str_is(m, "MFGR#1", 7) || str_is(m, "MFGR#2", 7)) ph.insert(i, t.part.col<Part::KEY>().data()[i]);
            }
        });
    for (auto& x : th) x.join();
    th.clear();
    for (uint32_t w = 0; w < workers; ++w)
        th.emplace_back([&, w] {
            auto [s, e] = lsl[w];
            std::unordered_map<HQ41, uint64_t, HQ41Hash> local;
            for (uint64_t i = s; i < e; ++i) {
                const uint64_t cm = ch.probe(t.lineorder.col<Lineorder::CUSTKEY>().data()[i]);
                if (cm == (uint64_t)-1) continue;
                const uint64_t sm = sh.probe(t.lineorder.col<Lineorder::SUPPKEY>().data()[i]);
                if (sm == (uint64_t)-1) continue;
                const uint64_t dm = dh.probe(t.lineorder.col<Lineorder::ORDERDATE>().data()[i]);
                if (dm == (uint64_t)-1) continue;
                const uint64_t pm = ph.probe(t.lineorder.col<Lineorder::PARTKEY>().data()[i]);
                if (pm == (uint64_t)-1) continue;
                const uint64_t profit = t.lineorder.col<Lineorder::REVENUE>().data()[i] -
                                        t.lineorder.col<Lineorder::SUPPLYCOST>().data()[i];
                local[HQ41{t.date.col<Date::YEAR>().data()[dm], t.customer.col<Customer::NATION>().data()[cm]}] +=
                    profit;
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

static int part_code(const char* mfgr_str) { return mfgr_str[5] - '1'; }

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

// Q2.1 and Q4.1 on the reference tables: out = {q21_groups, q21_sum,
// q41_groups, q41_sum}.
__attribute__((visibility("default"))) int ref_ssb_golden_flights(uint32_t sf, uint32_t workers, int64_t* out) {
    Tables t(sf, 1);
    t.init();
    t.populate();
    uint64_t ng = 0, tot = 0;
    run_q21(t, workers, &ng, &tot);
    out[0] = (int64_t)ng;
    out[1] = (int64_t)tot;
    run_q41(t, workers, &ng, &tot);
    out[2] = (int64_t)ng;
    out[3] = (int64_t)tot;
    return 0;
}

// The part and lineorder columns the Q2/Q4 flights read, as integer codes
// (p_mfgr "MFGR#m" -> m-1, p_category "MFGR#mn" -> 5(m-1)+(n-1), p_brand1
// "MFGR#mnbb" -> 40*category + bb-1) for cross-checking the oracle.
__attribute__((visibility("default"))) int64_t ref_ssb_part_columns(uint32_t sf, int32_t* p_mfgr, int32_t* p_category,
                                                                    int32_t* p_brand1, int32_t* lo_partkey,
                                                                    int32_t* lo_supplycost) {
    Tables t(sf, 1);
    t.init();
    t.populate();
    for (uint64_t i = 0; i < t.part.num_tuples; ++i) {
        const char* m = t.part.col<Part::MFGR>().data()[i].d;
        const char* c = t.part.col<Part::CATEGORY>().data()[i].d;
        const char* b = t.part.col<Part::BRAND1>().data()[i].d;
        p_mfgr[i] = part_code(m);
        p_category[i] = 5 * part_code(m) + (c[6] - '1');
        p_brand1[i] = 40 * p_category[i] + (b[7] - '0') * 10 + (b[8] - '0') - 1;
    }
    for (uint64_t i = 0; i < t.lineorder.num_tuples; ++i) {
        lo_partkey[i] = (int32_t)t.lineorder.col<Lineorder::PARTKEY>().data()[i];
        lo_supplycost[i] = (int32_t)t.lineorder.col<Lineorder::SUPPLYCOST>().data()[i];
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

// ---------------------------------------------------------------------------
// CPU baselines over the compressed columns the GPU path scans (the same
// bytes): LZ4 blocks decoded by the reference's LZ4CPUManager
// (core/comp_cpu.hpp:22-32); cascaded blocks (the build's own format, for
// which the reference has no CPU decoder) decoded by casc_cpu_block below,
// labelled as such by the caller.  Columns arrive as {payload, blocks} where
// blocks[4*k..] = {offset, size, payload bytes, tuples} of the k-th present
// block in slot order (gx_column_blocks, the reference's BlockInfo layout,
// core/comp.cuh:23-32).
// ---------------------------------------------------------------------------

// Cascaded page / block decode (format in golap_public_b200/csrc/gx_internal.h).
static inline uint32_t cc_unpack(const uint32_t* w, uint64_t i, uint32_t bits) {
    if (bits == 0) return 0;
    const uint64_t bit = i * bits;
    const uint64_t two = (uint64_t)w[bit >> 5] | ((uint64_t)w[(bit >> 5) + 1] << 32);
    return (uint32_t)((two >> (bit & 31)) & (bits == 32 ? 0xFFFFFFFFull : ((1ull << bits) - 1)));
}
static bool casc_cpu_page(const uint8_t* pg, uint32_t bytes, int32_t* out, uint32_t rows) {
    if (bytes < 32) return false;
    uint32_t h[8];
    std::memcpy(h, pg, 32);
    const uint32_t n_rows = h[0], n_runs = h[1], flags = h[2] & 255, vbits = (h[2] >> 8) & 255,
                   lbits = (h[2] >> 16) & 255, vbase = h[4], lbase = h[5], voff = h[6], loff = h[7];
    const bool rle = flags & 1, delta = flags & 2;
    if (n_rows != rows || vbits > 32 || lbits > 32 || (!rle && n_runs != rows)) return false;
    if ((uint64_t)voff + 4ull * (((uint64_t)n_runs * vbits + 31) / 32 + 1) > bytes) return false;
    if (rle && (uint64_t)loff + 4ull * (((uint64_t)n_runs * lbits + 31) / 32 + 1) > bytes) return false;
    const uint32_t* vw = (const uint32_t*)(pg + voff);
    const uint32_t* lw = (const uint32_t*)(pg + loff);
    uint32_t acc = h[3], r = 0;
    for (uint32_t i = 0; i < n_runs; ++i) {
        const uint32_t e = cc_unpack(vw, i, vbits) + vbase;
        const uint32_t v = delta ? (i ? (acc += e) : acc) : e;
        const uint32_t len = rle ? cc_unpack(lw, i, lbits) + lbase : 1;
        if (r + len > rows) return false;
        for (uint32_t k = 0; k < len; ++k) out[r + k] = (int32_t)v;
        r += len;
    }
    return r == rows;
}
static bool casc_cpu_block(const uint8_t* blk, uint64_t bytes, int32_t* out, uint32_t rows) {
    if (bytes < 8) return false;
    uint32_t np, pr;
    std::memcpy(&np, blk, 4);
    std::memcpy(&pr, blk + 4, 4);
    if (pr == 0 || 8 + 4ull * (np + 1) > bytes) return false;
    uint32_t done = 0;
    for (uint32_t p = 0; p < np; ++p) {
        uint32_t a, b;
        std::memcpy(&a, blk + 8 + 4ull * p, 4);
        std::memcpy(&b, blk + 8 + 4ull * (p + 1), 4);
        const uint32_t n = std::min(pr, rows - done);
        if (a > b || b > bytes || !casc_cpu_page(blk + a, b - a, out + done, n)) return false;
        done += n;
    }
    return done == rows;
}

struct CompCol {
    const uint8_t* payload;
    const uint64_t* blocks;  // 4 words per present block
    uint32_t codec;          // 1 LZ4, 2 cascaded
};

// Decode present block k of a column into out (rows values).
static bool decode_block(const CompCol& c, uint64_t k, int32_t* out, uint32_t rows, golap::LZ4CPUManager& m) {
    const uint64_t off = c.blocks[4 * k], used = c.blocks[4 * k + 2];
    if (c.codec == 1) return m.decompress((char*)out, (const char*)(c.payload + off), (int)used, (int)(rows * 4)) ==
                             (int)(rows * 4);
    return casc_cpu_block(c.payload + off, used, out, rows);
}

// Present blocks of the table in slot order: first row and row count; those
// of chunks that pass the min/max check (MinMaxMeta::check_pred_host,
// core/metadata.cuh:195-200) go into `work`.
static void table_blocks(uint64_t n_rows, uint64_t rpc, uint64_t rpb, const int32_t* mins, const int32_t* maxs,
                         int32_t lo, int32_t hi, std::vector<uint64_t>& work, std::vector<uint64_t>& row0,
                         std::vector<uint32_t>& rows, uint64_t* chunks_kept) {
    const uint64_t n_chunks = (n_rows + rpc - 1) / rpc;
    uint64_t kept = 0;
    for (uint64_t c = 0; c < n_chunks; ++c) {
        const uint64_t r0 = c * rpc, r1 = std::min(n_rows, r0 + rpc);
        const bool keep = !mins || (lo <= maxs[c] && hi >= mins[c]);
        kept += keep;
        for (uint64_t b0 = r0; b0 < r1; b0 += rpb) {
            if (keep) work.push_back(row0.size());
            row0.push_back(b0);
            rows.push_back((uint32_t)std::min(rpb, r1 - b0));
        }
    }
    *chunks_kept = kept;
}

// Q1 shape (query1inmem loop body, usecases/ssb/queries/01inmem.hpp:109-130)
// over compressed date_key / discount / quantity / extended_price: date table
// HostHashMap built from the flagged dimension rows, chunk pruning on the
// date_key min/max, then the surviving blocks split evenly over `workers`
// threads (SliceSeq), each decoding its blocks and running the probe loop.
__attribute__((visibility("default"))) int64_t ref_cpu_q1_comp(
    uint32_t workers, uint64_t n_rows, uint64_t rows_per_chunk, uint64_t rows_per_block, const CompCol* cols /* 4 */,
    const int32_t* date_mins, const int32_t* date_maxs, const int32_t* d_key, const uint8_t* d_ok, uint64_t n_date,
    int32_t date_lo, int32_t date_hi, int32_t dlo, int32_t dhi, int32_t qlo, int32_t qhi, double* elapsed_ms,
    uint64_t* chunks_scanned, uint64_t* rows_scanned) {
    std::vector<uint64_t> work, row0;
    std::vector<uint32_t> brows;
    table_blocks(n_rows, rows_per_chunk, rows_per_block, date_mins, date_maxs, date_lo, date_hi, work, row0, brows,
                 chunks_scanned);
    std::vector<uint64_t> dkeys(n_date);
    for (uint64_t i = 0; i < n_date; ++i) dkeys[i] = (uint64_t)d_key[i];
    util::Timer timer;
    golap::HostHashMap<uint64_t> hm(n_date, dkeys.data());
    for (uint64_t i = 0; i < n_date; ++i)
        if (d_ok[i]) hm.insert(i, dkeys[i]);
    std::atomic<uint64_t> agg{0}, scanned{0};
    std::atomic<int> bad{0};
    util::SliceSeq sl{work.size(), workers};
    std::vector<std::tuple<uint64_t, uint64_t>> sls(workers);
    for (auto& [s, e] : sls) sl.get(s, e);
    std::vector<std::thread> th;
    for (uint32_t w = 0; w < workers; ++w)
        th.emplace_back([&, w] {
            golap::LZ4CPUManager m;
            std::vector<int32_t> buf[4];
            for (auto& b : buf) b.resize(rows_per_block);
            uint64_t part = 0, nr = 0;
            auto [s, e] = sls[w];
            for (uint64_t t = s; t < e; ++t) {
                const uint64_t k = work[t];
                const uint32_t rows = brows[k];
                for (int c = 0; c < 4; ++c)
                    if (!decode_block(cols[c], k, buf[c].data(), rows, m)) bad = 1;
                const int32_t *od = buf[0].data(), *disc = buf[1].data(), *qty = buf[2].data(), *ext = buf[3].data();
                for (uint32_t i = 0; i < rows; ++i) {
                    if (disc[i] < dlo || disc[i] > dhi || qty[i] < qlo || qty[i] > qhi) continue;
                    if (hm.probe((uint64_t)od[i]) == (uint64_t)-1) continue;
                    part += (uint64_t)((int64_t)ext[i] * disc[i]);
                }
                nr += rows;
            }
            agg.fetch_add(part, std::memory_order_relaxed);
            scanned.fetch_add(nr, std::memory_order_relaxed);
        });
    for (auto& x : th) x.join();
    *elapsed_ms = timer.elapsed();
    *rows_scanned = scanned.load();
    return bad ? INT64_MIN : (int64_t)agg.load();
}

// Group of the int32 star-join schema: (c_nation, s_nation, year), the
// integer form of Q3NATION_GROUP (usecases/ssb/queries/03.cuh:29-59) with the
// same hash shape.
struct HIGroup {
    int32_t c_nation, s_nation, year;
    uint64_t hash() const { return (((uint64_t)(uint32_t)c_nation << 32) | (uint32_t)s_nation) ^ (uint64_t)year; }
    bool operator==(const HIGroup& o) const {
        return c_nation == o.c_nation && s_nation == o.s_nation && year == o.year;
    }
};
struct HIGroupHash {
    std::size_t operator()(const HIGroup& g) const { return g.hash(); }
};

// Q3 shape (query3_inmem, usecases/ssb/queries/03inmem.hpp:70-226) over
// compressed date_key / cust_key / supp_key / revenue: filtered HostHashMap
// builds of customer (region), supplier (region) and date (year range) split
// over the workers, chunk pruning on the date_key min/max against the year
// range, then the surviving blocks split over the workers; per row the
// probes in customer -> supplier -> date order, a thread-local map per group
// and HostHashAggregate::add of the local sums (the reference's own
// sequence).  Groups are returned unordered: keys as
// (c_nation * 25 + s_nation) * n_years + (year - ylo), their sums, *n_groups.
__attribute__((visibility("default"))) int64_t ref_cpu_q3_comp(
    uint32_t workers, uint64_t n_rows, uint64_t rows_per_chunk, uint64_t rows_per_block, const CompCol* cols /* 4 */,
    const int32_t* date_mins, const int32_t* date_maxs, const int32_t* c_key, const int32_t* c_nation,
    const int32_t* c_region, uint64_t n_cust, const int32_t* s_key, const int32_t* s_nation, const int32_t* s_region,
    uint64_t n_supp, const int32_t* d_key, const int32_t* d_year, uint64_t n_date, int32_t region, int32_t ylo,
    int32_t yhi, int64_t* group_keys, int64_t* group_sums, uint64_t cap, uint64_t* n_groups, double* elapsed_ms,
    uint64_t* chunks_scanned, uint64_t* rows_scanned) {
    std::vector<uint64_t> work, row0;
    std::vector<uint32_t> brows;
    table_blocks(n_rows, rows_per_chunk, rows_per_block, date_mins, date_maxs, ylo * 10000 + 101, yhi * 10000 + 1231,
                 work, row0, brows, chunks_scanned);
    std::vector<uint64_t> ck(n_cust), sk(n_supp), dk(n_date);
    for (uint64_t i = 0; i < n_cust; ++i) ck[i] = (uint64_t)c_key[i];
    for (uint64_t i = 0; i < n_supp; ++i) sk[i] = (uint64_t)s_key[i];
    for (uint64_t i = 0; i < n_date; ++i) dk[i] = (uint64_t)d_key[i];
    const uint64_t num_groups = 800;
    std::vector<HIGroup> groups(num_groups);
    auto aggs = std::make_unique<std::atomic<uint64_t>[]>(num_groups);
    for (uint64_t i = 0; i < num_groups; ++i) aggs[i] = 0;
    util::Timer timer;
    golap::HostHashMap<uint64_t> ch(n_cust, ck.data()), sh(n_supp, sk.data()), dh(n_date, dk.data());
    golap::HostHashAggregate<HIGroup, std::atomic<uint64_t>> ha(num_groups, groups.data(), aggs.get());
    util::SliceSeq cs{n_cust, workers}, ss{n_supp, workers}, dss{n_date, workers}, ls{work.size(), workers};
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
                if (c_region[i] == region) ch.insert(i, ck[i]);
            std::tie(s, e) = ssl[w];
            for (uint64_t i = s; i < e; ++i)
                if (s_region[i] == region) sh.insert(i, sk[i]);
            std::tie(s, e) = dsl[w];
            for (uint64_t i = s; i < e; ++i)
                if (d_year[i] >= ylo && d_year[i] <= yhi) dh.insert(i, dk[i]);
        });
    for (auto& x : th) x.join();
    th.clear();
    std::atomic<uint64_t> scanned{0};
    std::atomic<int> bad{0};
    for (uint32_t w = 0; w < workers; ++w)
        th.emplace_back([&, w] {
            golap::LZ4CPUManager m;
            std::vector<int32_t> buf[4];
            for (auto& b : buf) b.resize(rows_per_block);
            std::unordered_map<HIGroup, uint64_t, HIGroupHash> local;
            uint64_t nr = 0;
            auto [s, e] = lsl[w];
            for (uint64_t t = s; t < e; ++t) {
                const uint64_t k = work[t];
                const uint32_t rows = brows[k];
                for (int c = 0; c < 4; ++c)
                    if (!decode_block(cols[c], k, buf[c].data(), rows, m)) bad = 1;
                const int32_t *od = buf[0].data(), *cu = buf[1].data(), *su = buf[2].data(), *rev = buf[3].data();
                for (uint32_t i = 0; i < rows; ++i) {
                    const uint64_t cm = ch.probe((uint64_t)cu[i]);
                    if (cm == (uint64_t)-1) continue;
                    const uint64_t sm = sh.probe((uint64_t)su[i]);
                    if (sm == (uint64_t)-1) continue;
                    const uint64_t dm = dh.probe((uint64_t)od[i]);
                    if (dm == (uint64_t)-1) continue;
                    local[HIGroup{c_nation[cm], s_nation[sm], d_year[dm]}] += (uint64_t)(uint32_t)rev[i];
                }
                nr += rows;
            }
            for (auto& [g, v] : local) ha.add(g, v, HostSumAtomic());
            scanned.fetch_add(nr, std::memory_order_relaxed);
        });
    for (auto& x : th) x.join();
    *elapsed_ms = timer.elapsed();
    *rows_scanned = scanned.load();
    const int32_t ny = yhi - ylo + 1;
    uint64_t ng = 0;
    int64_t total = 0;
    for (uint64_t i = 0; i < num_groups; ++i) {
        if (ha.wrote_group[i] == 0) continue;
        const HIGroup& g = groups[i];
        if (ng < cap) {
            group_keys[ng] = ((int64_t)g.c_nation * 25 + g.s_nation) * ny + (g.year - ylo);
            group_sums[ng] = (int64_t)aggs[i].load();
        }
        ++ng;
        total += (int64_t)aggs[i].load();
    }
    *n_groups = ng;
    return bad ? INT64_MIN : total;
}

}  // extern "C"

// libnuma and snappy are declared by shims but never called; definitions
// keep the shared object self-contained if the linker asks for them.
extern "C" long get_mempolicy(int*, unsigned long*, unsigned long, void*, unsigned) { return -1; }
namespace snappy {
bool RawUncompress(const char*, size_t, char*) { return false; }
void RawCompress(const char*, size_t, char*, size_t* n) { *n = 0; }
}  // namespace snappy
