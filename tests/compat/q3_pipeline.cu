// q3_pipeline.cu -- a GOLAP-style Q3 pipeline written against the drop-in
// header include/golap_compat/golap_compat.cuh, in the shape of the
// reference's query3 driver (usecases/ssb/queries/03.hpp:249-547) and its
// kernels pipeline_customer_q3 / pipeline_q3 (usecases/ssb/queries/03.cuh:
// 94-170):
//   * per-chunk min/max of the fact date_key through MinMaxMeta(chunk_num,
//     max_tuples) + init_chunk on decompressed chunks, checked against the
//     ingest min/max; MetaChecker::add_minmax on a std::any holding it;
//   * the customer join table built from compressed customer chunks
//     (ChunkDecompressor steps, then a kernel that filters on region,
//     compacts the customers into a buffer with an atomic counter and inserts
//     them -- pipeline_customer_q3's shape);
//   * supplier and date tables built with hash_map_build_pred_other<<<>>>
//     and PredInfo predicates;
//   * per fact chunk skip_step or four ChunkDecompressor steps, then a kernel
//     probing customer -> supplier -> date and adding revenue into
//     HashAggregate<NationGroup, uint64_t> with SumAgg (NationGroup has the
//     layout of Q3NATION_GROUP, 03.cuh:29-59, filled supplier nation first as
//     the reference fills it, 03.cuh:159);
//   * Aggregate(aggs, total, 800, sum, 0).execute() over the group sums;
//   * the same query through the fused gx_scan.
// Input: raw int32 files in a directory.  Output: one "g <c_nation>
// <s_nation> <year> <sum>" line per group, then "groups=.. total=..
// agg_total=.. fused_total=.. chunks=kept/total minmax_ok=0|1".
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "golap_compat/golap_compat.cuh"

using golap::HashMap;

// nation index -> 16-byte padded name (the SSB nation list)
struct Name16 {
    char d[16];
};
static const char* kNations[25] = {"ALGERIA", "ARGENTINA", "BRAZIL",  "CANADA",         "EGYPT",
                                   "ETHIOPIA", "FRANCE",   "GERMANY", "INDIA",          "INDONESIA",
                                   "IRAN",     "IRAQ",     "JAPAN",   "JORDAN",         "KENYA",
                                   "MOROCCO",  "MOZAMBIQUE", "PERU",  "CHINA",          "ROMANIA",
                                   "SAUDI ARABIA", "VIETNAM", "RUSSIA", "UNITED KINGDOM", "UNITED STATES"};

struct NationGroup {
    Name16 c_nation;
    Name16 s_nation;
    uint16_t d_year;
    __host__ __device__ uint64_t hash() const {
        uint64_t h;
        uint32_t a, b;
        memcpy(&a, c_nation.d, 4);
        memcpy(&b, s_nation.d, 4);
        h = a;
        h <<= 32;
        h |= b;
        h ^= d_year;
        return h;
    }
    __host__ __device__ bool operator==(const NationGroup& o) const {
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

struct Customer {
    int32_t c_key;
    Name16 c_nation;
};
struct CustomerKey {
    __host__ __device__ uint64_t operator()(Customer* t) const { return (uint64_t)t->c_key; }
};
struct SumAgg {
    __device__ void operator()(uint64_t* agg, uint64_t v) const { atomicAdd((unsigned long long*)agg, (unsigned long long)v); }
};
struct EqPred {
    int32_t v;
    __host__ __device__ bool operator()(int32_t* p) const { return *p == v; }
};
struct Plus {
    __host__ __device__ uint64_t operator()(uint64_t a, uint64_t b) const { return a + b; }
};

// pipeline_customer_q3's shape: filter, compact with an atomic counter, insert.
template <typename PRED>
__global__ void build_customer(HashMap<Customer, uint64_t> customer_hashmap, const int32_t* c_key,
                               const int32_t* c_nation, PRED pred_info, const Name16* names, Customer* customer_buffer,
                               unsigned long long* customer_counter, uint64_t num) {
    for (uint64_t r = blockDim.x * (uint64_t)blockIdx.x + threadIdx.x; r < num; r += (uint64_t)blockDim.x * gridDim.x) {
        if (!pred_info.pred(&pred_info.col[r])) continue;
        const uint64_t cur = atomicAdd(customer_counter, 1ull);
        customer_buffer[cur] = Customer{c_key[r], names[c_nation[r]]};
        customer_hashmap.insert(cur, (uint64_t)c_key[r]);
    }
}

// pipeline_q3's shape (Q3NATION_GROUP branch).
__global__ void probe_aggregate(HashMap<Customer, uint64_t> customer_hashmap, HashMap<int32_t, uint64_t> supplier_hashmap,
                                HashMap<int32_t, uint64_t> date_hashmap, golap::HashAggregate<NationGroup, uint64_t> hashagg,
                                const int32_t* lo_custkey, const int32_t* lo_suppkey, const int32_t* lo_orderdate,
                                const int32_t* lo_revenue, const Name16* s_nation, const int32_t* d_year,
                                const Customer* customer_dev, uint64_t num) {
    for (uint64_t r = blockDim.x * (uint64_t)blockIdx.x + threadIdx.x; r < num; r += (uint64_t)blockDim.x * gridDim.x) {
        const uint64_t cm = customer_hashmap.probe((uint64_t)lo_custkey[r], CustomerKey());
        if (cm == (uint64_t)-1) continue;
        const uint64_t sm = supplier_hashmap.probe((uint64_t)lo_suppkey[r]);
        if (sm == (uint64_t)-1) continue;
        const uint64_t dm = date_hashmap.probe((uint64_t)lo_orderdate[r]);
        if (dm == (uint64_t)-1) continue;
        hashagg.add(NationGroup{s_nation[sm], customer_dev[cm].c_nation, (uint16_t)d_year[dm]},
                    (uint64_t)(uint32_t)lo_revenue[r], SumAgg());
    }
}

__global__ void nation_names(const int32_t* nation, const Name16* names, Name16* out, uint64_t n) {
    for (uint64_t i = blockDim.x * (uint64_t)blockIdx.x + threadIdx.x; i < n; i += (uint64_t)blockDim.x * gridDim.x)
        out[i] = names[nation[i]];
}

static std::vector<int32_t> read_col(const std::string& path) {
    FILE* f = fopen(path.c_str(), "rb");
    if (!f) {
        perror(path.c_str());
        exit(2);
    }
    fseek(f, 0, SEEK_END);
    long n = ftell(f) / 4;
    fseek(f, 0, SEEK_SET);
    std::vector<int32_t> v(n);
    if (fread(v.data(), 4, n, f) != (size_t)n) exit(2);
    fclose(f);
    return v;
}
template <typename T>
static T* to_dev(const std::vector<T>& v) {
    T* p = nullptr;
    golap::cuda_check(cudaMalloc(&p, sizeof(T) * (v.size() ? v.size() : 1)), "cudaMalloc");
    golap::cuda_check(cudaMemcpy(p, v.data(), sizeof(T) * v.size(), cudaMemcpyHostToDevice), "cudaMemcpy");
    return p;
}
static int nation_of(const Name16& n) {
    for (int i = 0; i < 25; ++i)
        if (strncmp(n.d, kNations[i], 16) == 0) return i;
    return -1;
}

int main(int argc, char** argv) {
    if (argc != 6) {
        fprintf(stderr, "usage: %s dir region ylo yhi cust_chunk_rows\n", argv[0]);
        return 2;
    }
    const std::string dir = argv[1];
    const int32_t region = atoi(argv[2]), ylo = atoi(argv[3]), yhi = atoi(argv[4]);
    const uint64_t cust_chunk_rows = strtoull(argv[5], nullptr, 10);
    auto od = read_col(dir + "/date_key.bin"), ck = read_col(dir + "/cust_key.bin"),
         sk = read_col(dir + "/supp_key.bin"), rev = read_col(dir + "/revenue.bin");
    auto c_key = read_col(dir + "/c_key.bin"), c_nat = read_col(dir + "/c_nation.bin"),
         c_reg = read_col(dir + "/c_region.bin");
    auto s_key = read_col(dir + "/s_key.bin"), s_nat = read_col(dir + "/s_nation.bin"),
         s_reg = read_col(dir + "/s_region.bin");
    auto d_key = read_col(dir + "/d_key.bin"), d_year = read_col(dir + "/d_year.bin");
    const uint64_t n = od.size(), chunk_rows = 1000000, chunk_bytes = chunk_rows * 4;
    cudaStream_t stream;
    cudaStreamCreate(&stream);
    try {
        std::vector<Name16> names(25);
        for (int i = 0; i < 25; ++i) {
            memset(names[i].d, 0, 16);
            strncpy(names[i].d, kNations[i], 15);
        }
        Name16* names_dev = to_dev(names);

        // ---- ingest (prepare_compressed) of the fact and customer columns
        auto ci_date = golap::prepare_compressed(od.data(), n, chunk_bytes, "Cascaded", 1, stream);
        auto ci_cust = golap::prepare_compressed(ck.data(), n, chunk_bytes, "LZ4", 1, stream);
        auto ci_supp = golap::prepare_compressed(sk.data(), n, chunk_bytes, "LZ4", 1, stream);
        auto ci_rev = golap::prepare_compressed(rev.data(), n, chunk_bytes, "LZ4", 1, stream);
        auto ci_ckey = golap::prepare_compressed(c_key.data(), c_key.size(), cust_chunk_rows * 4, "LZ4", 1, stream);
        auto ci_cnat = golap::prepare_compressed(c_nat.data(), c_key.size(), cust_chunk_rows * 4, "Cascaded", 1, stream);
        auto ci_creg = golap::prepare_compressed(c_reg.data(), c_key.size(), cust_chunk_rows * 4, "Cascaded", 1, stream);
        const uint64_t chunk_num = ci_date.chunk_num();

        // ---- date_key min/max per chunk: MinMaxMeta(chunk_num, max_tuples) + init_chunk
        int32_t* scratch = nullptr;
        golap::cuda_check(cudaMalloc(&scratch, chunk_bytes), "cudaMalloc");
        auto mgr_date0 = golap::build_gpucomp_manager(ci_date);
        golap::MinMaxMeta<int32_t> meta(chunk_num, chunk_rows);
        {
            golap::ChunkDecompressor d(chunk_bytes, nullptr, (char*)scratch, false, false, *mgr_date0,
                                       ci_date.chunk_size_vec);
            for (uint64_t c = 0; c < chunk_num; ++c) {
                d.step(stream);
                meta.init_chunk(c, scratch, ci_date.chunk_size_vec[c] / 4, stream);
            }
        }
        meta.to_host(stream);
        golap::cuda_check(cudaStreamSynchronize(stream), "sync");
        golap::MinMaxMeta<int32_t> ingest(ci_date);
        int minmax_ok = 1;
        for (uint64_t c = 0; c < chunk_num; ++c)
            minmax_ok &= meta.mins_hst[c] == ingest.mins_hst[c] && meta.maxs_hst[c] == ingest.maxs_hst[c];

        // ---- pruning (MetaChecker::add_minmax on a std::any, 03.hpp:328-370)
        uint16_t *combined, *tmp;
        cudaMalloc(&combined, 2 * chunk_num);
        cudaMalloc(&tmp, 2 * chunk_num);
        golap::MetaChecker checker(1, chunk_num, combined, tmp, stream);
        std::any any_meta = meta;
        checker.add_minmax<int32_t>(any_meta, ylo * 10000 + 101, yhi * 10000 + 1231);
        std::vector<uint16_t> keep(chunk_num);
        cudaMemcpyAsync(keep.data(), combined, 2 * chunk_num, cudaMemcpyDeviceToHost, stream);
        golap::cuda_check(cudaStreamSynchronize(stream), "sync");

        // ---- customer table from compressed customer chunks (pipeline_customer_q3's shape)
        const uint64_t n_cust = c_key.size();
        Customer* cust_buf = nullptr;
        cudaMalloc(&cust_buf, sizeof(Customer) * n_cust);
        unsigned long long* cust_count = nullptr;
        cudaMalloc(&cust_count, 8);
        cudaMemsetAsync(cust_count, 0, 8, stream);
        HashMap<Customer, uint64_t> customer_hashmap(n_cust, cust_buf);
        int32_t *cb_key, *cb_nat, *cb_reg;
        cudaMalloc(&cb_key, cust_chunk_rows * 4);
        cudaMalloc(&cb_nat, cust_chunk_rows * 4);
        cudaMalloc(&cb_reg, cust_chunk_rows * 4);
        {
            auto m1 = golap::build_gpucomp_manager(ci_ckey), m2 = golap::build_gpucomp_manager(ci_cnat),
                 m3 = golap::build_gpucomp_manager(ci_creg);
            golap::ChunkDecompressor d1(cust_chunk_rows * 4, nullptr, (char*)cb_key, false, false, *m1,
                                        ci_ckey.chunk_size_vec);
            golap::ChunkDecompressor d2(cust_chunk_rows * 4, nullptr, (char*)cb_nat, false, false, *m2,
                                        ci_cnat.chunk_size_vec);
            golap::ChunkDecompressor d3(cust_chunk_rows * 4, nullptr, (char*)cb_reg, false, false, *m3,
                                        ci_creg.chunk_size_vec);
            for (uint64_t c = 0; c < ci_ckey.chunk_num(); ++c) {
                d1.step(stream);
                d2.step(stream);
                d3.step(stream);
                const uint64_t rows = ci_ckey.chunk_size_vec[c] / 4;
                build_customer<<<(unsigned)((rows + 511) / 512), 512, 0, stream>>>(
                    customer_hashmap, cb_key, cb_nat, golap::PredInfo<int32_t, EqPred>{cb_reg, EqPred{region}},
                    names_dev, cust_buf, cust_count, rows);
            }
        }

        // ---- supplier and date tables (hash_map_build_pred_other, 03.hpp:306-326)
        int32_t *sk_dev = to_dev(s_key), *sn_dev = to_dev(s_nat), *sr_dev = to_dev(s_reg);
        int32_t *dk_dev = to_dev(d_key), *dy_dev = to_dev(d_year);
        Name16* sname_dev = nullptr;
        cudaMalloc(&sname_dev, sizeof(Name16) * s_key.size());
        nation_names<<<64, 256, 0, stream>>>(sn_dev, names_dev, sname_dev, s_key.size());
        HashMap<int32_t, uint64_t> supplier_hashmap(s_key.size(), sk_dev);
        HashMap<int32_t, uint64_t> date_hashmap(d_key.size(), dk_dev);
        hash_map_build_pred_other<<<(unsigned)((s_key.size() + 511) / 512), 512, 0, stream>>>(
            supplier_hashmap, s_key.size(), golap::DirectKey<int32_t>(),
            golap::PredInfo<int32_t, EqPred>{sr_dev, EqPred{region}});
        hash_map_build_pred_other<<<(unsigned)((d_key.size() + 511) / 512), 512, 0, stream>>>(
            date_hashmap, d_key.size(), golap::DirectKey<int32_t>(),
            golap::PredInfo<int32_t, golap::RangePredFn<int32_t>>{dy_dev, golap::RangePredFn<int32_t>{ylo, yhi}});

        // ---- fact chunks: skip or decompress, then probe + aggregate (03.hpp:487-547)
        const uint64_t num_groups = 800;
        NationGroup* groups_dev = nullptr;
        uint64_t* aggs_dev = nullptr;
        cudaMalloc(&groups_dev, sizeof(NationGroup) * num_groups);
        cudaMalloc(&aggs_dev, 8 * num_groups);
        cudaMemsetAsync(aggs_dev, 0, 8 * num_groups, stream);
        golap::HashAggregate<NationGroup, uint64_t> hashagg(num_groups, groups_dev, aggs_dev);
        int32_t* buf[4];
        for (auto& b : buf) cudaMalloc(&b, chunk_bytes);
        auto md = golap::build_gpucomp_manager(ci_date), mc = golap::build_gpucomp_manager(ci_cust),
             ms = golap::build_gpucomp_manager(ci_supp), mr = golap::build_gpucomp_manager(ci_rev);
        golap::ChunkDecompressor dec[4] = {
            {chunk_bytes, nullptr, (char*)buf[0], false, false, *md, ci_date.chunk_size_vec},
            {chunk_bytes, nullptr, (char*)buf[1], false, false, *mc, ci_cust.chunk_size_vec},
            {chunk_bytes, nullptr, (char*)buf[2], false, false, *ms, ci_supp.chunk_size_vec},
            {chunk_bytes, nullptr, (char*)buf[3], false, false, *mr, ci_rev.chunk_size_vec}};
        uint64_t kept = 0;
        for (uint64_t c = 0; c < chunk_num; ++c) {
            if (!keep[c]) {
                for (auto& d : dec) d.skip_step(stream);
                continue;
            }
            ++kept;
            for (auto& d : dec) d.step(stream);
            const uint64_t rows = std::min(chunk_rows, n - c * chunk_rows);
            probe_aggregate<<<148, 512, 0, stream>>>(customer_hashmap, supplier_hashmap, date_hashmap, hashagg, buf[1],
                                                     buf[2], buf[0], buf[3], sname_dev, dy_dev, cust_buf, rows);
        }
        golap::gx_check(gx_scan_check(stream));
        hashagg.check();
        if (customer_hashmap.num_filled(stream) == 0 || supplier_hashmap.num_filled(stream) == 0) return 4;

        // ---- results: groups, and their total through Aggregate (core/agg.cuh)
        std::vector<NationGroup> groups(num_groups);
        std::vector<uint64_t> aggs(num_groups);
        std::vector<uint32_t> wrote(num_groups);
        cudaMemcpy(groups.data(), groups_dev, sizeof(NationGroup) * num_groups, cudaMemcpyDeviceToHost);
        cudaMemcpy(aggs.data(), aggs_dev, 8 * num_groups, cudaMemcpyDeviceToHost);
        cudaMemcpy(wrote.data(), hashagg.wrote_group, 4 * num_groups, cudaMemcpyDeviceToHost);
        uint64_t total = 0, ngroups = 0;
        for (uint64_t i = 0; i < num_groups; ++i) {
            if (!wrote[i]) continue;
            ++ngroups;
            total += aggs[i];
            // the reference fills the group supplier nation first (03.cuh:159)
            printf("g %d %d %d %llu\n", nation_of(groups[i].s_nation), nation_of(groups[i].c_nation),
                   (int)groups[i].d_year, (unsigned long long)aggs[i]);
        }
        uint64_t* total_dev = nullptr;
        cudaMalloc(&total_dev, 8);
        golap::Aggregate<uint64_t, uint64_t, Plus> sum(aggs_dev, total_dev, (uint32_t)num_groups, Plus{}, 0);
        sum.execute(stream);
        uint64_t agg_total = 0;
        cudaMemcpyAsync(&agg_total, total_dev, 8, cudaMemcpyDeviceToHost, stream);
        golap::cuda_check(cudaStreamSynchronize(stream), "sync");

        // ---- the same query through the fused scan (join tables with nation / year payloads)
        int32_t *ck_dev = to_dev(c_key), *cn_dev = to_dev(c_nat), *cr_dev = to_dev(c_reg);
        HashMap<int32_t, uint64_t> hc(n_cust), hs(s_key.size()), hd(d_key.size());
        hc.build(ck_dev, n_cust, {golap::RangePred{cr_dev, region, region}}, cn_dev, stream);
        hs.build(sk_dev, s_key.size(), {golap::RangePred{sr_dev, region, region}}, sn_dev, stream);
        hd.build(dk_dev, d_key.size(), {golap::RangePred{dy_dev, ylo, yhi}}, dy_dev, stream);
        golap::GroupTable gt(25 * 25 * (yhi - ylo + 1));
        gx_scan_plan plan{};
        plan.n_steps = 4;
        plan.steps[0] = gx_scan_step{ci_cust.column.get(), GX_STEP_PROBE, 0, 0, hc.handle(), 0, 25};
        plan.steps[1] = gx_scan_step{ci_supp.column.get(), GX_STEP_PROBE, 0, 0, hs.handle(), 0, 25};
        plan.steps[2] = gx_scan_step{ci_date.column.get(), GX_STEP_PROBE, 0, 0, hd.handle(), ylo,
                                     (uint32_t)(yhi - ylo + 1)};
        plan.steps[3] = gx_scan_step{ci_rev.column.get(), GX_STEP_VALUE, 0, 0, nullptr, 0, 0};
        plan.agg = GX_AGG_SUM;
        plan.groupby = gt.handle();
        plan.keep_chunks_dev = combined;
        golap::gx_check(gx_scan_sync(&plan, stream, nullptr));
        long long fused_total = 0;
        for (auto& kv : gt.read(4096, stream)) fused_total += kv.second;
        printf("groups=%llu total=%llu agg_total=%llu fused_total=%lld chunks=%llu/%llu minmax_ok=%d\n",
               (unsigned long long)ngroups, (unsigned long long)total, (unsigned long long)agg_total, fused_total,
               (unsigned long long)kept, (unsigned long long)chunk_num, minmax_ok);
        return total == agg_total && (long long)total == fused_total && minmax_ok ? 0 : 1;
    } catch (const std::exception& e) {
        fprintf(stderr, "error: %s\n", e.what());
        return 3;
    }
}
