// q1_pipeline.cu -- a GOLAP-style Q1 pipeline written against the drop-in
// header include/golap_compat/golap_compat.cuh, in the shape of the
// reference's query1 worker loop (usecases/ssb/queries/01.hpp:350-424) and
// its kernel pipeline_q1_lineorder (usecases/ssb/queries/01.cuh:27-54):
// per chunk either skip_step (pruned by MetaChecker) or decompress the four
// columns and launch the probe/filter/sum kernel.  The same query also runs
// through the fused gx_scan.  Input: raw int32 column files; prints
// "pipeline=<sum> fused=<sum> chunks=<kept>/<total>".
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "golap_compat/golap_compat.cuh"

using golap::HashMap;

__global__ void pipeline_q1(HashMap<int32_t, uint64_t> hashmap, const int32_t* orderdate, const int32_t* discount,
                            int32_t dlo, int32_t dhi, const int32_t* quantity, int32_t qlo, int32_t qhi,
                            const int32_t* extprice, unsigned long long* agg, uint64_t num) {
    for (uint64_t r = blockDim.x * (uint64_t)blockIdx.x + threadIdx.x; r < num; r += (uint64_t)blockDim.x * gridDim.x) {
        if (discount[r] < dlo || discount[r] > dhi || quantity[r] < qlo || quantity[r] > qhi) continue;
        if (hashmap.probe((uint64_t)orderdate[r]) == (uint64_t)-1) continue;
        atomicAdd(agg, (unsigned long long)((int64_t)extprice[r] * discount[r]));
    }
}

static std::vector<int32_t> read_col(const char* path) {
    FILE* f = fopen(path, "rb");
    if (!f) {
        perror(path);
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

int main(int argc, char** argv) {
    if (argc != 10) {
        fprintf(stderr, "usage: %s dir d_key.bin d_ok.bin date_lo date_hi dlo dhi qlo qhi\n", argv[0]);
        return 2;
    }
    std::string dir = argv[1];
    auto od = read_col((dir + "/date_key.bin").c_str());
    auto disc = read_col((dir + "/discount.bin").c_str());
    auto qty = read_col((dir + "/quantity.bin").c_str());
    auto price = read_col((dir + "/extended_price.bin").c_str());
    auto dkey = read_col(argv[2]);
    auto dok = read_col(argv[3]);
    const int32_t date_lo = atoi(argv[4]), date_hi = atoi(argv[5]);
    const int32_t dlo = atoi(argv[6]), dhi = atoi(argv[7]), qlo = atoi(argv[8]), qhi = atoi(argv[9]);
    const uint64_t n = od.size(), chunk_rows = 1000000, chunk_bytes = chunk_rows * 4;
    cudaStream_t stream;
    cudaStreamCreate(&stream);
    try {
        // ingest (prepare_compressed)
        auto ci_date = golap::prepare_compressed(od.data(), n, chunk_bytes, "Cascaded", 1, stream);
        auto ci_disc = golap::prepare_compressed(disc.data(), n, chunk_bytes, "LZ4", 1, stream);
        auto ci_qty = golap::prepare_compressed(qty.data(), n, chunk_bytes, "LZ4", 1, stream);
        auto ci_price = golap::prepare_compressed(price.data(), n, chunk_bytes, "LZ4", 1, stream);
        const uint64_t chunk_num = ci_date.chunk_num();

        // date hash table build (hash_map_build_pred_other, 01.hpp:241)
        int32_t *d_key, *d_ok;
        cudaMalloc(&d_key, 4 * dkey.size());
        cudaMalloc(&d_ok, 4 * dok.size());
        cudaMemcpy(d_key, dkey.data(), 4 * dkey.size(), cudaMemcpyHostToDevice);
        cudaMemcpy(d_ok, dok.data(), 4 * dok.size(), cudaMemcpyHostToDevice);
        HashMap<int32_t, uint64_t> hashmap(dkey.size());
        hashmap.build(d_key, dkey.size(), {golap::RangePred{d_ok, 1, 1}}, nullptr, stream);

        // pruning (MetaChecker::add_minmax, 01.hpp:263-281)
        golap::MinMaxMeta<int32_t> meta(ci_date);
        uint16_t *combined, *tmp;
        cudaMalloc(&combined, 2 * chunk_num);
        cudaMalloc(&tmp, 2 * chunk_num);
        golap::MetaChecker checker(1, chunk_num, combined, tmp, stream);
        checker.add_minmax(meta, date_lo, date_hi);
        std::vector<uint16_t> keep(chunk_num);
        cudaMemcpyAsync(keep.data(), combined, 2 * chunk_num, cudaMemcpyDeviceToHost, stream);
        cudaStreamSynchronize(stream);

        // per-chunk worker loop (01.hpp:350-424)
        int32_t* buf[4];
        for (auto& b : buf) cudaMalloc(&b, chunk_bytes);
        golap::ChunkDecompressor dec[4] = {{ci_date, (char*)buf[0], false}, {ci_disc, (char*)buf[1], false},
                                           {ci_qty, (char*)buf[2], false}, {ci_price, (char*)buf[3], false}};
        unsigned long long* agg;
        cudaMalloc(&agg, 8);
        cudaMemsetAsync(agg, 0, 8, stream);
        uint64_t kept = 0;
        for (uint64_t c = 0; c < chunk_num; ++c) {
            if (!keep[c]) {
                for (auto& d : dec) d.skip_step(stream);
                continue;
            }
            ++kept;
            for (auto& d : dec) d.step(stream);
            const uint64_t rows = std::min(chunk_rows, n - c * chunk_rows);
            pipeline_q1<<<148, 512, 0, stream>>>(hashmap, buf[0], buf[1], dlo, dhi, buf[2], qlo, qhi, buf[3], agg, rows);
        }
        unsigned long long pipe = 0;
        cudaMemcpyAsync(&pipe, agg, 8, cudaMemcpyDeviceToHost, stream);
        golap::gx_check(gx_scan_check(stream));

        // the same query through the fused scan
        int64_t* res;
        cudaMalloc(&res, 8);
        cudaMemsetAsync(res, 0, 8, stream);
        gx_scan_plan plan{};
        plan.n_steps = 4;
        plan.steps[0] = gx_scan_step{ci_date.column.get(), GX_STEP_PROBE, 0, 0, hashmap.handle(), 0, 0};
        plan.steps[1] = gx_scan_step{ci_disc.column.get(), GX_STEP_FILTER | GX_STEP_CARRY, dlo, dhi, nullptr, 0, 0};
        plan.steps[2] = gx_scan_step{ci_qty.column.get(), GX_STEP_FILTER, qlo, qhi, nullptr, 0, 0};
        plan.steps[3] = gx_scan_step{ci_price.column.get(), GX_STEP_VALUE, 0, 0, nullptr, 0, 0};
        plan.agg = GX_AGG_SUM_PRODUCT;
        plan.keep_chunks_dev = combined;
        plan.result_dev = res;
        golap::gx_check(gx_scan_sync(&plan, stream, nullptr));
        int64_t fused = 0;
        cudaMemcpy(&fused, res, 8, cudaMemcpyDeviceToHost);
        printf("pipeline=%llu fused=%lld chunks=%llu/%llu\n", pipe, (long long)fused, (unsigned long long)kept,
               (unsigned long long)chunk_num);
        return pipe == (unsigned long long)fused ? 0 : 1;
    } catch (const std::exception& e) {
        fprintf(stderr, "error: %s\n", e.what());
        return 3;
    }
}
