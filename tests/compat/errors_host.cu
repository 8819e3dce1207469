// The drop-in layer's host-side error behaviour, without a GPU: bad ingest
// arguments throw std::runtime_error carrying the library's message (the
// reference's checkCudaErrors would exit the process instead).
#include <cstdio>
#include <cstring>

#include "golap_compat/golap_compat.cuh"

template <class F>
static int expect_throw(const char* what, F f) {
    try {
        f();
    } catch (const std::runtime_error& e) {
        std::printf("%s: threw: %s\n", what, e.what());
        return 0;
    }
    std::printf("%s: did not throw\n", what);
    return 1;
}

int main() {
    int bad = 0;
    const int32_t* none = nullptr;
    bad += expect_throw("host ingest of a null column",
                        [&] { golap::prepare_compressed(none, 10, 4000000, "LZ4"); });
    bad += expect_throw("device ingest of a null column",
                        [&] { golap::prepare_compressed_device(none, 10, 4000000, "Cascaded"); });
    const int32_t* fake = reinterpret_cast<const int32_t*>(0x1000);  // never dereferenced
    bad += expect_throw("device ingest of an empty column",
                        [&] { golap::prepare_compressed_device(fake, 0, 4000000, "LZ4"); });
    bad += expect_throw("device ingest with oversized blocks",
                        [&] { golap::prepare_compressed_device(fake, 10, 4000000, "LZ4", 0, 1 << 20); });
    return bad;
}
