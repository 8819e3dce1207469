/* Declaration-only stand-in for <snappy.h> (absent in this image).  The
 * reference's SnappyCPUManager (core/comp_cpu.hpp:34-49) names these two
 * functions; the oracle harness never constructs it. */
#pragma once
#include <cstddef>
namespace snappy {
bool RawUncompress(const char* compressed, size_t compressed_length, char* uncompressed);
void RawCompress(const char* input, size_t input_length, char* compressed, size_t* compressed_length);
}
