/* Prototypes of the public liblz4 block API used by the reference's
 * LZ4CPUManager (core/comp_cpu.hpp:22-32).  The image ships the shared
 * library liblz4.so.1 (1.9.4) without its header; the oracle harness links it
 * directly.  Signatures follow liblz4's documented public interface. */
#pragma once
#ifdef __cplusplus
extern "C" {
#endif
int LZ4_versionNumber(void);
int LZ4_compressBound(int inputSize);
int LZ4_compress_default(const char* src, char* dst, int srcSize, int dstCapacity);
int LZ4_decompress_safe(const char* src, char* dst, int compressedSize, int dstCapacity);
int LZ4_decompress_safe_partial(const char* src, char* dst, int srcSize, int targetOutputSize, int dstCapacity);
#ifdef __cplusplus
}
#endif
