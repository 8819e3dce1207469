/*
 * gx_hash.h -- the hash functions and slot formats of the device join and
 * group tables, shared by libgx.so and by code that probes the tables from
 * its own kernels (include/golap_compat/golap_compat.cuh).
 *
 * Join table slot (64 bit): low 32 bits = key (int32), high 32 bits =
 *   payload (int32); an empty slot holds key INT32_MIN (a reserved key).
 * Group table: two arrays of int64 (keys, sums); an empty key is INT64_MIN.
 * Both tables use linear probing from the hash below over a power-of-two
 * capacity 2^log2cap.
 * Dense join table (GX_HT_DENSE): slot 0 is a header, low 32 bits = base
 * (int32, the smallest key), high 32 bits = span (keys base .. base+span-1);
 * slot 1 + (key - base) holds the key's slot as above, or an empty slot.
 */
#ifndef GX_HASH_H
#define GX_HASH_H
#include <stdint.h>

#if defined(__CUDACC__)
#define GX_HASH_FN __host__ __device__ static inline
#else
#define GX_HASH_FN static inline
#endif

/* Fibonacci (multiplicative) hashing of a 32-bit key. */
GX_HASH_FN uint32_t gx_hash32(int32_t key, uint32_t log2cap) {
    uint32_t h = (uint32_t)key * 0x9E3779B1u;
    return log2cap ? (h >> (32 - log2cap)) : 0u;
}
/* Fibonacci hashing of a 64-bit key. */
GX_HASH_FN uint32_t gx_hash64(int64_t key, uint32_t log2cap) {
    uint64_t h = (uint64_t)key * 0x9E3779B97F4A7C15ull;
    return log2cap ? (uint32_t)(h >> (64 - log2cap)) : 0u;
}

#define GX_EMPTY_KEY ((int32_t)INT32_MIN)
#define GX_EMPTY_GROUP ((int64_t)INT64_MIN)

#endif /* GX_HASH_H */
