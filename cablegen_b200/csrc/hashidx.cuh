// hashidx.cuh -- home slot of a key in the open-addressing lookup index.
//
// Host and device code share these functions (the host compiles them for the
// capacity checks of its tests).  The index is an array of `cap` slots with
// linear probing; a key's home slot is a hash of the key range-reduced into
// [0, cap) by a multiply-high.  Below 2^32 slots a 32-bit hash and a 32x32
// multiply-high suffice; from 2^32 slots on (layers of more than ~1.9e9
// boards at a 45 % load) a 64-bit hash and a 64x64 multiply-high keep every
// slot of the table reachable.
#pragma once
#include <stdint.h>

namespace cgb {

// 32-bit hash of a board: both halves multiplied by odd constants, then
// xor-shift / multiply rounds (constants of the murmur3 and xxhash32
// finalisers)
__host__ __device__ __forceinline__ uint32_t hash32(uint64_t k)
{
    uint32_t x = ((uint32_t)(k >> 32) * 0x9E3779B1u) ^ ((uint32_t)k * 0x85EBCA77u);
    x ^= x >> 15;
    x *= 0xC2B2AE3Du;
    x ^= x >> 13;
    return x;
}

// 64-bit hash: the SplitMix64 finaliser (Steele, Lea, Flood 2014)
__host__ __device__ __forceinline__ uint64_t hash64(uint64_t z)
{
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

__host__ __device__ __forceinline__ uint64_t mulhi64(uint64_t a, uint64_t b)
{
#ifdef __CUDA_ARCH__
    return __umul64hi(a, b);
#else
    return (uint64_t)(((unsigned __int128)a * b) >> 64);
#endif
}

// home slot in [0, cap), cap >= 1
__host__ __device__ __forceinline__ uint64_t home_slot(uint64_t key, uint64_t cap)
{
    if (cap <= 0xFFFFFFFFull) return ((uint64_t)hash32(key) * cap) >> 32;
    return mulhi64(hash64(key), cap);
}

// slots for n keys at a load factor of at most pct percent, a multiple of 64
__host__ __device__ __forceinline__ uint64_t hash_capacity_for(uint64_t n, uint64_t pct)
{
    return ((n * 100 + pct - 1) / pct + 63) / 64 * 64;
}

}  // namespace cgb
