// hashidx.cuh -- home slot of a key in the open-addressing lookup index
// (16-byte {key, value} slots) and the tags of its 8-byte-slot form.
//
// Host and device code share these functions (the host compiles them for the
// checks of its tests).  The index is an array of `cap` slots with
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

// INDEX_HASH with 8-byte slots {32-bit tag, f32 value} (FP32 tables whose keys
// vary in few bytes): the layer's constant bytes, the byte permutes that
// gather its varying bytes, and the tag layout
struct CompactHash {
    int on = 0;
    uint64_t cmask = 0, cval = 0;     // key & cmask == cval for every key of the layer
    uint32_t sel_lo = 0, sel_hi = 0;  // __byte_perm selectors gathering the varying bytes
    uint64_t vmask = 0;               // 2^v - 1, v = bits of the varying bytes
    int r = 0;                   // remainder bits kept in the tag (v - log2(cap), >= 0)
    int dbits = 0;               // tag bits of the probe distance + 1
    int lshift = 0;              // log2(cap) - v when v < log2(cap), else 0
};

__host__ __device__ __forceinline__ uint64_t cgb_make64(uint32_t hi, uint32_t lo) { return ((uint64_t)hi << 32) | lo; }

// ---- compact hash slots (FP32 tables) ---------------------------------------
// An FP32 table whose keys agree on most of their bytes (canonical boards of
// one formation hold the same 0xf bytes) is stored in 8-byte slots
// {32-bit tag, f32 value}: the key's varying bytes k' (v bits, 8 per varying
// byte) are mixed by a multiplication with an odd constant modulo 2^v, a bijection;
// the top c bits of the product pick the home slot of a table of 2^c slots and
// its low r = v - c bits ("remainder") go into the tag with the probe distance
// t + 1 of the slot: together they give back k', so a tag match is an exact
// key match.  The constant bytes are tested before any load.  Four slots share
// a 32-byte sector and the table takes half the bytes of 16-byte slots.
constexpr uint64_t COMPACT_MUL = 0x9E3779B97F4A7C15ull;

__host__ __device__ __forceinline__ uint64_t compact_varying(const CompactHash &c, uint64_t key)
{
    const uint32_t lo = (uint32_t)key, hi = (uint32_t)(key >> 32);
#ifdef __CUDA_ARCH__
    const uint64_t kp = cgb_make64(__byte_perm(lo, hi, c.sel_hi), __byte_perm(lo, hi, c.sel_lo));
#else
    auto perm = [](uint32_t a, uint32_t b, uint32_t sel) {
        const uint64_t x = ((uint64_t)b << 32) | a;
        uint32_t o = 0;
        for (int i = 0; i < 4; i++) o |= (uint32_t)((x >> (8 * ((sel >> (4 * i)) & 7))) & 0xFF) << (8 * i);
        return o;
    };
    const uint64_t kp = cgb_make64(perm(lo, hi, c.sel_hi), perm(lo, hi, c.sel_lo));
#endif
    return kp & c.vmask;
}

// home slot of a key; *tag0 = its tag at probe distance 0
__host__ __device__ __forceinline__ uint64_t compact_home(const CompactHash &c, uint64_t key, uint32_t *tag0)
{
    const uint64_t h = (compact_varying(c, key) * COMPACT_MUL) & c.vmask;
    const uint32_t rem = c.r ? (uint32_t)h & ((1u << c.r) - 1u) : 0u;
    *tag0 = (rem << c.dbits) | 1u;
    return c.lshift ? (h << c.lshift) : (h >> c.r);
}

// The plan of a layer of n keys whose AND and OR over all keys are given: the
// table is the power of two at or above 2n (at least 64 slots; load 25-50 %);
// on = 0 when the remainder needs more than 26 bits (a tag of 32 bits keeps at
// least 6 for the probe distance) or no byte varies.
inline CompactHash plan_compact(uint64_t and_bits, uint64_t or_bits, uint64_t n, int *log2_cap)
{
    CompactHash ch;
    const uint64_t vary = and_bits ^ or_bits;
    int nv = 0;
    uint32_t sel[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    for (int b = 0; b < 8; b++) {
        if ((vary >> (8 * b)) & 0xFF) sel[nv++] = (uint32_t)b;
        else ch.cmask |= 0xFFull << (8 * b);
    }
    ch.cval = and_bits & ch.cmask;
    int cbits = 6;
    while ((1ull << cbits) < 2 * n) cbits++;
    *log2_cap = cbits;
    const int v = 8 * nv;
    ch.r = v > cbits ? v - cbits : 0;
    ch.lshift = v < cbits ? cbits - v : 0;
    if (nv == 0 || ch.r > 26) return ch;
    ch.dbits = 32 - ch.r < 16 ? 32 - ch.r : 16;
    for (int i = 0; i < 4; i++) {
        ch.sel_lo |= sel[i] << (4 * i);
        ch.sel_hi |= sel[4 + i] << (4 * i);
    }
    ch.vmask = v >= 64 ? ~0ull : (1ull << v) - 1;
    ch.on = 1;
    return ch;
}

}  // namespace cgb
