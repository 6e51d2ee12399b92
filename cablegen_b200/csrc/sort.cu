// sort.cu -- device-wide u64 sort, unique and merge for board sets.
//
// Replaces the reference's per-thread fluxsort + serial k-way merge
// (src/array.c:246-291, inc/external/fluxsort.h:112-120): layers must come out
// ascending and duplicate-free, bit-for-bit.
//
// * LSD radix sort with 8-bit digits in the single-pass "onesweep" form
//   (Adinets & Merrill 2022): one histogram pass for all eight digits, then
//   one pass per non-constant digit that ranks a 4096-key tile in shared
//   memory and finds its global bin offsets by a decoupled look-back.  Digits
//   on which every key agrees (the 0xff prefix that canonical formation
//   boards share) are skipped.
// * unique: adjacent-difference flags, ballot/popc compaction, decoupled
//   look-back for the tile prefix.
// * merge_unique: merge-path partition of two sorted runs, per-thread
//   sequential merge in shared memory, the same compaction (repeats inside a
//   run are dropped like repeats across the runs).
//
// Every look-back wait is bounded (SPIN_LIMIT polls); on timeout the kernel
// sets ERR_LOOKBACK_TIMEOUT in the error word and finishes without waiting.
#include "common.cuh"
#include "engine.h"
#include <cstring>

namespace cgb {

constexpr int SORT_THREADS = 256;
constexpr int SORT_KPT = 16;
constexpr int SORT_TILE = SORT_THREADS * SORT_KPT;  // 4096 keys per tile
constexpr int RADIX = 256;
constexpr u32 LB_AGG = 1u << 30, LB_PRE = 2u << 30, LB_MASK = (1u << 30) - 1;

constexpr int UNQ_THREADS = 256;
constexpr int UNQ_KPT = 16;
constexpr int UNQ_TILE = UNQ_THREADS * UNQ_KPT;

constexpr int MRG_THREADS = 256;
constexpr int MRG_KPT = 16;
constexpr int MRG_TILE = MRG_THREADS * MRG_KPT;

// Walk back over the look-back words of one bin (or of the whole tile),
// LB_BATCH predecessors per round trip, polling with a short sleep while a
// predecessor has not published.  Each word carries its own flag, so relaxed
// accesses suffice.  Returns the sum of the predecessors' counts up to and
// including the first inclusive prefix.
#ifndef LB_BATCH
#define LB_BATCH 4
#endif
// Polls a look-back wait makes before it gives up (SPIN_LIMIT unless a test
// lowers it), and a test switch that keeps tile 0 of a digit pass from
// publishing its counts: tile 1 then waits on a flag that nothing sets, runs
// out of polls and reports ERR_LOOKBACK_TIMEOUT (the bounded-wait path).
__device__ u32 g_spin_limit = SPIN_LIMIT;
__device__ u32 g_hold_first_tile = 0;

__device__ __forceinline__ u32 lookback_sum(const u32 *words, u64 stride, int j, u32 *err)
{
    u32 excl = 0;
    u32 spins = 0;
    const u32 limit = g_spin_limit;
    while (j >= 0) {
        u32 v[LB_BATCH];
#pragma unroll
        for (int q = 0; q < LB_BATCH; q++) v[q] = (j - q >= 0) ? ld_relaxed(words + (u64)(j - q) * stride) : LB_PRE;
        bool done = false, stalled = false;
#pragma unroll
        for (int q = 0; q < LB_BATCH; q++) {
            if (done || stalled) continue;
            const u32 flag = v[q] & ~LB_MASK;
            if (flag == 0) {
                stalled = true;  // not published yet: poll again from here
            } else {
                excl += v[q] & LB_MASK;
                if (flag == LB_PRE) done = true;
                else j--;
            }
        }
        if (done) break;
        if (stalled) {
            if (++spins > limit) {
                atomicOr(err, ERR_LOOKBACK_TIMEOUT);
                break;
            }
            __nanosleep(32);
        }
    }
    return excl;
}

__device__ __forceinline__ u64 ld_relaxed64(const u64 *p)
{
    u64 v;
    asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_relaxed64(u64 *p, u64 v)
{
    asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

// Warp-wide form of the walk back over one count per tile, called by all 32
// lanes of one warp: lane i reads the word of tile j - i, so one round trip
// covers 32 predecessors.  The words from tile j down to the nearest inclusive
// prefix (or down to the first one not yet published, which is polled again)
// are summed with a warp reduction.  Every lane returns the same prefix.
template <typename W>
__device__ __forceinline__ W warp_lookback_sum(const W *words, int j, u32 *err)
{
    constexpr W PRE = (W)2 << (8 * sizeof(W) - 2);
    constexpr W MASK = ((W)1 << (8 * sizeof(W) - 2)) - 1;
    const int lane = threadIdx.x & 31;
    W excl = 0;
    u32 spins = 0;
    const u32 limit = g_spin_limit;
    while (j >= 0) {
        const int k = j - lane;
        W v;
        if (k >= 0) {
            if constexpr (sizeof(W) == 8) v = ld_relaxed64((const u64 *)words + k);
            else v = ld_relaxed((const u32 *)words + k);
        } else {
            v = PRE;  // before tile 0: an empty inclusive prefix ends the walk
        }
        const W flag = v & ~MASK;
        const u32 pre = __ballot_sync(0xffffffffu, flag == PRE);
        const u32 unready = __ballot_sync(0xffffffffu, flag == 0);
        // lanes that count: up to the nearest inclusive prefix, and short of
        // the first word not yet published
        const u32 upto = pre ? ((pre & (0u - pre)) << 1) - 1 : 0xffffffffu;
        const u32 stop = unready & upto;
        const u32 take = stop ? (stop & (0u - stop)) - 1 : upto;
        W c = ((take >> lane) & 1) ? (v & MASK) : (W)0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
        excl += c;
        if (!stop && pre) break;
        j -= __popc(take);
        // a round trip to L2 per poll is the wait; the poll count bounds it
        if (stop && ++spins > limit) {
            if (lane == 0) atomicOr(err, ERR_LOOKBACK_TIMEOUT);
            break;
        }
    }
    return excl;
}


// ---------------------------------------------------------------------------
// histogram of all eight byte digits in one pass
__global__ void __launch_bounds__(256) digit_histogram_kernel(const u64 *__restrict__ keys, u64 n,
                                                              u32 *__restrict__ hist)
{
    __shared__ u32 sh[2][8 * RADIX];  // two copies halve same-bin contention
    for (int i = threadIdx.x; i < 2 * 8 * RADIX; i += blockDim.x) (&sh[0][0])[i] = 0;
    __syncthreads();
    u32 *mine = sh[(threadIdx.x >> 5) & 1];
    const int lane = threadIdx.x & 31;
    const u64 stride = (u64)gridDim.x * blockDim.x;
    for (u64 base = (u64)blockIdx.x * blockDim.x; base < n; base += stride) {
        const u64 i = base + threadIdx.x;
        const bool ok = i < n;
        const u64 k = ok ? keys[i] : 0;
        const u32 act = __ballot_sync(0xffffffffu, ok);
#pragma unroll
        for (int d = 0; d < 8; d++) {
            const u32 dig = (u32)(k >> (8 * d)) & 0xFF;
            // a warp whose keys all share this digit adds once
            const u32 first = __shfl_sync(0xffffffffu, dig, 0);
            const bool uniform = __all_sync(0xffffffffu, !ok || dig == first) && act == 0xffffffffu;
            if (uniform) {
                if (lane == 0) atomicAdd(&mine[d * RADIX + dig], 32u);
            } else if (ok) {
                atomicAdd(&mine[d * RADIX + dig], 1u);
            }
        }
    }
    __syncthreads();
    for (int i = threadIdx.x; i < 8 * RADIX; i += blockDim.x) {
        const u32 v = sh[0][i] + sh[1][i];
        if (v) atomicAdd(&hist[i], v);
    }
}

// the exclusive prefix of each digit's histogram (block d scans digit d): the
// global start of every bin, read by the byte-digit passes instead of a block
// scan per tile
__global__ void __launch_bounds__(RADIX) digit_offsets_kernel(const u32 *__restrict__ hist, u32 *__restrict__ offs)
{
    __shared__ u32 scratch[33];
    u32 total;
    offs[blockIdx.x * RADIX + threadIdx.x] =
        block_exclusive_scan<u32>(hist[blockIdx.x * RADIX + threadIdx.x], scratch, &total);
}

// ---------------------------------------------------------------------------
// one digit pass: src -> dst, stable by the digit at `shift`
__global__ void __launch_bounds__(SORT_THREADS) onesweep_kernel(const u64 *__restrict__ src, u64 *__restrict__ dst,
                                                                u32 n, int shift, const u32 *__restrict__ digit_hist,
                                                                u32 *lookback, u32 *tile_counter, u32 *err)
{
    __shared__ u64 keys_sh[SORT_TILE];
    __shared__ u32 warp_hist[SORT_THREADS / 32][RADIX];
    __shared__ u32 bin_local[RADIX];
    __shared__ u32 bin_global[RADIX];
    __shared__ u32 scan_scratch[33];
    __shared__ u32 tile_sh;

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (threadIdx.x == 0) tile_sh = atomicAdd(tile_counter, 1u);
    for (int i = threadIdx.x; i < (SORT_THREADS / 32) * RADIX; i += SORT_THREADS) (&warp_hist[0][0])[i] = 0;
    __syncthreads();
    const u32 tile = tile_sh;
    const u32 tile_base = tile * SORT_TILE;
    const u32 warp_base = tile_base + warp * (SORT_KPT * 32);

    u64 k[SORT_KPT];
    u32 rank[SORT_KPT];
#pragma unroll
    for (int i = 0; i < SORT_KPT; i++) {
        const u32 idx = warp_base + i * 32 + lane;
        k[i] = idx < n ? src[idx] : 0;
    }
    const u32 lt = lanemask_lt();
#pragma unroll
    for (int i = 0; i < SORT_KPT; i++) {
        const u32 idx = warp_base + i * 32 + lane;
        const bool ok = idx < n;
        const u32 d = ok ? (u32)(k[i] >> shift) & 0xFF : 0x100u;
        const u32 peers = __match_any_sync(0xffffffffu, d);
        const int leader = __ffs(peers) - 1;
        u32 base = 0;
        if (ok && lane == leader) {
            base = warp_hist[warp][d];
            warp_hist[warp][d] = base + __popc(peers);
        }
        base = __shfl_sync(0xffffffffu, base, leader);
        rank[i] = base + __popc(peers & lt);
        __syncwarp();
    }
    __syncthreads();

    // per bin: warp offsets inside the tile, tile count, look-back
    const u32 d = threadIdx.x;  // SORT_THREADS == RADIX
    u32 cnt = 0;
#pragma unroll
    for (int w = 0; w < SORT_THREADS / 32; w++) {
        const u32 c = warp_hist[w][d];
        warp_hist[w][d] = cnt;
        cnt += c;
    }
    u32 *lb = lookback + (u64)tile * RADIX + d;
    u32 excl = 0;
    if (tile == 0) {
        if (!g_hold_first_tile) st_relaxed(lb, LB_PRE | cnt);
    } else {
        st_relaxed(lb, LB_AGG | cnt);
        excl = lookback_sum(lookback + d, RADIX, (int)tile - 1, err);
        st_relaxed(lb, LB_PRE | (excl + cnt));
    }
    u32 total;
    const u32 gexcl = block_exclusive_scan<u32>(digit_hist[d], scan_scratch, &total);
    const u32 lstart = block_exclusive_scan<u32>(cnt, scan_scratch, &total);
    bin_local[d] = lstart;
    bin_global[d] = gexcl + excl;
    __syncthreads();

#pragma unroll
    for (int i = 0; i < SORT_KPT; i++) {
        const u32 idx = warp_base + i * 32 + lane;
        if (idx < n) {
            const u32 dd = (u32)(k[i] >> shift) & 0xFF;
            keys_sh[bin_local[dd] + warp_hist[warp][dd] + rank[i]] = k[i];
        }
    }
    __syncthreads();
    const u32 tile_n = min((u32)SORT_TILE, n - tile_base);
    for (u32 j = threadIdx.x; j < tile_n; j += SORT_THREADS) {
        const u64 key = keys_sh[j];
        const u32 dd = (u32)(key >> shift) & 0xFF;
        const u32 g = bin_global[dd] + (j - bin_local[dd]);
        if (g < n) dst[g] = key;
        else atomicOr(err, ERR_CAPACITY);
    }
}

// ---------------------------------------------------------------------------
// Second form of the digit pass: lanes find their equal-digit peers with eight
// ballots (one per digit bit) instead of a match instruction, ranks are packed
// two per register so four CTAs fit per SM, and the tile is scattered into
// shared memory before the look-back so that wait overlaps useful work.
// Walk back over the per-tile look-back words of one bin, eight predecessors
// per round trip: the eight loads are independent, so a long walk costs one
// latency per eight tiles instead of one per tile.  Returns the sum of the
// predecessors' counts up to and including the first inclusive prefix.
constexpr int BAL_KPT = 16;
constexpr int BAL_TILE = SORT_THREADS * BAL_KPT;  // 4096 keys per tile

// the digit of a pass: 8 bits of the key, or (batched sweeps) the formation
// id, which orders a layer holding several formations by formation
struct ShiftDigit {
    int shift;
    __device__ __forceinline__ u32 operator()(u64 k) const { return (u32)(k >> shift) & 0xFF; }
};
struct FormationDigit {
    const unsigned char *fid;
    __device__ __forceinline__ u32 operator()(u64 k) const { return __ldg(fid + fixed_pattern(k)); }
};

template <class Digit>
__global__ void __launch_bounds__(SORT_THREADS, 5)
    onesweep_ballot_kernel(const u64 *__restrict__ src, u64 *__restrict__ dst, u32 n, Digit digit,
                           const u32 *__restrict__ digit_hist, u32 *lookback, u32 *tile_counter, u32 *err)
{
    __shared__ u64 keys_sh[BAL_TILE];
    __shared__ u32 warp_hist[SORT_THREADS / 32][RADIX];
    __shared__ u32 bin_local[RADIX];
    __shared__ u32 bin_global[RADIX];
    __shared__ u32 scan_scratch[33];
    __shared__ u32 tile_sh;

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (threadIdx.x == 0) tile_sh = atomicAdd(tile_counter, 1u);
    for (int i = threadIdx.x; i < (SORT_THREADS / 32) * RADIX; i += SORT_THREADS) (&warp_hist[0][0])[i] = 0;
    __syncthreads();
    const u32 tile = tile_sh;
    const u32 tile_base = tile * BAL_TILE;
    const u32 warp_base = tile_base + warp * (BAL_KPT * 32);

    // only the digits stay in registers (four per word); the keys are read
    // again for the local scatter, from L2
    u32 dg[BAL_KPT / 4];
#pragma unroll
    for (int i = 0; i < BAL_KPT; i++) {
        const u32 idx = warp_base + i * 32 + lane;
        const u32 dd = idx < n ? digit(src[idx]) : 0;
        if (i % 4 == 0) dg[i / 4] = dd;
        else dg[i / 4] |= dd << (8 * (i % 4));
    }
    const u32 lt = lanemask_lt();
    u32 rank2[BAL_KPT / 2];
#pragma unroll
    for (int i = 0; i < BAL_KPT; i++) {
        const u32 idx = warp_base + i * 32 + lane;
        const u32 valid = __ballot_sync(0xffffffffu, idx < n);
        const u32 d = (dg[i / 4] >> (8 * (i % 4))) & 0xFF;
        u32 peers = valid;
#pragma unroll
        for (int j = 0; j < 8; j++) {
            const u32 bj = __ballot_sync(0xffffffffu, (d >> j) & 1);
            peers &= ((d >> j) & 1) ? bj : ~bj;
        }
        const u32 base = warp_hist[warp][d];   // every peer reads the same word
        __syncwarp();
        if (idx < n && (peers & lt) == 0) warp_hist[warp][d] = base + __popc(peers);
        __syncwarp();
        const u32 r = base + __popc(peers & lt);
        if (i & 1) rank2[i >> 1] |= r << 16;
        else rank2[i >> 1] = r;
    }
    __syncthreads();

    // per bin: warp offsets inside the tile, tile count; publish the aggregate
    const u32 d = threadIdx.x;  // SORT_THREADS == RADIX
    u32 cnt = 0;
#pragma unroll
    for (int w = 0; w < SORT_THREADS / 32; w++) {
        const u32 c = warp_hist[w][d];
        warp_hist[w][d] = cnt;
        cnt += c;
    }
    u32 *lb = lookback + (u64)tile * RADIX + d;
    if (tile != 0 || !g_hold_first_tile) st_relaxed(lb, (tile == 0 ? LB_PRE : LB_AGG) | cnt);
    u32 total;
    const u32 lstart = block_exclusive_scan<u32>(cnt, scan_scratch, &total);
    bin_local[d] = lstart;
    __syncthreads();
    // local scatter: the tile sorted by this digit, in shared memory
#pragma unroll
    for (int i = 0; i < BAL_KPT; i++) {
        const u32 idx = warp_base + i * 32 + lane;
        if (idx < n) {
            const u64 key = src[idx];
            const u32 dd = (dg[i / 4] >> (8 * (i % 4))) & 0xFF;
            const u32 r = (rank2[i >> 1] >> ((i & 1) * 16)) & 0xFFFF;
            keys_sh[bin_local[dd] + warp_hist[warp][dd] + r] = key;
        }
    }
    // look-back for this bin's global offset
    u32 excl = 0;
    if (tile != 0) {
        excl = lookback_sum(lookback + d, RADIX, (int)tile - 1, err);
        st_relaxed(lb, LB_PRE | (excl + cnt));
    }
    const u32 gexcl = block_exclusive_scan<u32>(digit_hist[d], scan_scratch, &total);
    bin_global[d] = gexcl + excl;
    __syncthreads();
    const u32 tile_n = min((u32)BAL_TILE, n - tile_base);
    for (u32 j = threadIdx.x; j < tile_n; j += SORT_THREADS) {
        const u64 key = keys_sh[j];
        const u32 dd = digit(key);
        const u32 g = bin_global[dd] + (j - bin_local[dd]);
        if (g < n) dst[g] = key;
        else atomicOr(err, ERR_CAPACITY);
    }
}

// ---------------------------------------------------------------------------
// Third form of the ballot pass, for byte digits of the key: the tile's body
// is specialised for full tiles (no bounds tests on all but the last tile),
// the ranking phase reads only the 32-bit word that holds the digit, digits
// come out of words with one byte permute, and each bin keeps one combined
// offset (global start - local start) for the final write.  THREADS x 16 keys
// per tile: 256 threads (4096 keys, five CTAs per SM) or 512 (8192 keys, two
// CTAs per SM, half the per-tile look-back and scans per key).
template <int THREADS>
struct BytePassSmem {
    static constexpr int TILE = THREADS * BAL_KPT;
    u64 keys[TILE];
    u32 warp_hist[THREADS / 32][RADIX];
    u32 bin_local[RADIX];
    u32 bin_delta[RADIX];
    u32 scan[33];
    u32 tile;
};

template <int THREADS, bool FULL, bool MATCH>
__device__ __forceinline__ void byte_pass_tile(const u64 *__restrict__ src, u64 *__restrict__ dst, u32 n, int shift,
                                               const u32 *__restrict__ bin_base, u32 *lookback, u32 tile, u32 *err,
                                               BytePassSmem<THREADS> &S)
{
    constexpr u32 TILE = (u32)BytePassSmem<THREADS>::TILE;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const u32 tile_base = tile * TILE;
    const u32 warp_base = tile_base + warp * (BAL_KPT * 32);
    const u32 *src_w = (const u32 *)src + (shift >= 32 ? 1 : 0);   // little-endian words of the keys
    const u32 sel = 0x4440u | (u32)((shift >> 3) & 3);              // the digit's byte, zero above it
    u32 dg[BAL_KPT / 4];
#pragma unroll
    for (int i = 0; i < BAL_KPT; i++) {
        const u32 idx = warp_base + i * 32 + lane;
        const u32 dd = (FULL || idx < n) ? __byte_perm(__ldg(src_w + 2 * (u64)idx), 0, sel) : 0u;
        if (i % 4 == 0) dg[i / 4] = dd;
        else dg[i / 4] |= dd << (8 * (i % 4));
    }
    const u32 lt = lanemask_lt();
    u32 rank2[BAL_KPT / 2];
#pragma unroll
    for (int i = 0; i < BAL_KPT; i++) {
        const u32 d = __byte_perm(dg[i / 4], 0, 0x4440u | (u32)(i % 4));
        u32 peers;
        if (FULL) {
            peers = 0xffffffffu;
        } else {
            const u32 idx = warp_base + i * 32 + lane;
            peers = __ballot_sync(0xffffffffu, idx < n);
        }
        if (MATCH) {
            // one match instruction in place of eight ballots; a lane past the
            // end matches only itself
            const u32 idx = warp_base + i * 32 + lane;
            peers &= __match_any_sync(0xffffffffu, (FULL || idx < n) ? d : RADIX + lane);
        } else {
#pragma unroll
            for (int j = 0; j < 8; j++) {
                const u32 bj = __ballot_sync(0xffffffffu, (d >> j) & 1);
                peers &= ((d >> j) & 1) ? bj : ~bj;
            }
        }
        const u32 base = S.warp_hist[warp][d];   // every peer reads the same word
        __syncwarp();
        const bool leader = (peers & lt) == 0;
        if (FULL) {
            if (leader) S.warp_hist[warp][d] = base + __popc(peers);
        } else {
            const u32 idx = warp_base + i * 32 + lane;
            if (idx < n && leader) S.warp_hist[warp][d] = base + __popc(peers);
        }
        __syncwarp();
        const u32 r = base + __popc(peers & lt);
        if (i & 1) rank2[i >> 1] |= r << 16;
        else rank2[i >> 1] = r;
    }
    __syncthreads();
    const u32 d = threadIdx.x;  // threads below RADIX own one bin each
    u32 cnt = 0;
    if (d < RADIX) {
#pragma unroll
        for (int w = 0; w < THREADS / 32; w++) {
            const u32 c = S.warp_hist[w][d];
            S.warp_hist[w][d] = cnt;
            cnt += c;
        }
        if (tile != 0 || !g_hold_first_tile)
            st_relaxed(lookback + (u64)tile * RADIX + d, (tile == 0 ? LB_PRE : LB_AGG) | cnt);
    }
    u32 total;
    const u32 lstart = block_exclusive_scan<u32>(cnt, S.scan, &total);
    if (d < RADIX) S.bin_local[d] = lstart;
    __syncthreads();
#pragma unroll
    for (int i = 0; i < BAL_KPT; i++) {
        const u32 idx = warp_base + i * 32 + lane;
        if (FULL || idx < n) {
            const u64 key = src[idx];
            const u32 dd = __byte_perm(dg[i / 4], 0, 0x4440u | (u32)(i % 4));
            const u32 r = (rank2[i >> 1] >> ((i & 1) * 16)) & 0xFFFF;
            S.keys[S.bin_local[dd] + S.warp_hist[warp][dd] + r] = key;
        }
    }
    u32 excl = 0;
    if (d < RADIX && tile != 0) {
        excl = lookback_sum(lookback + d, RADIX, (int)tile - 1, err);
        st_relaxed(lookback + (u64)tile * RADIX + d, LB_PRE | (excl + cnt));
    }
    // bin_base: the digit's exclusive prefix over all keys, scanned once per pass
    if (d < RADIX) S.bin_delta[d] = bin_base[d] + excl - lstart;
    __syncthreads();
    const bool hiw = shift >= 32;
    const u32 tile_n = FULL ? TILE : min(TILE, n - tile_base);
#pragma unroll 4
    for (u32 j = threadIdx.x; j < tile_n; j += THREADS) {
        const u64 key = S.keys[j];
        const u32 dd = __byte_perm(hiw ? (u32)(key >> 32) : (u32)key, 0, sel);
        const u32 g = S.bin_delta[dd] + j;
        if (g < n) dst[g] = key;
        else atomicOr(err, ERR_CAPACITY);
    }
}

template <int THREADS, bool MATCH = false>
__global__ void __launch_bounds__(THREADS, THREADS == 256 ? 5 : 2)
    onesweep_byte_kernel(const u64 *__restrict__ src, u64 *__restrict__ dst, u32 n, int shift,
                         const u32 *__restrict__ bin_base, u32 *lookback, u32 *tile_counter, u32 *err)
{
    extern __shared__ __align__(16) unsigned char byte_smem[];
    BytePassSmem<THREADS> &S = *reinterpret_cast<BytePassSmem<THREADS> *>(byte_smem);
    if (threadIdx.x == 0) S.tile = atomicAdd(tile_counter, 1u);
    for (int i = threadIdx.x; i < (THREADS / 32) * RADIX; i += THREADS) (&S.warp_hist[0][0])[i] = 0;
    __syncthreads();
    const u32 tile = S.tile;
    if ((u64)(tile + 1) * BytePassSmem<THREADS>::TILE <= n)
        byte_pass_tile<THREADS, true, MATCH>(src, dst, n, shift, bin_base, lookback, tile, err, S);
    else
        byte_pass_tile<THREADS, false, MATCH>(src, dst, n, shift, bin_base, lookback, tile, err, S);
}

// ---------------------------------------------------------------------------
// Persistent, software-pipelined digit pass.  Each CTA loops over tiles taken
// in order from the tile counter; while it ranks and scatters tile t, the
// bulk-copy engine already loads tile t+1 into the CTA's second shared
// buffer, so the load latency leaves the critical path.  The keys of the
// current tile sit in registers during ranking, which frees their shared
// buffer for the tile's local (digit-sorted) scatter.  The grid never exceeds
// the resident CTA count, so every tile taken is processed and the look-back
// always progresses.  Measured on B200 (88M LL-like keys, 8-bit digit): 0.74 ms
// per pass against 0.61 ms for the ballot kernel -- three resident CTAs per SM
// (shared memory) hide less of the integer-ALU-bound ranking, and CTAs that
// advance in step walk longer look-back chains -- so it is an option, not the
// default.
constexpr int PIPE_KPT = 16;
constexpr int PIPE_TILE = SORT_THREADS * PIPE_KPT;  // 4096 keys, 32 KiB
constexpr int PIPE_MINB = 3;

struct PipeSmem {
    u64 buf[2][PIPE_TILE];
    uint64_t bar[2];
    unsigned short warp_hist[SORT_THREADS / 32][RADIX];  // per-warp bin counts, then offsets (< 4096)
    u32 bin_local[RADIX];
    u32 bin_global[RADIX];
    u32 scan[33];
    u32 tile_next;
};

__global__ void __launch_bounds__(SORT_THREADS, PIPE_MINB)
    onesweep_pipe_kernel(const u64 *__restrict__ src, u64 *__restrict__ dst, u32 n, int shift,
                         const u32 *__restrict__ digit_hist, u32 *lookback, u32 *tile_counter, u32 *err)
{
    extern __shared__ __align__(128) unsigned char pipe_smem_raw[];
    PipeSmem &S = *reinterpret_cast<PipeSmem *>(pipe_smem_raw);
    const u32 ntiles = (n + PIPE_TILE - 1) / PIPE_TILE;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const u32 d = threadIdx.x;  // SORT_THREADS == RADIX: thread d owns bin d
    u32 total;
    const u32 gexcl = block_exclusive_scan<u32>(digit_hist[d], S.scan, &total);  // once per CTA
    if (threadIdx.x == 0) {
        mbar_init(&S.bar[0], 1);
        mbar_init(&S.bar[1], 1);
        fence_mbar_init();
        S.tile_next = atomicAdd(tile_counter, 1u);
    }
    __syncthreads();
    u32 tile = S.tile_next;
    // tile t holds keys [t*TILE, t*TILE + tile_n); the even-length prefix is
    // bulk-copied (16-byte granules), an odd last key is read directly
    auto dma_len = [&](u32 t) -> u32 { return min((u32)PIPE_TILE, n - t * PIPE_TILE) & ~1u; };
    if (threadIdx.x == 0 && tile < ntiles && dma_len(tile)) {
        fence_proxy_async_smem();
        mbar_expect_tx(&S.bar[0], dma_len(tile) * 8);
        bulk_load(S.buf[0], src + (u64)tile * PIPE_TILE, dma_len(tile) * 8, &S.bar[0]);
    }
    u32 parity[2] = {0, 0};
    int cur = 0;
    const u32 lt = lanemask_lt();
    while (tile < ntiles) {
        // (A) the previous tile is fully scattered: its buffer may be refilled
        __syncthreads();
        if (threadIdx.x == 0) {
            const u32 nt = atomicAdd(tile_counter, 1u);
            S.tile_next = nt;
            if (nt < ntiles && dma_len(nt)) {
                fence_proxy_async_smem();
                mbar_expect_tx(&S.bar[cur ^ 1], dma_len(nt) * 8);
                bulk_load(S.buf[cur ^ 1], src + (u64)nt * PIPE_TILE, dma_len(nt) * 8, &S.bar[cur ^ 1]);
            }
        }
        const u32 tile_base = tile * PIPE_TILE;
        const u32 tile_n = min((u32)PIPE_TILE, n - tile_base);
        const u32 n_dma = tile_n & ~1u;
        // each warp clears its own count row (all reads of it ended before (A))
        for (int b = lane; b < RADIX; b += 32) S.warp_hist[warp][b] = 0;
        if (n_dma) {
            mbar_wait(&S.bar[cur], parity[cur], err);
            parity[cur] ^= 1;
        }
        __syncwarp();
        const u32 wbase = warp * (PIPE_KPT * 32);
        // an odd last key is not part of the bulk copy: put it in place
        if (n_dma < tile_n && wbase <= n_dma && n_dma < wbase + PIPE_KPT * 32 && lane == 0)
            S.buf[cur][n_dma] = src[tile_base + n_dma];
        __syncwarp();
        u32 rank2[PIPE_KPT / 2];
#pragma unroll
        for (int i = 0; i < PIPE_KPT; i++) {
            const u32 j = wbase + i * 32 + lane;
            const u32 valid = __ballot_sync(0xffffffffu, j < tile_n);
            const u32 dg = j < tile_n ? (u32)(S.buf[cur][j] >> shift) & 0xFF : 0;
            u32 peers = valid;
#pragma unroll
            for (int b = 0; b < 8; b++) {
                const u32 bb = __ballot_sync(0xffffffffu, (dg >> b) & 1);
                peers &= ((dg >> b) & 1) ? bb : ~bb;
            }
            const u32 base = S.warp_hist[warp][dg];
            __syncwarp();
            if (j < tile_n && (peers & lt) == 0) S.warp_hist[warp][dg] = (unsigned short)(base + __popc(peers));
            __syncwarp();
            const u32 r = base + __popc(peers & lt);
            if (i & 1) rank2[i >> 1] |= r << 16;
            else rank2[i >> 1] = r;
        }
        // (B) counts complete
        __syncthreads();
        u32 cnt = 0;
#pragma unroll
        for (int w = 0; w < SORT_THREADS / 32; w++) {
            const u32 c = S.warp_hist[w][d];
            S.warp_hist[w][d] = (unsigned short)cnt;
            cnt += c;
        }
        u32 *lb = lookback + (u64)tile * RADIX + d;
        if (tile != 0 || !g_hold_first_tile) st_relaxed(lb, (tile == 0 ? LB_PRE : LB_AGG) | cnt);
        const u32 lstart = block_exclusive_scan<u32>(cnt, S.scan, &total);  // (C) inside
        S.bin_local[d] = lstart;
        // keys to registers, then (E) the local scatter may overwrite buf[cur]
        u64 k[PIPE_KPT];
#pragma unroll
        for (int i = 0; i < PIPE_KPT; i++) k[i] = S.buf[cur][wbase + i * 32 + lane];
        __syncthreads();
#pragma unroll
        for (int i = 0; i < PIPE_KPT; i++) {
            const u32 j = wbase + i * 32 + lane;
            if (j < tile_n) {
                const u32 dg = (u32)(k[i] >> shift) & 0xFF;
                const u32 r = (rank2[i >> 1] >> ((i & 1) * 16)) & 0xFFFF;
                S.buf[cur][S.bin_local[dg] + S.warp_hist[warp][dg] + r] = k[i];
            }
        }
        u32 excl = 0;
        if (tile != 0) {
            excl = lookback_sum(lookback + d, RADIX, (int)tile - 1, err);
            st_relaxed(lb, LB_PRE | (excl + cnt));
        }
        S.bin_global[d] = gexcl + excl - lstart;
        // (D) sorted tile and bin offsets visible
        __syncthreads();
        for (u32 j = threadIdx.x; j < tile_n; j += SORT_THREADS) {
            const u64 key = S.buf[cur][j];
            const u32 g = S.bin_global[(u32)(key >> shift) & 0xFF] + j;
            if (g < n) dst[g] = key;
            else atomicOr(err, ERR_CAPACITY);
        }
        tile = S.tile_next;
        cur ^= 1;
    }
}

constexpr size_t PIPE_SMEM = sizeof(PipeSmem);

// resident CTAs of the pipelined pass (0 until first use)
static int pipe_grid(int device)
{
    static int dev = -1, grid = 0;
    if (dev != device) {
        cudaFuncSetAttribute(onesweep_pipe_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)PIPE_SMEM);
        int per_sm = 0, sms = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, onesweep_pipe_kernel, SORT_THREADS, PIPE_SMEM);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
        grid = per_sm * sms;
        dev = device;
    }
    return grid;
}

// 0: match ranking, 1: ballot ranking, 2: pipelined persistent, 3: byte-digit ballot
// (4096-key tiles), 4: byte-digit ballot with 8192-key tiles (the default: measured
// 9 % faster than 3 on the LL sweep), 5: 4 with match ranking
int g_sort_variant = 4;

// the 8192-key byte pass needs more than the default 48 KiB of shared memory
static bool byte512_attr()
{
    static bool done = false;
    if (!done) {
        if (!CGB_CUDA(cudaFuncSetAttribute(onesweep_byte_kernel<512, false>,
                                           cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(BytePassSmem<512>))) ||
            !CGB_CUDA(cudaFuncSetAttribute(onesweep_byte_kernel<512, true>,
                                           cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(BytePassSmem<512>))))
            return false;
        done = true;
    }
    return true;
}

// test switches of the look-back waits (see g_spin_limit); 0 restores the default limit
bool set_lookback_test(u32 spin_limit, int hold_first_tile)
{
    const u32 lim = spin_limit ? spin_limit : SPIN_LIMIT;
    const u32 hold = hold_first_tile ? 1u : 0u;
    return CGB_CUDA(cudaMemcpyToSymbol(g_spin_limit, &lim, sizeof lim)) &&
           CGB_CUDA(cudaMemcpyToSymbol(g_hold_first_tile, &hold, sizeof hold));
}

// ---------------------------------------------------------------------------
// 8-byte global -> shared copies that hold no registers while in flight
__device__ __forceinline__ void cp_async8(void *dst_smem, const void *src_gmem)
{
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(smem_addr(dst_smem)), "l"(src_gmem) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

// unique: in (sorted) -> out, dropping repeats; *out_count = number kept.
// The tile (and the key before it) is staged in shared memory by async
// copies, all of a thread's in flight at once and no registers held.  Warp w
// then owns keys [512w, 512w + 512) as 16 rows of 32: a key's predecessor is
// the shared word before it, the kept keys of a row are ranked with one
// ballot, and each row's kept keys go out as one coalesced store.  Warp 0
// scans the eight warp totals and runs the tile's look-back.
struct UniqueSmem {
    u64 keys[UNQ_TILE + 1];  // keys[0]: the key before the tile
    u32 warp_base[UNQ_THREADS / 32];
    u32 tile;
};

// empty cells (0 nibbles) of a board
__device__ __forceinline__ u32 zero_nibbles(u64 k)
{
    const u64 x = k | (k >> 1) | (k >> 2) | (k >> 3);
    return (u32)__popcll(~x & 0x1111111111111111ull);
}

template <bool FULL>
__device__ __forceinline__ void unique_tile(const u64 *__restrict__ in, u32 n, u64 *__restrict__ out, u32 *lookback,
                                            u32 tile, u32 *out_count, u32 *err, UniqueSmem &S,
                                            unsigned long long *empties)
{
    constexpr u32 ALL = 0xffffffffu;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const u32 tile_base = tile * UNQ_TILE;
    const u32 tile_n = FULL ? (u32)UNQ_TILE : n - tile_base;
#pragma unroll
    for (int q = 0; q < UNQ_KPT; q++) {
        const u32 j = q * UNQ_THREADS + threadIdx.x;
        if (FULL || j < tile_n) cp_async8(&S.keys[1 + j], in + tile_base + j);
    }
    if (threadIdx.x == 0 && tile_base > 0) cp_async8(&S.keys[0], in + tile_base - 1);
    cp_async_wait_all();
    __syncthreads();
    const u32 wfirst = warp * (UNQ_KPT * 32);
    u32 mask[UNQ_KPT];
    u32 total = 0;
    bool descent = false;
#pragma unroll
    for (int q = 0; q < UNQ_KPT; q++) {
        const u32 j = wfirst + q * 32 + lane;
        const bool valid = FULL || j < tile_n;
        const bool has_prev = tile_base + j > 0;
        const u64 v = valid ? S.keys[1 + j] : 0ull;
        const u64 prev = (valid && has_prev) ? S.keys[j] : 0ull;
        descent |= valid && has_prev && v < prev;
        mask[q] = __ballot_sync(ALL, valid && (!has_prev || v != prev));
        total += __popc(mask[q]);
    }
    if (descent) atomicOr(err, ERR_UNSORTED);
    if (lane == 0) S.warp_base[warp] = total;
    __syncthreads();
    if (warp == 0) {
        const u32 c = lane < UNQ_THREADS / 32 ? S.warp_base[lane] : 0u;
        const u32 incl = warp_inclusive_scan(c);
        const u32 tile_total = __shfl_sync(ALL, incl, 31);
        u32 prefix = 0;
        if (tile == 0) {
            if (lane == 0) st_relaxed(lookback, LB_PRE | tile_total);
        } else {
            if (lane == 0) st_relaxed(lookback + tile, LB_AGG | tile_total);
            prefix = warp_lookback_sum<u32>(lookback, (int)tile - 1, err);
            if (lane == 0) st_relaxed(lookback + tile, LB_PRE | (prefix + tile_total));
        }
        if (lane < UNQ_THREADS / 32) S.warp_base[lane] = prefix + incl - c;
        if (lane == 0 && tile_base + UNQ_TILE >= n) *out_count = prefix + tile_total;
    }
    __syncthreads();
    u32 pos = S.warp_base[warp];
    const u32 lt = lanemask_lt();
    u32 ecount = 0;  // empty cells of this thread's kept keys (when asked for)
#pragma unroll
    for (int q = 0; q < UNQ_KPT; q++) {
        if ((mask[q] >> lane) & 1) {
            const u32 g = pos + __popc(mask[q] & lt);
            const u64 v = S.keys[1 + wfirst + q * 32 + lane];
            if (empties) ecount += zero_nibbles(v);
            if (g < n) out[g] = v;
            else atomicOr(err, ERR_CAPACITY);
        }
        pos += __popc(mask[q]);
    }
    if (empties) {
        const u32 w = __reduce_add_sync(0xffffffffu, ecount);
        if (lane == 0 && w) atomicAdd(empties, (unsigned long long)w);
    }
}

// empties: null, or a word that receives the number of empty cells over the
// kept keys (boards) -- the size of their spawn streams
__global__ void __launch_bounds__(UNQ_THREADS, 5) unique_kernel(const u64 *__restrict__ in, u32 n, u64 *__restrict__ out,
                                                                u32 *lookback, u32 *tile_counter, u32 *out_count,
                                                                u32 *err, unsigned long long *empties)
{
    __shared__ UniqueSmem S;
    if (threadIdx.x == 0) S.tile = atomicAdd(tile_counter, 1u);
    __syncthreads();
    const u32 tile = S.tile;
    if ((u64)(tile + 1) * UNQ_TILE <= n) unique_tile<true>(in, n, out, lookback, tile, out_count, err, S, empties);
    else unique_tile<false>(in, n, out, lookback, tile, out_count, err, S, empties);
}

// ---------------------------------------------------------------------------
// merge path over the merge tile's padded shared layout (a[i] at
// buf[pad8(i)], b[i] at buf[pad8(la + i)]): for output diagonal `diag`, the
// number of elements taken from a (ties go to a first)
__device__ __forceinline__ u32 pad8(u32 j) { return j + (j >> 3); }
__device__ __forceinline__ u32 merge_path_padded(const u64 *buf, u32 la, u32 lb, u32 diag)
{
    u32 lo = diag > lb ? diag - lb : 0;
    u32 hi = diag < la ? diag : la;
    while (lo < hi) {
        const u32 mid = (lo + hi) >> 1;
        if (buf[pad8(mid)] <= buf[pad8(la + diag - 1 - mid)]) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}

// merge runs may exceed 2^30 keys (a layer of a large workload): 64-bit
// positions and a 64-bit look-back word (2 flag bits, 62-bit count)
constexpr u64 LB64_AGG = 1ull << 62, LB64_PRE = 2ull << 62, LB64_MASK = (1ull << 62) - 1;



__device__ __forceinline__ u64 merge_path64(const u64 *a, u64 na, const u64 *b, u64 nb, u64 diag)
{
    u64 lo = diag > nb ? diag - nb : 0;
    u64 hi = diag < na ? diag : na;
    while (lo < hi) {
        const u64 mid = (lo + hi) >> 1;
        if (a[mid] <= b[diag - 1 - mid]) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}

__global__ void merge_partition_kernel(const u64 *__restrict__ a, u64 na, const u64 *__restrict__ b, u64 nb,
                                       u64 *splits, u32 ntiles)
{
    const u32 t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t > ntiles) return;
    const u64 diag = min((u64)t * MRG_TILE, na + nb);
    splits[t] = merge_path64(a, na, b, nb, diag);
}

// One tile of MRG_TILE merged positions: the tile's runs of a and b are loaded
// with all of a thread's loads in flight, each thread merges MRG_KPT positions
// from its merge-path split (the heads of both runs held in registers), marks
// the first of each run of equal keys, and the kept keys are staged in the
// same shared buffer (the runs are no longer read by then) for one coalesced
// write.  Warp 0 scans the warp totals and runs the 64-bit look-back.
__global__ void __launch_bounds__(MRG_THREADS) merge_unique_kernel(const u64 *__restrict__ a, u64 na,
                                                                   const u64 *__restrict__ b, u64 nb,
                                                                   const u64 *__restrict__ splits,
                                                                   u64 *__restrict__ out, u64 *lookback,
                                                                   u32 *tile_counter, u64 *out_count, u32 *err)
{
    constexpr u32 ALL = 0xffffffffu;
    __shared__ u64 buf[MRG_TILE + MRG_TILE / 8];
    __shared__ u64 last_sh[MRG_THREADS];
    __shared__ u32 warp_sh[MRG_THREADS / 32];
    __shared__ u32 tile_sh, kept_sh;
    __shared__ u64 prefix_sh;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (threadIdx.x == 0) tile_sh = atomicAdd(tile_counter, 1u);
    __syncthreads();
    const u32 tile = tile_sh;
    const u64 total = na + nb;
    const u64 d0 = min((u64)tile * MRG_TILE, total);
    const u64 d1 = min((u64)(tile + 1) * MRG_TILE, total);
    const u64 a0 = splits[tile], a1 = splits[tile + 1];
    const u64 b0 = d0 - a0, b1 = d1 - a1;
    const u32 la = (u32)(a1 - a0), lb = (u32)(b1 - b0);
    {
        u64 r[MRG_KPT];
#pragma unroll
        for (int i = 0; i < MRG_KPT; i++) {
            const u32 j = i * MRG_THREADS + threadIdx.x;
            r[i] = j < la ? a[a0 + j] : (j < la + lb ? b[b0 + (j - la)] : 0ull);
        }
#pragma unroll
        for (int i = 0; i < MRG_KPT; i++) {
            const u32 j = i * MRG_THREADS + threadIdx.x;
            if (j < la + lb) buf[pad8(j)] = r[i];
        }
    }
    // the merged element just before this tile
    const bool have_before = d0 > 0;
    u64 before = 0;
    if (have_before && threadIdx.x == 0) {
        if (a0 == 0) before = b[b0 - 1];
        else if (b0 == 0) before = a[a0 - 1];
        else before = max(a[a0 - 1], b[b0 - 1]);
    }
    __syncthreads();
    // a thread's runs start about MRG_KPT / 2 keys apart in each input: the
    // padded layout spreads their reads over the banks
    const u32 len = (u32)(d1 - d0);
    const u32 t0 = min((u32)(threadIdx.x * MRG_KPT), len);
    const u32 t1 = min(t0 + MRG_KPT, len);
    u32 ia = merge_path_padded(buf, la, lb, t0);
    u32 ib = t0 - ia;
    u64 xa = ia < la ? buf[pad8(ia)] : 0ull, xb = ib < lb ? buf[pad8(la + ib)] : 0ull;
    u64 v[MRG_KPT];
#pragma unroll
    for (int i = 0; i < MRG_KPT; i++) {
        if (t0 + i < t1) {
            const bool take_a = ib >= lb || (ia < la && xa <= xb);
            if (take_a) {
                v[i] = xa;
                ++ia;
                xa = ia < la ? buf[pad8(ia)] : 0ull;
            } else {
                v[i] = xb;
                ++ib;
                xb = ib < lb ? buf[pad8(la + ib)] : 0ull;
            }
        } else {
            v[i] = 0ull;
        }
    }
    u64 mylast = 0;
#pragma unroll
    for (int i = 0; i < MRG_KPT; i++)
        if (t0 + i < t1) mylast = v[i];
    last_sh[threadIdx.x] = mylast;
    __syncthreads();  // after this the runs in buf are no longer read
    u64 prev;
    bool have_prev;
    if (threadIdx.x == 0) {
        prev = before;
        have_prev = have_before;
    } else {
        // the previous thread always owns MRG_KPT elements when this one owns any
        prev = last_sh[threadIdx.x - 1];
        have_prev = true;
    }
    u32 flags = 0;
    bool descent = false;  // sorted inputs merge into a non-decreasing sequence
#pragma unroll
    for (int i = 0; i < MRG_KPT; i++) {
        if (t0 + i < t1) {
            if (!have_prev || v[i] != prev) flags |= 1u << i;
            descent |= have_prev && v[i] < prev;
            prev = v[i];
            have_prev = true;
        }
    }
    if (descent) atomicOr(err, ERR_UNSORTED);
    const u32 cnt = __popc(flags);
    const u32 inc = warp_inclusive_scan(cnt);
    if (lane == 31) warp_sh[warp] = inc;
    __syncthreads();
    if (warp == 0) {
        const u32 c = lane < MRG_THREADS / 32 ? warp_sh[lane] : 0u;
        const u32 wi = warp_inclusive_scan(c);
        const u32 tile_total = __shfl_sync(ALL, wi, 31);
        u64 prefix = 0;
        if (tile == 0) {
            if (lane == 0) st_relaxed64(lookback, LB64_PRE | tile_total);
        } else {
            if (lane == 0) st_relaxed64(lookback + tile, LB64_AGG | tile_total);
            prefix = warp_lookback_sum<u64>(lookback, (int)tile - 1, err);
            if (lane == 0) st_relaxed64(lookback + tile, LB64_PRE | (prefix + tile_total));
        }
        if (lane < MRG_THREADS / 32) warp_sh[lane] = wi - c;
        if (lane == 0) {
            prefix_sh = prefix;
            kept_sh = tile_total;
            if ((u64)(tile + 1) * MRG_TILE >= total) *out_count = prefix + tile_total;
        }
    }
    __syncthreads();
    u32 w = warp_sh[warp] + inc - cnt;
#pragma unroll
    for (int i = 0; i < MRG_KPT; i++)
        if (flags & (1u << i)) {
            buf[pad8(w)] = v[i];
            w++;
        }
    __syncthreads();
    const u64 prefix = prefix_sh;
    const u32 kept = kept_sh;
    for (u32 j = threadIdx.x; j < kept; j += MRG_THREADS) {
        if (prefix + j < total) out[prefix + j] = buf[pad8(j)];
        else atomicOr(err, ERR_CAPACITY);
    }
}

// ---------------------------------------------------------------------------
// host side

static inline u32 ceil_div(u64 a, u64 b) { return (u32)((a + b - 1) / b); }

// look-back words needed: one per bin per tile for a digit pass (the largest
// user), one per tile for unique, four per tile for a merge
bool SortWorkspace::reserve(u64 words, cudaStream_t s)
{
    const u64 need = (words + 64) * sizeof(u32);
    if (need <= lookback_bytes && small) return true;
    if (lookback) cudaFreeAsync(lookback, s);
    lookback = nullptr;
    if (!small) {
        if (!CGB_CUDA(cudaMallocAsync((void **)&small, SMALL_WORDS * sizeof(u32), s))) return false;
    }
    if (!CGB_CUDA(cudaMallocAsync((void **)&lookback, need, s))) return false;
    lookback_bytes = need;
    return true;
}

void SortWorkspace::release(cudaStream_t s)
{
    if (lookback) cudaFreeAsync(lookback, s);
    if (small) cudaFreeAsync(small, s);
    lookback = nullptr;
    small = nullptr;
    lookback_bytes = 0;
}

// small words: [0,2048) histograms, [2048,2064) tile counters, 2064 err, 2065 count,
// 2066-2067 a 64-bit count (8-byte aligned)
static constexpr int W_HIST = 0, W_CTR = 2048, W_ERR = 2064, W_COUNT = 2065, W_COUNT64 = 2066, W_EMPTIES = 2068,
                     W_OFFS = 4096;

static bool check_err(SortWorkspace &ws, cudaStream_t s, const char *what)
{
    u32 e = 0;
    if (!CGB_CUDA(cudaMemcpyAsync(&e, ws.small + W_ERR, sizeof(u32), cudaMemcpyDeviceToHost, s))) return false;
    if (!CGB_CUDA(cudaStreamSynchronize(s))) return false;
    if (e) {
        set_error(std::string(what) + ": device error " + err_string(e));
        return false;
    }
    return true;
}

bool sort_check(SortWorkspace &ws, cudaStream_t s)
{
    if (!ws.err_dirty) return true;
    ws.err_dirty = false;
    if (!check_err(ws, s, "sort_keys")) return false;
    kclock().flush();
    return true;
}

int sort_plan(const u32 *hist_host, u64 n, int *digits)
{
    int np = 0;
    for (int d = 0; d < 8; d++) {
        bool constant = false;
        for (int b = 0; b < RADIX; b++)
            if (hist_host[d * RADIX + b] == n) constant = true;
        if (!constant) digits[np++] = d;
    }
    return np;
}

bool sort_keys(u64 *keys, u64 *tmp, u64 n, u64 **sorted, SortWorkspace &ws, cudaStream_t s, SortStats *stats)
{
    *sorted = keys;
    if (stats) *stats = SortStats{};
    if (n <= 1) return true;
    if (n > (u64)LB_MASK) {
        set_error("sort_keys: more than 2^30 keys in one call");
        return false;
    }
    if (!ws.reserve(((n + SORT_TILE - 1) / SORT_TILE + 1) * RADIX, s)) return false;
    // histograms and tile counters start at zero; the error word keeps what an
    // earlier sort left for the next unique or merge to report
    if (!CGB_CUDA(cudaMemsetAsync(ws.small, 0, (ws.err_dirty ? W_ERR : W_COUNT + 1) * sizeof(u32), s))) return false;
    const int hist_blocks = (int)std::min<u64>((n + 255) / 256, (u64)NUM_SMS_B200 * 8);
    kclock().begin(s, &kstats().hist_ms);
    digit_histogram_kernel<<<hist_blocks, 256, 0, s>>>(keys, n, ws.small + W_HIST);
    kclock().end(s);
    kstats().hist_bytes += 8 * n;
    if (!CGB_CUDA(cudaGetLastError())) return false;
    u32 hist[8 * RADIX];
    if (g_sort_variant >= 3) {
        digit_offsets_kernel<<<8, RADIX, 0, s>>>(ws.small + W_HIST, ws.small + W_OFFS);
        kstats().launches++;
        if (!CGB_CUDA(cudaGetLastError())) return false;
    }
    if (!CGB_CUDA(cudaMemcpyAsync(hist, ws.small + W_HIST, sizeof(hist), cudaMemcpyDeviceToHost, s))) return false;
    if (!CGB_CUDA(cudaStreamSynchronize(s))) return false;
    int digits[8];
    const int np = sort_plan(hist, n, digits);
    const u32 tiles = ceil_div(n, SORT_TILE);
    // the pipelined pass needs 16-byte aligned buffers for its bulk copies
    int variant = g_sort_variant;
    int pgrid = 0;
    if (variant == 2) {
        int dev = 0;
        cudaGetDevice(&dev);
        pgrid = pipe_grid(dev);
        if (pgrid <= 0 || (((uintptr_t)keys | (uintptr_t)tmp) & 15)) variant = 1;
    }
    const u32 pass_tiles = variant == 2   ? ceil_div(n, PIPE_TILE)
                           : variant >= 4 ? ceil_div(n, 512 * BAL_KPT)
                           : (variant == 1 || variant == 3) ? ceil_div(n, BAL_TILE)
                                                            : tiles;
    if (variant >= 4 && !byte512_attr()) return false;
    u64 *src = keys, *dst = tmp;
    for (int p = 0; p < np; p++) {
        const int d = digits[p];
        if (!CGB_CUDA(cudaMemsetAsync(ws.lookback, 0, (u64)pass_tiles * RADIX * sizeof(u32), s))) return false;
        kclock().begin(s, &kstats().onesweep_ms);
        if (variant == 2)
            onesweep_pipe_kernel<<<std::min<u32>(pass_tiles, (u32)pgrid), SORT_THREADS, PIPE_SMEM, s>>>(
                src, dst, (u32)n, 8 * d, ws.small + W_HIST + d * RADIX, ws.lookback, ws.small + W_CTR + p,
                ws.small + W_ERR);
        else if (variant == 1)
            onesweep_ballot_kernel<<<ceil_div(n, BAL_TILE), SORT_THREADS, 0, s>>>(src, dst, (u32)n, ShiftDigit{8 * d},
                                                                  ws.small + W_HIST + d * RADIX, ws.lookback,
                                                                  ws.small + W_CTR + p, ws.small + W_ERR);
        else if (variant == 3)
            onesweep_byte_kernel<256><<<ceil_div(n, 256 * BAL_KPT), 256, sizeof(BytePassSmem<256>), s>>>(
                src, dst, (u32)n, 8 * d, ws.small + W_OFFS + d * RADIX, ws.lookback, ws.small + W_CTR + p,
                ws.small + W_ERR);
        else if (variant == 4)
            onesweep_byte_kernel<512><<<ceil_div(n, 512 * BAL_KPT), 512, sizeof(BytePassSmem<512>), s>>>(
                src, dst, (u32)n, 8 * d, ws.small + W_OFFS + d * RADIX, ws.lookback, ws.small + W_CTR + p,
                ws.small + W_ERR);
        else if (variant == 5)
            onesweep_byte_kernel<512, true><<<ceil_div(n, 512 * BAL_KPT), 512, sizeof(BytePassSmem<512>), s>>>(
                src, dst, (u32)n, 8 * d, ws.small + W_OFFS + d * RADIX, ws.lookback, ws.small + W_CTR + p,
                ws.small + W_ERR);
        else
            onesweep_kernel<<<tiles, SORT_THREADS, 0, s>>>(src, dst, (u32)n, 8 * d, ws.small + W_HIST + d * RADIX,
                                                           ws.lookback, ws.small + W_CTR + p, ws.small + W_ERR);
        kclock().end(s);
        kstats().onesweep_bytes += 16 * n;
        kstats().onesweep_launches++;
        if (!CGB_CUDA(cudaGetLastError())) return false;
        std::swap(src, dst);
    }
    *sorted = src;
    if (stats) {
        stats->passes = np;
        stats->n = n;
    }
    // errors of the passes stay in the error word; unique_keys reports them
    ws.err_dirty = true;
    return true;
}

bool unique_keys(const u64 *in, u64 n, u64 *out, u64 *n_out, SortWorkspace &ws, cudaStream_t s, u64 *empties)
{
    *n_out = 0;
    if (empties) *empties = 0;
    if (n == 0) return true;
    if (n > (u64)LB_MASK) {
        set_error("unique_keys: more than 2^30 keys in one call");
        return false;
    }
    if (!ws.reserve((n + UNQ_TILE - 1) / UNQ_TILE + 1, s)) return false;
    const u32 tiles = ceil_div(n, UNQ_TILE);
    if (!CGB_CUDA(cudaMemsetAsync(ws.small + W_CTR, 0, (W_ERR - W_CTR) * sizeof(u32), s))) return false;
    // the count, the 64-bit count slot and the empty-cell sum start at zero
    if (!CGB_CUDA(cudaMemsetAsync(ws.small + W_COUNT, 0, (W_EMPTIES + 2 - W_COUNT) * sizeof(u32), s))) return false;
    if (!ws.err_dirty && !CGB_CUDA(cudaMemsetAsync(ws.small + W_ERR, 0, sizeof(u32), s))) return false;
    ws.err_dirty = false;
    if (!CGB_CUDA(cudaMemsetAsync(ws.lookback, 0, (u64)tiles * sizeof(u32), s))) return false;
    kclock().begin(s, &kstats().unique_ms);
    unique_kernel<<<tiles, UNQ_THREADS, 0, s>>>(in, (u32)n, out, ws.lookback, ws.small + W_CTR,
                                                ws.small + W_COUNT, ws.small + W_ERR,
                                                empties ? (unsigned long long *)(ws.small + W_EMPTIES) : nullptr);
    kclock().end(s);
    if (!CGB_CUDA(cudaGetLastError())) return false;
    u32 ec[W_EMPTIES + 2 - W_ERR];  // error word, count, (64-bit count), empty-cell sum
    if (!CGB_CUDA(cudaMemcpyAsync(ec, ws.small + W_ERR, sizeof(ec), cudaMemcpyDeviceToHost, s))) return false;
    if (!CGB_CUDA(cudaStreamSynchronize(s))) return false;
    kclock().flush();
    if (ec[0]) {
        set_error(std::string("sort/unique: device error ") + err_string(ec[0]));
        return false;
    }
    const u32 cnt = ec[1];
    kstats().unique_bytes += 8 * (n + cnt);
    *n_out = cnt;
    if (empties) memcpy(empties, &ec[W_EMPTIES - W_ERR], sizeof(u64));
    return true;
}

bool merge_unique(const u64 *a, u64 na, const u64 *b, u64 nb, u64 *out, u64 *n_out, SortWorkspace &ws,
                  cudaStream_t s)
{
    *n_out = 0;
    const u64 total = na + nb;
    if (total == 0) return true;
    const u64 tiles64 = (total + MRG_TILE - 1) / MRG_TILE;
    if (tiles64 >= (1ull << 31)) {
        set_error("merge_unique: too many keys");
        return false;
    }
    const u32 tiles = (u32)tiles64;
    if (!ws.reserve(4 * ((u64)tiles + 1), s)) return false;
    // 64-bit look-back words, then the splits (both fit in the u32 look-back area)
    u64 *lb = (u64 *)ws.lookback;
    u64 *splits = lb + ((u64)tiles + 1);
    // tile counters and counts start at zero; the error word too, unless sorts
    // before this merge left errors in it (reported below with the merge's own)
    if (ws.err_dirty) {
        if (!CGB_CUDA(cudaMemsetAsync(ws.small + W_CTR, 0, (W_ERR - W_CTR) * sizeof(u32), s)) ||
            !CGB_CUDA(cudaMemsetAsync(ws.small + W_COUNT, 0, (W_COUNT64 + 2 - W_COUNT) * sizeof(u32), s)))
            return false;
    } else if (!CGB_CUDA(cudaMemsetAsync(ws.small + W_CTR, 0, (W_COUNT64 + 2 - W_CTR) * sizeof(u32), s))) {
        return false;
    }
    ws.err_dirty = false;
    if (!CGB_CUDA(cudaMemsetAsync(lb, 0, ((u64)tiles + 1) * sizeof(u64), s))) return false;
    kclock().begin(s, &kstats().merge_ms);
    merge_partition_kernel<<<ceil_div(tiles + 1, 256), 256, 0, s>>>(a, na, b, nb, splits, tiles);
    merge_unique_kernel<<<tiles, MRG_THREADS, 0, s>>>(a, na, b, nb, splits, out, lb, ws.small + W_CTR,
                                                      (u64 *)(ws.small + W_COUNT64), ws.small + W_ERR);
    kclock().end(s);
    kstats().launches++;
    if (!CGB_CUDA(cudaGetLastError())) return false;
    u32 ec[4];  // error word, (count u32 unused), 64-bit count
    if (!CGB_CUDA(cudaMemcpyAsync(ec, ws.small + W_ERR, 4 * sizeof(u32), cudaMemcpyDeviceToHost, s))) return false;
    if (!CGB_CUDA(cudaStreamSynchronize(s))) return false;
    kclock().flush();
    if (ec[0]) {
        set_error(std::string("merge_unique: device error ") + err_string(ec[0]));
        return false;
    }
    u64 cnt;
    memcpy(&cnt, &ec[2], 8);
    kstats().merge_bytes += 8 * (total + cnt);
    *n_out = cnt;
    return true;
}


// ---------------------------------------------------------------------------
// batched sweeps: stable partition of a layer by formation id
__global__ void __launch_bounds__(256) formation_histogram_kernel(const u64 *__restrict__ keys, u64 n,
                                                                  const unsigned char *__restrict__ fid,
                                                                  u32 *__restrict__ hist)
{
    __shared__ u32 sh[RADIX];
    sh[threadIdx.x] = 0;
    __syncthreads();
    for (u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (u64)gridDim.x * blockDim.x)
        atomicAdd(&sh[__ldg(fid + fixed_pattern(keys[i]))], 1u);
    __syncthreads();
    if (sh[threadIdx.x]) atomicAdd(&hist[threadIdx.x], sh[threadIdx.x]);
}

bool partition_by_formation(const u64 *in, u64 n, u64 *out, const unsigned char *fid, u32 counts[256],
                            SortWorkspace &ws, cudaStream_t s)
{
    memset(counts, 0, 256 * sizeof(u32));
    if (n == 0) return true;
    if (n > (u64)LB_MASK) {
        set_error("partition_by_formation: more than 2^30 keys in one call");
        return false;
    }
    const u32 tiles = ceil_div(n, BAL_TILE);
    if (!ws.reserve(((u64)tiles + 1) * RADIX, s)) return false;
    if (!CGB_CUDA(cudaMemsetAsync(ws.small, 0, (W_COUNT + 1) * sizeof(u32), s))) return false;
    if (!CGB_CUDA(cudaMemsetAsync(ws.lookback, 0, (u64)tiles * RADIX * sizeof(u32), s))) return false;
    const int hist_blocks = (int)std::min<u64>((n + 255) / 256, (u64)NUM_SMS_B200 * 4);
    formation_histogram_kernel<<<hist_blocks, 256, 0, s>>>(in, n, fid, ws.small + W_HIST);
    onesweep_ballot_kernel<<<tiles, SORT_THREADS, 0, s>>>(in, out, (u32)n, FormationDigit{fid}, ws.small + W_HIST,
                                                          ws.lookback, ws.small + W_CTR, ws.small + W_ERR);
    kstats().launches += 2;
    if (!CGB_CUDA(cudaGetLastError())) return false;
    u32 e = 0;
    if (!CGB_CUDA(cudaMemcpyAsync(counts, ws.small + W_HIST, 256 * sizeof(u32), cudaMemcpyDeviceToHost, s)) ||
        !CGB_CUDA(cudaMemcpyAsync(&e, ws.small + W_ERR, sizeof(u32), cudaMemcpyDeviceToHost, s)) ||
        !CGB_CUDA(cudaStreamSynchronize(s)))
        return false;
    ws.err_dirty = false;
    if (e) {
        set_error("partition_by_formation: device error " + err_string(e));
        return false;
    }
    return true;
}

}  // namespace cgb
