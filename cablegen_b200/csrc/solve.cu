// solve.cu -- backward expectimax over one layer (src/solve.c:226-302).
//
// One thread per board of layer s:
//   * satisfied (src/solve.c:233-244): with nox the board wins (1.0) when it
//     holds tile nox; otherwise when it matches any winstate image.
//   * otherwise expectimax (src/solve.c:257-281): for every empty cell in
//     cell order 0..15, a 2 (weight 0.9) and a 4 (weight 0.1) are placed; the
//     value of each spawn is the best of the four moves (src/solve.c:246-256),
//     each successor looked up, canonicalised, in the s+2 / s+4 table; a miss
//     is 0.0 (src/solve.c:108-164).  res = 0.9*S2/k + 0.1*S4/k.
//
// Two kernels: solve_items_kernel (the default) spreads the (board, empty
// cell) pairs of 32 boards over a warp's lanes; solve_direct_kernel runs one
// thread per board.  Canonical forms take the maximum over the images a
// CanonPlan allows for the board's 0xf mask (all eight without a plan).
//
// FP64 evaluates exactly the reference's operation sequence with
// round-to-nearest intrinsics (no FMA contraction): bit-identical values.
// FP32 keeps table values in FP32, accumulates the two spawn sums with Kahan
// compensation and forms the weighted mean in FP64 before rounding once (a
// 0.9f weight alone would bias every layer by 2.6e-8 relative).
//
// Lookup structures (all exact; a miss returns 0 like the reference):
//   INDEX_BISECT  branch-free bisection over the sorted layer
//   INDEX_BUCKET  top bits after the layer's common prefix select a bucket of
//                 the sorted layer, then bisection inside it
//   INDEX_HASH    open addressing with linear probing; a 16-byte slot holds
//                 the key and the value, so a hit costs one sector
#include "engine.h"
#include "hashidx.cuh"

namespace cgb {

constexpr int TABLE_BYTES_S = 65536 * 2;  // left-move rows, ROW_LOCKED for locked ones

// ---- lookup ---------------------------------------------------------------
template <typename V>
struct DevTable {
    int kind;
    const u64 *keys;
    const V *vals;
    u64 n;
    const u32 *bucket;
    int prefix, bits;
    u64 prefix_value;
    const ulonglong2 *slots;
    u64 cap;
    CompactHash ch;  // INDEX_HASH with 8-byte slots (ch.on)
};

template <typename V>
__device__ __forceinline__ V from_bits(u64 b);
template <>
__device__ __forceinline__ double from_bits<double>(u64 b) { return __longlong_as_double((long long)b); }
template <>
__device__ __forceinline__ float from_bits<float>(u64 b) { return __uint_as_float((u32)b); }

template <typename V>
__device__ __forceinline__ u64 to_bits(V v);
template <>
__device__ __forceinline__ u64 to_bits<double>(double v) { return (u64)__double_as_longlong(v); }
template <>
__device__ __forceinline__ u64 to_bits<float>(float v) { return (u64)__float_as_uint(v); }

template <typename V>
__device__ __forceinline__ V sorted_lookup(const DevTable<V> &t, u64 key)
{
    if (t.n == 0) return V(0);
    u64 lo = 0, len = t.n;
    if (t.kind == INDEX_BUCKET) {
        if (t.prefix > 0 && (key >> (64 - t.prefix)) != t.prefix_value) return V(0);
        const u32 bk = (u32)((key << t.prefix) >> (64 - t.bits));
        const u32 b0 = __ldg(t.bucket + bk), b1 = __ldg(t.bucket + bk + 1);
        lo = b0;
        len = b1 - b0;
        if (len == 0) return V(0);
    }
    while (len > 1) {
        const u64 half = len >> 1;
        lo = (__ldg(t.keys + lo + half) <= key) ? lo + half : lo;
        len -= half;
    }
    return __ldg(t.keys + lo) == key ? __ldg(t.vals + lo) : V(0);
}

// continue a linear probe after the first slot missed (plain arguments: a
// reference to the kernel's table would force a copy of it to local memory)
template <typename V>
__device__ __noinline__ V hash_probe_rest(const ulonglong2 *slots, u64 cap, u64 key, u64 s)
{
    for (u64 i = 1; i < cap; i++) {
        s = (s + 1 == cap) ? 0 : s + 1;
        const ulonglong2 e = __ldg(slots + s);
        if (e.x == key) return from_bits<V>(e.y);
        if (e.x == 0) return V(0);
    }
    return V(0);
}

// continue a compact probe after the home slot held another key
template <typename V>
__device__ __noinline__ V compact_probe_rest(const u64 *slots, u64 cap, int dbits, u64 home, u32 tag0)
{
    const u32 last = (1u << dbits) - 1u;  // probe distances stay below it (the build checks)
    for (u32 d = 1; d + 1 < last; d++) {
        const u64 e = __ldg(slots + ((home + d) & (cap - 1)));
        if ((u32)e == tag0 + d) return from_bits<V>(e >> 32);
        if ((u32)e == 0u) return V(0);
    }
    return V(0);
}

template <typename V>
__device__ __forceinline__ V vmax(V a, V b) { return a > b ? a : b; }

template <typename V>
__device__ __forceinline__ V table_value(const DevTable<V> &t, u64 key)
{
    if (t.kind == INDEX_HASH && t.ch.on) {
        if ((key & t.ch.cmask) != t.ch.cval) return V(0);
        u32 tag0;
        const u64 h = compact_home(t.ch, key, &tag0);
        const u64 e = __ldg((const u64 *)t.slots + h);
        if ((u32)e == tag0) return from_bits<V>(e >> 32);
        if ((u32)e == 0u) return V(0);
        return compact_probe_rest<V>((const u64 *)t.slots, t.cap, t.ch.dbits, h, tag0);
    }
    if (t.kind == INDEX_HASH) {
        if (t.cap == 0) return V(0);
        const u64 s = home_slot(key, t.cap);
        const ulonglong2 e = __ldg(t.slots + s);
        if (e.x == key) return from_bits<V>(e.y);
        if (e.x == 0) return V(0);
        return hash_probe_rest<V>(t.slots, t.cap, key, s);
    }
    return sorted_lookup(t, key);
}

__device__ __forceinline__ void add_probes(u32 probes, u64 *counter)
{
    const u32 w = __reduce_add_sync(0xffffffffu, probes);
    if ((threadIdx.x & 31) == 0 && w) atomicAdd((unsigned long long *)counter, (unsigned long long)w);
}

__device__ __forceinline__ bool satisfied(u64 b, const SolveRules &r)
{
    if (r.nox && !r.score) return has_tile(b, r.nox);
    if (r.score) return false;
    int lo = 0, hi = r.n_winstates;
    if (r.fid) {
        const u32 f = __ldg(r.fid + fixed_pattern(b));
        if (f == 0xFF) return false;
        lo = (int)__ldg(r.ws_begin + f);
        hi = (int)__ldg(r.ws_begin + f + 1);
    }
    for (int i = lo; i < hi; i++)
        if (matches(b, __ldg(r.winstates + i))) return true;
    return false;
}

__device__ __forceinline__ void stage_table_s(unsigned char *smem, const unsigned short *g_move)
{
    const uint4 *src = (const uint4 *)g_move;
    uint4 *dst = (uint4 *)smem;
    for (int i = threadIdx.x; i < TABLE_BYTES_S / 16; i += blockDim.x) dst[i] = __ldg(src + i);
    __syncthreads();
}

// Spawn-weighted mean of one board from its per-cell best values, in cell
// order (src/solve.c:257-281): FP64 adds in order, FP32 Kahan-compensated sums;
// the weighted mean is formed in FP64 and rounded once.
template <typename V>
struct SpawnSums {
    V s2 = 0, s4 = 0, c2 = 0, c4 = 0;
    __device__ __forceinline__ void add(V best2, V best4)
    {
        if constexpr (sizeof(V) == 8) {  // cell order, plain IEEE adds
            s2 = __dadd_rn(s2, best2);
            s4 = __dadd_rn(s4, best4);
        } else {  // Kahan-compensated
            const float y2 = __fsub_rn(best2, c2), u2 = __fadd_rn(s2, y2);
            c2 = __fsub_rn(__fsub_rn(u2, s2), y2);
            s2 = u2;
            const float y4 = __fsub_rn(best4, c4), u4 = __fadd_rn(s4, y4);
            c4 = __fsub_rn(__fsub_rn(u4, s4), y4);
            s4 = u4;
        }
    }
    __device__ __forceinline__ V result(int spaces, u64 b, const SolveRules &r) const
    {
        double d = 0.0;
        if (spaces) {
            const double k = (double)spaces;
            const double S2 = (double)s2 - (double)c2, S4 = (double)s4 - (double)c4;
            d = __dadd_rn(__ddiv_rn(__dmul_rn(0.9, S2), k), __ddiv_rn(__dmul_rn(0.1, S4), k));
        }
        if (r.score && d == 0.0) d = (double)tile_sum(b);
        return (V)d;
    }
};

// Direct variant: one thread per board, no queue.  The eight successors of
// one cell (2 spawns x 4 moves) are formed from the board's four views (the
// spawned nibble is OR-ed into each view), canonicalised and probed together,
// so a thread keeps up to eight independent loads in flight.
constexpr int DIRECT_THREADS = 1024;

template <typename V>
__device__ __forceinline__ void probe4(const DevTable<V> &t, const u64 *key, u32 legal, V *out)
{
    if (t.kind == INDEX_HASH && t.ch.on) {
        u64 h[4], e[4];
        u32 tag[4];
#pragma unroll
        for (int j = 0; j < 4; j++) {
            const bool on = (legal >> j) & 1 && (key[j] & t.ch.cmask) == t.ch.cval;
            h[j] = compact_home(t.ch, key[j], &tag[j]);
            e[j] = on ? __ldg((const u64 *)t.slots + h[j]) : 0ull;
        }
#pragma unroll
        for (int j = 0; j < 4; j++) {
            if ((u32)e[j] == tag[j]) out[j] = from_bits<V>(e[j] >> 32);
            else if ((u32)e[j] == 0u) out[j] = V(0);
            else out[j] = compact_probe_rest<V>((const u64 *)t.slots, t.cap, t.ch.dbits, h[j], tag[j]);
        }
        return;
    }
    if (t.kind == INDEX_HASH) {
        u64 s[4];
        ulonglong2 e[4];
#pragma unroll
        for (int j = 0; j < 4; j++) {
            const bool on = (legal >> j) & 1 && t.cap;
            s[j] = on ? home_slot(key[j], t.cap) : 0;
            e[j] = on ? __ldg(t.slots + s[j]) : make_ulonglong2(0, 0);
        }
#pragma unroll
        for (int j = 0; j < 4; j++) {
            if (!((legal >> j) & 1) || e[j].x == 0) out[j] = V(0);
            else if (e[j].x == key[j]) out[j] = from_bits<V>(e[j].y);
            else out[j] = hash_probe_rest<V>(t.slots, t.cap, key[j], s[j]);
        }
    } else {
#pragma unroll
        for (int j = 0; j < 4; j++) out[j] = ((legal >> j) & 1) ? sorted_lookup(t, key[j]) : V(0);
    }
}

// The best values of one empty cell: its eight successors (2 and 4 spawned
// into each of the board's four views, then the left move), canonicalised --
// over the plan's images when PLANNED, which the caller picks once per warp so
// that the image choice is a uniform branch -- and looked up in the s+2 and s+4
// tables, eight loads in flight.
template <bool PLANNED, typename V>
__device__ __forceinline__ void cell_bests(const RowTable &rt, const u64 v[4], int cell, const CanonPlan &plan,
                                           const DevTable<V> &t2, const DevTable<V> &t4, V &best2, V &best4,
                                           u32 &probes)
{
    u64 k2[4], k4[4];
    u32 l2 = 0, l4 = 0;
#pragma unroll
    for (int k = 0; k < 4; k++) {
        const int sh = 60 - 4 * view_cell(k, cell);
        u64 m;
        if (move_left(rt, v[k] | (1ull << sh), &m) == 2) l2 |= 1u << k;
        k2[k] = PLANNED ? canon_cand(m, plan.cand(k)) : canonical(m);
        if (move_left(rt, v[k] | (2ull << sh), &m) == 2) l4 |= 1u << k;
        k4[k] = PLANNED ? canon_cand(m, plan.cand(k)) : canonical(m);
    }
    probes += __popc(l2) + __popc(l4);
    V p2[4], p4[4];
    probe4(t2, k2, l2, p2);
    probe4(t4, k4, l4, p4);
    best2 = vmax(vmax(p2[0], p2[1]), vmax(p2[2], p2[3]));
    best4 = vmax(vmax(p4[0], p4[1]), vmax(p4[2], p4[3]));
}

// One probe of a table (the successor is looked up only when its move was legal).
template <typename V>
__device__ __forceinline__ V probe1(const DevTable<V> &t, u64 key, bool legal)
{
    if (!legal) return V(0);
    if (t.kind == INDEX_HASH && t.ch.on) {
        if ((key & t.ch.cmask) != t.ch.cval) return V(0);
        u32 tag0;
        const u64 h = compact_home(t.ch, key, &tag0);
        const u64 e = __ldg((const u64 *)t.slots + h);
        if ((u32)e == tag0) return from_bits<V>(e >> 32);
        if ((u32)e == 0u) return V(0);
        return compact_probe_rest<V>((const u64 *)t.slots, t.cap, t.ch.dbits, h, tag0);
    }
    if (t.kind == INDEX_HASH) {
        if (t.cap == 0) return V(0);
        const u64 s = home_slot(key, t.cap);
        const ulonglong2 e = __ldg(t.slots + s);
        if (e.x == key) return from_bits<V>(e.y);
        if (e.x == 0) return V(0);
        return hash_probe_rest<V>(t.slots, t.cap, key, s);
    }
    return sorted_lookup(t, key);
}

// cell_bests with the four views in a loop that is not unrolled: one view's
// two successors per iteration (two loads in flight per lane, hidden by the
// other warps), a quarter of the code.  The unrolled body of all eight
// successors is large enough that warps wait on instruction fetch.
template <bool PLANNED, typename V>
__device__ __forceinline__ void cell_bests_rolled(const RowTable &rt, u64 b, int cell, const CanonPlan &plan,
                                                  const DevTable<V> &t2, const DevTable<V> &t4, V &best2, V &best4,
                                                  u32 &probes)
{
    const Half h = halves(b), t = transpose(h);
    const int r0 = cell >> 2, q0 = cell & 3;
    best2 = V(0);
    best4 = V(0);
#pragma unroll 1
    for (int k = 0; k < 4; k++) {
        // view k: id, H, T, H.T; the cell of the spawn in it
        const Half x = (k & 2) ? t : h;
        const u64 y = (k & 1) ? whole(flip_h(x)) : whole(x);
        const int row = (k & 2) ? q0 : r0;
        const int col = ((k & 2) ? r0 : q0) ^ ((k & 1) ? 3 : 0);
        const int sh = 60 - 4 * (4 * row + col);
        u64 m2, m4;
        const bool ok2 = move_left(rt, y | (1ull << sh), &m2) == 2;
        const bool ok4 = move_left(rt, y | (2ull << sh), &m4) == 2;
        const u64 c2 = PLANNED ? canon_cand(m2, plan.cand(k)) : canonical(m2);
        const u64 c4 = PLANNED ? canon_cand(m4, plan.cand(k)) : canonical(m4);
        probes += (u32)ok2 + (u32)ok4;
        best2 = vmax(best2, probe1(t2, c2, ok2));
        best4 = vmax(best4, probe1(t4, c4, ok4));
    }
}

template <typename V>
__global__ void __launch_bounds__(DIRECT_THREADS, 1) solve_direct_kernel(const u64 *__restrict__ keys, u64 n,
                                                                         V *__restrict__ out, DevTable<V> t2,
                                                                         DevTable<V> t4, SolveRules r,
                                                                         const unsigned short *g_move,
                                                                         u64 *probes_out, CanonPlan plan)
{
    extern __shared__ __align__(16) unsigned char smem[];
    stage_table_s(smem, g_move);
    const RowTable rt{(const unsigned short *)smem};
    u32 probes = 0;
    for (u64 i = (u64)blockIdx.x * DIRECT_THREADS + threadIdx.x; i < n; i += (u64)gridDim.x * DIRECT_THREADS) {
        const u64 b = keys[i];
        // the images that can be canonical: the plan's when every board of the warp has its mask
        const bool planned = __all_sync(__activemask(), fixed_pattern(b) == plan.mask);
        V res;
        if (satisfied(b, r)) {
            res = V(1);
        } else {
            u64 e = empty_mask(b);
            const int spaces = popc64(e);
            u64 v[4];
            views(b, v);
            SpawnSums<V> sums;
            while (e) {  // cells in order 0..15 = highest nibble first
                const int bit = 63 - __clzll(e);
                e &= ~(1ull << bit);
                const int cell = (60 - bit) >> 2;
                V best2, best4;
                if (planned) cell_bests<true>(rt, v, cell, plan, t2, t4, best2, best4, probes);
                else cell_bests<false>(rt, v, cell, plan, t2, t4, best2, best4, probes);
                sums.add(best2, best4);
            }
            res = sums.result(spaces, b, r);
        }
        out[i] = res;
    }
    add_probes(probes, probes_out);
}

// Item form: the work of a warp is its boards' (board, empty cell) pairs, not
// its boards.  Boards have 0..16 empty cells, so one thread per board leaves a
// warp waiting on its fullest board; here the 32 lanes take the pairs of 32
// boards 32 at a time, every lane busy except in the last round.  A pair forms
// the eight successors of its cell (2 spawns x 4 moves, from the owner's four
// views), canonicalises them over the images its CanonPlan allows, probes the
// s+2 and s+4 tables, and leaves the two best values in shared memory; the
// owning lane then adds its pairs' values in cell order.
constexpr int ITEM_THREADS = 1024;
constexpr int ITEM_WARPS = ITEM_THREADS / 32;
constexpr int ITEM_MAX = 32 * 16;  // pairs of 32 boards at most
template <typename V>
constexpr int item_smem() { return TABLE_BYTES_S + ITEM_WARPS * (ITEM_MAX * 2 + 2 * 32 * (int)sizeof(V)); }

template <typename V>
__global__ void __launch_bounds__(ITEM_THREADS, 1)
    solve_items_kernel(const u64 *__restrict__ keys, u64 n, V *__restrict__ out, DevTable<V> t2, DevTable<V> t4,
                       SolveRules r, const unsigned short *g_move, u64 *probes_out, CanonPlan plan)
{
    extern __shared__ __align__(16) unsigned char smem[];
    stage_table_s(smem, g_move);
    const RowTable rt{(const unsigned short *)smem};
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    unsigned short *items = (unsigned short *)(smem + TABLE_BYTES_S) + warp * ITEM_MAX;  // (lane << 4) | cell
    V *best_sh = (V *)(smem + TABLE_BYTES_S + ITEM_WARPS * ITEM_MAX * 2) + warp * 64;   // [2][32]
    u32 probes = 0;
    const u64 stride = (u64)gridDim.x * ITEM_THREADS;
    for (u64 base = (u64)blockIdx.x * ITEM_THREADS + warp * 32; base < n; base += stride) {
        const u64 i = base + lane;
        const bool active = i < n;
        const u64 b = active ? keys[i] : 0;
        const bool sat = active && satisfied(b, r);
        u64 e = (active && !sat) ? empty_mask(b) : 0;
        const int spaces = popc64(e);
        const u32 inc = warp_inclusive_scan((u32)spaces);
        const u32 off = inc - (u32)spaces;
        const u32 total = __shfl_sync(0xffffffffu, inc, 31);
        // this board's pairs, cells in order 0..15 (highest nibble first)
        for (u32 j = off; e; j++) {
            const int bit = 63 - __clzll(e);
            e &= ~(1ull << bit);
            items[j] = (unsigned short)((lane << 4) | ((60 - bit) >> 2));
        }
        // the images that can be canonical: the plan's when every board of the batch has its mask
        const bool planned = __all_sync(0xffffffffu, !active || fixed_pattern(b) == plan.mask);
        __syncwarp();
        SpawnSums<V> sums;
        for (u32 r0 = 0; r0 < total; r0 += 32) {
            const u32 j = r0 + (u32)lane;
            const bool has = j < total;
            const u32 it = has ? items[j] : 0u;
            const int owner = (int)(it >> 4), cell = (int)(it & 15u);
            const u64 ob = __shfl_sync(0xffffffffu, b, owner);
            V best2 = 0, best4 = 0;
            if (has) {
                if (planned) cell_bests_rolled<true>(rt, ob, cell, plan, t2, t4, best2, best4, probes);
                else cell_bests_rolled<false>(rt, ob, cell, plan, t2, t4, best2, best4, probes);
            }
            best_sh[lane] = best2;
            best_sh[32 + lane] = best4;
            __syncwarp();
            // the owner adds the pairs of this round that are its own, in cell order
            const u32 lo = off > r0 ? off : r0;
            const u32 hi = (off + (u32)spaces) < r0 + 32 ? off + (u32)spaces : r0 + 32;
            for (u32 q = lo; q < hi; q++) sums.add(best_sh[q - r0], best_sh[32 + q - r0]);
            __syncwarp();
        }
        if (active) out[i] = sat ? V(1) : sums.result(spaces, b, r);
        __syncwarp();
    }
    add_probes(probes, probes_out);
}

// ---- index construction ----------------------------------------------------
__global__ void bucket_offsets_kernel(const u64 *__restrict__ keys, u64 n, u32 *__restrict__ off, int prefix,
                                      int bits)
{
    const u64 nb = 1ull << bits;
    for (u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x; i <= n; i += (u64)gridDim.x * blockDim.x) {
        const u64 bk = i < n ? (keys[i] << prefix) >> (64 - bits) : nb;
        const u64 bp = i ? (keys[i - 1] << prefix) >> (64 - bits) : 0;
        const u64 from = i ? bp + 1 : 0;
        for (u64 j = from; j <= bk && j <= nb; j++) off[j] = (u32)i;
    }
}

template <typename V>
__global__ void hash_build_kernel(const u64 *__restrict__ keys, const V *__restrict__ vals, u64 n,
                                  ulonglong2 *slots, u64 cap, u32 *err)
{
    for (u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (u64)gridDim.x * blockDim.x) {
        const u64 key = keys[i];
        u64 s = home_slot(key, cap);
        bool placed = false;
        for (u64 p = 0; p < cap; p++) {
            const u64 prev = atomicCAS((unsigned long long *)&slots[s].x, 0ull, (unsigned long long)key);
            if (prev == 0) {
                slots[s].y = to_bits<V>(vals[i]);
                placed = true;
                break;
            }
            s = (s + 1 == cap) ? 0 : s + 1;
        }
        if (!placed) atomicOr(err, ERR_CAPACITY);
    }
}

__global__ void key_bits_kernel(const u64 *__restrict__ keys, u64 n, unsigned long long *and_or)
{
    u64 a = ~0ull, o = 0;
    for (u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (u64)gridDim.x * blockDim.x) {
        const u64 k = keys[i];
        a &= k;
        o |= k;
    }
    for (int d = 16; d; d >>= 1) {
        a &= __shfl_xor_sync(0xffffffffu, a, d);
        o |= __shfl_xor_sync(0xffffffffu, o, d);
    }
    if ((threadIdx.x & 31) == 0) {
        atomicAnd(and_or, (unsigned long long)a);
        atomicOr(and_or + 1, (unsigned long long)o);
    }
}

__global__ void compact_build_kernel(const u64 *__restrict__ keys, const float *__restrict__ vals, u64 n,
                                     unsigned long long *slots, CompactHash c, u64 cap, u32 *err)
{
    const u32 last = (1u << c.dbits) - 1u;
    for (u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (u64)gridDim.x * blockDim.x) {
        u32 tag0;
        const u64 h = compact_home(c, keys[i], &tag0);
        const u64 vbits = (u64)__float_as_uint(vals[i]) << 32;
        bool placed = false;
        for (u32 d = 0; d + 1 < last; d++) {
            const unsigned long long prev =
                atomicCAS(slots + ((h + d) & (cap - 1)), 0ull, (unsigned long long)(vbits | (tag0 + d)));
            if (prev == 0ull) {
                placed = true;
                break;
            }
        }
        if (!placed) atomicOr(err, ERR_CAPACITY);  // the host falls back to 16-byte slots
    }
}

// ---- region-partitioned build of the 16-byte-slot index ----------------------
// The atomic build inserts every key with a compare-and-swap on a random slot of
// a table that was zeroed first: a random read-modify-write per key.  This form
// partitions the keys by region of their home slot (2048 slots = 32 KiB), builds
// each region in shared memory and writes it out whole: the table is written
// once, sequentially, and never zeroed.  A key whose linear probe runs past its
// region's end (or whose region's bucket is full) goes to an overflow list,
// inserted afterwards into the finished table with the atomic probe from its
// home slot; the slots a placed key skipped were taken when it was placed and
// stay taken, so every key stays reachable by the linear probe from its home.
constexpr u32 BUILD_REGION = 2048;

// Each region owns a bucket of `bcap` pairs in the scratch (the mean count of
// a region plus eight standard deviations and a margin, so that a bucket runs
// full almost never); a pair that finds its bucket full joins the overflow
// list.  Four keys per thread per step keep four cursor atomics in flight.
template <typename V>
__global__ void __launch_bounds__(256) region_scatter_kernel(const u64 *__restrict__ keys, const V *__restrict__ vals,
                                                             u64 n, u64 cap, u32 bcap, u32 *cursor,
                                                             ulonglong2 *tmp, ulonglong2 *overflow, u32 max_over,
                                                             u32 *n_over, u32 *err)
{
    constexpr int U = 4;
    const u64 stride = (u64)gridDim.x * blockDim.x;
    for (u64 i0 = (u64)blockIdx.x * blockDim.x + threadIdx.x; i0 < n; i0 += U * stride) {
        u64 key[U];
        V val[U];
        u32 r[U], p[U];
#pragma unroll
        for (int u = 0; u < U; u++) {
            const u64 i = i0 + u * stride;
            key[u] = i < n ? keys[i] : 0ull;
            val[u] = i < n ? vals[i] : V(0);
        }
#pragma unroll
        for (int u = 0; u < U; u++) {
            r[u] = (u32)(home_slot(key[u], cap) / BUILD_REGION);
            p[u] = i0 + u * stride < n ? atomicAdd(cursor + r[u], 1u) : 0u;
        }
#pragma unroll
        for (int u = 0; u < U; u++) {
            if (i0 + u * stride >= n) continue;
            const ulonglong2 e = make_ulonglong2(key[u], to_bits<V>(val[u]));
            if (p[u] < bcap) {
                tmp[(u64)r[u] * bcap + p[u]] = e;
            } else {
                const u32 k = atomicAdd(n_over, 1u);
                if (k < max_over) overflow[k] = e;
                else atomicOr(err, ERR_CAPACITY);
            }
        }
    }
}

__global__ void __launch_bounds__(512) region_build_kernel(const ulonglong2 *__restrict__ tmp,
                                                           const u32 *__restrict__ cursor, u32 bcap, u32 nreg,
                                                           u64 cap, ulonglong2 *slots, ulonglong2 *overflow,
                                                           u32 max_over, u32 *n_over, u32 *err)
{
    __shared__ ulonglong2 tab[BUILD_REGION];
    for (u32 r = blockIdx.x; r < nreg; r += gridDim.x) {
        for (u32 j = threadIdx.x; j < BUILD_REGION; j += blockDim.x) tab[j] = make_ulonglong2(0, 0);
        __syncthreads();
        const u64 base = (u64)r * BUILD_REGION;
        const u32 len = (u32)min((u64)BUILD_REGION, cap - base);
        const u32 cnt = min(cursor[r], bcap);
        const ulonglong2 *bucket = tmp + (u64)r * bcap;
        for (u32 j = threadIdx.x; j < cnt; j += blockDim.x) {
            const ulonglong2 e = bucket[j];
            bool placed = false;
            for (u32 sl = (u32)(home_slot(e.x, cap) - base); sl < len; sl++) {
                if (atomicCAS((unsigned long long *)&tab[sl].x, 0ull, (unsigned long long)e.x) == 0ull) {
                    tab[sl].y = e.y;
                    placed = true;
                    break;
                }
            }
            if (!placed) {
                const u32 k = atomicAdd(n_over, 1u);
                if (k < max_over) overflow[k] = e;
                else atomicOr(err, ERR_CAPACITY);
            }
        }
        __syncthreads();
        for (u32 j = threadIdx.x; j < len; j += blockDim.x) slots[base + j] = tab[j];
        __syncthreads();
    }
}

// the overflow keys, inserted into the finished table by the atomic linear probe
__global__ void overflow_insert_kernel(const ulonglong2 *__restrict__ over, u32 n, ulonglong2 *slots, u64 cap,
                                       u32 *err)
{
    for (u32 i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const ulonglong2 e = over[i];
        u64 s = home_slot(e.x, cap);
        bool placed = false;
        for (u64 p = 0; p < cap; p++) {
            if (atomicCAS((unsigned long long *)&slots[s].x, 0ull, (unsigned long long)e.x) == 0ull) {
                slots[s].y = e.y;
                placed = true;
                break;
            }
            s = (s + 1 == cap) ? 0 : s + 1;
        }
        if (!placed) atomicOr(err, ERR_CAPACITY);
    }
}

static int grid_for(u64 n, int threads, int per_sm)
{
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (sms <= 0) sms = NUM_SMS_B200;
    const u64 need = (n + threads - 1) / threads;
    return (int)std::max<u64>(1, std::min<u64>(need, (u64)sms * per_sm));
}

static bool ensure_storage(IndexStorage &st, u64 bytes, cudaStream_t s)
{
    if (st.bytes >= bytes && st.p) return true;
    if (st.p) dev_free(st.p, s);
    st.p = nullptr;
    st.bytes = 0;
    if (!dev_alloc(&st.p, bytes, s)) return false;
    st.bytes = bytes;
    return true;
}

int g_hash_compact = 1;  // FP32 hash tables in 8-byte slots where the keys allow it

// plans and builds the 8-byte-slot index of an FP32 layer: AND/OR of the keys
// give the constant bytes; the table is the power of two at or above twice the
// layer; the tag holds the remainder bits (at most 26) and the probe distance.
// Leaves ix.kind == INDEX_BISECT (nothing built) when the keys vary in too many
// bytes or a key would sit further from home than the tag can say.
static bool build_compact(LayerIndex &ix, IndexStorage &st, Counters &c, cudaStream_t s)
{
    unsigned long long init[2] = {~0ull, 0ull};
    if (!CGB_CUDA(cudaMemcpyAsync(c.d + 3, init, 16, cudaMemcpyHostToDevice, s))) return false;
    key_bits_kernel<<<grid_for(ix.n, 256, 8), 256, 0, s>>>(ix.keys, ix.n, (unsigned long long *)(c.d + 3));
    u64 ao[2];
    if (!CGB_CUDA(cudaGetLastError()) || !CGB_CUDA(cudaMemcpyAsync(ao, c.d + 3, 16, cudaMemcpyDeviceToHost, s)) ||
        !CGB_CUDA(cudaStreamSynchronize(s)))
        return false;
    int cbits = 0;
    const CompactHash ch = plan_compact(ao[0], ao[1], ix.n, &cbits);
    if (!ch.on) return true;
    const u64 cap = 1ull << cbits;
    if (!ensure_storage(st, cap * 8, s)) return false;
    if (!CGB_CUDA(cudaMemsetAsync(st.p, 0, cap * 8, s))) return false;
    if (!CGB_CUDA(cudaMemsetAsync(c.err, 0, sizeof(u32), s))) return false;
    kclock().begin(s, &kstats().index_ms);
    compact_build_kernel<<<grid_for(ix.n, 256, 16), 256, 0, s>>>(ix.keys, (const float *)ix.vals, ix.n,
                                                                 (unsigned long long *)st.p, ch, cap, c.err);
    kclock().end(s);
    u32 e = 0;
    if (!CGB_CUDA(cudaGetLastError()) || !CGB_CUDA(cudaMemcpyAsync(&e, c.err, sizeof(u32), cudaMemcpyDeviceToHost, s)) ||
        !CGB_CUDA(cudaStreamSynchronize(s)))
        return false;
    kclock().flush();
    if (e) return true;  // a probe ran past what the tag can hold: 16-byte slots instead
    ix.kind = INDEX_HASH;
    ix.slots = st.p;
    ix.cap = cap;
    ix.ch = ch;
    kstats().index_builds++;
    kstats().compact_index_builds++;
    return true;
}

int g_region_build = 1;  // 16-byte-slot indexes of 2^16..2^28 keys built region by region

// the region-partitioned build (above); leaves ix.kind == INDEX_BISECT when the
// overflow list ran out (the caller then builds with the atomic form)
static bool build_regions(LayerIndex &ix, int vbytes, IndexStorage &st, Counters &c, cudaStream_t s)
{
    const u64 n = ix.n;
    const u64 cap = hash_capacity(n);
    const u32 nreg = (u32)((cap + BUILD_REGION - 1) / BUILD_REGION);
    const u32 max_over = (u32)(n / 32 + 4096);
    // bucket size: the mean pairs of a region plus eight standard deviations and a margin
    const double mean = (double)n * BUILD_REGION / (double)cap;
    const u32 bcap = (u32)((mean + 8.0 * sqrt(mean) + 64.0 + 15.0) / 16.0) * 16u;
    if (!ensure_storage(st, cap * 16, s)) return false;
    // scratch: the cursors (u32), the region buckets, the overflow list
    const u64 bytes = 4ull * nreg + 64 + 16ull * nreg * bcap + 16ull * max_over;
    void *scratch = nullptr;
    if (!dev_alloc(&scratch, bytes, s)) return false;
    u32 *cursor = (u32 *)scratch;
    ulonglong2 *tmp = (ulonglong2 *)(((uintptr_t)(cursor + nreg) + 15) & ~(uintptr_t)15);
    ulonglong2 *over = tmp + (u64)nreg * bcap;
    bool ok = CGB_CUDA(cudaMemsetAsync(cursor, 0, 4ull * nreg, s)) &&
              CGB_CUDA(cudaMemsetAsync(c.d + 6, 0, sizeof(u64), s)) && CGB_CUDA(cudaMemsetAsync(c.err, 0, 4, s));
    u32 *n_over = (u32 *)(c.d + 6);
    if (ok) {
        kclock().begin(s, &kstats().index_ms);
        const int grid = grid_for((n + 3) / 4, 256, 8);
        if (vbytes == 8)
            region_scatter_kernel<double><<<grid, 256, 0, s>>>(ix.keys, (const double *)ix.vals, n, cap, bcap,
                                                                cursor, tmp, over, max_over, n_over, c.err);
        else
            region_scatter_kernel<float><<<grid, 256, 0, s>>>(ix.keys, (const float *)ix.vals, n, cap, bcap,
                                                               cursor, tmp, over, max_over, n_over, c.err);
        region_build_kernel<<<std::min<u32>(nreg, (u32)NUM_SMS_B200 * 4), 512, 0, s>>>(
            tmp, cursor, bcap, nreg, cap, (ulonglong2 *)st.p, over, max_over, n_over, c.err);
        kclock().end(s);
        kstats().launches += 2;
        ok = CGB_CUDA(cudaGetLastError());
    }
    u32 h[2] = {0, 0};  // overflow count, error word
    ok = ok && CGB_CUDA(cudaMemcpyAsync(&h[0], n_over, 4, cudaMemcpyDeviceToHost, s)) &&
         CGB_CUDA(cudaMemcpyAsync(&h[1], c.err, 4, cudaMemcpyDeviceToHost, s)) && CGB_CUDA(cudaStreamSynchronize(s));
    kclock().flush();
    if (ok && h[1] == 0 && h[0]) {
        kclock().begin(s, &kstats().index_ms);
        overflow_insert_kernel<<<std::max<u32>(1, std::min<u32>((h[0] + 255) / 256, 1024)), 256, 0, s>>>(
            over, h[0], (ulonglong2 *)st.p, cap, c.err);
        kclock().end(s);
        kstats().launches++;
        ok = CGB_CUDA(cudaGetLastError()) && CGB_CUDA(cudaMemcpyAsync(&h[1], c.err, 4, cudaMemcpyDeviceToHost, s)) &&
             CGB_CUDA(cudaStreamSynchronize(s));
        kclock().flush();
    }
    dev_free(scratch, s);
    if (!ok) return false;
    if (h[1]) return true;  // the overflow list ran out: the atomic build instead
    ix.kind = INDEX_HASH;
    ix.slots = st.p;
    ix.cap = cap;
    kstats().index_builds++;
    return true;
}

bool build_index(LayerIndex &ix, int kind, int vbytes, IndexStorage &st, int bucket_bits, Counters &c,
                 cudaStream_t s)
{
    ix.kind = INDEX_BISECT;
    ix.bucket = nullptr;
    ix.slots = nullptr;
    ix.cap = 0;
    if (ix.n == 0 || kind == INDEX_BISECT) return true;
    ix.ch = CompactHash{};
    if (kind == INDEX_HASH && vbytes == 4 && g_hash_compact && ix.n >= 64) {
        if (!build_compact(ix, st, c, s)) return false;
        if (ix.kind == INDEX_HASH) return true;
    }
    if (kind == INDEX_HASH && g_region_build && ix.n >= (1u << 16) && ix.n <= (1u << 28)) {
        if (!build_regions(ix, vbytes, st, c, s)) return false;
        if (ix.kind == INDEX_HASH) return true;
    }
    if (kind == INDEX_HASH) {
        // load factor <= g_hash_load_pct: capacity rounded up to a multiple of 64 slots
        const u64 cap = hash_capacity(ix.n);
        if (!ensure_storage(st, cap * 16, s)) return false;
        if (!CGB_CUDA(cudaMemsetAsync(st.p, 0, cap * 16, s))) return false;
        if (!CGB_CUDA(cudaMemsetAsync(c.err, 0, sizeof(u32), s))) return false;
        kclock().begin(s, &kstats().index_ms);
        if (vbytes == 8)
            hash_build_kernel<double><<<grid_for(ix.n, 256, 16), 256, 0, s>>>(
                ix.keys, (const double *)ix.vals, ix.n, (ulonglong2 *)st.p, cap, c.err);
        else
            hash_build_kernel<float><<<grid_for(ix.n, 256, 16), 256, 0, s>>>(
                ix.keys, (const float *)ix.vals, ix.n, (ulonglong2 *)st.p, cap, c.err);
        kclock().end(s);
        if (!CGB_CUDA(cudaGetLastError())) return false;
        u32 e = 0;
        if (!CGB_CUDA(cudaMemcpyAsync(&e, c.err, sizeof(u32), cudaMemcpyDeviceToHost, s))) return false;
        if (!CGB_CUDA(cudaStreamSynchronize(s))) return false;
        kclock().flush();
        if (e) {
            set_error("build_index: device error " + err_string(e));
            return false;
        }
        ix.kind = INDEX_HASH;
        ix.slots = st.p;
        ix.cap = cap;
        kstats().index_builds++;
        return true;
    }
    // INDEX_BUCKET
    if (ix.n < 64 || bucket_bits <= 0) return true;
    u64 first, last;
    if (!CGB_CUDA(cudaMemcpyAsync(&first, ix.keys, 8, cudaMemcpyDeviceToHost, s))) return false;
    if (!CGB_CUDA(cudaMemcpyAsync(&last, ix.keys + ix.n - 1, 8, cudaMemcpyDeviceToHost, s))) return false;
    if (!CGB_CUDA(cudaStreamSynchronize(s))) return false;
    const u64 x = first ^ last;
    const int prefix = x ? __builtin_clzll(x) : 64;
    int bits = bucket_bits;
    if (bits > 64 - prefix) bits = 64 - prefix;
    if (bits <= 0) return true;
    const u64 need = ((1ull << bits) + 1) * sizeof(u32);
    if (!ensure_storage(st, need, s)) return false;
    kclock().begin(s, &kstats().index_ms);
    bucket_offsets_kernel<<<grid_for(ix.n + 1, 256, 16), 256, 0, s>>>(ix.keys, ix.n, (u32 *)st.p, prefix, bits);
    kclock().end(s);
    if (!CGB_CUDA(cudaGetLastError())) return false;
    ix.kind = INDEX_BUCKET;
    ix.bucket = (const u32 *)st.p;
    ix.prefix = prefix;
    ix.bits = bits;
    ix.prefix_value = prefix ? first >> (64 - prefix) : 0;
    return true;
}

template <typename V>
static DevTable<V> dev_table(const LayerIndex &ix)
{
    DevTable<V> t;
    t.kind = ix.kind;
    t.keys = ix.keys;
    t.vals = (const V *)ix.vals;
    t.n = ix.n;
    t.bucket = ix.bucket;
    t.prefix = ix.prefix;
    t.bits = ix.bits;
    t.prefix_value = ix.prefix_value;
    t.slots = (const ulonglong2 *)ix.slots;
    t.cap = ix.kind == INDEX_HASH ? ix.cap : 0;
    t.ch = ix.ch;
    return t;
}

int g_solve_variant = 1;  // 0: direct (one thread per board), 1: (board, cell) pairs per warp

static bool solve_attrs()
{
    static bool attr = false;
    if (!attr) {
        if (!CGB_CUDA(cudaFuncSetAttribute(solve_items_kernel<double>,
                                           cudaFuncAttributeMaxDynamicSharedMemorySize, item_smem<double>())) ||
            !CGB_CUDA(cudaFuncSetAttribute(solve_items_kernel<float>,
                                           cudaFuncAttributeMaxDynamicSharedMemorySize, item_smem<float>())) ||
            !CGB_CUDA(cudaFuncSetAttribute(solve_direct_kernel<double>,
                                           cudaFuncAttributeMaxDynamicSharedMemorySize, TABLE_BYTES_S)) ||
            !CGB_CUDA(cudaFuncSetAttribute(solve_direct_kernel<float>,
                                           cudaFuncAttributeMaxDynamicSharedMemorySize, TABLE_BYTES_S)))
            return false;
        attr = true;
    }
    return true;
}

// the kernel launch alone: no host round trip, so it may be captured in a graph
template <class V>
static void enqueue_solve(const u64 *keys, u64 n, V *out, const LayerIndex &t2, const LayerIndex &t4,
                          const SolveRules &r, const DeviceRowTable &rt, u64 *probes, cudaStream_t s,
                          const CanonPlan &plan)
{
    if (g_solve_variant == 1)
        solve_items_kernel<V><<<grid_for(n, ITEM_THREADS, 1), ITEM_THREADS, item_smem<V>(), s>>>(
            keys, n, out, dev_table<V>(t2), dev_table<V>(t4), r, rt.move, probes, plan);
    else
        solve_direct_kernel<V><<<grid_for(n, DIRECT_THREADS, 1), DIRECT_THREADS, TABLE_BYTES_S, s>>>(
            keys, n, out, dev_table<V>(t2), dev_table<V>(t4), r, rt.move, probes, plan);
}

template <class V>
static bool launch_solve(const u64 *keys, u64 n, V *out, const LayerIndex &t2, const LayerIndex &t4,
                         const SolveRules &r, const DeviceRowTable &rt, Counters &c, cudaStream_t s,
                         const CanonPlan &plan)
{
    if (n == 0) return true;
    if (!solve_attrs()) return false;
    if (!CGB_CUDA(cudaMemsetAsync(c.d + 2, 0, sizeof(u64), s))) return false;
    kclock().begin(s, &kstats().solve_ms);
    enqueue_solve<V>(keys, n, out, t2, t4, r, rt, c.d + 2, s, plan);
    kclock().end(s);
    if (!CGB_CUDA(cudaGetLastError())) return false;
    u64 probes = 0;
    if (!CGB_CUDA(cudaMemcpyAsync(&probes, c.d + 2, sizeof(u64), cudaMemcpyDeviceToHost, s))) return false;
    if (!CGB_CUDA(cudaStreamSynchronize(s))) return false;
    kclock().flush();
    KernelStats &k = kstats();
    k.solve_launches++;
    k.solve_boards += n;
    k.lookups += probes;
    // keys in, values out, one key sector and one value sector per probe
    k.solve_bytes += (8 + sizeof(V)) * n + 64 * probes;
    return true;
}

bool solve_layer_enqueue(const u64 *keys, u64 n, void *out, int vbytes, const LayerIndex &t2, const LayerIndex &t4,
                         const SolveRules &r, const DeviceRowTable &rt, u64 *probes, cudaStream_t s)
{
    if (n == 0) return true;
    if (!solve_attrs()) return false;
    if (vbytes == 4) enqueue_solve<float>(keys, n, (float *)out, t2, t4, r, rt, probes, s, CanonPlan{});
    else enqueue_solve<double>(keys, n, (double *)out, t2, t4, r, rt, probes, s, CanonPlan{});
    KernelStats &k = kstats();
    k.solve_launches++;
    k.solve_boards += n;
    return CGB_CUDA(cudaGetLastError());
}

bool solve_prepare() { return solve_attrs(); }

// target load factor of the hash index, percent; 0 = by size: 25 % (64 bytes
// of slots per board: fewer probes, measured 10 % faster solve + build on LL
// layers than 45 %) up to 2^27 keys, 45 % above, where table memory counts
int g_hash_load_pct = 0;

u64 hash_capacity(u64 n)
{
    const u64 pct = g_hash_load_pct ? (u64)g_hash_load_pct : (n <= (1ull << 27) ? 25 : 45);
    return hash_capacity_for(n, pct);
}

bool build_hash_enqueue(LayerIndex &ix, int vbytes, void *slots, u64 cap, u32 *err, cudaStream_t s)
{
    ix.ch = CompactHash{};
    ix.kind = INDEX_BISECT;
    ix.bucket = nullptr;
    ix.slots = nullptr;
    ix.cap = 0;
    if (ix.n == 0) return true;
    if (!CGB_CUDA(cudaMemsetAsync(slots, 0, cap * 16, s))) return false;
    if (vbytes == 8)
        hash_build_kernel<double><<<grid_for(ix.n, 256, 16), 256, 0, s>>>(ix.keys, (const double *)ix.vals, ix.n,
                                                                         (ulonglong2 *)slots, cap, err);
    else
        hash_build_kernel<float><<<grid_for(ix.n, 256, 16), 256, 0, s>>>(ix.keys, (const float *)ix.vals, ix.n,
                                                                        (ulonglong2 *)slots, cap, err);
    ix.kind = INDEX_HASH;
    ix.slots = slots;
    ix.cap = cap;
    return CGB_CUDA(cudaGetLastError());
}

bool solve_layer_f64(const u64 *keys, u64 n, double *out, const LayerIndex &t2, const LayerIndex &t4,
                     const SolveRules &r, const DeviceRowTable &rt, Counters &c, cudaStream_t s, const CanonPlan &plan)
{
    return launch_solve<double>(keys, n, out, t2, t4, r, rt, c, s, plan);
}

bool solve_layer_f32(const u64 *keys, u64 n, float *out, const LayerIndex &t2, const LayerIndex &t4,
                     const SolveRules &r, const DeviceRowTable &rt, Counters &c, cudaStream_t s, const CanonPlan &plan)
{
    return launch_solve<float>(keys, n, out, t2, t4, r, rt, c, s, plan);
}

// ---- batch lookup (lookup(), src/solve.c:108-164, for many boards) --------
template <typename V>
__global__ void __launch_bounds__(256) lookup_batch_kernel(DevTable<V> t, const u64 *__restrict__ boards, u64 m,
                                                           int canon, double *__restrict__ out)
{
    for (u64 i = (u64)blockIdx.x * 256 + threadIdx.x; i < m; i += (u64)gridDim.x * 256) {
        const u64 b = boards[i];
        out[i] = (double)table_value(t, canon ? canonical(b) : b);
    }
}

bool lookup_batch(const LayerIndex &ix, int vbytes, const u64 *boards, u64 m, bool canon, double *out,
                  cudaStream_t s)
{
    if (m == 0) return true;
    const int grid = grid_for(m, 256, 8);
    if (vbytes == 4)
        lookup_batch_kernel<float><<<grid, 256, 0, s>>>(dev_table<float>(ix), boards, m, canon ? 1 : 0, out);
    else
        lookup_batch_kernel<double><<<grid, 256, 0, s>>>(dev_table<double>(ix), boards, m, canon ? 1 : 0, out);
    kstats().launches++;
    return CGB_CUDA(cudaGetLastError());
}

}  // namespace cgb
