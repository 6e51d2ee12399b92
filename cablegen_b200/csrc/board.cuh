// board.cuh -- device-side board primitives for the 2048 tablebase engine.
//
// A board is a u64 of 16 nibbles; nibble 0 (bits 63..60) is the top-left cell,
// cells run row-major (api/cablegen.h:9-12).  Row k (cells 4k..4k+3) occupies
// bits 63-16k .. 48-16k, its leftmost cell in the row's high nibble.
//
// Geometry is expressed through three involutions that map onto cheap
// 32-bit byte permutes: V (reverse the row order), H (reverse each row) and
// T (transpose).  The eight symmetries of the square are {X, X.T} for
// X in {id, V, H, VH}; the canonical board is the unsigned maximum over that
// orbit, which equals the reference's scalar canonicalize_b
// (src/board.c:314-337) because both take the maximum over the same set.
//
// Moves: the reference moves up by rotating clockwise and moving right, down
// by rotating clockwise and moving left (src/board.c:195-214), and right uses
// the mirrored LUT.  Since rot_cw = H.T and right(x) = H(left(H x)) (checked
// exhaustively against the reference LUT for every settings combination), the
// canonical results of the four directions are canon(left(y)) for the four
// "views" y in {b, H b, T b, H T b}; only the left-move row table is needed.
#pragma once
#include <stdint.h>

namespace cgb {

typedef uint64_t u64;
typedef unsigned int u32;

__host__ __device__ __forceinline__ u64 make64(u32 hi, u32 lo) { return ((u64)hi << 32) | lo; }

#ifdef __CUDA_ARCH__
__device__ __forceinline__ u32 prmt(u32 a, u32 sel) { return __byte_perm(a, 0, sel); }
#else
inline u32 prmt(u32 a, u32 sel)
{
    u32 out = 0;
    for (int i = 0; i < 4; i++) {
        u32 s = (sel >> (4 * i)) & 7;
        u32 byte = s < 4 ? (a >> (8 * s)) & 0xFF : 0;
        out |= byte << (8 * i);
    }
    return out;
}
#endif

// reverse the nibbles of each 16-bit half-word of a 32-bit word
__host__ __device__ __forceinline__ u32 rev_rows32(u32 x)
{
    x = prmt(x, 0x2301);                                      // swap bytes inside each half-word
    return ((x >> 4) & 0x0F0F0F0Fu) | ((x << 4) & 0xF0F0F0F0u); // swap nibbles inside each byte
}

// A board as two 32-bit words: hi = rows 0-1 (cells 0..7), lo = rows 2-3.
struct Half {
    u32 hi, lo;
};
__host__ __device__ __forceinline__ Half halves(u64 b) { return Half{(u32)(b >> 32), (u32)b}; }
__host__ __device__ __forceinline__ u64 whole(Half h) { return make64(h.hi, h.lo); }

// V: reverse the order of the four rows
__host__ __device__ __forceinline__ Half flip_v(Half b) { return Half{prmt(b.lo, 0x1032), prmt(b.hi, 0x1032)}; }
// H: mirror every row left<->right
__host__ __device__ __forceinline__ Half flip_h(Half b) { return Half{rev_rows32(b.hi), rev_rows32(b.lo)}; }
// T: transpose the 4x4 nibble matrix (cell (r,c) <-> (c,r)): inside each
// 2x2 block by one delta swap per word (cells 1<->4, 3<->6, 9<->12, 11<->14),
// then the off-diagonal 2x2 blocks by two byte permutes across the words
// (cells 2,3 <-> 8,9 and 6,7 <-> 12,13).
__host__ __device__ __forceinline__ Half transpose(Half b)
{
    u32 t = ((b.hi >> 12) ^ b.hi) & 0x0000F0F0u;
    const u32 hi = b.hi ^ t ^ (t << 12);
    t = ((b.lo >> 12) ^ b.lo) & 0x0000F0F0u;
    const u32 lo = b.lo ^ t ^ (t << 12);
#ifdef __CUDA_ARCH__
    return Half{__byte_perm(hi, lo, 0x3715), __byte_perm(hi, lo, 0x2604)};
#else
    auto perm2 = [](u32 x, u32 y, u32 sel) {
        const u64 v = ((u64)y << 32) | x;
        u32 out = 0;
        for (int i = 0; i < 4; i++) out |= (u32)((v >> (8 * ((sel >> (4 * i)) & 7))) & 0xFF) << (8 * i);
        return out;
    };
    return Half{perm2(hi, lo, 0x3715), perm2(hi, lo, 0x2604)};
#endif
}

__host__ __device__ __forceinline__ u64 flip_v(u64 b) { return whole(flip_v(halves(b))); }
__host__ __device__ __forceinline__ u64 flip_h(u64 b) { return whole(flip_h(halves(b))); }
__host__ __device__ __forceinline__ u64 transpose(u64 b) { return whole(transpose(halves(b))); }

__host__ __device__ __forceinline__ u64 umax64(u64 a, u64 b) { return a > b ? a : b; }

// the 8 images of the square's symmetry group: {X, X.T} for X in {id, V, H, VH}
__host__ __device__ __forceinline__ void images(u64 b, u64 img[8])
{
    const Half h = halves(b), t = transpose(h);
    const Half hv = flip_v(h), tv = flip_v(t), hh = flip_h(h), th = flip_h(t);
    img[0] = whole(h);
    img[1] = whole(hv);
    img[2] = whole(hh);
    img[3] = whole(flip_v(hh));
    img[4] = whole(t);
    img[5] = whole(tv);
    img[6] = whole(th);
    img[7] = whole(flip_v(th));
}

// canonical representative: unsigned max over the 8 symmetries
__host__ __device__ __forceinline__ u64 canonical(u64 b)
{
    u64 im[8];
    images(b, im);
    return umax64(umax64(umax64(im[0], im[1]), umax64(im[2], im[3])),
                  umax64(umax64(im[4], im[5]), umax64(im[6], im[7])));
}

// Cell permutations of the images: image k of (b with cell c set) equals
// image k of b with cell image_cell(k, c) set.  Cell c = 4r + q.
//   V: (r,q)->(3-r,q)  H: (r,q)->(r,3-q)  T: (r,q)->(q,r)
__host__ __device__ __forceinline__ int image_cell(int k, int c)
{
    const int r = c >> 2, q = c & 3;
    switch (k) {
    case 0: return c;                          // id
    case 1: return 4 * (3 - r) + q;            // V
    case 2: return 4 * r + (3 - q);            // H
    case 3: return 4 * (3 - r) + (3 - q);      // VH
    case 4: return 4 * q + r;                  // T
    case 5: return 4 * (3 - q) + r;            // V.T
    case 6: return 4 * q + (3 - r);            // H.T
    default: return 4 * (3 - q) + (3 - r);     // VH.T
    }
}

// reference rotate_clockwise (src/board.c:239-248): new (r,c) = old (3-c, r)
__host__ __device__ __forceinline__ u64 rot_cw(u64 b) { return flip_h(transpose(b)); }
__host__ __device__ __forceinline__ u64 rot_ccw(u64 b) { return transpose(flip_h(b)); }

__host__ __device__ __forceinline__ int tile_at(u64 b, int cell) { return (int)((b >> (60 - 4 * cell)) & 0xF); }
__host__ __device__ __forceinline__ u64 set_tile(u64 b, int cell, u64 v)
{
    const int sh = 60 - 4 * cell;
    return (b & ~(0xFull << sh)) | (v << sh);
}

// one bit per nibble (in the nibble's low bit) for every empty cell
__host__ __device__ __forceinline__ u64 empty_mask(u64 b)
{
    u64 x = b | (b >> 2);
    x |= x >> 1;
    return ~x & 0x1111111111111111ull;
}

#ifdef __CUDA_ARCH__
__device__ __forceinline__ int popc64(u64 x) { return __popcll(x); }
#else
inline int popc64(u64 x) { return __builtin_popcountll(x); }
#endif

// tile sum (src/board.c:340-347): 2^e for e not in {0, 0xe, 0xf}
__host__ __device__ __forceinline__ int tile_sum(u64 b)
{
    int s = 0;
#pragma unroll
    for (int c = 0; c < 16; c++) {
        int e = (int)((b >> (4 * c)) & 0xF);
        s += (e != 0 && e < 0xE) ? (1 << e) : 0;
    }
    return s;
}

// 16-bit mask of the cells holding 0xf (a fixed formation cell): bit i is set
// when nibble i, counted from the least significant nibble, is 0xf.  With
// fixed cells that never move, the mask of a canonical board is one of the 8
// images of its formation's mask, so it tells formations with disjoint mask
// orbits apart.
__host__ __device__ __forceinline__ u32 fixed_pattern(u64 b)
{
    u64 x = b & (b >> 1) & (b >> 2) & (b >> 3) & 0x1111111111111111ull;
    x = (x | (x >> 3)) & 0x0303030303030303ull;
    x = (x | (x >> 6)) & 0x000F000F000F000Full;
    x = (x | (x >> 12)) & 0x000000FF000000FFull;
    x = (x | (x >> 24)) & 0xFFFFull;
    return (u32)x;
}

// batched sweeps: formation id of a board from its fixed-cell mask (0xff: no
// formation of the batch) and whether that formation still generates
struct FormationFilter {
    const unsigned char *fid = nullptr;     // 65536 entries, by fixed_pattern()
    const unsigned char *active = nullptr;  // 256 entries
};

// prune predicate (src/generate.c:98-131).  It depends only on the multiset of
// tile values, so it may be evaluated on any orientation of the board.
struct PruneParams {
    long long stsl, ltc, smallest_large;
    int enabled;
};

__host__ __device__ __forceinline__ bool prune_board(u64 b, const PruneParams &p)
{
    // one-hot bit of each tile value: values below smallest_large are small (their
    // one-hot bit is their weight 2^e, an empty cell weighing 1), values from it up
    // to 0xd are large.  Copies of a large value other than smallest_large pass
    // through once/twice/thrice; smallest_large's first three copies are free, so
    // it dies at its sixth copy.
    const long long sl = p.smallest_large;
    const u32 small_mask = sl <= 0 ? 0u : (sl >= 14 ? 0x3FFFu : (1u << sl) - 1u);
    const u32 large_mask = 0x3FFFu & ~small_mask;
    const u32 sl_bit = (sl >= 0 && sl < 14) ? (1u << sl) : 0u;
    const u32 chain_mask = large_mask & ~sl_bit;
    const u32 w[2] = {(u32)(b >> 32), (u32)b};
    u32 once = 0, twice = 0, thrice = 0, small = 0;
    int large = 0, sl_count = 0;
#pragma unroll
    for (int k = 0; k < 16; k++) {
        const u32 bit = 1u << ((w[k >> 3] >> (4 * (k & 7))) & 0xF);
        small += bit & small_mask;
        large += (bit & large_mask) != 0;
        sl_count += bit == sl_bit;
        const u32 c = bit & chain_mask;
        thrice |= twice & c;
        twice |= once & c;
        once |= c;
    }
    return thrice != 0 || sl_count >= 6 || (long long)small > p.stsl + 64 || large > p.ltc;
}

// The same predicate from per-byte tables: a board is 8 bytes of two cells
// each, so 8 lookups give the small-tile weight (u32), and the number of copies
// of every large value as byte-wide counters (values 0-7 in one u64, 8-15 in
// the other; a value is counted only when it is large).  Then the large count
// is the sum of the counters, the third-copy rule is "a chain value's counter
// is at least 3" (0x7D added to a byte reaches 0x80 exactly at 3), and the
// smallest_large rule is its own counter reaching 6.  About 90 operations per
// board instead of about 220 for the per-cell loop; prune_board is the
// definition, PruneTable the fast form (the host test checks both).
struct PruneTable {
    u32 small[256];
    u64 cnt_lo[256], cnt_hi[256];
    u64 chain_lo, chain_hi;  // 0x80 in the bytes of chain values (large, not smallest_large)
    int sl_field;            // byte index (0-15) of smallest_large's counter, -1 if none
    long long stsl, ltc;
};

inline void build_prune_table(const PruneParams &p, PruneTable *t)
{
    const long long sl = p.smallest_large;
    const u32 small_mask = sl <= 0 ? 0u : (sl >= 14 ? 0x3FFFu : (1u << sl) - 1u);
    const u32 large_mask = 0x3FFFu & ~small_mask;
    const u32 sl_bit = (sl >= 0 && sl < 14) ? (1u << sl) : 0u;
    const u32 chain_mask = large_mask & ~sl_bit;
    for (int b = 0; b < 256; b++) {
        u32 sm = 0;
        u64 lo = 0, hi = 0;
        for (int h = 0; h < 2; h++) {
            const int x = h ? (b & 15) : (b >> 4);
            const u32 bit = 1u << x;
            sm += bit & small_mask;
            if (bit & large_mask) {
                if (x < 8) lo += 1ull << (8 * x);
                else hi += 1ull << (8 * (x - 8));
            }
        }
        t->small[b] = sm;
        t->cnt_lo[b] = lo;
        t->cnt_hi[b] = hi;
    }
    t->chain_lo = t->chain_hi = 0;
    for (int x = 0; x < 16; x++) {
        if (!((1u << x) & chain_mask)) continue;
        if (x < 8) t->chain_lo |= 0x80ull << (8 * x);
        else t->chain_hi |= 0x80ull << (8 * (x - 8));
    }
    t->sl_field = sl_bit ? (int)sl : -1;
    t->stsl = p.stsl;
    t->ltc = p.ltc;
}

__host__ __device__ __forceinline__ bool prune_by_table(u64 b, const PruneTable &t)
{
    u32 small = 0;
    u64 lo = 0, hi = 0;
#pragma unroll
    for (int i = 0; i < 8; i++) {
        const u32 byte = (u32)(b >> (8 * i)) & 0xFFu;
        small += t.small[byte];
        lo += t.cnt_lo[byte];
        hi += t.cnt_hi[byte];
    }
    const u64 ones = 0x0101010101010101ull;
    const int large = (int)(((lo + hi) * ones) >> 56);  // counters <= 16, their sum <= 16
    const bool thrice = (((lo + 0x7D * ones) & t.chain_lo) | ((hi + 0x7D * ones) & t.chain_hi)) != 0;
    const int slc = t.sl_field < 0 ? 0 : (int)(((t.sl_field < 8 ? lo : hi) >> (8 * (t.sl_field & 7))) & 0xFF);
    return thrice || slc >= 6 || (long long)small > t.stsl + 64 || large > t.ltc;
}

// contains tile x?  (src/generate.c:89-96 returns the negation)
__host__ __device__ __forceinline__ bool has_tile(u64 b, int x)
{
    if (x < 0 || x > 15) return false;
    u64 y = b ^ (0x1111111111111111ull * (u64)x);
    return empty_mask(y) != 0;
}

// winstate pattern test (src/solve.c:226-231): every nonzero nibble of w must match
__host__ __device__ __forceinline__ bool matches(u64 b, u64 w)
{
    u64 m = w | (w >> 2);
    m = (m | (m >> 1)) & 0x1111111111111111ull;
    return (b & (m * 0xF)) == w;
}

// ---- the row table in shared memory -------------------------------------
// move[row]: the row after a left move.  A row whose move would take a 0xf
// cell out of place (the reference's _locked_lut, src/board.c:29-38,117) holds
// ROW_LOCKED instead: a left move never yields 0x0001 (empty cells, then a
// tile that did not slide), so the value is free to mark "illegal" and the
// table needs no second bitset (build_row_table checks this for every row).
constexpr unsigned short ROW_LOCKED = 0x0001;

struct RowTable {
    const unsigned short *move;  // 65536 entries, ROW_LOCKED for locked rows
};

// left move of the four rows of y; returns 0 when any row is locked, else
// sets *out and returns 1 + (changed ? 1 : 0)
__device__ __forceinline__ int move_left(const RowTable &t, u64 y, u64 *out)
{
    const u32 hi = (u32)(y >> 32), lo = (u32)y;
    const u32 m0 = t.move[hi >> 16], m1 = t.move[hi & 0xFFFFu];
    const u32 m2 = t.move[lo >> 16], m3 = t.move[lo & 0xFFFFu];
    const bool locked = (m0 == ROW_LOCKED) | (m1 == ROW_LOCKED) | (m2 == ROW_LOCKED) | (m3 == ROW_LOCKED);
    const u64 r = make64(__byte_perm(m1, m0, 0x5410), __byte_perm(m3, m2, 0x5410));
    *out = r;
    return locked ? 0 : 1 + (int)(r != y);
}

// ---- canonical form from a subset of the images ---------------------------
// A 0xf nibble is larger than any tile, so among the 8 images of a board the
// maximum is one whose run of leading 0xf cells (from cell 0) is longest.
// With fixed formation cells (free_formation off) a legal move keeps every
// 0xf cell in place, so the 0xf-mask of a move result in view k of a board is
// the view of the board's mask, and the images that can be the maximum are
// known before the move: canon_cand() takes the maximum over those only.
// CanonPlan holds them for boards whose fixed_pattern() equals `mask`; a
// board with any other mask uses all eight (cand 0xff).
struct CanonPlan {
    u32 mask = 0xFFFFFFFFu;   // fixed_pattern() the plan is for (never equal: no plan)
    u32 views = 0xFFFFFFFFu;  // byte k: images for a move result in view k
    __host__ __device__ __forceinline__ u32 cand(int k) const { return (views >> (8 * k)) & 0xFFu; }
};

// cand: bit i = image i of images() (id, V, H, VH, T, VT, HT, VHT)
__host__ __device__ __forceinline__ u64 canon_cand(u64 m, u32 cand)
{
    if (cand == 0xFFu) return canonical(m);
    const Half h = halves(m);
    u64 best = 0;
    if (cand & 0x0Fu) {
        if (cand & 0x01u) best = umax64(best, m);
        if (cand & 0x02u) best = umax64(best, whole(flip_v(h)));
        if (cand & 0x0Cu) {
            const Half hh = flip_h(h);
            if (cand & 0x04u) best = umax64(best, whole(hh));
            if (cand & 0x08u) best = umax64(best, whole(flip_v(hh)));
        }
    }
    if (cand & 0xF0u) {
        const Half t = transpose(h);
        if (cand & 0x10u) best = umax64(best, whole(t));
        if (cand & 0x20u) best = umax64(best, whole(flip_v(t)));
        if (cand & 0xC0u) {
            const Half th = flip_h(t);
            if (cand & 0x40u) best = umax64(best, whole(th));
            if (cand & 0x80u) best = umax64(best, whole(flip_v(th)));
        }
    }
    return best;
}

__host__ __device__ __forceinline__ int leading_f(u64 b)
{
    int n = 0;
    while (n < 16 && ((b >> (60 - 4 * n)) & 0xF) == 0xF) n++;
    return n;
}

// the four move views of b: {b, H b, T b, H T b} for left, right, up, down
__host__ __device__ __forceinline__ void views(u64 b, u64 v[4])
{
    const Half h = halves(b), t = transpose(h);
    v[0] = b;
    v[1] = whole(flip_h(h));
    v[2] = whole(t);
    v[3] = whole(flip_h(t));
}

// cell of view k (id, H, T, H.T) that holds cell c of the board
__host__ __device__ __forceinline__ int view_cell(int k, int c)
{
    return image_cell(k == 0 ? 0 : k == 1 ? 2 : k == 2 ? 4 : 6, c);
}

// the plan for boards whose 0xf cells are those of `b` (host side, once per
// sweep): for each view k, the images of view_k(mask) with the longest run of
// leading 0xf cells.  free_formation lets 0xf cells move: no plan.
inline CanonPlan make_canon_plan(u64 b, bool free_formation)
{
    CanonPlan p;
    if (free_formation) return p;
    u64 x = 0;  // the 0xf cells of b, every other cell empty
    for (int c = 0; c < 16; c++)
        if (((b >> (60 - 4 * c)) & 0xF) == 0xF) x |= 0xFull << (60 - 4 * c);
    if (x == 0) return p;
    u64 v[4];
    views(x, v);
    for (int k = 0; k < 4; k++) {
        u64 im[8];
        images(v[k], im);
        int best = -1;
        for (int i = 0; i < 8; i++) best = leading_f(im[i]) > best ? leading_f(im[i]) : best;
        unsigned char cand = 0;
        for (int i = 0; i < 8; i++)
            if (leading_f(im[i]) == best) cand |= (unsigned char)(1u << i);
        p.views = (p.views & ~(0xFFu << (8 * k))) | ((u32)(best > 0 ? cand : 0xFF) << (8 * k));
    }
    p.mask = fixed_pattern(b);
    return p;
}

}  // namespace cgb
