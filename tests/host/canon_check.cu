// Host-side check of the canonical-form plans of cablegen_b200/csrc/board.cuh:
// for formation masks given as hex 16-bit cell sets in argv[1..] (bit c = cell c
// holds 0xf), random boards with those 0xf cells (in every orientation) are
// moved into each view, their non-0xf cells redrawn, and canon_cand() with the
// plan's images for that view is compared with the full canonical().  Prints
// "<mask> <boards checked> <mismatches> <images per view...>" per mask.
#include "../../cablegen_b200/csrc/board.cuh"
#include <cstdio>
#include <cstdlib>

static uint64_t state = 0x9E3779B97F4A7C15ull;
static uint64_t next()
{
    uint64_t z = (state += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

int main(int argc, char **argv)
{
    using namespace cgb;
    for (int a = 1; a < argc; a++) {
        const unsigned cells = (unsigned)std::strtoul(argv[a], nullptr, 16);
        u64 base = 0;
        for (int c = 0; c < 16; c++)
            if (cells >> c & 1) base |= 0xFull << (60 - 4 * c);
        u64 checked = 0, bad = 0;
        CanonPlan plan0 = make_canon_plan(base, false);
        for (int orient = 0; orient < 8; orient++) {
            u64 img[8];
            images(base, img);
            const u64 shape = img[orient];  // the 0xf cells in one orientation
            const CanonPlan plan = make_canon_plan(shape, false);
            for (int it = 0; it < 20000; it++) {
                // a board with exactly these 0xf cells: other cells empty or tiles 1..14
                u64 x = shape;
                for (int c = 0; c < 16; c++) {
                    if (((shape >> (60 - 4 * c)) & 0xF) == 0xF) continue;
                    const u64 r = next() % 20;
                    const u64 v = r < 6 ? 0 : (r - 5);  // 0 (often), 1..14
                    x |= v << (60 - 4 * c);
                }
                if (fixed_pattern(x) != plan.mask) { bad++; continue; }
                u64 v[4];
                views(x, v);
                for (int k = 0; k < 4; k++) {
                    checked++;
                    if (canon_cand(v[k], plan.cand(k)) != canonical(v[k])) bad++;
                }
            }
        }
        std::printf("%04x %llu %llu", cells, (unsigned long long)checked, (unsigned long long)bad);
        for (int k = 0; k < 4; k++) std::printf(" %d", __builtin_popcount(plan0.cand(k)));
        std::printf("\n");
    }
    return 0;
}
