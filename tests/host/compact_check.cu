// Host-side check of the 8-byte-slot hash index (cablegen_b200/csrc/hashidx.cuh):
// reads member keys from argv[1] and non-member queries from argv[2], plans the
// table from the members' AND/OR, inserts every member with the build's probe
// rule (tag = remainder | distance + 1), then looks every member and every query
// up with the lookup's rule.  Prints "on r dbits log2cap max_distance
// members_found members_wrong queries_hit".
#include "../../cablegen_b200/csrc/hashidx.cuh"
#include <cstdio>
#include <vector>

static std::vector<uint64_t> load(const char *p)
{
    std::vector<uint64_t> v;
    FILE *f = std::fopen(p, "rb");
    uint64_t x;
    while (f && std::fread(&x, 8, 1, f) == 1) v.push_back(x);
    if (f) std::fclose(f);
    return v;
}

int main(int argc, char **argv)
{
    using namespace cgb;
    if (argc < 3) return 2;
    const std::vector<uint64_t> keys = load(argv[1]), queries = load(argv[2]);
    uint64_t a = ~0ull, o = 0;
    for (uint64_t k : keys) a &= k, o |= k;
    int cbits = 0;
    const CompactHash c = plan_compact(a, o, keys.size(), &cbits);
    if (!c.on) {
        std::printf("0 %d %d %d 0 0 0 0\n", c.r, c.dbits, cbits);
        return 0;
    }
    const uint64_t cap = 1ull << cbits;
    std::vector<uint64_t> slots(cap, 0);
    const uint32_t last = (1u << c.dbits) - 1u;
    uint32_t maxd = 0;
    for (size_t i = 0; i < keys.size(); i++) {
        uint32_t tag0;
        const uint64_t h = compact_home(c, keys[i], &tag0);
        if (h >= cap) return 3;
        uint32_t d = 0;
        for (; d + 1 < last; d++) {
            uint64_t &s = slots[(h + d) & (cap - 1)];
            if (s == 0) {
                s = ((uint64_t)(i + 1) << 32) | (tag0 + d);  // value = member index + 1
                break;
            }
        }
        if (d + 1 >= last) return 4;
        if (d > maxd) maxd = d;
    }
    auto find = [&](uint64_t key) -> uint64_t {
        if ((key & c.cmask) != c.cval) return 0;
        uint32_t tag0;
        const uint64_t h = compact_home(c, key, &tag0);
        for (uint32_t d = 0; d + 1 < last; d++) {
            const uint64_t e = slots[(h + d) & (cap - 1)];
            if ((uint32_t)e == tag0 + d) return e >> 32;
            if ((uint32_t)e == 0) return 0;
        }
        return 0;
    };
    uint64_t found = 0, wrong = 0, qhit = 0;
    for (size_t i = 0; i < keys.size(); i++) {
        const uint64_t v = find(keys[i]);
        if (v == i + 1) found++;
        else wrong++;
    }
    for (uint64_t q : queries) qhit += find(q) != 0;
    std::printf("1 %d %d %d %u %llu %llu %llu\n", c.r, c.dbits, cbits, maxd, (unsigned long long)found,
                (unsigned long long)wrong, (unsigned long long)qhit);
    return 0;
}
