// Host-side check of the lookup index's home slots (cablegen_b200/csrc/hashidx.cuh):
// reads keys (u64, raw) from argv[1] and capacities from argv[2..]; for each
// capacity prints "cap max_slot distinct_slots out_of_range".
#include "../../cablegen_b200/csrc/hashidx.cuh"
#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <vector>

int main(int argc, char **argv)
{
    if (argc < 3) return 2;
    FILE *f = std::fopen(argv[1], "rb");
    if (!f) return 2;
    std::vector<uint64_t> k;
    uint64_t x;
    while (std::fread(&x, 8, 1, f) == 1) k.push_back(x);
    std::fclose(f);
    for (int a = 2; a < argc; a++) {
        const uint64_t cap = std::strtoull(argv[a], nullptr, 10);
        std::vector<uint64_t> s(k.size());
        uint64_t bad = 0;
        for (size_t i = 0; i < k.size(); i++) {
            s[i] = cgb::home_slot(k[i], cap);
            bad += s[i] >= cap;
        }
        std::sort(s.begin(), s.end());
        const uint64_t distinct = (uint64_t)(std::unique(s.begin(), s.end()) - s.begin());
        std::printf("%llu %llu %llu %llu\n", (unsigned long long)cap, (unsigned long long)(s.empty() ? 0 : s[distinct - 1]),
                    (unsigned long long)distinct, (unsigned long long)bad);
    }
    return 0;
}
