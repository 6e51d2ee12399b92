// Host-side check of the board algebra in cablegen_b200/csrc/board.cuh: reads
// boards (u64, raw) from argv[1] and prune parameter sets "stsl,ltc,sl" from
// argv[2..], writes one byte per (parameter set, board) to stdout: bit 0 the
// verdict of prune_board, bit 1 that of prune_by_table (the table-driven form).
#include "../../cablegen_b200/csrc/board.cuh"
#include <cstdio>
#include <cstdlib>
#include <vector>

int main(int argc, char **argv)
{
    if (argc < 3) return 2;
    FILE *f = std::fopen(argv[1], "rb");
    if (!f) return 2;
    std::vector<cgb::u64> b;
    cgb::u64 x;
    while (std::fread(&x, 8, 1, f) == 1) b.push_back(x);
    std::fclose(f);
    for (int a = 2; a < argc; a++) {
        long long stsl, ltc, sl;
        if (std::sscanf(argv[a], "%lld,%lld,%lld", &stsl, &ltc, &sl) != 3) return 2;
        cgb::PruneParams p{stsl, ltc, sl, 1};
        static cgb::PruneTable t;
        cgb::build_prune_table(p, &t);
        std::vector<unsigned char> out(b.size());
        for (size_t i = 0; i < b.size(); i++)
            out[i] = (cgb::prune_board(b[i], p) ? 1 : 0) | (cgb::prune_by_table(b[i], t) ? 2 : 0);
        std::fwrite(out.data(), 1, out.size(), stdout);
    }
    return 0;
}
