"""Stand-alone kernel cases for profiling (small enough for ncu --set full).

    python -m cablegen_b200.kernel_cases sort            # ~88M LL-like canonical keys, sort + unique
    python -m cablegen_b200.kernel_cases expand          # 30M LL-like boards, moves (prune 58/5/6) + spawns
    python -m cablegen_b200.kernel_cases solve 260       # LL pruned sweep to tile sum 260, FP64 solve

Boards are seeded random LL/4422 boards (cells 10,11,14,15 fixed), tiles up
to 512; the solve case is the real LL pruned workload truncated at the given
end sum.  Prints the engine's kernel statistics.
"""
import sys

import numpy as np
import torch

from . import configs, device

LL_CELLS = (10, 11, 14, 15)


def random_boards(rng, n, cells=LL_CELLS, max_exp=9, p_empty=0.35):
    free = np.array([c for c in range(16) if c not in cells])
    out = np.zeros(n, dtype=np.uint64)
    for c in cells:
        out |= np.uint64(0xF) << np.uint64(60 - 4 * c)
    exps = rng.integers(1, max_exp + 1, size=(n, len(free))).astype(np.uint64)
    exps[rng.random((n, len(free))) < p_empty] = 0
    for j, c in enumerate(free):
        out |= exps[:, j] << np.uint64(60 - 4 * int(c))
    return out


def main(argv):
    mode = argv[0]
    device.init(0)
    w = configs.get("ll_pruned")
    device.set_rules(w.settings)
    rng = np.random.default_rng(5)
    if mode == "sort":
        c = device.canonicalize(device.to_device(random_boards(rng, 25_000_000)))
        x = torch.cat([c, c.flip(0), c[1::2], c[::2], c[::3], c[::5]])
        s, p = device.sort(x)
        u = device.unique(s)
        print("keys", x.numel(), "passes", p, "unique", u.numel())
    elif mode == "expand":
        b = device.to_device(random_boards(rng, 30_000_000))
        o = device.expand_moves(b)
        o2, _ = device.expand_spawns(b)
        print("moves", o.numel(), "spawns", o2.numel())
    elif mode == "solve":
        f = w.formations[0]
        end = int(argv[1]) if len(argv) > 1 else 260
        _, _, st = device.tablebase(f.initial, f.start, end, f.start, f.winstates, 64)
        print(st)
    else:
        raise SystemExit(f"unknown case {mode}")
    print(device.kernel_stats())


if __name__ == "__main__":
    main(sys.argv[1:])
