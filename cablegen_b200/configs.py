"""Seeded synthetic workloads (formations, initial boards, winstates, settings).

A board is one u64 of 16 nibbles, nibble 0 (the most significant) being the
top-left cell; 0xf marks a fixed formation cell (api/cablegen.h:9-12,
README.md:63-75).  Every initial set shares one tile sum because the reference
CLI refuses mixed sums (frontends/cli/main.c:87-92).

The five workloads restate the benchmark configurations of the generator:

* ``plain_2x4``  -- 2x4 formation, no pruning, end 300 (small, CPU-runnable).
* ``ll_pruned``  -- LL/4422 formation, prune 58/5/6, end 600, 256 goal.
* ``dpdf``       -- DPDF-style formation (6 fixed cells), prune 58/5/6, end 1200.
* ``batch64``    -- 64 seeded formations with 6-10 free cells.
* ``ll_large``   -- LL, free formation, nox=10, prune 64/6/6, end 1400.

All randomness comes from SplitMix64 with a fixed seed, so every run, on every
machine, sees the same boards.
"""
from __future__ import annotations

import dataclasses
from collections import Counter
from typing import List, Tuple

SEED = 20261204
MASK64 = (1 << 64) - 1


class SplitMix64:
    """SplitMix64 (Steele, Lea, Flood 2014) -- the published 64-bit mixer."""

    def __init__(self, seed: int):
        self.state = seed & MASK64

    def next(self) -> int:
        self.state = (self.state + 0x9E3779B97F4A7C15) & MASK64
        z = self.state
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & MASK64
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & MASK64
        return z ^ (z >> 31)

    def below(self, n: int) -> int:
        return self.next() % n

    def uniform(self) -> float:
        return (self.next() >> 11) * (1.0 / (1 << 53))


def set_tile(board: int, cell: int, value: int) -> int:
    shift = 60 - 4 * cell
    return (board & ~(0xF << shift) & MASK64) | ((value & 0xF) << shift)


def get_tile(board: int, cell: int) -> int:
    return (board >> (60 - 4 * cell)) & 0xF


def tile_sum(board: int) -> int:
    """Sum of 2^e over tiles e not in {0, 0xe, 0xf} (src/board.c:340-347)."""
    s = 0
    for c in range(16):
        e = get_tile(board, c)
        if e not in (0, 0xE, 0xF):
            s += 1 << e
    return s


def formation_board(fixed_cells) -> int:
    b = 0
    for c in fixed_cells:
        b = set_tile(b, c, 0xF)
    return b


@dataclasses.dataclass
class Settings:
    """The generator/solver knobs the hot path reads (src/settings.c:34-59)."""
    free_formation: bool = False
    ignore_f: bool = False
    nox: int = 0
    prune: bool = False
    stsl: int = 200
    ltc: int = 5
    smallest_large: int = 6
    score: bool = False


@dataclasses.dataclass
class Formation:
    name: str
    fixed_cells: Tuple[int, ...]
    initial: List[int]
    winstates: List[int]
    end_gen: int
    end_solve: int = 0

    @property
    def start(self) -> int:
        return tile_sum(self.initial[0])


@dataclasses.dataclass
class Workload:
    name: str
    settings: Settings
    formations: List[Formation]
    description: str = ""


def _draw_sets(rng: SplitMix64, free_cells, count: int, draw_tiles) -> List[int]:
    """Draw boards until `count` distinct ones share the modal tile sum.

    `draw_tiles(rng)` returns a list of (cell, exponent) placements.
    """
    def one():
        b = 0
        for cell, e in draw_tiles(rng):
            b = set_tile(b, cell, e)
        return b

    pool = [one() for _ in range(64 * count)]
    modal = Counter(tile_sum(b) for b in pool).most_common(1)[0][0]
    out, seen = [], set()
    draws = 0
    while len(out) < count:
        b = pool[draws] if draws < len(pool) else one()
        draws += 1
        if tile_sum(b) == modal and b not in seen:
            seen.add(b)
            out.append(b)
        assert draws < 1_000_000, "cannot draw enough boards with the modal sum"
    return out


def _distinct_cells(rng: SplitMix64, free_cells, k: int) -> List[int]:
    cells = list(free_cells)
    chosen = []
    for _ in range(k):
        i = rng.below(len(cells))
        chosen.append(cells.pop(i))
    return chosen


def _with_formation(boards: List[int], fixed_cells) -> List[int]:
    f = formation_board(fixed_cells)
    return [b | f for b in boards]


LL_CELLS = (10, 11, 14, 15)
TWOBYFOUR_CELLS = tuple(range(8, 16))
DPDF_CELLS = (2, 3, 6, 7, 10, 11)


def plain_2x4(seed: int = SEED) -> Workload:
    rng = SplitMix64(seed ^ 0x2A4)
    free = [c for c in range(16) if c not in TWOBYFOUR_CELLS]

    def draw(r):
        cells = _distinct_cells(r, free, 2)
        return [(c, 2 if r.uniform() < 0.1 else 1) for c in cells]

    init = _with_formation(_draw_sets(rng, free, 16, draw), TWOBYFOUR_CELLS)
    return Workload(
        "plain_2x4", Settings(),
        [Formation("2x4", TWOBYFOUR_CELLS, init, [set_tile(0, 0, 7)], 300)],
        "2x4 formation, 16 seeded boards with two tiles, 128 goal in the top-left, end 300, no pruning")


def plain_2x4_nearwall(seed: int = SEED) -> Workload:
    w = plain_2x4(seed)
    w.name = "plain_2x4_nearwall"
    w.formations[0].winstates = [set_tile(0, 4, 7)]
    w.description = "as plain_2x4 with the 128 goal at cell 4 (reachable)"
    return w


def ll_pruned(seed: int = SEED, end_gen: int = 600) -> Workload:
    rng = SplitMix64(seed ^ 0x4422)
    free = [c for c in range(16) if c not in LL_CELLS]

    def draw(r):
        cells = _distinct_cells(r, free, 4)
        return [(c, 1 + r.below(3)) for c in cells]

    init = _with_formation(_draw_sets(rng, free, 64, draw), LL_CELLS)
    return Workload(
        "ll_pruned",
        Settings(prune=True, stsl=58, ltc=5, smallest_large=6),
        [Formation("LL", LL_CELLS, init, [set_tile(0, 0, 8)], end_gen)],
        "LL/4422 formation, 64 seeded 4-tile boards, 256 goal in the top-left, "
        f"end {end_gen}, prune stsl=58 ltc=5 smallest_large=6")


def ll_unpruned(seed: int = SEED, end_gen: int = 120) -> Workload:
    w = ll_pruned(seed, end_gen)
    w.name = "ll_unpruned"
    w.settings = Settings()
    w.description = f"LL/4422 formation, seeded 4-tile boards, no pruning, end {end_gen}"
    return w


def dpdf(seed: int = SEED, end_gen: int = 1200) -> Workload:
    rng = SplitMix64(seed ^ 0xD9DF)
    free = [c for c in range(16) if c not in DPDF_CELLS]
    top_row = [c for c in (0, 1, 2, 3) if c not in DPDF_CELLS]

    def draw(r):
        k = 4 + r.below(3)
        exps = sorted((1 + r.below(8) for _ in range(k)), reverse=True)
        cells = list(top_row)
        rest = [c for c in free if c not in cells]
        placed = []
        for i, e in enumerate(exps):
            if i < len(cells):
                placed.append((cells[i], e))
            else:
                j = r.below(len(rest))
                placed.append((rest.pop(j), e))
        return placed

    init = _with_formation(_draw_sets(rng, free, 32, draw), DPDF_CELLS)
    return Workload(
        "dpdf",
        Settings(prune=True, stsl=58, ltc=5, smallest_large=6),
        [Formation("DPDF", DPDF_CELLS, init, [set_tile(0, 0, 9)], end_gen)],
        f"DPDF-style formation (cells 2,3,6,7,10,11 fixed), 32 seeded boards, 512 goal, end {end_gen}, prune 58/5/6")


def _cell_image(sym: int, cell: int) -> int:
    """Cell under one of the 8 board symmetries: sym % 4 clockwise quarter turns, then a
    left-right mirror when sym >= 4."""
    r, c = divmod(cell, 4)
    for _ in range(sym % 4):
        r, c = c, 3 - r
    if sym >= 4:
        c = 3 - c
    return 4 * r + c


def batch64(seed: int = SEED, n_formations: int = 64) -> Workload:
    """Formations whose fixed cells sit at the end of their rows (each row keeps a left-aligned
    run of free cells), turned by a seeded symmetry: then the moves toward the fixed cells are
    always legal (fixed cells never move under free_formation off), so every formation grows real
    layers, while rows of different widths give masks with distinct symmetry orbits."""
    rng = SplitMix64(seed ^ 0xB64)
    forms = []
    for fi in range(n_formations):
        n_free = 6 + rng.below(5)
        while True:
            widths = [rng.below(5) for _ in range(4)]
            if sum(widths) == n_free:
                break
        sym = rng.below(8)
        free = sorted(_cell_image(sym, 4 * r + c) for r in range(4) for c in range(widths[r]))
        fixed = tuple(c for c in range(16) if c not in free)
        goal_exp = 6 + rng.below(3)
        goal_cell = free[rng.below(len(free))]
        end_gen = 200 + 2 * rng.below(201)
        r2 = SplitMix64(rng.next())

        def draw(r, free=free):
            cs = _distinct_cells(r, free, 2)
            return [(c, 2 if r.uniform() < 0.1 else 1) for c in cs]

        init = _with_formation(_draw_sets(r2, free, 4, draw), fixed)
        forms.append(Formation(f"F{fi:02d}", fixed, init, [set_tile(0, goal_cell, goal_exp)], end_gen))
    return Workload("batch64", Settings(), forms,
                    f"{n_formations} seeded formations (6-10 free cells), 4 boards each, end 200-600")


def ll_large(seed: int = SEED, end_gen: int = 1400) -> Workload:
    w = ll_pruned(seed, end_gen)
    w.name = "ll_large"
    w.settings = Settings(free_formation=True, ignore_f=False, nox=10, prune=True,
                          stsl=64, ltc=6, smallest_large=6)
    w.formations[0].winstates = [set_tile(0, 0, 9)]
    w.description = f"LL, free formation, nox=10, prune 64/6/6, end {end_gen}"
    return w


def reference_conf(path: str, wl: Workload, form: Formation, bdir: str, tdir: str, cores: int,
                   end_gen: int = None, end_solve: int = None, initial: str = None, winstates: str = None) -> None:
    """Write the reference's INI configuration for one formation of a workload.

    Keys, sections and value spellings are those the reference reads
    (src/settings.c:34-86): [Cablegen] rules, [Generate] and [Solve] paths and
    ends.  `initial` and `winstates` default to files of those names beside
    `path`.  Used to drive the reference CLI (the CPU baseline, the golden
    fixtures) and the same CLI linked to this library.
    """
    import os
    s = wl.settings
    tf = lambda v: "true" if v else "false"  # noqa: E731
    here = os.path.dirname(path)
    initial = initial if initial is not None else os.path.join(here, "initial")
    winstates = winstates if winstates is not None else os.path.join(here, "winstates")
    with open(path, "w") as f:
        f.write(f"""[Cablegen]
free_formation = {tf(s.free_formation)}
ignore_f = {tf(s.ignore_f)}
cores = {cores}
nox = {s.nox}
use_gpu = false

[Generate]
dir = {bdir}
initial = {initial}
end = {end_gen if end_gen is not None else form.end_gen}
stsl = {s.stsl}
ltc = {s.ltc}
smallest_large = {s.smallest_large}
prune = {tf(s.prune)}

[Solve]
dir = {tdir}
winstates = {winstates}
end = {end_solve if end_solve is not None else form.end_solve}
score = {tf(s.score)}
delete_boards = false
""")


def free_2x4_nox(seed: int = SEED, end_gen: int = 300) -> Workload:
    """Config 5's rules (free formation: the 0xf cells move like tiles; nox: a board holding
    the nox tile wins) on the small 2x4 formation, where a 64 tile (nox 6) is reachable, so
    the nox path yields nonzero probabilities."""
    w = plain_2x4(seed)
    w.name = "free_2x4_nox"
    w.settings = Settings(free_formation=True, ignore_f=False, nox=6)
    w.formations[0].end_gen = end_gen
    w.description = f"2x4 formation, free formation, nox 6 (a 64 tile wins), end {end_gen}"
    return w


WORKLOADS = {
    "plain_2x4": plain_2x4,
    "plain_2x4_nearwall": plain_2x4_nearwall,
    "ll_pruned": ll_pruned,
    "ll_unpruned": ll_unpruned,
    "dpdf": dpdf,
    "batch64": batch64,
    "ll_large": ll_large,
    "free_2x4_nox": free_2x4_nox,
}


def get(name: str, **kw) -> Workload:
    return WORKLOADS[name](**kw)
