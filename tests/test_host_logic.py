"""Host-side logic without a GPU: the seeded workloads (determinism and the invariants the
batched sweep relies on) and the autotuner's coordinate descent and cache, driven through a
stand-in for the device module."""
import json

import pytest

from cablegen_b200 import autotune, configs


def _fixed(board):
    return {c for c in range(16) if configs.get_tile(board, c) == 0xF}


def test_workloads_are_deterministic():
    for name in ("plain_2x4", "plain_2x4_nearwall", "ll_pruned", "dpdf", "batch64", "ll_large"):
        a, b = configs.get(name), configs.get(name)
        assert [(f.initial, f.winstates, f.end_gen) for f in a.formations] == \
               [(f.initial, f.winstates, f.end_gen) for f in b.formations], name


def test_batch64_formations():
    w = configs.get("batch64")
    assert len(w.formations) == 64 and not w.settings.free_formation
    for f in w.formations:
        free = [c for c in range(16) if c not in f.fixed_cells]
        assert 6 <= len(free) <= 10
        assert 200 <= f.end_gen <= 600 and f.end_gen % 2 == 0
        assert len(f.initial) == 4 and len({configs.tile_sum(b) for b in f.initial}) == 1
        assert all(_fixed(b) == set(f.fixed_cells) for b in f.initial)
        (ws,) = f.winstates
        goal = [c for c in range(16) if configs.get_tile(ws, c)]
        assert len(goal) == 1 and goal[0] in free and 6 <= configs.get_tile(ws, goal[0]) <= 8
        # some symmetry image of the mask keeps a left-aligned run of free cells in every row,
        # so moves toward the fixed cells never move them
        def left_aligned(cells):
            return all(sorted(c % 4 for c in cells if c // 4 == r) == list(range(sum(1 for c in cells if c // 4 == r)))
                       for r in range(4))
        assert any(left_aligned({configs._cell_image(k, c) for c in free}) for k in range(8))


def test_cell_images_form_the_square_group():
    cells = (0, 1, 5, 14)  # no symmetry of its own: eight distinct images
    imgs = {frozenset(configs._cell_image(k, c) for c in cells) for k in range(8)}
    assert len(imgs) == 8
    for k in range(8):
        assert sorted(configs._cell_image(k, c) for c in range(16)) == list(range(16))


class FakeDevice:
    """Knob values and a run time that depends on them (the minimum at sort 2, solve 1, load 25)."""

    def __init__(self):
        self.opts = {"sort_variant": 1, "solve_variant": 0, "hash_load_pct": 0, "move_window": 1}
        self.runs = 0

    def set_option(self, k, v):
        self.opts[k] = v

    def get_option(self, k):
        return self.opts[k]

    def set_rules(self, s):
        pass

    def batch(self, forms, precision=32):
        self.runs += 1
        o = self.opts
        ms = 100 + {3: 8, 4: 9, 5: 11, 1: 10, 0: 5, 2: 0}[o["sort_variant"]] + {0: 7, 1: 0}[o["solve_variant"]] + \
            {0: 3, 25: 0, 45: 6}[o["hash_load_pct"]] + {1: 0, 2: 1, 4: 2}[o["move_window"]]
        return {}, {}, {"total_ms": float(ms)}


def test_autotune_coordinate_descent_and_cache(monkeypatch, tmp_path):
    fake = FakeDevice()
    monkeypatch.setattr(autotune, "device", fake)
    monkeypatch.setattr(autotune, "_gpu_name", lambda: "test-gpu")
    cache = str(tmp_path / "tune.json")
    r = autotune.tune("batch64", end_cap=60, precision=32, repeats=1, cache=cache)
    assert r["params"] == {"sort_variant": 2, "solve_variant": 1, "hash_load_pct": 25, "move_window": 1}
    assert r["ms"] == 100.0 and not r["cached"]
    assert fake.opts == r["params"]          # the winners are applied
    assert len(r["trials"]) == 1 + sum(len(v) - 1 for v in autotune.KNOBS.values())
    with open(cache) as f:
        assert "test-gpu|batch64|60|32" in json.load(f)
    runs = fake.runs
    fake.opts.update(sort_variant=1, solve_variant=0, hash_load_pct=0, move_window=2)
    again = autotune.tune("batch64", end_cap=60, precision=32, repeats=1, cache=cache)
    assert again["cached"] and fake.runs == runs and fake.opts == r["params"]
