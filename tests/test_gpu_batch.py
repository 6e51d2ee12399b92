"""Batched sweeps (cgb_batch_run): many formations advanced together must give, formation by
formation, the layers and FP64 tables of the oracle (the reference's algorithm); FP32 tables stay
within 1e-6; CUDA-graph capture changes nothing; formations whose fixed-cell masks are images of
one another run in separate groups."""
import dataclasses

import numpy as np
import pytest

import py_oracle as O
from cablegen_b200 import configs

pytestmark = pytest.mark.gpu


def _small_batch(n, end_cap):
    w = configs.get("batch64")
    forms = []
    for f in w.formations[:n]:
        forms.append(dataclasses.replace(f, end_gen=min(f.end_gen, end_cap)))
    return w, forms


def _expected_groups(forms):
    """Greedy grouping by disjoint fixed-cell mask orbits (the batch's own rule)."""
    groups = []
    for f in forms:
        orbit = {frozenset(configs._cell_image(k, c) for c in f.fixed_cells) for k in range(8)}
        for g in groups:
            if not (g & orbit):
                g |= orbit
                break
        else:
            groups.append(set(orbit))
    return len(groups)


def _oracle(w, forms):
    lut = O.make_lut(0, 0)
    ost = O.settings(w.settings)
    want_layers, want_vals = [], []
    for f in forms:
        layers = O.generate(lut, ost, f.initial, f.start, f.end_gen)
        want_layers.append(layers)
        want_vals.append(O.solve(lut, ost, layers, f.winstates, f.end_gen, f.end_solve))
    return want_layers, want_vals


@pytest.fixture(scope="module")
def batch_case():
    w, forms = _small_batch(12, 70)
    return w, forms, _oracle(w, forms)


@pytest.mark.parametrize("graphs", [True, False])
def test_batch_fp64_matches_oracle(cuda, batch_case, graphs):
    w, forms, (want_layers, want_vals) = batch_case
    cuda.set_rules(w.settings)
    layers, tables, st = cuda.batch(forms, precision=64, use_graphs=graphs, keep_layers=True, keep_tables=True)
    for i, f in enumerate(forms):
        for s, want in want_layers[i].items():
            assert np.array_equal(layers[(i, s)], want), (i, s)
        for s, vals in want_vals[i].items():
            k, v = tables[(i, s)]
            assert np.array_equal(k, want_layers[i].get(s, np.zeros(0, np.uint64))), (i, s)
            assert np.array_equal(v, vals), (i, s)
    assert st["groups"] == _expected_groups(forms)
    assert st["boards_generated"] == sum(len(x) for L in want_layers for x in L.values())
    if graphs:
        assert st["graph_launches"] == st["solve_steps"] > 0
    else:
        assert st["graph_launches"] == 0


def test_batch_fp32_error(cuda, batch_case):
    w, forms, (want_layers, want_vals) = batch_case
    cuda.set_rules(w.settings)
    _, tables, _ = cuda.batch(forms, precision=32, keep_tables=True)
    err = 0.0
    for i in range(len(forms)):
        for s, vals in want_vals[i].items():
            k, v = tables[(i, s)]
            assert v.dtype == np.float32
            if len(vals):
                err = max(err, float(np.abs(v.astype(np.float64) - vals).max()))
    assert err <= 1e-6, err


def test_batch_symmetric_masks_split_into_groups(cuda):
    """LL and its mirror image share board space: they must run as two groups."""
    lut = O.make_lut(0, 0)
    st = configs.Settings()
    ost = O.settings(st)
    ll = configs.get("ll_pruned").formations[0]
    mirror_cells = (8, 9, 12, 13)   # LL (10, 11, 14, 15) mirrored left-right
    base = configs.formation_board(mirror_cells)
    init = [base | configs.set_tile(configs.set_tile(0, 0, 1), 5, 1), base | configs.set_tile(configs.set_tile(0, 2, 1), 7, 1)]
    forms = [dataclasses.replace(ll, end_gen=60, initial=ll.initial[:8]),
             configs.Formation("LLm", mirror_cells, init, [configs.set_tile(0, 3, 6)], 50)]
    cuda.set_rules(st)
    layers, tables, stats = cuda.batch(forms, precision=64, keep_layers=True, keep_tables=True)
    assert stats["groups"] == 2
    for i, f in enumerate(forms):
        want = O.generate(lut, ost, f.initial, f.start, f.end_gen)
        vals = O.solve(lut, ost, want, f.winstates, f.end_gen, f.end_solve)
        for s in want:
            assert np.array_equal(layers[(i, s)], want[s]), (i, s)
        for s in vals:
            assert np.array_equal(tables[(i, s)][1], vals[s]), (i, s)


def test_batch_knobs_do_not_change_results(cuda, batch_case):
    """Every tuned knob value gives the same FP64 tables (the autotuner picks speed only)."""
    w, forms, (want_layers, want_vals) = batch_case
    cuda.set_rules(w.settings)
    names = ("sort_variant", "solve_variant", "hash_load_pct", "move_window")
    old = {k: cuda.get_option(k) for k in names}
    try:
        for sv, so, hl, mw in ((2, 1, 60, 4), (0, 0, 25, 1), (3, 1, 45, 2), (4, 0, 0, 1), (5, 1, 0, 4)):
            cuda.set_option("sort_variant", sv)
            cuda.set_option("solve_variant", so)
            cuda.set_option("hash_load_pct", hl)
            cuda.set_option("move_window", mw)
            _, tables, _ = cuda.batch(forms, precision=64, keep_tables=True)
            for i in range(len(forms)):
                for s, vals in want_vals[i].items():
                    assert np.array_equal(tables[(i, s)][1], vals), (sv, so, hl, mw, i, s)
    finally:
        for k, v in old.items():
            cuda.set_option(k, v)


def test_autotune_applies_and_caches(cuda, tmp_path):
    from cablegen_b200 import autotune
    names = tuple(autotune.KNOBS)
    old = {k: cuda.get_option(k) for k in names}
    try:
        cache = str(tmp_path / "tune.json")
        r = autotune.tune("batch64", end_cap=60, precision=32, repeats=1, cache=cache)
        assert not r["cached"] and len(r["trials"]) == 1 + sum(len(v) - 1 for v in autotune.KNOBS.values())
        for k, v in r["params"].items():
            assert v in autotune.KNOBS[k] and cuda.get_option(k) == v
        again = autotune.tune("batch64", end_cap=60, precision=32, repeats=1, cache=cache)
        assert again["cached"] and again["params"] == r["params"]
    finally:
        for k, v in old.items():
            cuda.set_option(k, v)
