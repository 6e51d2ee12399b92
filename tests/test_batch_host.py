"""Batch planning on the host (cgb_batch_plan, no GPU): formations are grouped so that no two
formations of a group have fixed-cell masks in the same symmetry orbit; invalid formations are
refused."""
import ctypes as C

from cablegen_b200 import _lib, configs


def _formations(forms):
    keep = []
    arr = (_lib.Formation * len(forms))()
    for i, f in enumerate(forms):
        init = (C.c_uint64 * len(f.initial))(*[int(b) for b in f.initial])
        ws = (C.c_uint64 * max(len(f.winstates), 1))(*[int(x) for x in f.winstates])
        keep += [init, ws]
        arr[i].initial = init
        arr[i].n_initial = len(f.initial)
        arr[i].end_gen = f.end_gen
        arr[i].end_solve = 0
        arr[i].winstates = ws
        arr[i].n_winstates = len(f.winstates)
    return arr, keep


def _orbit(cells):
    return {frozenset(configs._cell_image(k, c) for c in cells) for k in range(8)}


def _greedy(forms):
    groups, out = [], []
    for f in forms:
        o = _orbit(f.fixed_cells)
        for gi, g in enumerate(groups):
            if not (g & o) and len(g) // 8 < 255:
                g |= o
                out.append(gi)
                break
        else:
            groups.append(set(o))
            out.append(len(groups) - 1)
    return out


def test_batch64_groups_match_orbit_rule():
    forms = configs.get("batch64").formations
    arr, keep = _formations(forms)
    g = (C.c_int * len(forms))()
    n = _lib.lib().cgb_batch_plan(arr, len(forms), g)
    want = _greedy(forms)
    assert n == max(want) + 1
    assert list(g) == want
    # within a group, masks never share an orbit
    for gi in range(n):
        seen = set()
        for f, x in zip(forms, g):
            if x == gi:
                o = _orbit(f.fixed_cells)
                assert not (seen & o)
                seen |= o


def test_mirrored_masks_split():
    ll = configs.get("ll_pruned").formations[0]
    base = configs.formation_board((8, 9, 12, 13))
    mirror = configs.Formation("LLm", (8, 9, 12, 13), [base | configs.set_tile(0, 0, 1)], [0], 40)
    arr, keep = _formations([ll, mirror, ll])
    g = (C.c_int * 3)()
    assert _lib.lib().cgb_batch_plan(arr, 3, g) == 3
    assert list(g) == [0, 1, 2]


def test_invalid_formations_refused():
    f = configs.get("ll_pruned").formations[0]
    bad = configs.Formation("mixed", f.fixed_cells, [f.initial[0], f.initial[0] | configs.set_tile(0, 0, 3)],
                            f.winstates, 40)
    arr, keep = _formations([bad])
    assert _lib.lib().cgb_batch_plan(arr, 1, None) == -1
    assert b"one tile sum" in _lib.lib().cgb_last_error()
