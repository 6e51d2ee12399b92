"""The CPU oracle is pinned to vectors the reference build produced (CPU only)."""
import ctypes as C

import numpy as np
import pytest

import py_oracle as O
from cablegen_b200 import configs
from helpers import digests, sha_layer, sha_table, unit

BOARDS = unit("boards.u64", np.uint64)


def test_canonical_matches_reference():
    assert np.array_equal(O.canon(BOARDS), unit("canon.u64", np.uint64))


def test_canonical_is_orbit_invariant():
    """test.c:219-234: every image of a board has the same canonical form."""
    L = O.lib()
    for b in BOARDS[:512]:
        imgs = O.expand_winstates([b])
        assert len({L.orc_canon(int(x)) for x in imgs}) == 1
        assert {L.orc_get_sum(int(x)) for x in imgs} == {L.orc_get_sum(int(b))}


def test_signed_variant_differs():
    """The AVX-512 build's signed maximum (board.c:271-313) is a different orbit representative."""
    L = O.lib()
    diff = sum(L.orc_canon(int(b)) != L.orc_canon_signed(int(b)) for b in BOARDS)
    assert diff > 0


@pytest.mark.parametrize("ff,ig", [(0, 0), (0, 1), (1, 0), (1, 1)])
def test_moves_match_reference(ff, ig):
    lut = O.make_lut(ff, ig)
    L = O.lib()
    tag = f"ff{ff}_ig{ig}"
    mv = unit(f"move_unstable_{tag}.u64", np.uint64).reshape(-1, 4)
    ok = unit(f"move_unstable_ok_{tag}.u8", np.uint8).reshape(-1, 4)
    mvs = unit(f"move_stable_{tag}.u64", np.uint64).reshape(-1, 4)
    oks = unit(f"move_stable_ok_{tag}.u8", np.uint8).reshape(-1, 4)
    for i, b in enumerate(BOARDS):
        for d in range(4):
            x = C.c_uint64(int(b))
            r = L.orc_movedir_unstable(C.byref(lut), C.byref(x), d)
            assert bool(r) == bool(ok[i, d])
            if r:
                assert x.value == mv[i, d]
            y = C.c_uint64(int(b))
            r = L.orc_movedir(C.byref(lut), C.byref(y), d)
            assert bool(r) == bool(oks[i, d]) and y.value == mvs[i, d]


def test_prune_matches_reference():
    import json, os
    from helpers import UNITS
    params = json.load(open(os.path.join(UNITS, "meta.json")))["prune_params"]
    pr = unit("prune.u8", np.uint8).reshape(len(params), -1)
    L = O.lib()
    for j, (stsl, ltc, sl) in enumerate(params):
        got = np.array([L.orc_prune(int(b), stsl, ltc, sl) for b in BOARDS], dtype=np.uint8)
        assert np.array_equal(got != 0, pr[j] != 0), (stsl, ltc, sl)


def test_cmpbrd_and_sum_match_reference():
    pats = unit("cmpbrd_patterns.u64", np.uint64)
    cm = unit("cmpbrd.u8", np.uint8).reshape(len(pats), -1)
    L = O.lib()
    for j, w in enumerate(pats):
        for i in range(cm.shape[1]):
            assert bool(L.orc_cmpbrd(int(BOARDS[i]), int(w))) == bool(cm[j, i])
    sums = unit("get_sum.i32", np.int32)
    assert all(L.orc_get_sum(int(b)) == s for b, s in zip(BOARDS, sums))


def test_lookup_matches_reference():
    keys = unit("lookup_keys.u64", np.uint64)
    vals = unit("lookup_vals.f64", np.float64)
    qs = unit("lookup_queries.u64", np.uint64)
    L = O.lib()
    kp = keys.ctypes.data_as(O.pu64)
    vp = vals.ctypes.data_as(O.pdbl)
    for canon, name in ((1, "lookup_canon.f64"), (0, "lookup_nocanon.f64")):
        want = unit(name, np.float64)
        got = np.array([L.orc_lookup(int(q), kp, vp, len(keys), canon) for q in qs])
        assert np.array_equal(got, want)


def test_lookup_kat():
    """test.c:22-52: keys 0..99 hold 99-i."""
    keys = np.arange(100, dtype=np.uint64)
    vals = (99 - np.arange(100)).astype(np.float64)
    L = O.lib()
    for i in range(100):
        assert L.orc_lookup(i, keys.ctypes.data_as(O.pu64), vals.ctypes.data_as(O.pdbl), 100, 0) == 99 - i
    assert L.orc_lookup(5, keys.ctypes.data_as(O.pu64), vals.ctypes.data_as(O.pdbl), 0, 0) == 0.0


def test_dedupe_kat():
    """test.c:147-167: dedupe of {2,5,6,5,4,5}; merge of three runs."""
    a = np.array([2, 5, 6, 5, 4, 5], dtype=np.uint64)
    n = O.lib().orc_sort_unique(a.ctypes.data_as(O.pu64), len(a))
    assert list(a[:n]) == [2, 4, 5, 6]
    m = O.merge_unique(O.merge_unique(a[:n], np.array([1, 5, 9], np.uint64)), np.array([0], np.uint64))
    assert list(m) == [0, 1, 2, 4, 5, 6, 9]


@pytest.mark.parametrize("name", ["plain_2x4", "plain_2x4_nearwall"])
def test_oracle_reproduces_reference_tablebase(name):
    w = configs.get(name)
    f = w.formations[0]
    lut = O.make_lut(w.settings.free_formation, w.settings.ignore_f)
    st = O.settings(w.settings)
    layers = O.generate(lut, st, f.initial, f.start, f.end_gen)
    d = digests(name)["layers"]
    for s, rec in d.items():
        assert sha_layer(layers[int(s)]) == rec["boards_sha256"], s
    vals = O.solve(lut, st, layers, f.winstates, f.end_gen, 0)
    for s, rec in d.items():
        assert sha_table(layers[int(s)], vals[int(s)]) == rec["tables_sha256"], s
