"""Whole sweeps on the GPU against the reference's own layer and table digests."""
import numpy as np
import pytest

import py_oracle as O
from cablegen_b200 import configs
from helpers import digests, sha_layer, sha_table

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", ["plain_2x4", "plain_2x4_nearwall"])
def test_generate_matches_reference(cuda, name):
    w = configs.get(name)
    f = w.formations[0]
    cuda.set_rules(w.settings)
    layers, st = cuda.generate(f.initial, f.start, f.end_gen)
    d = digests(name)["layers"]
    assert sorted(int(s) for s in d) == sorted(layers)
    for s, rec in d.items():
        assert len(layers[int(s)]) == rec["boards"], s
        assert sha_layer(layers[int(s)]) == rec["boards_sha256"], s
    assert st["boards_generated"] == sum(r["boards"] for r in d.values())


INDEX_KINDS = [0, 1, 2]  # bisection, top-bits buckets, hash


@pytest.fixture
def index_kind(cuda, request):
    old = cuda.get_option("index")
    cuda.set_option("index", request.param)
    yield request.param
    cuda.set_option("index", old)


@pytest.mark.parametrize("index_kind", INDEX_KINDS, indirect=True)
@pytest.mark.parametrize("name", ["plain_2x4", "plain_2x4_nearwall"])
def test_tablebase_fp64_bit_exact(cuda, name, index_kind):
    w = configs.get(name)
    f = w.formations[0]
    cuda.set_rules(w.settings)
    layers, tables, st = cuda.tablebase(f.initial, f.start, f.end_gen, 0, f.winstates, precision=64,
                                        keep_layers=True, keep_tables=True)
    d = digests(name)["layers"]
    for s, rec in d.items():
        k, v = tables[int(s)]
        assert sha_table(k, v) == rec["tables_sha256"], s
    # layers below the initial sum are solved as empty tables (solve.c:203-211)
    assert all(len(tables[s][0]) == 0 for s in tables if s < f.start)


@pytest.mark.parametrize("index_kind", INDEX_KINDS, indirect=True)
def test_tablebase_fp32_error(cuda, index_kind):
    """FP32 tables with Kahan sums stay within 1e-6 of FP64 (max-abs, every layer)."""
    w = configs.get("plain_2x4_nearwall")
    f = w.formations[0]
    cuda.set_rules(w.settings)
    _, t64, _ = cuda.tablebase(f.initial, f.start, f.end_gen, 0, f.winstates, precision=64, keep_tables=True)
    _, t32, _ = cuda.tablebase(f.initial, f.start, f.end_gen, 0, f.winstates, precision=32, keep_tables=True)
    err = max((np.abs(t64[s][1] - t32[s][1].astype(np.float64)).max() if len(t64[s][1]) else 0.0) for s in t64)
    assert err <= 1e-6, err
    # the side-by-side mode reports the same per-layer errors and still emits FP64 tables
    _, tb, st = cuda.tablebase(f.initial, f.start, f.end_gen, 0, f.winstates, precision=0, keep_tables=True)
    errs = st["layer_errors"]
    for s, (n, mx, mean) in errs.items():
        want = np.abs(t64[s][1] - t32[s][1].astype(np.float64))
        assert n == len(want) and mx == pytest.approx(want.max(), abs=0) and mean <= mx + 1e-18
        assert np.array_equal(tb[s][1], t64[s][1])
    assert st["max_abs_err"] == pytest.approx(err, abs=0)


@pytest.mark.parametrize("top", [0, 6])
def test_tablebase_fp32_fp64_window(cuda, top):
    """An FP32 sweep solves its `fp64_top_layers` highest layers in FP64 (bit-equal to the FP64
    sweep's tables there) and narrows them for the FP32 layers below, which stay within 1e-6."""
    w = configs.get("plain_2x4_nearwall")
    f = w.formations[0]
    cuda.set_rules(w.settings)
    old = cuda.get_option("fp64_top_layers")
    try:
        cuda.set_option("fp64_top_layers", top)
        _, t64, _ = cuda.tablebase(f.initial, f.start, f.end_gen, 0, f.winstates, precision=64, keep_tables=True)
        _, t32, _ = cuda.tablebase(f.initial, f.start, f.end_gen, 0, f.winstates, precision=32, keep_tables=True)
    finally:
        cuda.set_option("fp64_top_layers", old)
    window = [s for s in t32 if s > f.end_gen - 2 * top]
    assert len(window) == top
    for s in t32:
        if s in window:
            assert t32[s][1].dtype == np.float64 and np.array_equal(t32[s][1], t64[s][1]), s
        else:
            assert t32[s][1].dtype == np.float32, s
            if len(t32[s][1]):
                assert np.abs(t64[s][1] - t32[s][1].astype(np.float64)).max() <= 1e-6, s


@pytest.mark.parametrize("precision", [64, 32])
@pytest.mark.parametrize("name,end", [("plain_2x4_nearwall", None), ("ll_pruned", 200)])
def test_solve_variants_agree(cuda, precision, name, end):
    """Both solve kernels (one thread per board; board-cell pairs spread over a warp) give
    bit-identical tables: the same operations in the same order.  The full 2x4 workload's FP64
    tables also hash to the reference's files."""
    w = configs.get(name) if end is None else configs.get(name, end_gen=end)
    f = w.formations[0]
    cuda.set_rules(w.settings)
    old = cuda.get_option("solve_variant")
    got = {}
    try:
        for v in (0, 1):
            cuda.set_option("solve_variant", v)
            _, got[v], _ = cuda.tablebase(f.initial, f.start, f.end_gen, 0, f.winstates, precision=precision,
                                          keep_tables=True)
    finally:
        cuda.set_option("solve_variant", old)
    for v in (0,):
        for s in got[1]:
            assert np.array_equal(got[v][s][1], got[1][s][1]), (v, s)
    if precision == 64 and end is None:
        want = digests(name)["layers"]
        for s, rec in want.items():
            k, vals = got[1][int(s)]
            assert sha_table(k, vals) == rec["tables_sha256"], s


def test_region_built_index_matches_atomic_build(cuda):
    """The 16-byte-slot index built region by region in shared memory (layers of 2^16..2^28
    keys) answers exactly like the one built by atomic inserts: FP64 tables bit-equal."""
    w = configs.get("ll_pruned", end_gen=220)
    f = w.formations[0]
    cuda.set_rules(w.settings)
    old = cuda.get_option("region_build")
    got = {}
    try:
        for v in (0, 1):
            cuda.set_option("region_build", v)
            _, got[v], _ = cuda.tablebase(f.initial, f.start, f.end_gen, f.start, f.winstates, precision=64,
                                          keep_tables=True)
    finally:
        cuda.set_option("region_build", old)
    assert max(len(k) for k, _ in got[1].values()) >= (1 << 16)
    for s in got[0]:
        assert np.array_equal(got[0][s][1], got[1][s][1]), s


def test_move_windows_agree(cuda):
    """Every chunk size of the move expansion's repeat set (1..4 blocks of 1024 boards) gives
    the same layers: the set only decides how many repeats reach the sort."""
    w = configs.get("ll_pruned", end_gen=220)
    f = w.formations[0]
    cuda.set_rules(w.settings)
    old = cuda.get_option("move_window")
    got, kept = {}, {}
    try:
        for v in (1, 2, 4):
            cuda.set_option("move_window", v)
            before = cuda.kernel_stats()["moves_kept"]
            got[v], _ = cuda.generate(f.initial, f.start, f.end_gen)
            kept[v] = cuda.kernel_stats()["moves_kept"] - before
    finally:
        cuda.set_option("move_window", old)
    for v in (2, 4):
        assert got[v].keys() == got[1].keys()
        for s in got[1]:
            assert np.array_equal(got[v][s], got[1][s]), (v, s)
    assert kept[4] < kept[1]


def test_fp32_compact_index_matches_wide(cuda):
    """FP32 tables looked up through 8-byte slots equal those through 16-byte slots, bit for
    bit (both indexes are exact), and the large layers of LL do take the 8-byte form."""
    w = configs.get("ll_pruned", end_gen=230)
    f = w.formations[0]
    cuda.set_rules(w.settings)
    old = cuda.get_option("hash_compact")
    try:
        cuda.set_option("hash_compact", 0)
        _, wide, _ = cuda.tablebase(f.initial, f.start, f.end_gen, f.start, f.winstates, precision=32,
                                    keep_tables=True)
        cuda.set_option("hash_compact", 1)
        cuda.reset_kernel_stats()
        _, comp, _ = cuda.tablebase(f.initial, f.start, f.end_gen, f.start, f.winstates, precision=32,
                                    keep_tables=True)
        k = cuda.kernel_stats()
    finally:
        cuda.set_option("hash_compact", old)
    assert k["compact_index_builds"] > 0, k
    for s in wide:
        assert np.array_equal(wide[s][1], comp[s][1]), s


@pytest.mark.parametrize("host_layers_mb", [65536, 0])
def test_tablebase_async_copies_match(cuda, host_layers_mb):
    """Layers and tables copied out asynchronously equal the engine's own (LL, pruned, 40 layers),
    with the layers' host copies kept for the tables (default) and without (keys copied again)."""
    old = cuda.get_option("host_layers_mb")
    cuda.set_option("host_layers_mb", host_layers_mb)
    try:
        _async_copies_case(cuda, host_layers_mb)
    finally:
        cuda.set_option("host_layers_mb", old)


def _async_copies_case(cuda, host_layers_mb):
    w = configs.get("ll_pruned", end_gen=96)
    f = w.formations[0]
    cuda.set_rules(w.settings)
    lut = O.make_lut(0, 0)
    ost = O.settings(w.settings)
    want = O.generate(lut, ost, f.initial, f.start, 96)
    layers, tables, st = cuda.tablebase(f.initial, f.start, 96, f.start, f.winstates, precision=64,
                                        keep_layers=True, keep_tables=True)
    for s in want:
        assert np.array_equal(layers[s], want[s]), s
        assert np.array_equal(tables[s][0], want[s]), s
    vals = O.solve(lut, ost, want, f.winstates, 96, f.start)
    for s in want:
        assert np.array_equal(tables[s][1], vals[s]), s
    # with layers and tables both wanted, a layer's keys cross once (kept on the host for its
    # table), so the tables carry their f64 values only; without the host copies, keys again
    table_bytes = 8 if host_layers_mb else 16
    assert st["d2h_bytes"] == sum(table_bytes * len(v) for v in want.values()) + sum(8 * len(v) for v in want.values())


@pytest.mark.parametrize("index_kind", INDEX_KINDS, indirect=True)
def test_solve_layer_matches_oracle(cuda, index_kind):
    """One layer through cgb_solve_layer against the oracle, with nox and score variants."""
    w = configs.get("plain_2x4_nearwall")
    f = w.formations[0]
    lut = O.make_lut(0, 0)
    layers = O.generate(lut, O.settings(w.settings), f.initial, f.start, 60)
    for nox, score in ((0, 0), (5, 0), (0, 1)):
        st = configs.Settings(nox=nox, score=bool(score))
        cuda.set_rules(st)
        ost = O.settings(st)
        ws = O.expand_winstates(f.winstates)
        t4 = (layers[60], O.solve_layer(lut, ost, layers[60], (np.zeros(0, np.uint64),) * 2, (np.zeros(0, np.uint64),) * 2, ws))
        t2 = (layers[58], O.solve_layer(lut, ost, layers[58], t4, (np.zeros(0, np.uint64),) * 2, ws))
        want = O.solve_layer(lut, ost, layers[56], t2, t4, ws)
        got = cuda.solve_layer(cuda.to_device(layers[56]), (cuda.to_device(t2[0]), _f(cuda, t2[1])),
                               (cuda.to_device(t4[0]), _f(cuda, t4[1])), f.winstates, 64)
        assert np.array_equal(got.cpu().numpy(), want), (nox, score)


def _f(cuda, v):
    import torch
    return torch.from_numpy(np.ascontiguousarray(v, dtype=np.float64)).cuda()


def _hashing_sweep(cuda, w, end):
    f = w.formations[0]
    got_layers, got_tables = {}, {}

    def on_layer(s, ptr, n):
        got_layers[s] = sha_layer(np.ctypeslib.as_array(ptr, shape=(n,)) if n else np.zeros(0, np.uint64))

    def on_table(s, kptr, vptr, n, prec):
        import ctypes as C
        k = np.ctypeslib.as_array(kptr, shape=(n,)) if n else np.zeros(0, np.uint64)
        v = (np.ctypeslib.as_array(C.cast(vptr, C.POINTER(C.c_double)), shape=(n,)) if n
             else np.zeros(0, np.float64))
        got_tables[s] = sha_table(k, v)

    _, _, st = cuda.tablebase(f.initial, f.start, end, f.start, f.winstates, precision=64,
                              layer_fn=on_layer, table_fn=on_table)
    return got_layers, got_tables, st


def test_sliced_steps_and_spilled_layers_bit_exact(cuda):
    """Sliced layer steps (sorted unique runs merged) and layers spilled to host memory and
    brought back for the solve give the reference's layers and the unsliced run's tables."""
    w = configs.get("ll_pruned")
    cuda.set_rules(w.settings)
    end = 140
    base_layers, base_tables, _ = _hashing_sweep(cuda, w, end)
    names = ("max_sort_keys", "store_chunk_mb", "spill_reserve_mb")
    old = {k: cuda.get_option(k) for k in names}
    try:
        cuda.set_option("max_sort_keys", 1 << 18)
        cuda.set_option("store_chunk_mb", 8)
        cuda.set_option("spill_reserve_mb", 1 << 30)
        layers, tables, st = _hashing_sweep(cuda, w, end)
    finally:
        for k, v in old.items():
            cuda.set_option(k, v)
    want = digests("ll_pruned")["layers"]
    for s in range(16, end + 1, 2):
        assert layers[s] == want[str(s)]["boards_sha256"], s
    assert layers == base_layers
    assert tables == base_tables
    assert st["layer_slices"] > 0
    assert st["spilled_chunks"] > 0 and st["restored_chunks"] > 0
