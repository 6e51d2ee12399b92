"""Parity of the CUDA kernels with the oracle and the reference's vectors."""
import numpy as np
import pytest

import py_oracle as O
from cablegen_b200 import configs
from helpers import realistic_boards, unit

pytestmark = pytest.mark.gpu

BOARDS = unit("boards.u64", np.uint64)


def test_canonicalize(cuda):
    got = cuda.to_numpy(cuda.canonicalize(cuda.to_device(BOARDS)))
    assert np.array_equal(got, unit("canon.u64", np.uint64))


@pytest.mark.parametrize("ff,ig", [(0, 0), (0, 1), (1, 0), (1, 1)])
@pytest.mark.parametrize("prune", [(0, 200, 5, 6), (1, 58, 5, 6), (1, 64, 6, 6), (1, 0, 0, 0)])
def test_expand_moves(cuda, ff, ig, prune):
    rng = np.random.default_rng(7 + ff * 2 + ig)
    boards = np.concatenate([BOARDS, realistic_boards(rng, 20000), realistic_boards(rng, 5000, (8, 9, 10, 11, 12, 13, 14, 15))])
    st = configs.Settings(free_formation=bool(ff), ignore_f=bool(ig), prune=bool(prune[0]), stsl=prune[1],
                          ltc=prune[2], smallest_large=prune[3])
    cuda.set_rules(st)
    got = np.unique(cuda.to_numpy(cuda.expand_moves(cuda.to_device(boards))))
    want = O.move_layer(O.make_lut(ff, ig), O.settings(st), boards)
    assert np.array_equal(got, want)


def test_expand_spawns(cuda):
    rng = np.random.default_rng(3)
    boards = np.concatenate([BOARDS, realistic_boards(rng, 30000, p_empty=0.6)])
    o2, o4 = cuda.expand_spawns(cuda.to_device(boards))
    w2, w4 = O.spawn_layer(boards)
    assert np.array_equal(np.unique(cuda.to_numpy(o2)), w2)
    assert np.array_equal(np.unique(cuda.to_numpy(o4)), w4)
    assert cuda.count_spawns(cuda.to_device(boards)) == o2.numel()


SIZES = [0, 1, 2, 31, 4095, 4096, 4097, 8193, 100_000, 1_000_003, 5_000_001]


@pytest.fixture(params=[0, 1, 2, 3, 4, 5], ids=["match", "ballot", "pipelined", "byte", "byte8k", "byte8k_match"])
def sort_variant(cuda, request):
    old = cuda.get_option("sort_variant")
    cuda.set_option("sort_variant", request.param)
    yield request.param
    cuda.set_option("sort_variant", old)


@pytest.mark.parametrize("n", SIZES)
def test_sort_unique_random(cuda, n, sort_variant):
    rng = np.random.default_rng(n)
    x = rng.integers(0, 1 << 63, size=n, dtype=np.uint64) | (rng.integers(0, 2, size=n, dtype=np.uint64) << np.uint64(63))
    if n > 10:
        x[: n // 3] = x[n // 3: 2 * (n // 3)]   # duplicates
    s, passes = cuda.sort(cuda.to_device(x))
    assert np.array_equal(cuda.to_numpy(s), np.sort(x))
    u = cuda.unique(s)
    assert np.array_equal(cuda.to_numpy(u), np.unique(x))


def test_sort_unaligned_buffers(cuda, sort_variant):
    """Buffers 8 but not 16 bytes aligned (the pipelined pass falls back to direct loads)."""
    import ctypes as C
    import torch
    from cablegen_b200._lib import check, lib
    rng = np.random.default_rng(3)
    n = 700_001
    x = rng.integers(0, 1 << 63, size=n, dtype=np.uint64)
    keys = cuda.empty(n + 1)
    tmp = cuda.empty(n + 1)
    keys[1:].copy_(cuda.to_device(x))
    torch.cuda.synchronize()
    in_tmp, passes = C.c_int(), C.c_int()
    check(lib().cgb_sort(keys[1:].data_ptr(), tmp[1:].data_ptr(), n, C.byref(in_tmp), C.byref(passes)))
    out = (tmp if in_tmp.value else keys)[1:]
    assert np.array_equal(cuda.to_numpy(out), np.sort(x))


@pytest.mark.parametrize("kind", ["constant", "sorted", "reversed", "formation", "two_values", "top_bit"])
def test_sort_skewed(cuda, kind, sort_variant):
    rng = np.random.default_rng(11)
    n = 300_000
    if kind == "constant":
        x = np.full(n, 0xFF12FF0000000000, dtype=np.uint64)
    elif kind == "sorted":
        x = np.sort(rng.integers(0, 1 << 40, size=n, dtype=np.uint64))
    elif kind == "reversed":
        x = np.sort(rng.integers(0, 1 << 40, size=n, dtype=np.uint64))[::-1].copy()
    elif kind == "formation":
        x = O.canon(realistic_boards(rng, 50000))
        x = np.concatenate([x] * 6)
    elif kind == "two_values":
        x = np.where(rng.random(n) < 0.5, 0xFFFFFFFFFFFFFFFE, 1).astype(np.uint64)
    else:
        x = rng.integers(0, 2, size=n, dtype=np.uint64) << np.uint64(63)
    s, passes = cuda.sort(cuda.to_device(x))
    assert np.array_equal(cuda.to_numpy(s), np.sort(x))
    assert np.array_equal(cuda.to_numpy(cuda.unique(s)), np.unique(x))
    if kind == "constant":
        assert passes == 0


@pytest.mark.parametrize("na,nb", [(0, 0), (0, 5), (5, 0), (1, 1), (2047, 2049), (100_000, 3), (250_000, 310_000)])
def test_merge_unique(cuda, na, nb):
    rng = np.random.default_rng(na * 7 + nb)
    a = np.unique(rng.integers(0, 1 << 30, size=na, dtype=np.uint64))
    b = np.unique(rng.integers(0, 1 << 30, size=nb, dtype=np.uint64))
    if len(a) and len(b):
        b = np.unique(np.concatenate([b, a[::3]]))  # overlap
    got = cuda.to_numpy(cuda.merge_unique(cuda.to_device(a), cuda.to_device(b)))
    assert np.array_equal(got, np.union1d(a, b))


@pytest.mark.parametrize("na,nb", [(4095, 1), (4096, 4096), (4097, 8191), (3_000_017, 2_000_003)])
def test_merge_unique_repeats(cuda, na, nb):
    """Sorted inputs that keep repeats (the spawn streams): the merge drops them."""
    rng = np.random.default_rng(na + 31 * nb)
    a = np.sort(rng.integers(0, max(na // 3, 1), size=na, dtype=np.uint64))
    b = np.sort(rng.integers(0, max(nb // 2, 1), size=nb, dtype=np.uint64) * np.uint64(3))
    got = cuda.to_numpy(cuda.merge_unique(cuda.to_device(a), cuda.to_device(b)))
    assert np.array_equal(got, np.union1d(a, b))
