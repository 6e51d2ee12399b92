"""cgb_sort_unique_noalloc: the sort + unique entry point that allocates nothing.

It exists for callers that cannot let this library allocate device memory
(a host whose own allocator owns the GPU under a hard budget, or code that
cannot absorb cudaMalloc's device-wide synchronisation).  The test makes the
set-up call (n = 0) first, then calls the entry point through the C ABI twice
in a row and compares both results bit for bit (integer keys) with np.unique
of the input and with the allocating entry points cgb_sort + cgb_unique.
"""
import ctypes as C

import numpy as np
import pytest
import torch

import py_oracle as O
from cablegen_b200 import _lib
from helpers import realistic_boards

pytestmark = pytest.mark.gpu

MAX_KEYS = 1 << 20


def _fn():
    f = _lib.lib().cgb_sort_unique_noalloc
    f.restype = C.c_int
    f.argtypes = [C.c_void_p, C.c_uint64, C.c_void_p, C.POINTER(C.c_uint64), C.c_void_p]
    return f


def _inputs(seed, n):
    rng = np.random.default_rng(seed)
    boards = O.canon(realistic_boards(rng, n // 4))          # canonical formation keys
    x = np.concatenate([boards, boards[: n // 4], rng.integers(0, 1 << 64, n - 2 * (n // 4), dtype=np.uint64)])
    rng.shuffle(x)
    return x


def _noalloc(f, xd, n, out):
    cnt = C.c_uint64(0)
    torch.cuda.synchronize()
    rc = f(C.c_void_p(xd.data_ptr()), n, C.c_void_p(out.data_ptr()), C.byref(cnt), None)
    assert rc == 0, _lib.lib().cgb_last_error().decode()
    return out[: cnt.value]


def test_noalloc_matches_allocating_path(cuda):
    f = _fn()
    runs = [(101, 300_000), (202, MAX_KEYS)]
    # inputs and outputs are allocated by the caller, before the calls
    xs = [_inputs(seed, n) for seed, n in runs]
    xds = [cuda.to_device(x) for x in xs]
    outs = [torch.empty(n, dtype=torch.int64, device="cuda") for _, n in runs]
    # set-up only: places the fixed scratch array on this GPU (the one allocation, by the driver)
    cnt = C.c_uint64(5)
    assert f(None, 0, None, C.byref(cnt), None) == 0, _lib.lib().cgb_last_error().decode()
    assert cnt.value == 0
    results = []
    for i, (seed, n) in enumerate(runs):
        x, xd = xs[i], xds[i]
        torch.cuda.synchronize()
        free_before = torch.cuda.mem_get_info()[0]
        got = _noalloc(f, xd, n, outs[i])
        torch.cuda.synchronize()
        # after the set-up, nothing is allocated by a call (memory can only have been freed)
        assert torch.cuda.mem_get_info()[0] >= free_before
        assert np.array_equal(cuda.to_numpy(xd), x)   # input untouched
        results.append((xd, got))
    for (xd, got), x in zip(results, xs):
        assert np.array_equal(cuda.to_numpy(got), np.unique(x))
        want = cuda.sort_unique(xd)                     # cgb_sort + cgb_unique
        assert got.numel() == want.numel()
        assert torch.equal(got, want)


def test_noalloc_rejects_oversize_and_empty(cuda):
    f = _fn()
    xd = torch.zeros(MAX_KEYS + 1, dtype=torch.int64, device="cuda")
    out = torch.empty_like(xd)
    cnt = C.c_uint64(7)
    rc = f(C.c_void_p(xd.data_ptr()), MAX_KEYS + 1, C.c_void_p(out.data_ptr()), C.byref(cnt), None)
    assert rc == -1
    assert "exceed" in _lib.lib().cgb_last_error().decode()
    rc = f(C.c_void_p(xd.data_ptr()), 0, C.c_void_p(out.data_ptr()), C.byref(cnt), None)
    assert rc == 0 and cnt.value == 0
