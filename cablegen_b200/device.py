"""Device-level entry points of the engine on torch CUDA tensors.

Boards live in int64 tensors (the same 64 bits as the reference's uint64_t).
Every call hands raw device pointers to the C ABI (include/cablegen_b200.h),
which runs on the engine's own CUDA stream and returns only when its work is
complete; torch's current stream is synchronised before each call so inputs
written by torch are visible.
"""
from __future__ import annotations

import ctypes as C
from typing import Dict, Optional, Sequence, Tuple

import numpy as np
import torch

from . import _lib
from ._lib import check, lib
from .configs import Settings


def _ptr(t: torch.Tensor):
    assert t.is_cuda and t.is_contiguous()
    return C.c_void_p(t.data_ptr())


def _sync():
    torch.cuda.current_stream().synchronize()


def init(device: int = 0):
    check(lib().cgb_init(device))


def set_rules(settings: Settings):
    r = _lib.Rules(int(settings.free_formation), int(settings.ignore_f), int(settings.prune), settings.stsl,
                   settings.ltc, settings.smallest_large, settings.nox, int(settings.score))
    check(lib().cgb_set_rules(C.byref(r)))


def set_option(name: str, value: int):
    check(lib().cgb_set_option(name.encode(), int(value)))


def get_option(name: str) -> int:
    return int(lib().cgb_get_option(name.encode()))


def kernel_stats() -> dict:
    k = _lib.KernelStats()
    check(lib().cgb_get_kernel_stats(C.byref(k)))
    return k.as_dict()


def reset_kernel_stats():
    check(lib().cgb_reset_kernel_stats())


def to_device(a, device="cuda") -> torch.Tensor:
    a = np.ascontiguousarray(np.asarray(a, dtype=np.uint64))
    return torch.from_numpy(a.view(np.int64)).to(device)


def to_numpy(t: torch.Tensor) -> np.ndarray:
    return t.cpu().numpy().view(np.uint64)


def empty(n: int, device="cuda") -> torch.Tensor:
    return torch.empty(max(int(n), 1), dtype=torch.int64, device=device)


def canonicalize(x: torch.Tensor) -> torch.Tensor:
    _sync()
    out = empty(x.numel())
    check(lib().cgb_canonicalize(_ptr(x), x.numel(), _ptr(out)))
    return out[: x.numel()]


def expand_moves(x: torch.Tensor) -> torch.Tensor:
    _sync()
    n = x.numel()
    out = empty(4 * n)
    cnt = C.c_uint64()
    check(lib().cgb_expand_moves(_ptr(x), n, _ptr(out), 4 * n, C.byref(cnt)))
    return out[: cnt.value]


def count_spawns(x: torch.Tensor) -> int:
    _sync()
    tot = C.c_uint64()
    check(lib().cgb_count_spawns(_ptr(x), x.numel(), C.byref(tot)))
    return tot.value


def expand_spawns(x: torch.Tensor) -> Tuple[torch.Tensor, torch.Tensor]:
    total = count_spawns(x)
    o2, o4 = empty(total), empty(total)
    cnt = C.c_uint64()
    check(lib().cgb_expand_spawns(_ptr(x), x.numel(), _ptr(o2), _ptr(o4), total, C.byref(cnt)))
    return o2[: cnt.value], o4[: cnt.value]


def sort(x: torch.Tensor) -> Tuple[torch.Tensor, int]:
    """Ascending unsigned sort; returns (sorted tensor, digit passes)."""
    _sync()
    keys = x.clone()
    tmp = empty(x.numel())
    in_tmp, passes = C.c_int(), C.c_int()
    check(lib().cgb_sort(_ptr(keys), _ptr(tmp), x.numel(), C.byref(in_tmp), C.byref(passes)))
    return (tmp if in_tmp.value else keys)[: x.numel()], passes.value


def unique(x_sorted: torch.Tensor) -> torch.Tensor:
    _sync()
    out = empty(x_sorted.numel())
    cnt = C.c_uint64()
    check(lib().cgb_unique(_ptr(x_sorted), x_sorted.numel(), _ptr(out), C.byref(cnt)))
    return out[: cnt.value]


def sort_unique(x: torch.Tensor) -> torch.Tensor:
    s, _ = sort(x)
    return unique(s)


def merge_unique(a: torch.Tensor, b: torch.Tensor) -> torch.Tensor:
    _sync()
    out = empty(a.numel() + b.numel())
    cnt = C.c_uint64()
    check(lib().cgb_merge_unique(_ptr(a) if a.numel() else None, a.numel(), _ptr(b) if b.numel() else None,
                                 b.numel(), _ptr(out), C.byref(cnt)))
    return out[: cnt.value]


def solve_layer(keys: torch.Tensor, t2: Tuple[torch.Tensor, torch.Tensor], t4: Tuple[torch.Tensor, torch.Tensor],
                winstates: Sequence[int], precision: int = 64) -> torch.Tensor:
    _sync()
    dt = torch.float64 if precision == 64 else torch.float32
    out = torch.empty(max(keys.numel(), 1), dtype=dt, device=keys.device)
    ws = (C.c_uint64 * max(len(winstates), 1))(*[int(w) for w in winstates])

    def p(t):
        return _ptr(t) if t is not None and t.numel() else None

    check(lib().cgb_solve_layer(p(keys), keys.numel(), _ptr(out), precision, p(t2[0]), p(t2[1]), t2[0].numel(),
                                p(t4[0]), p(t4[1]), t4[0].numel(), ws, len(winstates)))
    return out[: keys.numel()]


def lookup_batch(keys: torch.Tensor, vals: torch.Tensor, boards: torch.Tensor, canonicalize: bool = False) -> torch.Tensor:
    """Values of `boards` in one solved layer (keys sorted, vals float64 or float32) through the
    engine's index; float64, 0.0 for a board not in the layer (lookup(), src/solve.c:108-164)."""
    _sync()
    precision = 32 if vals.dtype == torch.float32 else 64
    out = torch.empty(max(boards.numel(), 1), dtype=torch.float64, device=boards.device)

    def p(t):
        return _ptr(t) if t is not None and t.numel() else None

    check(lib().cgb_lookup_batch(p(keys), p(vals), keys.numel(), precision, p(boards), boards.numel(),
                                 1 if canonicalize else 0, _ptr(out)))
    return out[: boards.numel()]


def generate(initial: Sequence[int], start: int, end: int, keep: bool = True):
    """Generation sweep; returns ({sum: numpy layer}, stats dict)."""
    layers: Dict[int, np.ndarray] = {}

    def on_layer(user, s, ptr, n):
        if keep:
            layers[s] = np.ctypeslib.as_array(ptr, shape=(n,)).copy() if n else np.zeros(0, np.uint64)
        return 0

    cb = _lib.LAYER_FN(on_layer)
    init_a = (C.c_uint64 * max(len(initial), 1))(*[int(b) for b in initial])
    st = _lib.Stats()
    check(lib().cgb_generate(init_a, len(initial), start, end, cb, None, C.byref(st)))
    return layers, st.as_dict()


def tablebase(initial: Sequence[int], start: int, end_gen: int, end_solve: int, winstates: Sequence[int],
              precision: int = 64, keep_layers: bool = False, keep_tables: bool = False,
              layer_fn=None, table_fn=None, error_fn=None):
    """Generation + solve with layers resident in HBM (cgb_sweep_run).

    precision 64 / 32, or 0 to run both and report per-layer FP32 errors
    (error_fn(sum, n, max_abs, mean_abs); also returned as stats['layer_errors']).
    Returns (layers, tables, stats): layers {sum: keys}, tables {sum: (keys, values)} when kept.
    """
    layers, tables, errors = {}, {}, {}

    def on_layer(user, s, ptr, n):
        if keep_layers:
            layers[s] = np.ctypeslib.as_array(ptr, shape=(n,)).copy() if n else np.zeros(0, np.uint64)
        if layer_fn is not None:
            layer_fn(s, ptr, n)
        return 0

    def on_table(user, s, kptr, vptr, n, prec):
        if keep_tables:
            k = np.ctypeslib.as_array(kptr, shape=(n,)).copy() if n else np.zeros(0, np.uint64)
            vt = C.c_double if prec == 64 else C.c_float
            v = (np.ctypeslib.as_array(C.cast(vptr, C.POINTER(vt)), shape=(n,)).copy() if n
                 else np.zeros(0, np.float64 if prec == 64 else np.float32))
            tables[s] = (k, v)
        if table_fn is not None:
            table_fn(s, kptr, vptr, n, prec)
        return 0

    def on_error(user, s, n, mx, mean):
        errors[s] = (n, mx, mean)
        if error_fn is not None:
            error_fn(s, n, mx, mean)
        return 0

    want_layers = keep_layers or layer_fn is not None
    want_tables = keep_tables or table_fn is not None
    w = _lib.Sweep()
    init_a = (C.c_uint64 * max(len(initial), 1))(*[int(b) for b in initial])
    ws = (C.c_uint64 * max(len(winstates), 1))(*[int(x) for x in winstates])
    w.initial = init_a
    w.n_initial = len(initial)
    w.start, w.end_gen, w.end_solve = start, end_gen, end_solve
    w.winstates = ws
    w.n_winstates = len(winstates)
    w.precision = precision
    w.layer_fn = _lib.LAYER_FN(on_layer) if want_layers else _lib.LAYER_FN()
    w.table_fn = _lib.TABLE_FN(on_table) if want_tables else _lib.TABLE_FN()
    w.error_fn = _lib.ERROR_FN(on_error) if precision == 0 else _lib.ERROR_FN()
    st = _lib.Stats()
    check(lib().cgb_sweep_run(C.byref(w), C.byref(st)))
    stats = st.as_dict()
    if precision == 0:
        stats["layer_errors"] = errors
    return layers, tables, stats


def batch(formations, precision: int = 32, use_graphs: bool = True, keep_layers: bool = False,
          keep_tables: bool = False, layer_fn=None, table_fn=None):
    """Many formations in one sweep (cgb_batch_run).

    formations: objects with .initial, .end_gen, .end_solve, .winstates (configs.Formation).
    Returns (layers, tables, stats): layers {(formation, sum): keys}, tables {(formation, sum): (keys, values)}
    when kept.
    """
    layers, tables = {}, {}

    def on_layer(user, f, s, ptr, n):
        if keep_layers:
            layers[(f, s)] = np.ctypeslib.as_array(ptr, shape=(n,)).copy() if n else np.zeros(0, np.uint64)
        if layer_fn is not None:
            layer_fn(f, s, ptr, n)
        return 0

    def on_table(user, f, s, kptr, vptr, n, prec):
        if keep_tables:
            vt = C.c_double if prec == 64 else C.c_float
            k = np.ctypeslib.as_array(kptr, shape=(n,)).copy() if n else np.zeros(0, np.uint64)
            v = (np.ctypeslib.as_array(C.cast(vptr, C.POINTER(vt)), shape=(n,)).copy() if n
                 else np.zeros(0, np.float64 if prec == 64 else np.float32))
            tables[(f, s)] = (k, v)
        if table_fn is not None:
            table_fn(f, s, kptr, vptr, n, prec)
        return 0

    keep = []
    arr = (_lib.Formation * max(len(formations), 1))()
    for i, f in enumerate(formations):
        init = (C.c_uint64 * max(len(f.initial), 1))(*[int(b) for b in f.initial])
        ws = (C.c_uint64 * max(len(f.winstates), 1))(*[int(x) for x in f.winstates])
        keep += [init, ws]
        arr[i].initial = init
        arr[i].n_initial = len(f.initial)
        arr[i].end_gen = int(f.end_gen)
        arr[i].end_solve = int(getattr(f, "end_solve", 0))
        arr[i].winstates = ws
        arr[i].n_winstates = len(f.winstates)
    b = _lib.Batch()
    b.formations = arr
    b.n_formations = len(formations)
    b.precision = precision
    b.use_graphs = 1 if use_graphs else 0
    want_layers = keep_layers or layer_fn is not None
    want_tables = keep_tables or table_fn is not None
    lf = _lib.BATCH_LAYER_FN(on_layer) if want_layers else _lib.BATCH_LAYER_FN()
    tf = _lib.BATCH_TABLE_FN(on_table) if want_tables else _lib.BATCH_TABLE_FN()
    b.layer_fn = lf
    b.table_fn = tf
    st = _lib.BatchStats()
    _sync()
    check(lib().cgb_batch_run(C.byref(b), C.byref(st)))
    return layers, tables, st.as_dict()
