"""ctypes binding of the CPU oracle (oracle/cg_oracle.c) -- TEST INFRASTRUCTURE.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import
this module.  The product never does.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_build", "libcg_oracle.so")
REF_LIB = os.path.join(HERE, "_ref", "libcgref.so")
REF_CLI = os.path.join(HERE, "_ref", "cli")

u64 = C.c_uint64
pu64 = C.POINTER(C.c_uint64)
pdbl = C.POINTER(C.c_double)


class Lut(C.Structure):
    _fields_ = [("move", C.c_uint16 * (2 * 65536)), ("locked", C.c_uint8 * (2 * 65536))]


class Settings(C.Structure):
    _fields_ = [("free_formation", C.c_int), ("ignore_f", C.c_int), ("prune", C.c_int),
                ("stsl", C.c_long), ("ltc", C.c_long), ("smallest_large", C.c_long),
                ("nox", C.c_int), ("score", C.c_int)]


_L = None


def build():
    subprocess.run(["make", "-s", "-C", HERE, "oracle"], check=True)


def lib():
    global _L
    if _L is None:
        if not os.path.exists(LIB):
            build()
        L = C.CDLL(LIB)
        for f in ("orc_rot_cw", "orc_rot_ccw", "orc_rot_180", "orc_flip", "orc_canon", "orc_canon_signed"):
            getattr(L, f).restype = u64
            getattr(L, f).argtypes = [u64]
        L.orc_get_sum.restype = C.c_int
        L.orc_get_sum.argtypes = [u64]
        L.orc_build_lut.argtypes = [C.POINTER(Lut), C.c_int, C.c_int]
        L.orc_movedir_unstable.argtypes = [C.POINTER(Lut), pu64, C.c_int]
        L.orc_movedir.argtypes = [C.POINTER(Lut), pu64, C.c_int]
        L.orc_prune.argtypes = [u64, C.c_long, C.c_long, C.c_long]
        L.orc_checkx.argtypes = [u64, C.c_int]
        L.orc_move_layer.argtypes = [C.POINTER(Lut), C.POINTER(Settings), pu64, C.c_size_t,
                                     C.POINTER(pu64), C.POINTER(C.c_size_t)]
        L.orc_spawn_layer.argtypes = [pu64, C.c_size_t, C.POINTER(pu64), C.POINTER(C.c_size_t),
                                      C.POINTER(pu64), C.POINTER(C.c_size_t)]
        L.orc_merge_unique.restype = C.c_size_t
        L.orc_merge_unique.argtypes = [pu64, C.c_size_t, pu64, C.c_size_t, pu64]
        L.orc_sort_unique.restype = C.c_size_t
        L.orc_sort_unique.argtypes = [pu64, C.c_size_t]
        L.orc_cmpbrd.argtypes = [u64, u64]
        L.orc_lookup.restype = C.c_double
        L.orc_lookup.argtypes = [u64, pu64, pdbl, C.c_size_t, C.c_int]
        L.orc_solve_layer.argtypes = [C.POINTER(Lut), C.POINTER(Settings), pu64, C.c_size_t,
                                      pu64, pdbl, C.c_size_t, pu64, pdbl, C.c_size_t, pu64, C.c_size_t, pdbl]
        L.orc_solve_layer_mt.argtypes = L.orc_solve_layer.argtypes + [C.c_int]
        L.free.argtypes = [C.c_void_p]
        _L = L
    return _L


def _p(a, t=pu64):
    return a.ctypes.data_as(t)


def settings(s) -> Settings:
    """From cablegen_b200.configs.Settings."""
    return Settings(int(s.free_formation), int(s.ignore_f), int(s.prune), s.stsl, s.ltc, s.smallest_large,
                    int(s.nox), int(s.score))


def make_lut(free_formation=0, ignore_f=0) -> Lut:
    lut = Lut()
    lib().orc_build_lut(C.byref(lut), int(free_formation), int(ignore_f))
    return lut


def canon(boards) -> np.ndarray:
    L = lib()
    return np.array([L.orc_canon(int(b)) for b in boards], dtype=np.uint64)


def _take(ptr, n):
    a = np.ctypeslib.as_array(ptr, shape=(n,)).copy() if n else np.zeros(0, np.uint64)
    lib().free(C.cast(ptr, C.c_void_p))
    return a


def move_layer(lut, st, boards) -> np.ndarray:
    b = np.ascontiguousarray(boards, dtype=np.uint64)
    out, n = pu64(), C.c_size_t()
    lib().orc_move_layer(C.byref(lut), C.byref(st), _p(b), len(b), C.byref(out), C.byref(n))
    return _take(out, n.value)


def spawn_layer(moved):
    m = np.ascontiguousarray(moved, dtype=np.uint64)
    a, na, b, nb = pu64(), C.c_size_t(), pu64(), C.c_size_t()
    lib().orc_spawn_layer(_p(m), len(m), C.byref(a), C.byref(na), C.byref(b), C.byref(nb))
    return _take(a, na.value), _take(b, nb.value)


def merge_unique(a, b) -> np.ndarray:
    a = np.ascontiguousarray(a, dtype=np.uint64)
    b = np.ascontiguousarray(b, dtype=np.uint64)
    out = np.empty(len(a) + len(b) + 1, dtype=np.uint64)
    n = lib().orc_merge_unique(_p(a), len(a), _p(b), len(b), _p(out))
    return out[:n]


def generate(lut, st, initial, start, end):
    """Layer sweep (generate.c:551-615): {sum: sorted unique moved layer}."""
    layers = {}
    n = np.asarray(initial, dtype=np.uint64)
    n2 = np.zeros(0, np.uint64)
    for s in range(start, end + 1, 2):
        moved = move_layer(lut, st, n)
        layers[s] = moved
        s2, s4 = spawn_layer(moved)
        n = merge_unique(s2, n2)
        n2 = s4
    return layers


def expand_winstates(ws):
    L = lib()
    out = []
    for w in ws:
        w = int(w)
        f = L.orc_flip(w)
        out += [w, L.orc_rot_cw(w), L.orc_rot_180(w), L.orc_rot_ccw(w), f, L.orc_rot_cw(f), L.orc_rot_180(f),
                L.orc_rot_ccw(f)]
    return np.array(out, dtype=np.uint64)


def solve_layer(lut, st, keys, t2, t4, ws_expanded, threads=1) -> np.ndarray:
    keys = np.ascontiguousarray(keys, dtype=np.uint64)
    k2, v2 = (np.ascontiguousarray(t2[0], dtype=np.uint64), np.ascontiguousarray(t2[1], dtype=np.float64))
    k4, v4 = (np.ascontiguousarray(t4[0], dtype=np.uint64), np.ascontiguousarray(t4[1], dtype=np.float64))
    ws = np.ascontiguousarray(ws_expanded, dtype=np.uint64)
    out = np.zeros(max(len(keys), 1), dtype=np.float64)
    args = [C.byref(lut), C.byref(st), _p(keys), len(keys), _p(k2), _p(v2, pdbl), len(k2), _p(k4), _p(v4, pdbl),
            len(k4), _p(ws), len(ws), _p(out, pdbl)]
    if threads > 1:
        lib().orc_solve_layer_mt(*args, threads)
    else:
        lib().orc_solve_layer(*args)
    return out[: len(keys)]


def solve(lut, st, layers, winstates, top, bottom):
    """Top-down solve (solve.c:172-224) over in-memory layers: {sum: values}."""
    ws = expand_winstates(winstates)
    empty = (np.zeros(0, np.uint64), np.zeros(0, np.float64))
    t2 = t4 = empty
    out = {}
    s = top
    while s >= bottom and s > 0:
        keys = layers.get(s, np.zeros(0, np.uint64))
        vals = solve_layer(lut, st, keys, t2, t4, ws)
        out[s] = vals
        t4, t2 = t2, (keys, vals)
        s -= 2
    return out
