"""ctypes binding of libcablegen_b200.so (include/cablegen_b200.h, include/cablegen.h).

The product path has no fallback: if the shared library is missing or cannot
be loaded, every call raises ExtensionMissing.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libcablegen_b200.so")


class ExtensionMissing(RuntimeError):
    pass


class CablegenError(RuntimeError):
    pass


class Rules(C.Structure):
    """cgb_rules (include/cablegen_b200.h)."""
    _fields_ = [("free_formation", C.c_int), ("ignore_f", C.c_int), ("prune", C.c_int),
                ("stsl", C.c_longlong), ("ltc", C.c_longlong), ("smallest_large", C.c_longlong),
                ("nox", C.c_int), ("score", C.c_int)]


class Stats(C.Structure):
    """cgb_stats (include/cablegen_b200.h)."""
    _fields_ = [("layers", C.c_uint64), ("boards_generated", C.c_uint64), ("boards_solved", C.c_uint64),
                ("gen_ms", C.c_double), ("solve_ms", C.c_double), ("total_ms", C.c_double),
                ("expand_ms", C.c_double), ("sort_ms", C.c_double), ("unique_ms", C.c_double),
                ("merge_ms", C.c_double), ("solve_kernel_ms", C.c_double), ("index_ms", C.c_double),
                ("sorted_keys", C.c_uint64), ("sort_key_passes", C.c_uint64), ("lookups_bytes", C.c_uint64),
                ("h2d_bytes", C.c_uint64), ("d2h_bytes", C.c_uint64), ("max_abs_err", C.c_double),
                ("gpu_launches", C.c_uint64), ("spilled_chunks", C.c_uint64), ("restored_chunks", C.c_uint64),
                ("layer_slices", C.c_uint64)]

    def as_dict(self):
        return {name: getattr(self, name) for name, _ in self._fields_}


class KernelStats(C.Structure):
    """cgb_kernel_stats (include/cablegen_b200.h)."""
    _fields_ = [("launches", C.c_uint64)] + \
        [(f"{k}_ms", C.c_double) for k in ("hist", "onesweep", "unique", "merge", "expand", "spawn", "solve",
                                          "index")] + \
        [(f"{k}_bytes", C.c_uint64) for k in ("hist", "onesweep", "unique", "merge", "expand", "spawn",
                                             "solve")] + \
        [("onesweep_launches", C.c_uint64), ("solve_launches", C.c_uint64), ("solve_boards", C.c_uint64),
         ("lookups", C.c_uint64), ("index_builds", C.c_uint64), ("compact_index_builds", C.c_uint64),
         ("moves_raw", C.c_uint64), ("moves_kept", C.c_uint64), ("pool_trims", C.c_uint64)]

    def as_dict(self):
        return {name: getattr(self, name) for name, _ in self._fields_}


LAYER_FN = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_int, C.POINTER(C.c_uint64), C.c_uint64)
TABLE_FN = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_int, C.POINTER(C.c_uint64), C.c_void_p, C.c_uint64, C.c_int)

ERROR_FN = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_int, C.c_uint64, C.c_double, C.c_double)


class Sweep(C.Structure):
    """cgb_sweep (include/cablegen_b200.h)."""
    _fields_ = [("initial", C.POINTER(C.c_uint64)), ("n_initial", C.c_uint64), ("start", C.c_int),
                ("end_gen", C.c_int), ("end_solve", C.c_int), ("winstates", C.POINTER(C.c_uint64)),
                ("n_winstates", C.c_int), ("precision", C.c_int), ("layer_fn", LAYER_FN), ("table_fn", TABLE_FN),
                ("error_fn", ERROR_FN), ("user", C.c_void_p)]


class Formation(C.Structure):
    """cgb_formation (include/cablegen_b200.h)."""
    _fields_ = [("initial", C.POINTER(C.c_uint64)), ("n_initial", C.c_uint64), ("end_gen", C.c_int),
                ("end_solve", C.c_int), ("winstates", C.POINTER(C.c_uint64)), ("n_winstates", C.c_int)]


BATCH_LAYER_FN = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_int, C.c_int, C.POINTER(C.c_uint64), C.c_uint64)
BATCH_TABLE_FN = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_int, C.c_int, C.POINTER(C.c_uint64), C.c_void_p,
                             C.c_uint64, C.c_int)


class Batch(C.Structure):
    """cgb_batch (include/cablegen_b200.h)."""
    _fields_ = [("formations", C.POINTER(Formation)), ("n_formations", C.c_int), ("precision", C.c_int),
                ("use_graphs", C.c_int), ("layer_fn", BATCH_LAYER_FN), ("table_fn", BATCH_TABLE_FN),
                ("user", C.c_void_p)]


class BatchStats(C.Structure):
    """cgb_batch_stats (include/cablegen_b200.h)."""
    _fields_ = [("groups", C.c_uint64), ("gen_steps", C.c_uint64), ("solve_steps", C.c_uint64),
                ("boards_generated", C.c_uint64), ("boards_solved", C.c_uint64), ("gen_ms", C.c_double),
                ("solve_ms", C.c_double), ("total_ms", C.c_double), ("graph_launches", C.c_uint64),
                ("gpu_launches", C.c_uint64), ("lookups", C.c_uint64), ("h2d_bytes", C.c_uint64),
                ("d2h_bytes", C.c_uint64)]

    def as_dict(self):
        return {name: getattr(self, name) for name, _ in self._fields_}


_lib = None

u64 = C.c_uint64
pu64 = C.POINTER(C.c_uint64)
vp = C.c_void_p


def _declare(L):
    sig = {
        "cgb_last_error": (C.c_char_p, []),
        "cgb_init": (C.c_int, [C.c_int]),
        "cgb_set_rules": (C.c_int, [C.POINTER(Rules)]),
        "cgb_set_option": (C.c_int, [C.c_char_p, C.c_longlong]),
        "cgb_get_option": (C.c_longlong, [C.c_char_p]),
        "cgb_expand_moves": (C.c_int, [vp, u64, vp, u64, pu64]),
        "cgb_count_spawns": (C.c_int, [vp, u64, pu64]),
        "cgb_expand_spawns": (C.c_int, [vp, u64, vp, vp, u64, pu64]),
        "cgb_sort": (C.c_int, [vp, vp, u64, C.POINTER(C.c_int), C.POINTER(C.c_int)]),
        "cgb_unique": (C.c_int, [vp, u64, vp, pu64]),
        "cgb_merge_unique": (C.c_int, [vp, u64, vp, u64, vp, pu64]),
        "cgb_canonicalize": (C.c_int, [vp, u64, vp]),
        "cgb_get_kernel_stats": (C.c_int, [C.POINTER(KernelStats)]),
        "cgb_reset_kernel_stats": (C.c_int, []),
        "cgb_solve_layer": (C.c_int, [vp, u64, vp, C.c_int, vp, vp, u64, vp, vp, u64, pu64, C.c_int]),
        "cgb_lookup_batch": (C.c_int, [vp, vp, u64, C.c_int, vp, u64, C.c_int, vp]),
        "cgb_generate": (C.c_int, [pu64, u64, C.c_int, C.c_int, LAYER_FN, vp, C.POINTER(Stats)]),
        "cgb_sweep_run": (C.c_int, [C.POINTER(Sweep), C.POINTER(Stats)]),
        "cgb_batch_run": (C.c_int, [C.POINTER(Batch), C.POINTER(BatchStats)]),
        "cgb_batch_plan": (C.c_int, [C.POINTER(Formation), C.c_int, C.POINTER(C.c_int)]),
        "cgb_tablebase": (C.c_int, [pu64, u64, C.c_int, C.c_int, C.c_int, pu64, C.c_int, C.c_int, LAYER_FN,
                                    TABLE_FN, vp, C.POINTER(Stats)]),
    }
    for name, (res, args) in sig.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ExtensionMissing(f"{LIB_PATH} is not built; run `python -m cablegen_b200.build`")
        try:
            L = C.CDLL(LIB_PATH, mode=C.RTLD_LOCAL)
        except OSError as e:
            raise ExtensionMissing(f"cannot load {LIB_PATH}: {e}") from e
        _declare(L)
        _lib = L
    return _lib


def check(rc: int):
    if rc != 0:
        raise CablegenError(lib().cgb_last_error().decode(errors="replace"))
