"""Host side of the C ABI (no GPU needed): exported symbols, moves, lookup, arrays,
files, settings and string helpers, against the reference's own vectors."""
import ctypes as C
import json
import os
import re

import numpy as np
import pytest

from helpers import ROOT, UNITS, unit

LIB = os.path.join(ROOT, "cablegen_b200", "libcablegen_b200.so")
HEADERS = [os.path.join(ROOT, "include", h) for h in ("cablegen.h", "cablegen_b200.h", "cablegen_format.h")]


class MinSettings(C.Structure):
    _fields_ = [("free_formation", C.c_bool), ("ignore_f", C.c_bool), ("cores", C.c_longlong),
                ("nox", C.c_longlong), ("bdir", C.c_char_p), ("initial", C.c_char_p),
                ("end_gen", C.c_longlong), ("tdir", C.c_char_p), ("winstates", C.c_char_p),
                ("end_solve", C.c_longlong), ("delete_boards", C.c_bool)]


class SArr(C.Structure):
    _fields_ = [("valid", C.c_bool), ("bp", C.POINTER(C.c_uint64)), ("size", C.c_size_t)]


class DArr(C.Structure):
    _fields_ = [("valid", C.c_bool), ("bp", C.POINTER(C.c_uint64)), ("sp", C.POINTER(C.c_uint64)),
                ("size", C.c_size_t)]


class Table(C.Structure):
    _fields_ = [("key", SArr), ("value", SArr)]


@pytest.fixture(scope="module")
def lib(tmp_path_factory):
    os.environ["XDG_CONFIG_HOME"] = str(tmp_path_factory.mktemp("xdg"))
    L = C.CDLL(LIB)
    L.get_settings_min.restype = C.POINTER(MinSettings)
    L.movedir.argtypes = [C.POINTER(C.c_uint64), C.c_int]
    L.movedir.restype = C.c_bool
    L.lookup.argtypes = [C.c_uint64, C.POINTER(Table), C.c_bool]
    L.lookup.restype = C.c_double
    L.get_sum.argtypes = [C.c_uint64]
    L.push_back.argtypes = [C.POINTER(DArr), C.c_uint64]
    L.push_back.restype = C.c_bool
    L.init_darr.argtypes = [C.c_bool, C.c_size_t]
    L.init_darr.restype = DArr
    L.concat.argtypes = [C.POINTER(DArr), C.POINTER(DArr)]
    L.concat.restype = DArr
    L.read_boards.argtypes = [C.c_char_p]
    L.read_boards.restype = SArr
    L.write_boards.argtypes = [SArr, C.c_char_p, C.c_int]
    L.read_table.argtypes = [C.POINTER(Table), C.c_char_p]
    L.change_config.argtypes = [C.c_char_p]
    L.format_str.restype = C.c_void_p
    L.pun_uint64.argtypes = [C.c_uint64]
    L.pun_uint64.restype = C.c_double
    return L


def declared_functions(headers=HEADERS):
    names = set()
    for h in headers:
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"^[A-Za-z_][\w \*]*?\b(\w+)\s*\([^;{]*\)\s*;", text, flags=re.M):
            if not m.group(0).lstrip().startswith("typedef"):
                names.add(m.group(1))
    return names


def test_every_declared_symbol_is_exported():
    L = C.CDLL(LIB)
    names = declared_functions()
    assert {"generate", "solve", "lookup", "movedir", "cgb_sweep_run", "cgb_sort_unique_noalloc",
            "format_str"} <= names
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing


def test_cl_seam_exports_every_declared_function():
    """libcablegen_b200_cl.so (the reference's GPU plug-in seam on this engine) defines every
    cl_* function of include/cablegen_cl.h and leaves only get_settings_min() to the reference's
    objects it is linked with."""
    import subprocess
    lib = os.path.join(ROOT, "cablegen_b200", "libcablegen_b200_cl.so")
    names = declared_functions([os.path.join(ROOT, "include", "cablegen_cl.h")])
    assert len(names) == 11 and all(n.startswith("cl_") for n in names), names
    out = subprocess.run(["nm", "-D", lib], capture_output=True, text=True, check=True).stdout
    defined = {l.split()[-1] for l in out.splitlines() if " T " in l}
    undefined = {l.split()[-1] for l in out.splitlines() if l.split()[0] == "U" and "@" not in l}
    assert names <= defined, names - defined
    assert undefined == {"get_settings_min"}, undefined


@pytest.mark.parametrize("ff,ig", [(0, 0), (0, 1), (1, 0), (1, 1)])
def test_movedir_matches_reference(lib, ff, ig):
    s = lib.get_settings_min().contents
    s.free_formation, s.ignore_f = bool(ff), bool(ig)
    lib.generate_lut()
    boards = unit("boards.u64", np.uint64)
    tag = f"ff{ff}_ig{ig}"
    mv = unit(f"move_stable_{tag}.u64", np.uint64).reshape(-1, 4)
    ok = unit(f"move_stable_ok_{tag}.u8", np.uint8).reshape(-1, 4)
    for i, b in enumerate(boards):
        for d in range(4):
            x = C.c_uint64(int(b))
            assert bool(lib.movedir(C.byref(x), d)) == bool(ok[i, d])
            assert x.value == mv[i, d]
    s.free_formation, s.ignore_f = False, False
    lib.generate_lut()


def test_lookup_and_sum_match_reference(lib):
    keys = unit("lookup_keys.u64", np.uint64)
    vals = unit("lookup_vals.f64", np.float64)
    qs = unit("lookup_queries.u64", np.uint64)
    t = Table(SArr(True, keys.ctypes.data_as(C.POINTER(C.c_uint64)), len(keys)),
              SArr(True, vals.view(np.uint64).ctypes.data_as(C.POINTER(C.c_uint64)), len(keys)))
    for canon, name in ((1, "lookup_canon.f64"), (0, "lookup_nocanon.f64")):
        want = unit(name, np.float64)
        got = np.array([lib.lookup(int(q), C.byref(t), bool(canon)) for q in qs])
        assert np.array_equal(got, want)
    boards = unit("boards.u64", np.uint64)
    sums = unit("get_sum.i32", np.int32)
    assert all(lib.get_sum(int(b)) == s for b, s in zip(boards, sums))


def test_arrays(lib):
    """test.c:54-113: growth and concatenation."""
    for n in range(0, 20):
        for m in range(0, 20):
            a = lib.init_darr(False, n)
            b = lib.init_darr(False, m)
            for i in range(n):
                lib.push_back(C.byref(a), i)
            for i in range(m):
                lib.push_back(C.byref(b), i)
            c = lib.concat(C.byref(a), C.byref(b))
            cnt = (C.cast(c.sp, C.c_void_p).value - C.cast(c.bp, C.c_void_p).value) // 8 if n + m else 0
            assert cnt == n + m
            got = [c.bp[i] for i in range(n + m)]
            assert got == list(range(n)) + list(range(m))


def test_board_and_table_files_round_trip(lib, tmp_path):
    data = (np.arange(1000, dtype=np.uint64) * 0x9E3779B97F4A7C15) & np.uint64(0x7FFFFFFFFFFFFFFF)
    a = SArr(True, data.ctypes.data_as(C.POINTER(C.c_uint64)), len(data))
    fmt = str(tmp_path / "%d.boards").encode()
    lib.write_boards(a, fmt, 42)
    r = lib.read_boards(str(tmp_path / "42.boards").encode())
    assert r.valid and r.size == len(data)
    assert np.array_equal(np.ctypeslib.as_array(r.bp, shape=(r.size,)), data)
    keys = np.sort(data)
    vals = np.linspace(0, 1, len(keys))
    (tmp_path / "7.tables").write_bytes(keys.tobytes() + vals.tobytes())
    t = Table()
    lib.read_table(C.byref(t), str(tmp_path / "7.tables").encode())
    assert t.key.valid and t.key.size == len(keys)
    for i in (0, 17, 999):
        assert lib.lookup(int(keys[i]), C.byref(t), False) == vals[i]
    missing = lib.read_boards(str(tmp_path / "nope.boards").encode())
    assert not missing.valid


def test_truncated_boards_file_warns_and_counts_whole_boards(tmp_path):
    """A .boards file whose size is not a multiple of 8 is read with a warning and its whole
    boards only (src/generate.c:616-648)."""
    import subprocess
    import sys
    data = (np.arange(1, 101, dtype=np.uint64) * 0x0123456789ABCDEF)
    path = tmp_path / "t.boards"
    path.write_bytes(data.tobytes() + b"\x01\x02\x03")
    code = (
        "import ctypes as C, sys\n"
        "class SArr(C.Structure):\n"
        "    _fields_ = [('valid', C.c_bool), ('bp', C.POINTER(C.c_uint64)), ('size', C.c_size_t)]\n"
        f"L = C.CDLL({LIB!r})\n"
        "L.read_boards.argtypes = [C.c_char_p]\n"
        "L.read_boards.restype = SArr\n"
        f"r = L.read_boards({str(path)!r}.encode())\n"
        "sys.stdout.flush()\n"
        "print('RESULT', int(r.valid), r.size, r.bp[0], r.bp[r.size - 1])\n")
    out = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, check=True,
                         env=dict(os.environ, XDG_CONFIG_HOME=str(tmp_path))).stdout
    assert "[WARN] sz %8 != 0, this is probably not a real table!" in out
    res = [line for line in out.splitlines() if line.startswith("RESULT")][0].split()
    assert res[1:] == ["1", "100", str(int(data[0])), str(int(data[-1]))]


def test_settings_from_ini(lib, tmp_path):
    conf = tmp_path / "c.conf"
    conf.write_text("""; comment
[Cablegen]
free_formation = TRUE
cores = 12
nox = 10
[Generate]
dir = "./b/"
end = 640
[Solve]
dir = ./t/  ; trailing comment
end = 20
""")
    lib.change_config(str(conf).encode())
    s = lib.get_settings_min().contents
    assert s.free_formation and s.cores == 12 and s.nox == 10 and s.end_gen == 640 and s.end_solve == 20
    assert s.bdir == b"./b/" and s.tdir == b"./t/"
    empty = tmp_path / "empty.conf"
    empty.write_text("")
    lib.change_config(str(empty).encode())
    s = lib.get_settings_min().contents
    assert s.free_formation  # keys absent from a new file keep their values (src/settings.c:34-86)


def test_format_helpers(lib):
    p = lib.format_str(b"%s%d.boards", b"./x/", C.c_int(12))
    assert C.string_at(p) == b"./x/12.boards"
    assert lib.pun_uint64(0x3FF0000000000000) == 1.0
