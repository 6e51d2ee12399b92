"""Failure paths of the engine, made on purpose without faulting the GPU: every wait is
bounded and every device error is a bit in an error word that the host turns into -1 and
cgb_last_error() (the C API's functions log and exit, as the reference's do on allocation
failure: src/array.c, malloc_errcheck).

* a decoupled look-back wait that runs out: a test switch keeps tile 0 of a digit pass from
  publishing, so tile 1 waits on a flag that nothing sets; with the poll limit lowered the
  wait gives up, the pass reports "look-back wait timed out", and the context stays usable;
* merge of a run that is not sorted: "input not sorted";
* an output buffer one board short: "output capacity exceeded", nothing written past it;
* a capped device allocator: the engine's call returns -1, and the reference-API
  generate() logs the error and exits with EXIT_FAILURE in a child process.
"""
import ctypes as C
import os
import subprocess
import sys
import textwrap

import numpy as np
import pytest
import torch

import py_oracle as O
from cablegen_b200 import _lib, configs
from helpers import ROOT, realistic_boards

pytestmark = pytest.mark.gpu


def _keys(n, seed=7):
    rng = np.random.default_rng(seed)
    return O.canon(realistic_boards(rng, n))


def test_lookback_wait_runs_out_and_context_survives(cuda):
    x = cuda.to_device(_keys(300_000))
    try:
        cuda.set_option("lookback_spin_limit", 4096)
        cuda.set_option("lookback_hold_first_tile", 1)
        for variant in (0, 1, 2):
            old = cuda.get_option("sort_variant")
            cuda.set_option("sort_variant", variant)
            try:
                with pytest.raises(_lib.CablegenError, match="look-back wait timed out"):
                    cuda.sort(x)
            finally:
                cuda.set_option("sort_variant", old)
    finally:
        cuda.set_option("lookback_hold_first_tile", 0)
        cuda.set_option("lookback_spin_limit", 0)
    # the same context sorts correctly afterwards
    got, _ = cuda.sort(x)
    assert np.array_equal(cuda.to_numpy(got), np.sort(cuda.to_numpy(x)))


def test_merge_of_unsorted_run_is_reported(cuda):
    a = np.unique(_keys(50_000, 1))
    b = np.unique(_keys(50_000, 2))
    bad = a.copy()
    bad[1000], bad[30_000] = bad[30_000], bad[1000]   # two keys out of order
    with pytest.raises(_lib.CablegenError, match="input not sorted"):
        cuda.merge_unique(cuda.to_device(bad), cuda.to_device(b))
    got = cuda.merge_unique(cuda.to_device(a), cuda.to_device(b))
    assert np.array_equal(cuda.to_numpy(got), np.union1d(a, b))


def test_unique_of_unsorted_input_is_reported(cuda):
    x = np.sort(_keys(20_000, 3))
    x[10], x[5000] = x[5000], x[10]
    with pytest.raises(_lib.CablegenError, match="input not sorted"):
        cuda.unique(cuda.to_device(x))


def test_output_one_short_is_reported(cuda):
    w = configs.get("ll_pruned")
    cuda.set_rules(w.settings)
    x = cuda.to_device(realistic_boards(np.random.default_rng(4), 100_000))
    L = _lib.lib()
    total = cuda.count_spawns(x)
    o2 = torch.full((total + 8,), -1, dtype=torch.int64, device="cuda")
    o4 = torch.full((total + 8,), -1, dtype=torch.int64, device="cuda")
    cnt = C.c_uint64()
    torch.cuda.synchronize()
    assert L.cgb_expand_spawns(x.data_ptr(), x.numel(), o2.data_ptr(), o4.data_ptr(), total - 1, C.byref(cnt)) == -1
    assert "output capacity exceeded" in L.cgb_last_error().decode()
    assert int(o2[total - 1]) == -1 and int(o4[total - 1]) == -1   # nothing written past the capacity
    # the move expansion refuses an output below its 4n bound before launching
    out = torch.empty(4 * x.numel(), dtype=torch.int64, device="cuda")
    assert L.cgb_expand_moves(x.data_ptr(), x.numel(), out.data_ptr(), 4 * x.numel() - 1, C.byref(cnt)) == -1
    assert "4n" in L.cgb_last_error().decode()
    got2, got4 = cuda.expand_spawns(x)                # and the next call works
    assert got2.numel() == total and got4.numel() == total


def test_capped_allocator_engine_call_fails_cleanly(cuda):
    w = configs.get("ll_pruned", end_gen=120)
    f = w.formations[0]
    cuda.set_rules(w.settings)
    try:
        cuda.set_option("device_mem_cap_mb", 1)
        with pytest.raises(_lib.CablegenError, match="over the cap"):
            cuda.tablebase(f.initial, f.start, f.end_gen, f.start, f.winstates, precision=64)
    finally:
        cuda.set_option("device_mem_cap_mb", 0)
    _, _, st = cuda.tablebase(f.initial, f.start, f.end_gen, f.start, f.winstates, precision=64)
    assert st["layers"] == (f.end_gen - f.start) // 2 + 1


CHILD = textwrap.dedent("""
    import ctypes as C, os, sys
    import numpy as np
    sys.path.insert(0, {root!r})
    from cablegen_b200 import _lib, configs
    L = _lib.lib()
    class SArr(C.Structure):
        _fields_ = [("valid", C.c_bool), ("bp", C.POINTER(C.c_uint64)), ("size", C.c_size_t)]
    L.generate.argtypes = [C.c_int, C.c_int, C.c_char_p, C.POINTER(SArr)]
    L.change_config.argtypes = [C.c_char_p]
    work = {work!r}
    w = configs.get("ll_pruned", end_gen=200)
    f = w.formations[0]
    init = np.array(f.initial, dtype=np.uint64)
    init.tofile(os.path.join(work, "initial"))
    np.array(f.winstates, dtype=np.uint64).tofile(os.path.join(work, "winstates"))
    os.makedirs(os.path.join(work, "b"), exist_ok=True)
    conf = os.path.join(work, "cablegen.conf")
    configs.reference_conf(conf, w, f, os.path.join(work, "b") + "/", work + "/", 2)
    L.change_config(conf.encode())
    assert L.cgb_set_option(b"device_mem_cap_mb", 1) == 0
    si = SArr(True, init.ctypes.data_as(C.POINTER(C.c_uint64)), len(init))
    L.generate(f.start, 200, (os.path.join(work, "b") + "/%d.boards").encode(), C.byref(si))
    print("generate returned")
""")


def test_capped_allocator_generate_exits_with_failure(tmp_path):
    env = dict(os.environ, XDG_CONFIG_HOME=str(tmp_path))
    r = subprocess.run([sys.executable, "-c", CHILD.format(root=ROOT, work=str(tmp_path))], env=env,
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 1, (r.returncode, r.stdout[-2000:], r.stderr[-2000:])
    assert "generate returned" not in r.stdout
    assert "[ERROR] generate:" in r.stdout and "over the cap" in r.stdout
