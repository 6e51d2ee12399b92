"""Home slots of the hash lookup index compiled for the host (nvcc, no GPU): every slot
stays inside the table and keys spread over all of it, also for tables of 2^32 slots and
more (layers above ~1.9e9 boards at a 45 % load), where a 32-bit range reduction would
fold every key into the first slots."""
import os
import shutil
import subprocess

import numpy as np
import pytest

import py_oracle as O
from helpers import ROOT, realistic_boards

CAPS = [64, 1 << 20, (1 << 32) - 64, 1 << 32, (1 << 32) + 64, 1 << 33, 3 * (1 << 32) + 128, 1 << 40]


@pytest.fixture(scope="module")
def checker(tmp_path_factory):
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(nvcc):
        pytest.skip("nvcc not found")
    out = str(tmp_path_factory.mktemp("host") / "hash_check")
    subprocess.run([nvcc, "-std=c++17", "-O2", os.path.join(ROOT, "tests", "host", "hash_check.cu"), "-o", out],
                   check=True, capture_output=True)
    return out


def test_home_slots_cover_large_tables(checker, tmp_path):
    rng = np.random.default_rng(3)
    keys = np.unique(O.canon(realistic_boards(rng, 200_000)))
    path = tmp_path / "keys.u64"
    keys.tofile(path)
    r = subprocess.run([checker, str(path)] + [str(c) for c in CAPS], capture_output=True, text=True, check=True)
    rows = [tuple(int(v) for v in line.split()) for line in r.stdout.split("\n") if line.strip()]
    assert [row[0] for row in rows] == CAPS
    for cap, mx, distinct, bad in rows:
        assert bad == 0, cap
        assert mx < cap
        if cap >= (1 << 20):
            # no folding: nearly every key has its own home slot, spread over the whole table
            assert distinct >= 0.8 * len(keys), (cap, distinct)
            assert mx >= cap // 2, (cap, mx)



@pytest.fixture(scope="module")
def compact_checker(tmp_path_factory):
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(nvcc):
        pytest.skip("nvcc not found")
    out = str(tmp_path_factory.mktemp("host") / "compact_check")
    subprocess.run([nvcc, "-std=c++17", "-O2", os.path.join(ROOT, "tests", "host", "compact_check.cu"), "-o", out],
                   check=True, capture_output=True)
    return out


@pytest.mark.parametrize("const_bytes,n", [((7, 5), 3_000_000), ((7, 5, 4), 300_000), ((7, 6, 5, 4, 3), 5_000)])
def test_compact_slots_are_exact(compact_checker, tmp_path, const_bytes, n):
    """8-byte slots: every member is found with its own value, and keys that are not members
    -- neighbours differing in one nibble, other keys with the same constant bytes, keys with
    another constant byte -- never hit.  Keys share the bytes a layer's canonical boards
    share (the 0xf cells)."""
    rng = np.random.default_rng(11)
    keys = rng.integers(1, 1 << 63, 2 * n, dtype=np.uint64) * np.uint64(2) + np.uint64(1)
    for b in const_bytes:
        keys = (keys & ~np.uint64(0xFF << (8 * b))) | np.uint64(0xFF << (8 * b))
    keys = np.unique(keys)
    members = keys[: len(keys) // 2]
    others = keys[len(keys) // 2:]
    tweak = members ^ (np.uint64(1) << (np.uint64(4) * rng.integers(0, 16, len(members)).astype(np.uint64)))
    queries = np.setdiff1d(np.concatenate([others, tweak]), members)
    members.tofile(tmp_path / "m.u64")
    queries.tofile(tmp_path / "q.u64")
    r = subprocess.run([compact_checker, str(tmp_path / "m.u64"), str(tmp_path / "q.u64")], capture_output=True,
                       text=True, check=True)
    on, rbits, dbits, logcap, maxd, found, wrong, qhit = (int(x) for x in r.stdout.split())
    assert on == 1, r.stdout
    assert rbits + dbits <= 32 and (1 << logcap) >= 2 * len(members)
    assert found == len(members) and wrong == 0 and qhit == 0, r.stdout
    assert maxd < (1 << dbits) - 2
