"""The engine's board algebra compiled for the host (nvcc, no GPU): prune_board and its
table-driven form prune_by_table against the oracle's restatement of prune_board
(src/generate.c:98-131) on random boards, for the parameter sets of the workloads and the edge
values of smallest_large."""
import os
import shutil
import subprocess

import numpy as np
import pytest

import py_oracle as O
from helpers import ROOT, realistic_boards

PARAMS = [(58, 5, 6), (64, 6, 6), (200, 5, 6), (0, 0, 0), (10, 2, 3), (58, 5, 13), (58, 5, 14),
          (58, 5, -1), (1000, 16, 1), (30, 3, 8)]


@pytest.fixture(scope="module")
def checker(tmp_path_factory):
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(nvcc):
        pytest.skip("nvcc not found")
    out = str(tmp_path_factory.mktemp("host") / "board_check")
    subprocess.run([nvcc, "-std=c++17", "-O2", os.path.join(ROOT, "tests", "host", "board_check.cu"), "-o", out],
                   check=True, capture_output=True)
    return out


def test_prune_matches_oracle(checker, tmp_path):
    rng = np.random.default_rng(17)
    boards = np.concatenate([
        realistic_boards(rng, 20000, max_exp=13, p_empty=0.2),
        realistic_boards(rng, 20000, formation_cells=(), max_exp=8, p_empty=0.1),
        # many copies of one value (the smallest_large allowance and the third-copy rule)
        np.array([int("".join(rng.choice(list("6677889"), 16)), 16) for _ in range(5000)], dtype=np.uint64),
        np.array([0, 0x1111111111111111, 0x6666666666666666, 0xDDDDDDDDDDDDDDDD, 0xFFFFFFFFFFFFFFFF],
                 dtype=np.uint64),
    ])
    path = tmp_path / "boards.u64"
    boards.tofile(path)
    r = subprocess.run([checker, str(path)] + [f"{a},{b},{c}" for a, b, c in PARAMS], capture_output=True,
                       check=True)
    got = np.frombuffer(r.stdout, dtype=np.uint8).reshape(len(PARAMS), len(boards))
    L = O.lib()
    for i, (stsl, ltc, sl) in enumerate(PARAMS):
        want = np.array([L.orc_prune(int(b), stsl, ltc, sl) != 0 for b in boards], dtype=np.uint8)
        for form, bit in (("per-cell", 0), ("table", 1)):
            bad = np.nonzero(((got[i] >> bit) & 1) != want)[0]
            assert len(bad) == 0, (form, stsl, ltc, sl, [hex(int(boards[j])) for j in bad[:5]])
