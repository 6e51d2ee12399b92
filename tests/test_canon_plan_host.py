"""Canonical forms from a subset of the images (board.cuh: CanonPlan, canon_cand), compiled
for the host: for the formations of the workloads, every orientation of their 0xf cells, every
move view and random tiles in the other cells, the maximum over the plan's images equals the
maximum over all eight (the reference's canonicalize_b, src/board.c:314-337); and the plans
of the workloads' formations need two images or fewer where the 0xf cells reach a corner."""
import os
import shutil
import subprocess

import pytest

from helpers import ROOT


def cellmask(cells):
    return sum(1 << c for c in cells)


FORMATIONS = {
    "LL": (10, 11, 14, 15),
    "2x4": tuple(range(8, 16)),
    "DPDF": (2, 3, 6, 7, 10, 11),
    "corner": (15,),
    "centre": (5, 6, 9, 10),       # no 0xf cell on the border: all eight images stay
    "diagonal": (0, 5, 10, 15),
    "row": (12, 13, 14, 15),
    "L3": (0, 1, 4),
}


@pytest.fixture(scope="module")
def checker(tmp_path_factory):
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(nvcc):
        pytest.skip("nvcc not found")
    out = str(tmp_path_factory.mktemp("host") / "canon_check")
    subprocess.run([nvcc, "-std=c++17", "-O2", os.path.join(ROOT, "tests", "host", "canon_check.cu"), "-o", out],
                   check=True, capture_output=True)
    return out


def test_plans_give_the_canonical_form(checker):
    args = [f"{cellmask(c):04x}" for c in FORMATIONS.values()]
    r = subprocess.run([checker] + args, capture_output=True, text=True, check=True)
    rows = {}
    for line, name in zip(r.stdout.strip().split("\n"), FORMATIONS):
        f = line.split()
        rows[name] = (int(f[1]), int(f[2]), [int(x) for x in f[3:]])
    for name, (checked, bad, per_view) in rows.items():
        assert checked == 8 * 20000 * 4 and bad == 0, (name, checked, bad)
    for name in ("LL", "2x4", "DPDF", "row"):
        assert max(rows[name][2]) <= 2, (name, rows[name][2])
    assert rows["centre"][2] == [8, 8, 8, 8]
