"""Whole-sweep parity of the precision and large-table workloads: every layer and every FP64
table of the run hashes to the digest of the file the reference CLI itself wrote
(tests/golden/<workload>/digests.json, made by tests/golden/make_golden.py run).

* dpdf      -- DPDF-style formation, 6 fixed cells, prune 58/5/6, 512 goal, tile sums
               296..1200 (453 layers, 4.70e8 boards): the precision workload.
* ll_large  -- LL formation with free_formation (0xf cells move, src/board.c:29-38) and
               nox 10 (a board holding tile 1024 wins, src/solve.c:233-235), prune 64/6/6,
               tile sums 16..70 (28 layers, 2.18e9 boards; layers up to 3.2e8 boards run as
               sliced sort steps): the large-table workload up to the end the reference CLI
               finishes in reasonable time.
"""
import pytest

from cablegen_b200 import configs
from helpers import digests, sweep_digests

pytestmark = pytest.mark.gpu


def _check(cuda, workload, tag, **kw):
    want = digests(tag)
    w = configs.get(workload, end_gen=want["end_gen"])
    f = w.formations[0]
    assert f.start == want["start"]
    cuda.set_rules(w.settings)
    layers, tables, st = sweep_digests(cuda, f, **kw)
    want = want["layers"]
    assert st["boards_generated"] == sum(r["boards"] for r in want.values())
    bad_layers = [s for s, r in want.items() if layers.get(int(s)) != r["boards_sha256"]]
    bad_tables = [s for s, r in want.items() if tables.get(int(s)) != r["tables_sha256"]]
    assert not bad_layers, bad_layers[:10]
    assert not bad_tables, bad_tables[:10]
    return st


def test_dpdf_full_bit_exact(cuda):
    _check(cuda, "dpdf", "dpdf")


def test_ll_large_prefix_bit_exact(cuda):
    st = _check(cuda, "ll_large", "ll_large_end70")
    assert st["layers"] == 28


def test_free_formation_nox_bit_exact(cuda):
    _check(cuda, "free_2x4_nox", "free_2x4_nox")
