"""Full-size parity: the LL pruned workload (tile sums 16..600, 4.97e9 boards) generated and
solved in FP64 on one B200; every one of the 293 layers and tables must hash to the digest of
the file the reference itself wrote (tests/golden/ll_pruned/digests.json)."""
import pytest

from cablegen_b200 import configs
from helpers import digests, sweep_digests

pytestmark = pytest.mark.gpu


def test_ll_pruned_full_bit_exact(cuda):
    w = configs.get("ll_pruned")
    f = w.formations[0]
    cuda.set_rules(w.settings)
    want = digests("ll_pruned")["layers"]
    got_layers, got_tables, st = sweep_digests(cuda, f)
    assert st["boards_generated"] == sum(r["boards"] for r in want.values())
    bad_layers = [s for s, r in want.items() if got_layers.get(int(s)) != r["boards_sha256"]]
    bad_tables = [s for s, r in want.items() if got_tables.get(int(s)) != r["tables_sha256"]]
    assert not bad_layers, bad_layers[:10]
    assert not bad_tables, bad_tables[:10]
