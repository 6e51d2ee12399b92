"""Full-size parity: the LL pruned workload (tile sums 16..600, 4.97e9 boards) generated and
solved in FP64 on one B200; every one of the 293 layers and tables must hash to the digest of
the file the reference itself wrote (tests/golden/ll_pruned/digests.json)."""
import ctypes as C
import hashlib
import os
import threading
from concurrent.futures import ThreadPoolExecutor

import pytest

from cablegen_b200 import configs
from helpers import digests

pytestmark = pytest.mark.gpu


def test_ll_pruned_full_bit_exact(cuda):
    w = configs.get("ll_pruned")
    f = w.formations[0]
    cuda.set_rules(w.settings)
    want = digests("ll_pruned")["layers"]
    workers = max(2, min(16, (os.cpu_count() or 4) - 1))
    pool = ThreadPoolExecutor(max_workers=workers)
    gate = threading.Semaphore(2 * workers)   # bound the bytes waiting to be hashed
    got_layers, got_tables, futures = {}, {}, []

    def digest(store, key, parts):
        try:
            h = hashlib.sha256()
            for p in parts:
                h.update(p)
            store[key] = h.hexdigest()
        finally:
            gate.release()

    def on_layer(s, ptr, n):
        gate.acquire()
        data = C.string_at(ptr, 8 * n) if n else b""
        futures.append(pool.submit(digest, got_layers, s, [data]))

    def on_table(s, kptr, vptr, n, prec):
        assert prec == 64
        gate.acquire()
        keys = C.string_at(kptr, 8 * n) if n else b""
        vals = C.string_at(vptr, 8 * n) if n else b""
        futures.append(pool.submit(digest, got_tables, s, [keys, vals]))

    _, _, st = cuda.tablebase(f.initial, f.start, f.end_gen, f.start, f.winstates, precision=64,
                              layer_fn=on_layer, table_fn=on_table)
    for fu in futures:
        fu.result()
    pool.shutdown()
    assert st["boards_generated"] == sum(r["boards"] for r in want.values())
    bad_layers = [s for s, r in want.items() if got_layers.get(int(s)) != r["boards_sha256"]]
    bad_tables = [s for s, r in want.items() if got_tables.get(int(s)) != r["tables_sha256"]]
    assert not bad_layers, bad_layers[:10]
    assert not bad_tables, bad_tables[:10]
