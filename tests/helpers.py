"""Shared helpers of the test suite (fixtures loading, digests)."""
import hashlib
import json
import os

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")
UNITS = os.path.join(GOLDEN, "units")


def unit(name, dtype):
    return np.fromfile(os.path.join(UNITS, name), dtype=dtype)


def digests(tag):
    with open(os.path.join(GOLDEN, tag, "digests.json")) as f:
        return json.load(f)


def sha_layer(keys) -> str:
    return hashlib.sha256(np.ascontiguousarray(keys, dtype=np.uint64).tobytes()).hexdigest()


def sha_table(keys, vals) -> str:
    """SHA-256 of a .tables file: N u64 keys then N f64 values (src/solve.c:41-42)."""
    h = hashlib.sha256()
    h.update(np.ascontiguousarray(keys, dtype=np.uint64).tobytes())
    h.update(np.ascontiguousarray(vals, dtype=np.float64).tobytes())
    return h.hexdigest()


def sweep_digests(cuda, form, precision=64):
    """Generate and solve one formation (tile sums start..end_gen, solve down to start) and
    return ({sum: SHA-256 of the layer file}, {sum: SHA-256 of the table file}, stats): the
    digests the reference's .boards and .tables files would have.  Layers and tables reach
    the host through the sweep's callbacks and are hashed on a thread pool."""
    import ctypes as C
    import threading
    from concurrent.futures import ThreadPoolExecutor
    workers = max(2, min(16, (os.cpu_count() or 4) - 1))
    pool = ThreadPoolExecutor(max_workers=workers)
    gate = threading.Semaphore(2 * workers)   # bound the bytes waiting to be hashed
    got_layers, got_tables, futures = {}, {}, []

    def digest(store, key, parts):
        try:
            h = hashlib.sha256()
            for p in parts:
                mv = memoryview(p).cast("B")
                for o in range(0, len(mv), 1 << 28):   # 256 MiB at a time
                    h.update(mv[o:o + (1 << 28)])
            store[key] = h.hexdigest()
        finally:
            gate.release()

    def copy(ptr, n):
        # layers of large workloads exceed 2^31 bytes: copy through numpy, not string_at
        if not n:
            return np.zeros(0, np.uint64)
        return np.ctypeslib.as_array(C.cast(ptr, C.POINTER(C.c_uint64)), shape=(n,)).copy()

    def on_layer(s, ptr, n):
        gate.acquire()
        futures.append(pool.submit(digest, got_layers, s, [copy(ptr, n)]))

    def on_table(s, kptr, vptr, n, prec):
        assert prec == 64
        gate.acquire()
        futures.append(pool.submit(digest, got_tables, s, [copy(kptr, n), copy(vptr, n)]))

    _, _, st = cuda.tablebase(form.initial, form.start, form.end_gen, form.start, form.winstates,
                              precision=precision, layer_fn=on_layer, table_fn=on_table)
    for fu in futures:
        fu.result()
    pool.shutdown()
    return got_layers, got_tables, st


def realistic_boards(rng, n, formation_cells=(10, 11, 14, 15), max_exp=10, p_empty=0.35):
    """Random boards of a formation: 0xf fixed cells, empties and tiles."""
    cells = np.array([c for c in range(16) if c not in formation_cells])
    out = np.zeros(n, dtype=np.uint64)
    for c in formation_cells:
        out |= np.uint64(0xF) << np.uint64(60 - 4 * c)
    exps = rng.integers(1, max_exp + 1, size=(n, len(cells))).astype(np.uint64)
    empty = rng.random((n, len(cells))) < p_empty
    exps[empty] = 0
    for j, c in enumerate(cells):
        out |= exps[:, j] << np.uint64(60 - 4 * int(c))
    return out
