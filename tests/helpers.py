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
