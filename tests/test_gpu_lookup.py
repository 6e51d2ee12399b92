"""cgb_lookup_batch: many boards looked up in one solved layer through the engine's index, equal
to lookup()'s contract (src/solve.c:108-164: the value of the key, 0.0 when absent; the key
canonicalised first when asked), for every index kind and both precisions."""
import os
import sys

import numpy as np
import pytest
import torch

from cablegen_b200 import configs

sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle"))

pytestmark = pytest.mark.gpu


def expected(keys, vals, boards):
    idx = np.searchsorted(keys, boards)
    idx_c = np.minimum(idx, len(keys) - 1)
    hit = (idx < len(keys)) & (keys[idx_c] == boards)
    return np.where(hit, vals[idx_c].astype(np.float64), 0.0)


@pytest.fixture(params=[0, 1, 2], ids=["bisect", "bucket", "hash"])
def index_kind(cuda, request):
    old = cuda.get_option("index")
    cuda.set_option("index", request.param)
    yield request.param
    cuda.set_option("index", old)


@pytest.mark.parametrize("precision", [64, 32])
def test_lookup_batch_random_keys(cuda, index_kind, precision):
    rng = np.random.default_rng(11 * index_kind + precision)
    keys = np.unique(rng.integers(1, 1 << 63, size=300_000, dtype=np.uint64))
    vals = rng.random(len(keys)).astype(np.float64 if precision == 64 else np.float32)
    boards = np.concatenate([keys[rng.integers(0, len(keys), size=50_000)],
                             rng.integers(1, 1 << 63, size=50_000, dtype=np.uint64)])
    rng.shuffle(boards)
    got = cuda.lookup_batch(cuda.to_device(keys), torch.from_numpy(vals).cuda(), cuda.to_device(boards))
    assert np.array_equal(got.cpu().numpy(), expected(keys, vals, boards))


@pytest.mark.parametrize("precision", [64, 32])
def test_lookup_batch_layer_keys_canonicalised(cuda, index_kind, precision):
    """A real layer (its keys share the formation's 0xf bytes, so FP32 tables take the 8-byte
    slots), looked up through symmetric images of its boards with canonicalisation."""
    import py_oracle as O
    w = configs.get("ll_pruned", end_gen=120)
    f = w.formations[0]
    cuda.set_rules(w.settings)
    layers, _ = cuda.generate(f.initial, f.start, f.end_gen)
    keys = max(layers.values(), key=len)
    rng = np.random.default_rng(5 + index_kind + precision)
    vals = rng.random(len(keys)).astype(np.float64 if precision == 64 else np.float32)
    pick = keys[rng.integers(0, len(keys), size=20_000)]
    L = O.lib()
    images = np.array([L.orc_flip(int(b)) if i % 2 else L.orc_rot_cw(int(b)) for i, b in enumerate(pick)],
                      dtype=np.uint64)
    strangers = rng.integers(1, 1 << 63, size=5_000, dtype=np.uint64)
    boards = np.concatenate([images, strangers])
    canon = np.array([L.orc_canon(int(b)) for b in boards], dtype=np.uint64)
    got = cuda.lookup_batch(cuda.to_device(keys), torch.from_numpy(vals).cuda(), cuda.to_device(boards),
                            canonicalize=True)
    want = expected(keys, vals, canon)
    assert np.array_equal(got.cpu().numpy(), want)
    assert np.count_nonzero(want[:len(images)]) == len(images)  # every image found its board
    # without canonicalisation the images are looked up as they are
    plain = cuda.lookup_batch(cuda.to_device(keys), torch.from_numpy(vals).cuda(), cuda.to_device(boards))
    assert np.array_equal(plain.cpu().numpy(), expected(keys, vals, boards))
