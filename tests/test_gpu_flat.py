"""ShockHash2Flat<k> on the device vs the reference (golden fixtures from the compiled reference)."""
import glob
import os

import numpy as np
import pytest

import shockhash_b200 as shg

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
FLATS = sorted(os.path.basename(p)[:-4] for p in glob.glob(os.path.join(GOLDEN, "flat_k*.npz")))


def keys_of(g):
    data = g["data"].tobytes()
    offs = np.concatenate([[0], np.cumsum(g["lengths"])]).astype(np.int64)
    return [data[offs[i]:offs[i + 1]] for i in range(len(offs) - 1)]


@pytest.mark.parametrize("name", FLATS)
def test_flat_matches_golden(engine, name):
    g = np.load(os.path.join(GOLDEN, name + ".npz"))
    keys = keys_of(g)
    r = engine.build_flat_strings(int(g["k"]), keys)
    assert r.layers == int(g["layers"])
    assert np.array_equal(r.layer_bases, g["layer_bases"])
    assert np.array_equal(r.free_positions, g["free_positions"])
    assert np.array_equal(r.fallback_seed_buckets, g["fallback_buckets"])
    assert np.array_equal(r.fallback_seeds, g["fallback_seeds"])
    assert np.array_equal(r.thresholds_and_seeds, g["thresholds_and_seeds"])
    assert np.array_equal(r.ribbon_keys, g["ribbon_keys"])
    assert np.array_equal(r.ribbon_bits, g["ribbon_bits"])
    assert np.array_equal(r.query_strings(keys), g["query"])
    assert r.bits() == int(g["bits"])


def test_flat_is_a_minimal_perfect_hash_at_scale(engine):
    rng = np.random.default_rng(17)
    n = 400_003
    raw = rng.integers(0, 2**64, size=n, dtype=np.uint64)
    keys = [int(x).to_bytes(8, "little") + b"-" + int(i).to_bytes(3, "little") for i, x in enumerate(raw)]
    r = engine.build_flat_strings(100, keys)
    q = r.query_strings(keys)
    assert np.array_equal(np.sort(q), np.arange(n, dtype=np.uint64))


def test_flat_python_class():
    keys = [f"key-{i}" for i in range(5000)]
    h = shg.ShockHash2Flat[32](keys, 0, 0)
    vals = sorted(h(k) for k in keys)
    assert vals == list(range(5000))
