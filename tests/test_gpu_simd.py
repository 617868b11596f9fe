"""SIMDShockHash<l, rot> on the device (include/SIMDShockHash.hpp): the class the reference's SIMD
benchmark builds as its ShockHash<l>. Same tree, memo tables and leaf searches as ShockHash<l, rot>,
with its own split hash (remixAndRemap, SIMDShockHash.hpp:762-766) and start seeds. Every product is
compared bit for bit with the golden fixtures the reference made (tests/golden/simd*.npz) and with
the C++ restatement (variant 5) on random inputs."""
import glob
import os

import numpy as np
import pytest

import shockhash_b200 as shg
from conftest import rand_u64, unique_u64

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
SIMD_FIXTURES = sorted(os.path.basename(p)[:-4] for p in glob.glob(os.path.join(GOLDEN, "simd*.npz")))


def load(name):
    return np.load(os.path.join(GOLDEN, name + ".npz"))


def assert_products(r, want):
    assert np.array_equal(r.bucket_size_acc, want["size_acc"])
    assert np.array_equal(r.bucket_pos_acc, want["pos_acc"])
    assert np.array_equal(r.descriptors, want["desc"])
    assert np.array_equal(r.ribbon_keys, want["ribbon_keys"])
    assert np.array_equal(r.ribbon_bits, want["ribbon_bits"])


@pytest.mark.parametrize("name", SIMD_FIXTURES)
def test_simd_build_matches_golden(engine, name):
    g = load(name)
    variant = int(g["variant"])
    assert variant in (shg.SIMDSHOCKHASH, shg.SIMDSHOCKHASH_ROTATION)
    r = engine.build_hash128(variant, int(g["leaf"]), g["first"], g["second"], int(g["bucket_size"]), query=True)
    assert_products(r, g)
    assert np.array_equal(r._mphf.query_hash(g["first"], g["second"]), g["query"])
    assert np.array_equal(shg.DeviceMphf(r).query_hash(g["first"], g["second"]), g["query"])
    assert r._mphf.bits() == int(g["bits"])


@pytest.mark.parametrize("mode", [shg.MODE_LEVELS, shg.MODE_PER_LEAF, shg.MODE_PIPELINED, shg.MODE_QUEUE])
def test_simd_schedules_identical(engine, mode):
    for name in ("simd_l30_b2000", "simdrot_l40_b2000"):
        g = load(name)
        r = engine.build_hash128(int(g["variant"]), int(g["leaf"]), g["first"], g["second"], int(g["bucket_size"]),
                                 mode=mode)
        assert_products(r, g)


@pytest.mark.parametrize("leaf,n,b", [(8, 60_000, 100), (24, 60_000, 700), (30, 60_000, 2000), (40, 20_000, 2000),
                                      (2, 5_000, 9), (60, 300, 500)])
def test_simd_random_builds_match_port(engine, port, leaf, n, b):
    rng = np.random.default_rng(3 * n + leaf)
    f, s = rand_u64(rng, n), unique_u64(rng, n)
    p = port.build_hash(shg.SIMDSHOCKHASH, leaf, f, s, b)
    r = engine.build_hash128(shg.SIMDSHOCKHASH, leaf, f, s, b, query=True)
    assert_products(r, {"size_acc": p.size_acc, "pos_acc": p.pos_acc, "desc": p.desc, "ribbon_keys": p.ribbon_keys,
                        "ribbon_bits": p.ribbon_bits})
    assert np.array_equal(r._mphf.query_hash(f, s), p.query_hash(f, s))


def test_simd_strings_path_matches_port(engine, port):
    # the string constructor (SIMDShockHash.hpp:138-164): SpookyHash V2 fingerprints, then the build
    rng = np.random.default_rng(71)
    keys = list(dict.fromkeys(bytes(rng.integers(33, 127, size=int(rng.integers(16, 41)), dtype=np.uint8))
                              for _ in range(30_000)))
    f, s = port.spooky128(keys)
    p = port.build_hash(shg.SIMDSHOCKHASH, 30, f, s, 2000)
    r = engine.build_strings(shg.SIMDSHOCKHASH, 30, keys, 2000, query=True)
    assert np.array_equal(r.descriptors, p.desc) and np.array_equal(r.ribbon_bits, p.ribbon_bits)
    h = shg.SIMDShockHash[30](keys, 2000)
    got = h.query_many(keys)
    assert np.array_equal(np.sort(got), np.arange(len(keys), dtype=np.uint64))
    assert h(keys[17]) == int(got[17])


@pytest.mark.parametrize("variant,leaf", [(shg.SIMDSHOCKHASH, 30), (shg.SIMDSHOCKHASH_ROTATION, 30),
                                          (shg.SIMDSHOCKHASH, 40), (shg.SIMDSHOCKHASH_ROTATION, 48)])
def test_simd_at_scale_is_mphf(engine, variant, leaf):
    keys = unique_u64(np.random.default_rng(leaf + variant), 2_000_000)
    r = engine.build_u64(variant, leaf, keys, 2000, query=True)
    out = shg.DeviceMphf(r).query_u64(keys)
    assert np.array_equal(np.sort(out), np.arange(len(keys), dtype=np.uint64))
    idx = np.random.default_rng(3).choice(len(keys), 5000, replace=False)
    assert np.array_equal(r._mphf.query_strings([int(k).to_bytes(8, "little") for k in keys[idx]]), out[idx])


def test_simd_differs_from_shockhash_on_the_same_keys(engine):
    g = load("simd_l30_b2000")
    a = engine.build_hash128(shg.SHOCKHASH, 30, g["first"], g["second"], 2000)
    assert np.array_equal(a.bucket_size_acc, g["size_acc"])
    assert not np.array_equal(a.descriptors, g["desc"])
