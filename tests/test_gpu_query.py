"""Device query (shg_dmphf_*): operator() on the GPU for many keys per call, against the golden
query outputs of the reference and against the host query, key for key (runs on a B200)."""
import glob
import os

import numpy as np
import pytest

import shockhash_b200 as shg
from conftest import rand_u64, unique_u64

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
BUILD_FIXTURES = sorted(os.path.basename(p)[:-4] for p in glob.glob(os.path.join(GOLDEN, "sh*_*.npz"))
                        if "leaves" not in p)


@pytest.mark.parametrize("name", BUILD_FIXTURES)
def test_device_query_matches_golden(engine, name):
    g = np.load(os.path.join(GOLDEN, name + ".npz"))
    r = engine.build_hash128(int(g["variant"]), int(g["leaf"]), g["first"], g["second"], int(g["bucket_size"]))
    dq = shg.DeviceMphf(r)
    r.free()
    assert np.array_equal(dq.query_hash(g["first"], g["second"]), g["query"])
    assert dq.bits() == int(g["bits"])
    assert dq.size() == len(g["first"])


def test_device_query_readme_strings():
    g = np.load(os.path.join(GOLDEN, "strings.npz"))
    h = shg.ShockHash[30](["abc", "def", "123", "456"], 2000)
    dq = shg.DeviceMphf(h.result)
    assert list(dq.query_strings(["abc", "def", "123", "456"])) == list(g["readme_out"]) == [1, 3, 2, 0]


@pytest.mark.parametrize("variant,leaf,n", [(2, 64, 2_000_000), (1, 30, 500_000), (2, 100, 300_000), (1, 8, 200_000)])
def test_device_query_is_mphf_and_equals_host(engine, variant, leaf, n):
    keys = unique_u64(np.random.default_rng(600 + leaf), n)
    r = engine.build_u64(variant, leaf, keys, 2000, query=True)
    dq = shg.DeviceMphf(r)
    out = dq.query_u64(keys)
    assert np.array_equal(np.sort(out), np.arange(n, dtype=np.uint64))
    # host query on a sample, through the string path (the 8-byte little-endian encoding)
    idx = np.random.default_rng(1).choice(n, 20000, replace=False)
    sample = [int(k).to_bytes(8, "little") for k in keys[idx]]
    assert np.array_equal(r._mphf.query_strings(sample), out[idx])
    assert np.array_equal(dq.query_strings(sample), out[idx])


def test_device_query_foreign_keys_equal_host(engine):
    keys = unique_u64(np.random.default_rng(71), 100_000)
    r = engine.build_u64(2, 64, keys, 2000, query=True)
    dq = shg.DeviceMphf(r)
    rng = np.random.default_rng(72)
    first, second = rand_u64(rng, 50_000), rand_u64(rng, 50_000)
    assert np.array_equal(dq.query_hash(first, second), r._mphf.query_hash(first, second))
    assert np.array_equal(dq.query_hash(first[:0], second[:0]), np.zeros(0, np.uint64))


FLATS = sorted(os.path.basename(p)[:-4] for p in glob.glob(os.path.join(GOLDEN, "flat_k*.npz")))


def _flat_keys(g):
    data = g["data"].tobytes()
    offs = np.concatenate([[0], np.cumsum(g["lengths"])]).astype(np.int64)
    return [data[offs[i]:offs[i + 1]] for i in range(len(offs) - 1)]


@pytest.mark.parametrize("name", FLATS)
def test_device_flat_query_matches_golden(engine, name):
    g = np.load(os.path.join(GOLDEN, name + ".npz"))
    keys = _flat_keys(g)
    r = engine.build_flat_strings(int(g["k"]), keys)
    dq = r.device_query()
    assert np.array_equal(dq.query_strings(keys), g["query"])
    # foreign hashes reach the fallback PHF path too; device and host agree on them
    mhc = np.random.default_rng(5).integers(0, 2**64, size=20000, dtype=np.uint64)
    assert np.array_equal(dq.query_hash(mhc), r.query_hash(mhc))


def test_device_flat_query_at_scale(engine):
    rng = np.random.default_rng(19)
    n = 300_007
    raw = rng.integers(0, 2**64, size=n, dtype=np.uint64)
    keys = [int(x).to_bytes(8, "little") + b"#" + int(i).to_bytes(3, "little") for i, x in enumerate(raw)]
    r = engine.build_flat_strings(100, keys)
    q = r.device_query().query_strings(keys)
    assert np.array_equal(np.sort(q), np.arange(n, dtype=np.uint64))
    idx = rng.choice(n, 5000, replace=False)
    assert np.array_equal(r.query_strings([keys[i] for i in idx]), q[idx])


def test_saved_result_queries_on_device(engine, tmp_path):
    keys = unique_u64(np.random.default_rng(90), 200_000)
    r = engine.build_u64(2, 64, keys, 2000)
    path = str(tmp_path / "build.shg")
    r.save(path)
    back = shg.load_result(path)
    assert np.array_equal(shg.DeviceMphf(back).query_u64(keys), shg.DeviceMphf(r).query_u64(keys))
    assert np.array_equal(back.descriptors, r.descriptors)
