"""CUDA path vs the oracle: bit-exact products on the same seeded inputs (runs on a B200)."""
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
MODES = [shg.MODE_DEFAULT, shg.MODE_LEVELS]


def load(name):
    return np.load(os.path.join(GOLDEN, name + ".npz"))


def assert_same(r, g):
    assert np.array_equal(r.bucket_size_acc, g["size_acc"])
    assert np.array_equal(r.bucket_pos_acc, g["pos_acc"])
    assert np.array_equal(r.descriptors, g["desc"])
    assert np.array_equal(r.ribbon_keys, g["ribbon_keys"])
    assert np.array_equal(r.ribbon_bits, g["ribbon_bits"])


@pytest.mark.parametrize("name", BUILD_FIXTURES)
def test_build_matches_golden(engine, name):
    g = load(name)
    r = engine.build_hash128(int(g["variant"]), int(g["leaf"]), g["first"], g["second"], int(g["bucket_size"]),
                             query=True)
    assert_same(r, g)
    assert np.array_equal(r._mphf.query_hash(g["first"], g["second"]), g["query"])
    assert r._mphf.bits() == int(g["bits"])


def test_modes_identical(engine):
    g = load("sh2_l64_b2000")
    outs = [engine.build_hash128(2, 64, g["first"], g["second"], 2000, mode=m) for m in
            (shg.MODE_DEFAULT, shg.MODE_LEVELS, shg.MODE_PER_LEAF, shg.MODE_PIPELINED, shg.MODE_QUEUE)]
    for r in outs:
        assert_same(r, g)
    g = load("sh1_l30_b2000")
    for m in (shg.MODE_PER_LEAF, shg.MODE_LEVELS, shg.MODE_PIPELINED):
        assert_same(engine.build_hash128(1, 30, g["first"], g["second"], 2000, mode=m), g)


def test_pipelined_chunk_counts_identical(port):
    # the bucket chunking of the pipelined schedule must not change any product
    rng = np.random.default_rng(21)
    n = 30000
    f, s = rand_u64(rng, n), unique_u64(rng, n)
    p = port.build_hash(2, 24, f, s, 700)
    for chunks in ("1", "3", "64"):
        os.environ["SHG_PIPE_CHUNKS"] = chunks
        try:
            eng = shg.Engine(0)
        finally:
            del os.environ["SHG_PIPE_CHUNKS"]
        r = eng.build_hash128(2, 24, f, s, 700, mode=shg.MODE_PIPELINED)
        assert np.array_equal(r.descriptors, p.desc) and np.array_equal(r.ribbon_bits, p.ribbon_bits), chunks
        r.free()
        eng.close()


def test_sh2_leaves_match_golden(engine):
    g = load("sh2_leaves")
    seeds, bits = engine.sh2_construct_leaves(g["keys"], g["offsets"])
    assert np.array_equal(seeds, g["seeds"])
    assert np.array_equal(bits, g["bits"])


def test_sh1_leaves_match_golden(engine):
    g = load("sh1_leaves")
    offs, lv = g["offsets"], g["levels"]
    for level in (0, 1, 2):
        idx = np.nonzero(lv == level)[0]
        keys = np.concatenate([g["keys"][offs[j]:offs[j + 1]] for j in idx])
        sub = np.concatenate([[0], np.cumsum([offs[j + 1] - offs[j] for j in idx])]).astype(np.uint64)
        codes, kc, bits = engine.sh1_construct_leaves(keys, sub, level)
        assert np.array_equal(codes, g["codes"][idx])
        assert np.array_equal(kc, np.concatenate([g["keys_by_cell"][offs[j]:offs[j + 1]] for j in idx]))
        assert np.array_equal(bits, np.concatenate([g["bits"][offs[j]:offs[j + 1]] for j in idx]))


def test_string_hashing_matches_golden(engine):
    g = load("strings")
    data = g["data"].tobytes()
    offs = np.concatenate([[0], np.cumsum(g["lengths"])]).astype(np.uint64)
    keys = [data[offs[i]:offs[i + 1]] for i in range(len(offs) - 1)]
    f, s = engine.hash_strings(keys)
    bad = np.nonzero((f != g["first"]) | (s != g["second"]))[0]
    assert len(bad) == 0, f"lengths that differ: {g['lengths'][bad].tolist()}"


def test_readme_vector():
    keys = ["abc", "def", "123", "456"]
    h = shg.ShockHash[30](keys, 2000)
    assert [h(k) for k in keys] == [1, 3, 2, 0]


@pytest.mark.parametrize("variant,leaf,n,b", [(2, 64, 60000, 2000), (1, 30, 40000, 2000), (2, 24, 20000, 100),
                                              (1, 16, 20000, 64), (2, 128, 1500, 600), (1, 60, 2500, 900),
                                              (2, 2, 400, 3), (1, 3, 400, 5), (2, 11, 7, 2000), (1, 7, 1, 10)])
def test_build_matches_port_random(engine, port, variant, leaf, n, b):
    rng = np.random.default_rng(n * 7 + leaf)
    f, s = rand_u64(rng, n), unique_u64(rng, n)
    p = port.build_hash(variant, leaf, f, s, b)
    r = engine.build_hash128(variant, leaf, f, s, b)
    assert np.array_equal(r.bucket_size_acc, p.size_acc) and np.array_equal(r.bucket_pos_acc, p.pos_acc)
    assert np.array_equal(r.descriptors, p.desc)
    assert np.array_equal(r.ribbon_keys, p.ribbon_keys) and np.array_equal(r.ribbon_bits, p.ribbon_bits)


def test_u64_keys_match_strings_path(engine, port):
    rng = np.random.default_rng(77)
    keys = unique_u64(rng, 20000)
    r1 = engine.build_u64(2, 64, keys, 2000)
    strs = [int(k).to_bytes(8, "little") for k in keys]
    r2 = engine.build_strings(2, 64, strs, 2000)
    assert np.array_equal(r1.descriptors, r2.descriptors)
    f, s = port.spooky128(strs)
    p = port.build_hash(2, 64, f, s, 2000)
    assert np.array_equal(r1.descriptors, p.desc) and np.array_equal(r1.ribbon_bits, p.ribbon_bits)


def test_large_build_is_a_minimal_perfect_hash(engine):
    # Full-size property check: 2M keys, every key maps to a distinct value in [0, n).
    rng = np.random.default_rng(5)
    n = 2_000_000
    keys = unique_u64(rng, n)
    r = engine.build_u64(2, 64, keys, 2000, query=True)
    strs_f, strs_s = engine.hash_strings([int(k).to_bytes(8, "little") for k in keys[:1000]])
    q = r._mphf.query_hash(strs_f, strs_s)
    assert len(np.unique(q)) == 1000 and q.max() < n
    # all keys, through the 128-bit path
    first = np.empty(n, np.uint64)
    second = np.empty(n, np.uint64)
    step = 200000
    for i in range(0, n, step):
        a, b = engine.hash_strings([int(k).to_bytes(8, "little") for k in keys[i:i + step]])
        first[i:i + step], second[i:i + step] = a, b
    q = r._mphf.query_hash(first, second)
    assert np.array_equal(np.sort(q), np.arange(n, dtype=np.uint64))


def test_trial_cap_reports_error_and_engine_recovers(engine):
    # A trial cap below the answer turns a search into SHG_ERR_TRIAL_LIMIT (the reference has no cap
    # and would keep searching); the engine must stay usable afterwards.
    g = load("sh2_l10_b100")
    with pytest.raises(shg.ShgError) as ei:
        engine.build_hash128(1, 8, g["first"], g["second"], 100, max_trials=1)
    assert ei.value.status == 3
    assert_same(engine.build_hash128(2, 10, g["first"], g["second"], 100), g)


def test_duplicate_keys_match_oracle(engine, port):
    # Equal keys form a double edge (a 2-cycle), which a pseudoforest admits; the reference then
    # builds a structure that maps both copies to one value. The device must build the same one.
    rng = np.random.default_rng(3)
    f, s = rand_u64(rng, 3000), unique_u64(rng, 3000)
    s[10], f[10] = s[11], f[11]
    for variant, leaf in ((1, 8), (2, 12)):
        p = port.build_hash(variant, leaf, f, s, 100)
        r = engine.build_hash128(variant, leaf, f, s, 100)
        assert np.array_equal(r.descriptors, p.desc) and np.array_equal(r.ribbon_bits, p.ribbon_bits)


@pytest.mark.parametrize("variant,leaf", [(1, 30), (2, 64)])
def test_empty_key_set_matches_oracle(engine, port, variant, leaf):
    # no keys: one empty bucket, a descriptor stream holding only the sentinel (ShockHash.h:616-654)
    f = np.zeros(0, np.uint64)
    p = port.build_hash(variant, leaf, f, f, 2000)
    r = engine.build_hash128(variant, leaf, f, f, 2000)
    assert r.n == 0 and r.nbuckets == 1
    assert np.array_equal(r.bucket_size_acc, p.size_acc) and np.array_equal(r.bucket_pos_acc, p.pos_acc)
    assert np.array_equal(r.descriptors, p.desc) and len(r.ribbon_keys) == 0


def test_oversized_bucket_is_an_error(engine):
    # a bucket of >= 3000 keys exceeds MAX_BUCKET_SIZE (ShockHash.h:33); the reference's memo tables
    # stop there, so the engine refuses instead of reading past them, and stays usable
    rng = np.random.default_rng(8)
    n = 6000
    f = np.full(n, 12345, np.uint64)  # every key in the same bucket
    s = unique_u64(rng, n)
    with pytest.raises(shg.ShgError) as ei:
        engine.build_hash128(2, 64, f, s, 6000)
    assert ei.value.status == 5
    g = load("sh2_l10_b100")
    assert_same(engine.build_hash128(2, 10, g["first"], g["second"], 100), g)


ROT_FIXTURES = sorted(os.path.basename(p)[:-4] for p in glob.glob(os.path.join(GOLDEN, "rot_*.npz")))


@pytest.mark.parametrize("name", ROT_FIXTURES)
def test_rotation_fitting_matches_golden(engine, name):
    # ShockHash<l, true>: leaves of exactly l keys use rotation fitting (ShockHash.h:316-399)
    g = load(name)
    assert int(g["variant"]) == shg.SHOCKHASH_ROTATION
    r = engine.build_hash128(int(g["variant"]), int(g["leaf"]), g["first"], g["second"], int(g["bucket_size"]),
                             query=True)
    assert_same(r, g)
    assert np.array_equal(r._mphf.query_hash(g["first"], g["second"]), g["query"])
    assert np.array_equal(shg.DeviceMphf(r).query_hash(g["first"], g["second"]), g["query"])
    assert r._mphf.bits() == int(g["bits"])


@pytest.mark.parametrize("leaf", [30, 40])
def test_rotation_fitting_at_scale_is_mphf(engine, leaf):
    keys = unique_u64(np.random.default_rng(leaf + 900), 1_000_000)
    r = engine.build_u64(shg.SHOCKHASH_ROTATION, leaf, keys, 2000, query=True)
    out = shg.DeviceMphf(r).query_u64(keys)
    assert np.array_equal(np.sort(out), np.arange(len(keys), dtype=np.uint64))
    idx = np.random.default_rng(2).choice(len(keys), 5000, replace=False)
    assert np.array_equal(r._mphf.query_strings([int(k).to_bytes(8, "little") for k in keys[idx]]), out[idx])


@pytest.mark.parametrize("leaf,n,b", [(64, 300_000, 2000), (24, 60_000, 700), (9, 20_000, 50), (64, 3, 2000)])
def test_queue_schedule_equals_levels(engine, leaf, n, b):
    # every split node and leaf in one persistent launch gives the level schedule's products
    rng = np.random.default_rng(leaf + n)
    f, s = rand_u64(rng, n), unique_u64(rng, n)
    lv = engine.build_hash128(2, leaf, f, s, b, mode=shg.MODE_LEVELS)
    q = engine.build_hash128(2, leaf, f, s, b, mode=shg.MODE_QUEUE)
    assert_same(q, type("G", (), {"__getitem__": lambda self, k: {"size_acc": lv.bucket_size_acc,
                                                                  "pos_acc": lv.bucket_pos_acc, "desc": lv.descriptors,
                                                                  "ribbon_keys": lv.ribbon_keys,
                                                                  "ribbon_bits": lv.ribbon_bits}[k]})())
    assert q.work["split_evals"] == lv.work["split_evals"] and q.work["uf_edges"] == lv.work["uf_edges"]
