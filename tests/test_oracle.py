"""The CPU oracle, pinned: the C++ restatement (oracle/port) and the compiled reference
(oracle/_ref) against the golden fixtures generated by the reference itself (tests/golden)."""
import glob
import hashlib
import json
import os

import numpy as np
import pytest

from conftest import rand_u64, unique_u64

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
BUILD_FIXTURES = sorted(os.path.basename(p)[:-4] for p in glob.glob(os.path.join(GOLDEN, "sh*_*.npz"))
                        if "leaves" not in p)


def load(name):
    return np.load(os.path.join(GOLDEN, name + ".npz"))


def test_manifest_hashes():
    with open(os.path.join(GOLDEN, "MANIFEST.json")) as f:
        manifest = json.load(f)
    for name, digest in manifest.items():
        with open(os.path.join(GOLDEN, name), "rb") as fh:
            assert hashlib.sha256(fh.read()).hexdigest() == digest, name


def test_readme_vector_golden():
    # README.md:42-46 — ShockHash<30,false>({"abc","def","123","456"}, 2000) maps them to 1 3 2 0.
    assert list(load("strings")["readme_out"]) == [1, 3, 2, 0]


@pytest.mark.parametrize("name", BUILD_FIXTURES)
def test_port_matches_golden(port, name):
    g = load(name)
    r = port.build_hash(int(g["variant"]), int(g["leaf"]), g["first"], g["second"], int(g["bucket_size"]))
    assert np.array_equal(r.desc, g["desc"])
    assert np.array_equal(r.size_acc, g["size_acc"])
    assert np.array_equal(r.pos_acc, g["pos_acc"])
    assert np.array_equal(r.ribbon_keys, g["ribbon_keys"])
    assert np.array_equal(r.ribbon_bits, g["ribbon_bits"])
    assert np.array_equal(r.query_hash(g["first"], g["second"]), g["query"])


def test_port_leaves_match_golden(port):
    g = load("sh2_leaves")
    offs = g["offsets"]
    for j in range(len(offs) - 1):
        k = g["keys"][offs[j]:offs[j + 1]]
        seed, rk, rb = port.sh2_leaf(k)
        assert seed == g["seeds"][j]
        assert np.array_equal(rb, g["bits"][offs[j]:offs[j + 1]])
    g = load("sh1_leaves")
    offs = g["offsets"]
    for j in range(len(offs) - 1):
        k = g["keys"][offs[j]:offs[j + 1]]
        code, rk, rb = port.sh1_leaf(k, int(g["levels"][j]))
        assert code == g["codes"][j]
        assert np.array_equal(rk, g["keys_by_cell"][offs[j]:offs[j + 1]])
        assert np.array_equal(rb, g["bits"][offs[j]:offs[j + 1]])


def test_port_spooky_matches_golden(port):
    g = load("strings")
    data = g["data"].tobytes()
    offs = np.concatenate([[0], np.cumsum(g["lengths"])]).astype(np.uint64)
    keys = [data[offs[i]:offs[i + 1]] for i in range(len(offs) - 1)]
    f, s = port.spooky128(keys)
    assert np.array_equal(f, g["first"]) and np.array_equal(s, g["second"])


def test_ref_matches_golden(ref):
    for name in ("sh2_l64_b2000", "sh1_l30_b2000", "sh2_l9_b50", "rot_l30_b2000", "rot_l40_b2000"):
        g = load(name)
        r = ref.build_hash(int(g["variant"]), int(g["leaf"]), g["first"], g["second"], int(g["bucket_size"]), 1)
        assert np.array_equal(r.desc, g["desc"])
        assert np.array_equal(r.ribbon_bits, g["ribbon_bits"])


def test_ref_readme_vector(ref):
    keys = [b"abc", b"def", b"123", b"456"]
    b = ref.build_strings(1, 30, keys, 2000, 1)
    assert list(ref.query_strings(b, keys)) == [1, 3, 2, 0]


@pytest.mark.parametrize("variant,leaf,n,b,threads", [(2, 64, 12000, 2000, 4), (1, 24, 8000, 300, 3)])
def test_ref_thread_count_invariance(ref, variant, leaf, n, b, threads):
    rng = np.random.default_rng(leaf)
    f, s = rand_u64(rng, n), unique_u64(rng, n)
    r1 = ref.build_hash(variant, leaf, f, s, b, 1)
    rt = ref.build_hash(variant, leaf, f, s, b, threads)
    assert np.array_equal(r1.desc, rt.desc) and np.array_equal(r1.pos_acc, rt.pos_acc)


@pytest.mark.parametrize("variant,leaf,n,b", [(1, 12, 4000, 150), (2, 16, 4000, 150), (2, 48, 9000, 1200),
                                              (1, 32, 6000, 900), (2, 5, 500, 9), (1, 2, 300, 4)])
def test_port_matches_ref_random(port, ref, variant, leaf, n, b):
    rng = np.random.default_rng(n + leaf)
    f, s = rand_u64(rng, n), unique_u64(rng, n)
    r = ref.build_hash(variant, leaf, f, s, b, 2)
    p = port.build_hash(variant, leaf, f, s, b)
    assert np.array_equal(p.desc, r.desc)
    assert np.array_equal(p.size_acc, r.size_acc) and np.array_equal(p.pos_acc, r.pos_acc)
    assert np.array_equal(p.ribbon_keys, r.ribbon_keys) and np.array_equal(p.ribbon_bits, r.ribbon_bits)


def test_memo_tables_port_vs_ref(port, ref):
    for variant, leaves in ((1, [2, 3, 4, 5, 6, 7, 8, 10, 12, 13, 16, 20, 24, 25, 30, 32, 33, 40, 48, 60]),
                            (2, [2, 3, 4, 5, 6, 8, 9, 10, 11, 12, 16, 20, 24, 32, 33, 40, 48, 64, 100, 128])):
        for leaf in leaves:
            assert np.array_equal(port.memo(variant, leaf), ref.memo(variant, leaf)), (variant, leaf)


def test_mphf_property_port(port):
    rng = np.random.default_rng(9)
    n = 30000
    f, s = rand_u64(rng, n), unique_u64(rng, n)
    for variant, leaf in ((1, 20), (2, 24)):
        r = port.build_hash(variant, leaf, f, s, 1000)
        q = r.query_hash(f, s)
        assert np.array_equal(np.sort(q), np.arange(n, dtype=np.uint64))


def test_ref_rotation_fitting_is_mphf_and_differs_from_plain(ref):
    # ShockHash<l, true> stores x * l + r for full leaves; its structure is a different one
    rng = np.random.default_rng(44)
    f, s = rand_u64(rng, 6000), unique_u64(rng, 6000)
    r = ref.build_hash(3, 24, f, s, 500, 1)
    assert np.array_equal(np.sort(r.query_hash(f, s)), np.arange(6000, dtype=np.uint64))
    assert not np.array_equal(r.desc, ref.build_hash(1, 24, f, s, 500, 1).desc)


def _pseudoforest(m, c1, c2):
    """Union-find with a cycle flag per root: every component has at most as many keys (edges) as
    cells (vertices)."""
    parent = list(range(m))
    cyc = [False] * m

    def root(x):
        while parent[x] != x:
            parent[x] = parent[parent[x]]
            x = parent[x]
        return x

    for a, b in zip(c1.tolist(), c2.tolist()):
        ra, rb = root(a), root(b)
        if ra == rb:
            if cyc[ra]:
                return False
            cyc[ra] = True
        else:
            if cyc[ra] and cyc[rb]:
                return False
            parent[ra] = rb
            cyc[rb] = cyc[ra] or cyc[rb]
    return True


def test_ref_cuckoo_insertion_iff_pseudoforest(ref):
    """The equivalence the leaf kernels rely on: the reference's ordered cuckoo insertion
    (TinyBinaryCuckooHashTable.h:80-106,169-198) places every key exactly when the cell graph is a
    pseudoforest, in both directions, on 10^5 random leaves of 2..60 keys and random seeds."""
    rng = np.random.default_rng(2024)
    both = {True: 0, False: 0}
    for _ in range(100_000):
        m = int(rng.integers(2, 61))
        keys = rng.integers(0, 2**64, size=m, dtype=np.uint64)
        seed = int(rng.integers(0, 2**63))
        placed, c1, c2 = ref.cuckoo_construct(keys, seed)
        assert placed == _pseudoforest(m, c1, c2), (m, seed)
        both[placed] += 1
    assert both[True] > 5_000 and both[False] > 5_000


def _covering_rows(rng, L, n):
    """n hash rows of an L-key leaf, each covering all (L + 1) / 2 values, as candidates do."""
    c = (L + 1) // 2
    out = rng.integers(0, c, size=(n, L))
    for r in out:
        r[:c] = rng.permutation(c)
        rng.shuffle(r)
    return out.astype(np.uint8)


@pytest.mark.parametrize("L", [10, 16, 33, 64, 100, 128])
def test_ref_bipartite_pair_filter_and_union_find(ref, L):
    """The bipartite pair test of the reference (ShockHash2-internal.h:510-528) on random candidate
    pairs: its CuckooUnionFind accepts exactly the pseudoforests. The isolated-vertex filter
    (:34-44, :515-517) never skips a pseudoforest for even L; for odd L the two rows share cell
    L / 2 (rows hash to (L + 1) / 2 values, the new one shifted by L / 2), a key alone in its cell
    in each row can still lie on a larger component, and the filter skips some pairs that pass.
    The filter is therefore part of the result, and the device and the restatement apply it
    exactly as the reference does rather than treating it as a pure speed-up."""
    rng = np.random.default_rng(7 + L)
    A, B = _covering_rows(rng, L, 20000), _covering_rows(rng, L, 20000)
    skipped_forests = forests = 0
    for a, b in zip(A, B):
        skipped, forest = ref.sh2_pair_check(a, b)
        assert forest == _pseudoforest(L, a.astype(np.int64) + L // 2, b.astype(np.int64))
        forests += forest
        skipped_forests += skipped and forest
    if L % 2 == 0:
        assert skipped_forests == 0
    else:
        assert skipped_forests > 0
    if L <= 64:
        assert forests > 0


def test_ref_stats_phase_times(ref):
    """The reference's own STATS timers (oracle/ref_stats.py, one thread, a subprocess because the
    STATS build prints to stdout): leaf-search and split-level totals within the constructor time."""
    import subprocess
    import sys
    helper = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle", "ref_stats.py")
    if not os.path.exists(os.path.join(os.path.dirname(helper), "_ref", "libshref_stats.so")):
        pytest.skip("STATS build of the reference oracle not available")
    out = subprocess.run([sys.executable, helper, "--n", "20000"], capture_output=True, text=True, timeout=300,
                         check=True)
    res = json.loads(out.stdout.strip().splitlines()[-1])
    assert res["keys"] == 20000 and res["threads"] == 1
    assert 0 < res["leaves_ms"] and 0 < res["splits_ms"]
    assert res["leaves_ms"] + res["splits_ms"] <= res["total_ms"] * 1.02


def test_elegant_pairing_of_raw_seeds_is_float_accurate():
    # The bipartite leaf kernel skips isFloatAccurateElegant (PairingFunction.h:93-96) for raw seeds
    # below 2^24, where unpairing with an IEEE double square root is always exact: checked here
    # exhaustively below 2^11, around every power of two, and on random pairs below 2^24.
    def accurate(x, y):
        x, y = x.astype(np.uint64), y.astype(np.uint64)
        z = np.where(x < y, y * y + x, x * x + x + y)
        f = np.floor(np.sqrt(z.astype(np.float64))).astype(np.uint64)
        sq = f * f
        first = z - sq < f
        a = np.where(first, z - sq, f)
        b = np.where(first, f, z - sq - f)
        return (a == x) & (b == y)
    g = np.arange(2048, dtype=np.uint64)
    xs, ys = np.meshgrid(g, g)
    assert accurate(xs.ravel(), ys.ravel()).all()
    rng = np.random.default_rng(5)
    r = rng.integers(0, 1 << 24, size=(2, 4_000_000), dtype=np.uint64)
    assert accurate(r[0], r[1]).all()
    edges = np.array([(1 << e) + d for e in range(1, 25) for d in (-2, -1, 0, 1) if (1 << e) + d < (1 << 24)],
                     dtype=np.uint64)
    other = rng.integers(0, 1 << 24, size=(len(edges), 2000), dtype=np.uint64)
    ee = np.repeat(edges, 2000)
    assert accurate(ee, other.ravel()).all() and accurate(other.ravel(), ee).all()


# ---------------------------------------------------------------- SIMDShockHash (SIMDShockHash.hpp)
SIMD_FIXTURES = sorted(os.path.basename(p)[:-4] for p in glob.glob(os.path.join(GOLDEN, "simd*.npz")))


def simd_ref(lanes=None):
    from oracle import bindings
    path = bindings.SIMD_SO[lanes or 4]
    if not os.path.exists(path):
        pytest.skip("compiled SIMDShockHash oracle not available")
    if lanes == 8 and not bindings.host_has_avx512():
        pytest.skip("the 8-lane build needs an AVX-512 host")
    return bindings.RefSimdLib(lanes)


def fmix32(z):  # MurmurHash3's 32-bit finalizer, SIMDShockHash.hpp:76-83, on uint32 arrays
    z = z.astype(np.uint32)
    z ^= z >> np.uint32(16)
    z = (z * np.uint32(0x85EBCA6B)).astype(np.uint32)
    z ^= z >> np.uint32(13)
    z = (z * np.uint32(0xC2B2AE35)).astype(np.uint32)
    z ^= z >> np.uint32(16)
    return z


def test_simd_split_hash_restated(ref):
    # remixAndRemap (SIMDShockHash.hpp:762-766): remap16 of fmix32(hi ^ lo), as the device computes it
    R = simd_ref()
    rng = np.random.default_rng(5)
    x = rand_u64(rng, 20000)
    with np.errstate(over="ignore"):
        folded = fmix32((x >> np.uint64(32)).astype(np.uint32) ^ (x & np.uint64(0xFFFFFFFF)).astype(np.uint32))
    for m in (2, 7, 100, 961, 2999):
        want = ((folded.astype(np.uint64) & np.uint64(0xFFFF)) * np.uint64(m)) >> np.uint64(16)
        assert np.array_equal(R.remix_and_remap(x, m).astype(np.uint64), want), m


@pytest.mark.parametrize("rot,leaf,n,b", [(0, 8, 20000, 100), (0, 30, 20000, 2000), (1, 30, 12000, 2000),
                                          (1, 40, 6000, 2000), (0, 2, 3000, 7), (1, 8, 3000, 50), (0, 33, 4000, 500)])
def test_simd_ref_same_for_4_and_8_lanes(ref, rot, leaf, n, b):
    # The format does not depend on the vector width: every seed search scans seeds in increasing
    # order and keeps the first valid one, and the split hash folds each 64-bit lane on its own.
    a, w = simd_ref(4), simd_ref(8)
    assert (a.lanes, w.lanes) == (4, 8)
    rng = np.random.default_rng(n + leaf + rot)
    f, s = rand_u64(rng, n), unique_u64(rng, n)
    ra, rw = a.build_hash(rot, leaf, f, s, b), w.build_hash(rot, leaf, f, s, b)
    for k in ("desc", "size_acc", "pos_acc", "ribbon_keys", "ribbon_bits"):
        assert np.array_equal(getattr(ra, k), getattr(rw, k)), k
    assert np.array_equal(ra.query_hash(f, s), rw.query_hash(f, s))


@pytest.mark.parametrize("name", SIMD_FIXTURES)
def test_simd_ref_matches_golden(ref, name):
    g = load(name)
    R = simd_ref()
    r = R.build_hash(int(g["variant"]) == 6, int(g["leaf"]), g["first"], g["second"], int(g["bucket_size"]), 2)
    for k in ("desc", "size_acc", "pos_acc", "ribbon_keys", "ribbon_bits"):
        assert np.array_equal(getattr(r, k), g[k]), k
    assert np.array_equal(r.query_hash(g["first"], g["second"]), g["query"])
    assert r.bits == int(g["bits"])


@pytest.mark.parametrize("name", [n for n in SIMD_FIXTURES if n.startswith("simd_")])
def test_port_simd_matches_golden(port, name):
    # the restatement's variant 5 is SIMDShockHash<l, false>
    g = load(name)
    r = port.build_hash(5, int(g["leaf"]), g["first"], g["second"], int(g["bucket_size"]))
    for k in ("desc", "size_acc", "pos_acc", "ribbon_keys", "ribbon_bits"):
        assert np.array_equal(getattr(r, k), g[k]), k
    assert np.array_equal(r.query_hash(g["first"], g["second"]), g["query"])


@pytest.mark.parametrize("leaf,n,b", [(12, 6000, 150), (24, 9000, 700), (32, 6000, 900), (4, 2000, 11)])
def test_port_simd_matches_ref_random(port, ref, leaf, n, b):
    R = simd_ref()
    rng = np.random.default_rng(7 * n + leaf)
    f, s = rand_u64(rng, n), unique_u64(rng, n)
    r, p = R.build_hash(0, leaf, f, s, b, 2), port.build_hash(5, leaf, f, s, b)
    for k in ("desc", "size_acc", "pos_acc", "ribbon_keys", "ribbon_bits"):
        assert np.array_equal(getattr(r, k), getattr(p, k)), k


def test_simd_format_differs_from_shockhash(ref):
    # same keys, same leaf size: SIMDShockHash<l> stores other seeds than ShockHash<l>
    g = load("simd_l30_b2000")
    r = ref.build_hash(1, 30, g["first"], g["second"], 2000, 1)
    assert not np.array_equal(r.desc, g["desc"])
    assert np.array_equal(r.size_acc, g["size_acc"])  # the same buckets
