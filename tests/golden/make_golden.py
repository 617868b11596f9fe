"""Generates the golden fixtures in this folder by running the reference itself.

The reference (its unmodified headers and src/ShockHash2-precompiled.cpp, compiled with the
restated third-party stand-ins in oracle/shims) is built as oracle/_ref/libshref.so by
``make -C oracle ref`` in the container that holds the reference sources. This script seeds the
inputs, runs the reference constructors and stores inputs and products as .npz files together with
a SHA-256 manifest. The tests compare the CPU restatement (oracle/port) and the CUDA path against
these files; they never need the reference sources at run time.

The SIMDShockHash fixtures (simd_*, simdrot_*) come from the reference's SIMDShockHash.hpp compiled
with -DSIMD (oracle/_ref/libshref_simd.so and its 8-lane twin in oracle/_ref/v4/; their products are
the same for both lane counts, which tests/test_oracle.py checks).

Usage:  python tests/golden/make_golden.py [core] [simd]     (no argument: both groups)
"""
import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
from oracle.bindings import RefLib, RefSimdLib  # noqa: E402

# (name, variant, leaf, n, bucket_size, seed)
BUILDS = [
    ("sh1_l30_b2000", 1, 30, 20000, 2000, 101),
    ("sh1_l8_b100", 1, 8, 5000, 100, 102),
    ("sh1_l40_b2000", 1, 40, 6000, 2000, 103),
    ("sh1_l5_b7", 1, 5, 1500, 7, 104),
    ("sh1_l60_b500", 1, 60, 1500, 500, 105),
    ("sh2_l64_b2000", 2, 64, 20000, 2000, 201),
    ("sh2_l10_b100", 2, 10, 5000, 100, 202),
    ("sh2_l9_b50", 2, 9, 3000, 50, 203),
    ("sh2_l33_b500", 2, 33, 8000, 500, 204),
    ("sh2_l3_b5", 2, 3, 1000, 5, 205),
    ("sh2_l100_b1000", 2, 100, 2000, 1000, 206),
    ("sh2_l64_tiny", 2, 64, 3, 2000, 207),
    ("sh1_l30_tiny", 1, 30, 2, 2000, 208),
    # ShockHash<l, true> (rotation fitting); l > 32 shares set A's cells over eight seeds
    ("rot_l30_b2000", 3, 30, 20000, 2000, 111),
    ("rot_l40_b2000", 3, 40, 8000, 2000, 112),
    ("rot_l16_b100", 3, 16, 5000, 100, 113),
    ("rot_l8_b50", 3, 8, 3000, 50, 114),
    ("rot_l33_b500", 3, 33, 5000, 500, 115),
    ("rot_l48_b2000", 3, 48, 6000, 2000, 116),
]
# SIMDShockHash<leaf, rotation>: (name, rotation, leaf, n, bucket_size, seed)
SIMD_BUILDS = [
    ("simd_l30_b2000", 0, 30, 20000, 2000, 501),
    ("simd_l8_b100", 0, 8, 5000, 100, 502),
    ("simd_l40_b2000", 0, 40, 6000, 2000, 503),
    ("simd_l16_b300", 0, 16, 9000, 300, 504),
    ("simd_l2_b7", 0, 2, 1500, 7, 505),
    ("simd_l33_b500", 0, 33, 4000, 500, 506),
    ("simd_l48_b1000", 0, 48, 2000, 1000, 507),
    ("simd_l30_tiny", 0, 30, 2, 2000, 508),
    ("simdrot_l30_b2000", 1, 30, 20000, 2000, 511),
    ("simdrot_l16_b100", 1, 16, 5000, 100, 512),
    ("simdrot_l40_b2000", 1, 40, 8000, 2000, 513),
    ("simdrot_l8_b50", 1, 8, 3000, 50, 514),
    ("simdrot_l33_b500", 1, 33, 5000, 500, 515),
    ("simdrot_l48_b2000", 1, 48, 6000, 2000, 516),
]
# (k, n, seed) for ShockHash2Flat<k>
FLATS = [(16, 30000, 401), (32, 20000, 402), (64, 20003, 403), (100, 4100, 404), (8, 5000, 405)]
LEAVES_SH2 = [(m, 40 if m <= 64 else 4) for m in list(range(2, 65)) + [80, 100, 128]]
LEAVES_SH1 = [(m, 20) for m in range(2, 41)] + [(48, 3), (60, 2)]


def sha(path):
    h = hashlib.sha256()
    with open(path, "rb") as f:
        h.update(f.read())
    return h.hexdigest()


def simd(manifest):
    R = RefSimdLib()
    for name, rot, leaf, n, b, seed in SIMD_BUILDS:
        rng = np.random.default_rng(seed)
        first = rng.integers(0, 2**64, size=n, dtype=np.uint64)
        second = np.unique(rng.integers(0, 2**64, size=n + 8, dtype=np.uint64))[:n]
        rng.shuffle(second)
        r = R.build_hash(rot, leaf, first, second, b, 1)
        q = r.query_hash(first, second)
        path = os.path.join(HERE, name + ".npz")
        np.savez_compressed(path, variant=6 if rot else 5, leaf=leaf, bucket_size=b, first=first, second=second,
                            desc=r.desc, size_acc=r.size_acc, pos_acc=r.pos_acc, ribbon_keys=r.ribbon_keys,
                            ribbon_bits=r.ribbon_bits, query=q, bits=r.bits, lanes=R.lanes)
        manifest[name + ".npz"] = sha(path)
        r.free()


def main(groups):
    mpath = os.path.join(HERE, "MANIFEST.json")
    manifest = {}
    if os.path.exists(mpath):
        with open(mpath) as fh:
            manifest = json.load(fh)
    if "simd" in groups:
        simd(manifest)
    if "core" in groups:
        core(manifest)
    with open(mpath, "w") as fh:
        json.dump(manifest, fh, indent=1, sort_keys=True)
    print(json.dumps(manifest, indent=1))


def core(manifest):
    R = RefLib()
    for name, variant, leaf, n, b, seed in BUILDS:
        rng = np.random.default_rng(seed)
        first = rng.integers(0, 2**64, size=n, dtype=np.uint64)
        second = np.unique(rng.integers(0, 2**64, size=n + 8, dtype=np.uint64))[:n]
        rng.shuffle(second)
        r = R.build_hash(variant, leaf, first, second, b, 1)
        q = r.query_hash(first, second)
        path = os.path.join(HERE, name + ".npz")
        np.savez_compressed(path, variant=variant, leaf=leaf, bucket_size=b, first=first, second=second,
                            desc=r.desc, size_acc=r.size_acc, pos_acc=r.pos_acc, ribbon_keys=r.ribbon_keys,
                            ribbon_bits=r.ribbon_bits, query=q, bits=r.bits)
        manifest[name + ".npz"] = sha(path)
        r.free()
    # single leaves through the reference's leaf seams
    rng = np.random.default_rng(301)
    keys, offs, seeds, bits = [], [0], [], []
    for m, cnt in LEAVES_SH2:
        for _ in range(cnt):
            k = np.unique(rng.integers(0, 2**64, size=m + 4, dtype=np.uint64))[:m]
            rng.shuffle(k)
            s, rk, rb = R.sh2_leaf(k)
            assert np.array_equal(rk, k)
            keys.append(k)
            offs.append(offs[-1] + m)
            seeds.append(s)
            bits.append(rb)
    path = os.path.join(HERE, "sh2_leaves.npz")
    np.savez_compressed(path, keys=np.concatenate(keys), offsets=np.array(offs, np.uint64),
                        seeds=np.array(seeds, np.uint64), bits=np.concatenate(bits))
    manifest["sh2_leaves.npz"] = sha(path)
    rng = np.random.default_rng(302)
    keys, offs, codes, kc, bits, levels = [], [0], [], [], [], []
    for m, cnt in LEAVES_SH1:
        for t in range(cnt):
            k = np.unique(rng.integers(0, 2**64, size=m + 4, dtype=np.uint64))[:m]
            rng.shuffle(k)
            level = t % 3
            c, rk, rb = R.sh1_leaf(60, k, level)
            keys.append(k)
            offs.append(offs[-1] + m)
            codes.append(c)
            kc.append(rk)
            bits.append(rb)
            levels.append(level)
    path = os.path.join(HERE, "sh1_leaves.npz")
    np.savez_compressed(path, keys=np.concatenate(keys), offsets=np.array(offs, np.uint64),
                        codes=np.array(codes, np.uint64), keys_by_cell=np.concatenate(kc),
                        bits=np.concatenate(bits), levels=np.array(levels, np.int32))
    manifest["sh1_leaves.npz"] = sha(path)
    # ShockHash2Flat<k> over string keys (MurmurHash64 path)
    for k, n, seed in FLATS:
        rng = np.random.default_rng(seed)
        keys = [bytes(rng.integers(0, 256, size=int(rng.integers(8, 40)), dtype=np.uint8)) for _ in range(n)]
        keys = list(dict.fromkeys(keys))
        d = R.flat_build_strings(k, keys)
        path = os.path.join(HERE, f"flat_k{k}.npz")
        np.savez_compressed(path, k=k, data=np.frombuffer(b"".join(keys), np.uint8),
                            lengths=np.array([len(x) for x in keys], np.uint64), **d)
        manifest[f"flat_k{k}.npz"] = sha(path)
    # string hashing (short and long SpookyHash paths) and the README example
    rng = np.random.default_rng(303)
    strs = [bytes(rng.integers(0, 256, size=L, dtype=np.uint8)) for L in list(range(0, 260)) + [300, 511, 1000]]
    f, s = R.spooky128(strs)
    readme = [b"abc", b"def", b"123", b"456"]
    rb = R.build_strings(1, 30, readme, 2000, 1)
    readme_out = R.query_strings(rb, readme)
    path = os.path.join(HERE, "strings.npz")
    np.savez_compressed(path, data=np.frombuffer(b"".join(strs), np.uint8),
                        lengths=np.array([len(x) for x in strs], np.uint64), first=f, second=s,
                        murmur=R.murmur64(strs), readme_out=readme_out)
    manifest["strings.npz"] = sha(path)


if __name__ == "__main__":
    main(sys.argv[1:] or ["core", "simd"])
