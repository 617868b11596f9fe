"""Build results on disk (shg_result_save / shg_result_load) without a GPU: a result of the C++
restatement, taken into the library, written and read back, keeps every array and answers
operator() as the restatement does; the descriptors section is RiceBitVector's stream layout
(RiceBitVector.h:133-141: u64 word count, then the words); damaged files are rejected."""
import os
import struct
from types import SimpleNamespace

import numpy as np
import pytest

import shockhash_b200 as shg
from shockhash_b200 import shard
from conftest import rand_u64, unique_u64


def _library_result(port, variant, leaf, n, b, seed):
    rng = np.random.default_rng(seed)
    f, s = rand_u64(rng, n), unique_u64(rng, n)
    full = port.build_hash(variant, leaf, f, s, b)
    # one shard covering every bucket is the whole structure as a library-owned result
    return shg.merge_shards(variant, leaf, [shard._arrays(full)], b), full, f, s


@pytest.mark.parametrize("variant,leaf,n,b", [(2, 64, 20000, 2000), (1, 30, 5000, 2000), (2, 9, 3000, 50)])
def test_round_trip(tmp_path, port, variant, leaf, n, b):
    res, full, f, s = _library_result(port, variant, leaf, n, b, 70 + variant)
    path = str(tmp_path / "mphf.shg")
    res.save(path)
    back = shg.load_result(path)
    assert (back.params.variant, back.params.leaf_size, back.params.bucket_size) == (variant, leaf, b)
    for name in ("bucket_size_acc", "bucket_pos_acc", "descriptors", "ribbon_keys", "ribbon_bits"):
        assert np.array_equal(getattr(back, name), getattr(res, name)), name
    assert back.desc_bits == res.desc_bits and back.n == n
    assert np.array_equal(back.mphf().query_hash(f, s), full.query_hash(f, s))
    # descriptors section: word count, then the words
    with open(path, "rb") as fh:
        raw = fh.read()
    nb = res.nbuckets
    off = 8 + 8 + 40 + 16 * (nb + 1)
    (words,) = struct.unpack_from("<Q", raw, off)
    assert words == len(res.descriptors)
    assert np.array_equal(np.frombuffer(raw, dtype="<u8", count=words, offset=off + 8), res.descriptors)
    back.free()


def test_round_trip_rotation_fitting_golden(tmp_path):
    g = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "rot_l30_b2000.npz"))
    arrays = SimpleNamespace(size_acc=g["size_acc"], pos_acc=g["pos_acc"], desc=g["desc"],
                             ribbon_keys=g["ribbon_keys"], ribbon_bits=g["ribbon_bits"])
    res = shg.merge_shards(3, 30, [shard._arrays(arrays)], int(g["bucket_size"]))
    path = str(tmp_path / "rot.shg")
    res.save(path)
    back = shg.load_result(path)
    assert back.params.variant == 3
    assert np.array_equal(back.mphf().query_hash(g["first"], g["second"]), g["query"])
    assert back.mphf().bits() == int(g["bits"])


@pytest.mark.parametrize("name", ["simd_l30_b2000", "simd_l2_b7", "simd_l48_b1000", "simdrot_l30_b2000",
                                  "simdrot_l40_b2000", "simdrot_l8_b50"])
def test_round_trip_simd_golden(tmp_path, name):
    # SIMDShockHash<l, rot>: the host query's own split hash and start seeds answer as the reference
    g = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", name + ".npz"))
    arrays = SimpleNamespace(size_acc=g["size_acc"], pos_acc=g["pos_acc"], desc=g["desc"],
                             ribbon_keys=g["ribbon_keys"], ribbon_bits=g["ribbon_bits"])
    variant, leaf = int(g["variant"]), int(g["leaf"])
    res = shg.merge_shards(variant, leaf, [shard._arrays(arrays)], int(g["bucket_size"]))
    path = str(tmp_path / "simd.shg")
    res.save(path)
    back = shg.load_result(path)
    assert (back.params.variant, back.params.leaf_size) == (variant, leaf)
    assert np.array_equal(back.mphf().query_hash(g["first"], g["second"]), g["query"])
    assert back.mphf().bits() == int(g["bits"])


def test_damaged_files_are_rejected(tmp_path, port):
    res, _, _, _ = _library_result(port, 2, 64, 5000, 2000, 5)
    path = str(tmp_path / "a.shg")
    res.save(path)
    raw = open(path, "rb").read()
    cases = {"magic": b"XXXXXXXX" + raw[8:], "truncated": raw[:-3], "longer": raw + b"\0",
             "words": raw[:56 + 16 * (res.nbuckets + 1)] + struct.pack("<Q", 1) + raw[56 + 16 * (res.nbuckets + 1) + 8:]}
    nb = res.nbuckets
    acc0 = 56  # bucket_size_acc, then bucket_pos_acc, (nb + 1) words each
    def put(data, off, value):
        return data[:off] + struct.pack("<Q", value) + data[off + 8:]
    cases.update({
        "variant": raw[:8] + struct.pack("<I", 9) + raw[12:],
        "leaf_size": raw[:12] + struct.pack("<I", 500) + raw[16:],
        "size_acc_decreases": put(raw, acc0 + 8 * 2, 0),
        "size_acc_start": put(raw, acc0, 1),
        "pos_acc_decreases": put(raw, acc0 + 8 * (nb + 1) + 8 * 2, 0),
        "pos_acc_past_bits": put(raw, acc0 + 8 * (nb + 1) + 8 * nb, res.desc_bits + 64),
        "huge_ribbon_count": raw[:48] + struct.pack("<Q", (1 << 63) + 5) + raw[56:],
        "huge_bit_count": raw[:40] + struct.pack("<Q", (1 << 62)) + raw[48:],
    })
    for name, data in cases.items():
        p = str(tmp_path / (name + ".shg"))
        with open(p, "wb") as fh:
            fh.write(data)
        with pytest.raises(shg.ShgError):
            shg.load_result(p)
    with pytest.raises(shg.ShgError):
        shg.load_result(str(tmp_path / "missing.shg"))
