"""Generates tests/golden/config_digests.json: SHA-256 digests of what the reference itself builds for
the benchmark configurations at their own sizes (or, where the reference's build is slow, a stated
prefix of the same key stream), so that the GPU tests can check the device builds bit for bit at
those sizes without storing the products.

Runs the compiled reference (oracle/_ref, built by ``make -C oracle ref`` where the reference
sources are) on keys drawn by the oracle's generators (oracle/keygen.h), with all host threads
(its output does not depend on the thread count). Per configuration it records the digests of the
Golomb-Rice descriptor words, bucket_size_acc, bucket_pos_acc, the retrieval input (keys, bits) and
operator() of every key, plus their sizes and getBits(); for ShockHash2Flat<100> the thresholds
and seeds, layer bases, fallback seeds, free positions, retrieval input and operator().

Usage:  python tests/golden/make_config_digests.py
"""
import hashlib
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
from oracle import bindings  # noqa: E402

# name -> (variant (1 = ShockHash<l,false>, 2 = ShockHash2<l>, 'flat' = ShockHash2Flat<k>), leaf,
#          bucket size, key kind, seed, keys)
CONFIGS = {
    "c1_sh1_l30_printable_1M": (1, 30, 2000, "printable", 42, 1_000_000),
    "c2_sh2_l64_u64_10M": (2, 64, 2000, "u64", 7, 10_000_000),
    "c3_sh1_l40_u64_2M": (1, 40, 2000, "u64", 11, 2_000_000),
    "c4_flat_k100_zipf_500k": ("flat", 100, 0, "zipf", 23, 500_000),
}


def digest(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def keys_of(kind, seed, n):
    """(bytes, offsets) of the configuration's string keys (uint64 keys as 8-byte strings)."""
    if kind == "u64":
        k = bindings.keys_mt19937_64(seed, n)
        return np.ascontiguousarray(k, dtype="<u8").tobytes(), np.arange(0, 8 * (n + 1), 8, dtype=np.uint64)
    return bindings.strings_mt19937_64(bindings.STRINGS_PRINTABLE if kind == "printable" else bindings.STRINGS_ZIPF,
                                       seed, n)


def main():
    R = bindings.RefLib()
    threads = os.cpu_count() or 1
    out = {}
    for name, (variant, leaf, bucket, kind, seed, n) in CONFIGS.items():
        t0 = time.time()
        data, offs = keys_of(kind, seed, n)
        entry = {"variant": variant, "leaf": leaf, "bucket_size": bucket, "keys": {"kind": kind, "seed": seed, "n": n}}
        if variant == "flat":
            d = R.flat_build_strings(leaf, bindings.split_strings(data, offs))
            entry["sha256"] = {k: digest(d[k]) for k in ("thresholds_and_seeds", "layer_bases", "fallback_buckets",
                                                         "fallback_seeds", "free_positions", "ribbon_keys",
                                                         "ribbon_bits", "query")}
            entry["sizes"] = {k: int(len(d[k])) for k in entry["sha256"]}
            entry["bits"] = int(d["bits"])
            entry["layers"] = int(d["layers"])
        else:
            b, secs = R.build_strings_packed_timed(variant, leaf, data, offs, bucket, threads)
            q = R.query_packed(b, data, offs)
            assert np.array_equal(np.sort(q), np.arange(n, dtype=np.uint64)), name
            arrays = {"descriptors": b.desc, "bucket_size_acc": b.size_acc, "bucket_pos_acc": b.pos_acc,
                      "ribbon_keys": b.ribbon_keys, "ribbon_bits": b.ribbon_bits, "query": q}
            entry["sha256"] = {k: digest(v) for k, v in arrays.items()}
            entry["sizes"] = {k: int(len(v)) for k, v in arrays.items()}
            entry["bits"] = int(b.bits)
            b.free()
        out[name] = entry
        print(name, f"{time.time() - t0:.1f} s", flush=True)
    with open(os.path.join(HERE, "config_digests.json"), "w") as fh:
        json.dump({"generator": "tests/golden/make_config_digests.py", "reference_build": bindings.ref_build_info(),
                   "configs": out}, fh, indent=1, sort_keys=True)


if __name__ == "__main__":
    main()
