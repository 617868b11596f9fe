"""Bit-exact parity at the benchmark configurations' own sizes: the device builds of the configuration
key sets (ShockHash<30,false> over 1M printable strings, ShockHash2<64> over 10M uint64 keys,
ShockHash<40,false> over 2M uint64 keys, ShockHash2Flat<100> over 500k Zipf-length strings) against
SHA-256 digests of what the compiled reference builds from the same keys, and operator() of every
key on the device against the reference's. The digests come from tests/golden/make_config_digests.py
(committed with it); the keys from the oracle's generators, so no large fixture is stored."""
import hashlib
import json
import os

import numpy as np
import pytest

import shockhash_b200 as shg
from oracle import bindings

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
with open(os.path.join(GOLDEN, "config_digests.json")) as _f:
    DIGESTS = json.load(_f)["configs"]
RECSPLIT = sorted(k for k, v in DIGESTS.items() if v["variant"] != "flat")
FLAT = sorted(k for k, v in DIGESTS.items() if v["variant"] == "flat")


def digest(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def config_keys(c):
    kind, seed, n = c["keys"]["kind"], c["keys"]["seed"], c["keys"]["n"]
    if kind == "u64":
        return bindings.keys_mt19937_64(seed, n)
    return bindings.strings_mt19937_64(bindings.STRINGS_PRINTABLE if kind == "printable" else bindings.STRINGS_ZIPF,
                                       seed, n)


def check(c, arrays):
    bad = [k for k, v in arrays.items() if digest(v) != c["sha256"][k]]
    assert not bad, f"products differ from the reference: {bad}"
    assert {k: len(v) for k, v in arrays.items()} == {k: c["sizes"][k] for k in arrays}


@pytest.mark.parametrize("name", RECSPLIT)
def test_config_build_matches_reference(engine, port, name):
    c = DIGESTS[name]
    keys = config_keys(c)
    if c["keys"]["kind"] == "u64":
        r = engine.build_u64(c["variant"], c["leaf"], keys, c["bucket_size"])
        dq = shg.DeviceMphf(r)
        q = dq.query_u64(keys)
    else:
        r = engine.build_strings(c["variant"], c["leaf"], keys, c["bucket_size"])
        dq = shg.DeviceMphf(r)
        q = dq.query_strings(keys)
    check(c, {"descriptors": r.descriptors, "bucket_size_acc": r.bucket_size_acc, "bucket_pos_acc": r.bucket_pos_acc,
              "ribbon_keys": r.ribbon_keys, "ribbon_bits": r.ribbon_bits, "query": q})
    assert r.mphf().bits() == c["bits"]
    dq.close()
    r.free()


@pytest.mark.parametrize("name", FLAT)
def test_config_flat_matches_reference(engine, port, name):
    c = DIGESTS[name]
    keys = config_keys(c)
    f = engine.build_flat_strings(c["leaf"], keys)
    dq = f.device_query()
    q = dq.query_strings(keys)
    check(c, {"thresholds_and_seeds": f.thresholds_and_seeds, "layer_bases": f.layer_bases,
              "fallback_buckets": f.fallback_seed_buckets, "fallback_seeds": f.fallback_seeds,
              "free_positions": f.free_positions, "ribbon_keys": f.ribbon_keys, "ribbon_bits": f.ribbon_bits,
              "query": q})
    assert f.layers == c["layers"] and f.bits() == c["bits"]
    dq.close()
    f.free()
