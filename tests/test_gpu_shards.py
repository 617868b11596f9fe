"""Shard builds on the device (shg_build_shard_hash128) joined by shg_merge_shards equal one
device build of all keys, bit for bit (runs on a B200)."""
import numpy as np
import pytest

import shockhash_b200 as shg
from shockhash_b200 import shard
from conftest import rand_u64, unique_u64

pytestmark = pytest.mark.gpu


def _same(a, b):
    return (np.array_equal(a.bucket_size_acc, b.bucket_size_acc) and np.array_equal(a.bucket_pos_acc, b.bucket_pos_acc)
            and np.array_equal(a.descriptors, b.descriptors) and np.array_equal(a.ribbon_keys, b.ribbon_keys)
            and np.array_equal(a.ribbon_bits, b.ribbon_bits))


@pytest.mark.parametrize("variant,leaf,n,world", [(2, 64, 1_000_000, 4), (1, 30, 300_000, 3), (2, 100, 100_000, 2)])
def test_shard_builds_merge_to_one_build(engine, variant, leaf, n, world):
    rng = np.random.default_rng(31 + world)
    f, s = rand_u64(rng, n), unique_u64(rng, n)
    full = engine.build_hash128(variant, leaf, f, s, 2000)
    nb = shard.nbuckets(n, 2000)
    own = shard.owners(f, nb, world)
    parts = []
    for g, (b0, b1) in enumerate(shard.bucket_ranges(nb, world)):
        sel = own == g
        r = engine.build_shard_hash128(variant, leaf, f[sel], s[sel], nb, b0, b1)
        parts.append(shard._arrays(r))
        r.free()
    merged = shg.merge_shards(variant, leaf, parts)
    assert _same(merged, full)
    q = shg.DeviceMphf(merged)
    assert np.array_equal(q.query_hash(f, s), shg.DeviceMphf(full).query_hash(f, s))


def test_shard_rejects_keys_outside_its_range(engine):
    rng = np.random.default_rng(5)
    f, s = rand_u64(rng, 50_000), unique_u64(rng, 50_000)
    nb = shard.nbuckets(len(f), 2000)
    with pytest.raises(shg.ShgError) as ei:
        engine.build_shard_hash128(2, 64, f, s, nb, 0, nb // 2)
    assert ei.value.status == 1
    ok = shard.owners(f, nb, 2) == 0
    r = engine.build_shard_hash128(2, 64, f[ok], s[ok], nb, 0, nb // 2)  # the engine stays usable
    assert r.nbuckets == nb // 2 and r.n == int(ok.sum())
