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


@pytest.mark.parametrize("world,nb", [(1, 5000), (2, 5000), (3, 7), (8, 50_000), (64, 100_003), (5, 1)])
def test_device_partition_equals_host_partition(engine, world, nb):
    import torch
    from shockhash_b200 import shard
    rng = np.random.default_rng(world * 7 + nb)
    n = 1_000_003
    f = rng.integers(0, 2**64, size=n, dtype=np.uint64)
    s = rng.integers(0, 2**64, size=n, dtype=np.uint64)
    ft, st = torch.from_numpy(f.view(np.int64)), torch.from_numpy(s.view(np.int64))
    host_pairs, host_counts = shard.partition(ft, st, nb, world)
    dev_pairs, dev_counts = shard.partition(ft.cuda(), st.cuda(), nb, world, engine)
    assert np.array_equal(dev_counts, host_counts)
    assert torch.equal(dev_pairs.cpu(), host_pairs)


def test_device_shard_builds_merge_to_one_build(engine):
    import torch
    from shockhash_b200 import shard
    rng = np.random.default_rng(5)
    n, b, world = 300_000, 2000, 3
    f = rng.integers(0, 2**64, size=n, dtype=np.uint64)
    s = np.unique(rng.integers(0, 2**64, size=n + 64, dtype=np.uint64))[:n]
    full = engine.build_hash128(2, 64, f, s, b)
    nb = shard.nbuckets(n, b)
    pairs, counts = shard.partition(torch.from_numpy(f.view(np.int64)).cuda(), torch.from_numpy(s.view(np.int64)).cuda(),
                                    nb, world, engine)
    parts, at = [], 0
    for g, (b0, b1) in enumerate(shard.bucket_ranges(nb, world)):
        seg = pairs[at:at + int(counts[g])]
        at += int(counts[g])
        fg, sg = seg[:, 0].contiguous(), seg[:, 1].contiguous()
        torch.cuda.synchronize()  # torch's copies are done before the engine's stream reads them
        r = engine.build_shard_hash128_device(2, 64, fg.data_ptr(), sg.data_ptr(), fg.numel(), nb, b0, b1, b)
        parts.append(shard._arrays(r))
        r.free()
    m = shg.merge_shards(2, 64, parts, b)
    for name in ("bucket_size_acc", "bucket_pos_acc", "descriptors", "ribbon_keys", "ribbon_bits"):
        assert np.array_equal(getattr(m, name), getattr(full, name)), name
