"""Shards by bucket range (shockhash_b200.shard, shg_merge_shards) on the host: shard builds of
the C++ restatement joined by the library's merge equal one build of all keys, bit for bit; the
exchange and gather run as two gloo ranks."""
import os
import socket

import numpy as np
import pytest

import shockhash_b200 as shg
from shockhash_b200 import shard
from conftest import rand_u64, unique_u64


def _keys(seed, n):
    rng = np.random.default_rng(seed)
    return rand_u64(rng, n), unique_u64(rng, n)


def _same(m, full):
    assert np.array_equal(m.bucket_size_acc, full.size_acc)
    assert np.array_equal(m.bucket_pos_acc, full.pos_acc)
    assert np.array_equal(m.descriptors, full.desc)
    assert np.array_equal(m.ribbon_keys, full.ribbon_keys)
    assert np.array_equal(m.ribbon_bits, full.ribbon_bits)


def test_remap128_matches_integer_arithmetic():
    f = rand_u64(np.random.default_rng(1), 1000)
    for nb in (1, 7, 5000, 50000, (1 << 32) - 1):
        want = np.array([(int(x) * nb) >> 64 for x in f], dtype=np.uint64)
        assert np.array_equal(shard.remap128(f, nb), want)


@pytest.mark.parametrize("variant,leaf,n,b,world", [(2, 24, 30000, 700, 3), (1, 16, 20000, 500, 2),
                                                    (2, 64, 9000, 2000, 4), (2, 10, 300, 100, 5)])
def test_merged_port_shards_equal_one_build(port, variant, leaf, n, b, world):
    f, s = _keys(variant * 100 + world, n)
    full = port.build_hash(variant, leaf, f, s, b)
    nb = shard.nbuckets(n, b)
    own = shard.owners(f, nb, world)
    parts = []
    for g, (b0, b1) in enumerate(shard.bucket_ranges(nb, world)):
        if b1 > b0:
            sel = own == g
            parts.append(shard._arrays(port.build_shard(variant, leaf, f[sel], s[sel], nb, b0, b1, b)))
        else:
            assert not (own == g).any()
    m = shg.merge_shards(variant, leaf, parts, b)
    _same(m, full)
    assert m.desc_bits == int(full.pos_acc[-1]) + 1


def test_merge_rejects_shards_of_another_structure(port):
    f, s = _keys(9, 5000)
    nb = shard.nbuckets(5000, 500)
    own = shard.owners(f, nb, 2)
    b0, b1 = shard.bucket_ranges(nb, 2)[0]
    part = shard._arrays(port.build_shard(2, 24, f[own == 0], s[own == 0], nb, b0, b1, 500))
    with pytest.raises(shg.ShgError):
        shg.merge_shards(2, 24, [part], 500)  # half of the buckets only


def _free_port():
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        return sk.getsockname()[1]


def _rank_main(rank, world, port_no, variant, leaf, n, b, out_dir):
    import torch.distributed as dist
    from oracle.bindings import PortLib
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port_no)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        P = PortLib()
        f, s = _keys(77, n)
        mine = slice(rank, None, world)  # each rank starts with an interleaved slice of the keys
        part, nb, (b0, b1) = shard.build_sharded(
            lambda ff, ss, nbg, x0, x1: P.build_shard(variant, leaf, ff, ss, nbg, x0, x1, b), f[mine], s[mine], b)
        own = shard.owners(f, nb, world)
        assert part.n == int((own == rank).sum())
        koff, boff = shard.shard_offsets(part)
        full = P.build_hash(variant, leaf, f, s, b)
        assert koff == int(full.size_acc[b0]) and boff == int(full.pos_acc[b0])
        merged = shard.gather_merge(part, variant, leaf, b)
        if rank == 0:
            _same(merged, full)
            open(os.path.join(out_dir, "ok"), "w").write("ok")
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_exchange_build_and_merge(tmp_path):
    import torch.multiprocessing as mp
    mp.spawn(_rank_main, args=(2, _free_port(), 2, 24, 12000, 600, str(tmp_path)), nprocs=2, join=True)
    assert (tmp_path / "ok").exists()


@pytest.mark.parametrize("world,nb", [(1, 5), (2, 5000), (3, 7), (8, 1), (5, 123457), (64, 1000)])
def test_host_partition_is_the_stable_owner_order(world, nb):
    import torch
    f, s = _keys(world * 31 + nb, 20_011)
    pairs, counts = shard.partition(torch.from_numpy(f.view(np.int64)), torch.from_numpy(s.view(np.int64)), nb, world)
    own = shard.owners(f, nb, world)
    order = np.argsort(own, kind="stable")
    got = pairs.numpy().view(np.uint64)
    assert np.array_equal(got[:, 0], f[order]) and np.array_equal(got[:, 1], s[order])
    assert np.array_equal(counts, np.bincount(own, minlength=world))


def _tensor_rank_main(rank, world, port_no, variant, leaf, n, b, out_dir):
    import torch
    import torch.distributed as dist
    from oracle.bindings import PortLib
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port_no)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        P = PortLib()
        f, s = _keys(78, n)
        mine = slice(rank, None, world)
        ft = torch.from_numpy(np.ascontiguousarray(f[mine]).view(np.int64))
        st = torch.from_numpy(np.ascontiguousarray(s[mine]).view(np.int64))
        build = lambda ff, ss, nbg, x0, x1: P.build_shard(variant, leaf, ff.numpy().view(np.uint64),
                                                          ss.numpy().view(np.uint64), nbg, x0, x1, b)
        part, nb, (b0, b1) = shard.build_sharded_tensors(build, ft, st, b)
        own = shard.owners(f, nb, world)
        assert (part.n if part is not None else 0) == int((own == rank).sum())
        merged = shard.gather_merge_tensors(part, variant, leaf, b)
        if rank == 0:
            _same(merged, P.build_hash(variant, leaf, f, s, b))
            open(os.path.join(out_dir, "ok"), "w").write("ok")
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world,n,b", [(2, 12000, 600), (3, 900, 500)])
def test_gloo_ranks_tensor_exchange_build_and_merge(tmp_path, world, n, b):
    # (3, 900, 500): two buckets over three ranks, so one rank owns none
    import torch.multiprocessing as mp
    mp.spawn(_tensor_rank_main, args=(world, _free_port(), 2, 24, n, b, str(tmp_path)), nprocs=world, join=True)
    assert (tmp_path / "ok").exists()
