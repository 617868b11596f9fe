"""One structure over several GPUs or processes: shards by bucket range.

The bucket of a key is remap128(first, nb) with nb = max(1, ceil(N / bucket_size)) for the total
key count N (ShockHash.h:616, Sorter.hpp:15-36), and it is monotone in `first`; buckets are built
independently (the reference's compute_thread hands each thread a bucket range,
ShockHash.h:566-570). So rank g of G owns the buckets [nb*g/G, nb*(g+1)/G):

1. ``exchange``: one all-to-all of the 16-byte fingerprints sends every key to the rank that owns
   its bucket (NCCL over NVLink for CUDA tensors, gloo on the host);
2. each rank builds its bucket range (``Engine.build_shard_hash128`` on its GPU);
3. ``shard_offsets``: an all-gather of (keys, code bits) per rank gives every rank the global key
   and bit offsets of its buckets (the structure can stay sharded);
4. ``gather_merge``: or the shard arrays go to one rank, which joins them with
   ``merge_shards`` into exactly the result a single build of all keys gives.

Keys with equal `first` (probability about N^2 / 2^65) may reach a bucket in another order than in
a single build; the bucket sort orders ties by arrival.
"""
from types import SimpleNamespace

import numpy as np

from . import merge_shards


def remap128(first, nb):
    """High 64 bits of first * nb for uint64 arrays (nb < 2^32)."""
    first = np.asarray(first, dtype=np.uint64)
    nb = np.uint64(nb)
    hi, lo = first >> np.uint64(32), first & np.uint64(0xFFFFFFFF)
    return (hi * nb + ((lo * nb) >> np.uint64(32))) >> np.uint64(32)


def nbuckets(n_total, bucket_size):
    return max(1, (int(n_total) + bucket_size - 1) // bucket_size)


def bucket_ranges(nb, world):
    """[b0, b1) per rank; ranks past nb get empty ranges."""
    return [(nb * g // world, nb * (g + 1) // world) for g in range(world)]


def owners(first, nb, world):
    """Rank that owns each key's bucket."""
    starts = np.array([r[0] for r in bucket_ranges(nb, world)], dtype=np.uint64)
    return (np.searchsorted(starts, remap128(first, nb), side="right") - 1).astype(np.int64)


def _dist():
    import torch.distributed as dist
    return dist


def exchange(first, second, nb, group=None, device=None):
    """All-to-all of (first, second): afterwards each rank holds the keys of its bucket range, in
    the order (source rank, position on the source rank)."""
    import torch
    dist = _dist()
    world = dist.get_world_size(group)
    first = np.ascontiguousarray(first, dtype=np.uint64)
    second = np.ascontiguousarray(second, dtype=np.uint64)
    own = owners(first, nb, world)
    order = np.argsort(own, kind="stable")
    send = np.bincount(own, minlength=world).astype(np.int64)
    sc = torch.from_numpy(send).to(device)
    rc = torch.empty_like(sc)
    dist.all_to_all_single(rc, sc, group=group)
    recv_counts = rc.cpu().tolist()
    payload = np.stack([first[order], second[order]], axis=1).view(np.int64)
    out = torch.empty((int(sum(recv_counts)), 2), dtype=torch.int64, device=device)
    dist.all_to_all_single(out, torch.from_numpy(np.ascontiguousarray(payload)).to(device),
                           output_split_sizes=recv_counts, input_split_sizes=send.tolist(), group=group)
    got = out.cpu().numpy().view(np.uint64)
    return np.ascontiguousarray(got[:, 0]), np.ascontiguousarray(got[:, 1])


def build_sharded(build_shard, first, second, bucket_size, group=None, device=None):
    """Exchange this rank's keys and build its bucket range.

    ``build_shard(first, second, nb_global, b0, b1)`` builds one shard (for example
    ``lambda f, s, nb, b0, b1: engine.build_shard_hash128(2, 64, f, s, nb, b0, b1, 2000)``).
    Returns (shard result or None for an empty range, nb_global, (b0, b1))."""
    import torch
    dist = _dist()
    world, rank = dist.get_world_size(group), dist.get_rank(group)
    t = torch.tensor([len(first)], dtype=torch.int64, device=device)
    dist.all_reduce(t, group=group)
    nb = nbuckets(int(t.item()), bucket_size)
    f, s = exchange(first, second, nb, group, device)
    b0, b1 = bucket_ranges(nb, world)[rank]
    shard = build_shard(f, s, nb, b0, b1) if b1 > b0 else None
    if shard is None and len(f):
        raise RuntimeError("keys arrived at a rank without buckets")
    return shard, nb, (b0, b1)


def _arrays(shard):
    """The arrays of a shard result (engine BuildResult or oracle result naming)."""
    g = lambda *names: next(getattr(shard, x) for x in names if hasattr(shard, x))
    size_acc = np.asarray(g("bucket_size_acc", "size_acc"), dtype=np.uint64)
    pos_acc = np.asarray(g("bucket_pos_acc", "pos_acc"), dtype=np.uint64)
    return SimpleNamespace(
        n=int(size_acc[-1]), nbuckets=len(size_acc) - 1, bucket_size_acc=size_acc.copy(), bucket_pos_acc=pos_acc.copy(),
        descriptors=np.asarray(g("descriptors", "desc"), dtype=np.uint64).copy(), desc_bits=int(pos_acc[-1]) + 1,
        ribbon_keys=np.asarray(shard.ribbon_keys, dtype=np.uint64).copy(),
        ribbon_bits=np.asarray(shard.ribbon_bits, dtype=np.uint8).copy())


def shard_offsets(shard, group=None, device=None):
    """(key offset, bit offset) of this rank's buckets in the whole structure (all-gather of the
    per-rank key and code-bit counts, then an exclusive scan)."""
    import torch
    dist = _dist()
    world, rank = dist.get_world_size(group), dist.get_rank(group)
    a = _arrays(shard) if shard is not None else None
    mine = torch.tensor([a.n if a else 0, a.desc_bits - 1 if a else 0], dtype=torch.int64, device=device)
    allc = [torch.empty_like(mine) for _ in range(world)]
    dist.all_gather(allc, mine, group=group)
    counts = np.array([c.cpu().tolist() for c in allc], dtype=np.int64)
    return int(counts[:rank, 0].sum()), int(counts[:rank, 1].sum())


def gather_merge(shard, variant, leaf_size, bucket_size, dst=0, group=None):
    """Gather the shard arrays on rank `dst` and join them there; returns the merged result on
    `dst` and None elsewhere."""
    dist = _dist()
    world, rank = dist.get_world_size(group), dist.get_rank(group)
    mine = None if shard is None else vars(_arrays(shard))
    objs = [None] * world if rank == dst else None
    dist.gather_object(mine, objs, dst=dst, group=group)
    if rank != dst:
        return None
    parts = [SimpleNamespace(**o) for o in objs if o is not None]
    return merge_shards(variant, leaf_size, parts, bucket_size)
