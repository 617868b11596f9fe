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

Two forms of the same steps:
* host arrays (``exchange``, ``build_sharded``, ``gather_merge``): numpy fingerprints, any process
  group;
* tensors (``exchange_tensors``, ``build_sharded_tensors``, ``gather_merge_tensors``): fingerprints
  stay in torch tensors (int64 views of uint64). On a GPU the library's partition kernel
  (shg_shard_partition_device) writes the send buffer, NCCL's all-to-all moves it, and the shard
  build reads the received keys where they landed (shg_build_shard_hash128_device); only the
  per-rank counts go through host memory. Host tensors (gloo) take the library's host partition,
  which gives the same order.
"""
from types import SimpleNamespace

import numpy as np

from . import _ptr, lib, merge_shards, _check


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


# ------------------------------------------------------------------ tensor form
def partition(first, second, nb, world, engine=None):
    """Send buffer and split sizes of the exchange: (pairs [n, 2] int64 tensor in owner-rank order,
    stable; counts numpy int64 [world]). `first`/`second` are int64 tensors (uint64 bits); CUDA
    tensors need `engine` on their device."""
    import torch
    n = first.numel()
    pairs = torch.empty((n, 2), dtype=torch.int64, device=first.device)
    counts = np.zeros(world, dtype=np.uint64)
    if first.is_cuda:
        if engine is None:
            raise ValueError("partitioning device tensors needs an Engine on their device")
        torch.cuda.synchronize(first.device)  # the inputs are complete before the engine's stream reads them
        _check(lib().shg_shard_partition_device(engine._h, first.data_ptr(), second.data_ptr(), n, nb, world,
                                                pairs.data_ptr(), _ptr(counts)))
    else:
        f = np.ascontiguousarray(first.numpy()).view(np.uint64)
        s = np.ascontiguousarray(second.numpy()).view(np.uint64)
        out = pairs.numpy().view(np.uint64)
        _check(lib().shg_shard_partition(_ptr(f), _ptr(s), n, nb, world, _ptr(out), _ptr(counts)))
    return pairs, counts.astype(np.int64)


def exchange_tensors(first, second, nb, group=None, engine=None):
    """All-to-all of fingerprints held in tensors; returns this rank's (first, second) int64 tensors on
    the inputs' device, in (source rank, source position) order. The counts are exchanged first and
    read on the host (the split sizes the collective needs); the payload stays in tensors."""
    import torch
    dist = _dist()
    world = dist.get_world_size(group)
    pairs, counts = partition(first, second, nb, world, engine)
    send = torch.from_numpy(counts).to(first.device)
    recv = torch.empty_like(send)
    dist.all_to_all_single(recv, send, group=group)
    recv_sizes = [int(x) for x in recv.cpu().tolist()]
    out = torch.empty((sum(recv_sizes), 2), dtype=torch.int64, device=first.device)
    dist.all_to_all_single(out, pairs, output_split_sizes=recv_sizes, input_split_sizes=[int(x) for x in counts],
                           group=group)
    return out[:, 0].contiguous(), out[:, 1].contiguous()


def build_sharded_tensors(build_shard, first, second, bucket_size, group=None, engine=None):
    """``build_sharded`` for tensors: ``build_shard(first, second, nb_global, b0, b1)`` receives this
    rank's exchanged int64 tensors (on the GPU for CUDA inputs, e.g. ``lambda f, s, nb, b0, b1:
    engine.build_shard_hash128_device(2, 64, f.data_ptr(), s.data_ptr(), f.numel(), nb, b0, b1)``).
    Returns (shard result or None for an empty range, nb_global, (b0, b1))."""
    import torch
    dist = _dist()
    world, rank = dist.get_world_size(group), dist.get_rank(group)
    t = torch.tensor([first.numel()], dtype=torch.int64, device=first.device)
    dist.all_reduce(t, group=group)
    nb = nbuckets(int(t.item()), bucket_size)
    f, s = exchange_tensors(first, second, nb, group, engine)
    b0, b1 = bucket_ranges(nb, world)[rank]
    if b1 <= b0:
        if f.numel():
            raise RuntimeError("keys arrived at a rank without buckets")
        return None, nb, (b0, b1)
    if f.is_cuda:
        torch.cuda.synchronize(f.device)
    return build_shard(f, s, nb, b0, b1), nb, (b0, b1)


_FIELDS = (("bucket_size_acc", np.uint64), ("bucket_pos_acc", np.uint64), ("descriptors", np.uint64),
           ("ribbon_keys", np.uint64), ("ribbon_bits", np.uint8))


def gather_merge_tensors(shard, variant, leaf_size, bucket_size, dst=0, group=None, device=None):
    """``gather_merge`` with tensor collectives (all-gather of the lengths, then of each array padded
    to the longest; NCCL when `device` is a GPU, gloo on the host) instead of pickled objects; returns
    the merged result on `dst` and None elsewhere."""
    import torch
    dist = _dist()
    world, rank = dist.get_world_size(group), dist.get_rank(group)
    a = _arrays(shard) if shard is not None else None
    cols = [np.ascontiguousarray(getattr(a, k), dtype=dt) if a else np.zeros(0, dt) for k, dt in _FIELDS]
    lens = torch.tensor([len(c) for c in cols], dtype=torch.int64, device=device)
    all_lens = [torch.empty_like(lens) for _ in range(world)]
    dist.all_gather(all_lens, lens, group=group)
    all_lens = np.array([x.cpu().tolist() for x in all_lens], dtype=np.int64)
    parts = [dict() for _ in range(world)]
    for k, ((name, dt), col) in enumerate(zip(_FIELDS, cols)):
        width = max(1, int(all_lens[:, k].max()))
        buf = np.zeros(width, dtype=dt)
        buf[:len(col)] = col
        t = torch.from_numpy(buf.view(np.int64) if dt == np.uint64 else buf).to(device)
        got = [torch.empty_like(t) for _ in range(world)]
        dist.all_gather(got, t, group=group)
        if rank == dst:
            for g in range(world):
                arr = got[g].cpu().numpy()
                parts[g][name] = (arr.view(np.uint64) if dt == np.uint64 else arr)[:int(all_lens[g, k])].copy()
    if rank != dst:
        return None
    shards = []
    for g in range(world):
        if all_lens[g, 1] == 0:  # a rank without buckets
            continue
        d = parts[g]
        shards.append(SimpleNamespace(n=int(d["bucket_size_acc"][-1]), nbuckets=len(d["bucket_size_acc"]) - 1,
                                      desc_bits=int(d["bucket_pos_acc"][-1]) + 1, **d))
    return merge_shards(variant, leaf_size, shards, bucket_size)
