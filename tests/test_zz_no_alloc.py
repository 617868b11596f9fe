"""The no-allocation bipartite leaf entry point, through the C ABI, against the allocating one.

Collected last on purpose (file name): it runs after every other test in the suite, and also
passes alone in a fresh process. Callers without the right to allocate device memory pass their
own device buffers; the library works in a fixed scratch array of its own device image.
"""
import os

import numpy as np
import pytest

import shockhash_b200 as shg
from conftest import unique_u64

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def leaves_up_to_64():
    g = np.load(os.path.join(GOLDEN, "sh2_leaves.npz"))
    offs = g["offsets"].astype(np.int64)
    sizes = np.diff(offs)
    keep = np.nonzero(sizes <= 64)[0]
    keys = np.concatenate([g["keys"][offs[j]:offs[j + 1]] for j in keep])
    rng = np.random.default_rng(11)
    extra = []
    for _ in range(3000):  # plus a batch of full-size and uneven leaves, as a ShockHash2<64> build has
        extra.append(unique_u64(rng, int(rng.choice([64, 64, 64, 16, 48, 2, 9, 10, 33]))))
    all_keys = np.concatenate([keys] + extra).astype(np.uint64)
    sizes = np.concatenate([sizes[keep], [len(e) for e in extra]])
    leaf_offs = np.concatenate([[0], np.cumsum(sizes)]).astype(np.uint64)
    return all_keys, leaf_offs


def test_noalloc_matches_allocating_entry_point(engine):
    import torch
    keys, offs = leaves_up_to_64()
    nleaves = len(offs) - 1
    want_seeds, want_bits = engine.sh2_construct_leaves(keys, offs)
    dev = torch.device("cuda", 0)
    d_keys = torch.from_numpy(keys.view(np.int64)).to(dev)
    d_offs = torch.from_numpy(offs.view(np.int64)).to(dev)
    for call in range(2):  # the scratch keeps the previous call's contents; results must not depend on it
        d_seeds = torch.full((nleaves,), -1, dtype=torch.int64, device=dev)
        d_bits = torch.full((len(keys),), 7, dtype=torch.uint8, device=dev)
        stream = torch.cuda.current_stream(dev).cuda_stream
        shg.sh2_construct_leaves_noalloc(d_keys.data_ptr(), d_offs.data_ptr(), nleaves, d_seeds.data_ptr(),
                                         d_bits.data_ptr(), stream)
        got_seeds = d_seeds.cpu().numpy().view(np.uint64)
        got_bits = d_bits.cpu().numpy()
        assert np.array_equal(got_seeds, want_seeds), f"seeds differ on call {call}"
        assert np.array_equal(got_bits, want_bits), f"retrieval bits differ on call {call}"


def test_noalloc_rejects_oversized_leaf():
    import torch
    dev = torch.device("cuda", 0)
    rng = np.random.default_rng(12)
    keys = unique_u64(rng, 65 + 64)
    offs = np.array([0, 65, 129], dtype=np.uint64)  # a 65-key leaf is beyond this entry point's maximum
    d_keys = torch.from_numpy(keys.view(np.int64)).to(dev)
    d_offs = torch.from_numpy(offs.view(np.int64)).to(dev)
    d_seeds = torch.zeros(2, dtype=torch.int64, device=dev)
    d_bits = torch.zeros(129, dtype=torch.uint8, device=dev)
    with pytest.raises(shg.ShgError) as ei:
        shg.sh2_construct_leaves_noalloc(d_keys.data_ptr(), d_offs.data_ptr(), 2, d_seeds.data_ptr(),
                                         d_bits.data_ptr(), 0)
    assert ei.value.status == 1 and "64" in str(ei.value)
