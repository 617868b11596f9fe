"""Large inputs from pageable host memory (numpy arrays, Python bytes) take the engine's pinned
staging path (two buffers of 64 MB filled by host threads while the copy engine drains the other):
the products equal those of the same keys given another way."""
import numpy as np
import pytest

import shockhash_b200 as shg

pytestmark = pytest.mark.gpu


def same_products(a, b):
    return (np.array_equal(a.descriptors, b.descriptors) and np.array_equal(a.bucket_size_acc, b.bucket_size_acc)
            and np.array_equal(a.bucket_pos_acc, b.bucket_pos_acc) and np.array_equal(a.ribbon_keys, b.ribbon_keys)
            and np.array_equal(a.ribbon_bits, b.ribbon_bits))


def test_pageable_u64_and_string_inputs_equal_device_input(engine):
    import torch
    n = 20_000_000  # 160 MB of keys: above the staging threshold
    keys = shg.keys_mt19937_64(5, n)
    d = torch.from_numpy(keys.view(np.int64)).to("cuda")
    r_dev = engine.build_u64_device(shg.SHOCKHASH2, 64, d.data_ptr(), n, 2000)
    r_host = engine.build_u64(shg.SHOCKHASH2, 64, keys, 2000)
    assert same_products(r_dev, r_host)
    r_host.free()
    # the same keys as 8-byte strings: 160 MB of bytes and 160 MB of offsets, both staged
    data = np.ascontiguousarray(keys, dtype="<u8").tobytes()
    offs = np.arange(0, 8 * (n + 1), 8, dtype=np.uint64)
    r_str = engine.build_strings(shg.SHOCKHASH2, 64, (data, offs), 2000)
    assert same_products(r_dev, r_str)
    r_str.free()
    r_dev.free()
