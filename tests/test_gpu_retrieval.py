"""Device-built retrieval structure: every input key retrieves its bit (host and device queries),
the device build equals the Python restatement word for word, builds are independent of input
order, and the structure of a ShockHash2 build's retrieval input answers that build's bits."""
import numpy as np
import pytest
import torch

import shockhash_b200 as shg
import retrieval_model as rm

from conftest import unique_u64

pytestmark = pytest.mark.gpu


def _device_query(r, keys):
    d_keys = torch.from_numpy(keys.view(np.int64)).cuda()
    d_out = torch.zeros(len(keys), dtype=torch.uint8, device="cuda")
    r.query_device(d_keys.data_ptr(), len(keys), d_out.data_ptr())
    return d_out.cpu().numpy()


@pytest.mark.parametrize("n", [0, 1, 2, 241, 1000, 100_000, 2_000_000])
def test_every_key_retrieves_its_bit(engine, n):
    rng = np.random.default_rng(n)
    keys = unique_u64(rng, n)
    bits = rng.integers(0, 2, n).astype(np.uint8)
    r = shg.Retrieval.build(engine, keys, bits)
    assert np.array_equal(r.query(keys), bits)
    if n:
        assert np.array_equal(_device_query(r, keys), bits)
    if n >= 100_000:
        assert r.bits() / n < 1.16
        assert r.levels() <= 6
    r.close()


@pytest.mark.parametrize("n", [600, 3000])
def test_device_build_equals_restatement(engine, n):
    rng = np.random.default_rng(40 + n)
    keys = unique_u64(rng, n)
    bits = rng.integers(0, 2, n).astype(np.uint8)
    lb, sol, thr = rm.build([int(k) for k in keys], [int(b) for b in bits])
    r = shg.Retrieval.build(engine, keys, bits)
    lb2, sol2, thr2 = r.arrays()
    assert np.array_equal(lb2, np.array(lb, np.uint64))
    assert np.array_equal(thr2, np.array(thr, np.uint8))
    assert np.array_equal(sol2, np.array(sol, np.uint64))


def test_build_is_independent_of_input_order(engine):
    rng = np.random.default_rng(3)
    keys = unique_u64(rng, 300_000)
    bits = rng.integers(0, 2, len(keys)).astype(np.uint8)
    a = shg.Retrieval.build(engine, keys, bits).arrays()
    perm = rng.permutation(len(keys))
    b = shg.Retrieval.build(engine, keys[perm], bits[perm]).arrays()
    for x, y in zip(a, b):
        assert np.array_equal(x, y)


def test_device_input_and_reload(engine):
    rng = np.random.default_rng(9)
    keys = unique_u64(rng, 50_000)
    bits = rng.integers(0, 2, len(keys)).astype(np.uint8)
    d_keys = torch.from_numpy(keys.view(np.int64)).cuda()
    d_bits = torch.from_numpy(bits).cuda()
    r = shg.Retrieval.build_device(engine, d_keys.data_ptr(), d_bits.data_ptr(), len(keys))
    assert np.array_equal(r.query(keys), bits)
    again = shg.Retrieval.load(*r.arrays(), len(keys))
    assert np.array_equal(again.query(keys), bits)


def test_duplicates(engine):
    keys = np.array([5, 5, 9, 11], np.uint64)
    r = shg.Retrieval.build(engine, keys, np.array([1, 1, 0, 1], np.uint8))
    assert np.array_equal(r.query(keys), [1, 1, 0, 1])
    with pytest.raises(shg.ShgError) as ei:
        shg.Retrieval.build(engine, keys, np.array([1, 0, 0, 1], np.uint8))
    assert ei.value.status == 1  # SHG_ERR_ARG


def test_shockhash2_retrieval_input(engine):
    keys = shg.keys_mt19937_64(7, 1_000_000)
    res = engine.build_u64(shg.SHOCKHASH2, 64, keys, 2000)
    r = shg.Retrieval.build(engine, res.ribbon_keys, res.ribbon_bits)
    assert np.array_equal(r.query(res.ribbon_keys), res.ribbon_bits)
    assert r.bits() / len(res.ribbon_keys) < 1.16


@pytest.mark.parametrize("variant,leaf,n", [(2, 64, 1_000_000), (1, 30, 300_000)])
def test_device_query_with_compact_retrieval(engine, variant, leaf, n):
    keys = unique_u64(np.random.default_rng(800 + leaf), n)
    r = engine.build_u64(variant, leaf, keys, 2000)
    exact = shg.DeviceMphf(r)
    compact = shg.DeviceMphf(r, compact=True)
    out = compact.query_u64(keys)
    assert np.array_equal(out, exact.query_u64(keys))
    assert np.array_equal(np.sort(out), np.arange(n, dtype=np.uint64))
    assert compact.retrieval_bits() < exact.retrieval_bits() / 10
    assert compact.retrieval_bits() / len(r.ribbon_keys) < 1.2
