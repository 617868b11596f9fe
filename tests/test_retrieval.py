"""Retrieval structure without a GPU: the library's host query reads structures built by the Python
restatement of the format (tests/retrieval_model.py), and bad arguments are rejected."""
import numpy as np
import pytest

import shockhash_b200 as shg
import retrieval_model as rm

from conftest import unique_u64


def test_restatement_retrieves_every_bit():
    rng = np.random.default_rng(5)
    keys = [int(k) for k in unique_u64(rng, 2500)]
    bits = [int(b) for b in rng.integers(0, 2, len(keys))]
    lb, sol, thr = rm.build(keys, bits)
    assert all(rm.query(lb, sol, thr, k) == b for k, b in zip(keys, bits))
    assert len(lb) >= 1 and sum(lb) == len(thr) and len(sol) == 4 * len(thr)
    assert max(thr) <= rm.PRIO


@pytest.mark.parametrize("n", [0, 1, 7, 240, 3000])
def test_host_query_reads_restated_structure(n):
    rng = np.random.default_rng(100 + n)
    keys = unique_u64(rng, n)
    bits = rng.integers(0, 2, n).astype(np.uint8)
    lb, sol, thr = rm.build([int(k) for k in keys], [int(b) for b in bits])
    r = shg.Retrieval.load(lb, sol, thr, n)
    assert r.levels() == len(lb)
    assert np.array_equal(r.query(keys), bits)
    lb2, sol2, thr2 = r.arrays()
    assert np.array_equal(lb2, np.array(lb, np.uint64))
    assert np.array_equal(sol2, np.array(sol, np.uint64)) and np.array_equal(thr2, np.array(thr, np.uint8))
    assert r.bits() == 264 * len(thr) + 64 * len(lb)
    # keys outside the set get some bit, never an error
    other = r.query(unique_u64(np.random.default_rng(7), 100))
    assert set(np.unique(other)) <= {0, 1}
    r.close()


def test_load_rejects_bad_arrays():
    with pytest.raises(shg.ShgError):
        shg.Retrieval.load([2], np.zeros(4, np.uint64), np.zeros(1, np.uint8))  # counts disagree
    with pytest.raises(shg.ShgError):
        shg.Retrieval.load([0], np.zeros(0, np.uint64), np.zeros(0, np.uint8))  # empty level
    with pytest.raises(shg.ShgError):
        shg.Retrieval.load(np.ones(41, np.uint64), np.zeros(4 * 41, np.uint64), np.zeros(41, np.uint8))


def test_device_query_of_loaded_structure_is_refused():
    r = shg.Retrieval.load([1], np.zeros(4, np.uint64), np.zeros(1, np.uint8))
    with pytest.raises(shg.ShgError):
        r.query_device(0, 0, 0)
