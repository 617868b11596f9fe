"""The C ABI library without a GPU: it loads, exports every symbol include/shg.h declares, and its
host-side functions agree with the oracle."""
import os
import re
import subprocess

import numpy as np
import pytest

import shockhash_b200 as shg

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    with open(os.path.join(ROOT, "include", "shg.h")) as f:
        text = f.read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(shg_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_declared_symbols():
    shg.lib()
    out = subprocess.check_output(["nm", "-D", "--defined-only", shg.LIB_PATH]).decode()
    exported = set(re.findall(r" T (shg_\w+)", out))
    missing = [s for s in declared_symbols() if s not in exported]
    assert not missing, missing
    assert len(declared_symbols()) >= 20


def test_library_has_no_unresolved_own_symbols():
    out = subprocess.check_output(["nm", "-D", "--undefined-only", shg.LIB_PATH]).decode()
    assert not re.findall(r"\bshg_\w+", out)


def test_no_device_is_an_error_not_a_fallback():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(shg.ShgError) as ei:
        shg.Engine(0)
    assert ei.value.status == 6
    import ctypes
    p, r, h = shg._Params(2, 64, 2000, 0, 0), shg._Result(), ctypes.c_void_p()
    acc = np.zeros(2, np.uint64)
    r.nbuckets = 1
    r.bucket_size_acc = r.bucket_pos_acc = acc.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64))
    assert shg.lib().shg_dmphf_create(0, ctypes.byref(p), ctypes.byref(r), ctypes.byref(h)) == 6


@pytest.mark.parametrize("variant,leaves", [(1, [2, 5, 8, 24, 30, 40, 60]), (2, [2, 9, 10, 33, 64, 100, 128])])
def test_memo_tables_match_oracle(port, variant, leaves):
    for leaf in leaves:
        assert np.array_equal(shg.memo_table(variant, leaf), port.memo(variant, leaf))


def test_leaf_query_matches_oracle(port):
    rng = np.random.default_rng(4)
    for m in [1, 2, 3, 9, 10, 11, 33, 64, 100, 128]:
        for _ in range(50):
            seed = int(rng.integers(0, 2**40))
            key = int(rng.integers(0, 2**63))
            ret = int(rng.integers(0, 2))
            assert shg.sh2_query(m, seed, key, ret) == port.lib.port_sh2_leaf_query(m, seed, key, ret)


def test_invalid_arguments_rejected():
    with pytest.raises(shg.ShgError):
        shg.memo_table(1, 61)
    with pytest.raises(shg.ShgError):
        shg.memo_table(4, 10)
    # ShockHash<l, true> keeps the memo table of ShockHash<l, false> (ShockHash.h:145)
    assert np.array_equal(shg.memo_table(3, 30), shg.memo_table(1, 30))
