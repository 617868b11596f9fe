"""The benchmark key generators (oracle/keygen.h) without a GPU: the oracle's uint64 stream equals the
CUDA library's host generator draw for draw (the timed reference run and the GPU run build the same
keys while the reference process loads no library of this package), and the string generators
follow their stated definitions."""
import numpy as np
import pytest

from oracle import bindings


@pytest.mark.parametrize("seed,n", [(7, 1), (7, 100_000), (11, 250_000), (31, 3), (42, 0)])
def test_oracle_u64_stream_equals_library_generator(port, seed, n):
    import shockhash_b200 as shg
    a = bindings.keys_mt19937_64(seed, n)
    assert np.array_equal(a, shg.keys_mt19937_64(seed, n))
    assert len(np.unique(a)) == n


def test_u64_stream_is_std_mt19937_64(port):
    # the C++ standard's known answer: the 10000th draw of a default-seeded (5489) mt19937_64
    assert int(bindings.keys_mt19937_64(5489, 10000)[-1]) == 9981545732273789042


def test_ref_and_port_generators_agree(ref, port):
    import ctypes
    lib_p = ctypes.CDLL(bindings.PORT_SO)
    fn = lib_p.port_keys_mt19937_64
    fn.argtypes = [ctypes.c_uint64, ctypes.c_uint64, ctypes.c_void_p]
    out = np.empty(5000, np.uint64)
    fn(7, 5000, out.ctypes.data)
    assert np.array_equal(out, bindings.keys_mt19937_64(7, 5000))
    fs = lib_p.port_strings_mt19937_64
    fs.argtypes = [ctypes.c_int, ctypes.c_uint64, ctypes.c_uint64, ctypes.c_char_p, ctypes.c_void_p]
    fs.restype = ctypes.c_uint64
    total = fs(1, 23, 2000, None, None)
    buf = ctypes.create_string_buffer(int(total))
    offs = np.zeros(2001, np.uint64)
    fs(1, 23, 2000, buf, offs.ctypes.data)
    d, o = bindings.strings_mt19937_64(1, 23, 2000)
    assert buf.raw[:total] == d and np.array_equal(offs, o)


def test_printable_strings(port):
    d, o = bindings.strings_mt19937_64(bindings.STRINGS_PRINTABLE, 42, 20_000)
    keys = bindings.split_strings(d, o)
    lens = np.diff(o.astype(np.int64))
    assert lens.min() >= 16 and lens.max() <= 40 and len(set(lens.tolist())) == 25
    arr = np.frombuffer(d, dtype=np.uint8)
    assert arr.min() >= 33 and arr.max() <= 126
    assert len(set(keys)) == len(keys)
    d2, o2 = bindings.strings_mt19937_64(bindings.STRINGS_PRINTABLE, 42, 20_000)
    assert d2 == d and np.array_equal(o2, o)


def test_zipf_strings(port):
    n = 50_000
    d, o = bindings.strings_mt19937_64(bindings.STRINGS_ZIPF, 23, n)
    lens = np.diff(o.astype(np.int64))
    assert lens.min() >= 8 and lens.max() <= 200
    w = np.arange(1, 194, dtype=np.float64) ** -1.1
    p8 = w[0] / w.sum()  # P(l = 8)
    assert abs((lens == 8).mean() - p8) < 0.01
    assert abs(lens.mean() - (np.arange(8, 201) * w).sum() / w.sum()) < 1.0
    keys = bindings.split_strings(d, o)
    assert len(set(keys)) == n
    assert 0 in np.frombuffer(d, dtype=np.uint8)  # NUL bytes occur


def test_bench_synthetic_strings_follow_the_configuration_shapes():
    """bench.py's stand-ins for the string configurations (numpy streams, used by its GPU leg):
    the same lengths, byte ranges and length distribution as the oracle's generators define."""
    import bench
    d, o = bench.synthetic_strings("printable", 42, 20_000)
    lens = np.diff(o.astype(np.int64))
    assert lens.min() >= 16 and lens.max() <= 40 and len(set(lens.tolist())) == 25
    arr = np.frombuffer(d, dtype=np.uint8)
    assert arr.min() >= 33 and arr.max() <= 126 and len(d) == int(o[-1])
    n = 200_000
    d, o = bench.synthetic_strings("zipf", 23, n)
    lens = np.diff(o.astype(np.int64))
    assert lens.min() >= 8 and lens.max() <= 200 and len(d) == int(o[-1])
    w = np.arange(1, 194, dtype=np.float64) ** -1.1
    assert abs((lens == 8).mean() - w[0] / w.sum()) < 0.01
    assert abs(lens.mean() - (np.arange(8, 201) * w).sum() / w.sum()) < 1.0
    d2, o2 = bench.synthetic_strings("zipf", 23, n)
    assert d2 == d and np.array_equal(o2, o)
