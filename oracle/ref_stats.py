"""Oracle helper (test and CPU-baseline infrastructure): phase times of the compiled reference.

Builds `--n` keys of the benchmark's std::mt19937_64 stream (each hashed as its 8-byte string with
the reference's SpookyV2) once, on ONE thread, through oracle/_ref/libshref_stats.so: the
reference's sources compiled with their own -DSTATS timers (ShockHash.h:37-44,
ShockHash2.h:268-290,314-388), whose counters are plain globals and so need a single thread.
Prints, as its last line on stdout, a JSON object with the constructor's wall time and the
reference's totals for the leaf searches and the split levels. Run it as a subprocess: the STATS
build prints its own report to stdout first.

    python oracle/ref_stats.py --n 200000 --variant 2 --leaf 64 --bucket 2000 --seed 7
"""
import argparse
import ctypes
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))

from oracle.bindings import STATS_SO, RefLib, _ptr  # noqa: E402


def phase_times(keys, variant, leaf, bucket):
    lib = RefLib(STATS_SO)
    L = lib.lib
    L.ref_spooky128.argtypes = [ctypes.c_char_p, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_void_p, ctypes.c_void_p]
    L.ref_stats_times.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
    data = keys.astype("<u8").tobytes()
    offs = np.arange(0, 8 * (len(keys) + 1), 8, dtype=np.uint64)
    first = np.zeros(len(keys), np.uint64)
    second = np.zeros(len(keys), np.uint64)
    L.ref_spooky128(data, _ptr(offs), len(keys), _ptr(first), _ptr(second))
    t = np.zeros(2, np.uint64)
    L.ref_stats_times(_ptr(t[:1]), _ptr(t[1:]))  # read and zero what earlier builds left
    t0 = time.perf_counter()
    b = lib.build_hash(variant, leaf, first, second, bucket, 1)
    wall = time.perf_counter() - t0
    b.free()
    leaves_ns, splits_ns = ctypes.c_uint64(0), ctypes.c_uint64(0)
    L.ref_stats_times(ctypes.byref(leaves_ns), ctypes.byref(splits_ns))
    return {"keys": len(keys), "threads": 1, "total_ms": round(wall * 1e3, 3),
            "leaves_ms": round(leaves_ns.value * 1e-6, 3), "splits_ms": round(splits_ns.value * 1e-6, 3)}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--n", type=int, default=200_000)
    ap.add_argument("--variant", type=int, default=2)
    ap.add_argument("--leaf", type=int, default=64)
    ap.add_argument("--bucket", type=int, default=2000)
    ap.add_argument("--seed", type=int, default=7)
    a = ap.parse_args()
    from oracle.bindings import keys_mt19937_64  # the benchmark's key stream, drawn by the oracle
    keys = keys_mt19937_64(a.seed, a.n)
    res = phase_times(keys, a.variant, a.leaf, a.bucket)
    ctypes.CDLL(None).fflush(None)  # the STATS report (C stdio) goes out before the JSON line
    sys.stdout.flush()
    print(json.dumps(res), flush=True)


if __name__ == "__main__":
    main()
