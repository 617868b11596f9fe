"""B200 ShockHash construction engine — Python host interface over ``libshg.so`` (include/shg.h).

Mirrors the reference's public classes (paths relative to the ShockHash reference project):

* ``ShockHash[l](keys, bucket_size, num_threads=1)``  — ``shockhash::ShockHash<l, false>``
  (include/ShockHash.h:134-191); ``ShockHash[l, True]`` — ``ShockHash<l, true>`` (rotation fitting)
* ``ShockHash2[l](keys, bucket_size, num_threads=1)`` — ``shockhash::ShockHash2<l>``
  (include/ShockHash2.h:117-170)

with ``obj(key)`` (operator()), ``obj.size()``, ``obj.getBits()`` and ``obj.printBits()``. ``keys``
is a list of ``str``/``bytes`` (hashed with SpookyHash V2 on the device, as the reference's string
constructors do), or a pair of uint64 arrays ``(first, second)`` standing for ``hash128_t`` values.
``num_threads`` is accepted for signature compatibility; construction runs on the GPU.

The CUDA library must be built (``python -m shockhash_b200.build``); there is no CPU fallback:
every entry point raises ``ShgError`` when the library or a CUDA device is missing.
"""
import ctypes
import os

import numpy as np

__all__ = ["ShgError", "Engine", "BuildResult", "ShockHash", "ShockHash2", "ShockHash2Flat", "SIMDShockHash", "lib",
           "LIB_PATH", "SHOCKHASH", "SHOCKHASH2", "SHOCKHASH_ROTATION", "SIMDSHOCKHASH", "SIMDSHOCKHASH_ROTATION",
           "MODE_DEFAULT", "MODE_LEVELS", "MODE_PER_LEAF", "MODE_PIPELINED"]

LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "_lib", "libshg.so")

SHOCKHASH, SHOCKHASH2, SHOCKHASH_ROTATION = 1, 2, 3
SIMDSHOCKHASH, SIMDSHOCKHASH_ROTATION = 5, 6  # shg_variant (4 is ShockHash2Flat's tuning-table key)
MODE_DEFAULT, MODE_LEVELS, MODE_PER_LEAF, MODE_PIPELINED, MODE_QUEUE = 0, 1, 2, 3, 4
_STATUS = {0: "OK", 1: "ERR_ARG", 2: "ERR_OOM", 3: "ERR_TRIAL_LIMIT", 4: "ERR_CUDA", 5: "ERR_BUCKET",
           6: "ERR_NO_DEVICE"}
STAGES = ("hash", "partition", "plan", "splits", "leaves", "encode", "copy_out", "total")
WORK = ("split_evals", "leaf_evals", "pairs", "pairs_filtered", "uf_edges", "leaves", "split_nodes", "launches")


class ShgError(RuntimeError):
    def __init__(self, status, msg):
        self.status = status
        super().__init__(f"shg {_STATUS.get(status, status)}: {msg}")


class _Params(ctypes.Structure):
    _fields_ = [("variant", ctypes.c_int), ("leaf_size", ctypes.c_int), ("bucket_size", ctypes.c_uint64),
                ("mode", ctypes.c_int), ("max_trials", ctypes.c_uint64)]


class _Result(ctypes.Structure):
    _fields_ = [("n", ctypes.c_uint64), ("nbuckets", ctypes.c_uint64),
                ("bucket_size_acc", ctypes.POINTER(ctypes.c_uint64)),
                ("bucket_pos_acc", ctypes.POINTER(ctypes.c_uint64)),
                ("descriptors", ctypes.POINTER(ctypes.c_uint64)), ("desc_words", ctypes.c_uint64),
                ("desc_bits", ctypes.c_uint64), ("ribbon_keys", ctypes.POINTER(ctypes.c_uint64)),
                ("ribbon_bits", ctypes.POINTER(ctypes.c_uint8)), ("ribbon_n", ctypes.c_uint64),
                ("stage_ms", ctypes.c_double * 8), ("work", ctypes.c_uint64 * 8), ("owner", ctypes.c_void_p)]


class _BatchItem(ctypes.Structure):
    _fields_ = [("keys", ctypes.c_void_p), ("first", ctypes.c_void_p), ("second", ctypes.c_void_p),
                ("n", ctypes.c_uint64), ("nb_global", ctypes.c_uint64), ("b0", ctypes.c_uint64), ("b1", ctypes.c_uint64)]


class _FlatResult(ctypes.Structure):
    _fields_ = [("n", ctypes.c_uint64), ("k", ctypes.c_uint64), ("nbuckets", ctypes.c_uint64), ("layers", ctypes.c_uint64),
                ("layer_bases", ctypes.c_uint64 * 3), ("threshold_bits", ctypes.c_uint32), ("seed_bits", ctypes.c_uint32),
                ("thresholds_and_seeds", ctypes.POINTER(ctypes.c_uint64)), ("nfallback_seeds", ctypes.c_uint64),
                ("fallback_seed_buckets", ctypes.POINTER(ctypes.c_uint64)),
                ("fallback_seeds", ctypes.POINTER(ctypes.c_uint64)), ("nfree", ctypes.c_uint64),
                ("free_positions", ctypes.POINTER(ctypes.c_uint64)), ("nfallback_keys", ctypes.c_uint64),
                ("fallback", _Result), ("ribbon_keys", ctypes.POINTER(ctypes.c_uint64)),
                ("ribbon_bits", ctypes.POINTER(ctypes.c_uint8)), ("ribbon_n", ctypes.c_uint64),
                ("stage_ms", ctypes.c_double * 8), ("owner", ctypes.c_void_p)]


_lib = None
_vp = ctypes.c_void_p
_u64 = ctypes.c_uint64


def lib():
    """The loaded ``libshg.so``; raises ShgError when it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ShgError(6, f"{LIB_PATH} is missing; build it with `python -m shockhash_b200.build`")
    L = ctypes.CDLL(LIB_PATH)
    P, R = ctypes.POINTER(_Params), ctypes.POINTER(_Result)
    sig = {
        "shg_engine_create": ([ctypes.c_int, ctypes.POINTER(_vp)], ctypes.c_int),
        "shg_engine_destroy": ([_vp], None),
        "shg_build_hash128": ([_vp, P, _vp, _vp, _u64, R], ctypes.c_int),
        "shg_build_hash128_device": ([_vp, P, _vp, _vp, _u64, R], ctypes.c_int),
        "shg_build_u64": ([_vp, P, _vp, _u64, R], ctypes.c_int),
        "shg_build_u64_device": ([_vp, P, _vp, _u64, R], ctypes.c_int),
        "shg_build_strings": ([_vp, P, ctypes.c_char_p, _vp, _u64, R], ctypes.c_int),
        "shg_result_free": ([R], None),
        "shg_result_save": ([P, R, ctypes.c_char_p], ctypes.c_int),
        "shg_result_load": ([ctypes.c_char_p, P, R], ctypes.c_int),
        "shg_build_batch_u64": ([_vp, P, _vp, _vp, _u64, _vp], ctypes.c_int),
        "shg_build_shard_hash128": ([_vp, P, _vp, _vp, _u64, _u64, _u64, _u64, R], ctypes.c_int),
        "shg_build_shard_hash128_device": ([_vp, P, _vp, _vp, _u64, _u64, _u64, _u64, R], ctypes.c_int),
        "shg_shard_partition": ([_vp, _vp, _u64, _u64, ctypes.c_int, _vp, _vp], ctypes.c_int),
        "shg_hash_u64_device": ([_vp, _vp, _u64, _vp, _vp], ctypes.c_int),
        "shg_hash_u64_host": ([_vp, _u64, _vp, _vp, ctypes.c_int], ctypes.c_int),
        "shg_partition_u64": ([_vp, _vp, _u64, _u64, ctypes.c_int, _vp, _vp], ctypes.c_int),
        "shg_build_batch_items": ([_vp, P, _vp, _u64, _vp], ctypes.c_int),
        "shg_shard_partition_device": ([_vp, _vp, _vp, _u64, _u64, ctypes.c_int, _vp, _vp], ctypes.c_int),
        "shg_merge_shards": ([P, _vp, _u64, R], ctypes.c_int),
        "shg_hash_strings": ([_vp, ctypes.c_char_p, _vp, _u64, _vp, _vp], ctypes.c_int),
        "shg_sh2_construct_leaves": ([_vp, _vp, _vp, _u64, _vp, _vp], ctypes.c_int),
        "shg_sh1_construct_leaves": ([_vp, _vp, _vp, _u64, ctypes.c_int, _vp, _vp, _vp], ctypes.c_int),
        "shg_sh2_query": ([_u64, _u64, _u64, _u64], _u64),
        "shg_memo_table": ([ctypes.c_int, ctypes.c_int, _vp], ctypes.c_int),
        "shg_last_error": ([], ctypes.c_char_p),
        "shg_mphf_create": ([P, R, ctypes.POINTER(_vp)], ctypes.c_int),
        "shg_mphf_destroy": ([_vp], None),
        "shg_mphf_query_hash": ([_vp, _vp, _vp, _u64, _vp], ctypes.c_int),
        "shg_mphf_query_strings": ([_vp, ctypes.c_char_p, _vp, _u64, _vp], ctypes.c_int),
        "shg_mphf_bits": ([_vp], _u64),
        "shg_mphf_size": ([_vp], _u64),
        "shg_dmphf_create": ([ctypes.c_int, P, R, ctypes.POINTER(_vp)], ctypes.c_int),
        "shg_dmphf_destroy": ([_vp], None),
        "shg_dmphf_query_hash128": ([_vp, _vp, _vp, _u64, _vp], ctypes.c_int),
        "shg_dmphf_query_u64": ([_vp, _vp, _u64, _vp], ctypes.c_int),
        "shg_dmphf_query_strings": ([_vp, ctypes.c_char_p, _vp, _u64, _vp], ctypes.c_int),
        "shg_dmphf_query_hash128_device": ([_vp, _vp, _vp, _u64, _vp], ctypes.c_int),
        "shg_dmphf_query_u64_device": ([_vp, _vp, _u64, _vp], ctypes.c_int),
        "shg_dmphf_bits": ([_vp], _u64),
        "shg_dmphf_size": ([_vp], _u64),
        "shg_dmphf_last_kernel_ms": ([_vp], ctypes.c_float),
        "shg_dmphf_create_compact": ([ctypes.c_int, P, R, ctypes.POINTER(_vp)], ctypes.c_int),
        "shg_dmphf_retrieval_bits": ([_vp], _u64),
        "shg_dflat_create": ([ctypes.c_int, ctypes.POINTER(_FlatResult), ctypes.POINTER(_vp)], ctypes.c_int),
        "shg_dflat_destroy": ([_vp], None),
        "shg_dflat_query_strings": ([_vp, ctypes.c_char_p, _vp, _u64, _vp], ctypes.c_int),
        "shg_dflat_query_hash": ([_vp, _vp, _u64, _vp], ctypes.c_int),
        "shg_dflat_last_kernel_ms": ([_vp], ctypes.c_float),
        "shg_sh2_construct_leaves_noalloc": ([_vp, _vp, _u64, _vp, _vp, _vp], ctypes.c_int),
        "shg_build_flat_strings": ([_vp, _u64, ctypes.c_char_p, _vp, _u64, ctypes.POINTER(_FlatResult)], ctypes.c_int),
        "shg_flat_result_free": ([ctypes.POINTER(_FlatResult)], None),
        "shg_flat_create": ([ctypes.POINTER(_FlatResult), ctypes.POINTER(_vp)], ctypes.c_int),
        "shg_flat_destroy": ([_vp], None),
        "shg_flat_query_strings": ([_vp, ctypes.c_char_p, _vp, _u64, _vp], ctypes.c_int),
        "shg_flat_query_hash": ([_vp, _vp, _u64, _vp], ctypes.c_int),
        "shg_flat_bits": ([_vp], _u64),
        "shg_retrieval_build": ([_vp, _vp, _vp, _u64, ctypes.POINTER(_vp)], ctypes.c_int),
        "shg_retrieval_build_device": ([_vp, _vp, _vp, _u64, ctypes.POINTER(_vp)], ctypes.c_int),
        "shg_retrieval_load": ([_vp, ctypes.c_uint32, _vp, _vp, _u64, ctypes.POINTER(_vp)], ctypes.c_int),
        "shg_retrieval_destroy": ([_vp], None),
        "shg_retrieval_query": ([_vp, _vp, _u64, _vp], ctypes.c_int),
        "shg_retrieval_query_device": ([_vp, _vp, _u64, _vp], ctypes.c_int),
        "shg_retrieval_levels": ([_vp], ctypes.c_uint32),
        "shg_retrieval_buckets": ([_vp, ctypes.c_uint32], _u64),
        "shg_retrieval_solutions": ([_vp], _vp),
        "shg_retrieval_thresholds": ([_vp], _vp),
        "shg_retrieval_bits": ([_vp], _u64),
        "shg_retrieval_build_ms": ([_vp], ctypes.c_float),
        "shg_retrieval_query_ms": ([_vp], ctypes.c_float),
        "shg_device_memory": ([ctypes.c_int, ctypes.POINTER(_u64), ctypes.POINTER(_u64)], ctypes.c_int),
        "shg_engine_last_work": ([_vp, _vp, ctypes.c_int], ctypes.c_int),
        "shg_engine_set_tuning": ([_vp, ctypes.c_int, ctypes.c_int, ctypes.c_char_p, ctypes.c_int64], ctypes.c_int),
        "shg_engine_get_tuning": ([_vp, ctypes.c_int, ctypes.c_int, ctypes.c_char_p, ctypes.POINTER(ctypes.c_int64)],
                                  ctypes.c_int),
        "shg_engine_load_tuning": ([_vp, ctypes.c_char_p], ctypes.c_int),
        "shg_engine_tuning_source": ([_vp], ctypes.c_char_p),
        "shg_keys_mt19937_64": ([_u64, _u64, _vp], None),
        "shg_keys_mix": ([_u64, _u64, _vp, ctypes.c_int], None),
        "shg_int_peak": ([ctypes.c_int, _u64, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double)],
                         ctypes.c_int),
        "shg_int_peak_kind": ([ctypes.c_int, ctypes.c_int, _u64, ctypes.POINTER(ctypes.c_double),
                               ctypes.POINTER(ctypes.c_double)], ctypes.c_int),
    }
    for name, (args, res) in sig.items():
        fn = getattr(L, name)
        fn.argtypes = args
        fn.restype = res
    _lib = L
    return L


def _check(st):
    if st != 0:
        raise ShgError(st, lib().shg_last_error().decode())


def _ptr(a):
    return ctypes.c_void_p(a.ctypes.data)


def pack_strings(keys):
    """list of str/bytes -> (bytes, offsets[n+1] uint64); an already packed (bytes, offsets) pair
    passes through unchanged."""
    if isinstance(keys, tuple) and len(keys) == 2 and isinstance(keys[0], (bytes, bytearray)):
        return bytes(keys[0]), np.ascontiguousarray(keys[1], dtype=np.uint64)
    bs = [k.encode() if isinstance(k, str) else bytes(k) for k in keys]
    data = b"".join(bs)
    offs = np.zeros(len(bs) + 1, dtype=np.uint64)
    if bs:
        np.cumsum(np.fromiter((len(k) for k in bs), dtype=np.uint64, count=len(bs)), out=offs[1:])
    return data, offs


def keys_mt19937_64(seed, n):
    """n uint64 keys from std::mt19937_64(seed), duplicates redrawn (the benchmark key sets)."""
    out = np.zeros(n, dtype=np.uint64)
    lib().shg_keys_mt19937_64(seed, n, _ptr(out))
    return out


def hash_u64_host(keys, threads=8):
    """128-bit fingerprints (first, second) of uint64 keys hashed as 8-byte strings, on the host."""
    keys = np.ascontiguousarray(keys, dtype=np.uint64)
    f = np.empty(len(keys), np.uint64)
    s = np.empty(len(keys), np.uint64)
    _check(lib().shg_hash_u64_host(_ptr(keys), len(keys), _ptr(f), _ptr(s), threads))
    return f, s


def keys_mix(seed, n, threads=8):
    """n distinct uint64 keys remix(seed ^ (j * 0x9E3779B97F4A7C15)), j < n (the serving stream's
    per-request key sets; fast enough to draw at submit time)."""
    out = np.empty(n, dtype=np.uint64)
    lib().shg_keys_mix(seed, n, _ptr(out), threads)
    return out


def device_memory(device=0):
    """(free, total) device memory in bytes."""
    f, t = _u64(), _u64()
    _check(lib().shg_device_memory(device, ctypes.byref(f), ctypes.byref(t)))
    return f.value, t.value


def int_peak(device=0, iters=1 << 16, kind=0):
    """Measured evaluations/s of a search's inner-loop arithmetic with no memory traffic
    (kind 0 = split quarter moments, 1 = original leaf coverage, 2 = bipartite raw seeds,
    3 / 4 / 5 = split compare-and-count with 1 / 2 / 3 part thresholds)."""
    e, ms = ctypes.c_double(), ctypes.c_double()
    _check(lib().shg_int_peak_kind(device, kind, iters, ctypes.byref(e), ctypes.byref(ms)))
    return e.value, ms.value


SPLIT_KINDS = ("thresholds_1", "thresholds_2", "thresholds_3", "quarter_moments")
# Launch parameters of the search kernels (shg_engine_set_tuning); FLAT is the tuning table's
# variant key of ShockHash2Flat<k>.
TUNING_PARAMS = ("split_seeds_per_lane", "split_threads", "split_round_div", "split_arith", "leaf_blocks_per_sm",
                 "leaf_min_blocks", "sh1_seeds_per_lane", "queue_lag_rounds")
TUNING_FLAT = 4


def split_peaks(device=0, iters=1 << 15, detail=None, simd=False):
    """Measured evaluations/s of each split inner loop, keyed as SPLIT_KINDS: the faster of the two
    arithmetic forms the split kernel can run (split_arith 0 and 1), so the ceiling holds for both.
    `detail`, a dict, receives both forms' rates per kind. `simd`: the loops under SIMDShockHash's
    split hash, which has one form."""
    if simd:
        out = {name: int_peak(device, iters, k)[0] for name, k in zip(SPLIT_KINDS, (17, 18, 19, 16))}
        if detail is not None:
            detail.update({name: {"simd": v} for name, v in out.items()})
        return out
    plain, pipes = (3, 4, 5, 0), (10, 11, 12, 9)
    out = {}
    for name, a, b in zip(SPLIT_KINDS, plain, pipes):
        ra, rb = int_peak(device, iters, a)[0], int_peak(device, iters, b)[0]
        out[name] = max(ra, rb)
        if detail is not None:
            detail[name] = {"arith_0": ra, "arith_1": rb}
    return out


LEAF_OPS = ("hash_evals", "scan_tests", "pair_tests", "uf_edges")


def leaf_peaks(device=0, iters=1 << 15, large=False):
    """Measured operations/s of the bipartite leaf search's inner loops, keyed as LEAF_OPS:
    hashing (remix, fastrange64, mask), candidate-scan mask pairs, isolated-key pair filter,
    pseudoforest (union-find) edges; `large` for leaves of more than 64 keys."""
    kinds = (2, 13, 14, 15) if large else (2, 6, 7, 8)
    out = {name: int_peak(device, iters, k)[0] for name, k in zip(LEAF_OPS, kinds)}
    if large:  # the scan's mask test in both of its forms: the faster one bounds the loop
        out["scan_tests"] = max(out["scan_tests"], int_peak(device, iters, 20)[0])
    return out


def leaf_ceiling_s(counts, peaks):
    """Seconds the bipartite leaf stage's operations take at their loops' measured peaks (the
    stage's roofline: the sum over the four operation kinds of count / peak)."""
    return sum(counts[k] / peaks[k] for k in LEAF_OPS if counts.get(k))


def weighted_split_peak(kind_evals, peaks):
    """The split stage's ceiling for a build: its useful evaluations over the time each node kind's
    evaluations take at that kind's measured peak (a harmonic mean weighted by evaluations)."""
    total = sum(kind_evals[k] for k in SPLIT_KINDS)
    t = sum(kind_evals[k] / peaks[k] for k in SPLIT_KINDS if kind_evals[k])
    return total / t if t > 0 else float("nan")


def sh2_construct_leaves_noalloc(d_keys, d_leaf_offsets, nleaves, d_seeds, d_bits, stream=0):
    """Bipartite leaf search without any device allocation (fixed 16 MiB library scratch).

    All arguments are device addresses (ints) on the current device: keys, leaf_offsets[nleaves+1]
    (leaves of 2..64 keys), seeds[nleaves], bits[total keys]; ``stream`` a cudaStream_t handle."""
    _check(lib().shg_sh2_construct_leaves_noalloc(_vp(d_keys), _vp(d_leaf_offsets), nleaves, _vp(d_seeds),
                                                   _vp(d_bits), _vp(stream)))


def load_result(path):
    """A build result saved with ``BuildResult.save`` (its configuration in ``.params``)."""
    p, res = _Params(), _Result()
    _check(lib().shg_result_load(os.fsencode(path), ctypes.byref(p), ctypes.byref(res)))
    return BuildResult(p, res, None)


def memo_table(variant, leaf_size):
    out = np.zeros(3000, dtype=np.uint64)
    _check(lib().shg_memo_table(variant, leaf_size, _ptr(out)))
    return out


def sh2_query(leaf_size, seed, key, retrieved):
    return int(lib().shg_sh2_query(leaf_size, seed, key, retrieved))


class BuildResult:
    """Products of one device build. The arrays are numpy views of the engine's pinned host block
    (no copy); they stay valid until ``free()`` (also called on garbage collection) or until the
    engine is destroyed."""

    def __init__(self, params, res, engine):
        self.params, self._res, self._engine = params, res, engine
        n, nb = res.n, res.nbuckets
        self.n, self.nbuckets = n, nb
        view = np.ctypeslib.as_array
        self.bucket_size_acc = view(res.bucket_size_acc, (nb + 1,))
        self.bucket_pos_acc = view(res.bucket_pos_acc, (nb + 1,))
        self.descriptors = view(res.descriptors, (res.desc_words,))
        self.desc_bits = res.desc_bits
        rn = res.ribbon_n
        self.ribbon_keys = view(res.ribbon_keys, (max(rn, 1),))[:rn]
        self.ribbon_bits = view(res.ribbon_bits, (max(rn, 1),))[:rn]
        self.stage_ms = dict(zip(STAGES, list(res.stage_ms)))
        self.work = dict(zip(WORK, [int(x) for x in res.work]))

    def free(self):
        if self._res is not None:
            lib().shg_result_free(ctypes.byref(self._res))
            self._res = None

    def save(self, path):
        """Write the result to a file (``shg_result_save``); ``load_result`` reads it back."""
        if self._res is None:
            raise ShgError(1, "build result already freed")
        _check(lib().shg_result_save(ctypes.byref(self.params), ctypes.byref(self._res), os.fsencode(path)))

    def mphf(self):
        """Host query object (``operator()``, ``getBits()``) over this result."""
        return _Mphf(self.params, self._res)

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


class Engine:
    """One CUDA device + stream with resident buffers (shg_engine)."""

    def __init__(self, device=0):
        h = _vp()
        _check(lib().shg_engine_create(device, ctypes.byref(h)))
        self._h = h

    def close(self):
        if getattr(self, "_h", None):
            lib().shg_engine_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_tuning(self, variant, leaf_size, **params):
        """Set launch parameters of one configuration (names in TUNING_PARAMS; speed only)."""
        for name, v in params.items():
            _check(lib().shg_engine_set_tuning(self._h, variant, leaf_size, name.encode(), int(v)))

    def get_tuning(self, variant, leaf_size):
        """The launch parameters this engine uses for a configuration, as a dict."""
        out = {}
        for name in TUNING_PARAMS:
            v = ctypes.c_int64()
            _check(lib().shg_engine_get_tuning(self._h, variant, leaf_size, name.encode(), ctypes.byref(v)))
            out[name] = int(v.value)
        return out

    def load_tuning(self, path):
        _check(lib().shg_engine_load_tuning(self._h, os.fsencode(path)))

    def tuning_source(self):
        """Path of the tuning table loaded at creation ("" if none)."""
        return lib().shg_engine_tuning_source(self._h).decode()

    def last_work(self):
        """Work counts of this engine's last build beyond BuildResult.work: useful split evaluations
        by inner loop (SPLIT_KINDS), split level launches, bipartite candidate-scan mask tests."""
        k = np.zeros(13, np.uint64)
        _check(lib().shg_engine_last_work(self._h, _ptr(k), 13))
        out = {name: int(v) for name, v in zip(SPLIT_KINDS, k[:4])}
        out["split_launches"] = int(k[4])
        out["leaf_scan_tests"] = int(k[5])
        out["flat_leaves"] = {"hash_evals": int(k[8]), "pair_tests": int(k[9]), "pairs_filtered": int(k[10]),
                              "uf_edges": int(k[11]), "scan_tests": int(k[12])}
        return out

    @staticmethod
    def params(variant, leaf_size, bucket_size=2000, mode=MODE_DEFAULT, max_trials=0):
        return _Params(variant, leaf_size, bucket_size, mode, max_trials)

    def _finish(self, p, st, res, keep_raw=False):
        if st != 0:
            _check(st)
        out = BuildResult(p, res, self)
        if keep_raw:
            out._mphf = _Mphf(p, res)
        return out

    def build_hash128(self, variant, leaf_size, first, second, bucket_size=2000, mode=MODE_DEFAULT, max_trials=0,
                      query=False):
        first = np.ascontiguousarray(first, dtype=np.uint64)
        second = np.ascontiguousarray(second, dtype=np.uint64)
        p, res = self.params(variant, leaf_size, bucket_size, mode, max_trials), _Result()
        st = lib().shg_build_hash128(self._h, ctypes.byref(p), _ptr(first), _ptr(second), len(first), ctypes.byref(res))
        return self._finish(p, st, res, query)

    def build_u64(self, variant, leaf_size, keys, bucket_size=2000, mode=MODE_DEFAULT, max_trials=0, query=False):
        keys = np.ascontiguousarray(keys, dtype=np.uint64)
        p, res = self.params(variant, leaf_size, bucket_size, mode, max_trials), _Result()
        st = lib().shg_build_u64(self._h, ctypes.byref(p), _ptr(keys), len(keys), ctypes.byref(res))
        return self._finish(p, st, res, query)

    def build_batch_u64(self, variant, leaf_size, key_arrays, bucket_size=2000, mode=MODE_DEFAULT):
        """One batched construction of several independent uint64 key sets; returns one
        BuildResult per key set (each identical to building that set alone)."""
        arrays = [np.ascontiguousarray(k, dtype=np.uint64) for k in key_arrays]
        R = len(arrays)
        ptrs = (ctypes.c_void_p * R)(*[a.ctypes.data for a in arrays])
        ns = np.array([len(a) for a in arrays], dtype=np.uint64)
        outs = (_Result * R)()
        p = self.params(variant, leaf_size, bucket_size, mode, 0)
        st = lib().shg_build_batch_u64(self._h, ctypes.byref(p), ptrs, _ptr(ns), R, outs)
        _check(st)
        results = []
        for r in range(R):
            res = _Result()
            ctypes.memmove(ctypes.byref(res), ctypes.byref(outs[r]), ctypes.sizeof(_Result))
            results.append(BuildResult(p, res, self))
        return results

    def build_batch_items(self, variant, leaf_size, items, bucket_size=2000, mode=MODE_DEFAULT):
        """One batched construction of mixed items (shg_build_batch_items): each item a dict with
        "keys" (uint64 keys) or "first"/"second" (fingerprints), optionally "nb_global", "b0", "b1"
        for a bucket-range piece of a larger structure. Returns one BuildResult per item."""
        keep, arr = [], (_BatchItem * len(items))()
        for it, d in zip(arr, items):
            if d.get("keys") is not None:
                k = np.ascontiguousarray(d["keys"], dtype=np.uint64)
                keep.append(k)
                it.keys, it.n = k.ctypes.data, len(k)
            else:
                f = np.ascontiguousarray(d["first"], dtype=np.uint64)
                sc = np.ascontiguousarray(d["second"], dtype=np.uint64)
                keep += [f, sc]
                it.first, it.second, it.n = f.ctypes.data, sc.ctypes.data, len(f)
            it.nb_global, it.b0, it.b1 = d.get("nb_global", 0), d.get("b0", 0), d.get("b1", 0)
        outs = (_Result * len(items))()
        p = self.params(variant, leaf_size, bucket_size, mode, 0)
        _check(lib().shg_build_batch_items(self._h, ctypes.byref(p), arr, len(items), outs))
        results = []
        for r in range(len(items)):
            res = _Result()
            ctypes.memmove(ctypes.byref(res), ctypes.byref(outs[r]), ctypes.sizeof(_Result))
            results.append(BuildResult(p, res, self))
        return results

    def build_shard_hash128(self, variant, leaf_size, first, second, nb_global, b0, b1, bucket_size=2000,
                            mode=MODE_DEFAULT):
        """Buckets [b0, b1) of a structure with nb_global buckets, from exactly the keys in them."""
        first = np.ascontiguousarray(first, dtype=np.uint64)
        second = np.ascontiguousarray(second, dtype=np.uint64)
        p, res = self.params(variant, leaf_size, bucket_size, mode, 0), _Result()
        st = lib().shg_build_shard_hash128(self._h, ctypes.byref(p), _ptr(first), _ptr(second), len(first), nb_global,
                                           b0, b1, ctypes.byref(res))
        return self._finish(p, st, res)

    def partition_u64(self, keys, nb, parts):
        """Fingerprints of host uint64 keys made and ordered by bucket range on this engine's GPU
        (shg_partition_u64): an (n, 2) uint64 array of (first, second) pairs, range by range in
        input order, and the key count of each of the `parts` ranges of nb buckets."""
        keys = np.ascontiguousarray(keys, dtype=np.uint64)
        pairs = np.empty((len(keys), 2), np.uint64)
        counts = np.zeros(parts, np.uint64)
        _check(lib().shg_partition_u64(self._h, _ptr(keys), len(keys), nb, parts, _ptr(pairs), _ptr(counts)))
        return pairs, counts

    def hash_u64_device(self, d_keys_ptr, n, d_first_ptr, d_second_ptr):
        """Fingerprints of n device-resident uint64 keys into device buffers (synchronous)."""
        _check(lib().shg_hash_u64_device(self._h, _vp(d_keys_ptr), n, _vp(d_first_ptr), _vp(d_second_ptr)))

    def build_shard_hash128_device(self, variant, leaf_size, d_first_ptr, d_second_ptr, n, nb_global, b0, b1,
                                   bucket_size=2000, mode=MODE_DEFAULT):
        """build_shard_hash128 with the fingerprints in device memory (pointers on the engine's device)."""
        p, res = self.params(variant, leaf_size, bucket_size, mode, 0), _Result()
        st = lib().shg_build_shard_hash128_device(self._h, ctypes.byref(p), _vp(d_first_ptr), _vp(d_second_ptr), n,
                                                  nb_global, b0, b1, ctypes.byref(res))
        return self._finish(p, st, res)

    def build_u64_device(self, variant, leaf_size, d_keys_ptr, n, bucket_size=2000, mode=MODE_DEFAULT):
        p, res = self.params(variant, leaf_size, bucket_size, mode, 0), _Result()
        st = lib().shg_build_u64_device(self._h, ctypes.byref(p), _vp(d_keys_ptr), n, ctypes.byref(res))
        return self._finish(p, st, res)

    def build_strings(self, variant, leaf_size, keys, bucket_size=2000, mode=MODE_DEFAULT, max_trials=0,
                      query=False):
        data, offs = pack_strings(keys)
        p, res = self.params(variant, leaf_size, bucket_size, mode, max_trials), _Result()
        st = lib().shg_build_strings(self._h, ctypes.byref(p), data, _ptr(offs), len(offs) - 1, ctypes.byref(res))
        return self._finish(p, st, res, query)

    def build_flat_strings(self, k, keys):
        """ShockHash2Flat<k>(keys) on the device (include/ShockHash2Flat.h:66-171)."""
        data, offs = pack_strings(keys)
        res = _FlatResult()
        _check(lib().shg_build_flat_strings(self._h, k, data, _ptr(offs), len(offs) - 1, ctypes.byref(res)))
        return FlatBuild(res, self)

    def hash_strings(self, keys):
        data, offs = pack_strings(keys)
        n = len(offs) - 1
        f = np.zeros(n, np.uint64)
        s = np.zeros(n, np.uint64)
        _check(lib().shg_hash_strings(self._h, data, _ptr(offs), n, _ptr(f), _ptr(s)))
        return f, s

    def sh2_construct_leaves(self, keys, leaf_offsets):
        keys = np.ascontiguousarray(keys, dtype=np.uint64)
        offs = np.ascontiguousarray(leaf_offsets, dtype=np.uint64)
        nl = len(offs) - 1
        seeds = np.zeros(max(nl, 1), np.uint64)
        bits = np.zeros(max(len(keys), 1), np.uint8)
        _check(lib().shg_sh2_construct_leaves(self._h, _ptr(keys), _ptr(offs), nl, _ptr(seeds), _ptr(bits)))
        return seeds[:nl], bits[:len(keys)]

    def sh1_construct_leaves(self, keys, leaf_offsets, level=0):
        keys = np.ascontiguousarray(keys, dtype=np.uint64)
        offs = np.ascontiguousarray(leaf_offsets, dtype=np.uint64)
        nl = len(offs) - 1
        codes = np.zeros(max(nl, 1), np.uint64)
        kc = np.zeros(max(len(keys), 1), np.uint64)
        bits = np.zeros(max(len(keys), 1), np.uint8)
        _check(lib().shg_sh1_construct_leaves(self._h, _ptr(keys), _ptr(offs), nl, level, _ptr(codes), _ptr(kc),
                                              _ptr(bits)))
        return codes[:nl], kc[:len(keys)], bits[:len(keys)]


class FlatBuild:
    """Products of a ShockHash2Flat<k> build (views of the engine's pinned block) plus its query
    object: ``query_strings(keys)`` is operator()(const string&), ``bits()`` getBits()."""

    def __init__(self, res, engine):
        self._res, self._engine = res, engine
        v = np.ctypeslib.as_array
        self.n, self.k, self.nbuckets, self.layers = res.n, res.k, res.nbuckets, res.layers
        self.layer_bases = np.array(list(res.layer_bases)[:res.layers + 1], np.uint64)
        nb = max(res.nbuckets, 1)
        self.thresholds_and_seeds = v(res.thresholds_and_seeds, (nb,))[:res.nbuckets]
        nfs = max(res.nfallback_seeds, 1)
        self.fallback_seed_buckets = v(res.fallback_seed_buckets, (nfs,))[:res.nfallback_seeds]
        self.fallback_seeds = v(res.fallback_seeds, (nfs,))[:res.nfallback_seeds]
        self.free_positions = v(res.free_positions, (max(res.nfree, 1),))[:res.nfree]
        rn = max(res.ribbon_n, 1)
        self.ribbon_keys = v(res.ribbon_keys, (rn,))[:res.ribbon_n]
        self.ribbon_bits = v(res.ribbon_bits, (rn,))[:res.ribbon_n]
        self.nfallback_keys = res.nfallback_keys
        self.stage_ms = list(res.stage_ms)
        h = _vp()
        _check(lib().shg_flat_create(ctypes.byref(res), ctypes.byref(h)))
        self._q = h

    def query_strings(self, keys):
        data, offs = pack_strings(keys)
        out = np.zeros(len(offs) - 1, np.uint64)
        _check(lib().shg_flat_query_strings(self._q, data, _ptr(offs), len(offs) - 1, _ptr(out)))
        return out

    def query_hash(self, mhc):
        mhc = np.ascontiguousarray(mhc, dtype=np.uint64)
        out = np.zeros(len(mhc), np.uint64)
        _check(lib().shg_flat_query_hash(self._q, _ptr(mhc), len(mhc), _ptr(out)))
        return out

    def bits(self):
        return int(lib().shg_flat_bits(self._q))

    def device_query(self, device=0):
        """A DeviceFlat over this build (operator() on the GPU for many keys per call)."""
        return DeviceFlat(self, device)

    def free(self):
        if getattr(self, "_q", None):
            lib().shg_flat_destroy(self._q)
            self._q = None
        if self._res is not None:
            lib().shg_flat_result_free(ctypes.byref(self._res))
            self._res = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


class DeviceFlat:
    """ShockHash2Flat<k> operator() on the GPU (``shg_dflat_*``); outputs equal the host query."""

    def __init__(self, flat_build, device=0):
        if flat_build._res is None:
            raise ShgError(1, "flat build already freed")
        h = _vp()
        _check(lib().shg_dflat_create(device, ctypes.byref(flat_build._res), ctypes.byref(h)))
        self._h = h

    def query_strings(self, keys):
        data, offs = pack_strings(keys)
        out = np.zeros(len(offs) - 1, np.uint64)
        _check(lib().shg_dflat_query_strings(self._h, data, _ptr(offs), len(offs) - 1, _ptr(out)))
        return out

    def query_hash(self, mhc):
        mhc = np.ascontiguousarray(mhc, dtype=np.uint64)
        out = np.zeros(len(mhc), np.uint64)
        _check(lib().shg_dflat_query_hash(self._h, _ptr(mhc), len(mhc), _ptr(out)))
        return out

    def last_kernel_ms(self):
        return float(lib().shg_dflat_last_kernel_ms(self._h))

    def close(self):
        if self._h:
            lib().shg_dflat_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class _Mphf:
    def __init__(self, p, res):
        h = _vp()
        _check(lib().shg_mphf_create(ctypes.byref(p), ctypes.byref(res), ctypes.byref(h)))
        self._h = h

    def query_hash(self, first, second):
        first = np.ascontiguousarray(first, dtype=np.uint64)
        second = np.ascontiguousarray(second, dtype=np.uint64)
        out = np.zeros(len(first), np.uint64)
        _check(lib().shg_mphf_query_hash(self._h, _ptr(first), _ptr(second), len(first), _ptr(out)))
        return out

    def query_strings(self, keys):
        data, offs = pack_strings(keys)
        out = np.zeros(len(offs) - 1, np.uint64)
        _check(lib().shg_mphf_query_strings(self._h, data, _ptr(offs), len(offs) - 1, _ptr(out)))
        return out

    def bits(self):
        return int(lib().shg_mphf_bits(self._h))

    def __del__(self):
        try:
            if self._h:
                lib().shg_mphf_destroy(self._h)
        except Exception:
            pass


def merge_shards(variant, leaf_size, shards, bucket_size=2000):
    """Join shard results (bucket order) into the result of one build over all their keys.
    ``shards`` are BuildResults or objects with the same array attributes (numpy uint64/uint8)."""
    R = len(shards)
    arr = (_Result * R)()
    keep = []
    for g, sh in enumerate(shards):
        cols = {}
        for name, dt in (("bucket_size_acc", np.uint64), ("bucket_pos_acc", np.uint64), ("descriptors", np.uint64),
                         ("ribbon_keys", np.uint64), ("ribbon_bits", np.uint8)):
            a = np.ascontiguousarray(getattr(sh, name), dtype=dt)
            if a.size == 0:
                a = np.zeros(1, dt)
            keep.append(a)
            cols[name] = a
        r = arr[g]
        r.n = int(sh.n)
        r.nbuckets = int(sh.nbuckets)
        r.bucket_size_acc = cols["bucket_size_acc"].ctypes.data_as(ctypes.POINTER(ctypes.c_uint64))
        r.bucket_pos_acc = cols["bucket_pos_acc"].ctypes.data_as(ctypes.POINTER(ctypes.c_uint64))
        r.descriptors = cols["descriptors"].ctypes.data_as(ctypes.POINTER(ctypes.c_uint64))
        r.desc_words = len(sh.descriptors)
        r.desc_bits = int(cols["bucket_pos_acc"][-1]) + 1  # code bits + the sentinel
        r.ribbon_keys = cols["ribbon_keys"].ctypes.data_as(ctypes.POINTER(ctypes.c_uint64))
        r.ribbon_bits = cols["ribbon_bits"].ctypes.data_as(ctypes.POINTER(ctypes.c_uint8))
        r.ribbon_n = len(sh.ribbon_keys)
    p = Engine.params(variant, leaf_size, bucket_size)
    out = _Result()
    _check(lib().shg_merge_shards(ctypes.byref(p), arr, R, ctypes.byref(out)))
    return BuildResult(p, out, None)


class DeviceMphf:
    """operator() evaluated on the GPU for many keys per call (``shg_dmphf_*``), over a build result.
    Outputs equal the host query key for key. The result may be freed afterwards. ``compact=True``
    reads the retrieval bit from the compact structure built on the device (``Retrieval``) instead of
    an exact table; outputs then equal the host query for the keys of the build."""

    def __init__(self, result, device=0, compact=False):
        if result._res is None:
            raise ShgError(1, "build result already freed")
        h = _vp()
        create = lib().shg_dmphf_create_compact if compact else lib().shg_dmphf_create
        _check(create(device, ctypes.byref(result.params), ctypes.byref(result._res), ctypes.byref(h)))
        self._h = h

    def query_hash(self, first, second):
        first = np.ascontiguousarray(first, dtype=np.uint64)
        second = np.ascontiguousarray(second, dtype=np.uint64)
        out = np.zeros(len(first), np.uint64)
        _check(lib().shg_dmphf_query_hash128(self._h, _ptr(first), _ptr(second), len(first), _ptr(out)))
        return out

    def query_u64(self, keys):
        keys = np.ascontiguousarray(keys, dtype=np.uint64)
        out = np.zeros(len(keys), np.uint64)
        _check(lib().shg_dmphf_query_u64(self._h, _ptr(keys), len(keys), _ptr(out)))
        return out

    def query_strings(self, keys):
        data, offs = pack_strings(keys)
        out = np.zeros(len(offs) - 1, np.uint64)
        _check(lib().shg_dmphf_query_strings(self._h, data, _ptr(offs), len(offs) - 1, _ptr(out)))
        return out

    def query_u64_device(self, d_keys, n, d_out):
        """Device pointers (ints); synchronous."""
        _check(lib().shg_dmphf_query_u64_device(self._h, _vp(d_keys), n, _vp(d_out)))

    def last_kernel_ms(self):
        return float(lib().shg_dmphf_last_kernel_ms(self._h))

    def bits(self):
        return int(lib().shg_dmphf_bits(self._h))

    def retrieval_bits(self):
        """Size of the retrieval part actually held on the device (compact structure or table)."""
        return int(lib().shg_dmphf_retrieval_bits(self._h))

    def size(self):
        return int(lib().shg_dmphf_size(self._h))

    def close(self):
        if self._h:
            lib().shg_dmphf_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Retrieval:
    """Compact 1-bit retrieval structure built on the GPU from a retrieval input (``shg_retrieval_*``):
    the role of SimpleRibbon<1, w> in the reference (ShockHash.h:657, ShockHash2.h:497), in this
    library's own format (levels of ~240-key buckets, a 256-bit GF(2) solution and an 8-bit priority
    threshold per bucket). ``query`` returns the stored bit of every input key."""

    def __init__(self, handle):
        self._h = handle

    @classmethod
    def build(cls, engine, keys, bits):
        keys = np.ascontiguousarray(keys, dtype=np.uint64)
        bits = np.ascontiguousarray(bits, dtype=np.uint8)
        if len(keys) != len(bits):
            raise ShgError(1, "keys and bits differ in length")
        h = _vp()
        _check(lib().shg_retrieval_build(engine._h, _ptr(keys), _ptr(bits), len(keys), ctypes.byref(h)))
        return cls(h)

    @classmethod
    def build_device(cls, engine, d_keys, d_bits, n):
        """Device pointers (ints) to n uint64 keys and n uint8 bits."""
        h = _vp()
        _check(lib().shg_retrieval_build_device(engine._h, _vp(d_keys), _vp(d_bits), n, ctypes.byref(h)))
        return cls(h)

    @classmethod
    def load(cls, level_buckets, solutions, thresholds, n=0):
        """A structure from its arrays (host queries only)."""
        lb = np.ascontiguousarray(level_buckets, dtype=np.uint64)
        sol = np.ascontiguousarray(solutions, dtype=np.uint64)
        thr = np.ascontiguousarray(thresholds, dtype=np.uint8)
        if len(sol) != 4 * len(thr) or int(lb.sum()) != len(thr):
            raise ShgError(1, "solution, threshold and bucket counts disagree")
        h = _vp()
        _check(lib().shg_retrieval_load(_ptr(lb), len(lb), _ptr(sol), _ptr(thr), n, ctypes.byref(h)))
        return cls(h)

    def query(self, keys):
        keys = np.ascontiguousarray(keys, dtype=np.uint64)
        out = np.zeros(len(keys), np.uint8)
        _check(lib().shg_retrieval_query(self._h, _ptr(keys), len(keys), _ptr(out)))
        return out

    def query_device(self, d_keys, n, d_out):
        """Device pointers (ints); synchronous."""
        _check(lib().shg_retrieval_query_device(self._h, _vp(d_keys), n, _vp(d_out)))

    def levels(self):
        return int(lib().shg_retrieval_levels(self._h))

    def level_buckets(self):
        return np.array([lib().shg_retrieval_buckets(self._h, l) for l in range(self.levels())], dtype=np.uint64)

    def arrays(self):
        """(level buckets, solutions [4 words per bucket], thresholds) copied out."""
        lb = self.level_buckets()
        nb = int(lb.sum())
        if nb == 0:
            return lb, np.zeros(0, np.uint64), np.zeros(0, np.uint8)
        sol = np.ctypeslib.as_array(ctypes.cast(lib().shg_retrieval_solutions(self._h), ctypes.POINTER(ctypes.c_uint64)),
                                    (4 * nb,)).copy()
        thr = np.ctypeslib.as_array(ctypes.cast(lib().shg_retrieval_thresholds(self._h), ctypes.POINTER(ctypes.c_uint8)),
                                    (nb,)).copy()
        return lb, sol, thr

    def bits(self):
        return int(lib().shg_retrieval_bits(self._h))

    def build_ms(self):
        return float(lib().shg_retrieval_build_ms(self._h))

    def query_ms(self):
        return float(lib().shg_retrieval_query_ms(self._h))

    def close(self):
        if getattr(self, "_h", None):
            lib().shg_retrieval_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


_default_engines = {}


def default_engine(device=0):
    if device not in _default_engines:
        _default_engines[device] = Engine(device)
    return _default_engines[device]


class _RecSplitBase:
    VARIANT = None
    LEAF = None

    def __init__(self, keys, bucket_size, num_threads=1, mode=MODE_DEFAULT, engine=None):
        if self.LEAF is None:
            raise TypeError("pick a leaf size first, e.g. ShockHash2[64](keys, 2000)")
        eng = engine or default_engine()
        if isinstance(keys, tuple) and len(keys) == 2:
            self._strings = False
            r = eng.build_hash128(self.VARIANT, self.LEAF, keys[0], keys[1], bucket_size, mode, query=True)
        else:
            self._strings = True
            r = eng.build_strings(self.VARIANT, self.LEAF, keys, bucket_size, mode, query=True)
        self.result = r
        self._mphf = r._mphf
        self.keys_count = r.n

    def __call__(self, key):
        """operator(): a str/bytes key, or a (first, second) hash128 pair."""
        if isinstance(key, tuple):
            return int(self._mphf.query_hash(np.array([key[0]], np.uint64), np.array([key[1]], np.uint64))[0])
        return int(self._mphf.query_strings([key])[0])

    def query_many(self, keys):
        if isinstance(keys, tuple):
            return self._mphf.query_hash(keys[0], keys[1])
        return self._mphf.query_strings(keys)

    def size(self):
        return self.keys_count

    def getBits(self):
        return self._mphf.bits()

    def printBits(self):
        r, n = self.result, max(self.keys_count, 1)
        print("trees:  ", r.descriptors.size * 64 / n)
        print("ribbon: ", 8 * ((len(r.ribbon_keys) + 7) // 8) / n)


class _Templated(type):
    _cache = {}

    def __getitem__(cls, params):
        """cls[leaf], or ShockHash[leaf, rotation_fitting] like the reference's template arguments."""
        leaf, rot = (params if isinstance(params, tuple) else (params, False))
        key = (cls.__name__, int(leaf), bool(rot))
        if key not in _Templated._cache:
            attrs = {"LEAF": int(leaf)}
            if rot:
                rotated = {SHOCKHASH: SHOCKHASH_ROTATION, SIMDSHOCKHASH: SIMDSHOCKHASH_ROTATION}
                if cls.VARIANT not in rotated:
                    raise TypeError("rotation fitting exists for ShockHash<l, true> and SIMDShockHash<l, true> only")
                attrs["VARIANT"] = rotated[cls.VARIANT]
            _Templated._cache[key] = type(f"{cls.__name__}[{leaf}{', True' if rot else ''}]", (cls,), attrs)
        return _Templated._cache[key]


class ShockHash(_RecSplitBase, metaclass=_Templated):
    """shockhash::ShockHash<LEAF_SIZE, ROTATION_FITTING> (include/ShockHash.h:134); use ShockHash[l](keys, b)
    or ShockHash[l, True](keys, b) for rotation fitting."""
    VARIANT = SHOCKHASH


class SIMDShockHash(_RecSplitBase, metaclass=_Templated):
    """shockhash::SIMDShockHash<LEAF_SIZE, ROTATION_FITTING> (include/SIMDShockHash.hpp:105), the class the
    reference's SIMD benchmark builds as ShockHash<l>; use SIMDShockHash[l](keys, b) or
    SIMDShockHash[l, True](keys, b) for rotation fitting."""
    VARIANT = SIMDSHOCKHASH


class ShockHash2(_RecSplitBase, metaclass=_Templated):
    """shockhash::ShockHash2<LEAF_SIZE> (include/ShockHash2.h:117); use ShockHash2[l](keys, b)."""
    VARIANT = SHOCKHASH2


class ShockHash2Flat(metaclass=_Templated):
    """shockhash::ShockHash2Flat<k> (include/ShockHash2Flat.h:37); use ShockHash2Flat[k](keys).

    The two extra constructor arguments of the reference (ShockHash2Flat.h:60-64) are accepted and
    ignored, as there."""
    LEAF = None

    def __init__(self, keys, ignore=0, ignore2=0, engine=None):
        if self.LEAF is None:
            raise TypeError("pick k first, e.g. ShockHash2Flat[100](keys)")
        self.result = (engine or default_engine()).build_flat_strings(self.LEAF, keys)
        self.keys_count = self.result.n

    def __call__(self, key):
        if isinstance(key, int):
            return int(self.result.query_hash(np.array([key], np.uint64))[0])
        return int(self.result.query_strings([key])[0])

    def query_many(self, keys):
        return self.result.query_strings(keys)

    def getBits(self):
        return self.result.bits()

    def size(self):
        return self.keys_count
