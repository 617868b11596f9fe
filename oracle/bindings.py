"""Test infrastructure only (the oracle): ctypes bindings to the two CPU checkers.

* ``RefLib``  — ``oracle/_ref/libshref.so``: the reference's own headers compiled against the
  restated third-party stand-ins in ``oracle/shims`` (built by ``make -C oracle ref``).
* ``PortLib`` — ``oracle/_port/libshgport.so``: the C++ restatement in ``oracle/port``
  (built by ``make -C oracle port``).

Only the tests, ``__graft_entry__.smoke()`` and the CPU-baseline leg of ``bench.py`` use this
module. The shipped library never imports it.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def host_has_avx512():
    """Whether this host runs x86-64-v4 code (AVX-512 F, BW, CD, DQ, VL)."""
    try:
        with open("/proc/cpuinfo") as f:
            flags = next((ln for ln in f if ln.startswith("flags")), "").split()
    except OSError:
        return False
    return all(x in flags for x in ("avx512f", "avx512bw", "avx512cd", "avx512dq", "avx512vl"))


# The reference build whose SIMD width matches this host's -march=native (oracle/Makefile).
_V4_DIR = os.path.join(HERE, "_ref", "v4")
REF_DIR = _V4_DIR if host_has_avx512() and os.path.exists(os.path.join(_V4_DIR, "libshref.so")) else os.path.join(HERE, "_ref")
REF_SO = os.path.join(REF_DIR, "libshref.so")
STATS_SO = os.path.join(REF_DIR, "libshref_stats.so")
PORT_SO = os.path.join(HERE, "_port", "libshgport.so")
# SIMDShockHash.hpp built for 4 lanes of 64 bits (x86-64-v3) and for 8 (x86-64-v4)
SIMD_SO = {4: os.path.join(HERE, "_ref", "libshref_simd.so"), 8: os.path.join(_V4_DIR, "libshref_simd.so")}


def ref_build_info():
    """Which compiled reference this process uses: its directory, target ISA and the host's."""
    arch = None
    try:
        with open(os.path.join(REF_DIR, "build_arch.txt")) as f:
            arch = f.read().strip()
    except OSError:
        pass
    return {"dir": os.path.relpath(REF_DIR, os.path.dirname(HERE)), "march": arch, "host_avx512": host_has_avx512(),
            "flags": "-std=c++20 -O3 -DNDEBUG"}

_u64p = ctypes.c_void_p
_vp = ctypes.c_void_p
_sz = ctypes.c_size_t


def _ptr(a):
    return ctypes.c_void_p(a.ctypes.data) if a is not None else ctypes.c_void_p(0)


def pack_strings(keys):
    """bytes keys -> (concatenated bytes, offsets[n+1] uint64)."""
    data = b"".join(keys)
    offs = np.zeros(len(keys) + 1, dtype=np.uint64)
    np.cumsum([len(k) for k in keys], out=offs[1:])
    return data, offs


class Built:
    """Products of one construction, as numpy arrays."""

    def __init__(self, lib, prefix, h):
        self.lib, self.prefix, self.h = lib, prefix, h
        f = lambda name: getattr(lib, prefix + name)
        self.nbuckets = int(f("nbuckets")(_vp(h)))
        nw = int(f("desc_words")(_vp(h)))
        self.desc = np.zeros(nw, dtype=np.uint64)
        f("get_desc")(_vp(h), _ptr(self.desc))
        self.size_acc = np.zeros(self.nbuckets + 1, dtype=np.uint64)
        self.pos_acc = np.zeros(self.nbuckets + 1, dtype=np.uint64)
        f("get_acc")(_vp(h), _ptr(self.size_acc), _ptr(self.pos_acc))
        nr = int(f("ribbon_n")(_vp(h)))
        self.ribbon_keys = np.zeros(nr, dtype=np.uint64)
        self.ribbon_bits = np.zeros(nr, dtype=np.uint8)
        f("get_ribbon")(_vp(h), _ptr(self.ribbon_keys), _ptr(self.ribbon_bits))

    def query_hash(self, first, second):
        first = np.ascontiguousarray(first, dtype=np.uint64)
        second = np.ascontiguousarray(second, dtype=np.uint64)
        out = np.zeros(len(first), dtype=np.uint64)
        getattr(self.lib, self.prefix + "query_hash")(_vp(self.h), _ptr(first), _ptr(second), _sz(len(first)), _ptr(out))
        return out

    def free(self):
        if self.h:
            getattr(self.lib, self.prefix + "free")(_vp(self.h))
            self.h = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


class _Lib:
    prefix = ""

    def __init__(self, path):
        self.path = path
        self.lib = ctypes.CDLL(path)
        for name in ("nbuckets", "desc_words", "ribbon_n", "get_bits"):
            fn = getattr(self.lib, self.prefix + name, None)
            if fn is not None:
                fn.restype = ctypes.c_uint64
                fn.argtypes = [_vp]


class RefSimdLib(_Lib):
    """The reference's SIMDShockHash<leaf, rotation> (oracle/ref_simd_capi.cpp), built for `lanes`
    64-bit lanes (4: AVX2, 8: AVX-512; the 8-lane build needs an AVX-512 host)."""
    prefix = "refsimd_"

    def __init__(self, lanes=None):
        if lanes is None:
            lanes = 8 if host_has_avx512() and os.path.exists(SIMD_SO[8]) else 4
        super().__init__(SIMD_SO[lanes])
        L = self.lib
        L.refsimd_lanes.restype = ctypes.c_uint64
        L.refsimd_build_hash.restype = _vp
        L.refsimd_build_hash.argtypes = [ctypes.c_int, ctypes.c_int, _vp, _vp, _sz, _sz, _sz]
        L.refsimd_build_strings.restype = _vp
        L.refsimd_build_strings.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_char_p, _vp, _sz, _sz, _sz]
        L.refsimd_query_strings.argtypes = [_vp, ctypes.c_char_p, _vp, _sz, _vp]
        L.refsimd_remix_and_remap.argtypes = [_vp, _sz, ctypes.c_uint32, _vp]
        self.lanes = int(L.refsimd_lanes())

    def _built(self, h, leaf):
        if not h:
            raise ValueError(f"leaf size {leaf} not instantiated in the SIMDShockHash oracle")
        b = Built(self.lib, "refsimd_", h)
        b.bits = int(self.lib.refsimd_get_bits(_vp(h)))
        return b

    def build_hash(self, rotation, leaf, first, second, bucket_size=2000, threads=1):
        first = np.ascontiguousarray(first, dtype=np.uint64)
        second = np.ascontiguousarray(second, dtype=np.uint64)
        return self._built(self.lib.refsimd_build_hash(int(rotation), leaf, _ptr(first), _ptr(second), len(first),
                                                       bucket_size, threads), leaf)

    def build_strings(self, rotation, leaf, keys, bucket_size=2000, threads=1):
        data, offs = pack_strings(keys)
        b = self._built(self.lib.refsimd_build_strings(int(rotation), leaf, data, _ptr(offs), len(keys), bucket_size,
                                                       threads), leaf)
        b._strings = (data, offs)
        return b

    def build_strings_packed_timed(self, rotation, leaf, data, offs, bucket_size=2000, threads=1):
        """The constructor from packed string keys; returns (products, seconds of the call alone)."""
        L = self.lib
        L.refsimd_build_strings_timed.restype = _vp
        L.refsimd_build_strings_timed.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_char_p, _vp, _sz, _sz, _sz,
                                                  ctypes.POINTER(ctypes.c_double)]
        secs = ctypes.c_double(0)
        offs = np.ascontiguousarray(offs, dtype=np.uint64)
        h = L.refsimd_build_strings_timed(int(rotation), leaf, data, _ptr(offs), len(offs) - 1, bucket_size, threads,
                                          ctypes.byref(secs))
        return self._built(h, leaf), float(secs.value)

    def query_strings(self, built, keys):
        data, offs = pack_strings(keys)
        out = np.zeros(len(keys), dtype=np.uint64)
        self.lib.refsimd_query_strings(_vp(built.h), data, _ptr(offs), len(keys), _ptr(out))
        return out

    def remix_and_remap(self, x, n):
        """The format's split hash of each value for range n (SIMDShockHash.hpp:762-766)."""
        x = np.ascontiguousarray(x, dtype=np.uint64)
        out = np.zeros(len(x), np.uint32)
        self.lib.refsimd_remix_and_remap(_ptr(x), len(x), n, _ptr(out))
        return out


class RefLib(_Lib):
    prefix = "ref_"

    def __init__(self, path=REF_SO):
        super().__init__(path)
        L = self.lib
        L.ref_build_hash.restype = _vp
        L.ref_build_hash.argtypes = [ctypes.c_int, ctypes.c_int, _vp, _vp, _sz, _sz, _sz]
        L.ref_build_strings.restype = _vp
        L.ref_build_strings.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_char_p, _vp, _sz, _sz, _sz]
        L.ref_sh2_leaf.restype = ctypes.c_uint64
        L.ref_sh2_leaf.argtypes = [_sz, _vp, _vp, _vp]
        L.ref_sh2_leaf_query.restype = ctypes.c_uint64
        L.ref_sh2_leaf_query.argtypes = [_sz, ctypes.c_uint64, ctypes.c_uint64, ctypes.c_uint64]
        L.ref_sh2_pair_check.restype = ctypes.c_int
        L.ref_sh2_pair_check.argtypes = [_sz, _vp, _vp, _vp, _vp]
        L.ref_cuckoo_construct.restype = ctypes.c_int
        L.ref_cuckoo_construct.argtypes = [_vp, _sz, ctypes.c_uint64, _vp, _vp]
        L.ref_sh1_leaf.restype = ctypes.c_uint64
        L.ref_sh1_leaf.argtypes = [ctypes.c_int, _vp, _sz, ctypes.c_int, _vp, _vp]
        L.ref_memo.restype = ctypes.c_int
        L.ref_memo.argtypes = [ctypes.c_int, ctypes.c_int, _vp]
        L.ref_query_strings.argtypes = [_vp, ctypes.c_char_p, _vp, _sz, _vp]

    def build_hash(self, variant, leaf, first, second, bucket_size=2000, threads=1):
        first = np.ascontiguousarray(first, dtype=np.uint64)
        second = np.ascontiguousarray(second, dtype=np.uint64)
        h = self.lib.ref_build_hash(variant, leaf, _ptr(first), _ptr(second), len(first), bucket_size, threads)
        if not h:
            raise ValueError(f"leaf size {leaf} not instantiated in the reference oracle")
        b = Built(self.lib, "ref_", h)
        b.bits = int(self.lib.ref_get_bits(_vp(h)))
        return b

    def build_strings(self, variant, leaf, keys, bucket_size=2000, threads=1):
        data, offs = pack_strings(keys)
        h = self.lib.ref_build_strings(variant, leaf, data, _ptr(offs), len(keys), bucket_size, threads)
        if not h:
            raise ValueError(f"leaf size {leaf} not instantiated in the reference oracle")
        b = Built(self.lib, "ref_", h)
        b.bits = int(self.lib.ref_get_bits(_vp(h)))
        b._strings = (data, offs)
        return b

    def build_strings_packed_timed(self, variant, leaf, data, offs, bucket_size=2000, threads=1):
        """The reference constructor from string keys given packed; returns (products, seconds of the
        constructor call alone)."""
        L = self.lib
        L.ref_build_strings_timed.restype = _vp
        L.ref_build_strings_timed.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_char_p, _vp, _sz, _sz, _sz,
                                              ctypes.POINTER(ctypes.c_double)]
        secs = ctypes.c_double(0)
        offs = np.ascontiguousarray(offs, dtype=np.uint64)
        h = L.ref_build_strings_timed(variant, leaf, data, _ptr(offs), len(offs) - 1, bucket_size, threads,
                                      ctypes.byref(secs))
        if not h:
            raise ValueError(f"leaf size {leaf} not instantiated in the reference oracle")
        b = Built(L, "ref_", h)
        b.bits = int(L.ref_get_bits(_vp(h)))
        return b, float(secs.value)

    def query_packed(self, built, data, offs):
        """operator()(const string&) of a reference build for packed string keys."""
        offs = np.ascontiguousarray(offs, dtype=np.uint64)
        out = np.zeros(len(offs) - 1, dtype=np.uint64)
        self.lib.ref_query_strings(_vp(built.h), data, _ptr(offs), len(offs) - 1, _ptr(out))
        return out

    def query_strings(self, built, keys):
        data, offs = pack_strings(keys)
        out = np.zeros(len(keys), dtype=np.uint64)
        self.lib.ref_query_strings(_vp(built.h), data, _ptr(offs), len(keys), _ptr(out))
        return out

    def memo(self, variant, leaf):
        out = np.zeros(3000, dtype=np.uint64)
        if not self.lib.ref_memo(variant, leaf, _ptr(out)):
            return None
        return out

    def sh2_leaf(self, keys):
        keys = np.ascontiguousarray(keys, dtype=np.uint64)
        m = len(keys)
        rk = np.zeros(m, np.uint64)
        rb = np.zeros(m, np.uint8)
        seed = self.lib.ref_sh2_leaf(m, _ptr(keys), _ptr(rk), _ptr(rb))
        return int(seed), rk, rb

    def flat_build_strings(self, k, keys):
        """ShockHash2Flat<k>(keys) (ShockHash2Flat.h:66-171); returns a dict of its internals."""
        L = self.lib
        L.ref_flat_build_strings.restype = _vp
        L.ref_flat_build_strings.argtypes = [ctypes.c_int, ctypes.c_char_p, _vp, _sz]
        L.ref_flat_bits.restype = ctypes.c_uint64
        L.ref_flat_bits.argtypes = [_vp]
        L.ref_flat_dump.argtypes = [_vp] + [_vp] * 8
        L.ref_flat_query_strings.argtypes = [_vp, ctypes.c_char_p, _vp, _sz, _vp]
        L.ref_flat_free.argtypes = [_vp]
        data, offs = pack_strings(keys)
        h = L.ref_flat_build_strings(k, data, _ptr(offs), len(keys))
        if not h:
            raise ValueError(f"k={k} not instantiated")
        sizes = np.zeros(6, np.uint64)
        L.ref_flat_dump(_vp(h), _ptr(sizes), *([_vp(0)] * 7))
        lb, tas, fbb, fbs, fp = (np.zeros(int(sizes[i]), np.uint64) for i in (0, 1, 2, 2, 3))
        rk, rb = np.zeros(int(sizes[4]), np.uint64), np.zeros(int(sizes[4]), np.uint8)
        L.ref_flat_dump(_vp(h), _ptr(sizes), _ptr(lb), _ptr(tas), _ptr(fbb), _ptr(fbs), _ptr(fp), _ptr(rk), _ptr(rb))
        q = np.zeros(len(keys), np.uint64)
        L.ref_flat_query_strings(_vp(h), data, _ptr(offs), len(keys), _ptr(q))
        out = dict(layer_bases=lb, thresholds_and_seeds=tas, fallback_buckets=fbb, fallback_seeds=fbs,
                   free_positions=fp, ribbon_keys=rk, ribbon_bits=rb, layers=int(sizes[5]), query=q,
                   bits=int(L.ref_flat_bits(_vp(h))))
        L.ref_flat_free(_vp(h))
        return out

    def sh1_leaf(self, leaf, keys, level=0):
        keys = np.ascontiguousarray(keys, dtype=np.uint64)
        m = len(keys)
        rk = np.zeros(m, np.uint64)
        rb = np.zeros(m, np.uint8)
        code = self.lib.ref_sh1_leaf(leaf, _ptr(keys), m, level, _ptr(rk), _ptr(rb))
        return int(code), rk, rb

    def sh2_pair_check(self, a, b):
        """The reference's isolated-vertex filter and union-find on one candidate pair of hash rows:
        (skipped by the filter, all edges accepted)."""
        a = np.ascontiguousarray(a, dtype=np.uint8)
        b = np.ascontiguousarray(b, dtype=np.uint8)
        sk, fo = ctypes.c_int(0), ctypes.c_int(0)
        if not self.lib.ref_sh2_pair_check(len(a), _ptr(a), _ptr(b), ctypes.byref(sk), ctypes.byref(fo)):
            raise ValueError("leaf size not instantiated")
        return bool(sk.value), bool(fo.value)

    def cuckoo_construct(self, keys, seed):
        """The reference's ordered cuckoo insertion under `seed`: (all placed, cell1[], cell2[])."""
        keys = np.ascontiguousarray(keys, dtype=np.uint64)
        m = len(keys)
        c1 = np.zeros(m, np.uint32)
        c2 = np.zeros(m, np.uint32)
        ok = self.lib.ref_cuckoo_construct(_ptr(keys), m, seed, _ptr(c1), _ptr(c2))
        return bool(ok), c1, c2

    def spooky128(self, keys):
        data, offs = pack_strings(keys)
        f = np.zeros(len(keys), np.uint64)
        s = np.zeros(len(keys), np.uint64)
        self.lib.ref_spooky128.argtypes = [ctypes.c_char_p, _vp, _sz, _vp, _vp]
        self.lib.ref_spooky128(data, _ptr(offs), len(keys), _ptr(f), _ptr(s))
        return f, s

    def murmur64(self, keys):
        data, offs = pack_strings(keys)
        out = np.zeros(len(keys), np.uint64)
        self.lib.ref_murmur64.argtypes = [ctypes.c_char_p, _vp, _sz, _vp]
        self.lib.ref_murmur64(data, _ptr(offs), len(keys), _ptr(out))
        return out


class PortLib(_Lib):
    prefix = "port_"

    def __init__(self, path=PORT_SO):
        super().__init__(path)
        L = self.lib
        L.port_build.restype = _vp
        L.port_build.argtypes = [ctypes.c_int, ctypes.c_int, _vp, _vp, ctypes.c_uint64, ctypes.c_uint64]
        L.port_build_shard.restype = _vp
        L.port_build_shard.argtypes = [ctypes.c_int, ctypes.c_int, _vp, _vp, ctypes.c_uint64, ctypes.c_uint64,
                                       ctypes.c_uint64, ctypes.c_uint64, ctypes.c_uint64]
        L.port_node_count.restype = ctypes.c_uint64
        L.port_node_count.argtypes = [_vp]
        L.port_sh2_leaf.restype = ctypes.c_uint64
        L.port_sh2_leaf.argtypes = [ctypes.c_uint32, _vp, _vp, _vp, _vp]
        L.port_sh2_leaf_query.restype = ctypes.c_uint64
        L.port_sh2_leaf_query.argtypes = [ctypes.c_uint32, ctypes.c_uint64, ctypes.c_uint64, ctypes.c_uint64]
        L.port_sh1_leaf.restype = ctypes.c_uint64
        L.port_sh1_leaf.argtypes = [ctypes.c_uint32, ctypes.c_int, _vp, _vp, _vp]
        L.port_memo.argtypes = [ctypes.c_int, ctypes.c_int, _vp]

    def build_hash(self, variant, leaf, first, second, bucket_size=2000):
        first = np.ascontiguousarray(first, dtype=np.uint64)
        second = np.ascontiguousarray(second, dtype=np.uint64)
        h = self.lib.port_build(variant, leaf, _ptr(first), _ptr(second), len(first), bucket_size)
        if not h:
            raise ValueError("port build failed")
        b = Built(self.lib, "port_", h)
        nn = int(self.lib.port_node_count(_vp(h)))
        b.node_codes = np.zeros(nn, np.uint64)
        self.lib.port_get_node_codes(_vp(h), _ptr(b.node_codes))
        b.sorted_keys = np.zeros(len(first), np.uint64)
        self.lib.port_get_sorted_keys(_vp(h), _ptr(b.sorted_keys))
        b.work = np.zeros(7, np.uint64)
        self.lib.port_get_work(_vp(h), _ptr(b.work))
        return b

    def build_shard(self, variant, leaf, first, second, nb_global, b0, b1, bucket_size=2000):
        """Buckets [b0, b1) of a structure with nb_global buckets, from exactly the keys in them."""
        first = np.ascontiguousarray(first, dtype=np.uint64)
        second = np.ascontiguousarray(second, dtype=np.uint64)
        h = self.lib.port_build_shard(variant, leaf, _ptr(first), _ptr(second), len(first), bucket_size, nb_global, b0,
                                      b1)
        if not h:
            raise ValueError("port shard build failed")
        b = Built(self.lib, "port_", h)
        b.n = len(first)
        return b

    def memo(self, variant, leaf):
        out = np.zeros(3000, dtype=np.uint64)
        self.lib.port_memo(variant, leaf, _ptr(out))
        return out

    def spooky128(self, keys):
        data, offs = pack_strings(keys)
        f = np.zeros(len(keys), np.uint64)
        s = np.zeros(len(keys), np.uint64)
        self.lib.port_spooky128.argtypes = [ctypes.c_char_p, _vp, _sz, _vp, _vp]
        self.lib.port_spooky128(data, _ptr(offs), len(keys), _ptr(f), _ptr(s))
        return f, s

    def sh2_leaf(self, keys, with_work=False):
        keys = np.ascontiguousarray(keys, dtype=np.uint64)
        m = len(keys)
        rk = np.zeros(m, np.uint64)
        rb = np.zeros(m, np.uint8)
        w = np.zeros(7, np.uint64)
        seed = self.lib.port_sh2_leaf(m, _ptr(keys), _ptr(rk), _ptr(rb), _ptr(w))
        if with_work:
            return int(seed), rk, rb, w
        return int(seed), rk, rb

    def sh1_leaf(self, keys, level=0):
        keys = np.ascontiguousarray(keys, dtype=np.uint64)
        m = len(keys)
        rk = np.zeros(m, np.uint64)
        rb = np.zeros(m, np.uint8)
        code = self.lib.port_sh1_leaf(m, level, _ptr(keys), _ptr(rk), _ptr(rb))
        return int(code), rk, rb


def _keygen_lib():
    """The compiled reference when present, else the restatement: both export the same generators."""
    if ref_available():
        return ctypes.CDLL(REF_SO), "ref_"
    return ctypes.CDLL(PORT_SO), "port_"


def keys_mt19937_64(seed, n):
    """n uint64 keys from std::mt19937_64(seed), later duplicates redrawn (oracle/keygen.h); the same
    keys, draw for draw, as the CUDA library's benchmark generator."""
    lib, p = _keygen_lib()
    fn = getattr(lib, p + "keys_mt19937_64")
    fn.argtypes = [ctypes.c_uint64, ctypes.c_uint64, _vp]
    fn.restype = None
    out = np.empty(n, dtype=np.uint64)
    fn(seed, n, _ptr(out))
    return out


STRINGS_PRINTABLE, STRINGS_ZIPF = 0, 1


def strings_mt19937_64(kind, seed, n):
    """n distinct string keys from std::mt19937_64(seed) (oracle/keygen.h): kind 0 = lengths 16..40
    of bytes 33..126; kind 1 = Zipf(1.1) lengths 8..200 of bytes 0..255. Returns (bytes, offsets[n+1])."""
    lib, p = _keygen_lib()
    fn = getattr(lib, p + "strings_mt19937_64")
    fn.argtypes = [ctypes.c_int, ctypes.c_uint64, ctypes.c_uint64, ctypes.c_char_p, _vp]
    fn.restype = ctypes.c_uint64
    total = int(fn(kind, seed, n, None, None))
    buf = ctypes.create_string_buffer(max(1, total))
    offs = np.zeros(n + 1, dtype=np.uint64)
    fn(kind, seed, n, buf, _ptr(offs))
    return buf.raw[:total], offs


def split_strings(data, offs):
    """(bytes, offsets) -> list of bytes keys."""
    return [data[int(offs[i]):int(offs[i + 1])] for i in range(len(offs) - 1)]


def ref_available():
    return os.path.exists(REF_SO)


def port_available():
    return os.path.exists(PORT_SO)
