// Batched device query: operator() of ShockHash<l,false> / ShockHash2<l> for many keys at once
// (ShockHash.h:199-270, :277; ShockHash2.h:178-230, :237), over the arrays a construction produced.
//
// One thread per key: fingerprint (SpookyV2-128, fused for uint64 and string keys), bucket by
// remap128, Golomb-Rice walk down the bucket's tree (RiceBitVector.h:149-213 reader: unary part
// from a 64-bit window, fixed part at a separate bit offset, subtree skips by the memo's node and
// fixed-bit counts), the leaf hash, and the retrieval bit from a device hash table. The walk is
// a handful of dependent loads per key, so the kernel is bound by HBM latency and the number of
// loads in flight, not by the arithmetic.
//
// The retrieval structure is an exact open-addressing table (64-bit keys, one bit each, linear
// probing from remix(key)), built on the device from the construction's retrieval input; every
// key of the set retrieves the bit it was given, as with the reference's SimpleRibbon.
#include <cuda_runtime.h>
#include <cstdint>
#include <cstring>
#include <string>
#include "shg.h"
#include "shg_common.cuh"
#include "shg_internal.h"
#include "shg_retrieval.cuh"

using namespace shg;

namespace {

constexpr uint64_t kEmpty = ~0ull;     // empty table slot; the key kEmpty itself lives in `special`
constexpr uint32_t kQErrStream = 1;    // a walk ran past the end of the descriptor stream

struct DView {
    const uint64_t *size_acc, *pos_acc, *desc, *memo;
    const uint64_t *tkey;
    const uint32_t *tbits;
    const uint32_t *special;  // bit 1: key kEmpty present; bit 0: its retrieval bit
    const RetLevels *rlv;     // compact retrieval structure instead of the table (or null)
    const uint64_t *rsol;
    const uint8_t *rthr;
    uint64_t nb, nw, tmask;
    uint32_t lower, upper, leaf;
    int variant;
};

__device__ __forceinline__ uint64_t ldw(const DView &v, uint64_t i) { return i < v.nw ? __ldg(v.desc + i) : 0; }

// RiceBitVector::Reader (RiceBitVector.h:149-213) over device memory; every loop is bounded by the
// stream length, and `bad` is set instead of reading past it.
struct DReader {
    uint64_t fixed_off, window, ptr;
    int valid;
    bool bad;
    __device__ void reset(const DView &v, uint64_t bit_pos, uint64_t unary_off) {
        fixed_off = bit_pos;
        const uint64_t up = bit_pos + unary_off;
        ptr = up / 64;
        window = ldw(v, ptr++) >> (up & 63);
        valid = 64 - (int)(up & 63);
        bad = false;
    }
    __device__ uint64_t next(const DView &v, int g) {
        uint64_t result = 0;
        if (window == 0) {
            result += valid;
            window = ldw(v, ptr++);
            valid = 64;
            while (window == 0) {
                if (ptr > v.nw) {
                    bad = true;
                    return 0;
                }
                result += 64;
                window = ldw(v, ptr++);
            }
        }
        const int pos = __ffsll((long long)window) - 1;
        window >>= pos;
        window >>= 1;
        valid -= pos + 1;
        result += pos;
        result <<= g;
        const uint64_t lo = ldw(v, fixed_off / 64), hi = ldw(v, fixed_off / 64 + 1);
        const int sh = (int)(fixed_off % 64);
        uint64_t f = sh ? (lo >> sh) | (hi << (64 - sh)) : lo;
        f &= (g < 64) ? ((1ull << g) - 1) : ~0ull;
        fixed_off += g;
        return result | f;
    }
    __device__ void skip(const DView &v, uint64_t nodes, uint64_t fixed_len) {
        uint64_t missing = nodes, cnt;
        while ((cnt = (uint64_t)__popcll(window)) < missing) {
            if (ptr > v.nw) {
                bad = true;
                return;
            }
            window = ldw(v, ptr++);
            missing -= cnt;
            valid = 64;
        }
        uint64_t w = window;
        for (uint64_t i = 0; i + 1 < missing; i++) w &= w - 1;
        cnt = (uint64_t)(__ffsll((long long)w) - 1);
        window >>= cnt;
        window >>= 1;
        valid -= (int)cnt + 1;
        fixed_off += fixed_len;
    }
};

__device__ __forceinline__ uint64_t dretrieve(const DView &v, uint64_t key) {
    if (v.rlv) return ret_lookup(*v.rlv, v.rsol, v.rthr, key);
    if (key == kEmpty) return __ldg(v.special) & 1u;
    uint64_t s = remix(key) & v.tmask;
    for (uint64_t probe = 0; probe <= v.tmask; probe++) {
        const uint64_t k = __ldg(v.tkey + s);
        if (k == key) return (__ldg(v.tbits + (s >> 5)) >> (s & 31)) & 1u;
        if (k == kEmpty) return 0;
        s = (s + 1) & v.tmask;
    }
    return 0;
}

__device__ __forceinline__ int golomb(const DView &v, uint32_t m) { return (int)(__ldg(v.memo + m) >> 27); }
__device__ __forceinline__ uint32_t skip_bits(const DView &v, uint32_t m) { return (uint32_t)(__ldg(v.memo + m) & 0xFFFF); }
__device__ __forceinline__ uint32_t skip_nodes(const DView &v, uint32_t m) {
    return (uint32_t)((__ldg(v.memo + m) >> 16) & 0x7FF);
}

// operator()(const hash128_t&) (ShockHash.h:199-270, ShockHash2.h:178-230).
__device__ uint64_t dquery_one(const DView &v, uint64_t first, uint64_t second, bool &bad) {
    const uint64_t bucket = remap128(first, v.nb);
    uint64_t cum = __ldg(v.size_acc + bucket);
    uint32_t m = (uint32_t)(__ldg(v.size_acc + bucket + 1) - cum);
    if (m >= (uint32_t)kMaxBucket) {
        bad = true;
        return 0;
    }
    DReader rd;
    rd.reset(v, __ldg(v.pos_acc + bucket), skip_bits(v, m));
    int level = 0;
    // SIMDShockHash: its own split hash and fixed start seeds below the fanout-2 levels
    // (SIMDShockHash.hpp:785-843)
    const bool simd = is_simd(v.variant);
    auto split_hash = [simd](uint64_t z, uint32_t range) {
        return simd ? remap16(simd_split_low16(z), range) : remap16(remix(z), range);
    };
    while (m > v.upper) {
        const uint64_t d = rd.next(v, golomb(v, m));
        const uint32_t h = split_hash(second + d + start_seed(level), m);
        const uint32_t sp = (uint16_t(m / 2 + v.upper - 1) / v.upper) * v.upper;
        if (h < sp) {
            m = sp;
        } else {
            rd.skip(v, skip_nodes(v, sp), skip_bits(v, sp));
            m -= sp;
            cum += sp;
        }
        level++;
    }
    if (m > v.lower) {
        const uint64_t d = rd.next(v, golomb(v, m));
        const uint32_t h = split_hash(second + d + start_seed(simd ? kSimdSeedLower : level), m);
        const uint32_t part = uint16_t(h) / v.lower;
        m = min(v.lower, m - part * v.lower);
        cum += (uint64_t)v.lower * part;
        if (part) rd.skip(v, (uint64_t)skip_nodes(v, v.lower) * part, (uint64_t)skip_bits(v, v.lower) * part);
        level++;
    }
    if (m > v.leaf) {
        const uint64_t d = rd.next(v, golomb(v, m));
        const uint32_t h = split_hash(second + d + start_seed(simd ? kSimdSeedLeafAggr : level), m);
        const uint32_t part = uint16_t(h) / v.leaf;
        m = min(v.leaf, m - part * v.leaf);
        cum += (uint64_t)v.leaf * part;
        if (part) rd.skip(v, part, (uint64_t)skip_bits(v, v.leaf) * part);
        level++;
    }
    const uint64_t b = rd.next(v, golomb(v, m));
    bad = bad || rd.bad;
    const uint64_t ret = dretrieve(v, second);
    const int leaf_seed = simd ? kSimdSeedLeaf : level;
    if (is_rotation(v.variant) && m == v.leaf) {  // rotation fitting (ShockHash.h:251-265, SIMDShockHash.hpp:826-840)
        const uint32_t r = (uint32_t)(b % m);
        const uint64_t x = b / m + start_seed(leaf_seed);
        uint32_t c1, c2;
        if ((second & 1) == 0) {
            sh1_cells(second, x & ~(uint64_t)(m > 32 ? 7 : 0), m, c1, c2);
            return cum + (ret == 0 ? c1 : c2);
        }
        sh1_cells(second, x, m, c1, c2);
        return cum + ((ret == 0 ? c1 : c2) + r) % m;
    }
    if (is_sh1(v.variant)) {
        uint32_t c1, c2;
        sh1_cells(second, b + start_seed(leaf_seed), m, c1, c2);  // TinyBinaryCuckooHashTable.h:116-123
        return cum + (ret == 0 ? c1 : c2);
    }
    return cum + sh2_leaf_query(m, b, second, ret);
}

enum QIn { kInHash128 = 0, kInU64 = 1, kInStrings = 2 };

template <int IN>
__global__ void __launch_bounds__(256) k_dquery(DView v, const uint64_t *__restrict__ a, const uint64_t *__restrict__ b,
                                                const uint8_t *__restrict__ bytes, uint64_t n, uint64_t *__restrict__ out,
                                                uint32_t *__restrict__ err) {
    bool bad = false;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        uint64_t f, s;
        if (IN == kInHash128) {
            f = a[i];
            s = b[i];
        } else if (IN == kInU64) {
            spooky128_u64(a[i], 0, f, s);
        } else {
            const uint64_t lo = b[i], hi = b[i + 1];
            spooky128(bytes + lo, hi - lo, 0, f, s);
        }
        out[i] = dquery_one(v, f, s, bad);
    }
    if (bad) atomicOr(err, kQErrStream);
}

__global__ void k_table_insert(const uint64_t *__restrict__ keys, const uint8_t *__restrict__ bits, uint64_t n,
                               uint64_t *__restrict__ tkey, uint32_t *__restrict__ tbits, uint32_t *__restrict__ special,
                               uint64_t tmask) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t key = keys[i];
        const uint32_t bit = bits[i] & 1u;
        if (key == kEmpty) {
            atomicOr(special, 2u | bit);
            continue;
        }
        uint64_t s = remix(key) & tmask;
        for (uint64_t probe = 0; probe <= tmask; probe++) {
            const unsigned long long prev =
                atomicCAS((unsigned long long *)(tkey + s), (unsigned long long)kEmpty, (unsigned long long)key);
            if (prev == kEmpty || prev == key) {
                if (bit) atomicOr(tbits + (s >> 5), 1u << (s & 31));
                break;
            }
            s = (s + 1) & tmask;
        }
    }
}

// ---------------------------------------------------------------- ShockHash2Flat<k> on the device
struct FView {
    uint64_t lb[4];                 // layerBases
    uint32_t layers, tb, thr_mask;  // threshold bits, threshold range - 1
    uint32_t k;
    uint64_t nbuckets, nfree, nfs;
    const uint64_t *tas;            // thresholds and seeds, [nbuckets]
    const uint32_t *mapping;        // compact threshold -> 32-bit threshold
    const uint64_t *free_pos;       // freePositions
    const uint64_t *fs_bucket, *fs_seed;  // seedsFallback, ascending buckets
    const uint64_t *tkey;
    const uint32_t *tbits, *special;
    uint64_t tmask;
    bool has_fallback;
};

__device__ __forceinline__ uint64_t fretrieve(const FView &v, uint64_t key) {
    if (key == kEmpty) return __ldg(v.special) & 1u;
    uint64_t s = remix(key) & v.tmask;
    for (uint64_t probe = 0; probe <= v.tmask; probe++) {
        const uint64_t k = __ldg(v.tkey + s);
        if (k == key) return (__ldg(v.tbits + (s >> 5)) >> (s & 31)) & 1u;
        if (k == kEmpty) return 0;
        s = (s + 1) & v.tmask;
    }
    return 0;
}

// std::to_string(uint64_t): decimal digits, no terminator; returns the length.
__device__ __forceinline__ int u64_decimal(uint64_t x, uint8_t *buf) {
    uint8_t tmp[20];
    int n = 0;
    do {
        tmp[n++] = (uint8_t)('0' + x % 10);
        x /= 10;
    } while (x);
    for (int i = 0; i < n; i++) buf[i] = tmp[n - 1 - i];
    return n;
}

// operator()(uint64_t) (ShockHash2Flat.h:266-277) with evaluateKPerfect (:280-301).
__device__ uint64_t dflat_one(const FView &f, const DView &fb, uint64_t hash, bool &bad) {
    uint64_t mhc = hash, bucket = 0, seed = 0;
    bool found = false;
    for (uint32_t layer = 0; layer < f.layers && !found; layer++) {
        if (layer) mhc = remix(mhc);
        const uint64_t base = f.lb[layer];
        const uint32_t size = (uint32_t)(f.lb[layer + 1] - base);
        const uint64_t b = base + fastrange32((uint32_t)mhc, size);
        const uint64_t stored = __ldg(f.tas + b);
        if ((uint32_t)(mhc >> 32) <= __ldg(f.mapping + (stored & f.thr_mask))) {
            bucket = b;
            seed = stored >> f.tb;
            found = true;
        }
    }
    if (!found) {
        // fallback PHF over std::to_string(mhc) (:124-128, :292-300)
        uint64_t phf = 0;
        if (f.has_fallback) {
            uint8_t buf[24];
            const int len = u64_decimal(mhc, buf);
            uint64_t a, b;
            spooky128(buf, (size_t)len, 0, a, b);
            phf = dquery_one(fb, a, b, bad);
        }
        bucket = phf < f.nfree ? __ldg(f.free_pos + phf) : 0;  // select1(phf + 1) - phf
        if (bucket >= f.nbuckets) return bucket - f.nbuckets + (uint64_t)f.k * f.nbuckets;
        seed = __ldg(f.tas + bucket) >> f.tb;
    }
    if (seed == 0) {  // seedsFallback lookup (:271-273)
        uint64_t lo = 0, hi = f.nfs;
        while (lo < hi) {
            const uint64_t mid = (lo + hi) / 2;
            if (__ldg(f.fs_bucket + mid) < bucket) lo = mid + 1; else hi = mid;
        }
        seed = (lo < f.nfs && __ldg(f.fs_bucket + lo) == bucket) ? __ldg(f.fs_seed + lo) : 0;
    }
    const uint64_t retrieved = fretrieve(f, hash);
    return bucket * f.k + sh2_leaf_query(f.k, seed, hash, retrieved, true);  // QuadSplit for every k
}

template <bool STRINGS>
__global__ void __launch_bounds__(256) k_dflat(FView f, DView fb, const uint64_t *__restrict__ a,
                                               const uint8_t *__restrict__ bytes, uint64_t n, uint64_t *__restrict__ out,
                                               uint32_t *__restrict__ err) {
    bool bad = false;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        uint64_t h;
        if (STRINGS) {
            const uint64_t lo = a[i], hi = a[i + 1];
            h = murmur64a(bytes + lo, hi - lo, kMurmurSeed);
        } else {
            h = a[i];
        }
        out[i] = dflat_one(f, fb, h, bad);
    }
    if (bad) atomicOr(err, kQErrStream);
}

int grid_for(uint64_t n) {
    uint64_t g = (n + 255) / 256;
    if (g > 148ull * 16) g = 148ull * 16;
    return g < 1 ? 1 : (int)g;
}

struct QBuf {
    void *p = nullptr;
    size_t cap = 0;
    cudaError_t ensure(size_t bytes) {
        if (bytes <= cap) return cudaSuccess;
        if (p) cudaFree(p);
        p = nullptr;
        cap = 0;
        const size_t want = bytes < 256 ? 256 : bytes;
        cudaError_t e = cudaMalloc(&p, want);
        if (e == cudaSuccess) cap = want;
        return e;
    }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        cap = 0;
    }
};

// Exact retrieval table on the device: slot keys (kEmpty = free), one bit per slot, and the
// kEmpty key's own presence/bit in `special`. Capacity = power of two >= 1.5 n.
struct RTable {
    QBuf key, bits, special;
    uint64_t mask = 0;
    cudaError_t build(const uint64_t *hkeys, const uint8_t *hbits, uint64_t n, cudaStream_t s, QBuf &stage_keys,
                      QBuf &stage_bits) {
        uint64_t cap = 64;
        while (cap < n + n / 2 + 1) cap <<= 1;
        mask = cap - 1;
        cudaError_t e;
        if ((e = key.ensure(cap * 8)) || (e = bits.ensure(cap / 8)) || (e = special.ensure(4)) ||
            (e = stage_keys.ensure(n * 8 + 8)) || (e = stage_bits.ensure(n + 1)))
            return e;
        if ((e = cudaMemsetAsync(key.p, 0xFF, cap * 8, s)) || (e = cudaMemsetAsync(bits.p, 0, cap / 8, s)) ||
            (e = cudaMemsetAsync(special.p, 0, 4, s)))
            return e;
        if (n) {
            if ((e = cudaMemcpyAsync(stage_keys.p, hkeys, n * 8, cudaMemcpyHostToDevice, s)) ||
                (e = cudaMemcpyAsync(stage_bits.p, hbits, n, cudaMemcpyHostToDevice, s)))
                return e;
            k_table_insert<<<grid_for(n), 256, 0, s>>>((const uint64_t *)stage_keys.p, (const uint8_t *)stage_bits.p, n,
                                                     (uint64_t *)key.p, (uint32_t *)bits.p, (uint32_t *)special.p, mask);
            if ((e = cudaGetLastError())) return e;
        }
        return cudaStreamSynchronize(s);
    }
    void release() {
        key.release();
        bits.release();
        special.release();
    }
};

// Textbook Elias-Fano size (the same estimate shg_mphf_bits uses).
uint64_t ef_bits(const uint64_t *v, uint64_t n1) {
    if (!n1) return 0;
    const uint64_t u = v[n1 - 1] + 1;
    uint64_t q = u / n1, L = 0;
    while (q > 1) {
        q >>= 1;
        L++;
    }
    return n1 * L + n1 + (u >> L) + 1;
}

} // namespace

struct shg_dmphf {
    int device = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    DView v{};
    uint64_t n = 0, bits = 0;
    QBuf size_acc, pos_acc, desc, memo, err;
    RTable table;
    shg_retrieval *compact = nullptr;  // owned; replaces the table when set
    QBuf in_a, in_b, in_bytes, out;  // staging for host-buffer queries
    float last_ms = 0.f;
};

#define DQ_CU(call)                                                                                  \
    do {                                                                                             \
        cudaError_t e_ = (call);                                                                     \
        if (e_ != cudaSuccess) return shg_set_error(SHG_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

namespace {

shg_status dq_launch(shg_dmphf *f, int in, const uint64_t *a, const uint64_t *b, const uint8_t *bytes, uint64_t n,
                     uint64_t *out) {
    DQ_CU(cudaMemsetAsync(f->err.p, 0, sizeof(uint32_t), f->stream));
    DQ_CU(cudaEventRecord(f->ev0, f->stream));
    if (n) {
        const int g = grid_for(n);
        uint32_t *err = (uint32_t *)f->err.p;
        if (in == kInHash128)
            k_dquery<kInHash128><<<g, 256, 0, f->stream>>>(f->v, a, b, bytes, n, out, err);
        else if (in == kInU64)
            k_dquery<kInU64><<<g, 256, 0, f->stream>>>(f->v, a, b, bytes, n, out, err);
        else
            k_dquery<kInStrings><<<g, 256, 0, f->stream>>>(f->v, a, b, bytes, n, out, err);
        DQ_CU(cudaGetLastError());
    }
    DQ_CU(cudaEventRecord(f->ev1, f->stream));
    uint32_t herr = 0;
    DQ_CU(cudaMemcpyAsync(&herr, f->err.p, sizeof(uint32_t), cudaMemcpyDeviceToHost, f->stream));
    DQ_CU(cudaStreamSynchronize(f->stream));
    DQ_CU(cudaEventElapsedTime(&f->last_ms, f->ev0, f->ev1));
    if (herr) return shg_set_error(SHG_ERR_ARG, "device query: descriptor walk left the stream (corrupt result?)");
    return SHG_OK;
}

struct DeviceGuard {
    int prev = -1;
    explicit DeviceGuard(int d) {
        if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
        cudaSetDevice(d);
    }
    ~DeviceGuard() {
        if (prev >= 0) cudaSetDevice(prev);
    }
};

} // namespace

namespace shg {
shg_status retrieval_build_on(int device, cudaStream_t s, const uint64_t *d_keys, const uint8_t *d_bits, uint64_t n,
                              shg_retrieval **out);
const RetLevels *retrieval_device_view(const shg_retrieval *r, const uint64_t **sol, const uint8_t **thr);
} // namespace shg

static shg_status dmphf_create(int device, const shg_params *p, const shg_result *r, bool compact, shg_dmphf **out) {
    if (!p || !r || !out) return shg_set_error(SHG_ERR_ARG, "null argument");
    *out = nullptr;
    if (!is_sh1(p->variant) && p->variant != SHG_SHOCKHASH2) return shg_set_error(SHG_ERR_ARG, "unknown variant");
    const int maxleaf = is_sh1(p->variant) ? kMaxLeaf1 : kMaxLeaf2;
    if (p->leaf_size < 2 || p->leaf_size > maxleaf) return shg_set_error(SHG_ERR_ARG, "leaf size out of range");
    if (r->nbuckets == 0 || !r->bucket_size_acc || !r->bucket_pos_acc)
        return shg_set_error(SHG_ERR_ARG, "result has no buckets");
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) return shg_set_error(SHG_ERR_NO_DEVICE, "no CUDA device");
    if (device < 0 || device >= count) return shg_set_error(SHG_ERR_ARG, "device index out of range");
    cudaDeviceProp prop;
    DQ_CU(cudaGetDeviceProperties(&prop, device));
    if (prop.major != 10) return shg_set_error(SHG_ERR_NO_DEVICE, "libshg is built for sm_100a (B200)");
    DeviceGuard guard(device);
    auto *f = new shg_dmphf();
    f->device = device;
    auto bail = [&](shg_status st) {
        shg_dmphf_destroy(f);
        return st;
    };
    if (cudaStreamCreateWithFlags(&f->stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreate(&f->ev0) != cudaSuccess || cudaEventCreate(&f->ev1) != cudaSuccess)
        return bail(shg_set_error(SHG_ERR_CUDA, "stream/event creation failed"));
    const Config cfg(p->variant, p->leaf_size);
    const uint64_t nb = r->nbuckets, nw = r->desc_words, rn = r->ribbon_n;
    const size_t acc_bytes = (nb + 1) * sizeof(uint64_t);
    if (f->size_acc.ensure(acc_bytes) || f->pos_acc.ensure(acc_bytes) || f->desc.ensure((nw + 2) * 8) ||
        f->memo.ensure(kMaxBucket * 8) || f->err.ensure(4))
        return bail(shg_set_error(SHG_ERR_OOM, "device query: cudaMalloc failed"));
    cudaStream_t s = f->stream;
    auto up = [&](void *dst, const void *src, size_t bytes) {
        return bytes ? cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, s) : cudaSuccess;
    };
    if (up(f->size_acc.p, r->bucket_size_acc, acc_bytes) || up(f->pos_acc.p, r->bucket_pos_acc, acc_bytes) ||
        cudaMemsetAsync(f->desc.p, 0, (nw + 2) * 8, s) || up(f->desc.p, r->descriptors, nw * 8) ||
        up(f->memo.p, cfg.memo.data(), kMaxBucket * 8))
        return bail(shg_set_error(SHG_ERR_CUDA, "device query: upload failed"));
    DView &v = f->v;
    if (compact) {
        if (f->in_a.ensure(rn * 8 + 8) || f->in_bytes.ensure(rn + 1))
            return bail(shg_set_error(SHG_ERR_OOM, "device query: cudaMalloc failed"));
        if (up(f->in_a.p, r->ribbon_keys, rn * 8) || up(f->in_bytes.p, r->ribbon_bits, rn))
            return bail(shg_set_error(SHG_ERR_CUDA, "device query: upload failed"));
        const shg_status st = retrieval_build_on(device, s, (const uint64_t *)f->in_a.p, (const uint8_t *)f->in_bytes.p,
                                                 rn, &f->compact);
        if (st != SHG_OK) return bail(st);
        v.rlv = retrieval_device_view(f->compact, &v.rsol, &v.rthr);
    } else if (cudaError_t e = f->table.build(r->ribbon_keys, r->ribbon_bits, rn, s, f->in_a, f->in_bytes)) {
        return bail(shg_set_error(e == cudaErrorMemoryAllocation ? SHG_ERR_OOM : SHG_ERR_CUDA,
                                  std::string("device query: retrieval table: ") + cudaGetErrorString(e)));
    }
    v.size_acc = (const uint64_t *)f->size_acc.p;
    v.pos_acc = (const uint64_t *)f->pos_acc.p;
    v.desc = (const uint64_t *)f->desc.p;
    v.memo = (const uint64_t *)f->memo.p;
    v.tkey = (const uint64_t *)f->table.key.p;
    v.tbits = (const uint32_t *)f->table.bits.p;
    v.special = (const uint32_t *)f->table.special.p;
    v.nb = nb;
    v.nw = nw;
    v.tmask = f->table.mask;
    v.lower = cfg.lower;
    v.upper = cfg.upper;
    v.leaf = (uint32_t)p->leaf_size;
    v.variant = p->variant;
    f->n = r->n;
    const uint64_t obj = is_sh1(p->variant) ? 144 : 136;
    f->bits = ef_bits(r->bucket_size_acc, nb + 1) + ef_bits(r->bucket_pos_acc, nb + 1) + nw * 64 + 8 * ((rn + 7) / 8) +
              8 * obj;
    *out = f;
    return SHG_OK;
}

extern "C" {

shg_status shg_dmphf_create(int device, const shg_params *p, const shg_result *r, shg_dmphf **out) {
    return dmphf_create(device, p, r, false, out);
}

shg_status shg_dmphf_create_compact(int device, const shg_params *p, const shg_result *r, shg_dmphf **out) {
    return dmphf_create(device, p, r, true, out);
}

uint64_t shg_dmphf_retrieval_bits(const shg_dmphf *f) {
    if (!f) return 0;
    if (f->compact) return shg_retrieval_bits(f->compact);
    return (f->table.mask + 1) * 65 + 32;  // table keys and bits, and the special slot
}

void shg_dmphf_destroy(shg_dmphf *f) {
    if (!f) return;
    DeviceGuard guard(f->device);
    if (f->stream) cudaStreamSynchronize(f->stream);
    for (QBuf *b : {&f->size_acc, &f->pos_acc, &f->desc, &f->memo, &f->err, &f->in_a, &f->in_b, &f->in_bytes, &f->out})
        b->release();
    f->table.release();
    shg_retrieval_destroy(f->compact);
    if (f->ev0) cudaEventDestroy(f->ev0);
    if (f->ev1) cudaEventDestroy(f->ev1);
    if (f->stream) cudaStreamDestroy(f->stream);
    delete f;
}

shg_status shg_dmphf_query_hash128_device(shg_dmphf *f, const uint64_t *d_first, const uint64_t *d_second, uint64_t n,
                                          uint64_t *d_out) {
    if (!f || (n && (!d_first || !d_second || !d_out))) return shg_set_error(SHG_ERR_ARG, "null argument");
    DeviceGuard guard(f->device);
    return dq_launch(f, kInHash128, d_first, d_second, nullptr, n, d_out);
}

shg_status shg_dmphf_query_u64_device(shg_dmphf *f, const uint64_t *d_keys, uint64_t n, uint64_t *d_out) {
    if (!f || (n && (!d_keys || !d_out))) return shg_set_error(SHG_ERR_ARG, "null argument");
    DeviceGuard guard(f->device);
    return dq_launch(f, kInU64, d_keys, nullptr, nullptr, n, d_out);
}

shg_status shg_dmphf_query_hash128(shg_dmphf *f, const uint64_t *first, const uint64_t *second, uint64_t n, uint64_t *out) {
    if (!f || (n && (!first || !second || !out))) return shg_set_error(SHG_ERR_ARG, "null argument");
    DeviceGuard guard(f->device);
    if (f->in_a.ensure(n * 8 + 8) || f->in_b.ensure(n * 8 + 8) || f->out.ensure(n * 8 + 8))
        return shg_set_error(SHG_ERR_OOM, "device query: cudaMalloc failed");
    if (n) {
        DQ_CU(cudaMemcpyAsync(f->in_a.p, first, n * 8, cudaMemcpyHostToDevice, f->stream));
        DQ_CU(cudaMemcpyAsync(f->in_b.p, second, n * 8, cudaMemcpyHostToDevice, f->stream));
    }
    shg_status st = dq_launch(f, kInHash128, (const uint64_t *)f->in_a.p, (const uint64_t *)f->in_b.p, nullptr, n,
                              (uint64_t *)f->out.p);
    if (st) return st;
    if (n) {
        DQ_CU(cudaMemcpyAsync(out, f->out.p, n * 8, cudaMemcpyDeviceToHost, f->stream));
        DQ_CU(cudaStreamSynchronize(f->stream));
    }
    return SHG_OK;
}

shg_status shg_dmphf_query_u64(shg_dmphf *f, const uint64_t *keys, uint64_t n, uint64_t *out) {
    if (!f || (n && (!keys || !out))) return shg_set_error(SHG_ERR_ARG, "null argument");
    DeviceGuard guard(f->device);
    if (f->in_a.ensure(n * 8 + 8) || f->out.ensure(n * 8 + 8))
        return shg_set_error(SHG_ERR_OOM, "device query: cudaMalloc failed");
    if (n) DQ_CU(cudaMemcpyAsync(f->in_a.p, keys, n * 8, cudaMemcpyHostToDevice, f->stream));
    shg_status st = dq_launch(f, kInU64, (const uint64_t *)f->in_a.p, nullptr, nullptr, n, (uint64_t *)f->out.p);
    if (st) return st;
    if (n) {
        DQ_CU(cudaMemcpyAsync(out, f->out.p, n * 8, cudaMemcpyDeviceToHost, f->stream));
        DQ_CU(cudaStreamSynchronize(f->stream));
    }
    return SHG_OK;
}

shg_status shg_dmphf_query_strings(shg_dmphf *f, const char *bytes, const uint64_t *offsets, uint64_t n, uint64_t *out) {
    if (!f || !offsets || (n && !out)) return shg_set_error(SHG_ERR_ARG, "null argument");
    if (offsets[0] != 0) return shg_set_error(SHG_ERR_ARG, "offsets[0] must be 0");
    for (uint64_t i = 0; i < n; i++)
        if (offsets[i + 1] < offsets[i]) return shg_set_error(SHG_ERR_ARG, "offsets must be non-decreasing");
    const uint64_t total = offsets[n];
    if (total && !bytes) return shg_set_error(SHG_ERR_ARG, "null bytes");
    DeviceGuard guard(f->device);
    if (f->in_bytes.ensure(total + 16) || f->in_b.ensure((n + 1) * 8) || f->out.ensure(n * 8 + 8))
        return shg_set_error(SHG_ERR_OOM, "device query: cudaMalloc failed");
    if (total) DQ_CU(cudaMemcpyAsync(f->in_bytes.p, bytes, total, cudaMemcpyHostToDevice, f->stream));
    DQ_CU(cudaMemcpyAsync(f->in_b.p, offsets, (n + 1) * 8, cudaMemcpyHostToDevice, f->stream));
    shg_status st = dq_launch(f, kInStrings, nullptr, (const uint64_t *)f->in_b.p, (const uint8_t *)f->in_bytes.p, n,
                              (uint64_t *)f->out.p);
    if (st) return st;
    if (n) {
        DQ_CU(cudaMemcpyAsync(out, f->out.p, n * 8, cudaMemcpyDeviceToHost, f->stream));
        DQ_CU(cudaStreamSynchronize(f->stream));
    }
    return SHG_OK;
}

uint64_t shg_dmphf_bits(const shg_dmphf *f) { return f ? f->bits : 0; }
uint64_t shg_dmphf_size(const shg_dmphf *f) { return f ? f->n : 0; }
float shg_dmphf_last_kernel_ms(const shg_dmphf *f) { return f ? f->last_ms : 0.f; }

} // extern "C"

// ------------------------------------------------------------------ ShockHash2Flat<k> device query
struct shg_dflat {
    int device = 0;
    shg_dmphf *fallback = nullptr;  // owns the stream the queries run on
    shg_dmphf *owner = nullptr;     // stream/event/staging holder when there is no fallback PHF
    FView v{};
    QBuf tas, mapping, free_pos, fs_bucket, fs_seed;
    RTable table;
    uint64_t n = 0;
};

namespace {

shg_status dflat_launch(shg_dflat *f, bool strings, const uint64_t *a, const uint8_t *bytes, uint64_t n, uint64_t *out) {
    shg_dmphf *h = f->fallback ? f->fallback : f->owner;
    DQ_CU(cudaMemsetAsync(h->err.p, 0, sizeof(uint32_t), h->stream));
    DQ_CU(cudaEventRecord(h->ev0, h->stream));
    if (n) {
        const DView fb = f->fallback ? f->fallback->v : DView{};
        if (strings)
            k_dflat<true><<<grid_for(n), 256, 0, h->stream>>>(f->v, fb, a, bytes, n, out, (uint32_t *)h->err.p);
        else
            k_dflat<false><<<grid_for(n), 256, 0, h->stream>>>(f->v, fb, a, bytes, n, out, (uint32_t *)h->err.p);
        DQ_CU(cudaGetLastError());
    }
    DQ_CU(cudaEventRecord(h->ev1, h->stream));
    uint32_t herr = 0;
    DQ_CU(cudaMemcpyAsync(&herr, h->err.p, sizeof(uint32_t), cudaMemcpyDeviceToHost, h->stream));
    DQ_CU(cudaStreamSynchronize(h->stream));
    DQ_CU(cudaEventElapsedTime(&h->last_ms, h->ev0, h->ev1));
    if (herr) return shg_set_error(SHG_ERR_ARG, "device query: descriptor walk left the stream (corrupt result?)");
    return SHG_OK;
}

} // namespace

extern "C" {

shg_status shg_dflat_create(int device, const shg_flat_result *r, shg_dflat **out) {
    if (!r || !out) return shg_set_error(SHG_ERR_ARG, "null argument");
    *out = nullptr;
    if (r->k < 4 || r->k > (uint64_t)kMaxLeaf2 || r->layers < 1 || r->layers > 2)
        return shg_set_error(SHG_ERR_ARG, "not a ShockHash2Flat result");
    auto *f = new shg_dflat();
    f->device = device;
    auto bail = [&](shg_status st) {
        shg_dflat_destroy(f);
        return st;
    };
    shg_params fp{SHG_SHOCKHASH2, (int)r->k, 2000, SHG_MODE_DEFAULT, 0};
    shg_status st;
    if (r->nfallback_keys && r->fallback.nbuckets) {
        st = shg_dmphf_create(device, &fp, &r->fallback, &f->fallback);
    } else {
        // an empty one-bucket result only to own the stream, events and staging buffers
        static const uint64_t zeros[2] = {0, 0};
        shg_result empty{};
        empty.nbuckets = 1;
        empty.bucket_size_acc = const_cast<uint64_t *>(zeros);
        empty.bucket_pos_acc = const_cast<uint64_t *>(zeros);
        st = shg_dmphf_create(device, &fp, &empty, &f->owner);
    }
    if (st) return bail(st);
    shg_dmphf *h = f->fallback ? f->fallback : f->owner;
    DeviceGuard guard(device);
    const FlatConsts fc = flat_consts((uint32_t)r->k);
    cudaStream_t s = h->stream;
    const uint64_t nb = r->nbuckets;
    if (f->tas.ensure(nb * 8 + 8) || f->mapping.ensure(fc.mapping.size() * 4) || f->free_pos.ensure(r->nfree * 8 + 8) ||
        f->fs_bucket.ensure(r->nfallback_seeds * 8 + 8) || f->fs_seed.ensure(r->nfallback_seeds * 8 + 8))
        return bail(shg_set_error(SHG_ERR_OOM, "device flat query: cudaMalloc failed"));
    auto up = [&](void *dst, const void *src, size_t bytes) {
        return bytes ? cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, s) : cudaSuccess;
    };
    if (up(f->tas.p, r->thresholds_and_seeds, nb * 8) || up(f->mapping.p, fc.mapping.data(), fc.mapping.size() * 4) ||
        up(f->free_pos.p, r->free_positions, r->nfree * 8) ||
        up(f->fs_bucket.p, r->fallback_seed_buckets, r->nfallback_seeds * 8) ||
        up(f->fs_seed.p, r->fallback_seeds, r->nfallback_seeds * 8))
        return bail(shg_set_error(SHG_ERR_CUDA, "device flat query: upload failed"));
    if (cudaError_t e = f->table.build(r->ribbon_keys, r->ribbon_bits, r->ribbon_n, s, h->in_a, h->in_bytes))
        return bail(shg_set_error(e == cudaErrorMemoryAllocation ? SHG_ERR_OOM : SHG_ERR_CUDA,
                                  std::string("device flat query: retrieval table: ") + cudaGetErrorString(e)));
    FView &v = f->v;
    for (uint64_t i = 0; i <= r->layers; i++) v.lb[i] = r->layer_bases[i];
    v.layers = (uint32_t)r->layers;
    v.tb = fc.threshold_bits;
    v.thr_mask = fc.threshold_range - 1;
    v.k = (uint32_t)r->k;
    v.nbuckets = nb;
    v.nfree = r->nfree;
    v.nfs = r->nfallback_seeds;
    v.tas = (const uint64_t *)f->tas.p;
    v.mapping = (const uint32_t *)f->mapping.p;
    v.free_pos = (const uint64_t *)f->free_pos.p;
    v.fs_bucket = (const uint64_t *)f->fs_bucket.p;
    v.fs_seed = (const uint64_t *)f->fs_seed.p;
    v.tkey = (const uint64_t *)f->table.key.p;
    v.tbits = (const uint32_t *)f->table.bits.p;
    v.special = (const uint32_t *)f->table.special.p;
    v.tmask = f->table.mask;
    v.has_fallback = f->fallback != nullptr;
    f->n = r->n;
    *out = f;
    return SHG_OK;
}

void shg_dflat_destroy(shg_dflat *f) {
    if (!f) return;
    {
        DeviceGuard guard(f->device);
        shg_dmphf *h = f->fallback ? f->fallback : f->owner;
        if (h && h->stream) cudaStreamSynchronize(h->stream);
        for (QBuf *b : {&f->tas, &f->mapping, &f->free_pos, &f->fs_bucket, &f->fs_seed}) b->release();
        f->table.release();
    }
    shg_dmphf_destroy(f->fallback);
    shg_dmphf_destroy(f->owner);
    delete f;
}

shg_status shg_dflat_query_strings(shg_dflat *f, const char *bytes, const uint64_t *offsets, uint64_t n, uint64_t *out) {
    if (!f || !offsets || (n && !out)) return shg_set_error(SHG_ERR_ARG, "null argument");
    if (offsets[0] != 0) return shg_set_error(SHG_ERR_ARG, "offsets[0] must be 0");
    for (uint64_t i = 0; i < n; i++)
        if (offsets[i + 1] < offsets[i]) return shg_set_error(SHG_ERR_ARG, "offsets must be non-decreasing");
    const uint64_t total = offsets[n];
    if (total && !bytes) return shg_set_error(SHG_ERR_ARG, "null bytes");
    shg_dmphf *h = f->fallback ? f->fallback : f->owner;
    DeviceGuard guard(f->device);
    if (h->in_bytes.ensure(total + 16) || h->in_b.ensure((n + 1) * 8) || h->out.ensure(n * 8 + 8))
        return shg_set_error(SHG_ERR_OOM, "device flat query: cudaMalloc failed");
    if (total) DQ_CU(cudaMemcpyAsync(h->in_bytes.p, bytes, total, cudaMemcpyHostToDevice, h->stream));
    DQ_CU(cudaMemcpyAsync(h->in_b.p, offsets, (n + 1) * 8, cudaMemcpyHostToDevice, h->stream));
    shg_status st = dflat_launch(f, true, (const uint64_t *)h->in_b.p, (const uint8_t *)h->in_bytes.p, n, (uint64_t *)h->out.p);
    if (st) return st;
    if (n) {
        DQ_CU(cudaMemcpyAsync(out, h->out.p, n * 8, cudaMemcpyDeviceToHost, h->stream));
        DQ_CU(cudaStreamSynchronize(h->stream));
    }
    return SHG_OK;
}

shg_status shg_dflat_query_hash(shg_dflat *f, const uint64_t *mhc, uint64_t n, uint64_t *out) {
    if (!f || (n && (!mhc || !out))) return shg_set_error(SHG_ERR_ARG, "null argument");
    shg_dmphf *h = f->fallback ? f->fallback : f->owner;
    DeviceGuard guard(f->device);
    if (h->in_a.ensure(n * 8 + 8) || h->out.ensure(n * 8 + 8))
        return shg_set_error(SHG_ERR_OOM, "device flat query: cudaMalloc failed");
    if (n) DQ_CU(cudaMemcpyAsync(h->in_a.p, mhc, n * 8, cudaMemcpyHostToDevice, h->stream));
    shg_status st = dflat_launch(f, false, (const uint64_t *)h->in_a.p, nullptr, n, (uint64_t *)h->out.p);
    if (st) return st;
    if (n) {
        DQ_CU(cudaMemcpyAsync(out, h->out.p, n * 8, cudaMemcpyDeviceToHost, h->stream));
        DQ_CU(cudaStreamSynchronize(h->stream));
    }
    return SHG_OK;
}

float shg_dflat_last_kernel_ms(const shg_dflat *f) {
    if (!f) return 0.f;
    const shg_dmphf *h = f->fallback ? f->fallback : f->owner;
    return h ? h->last_ms : 0.f;
}

} // extern "C"
