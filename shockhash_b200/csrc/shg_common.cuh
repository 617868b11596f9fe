// Shared host/device arithmetic of the ShockHash construction path.
//
// Every function here is bit-for-bit the arithmetic the reference performs (file:line of the
// reference project given per item); the third-party ones are restated from their published
// algorithms (SpookyHash V2, MurmurHash64A, Stafford Mix13, Lemire range reduction) because the
// reference's submodules that define them are not vendored.
#pragma once
#include <cstdint>
#include <cstddef>

#define SHG_HD __host__ __device__ __forceinline__

namespace shg {

constexpr int kMaxBucket = 3000;   // ShockHash.h:33 MAX_BUCKET_SIZE
constexpr int kMaxLeaf1 = 60;      // ShockHash.h:35 MAX_LEAF_SIZE
constexpr int kMaxLeaf2 = 128;     // ShockHash2.h:29 MAX_LEAF_SIZE2
constexpr int kMaxLevels = 20;     // ShockHash.h:47-50, 20 start seeds

// Start seed per tree depth, ShockHash.h:47-49 (the table must be identical for the format).
#define SHG_START_SEEDS                                                                              \
    {0x106393c187cae21aULL, 0x6453cec3f7376937ULL, 0x643e521ddbd2be98ULL, 0x3740c6412f6572cbULL,   \
     0x717d47562f1ce470ULL, 0x4cd6eb4c63befb7cULL, 0x9bfd8c5e18c8da73ULL, 0x082f20e10092a9a3ULL,   \
     0x2ada2ce68d21defcULL, 0xe33cb4f3e7c6466bULL, 0x3980be458c509c59ULL, 0xc466fd9584828e8cULL,   \
     0x45f0aabe1a61ede6ULL, 0xf6e7b8b33ad9b98dULL, 0x4ef95e25f4b4983dULL, 0x81175195173b92d3ULL,   \
     0x4e50927d8dd15978ULL, 0x1ea2099d1fafae7fULL, 0x425c8a06fbaaa815ULL, 0xcd4216006c74052aULL}

static __constant__ const uint64_t d_start_seed[kMaxLevels] = SHG_START_SEEDS;
static const uint64_t h_start_seed[kMaxLevels] = SHG_START_SEEDS;

SHG_HD uint64_t start_seed(int level) {
#ifdef __CUDA_ARCH__
    return d_start_seed[level];
#else
    return h_start_seed[level];
#endif
}

// Stafford's Mix13 finalizer (`remix`, constants as in SimdUtils.h:42-46).
SHG_HD uint64_t remix(uint64_t z) {
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
    return z ^ (z >> 31);
}

// The low 16 bits of remix(z): all that remap16 looks at (sux remap16, SIMDShockHash.hpp:58-71).
// Only bits 0..46 of the second product matter, so its high word is needed only to bit 14.
SHG_HD uint32_t remix_low16(uint64_t z) {
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
    return (uint32_t)((z ^ (z >> 31)) & 0xFFFF);
}

// MurmurHash3's 32-bit finalizer (fmix32), as SIMDShockHash.hpp:76-83 (remix32) writes it.
SHG_HD uint32_t fmix32(uint32_t z) {
    z ^= z >> 16;
    z *= 0x85ebca6bu;
    z ^= z >> 13;
    z *= 0xc2b2ae35u;
    z ^= z >> 16;
    return z;
}
// SIMDShockHash's split hash before remap16: fmix32 of the xor of z's two 32-bit halves
// (remixAndRemap, SIMDShockHash.hpp:762-766; the vector form remap() at :58-71 combines the same
// halves lane by lane). Only the low 16 bits reach remap16.
SHG_HD uint32_t simd_split_low16(uint64_t z) { return fmix32((uint32_t)(z >> 32) ^ (uint32_t)z) & 0xFFFFu; }

#ifdef __CUDACC__
// remix's low 32 bits with the work split between the integer and multiply pipes: the high words
// of the two xor-shifts are taken as multiply-highs by the runtime constants K.four (4) and
// K.thirtytwo (32), which the compiler cannot turn back into shifts, so that they run on the
// multiply-add pipe next to the 64-bit products. Returns (lo, t): remix(z) = lo ^ t in the low 32
// bits, left unmerged so that the caller folds its own mask into the same logic operation.
struct PipeK {
    uint32_t four, thirtytwo, c18, two;  // 4, 32, 2^18, 2 (kernel arguments)
};
__device__ __forceinline__ void remix_lo32_pipes(uint64_t z, const PipeK &K, uint32_t &lo4, uint32_t &t) {
    uint32_t lo = (uint32_t)z, hi = (uint32_t)(z >> 32);
    lo ^= __funnelshift_r(lo, hi, 30);  // z ^= z >> 30
    hi ^= __umulhi(hi, K.four);
    uint64_t w = (uint64_t)lo * 0x1ce4e5b9u;  // z *= 0xbf58476d1ce4e5b9
    uint32_t lo2 = (uint32_t)w, hi2 = (uint32_t)(w >> 32) + lo * 0xbf58476du + hi * 0x1ce4e5b9u;
    lo2 ^= __funnelshift_r(lo2, hi2, 27);  // z ^= z >> 27
    hi2 ^= __umulhi(hi2, K.thirtytwo);
    w = (uint64_t)lo2 * 0x133111ebu;  // z *= 0x94d049bb133111eb (bits 0..46 matter)
    lo4 = (uint32_t)w;
    const uint32_t hi4 = (uint32_t)(w >> 32) + lo2 * 0x94d049bbu + hi2 * 0x133111ebu;
    t = __funnelshift_r(lo4, hi4, 31);  // z ^ (z >> 31)
}
// c + (x >> 31) as one multiply-add-high (x * 2 >> 32), on the multiply-add pipe.
__device__ __forceinline__ uint32_t add_sign_bit(uint32_t c, uint32_t x, uint32_t two) {
    uint32_t d;
    asm("mad.hi.u32 %0, %1, %2, %3;" : "=r"(d) : "r"(x), "r"(two), "r"(c));
    return d;
}
#endif

// Lemire range reduction. fastrange32 takes the low 32 bits of its argument
// (TinyBinaryCuckooHashTable.h:140-141, SimdUtils.h:48-51).
SHG_HD uint32_t fastrange32(uint32_t word, uint32_t p) { return (uint32_t)(((uint64_t)word * (uint64_t)p) >> 32); }
SHG_HD uint64_t fastrange64(uint64_t word, uint64_t p) {
#ifdef __CUDA_ARCH__
    return __umul64hi(word, p);
#else
    return (uint64_t)(((unsigned __int128)word * (unsigned __int128)p) >> 64);
#endif
}
SHG_HD uint32_t remap16(uint64_t x, uint32_t n) { return (uint32_t)(((x & 0xFFFF) * n) >> 16); }
SHG_HD uint64_t remap128(uint64_t x, uint64_t n) { return fastrange64(x, n); }

// ------------------------------------------------------------------ pairing (PairingFunction.h)
// The unpairing steps use IEEE double sqrt, which is correctly rounded on both host and device,
// so the float-accuracy checks agree with the reference bit for bit.
SHG_HD uint64_t pair_triangular(uint64_t x, uint64_t y) { return (x - 1) * x / 2 + y; }  // :47-50
SHG_HD void unpair_triangular(uint64_t z, uint64_t &x, uint64_t &y) {                     // :52-56
    x = (uint64_t)floor(0.5 + sqrt(0.25 + 2.0 * (double)z));
    y = z - ((x - 1) * x) / 2;
}
SHG_HD bool float_accurate_triangular(uint64_t x, uint64_t y) {  // :58-61
    uint64_t a, b;
    unpair_triangular(pair_triangular(x, y), a, b);
    return a == x && b == y;
}
SHG_HD uint64_t pair_elegant(uint64_t x, uint64_t y) { return x < y ? y * y + x : x * x + x + y; }  // :75-81
SHG_HD void unpair_elegant(uint64_t z, uint64_t &x, uint64_t &y) {                               // :83-91
    uint64_t f = (uint64_t)floor(sqrt((double)z));
    uint64_t sq = f * f;
    if (z - sq < f) { x = z - sq; y = f; } else { x = f; y = z - sq - f; }
}
SHG_HD bool float_accurate_elegant(uint64_t x, uint64_t y) {  // :93-96
    uint64_t a, b;
    unpair_elegant(pair_elegant(x, y), a, b);
    return a == x && b == y;
}
// The same test for raw seeds of a leaf search: below 2^24 it always holds, so the square root is
// skipped there. z = pair_elegant(x, y) lies in [f^2, (f + 1)^2 - 1] with f <= 2^24; sqrt(f^2) = f
// is exact, and sqrt((f + 1)^2 - 1) stays more than 2^-26 below f + 1 while doubles near f are at
// most 2^-28 apart, so the correctly rounded square root floors to f and unpairing is exact.
#ifdef __CUDA_ARCH__
// The square-root path out of line on the device: raw seeds of a leaf search stay far below 2^24 in
// practice, and the leaf kernels test many seed pairs at many places, so inlining it would only
// grow their code.
static __device__ __noinline__ bool float_accurate_elegant_cold(uint64_t x, uint64_t y) {
    return float_accurate_elegant(x, y);
}
#endif
SHG_HD bool float_accurate_elegant_seeds(uint64_t x, uint64_t y) {
#ifdef __CUDA_ARCH__
    return (x | y) < (1ull << 24) || float_accurate_elegant_cold(x, y);
#else
    return (x | y) < (1ull << 24) || float_accurate_elegant(x, y);
#endif
}

// ------------------------------------------------------------------ leaf cell hashes
// Original ShockHash candidate cells (TinyBinaryCuckooHashTable.h:138-149).
SHG_HD void sh1_cells(uint64_t key, uint64_t seed, uint32_t m, uint32_t &c1, uint32_t &c2) {
    const uint64_t r = remix(key + seed);
    c1 = fastrange32((uint32_t)r, m / 2);
    c2 = fastrange32((uint32_t)(r >> 32), (m + 1) / 2) + m / 2;
}
// Bipartite half-table cell (ShockHash2-internal.h:100-102, 473-477).
// fastrange64(word, p) for a range p below 2^32, exactly: with word = hi * 2^32 + lo,
// floor(word * p / 2^64) = floor((hi * p + floor(lo * p / 2^32)) / 2^32), the dropped fraction
// never carrying past an integer. Two 32-bit multiplies instead of a 64 x 64-bit high product.
SHG_HD uint32_t fastrange64_32(uint64_t word, uint32_t p) {
#ifdef __CUDA_ARCH__
    const uint64_t a = (uint64_t)(uint32_t)(word >> 32) * p + __umulhi((uint32_t)word, p);
    return (uint32_t)(a >> 32);
#else
    return (uint32_t)fastrange64(word, p);
#endif
}
SHG_HD uint32_t half_hash(uint64_t key, uint64_t s, uint32_t half) { return fastrange64_32(remix(key + s), half); }
// Cell of `key` under a bipartite candidate seed: the Basic finder's hash
// (ShockHash2-internal.h:100-102), or QuadSplit's (elegant pair; even keys use seedA, odd keys
// seedB, :473-477). The RecSplit leaves use QuadSplit from m = 10 on
// (ShockHash2-precompiled.cpp:11-13); ShockHash2Flat uses it for every k (ShockHash2Flat.h:39).
constexpr uint32_t kQuadMinRecSplit = 10, kQuadMinFlat = 0;
SHG_HD uint32_t sh2_cand_hash(uint64_t key, uint64_t seed, uint32_t m, bool quad) {
    const uint32_t half = (m + 1) / 2;
    if (!quad) return half_hash(key, seed, half);
    uint64_t a, b;
    unpair_elegant(seed, a, b);
    return half_hash(key, (key & 1) == 0 ? a : b, half);
}
SHG_HD uint32_t sh2_cand_hash(uint64_t key, uint64_t seed, uint32_t m) {
    return sh2_cand_hash(key, seed, m, m >= kQuadMinRecSplit);
}
// Leaf query (ShockHash2-internal.h:574-584); leaves of size <= 1 map to 0
// (ShockHash2-precompiled.cpp:6-9).
SHG_HD uint64_t sh2_leaf_query(uint32_t m, uint64_t seed, uint64_t key, uint64_t retrieved, bool quad) {
    if (m <= 1) return 0;
    uint64_t s1, s2;
    unpair_triangular(seed, s1, s2);
    return retrieved == 0 ? (uint64_t)sh2_cand_hash(key, s1, m, quad) + m / 2 : (uint64_t)sh2_cand_hash(key, s2, m, quad);
}
SHG_HD uint64_t sh2_leaf_query(uint32_t m, uint64_t seed, uint64_t key, uint64_t retrieved) {
    return sh2_leaf_query(m, seed, key, retrieved, m >= kQuadMinRecSplit);
}

// ------------------------------------------------------------------ SpookyHash V2 (Jenkins)
SHG_HD uint64_t rotl64(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }
constexpr uint64_t kSpookyConst = 0xdeadbeefdeadbeefULL;

SHG_HD void spooky_short_mix(uint64_t &h0, uint64_t &h1, uint64_t &h2, uint64_t &h3) {
    h2 = rotl64(h2, 50); h2 += h3; h0 ^= h2;
    h3 = rotl64(h3, 52); h3 += h0; h1 ^= h3;
    h0 = rotl64(h0, 30); h0 += h1; h2 ^= h0;
    h1 = rotl64(h1, 41); h1 += h2; h3 ^= h1;
    h2 = rotl64(h2, 54); h2 += h3; h0 ^= h2;
    h3 = rotl64(h3, 48); h3 += h0; h1 ^= h3;
    h0 = rotl64(h0, 38); h0 += h1; h2 ^= h0;
    h1 = rotl64(h1, 37); h1 += h2; h3 ^= h1;
    h2 = rotl64(h2, 62); h2 += h3; h0 ^= h2;
    h3 = rotl64(h3, 34); h3 += h0; h1 ^= h3;
    h0 = rotl64(h0, 5);  h0 += h1; h2 ^= h0;
    h1 = rotl64(h1, 36); h1 += h2; h3 ^= h1;
}
SHG_HD void spooky_short_end(uint64_t &h0, uint64_t &h1, uint64_t &h2, uint64_t &h3) {
    h3 ^= h2; h2 = rotl64(h2, 15); h3 += h2;
    h0 ^= h3; h3 = rotl64(h3, 52); h0 += h3;
    h1 ^= h0; h0 = rotl64(h0, 26); h1 += h0;
    h2 ^= h1; h1 = rotl64(h1, 51); h2 += h1;
    h3 ^= h2; h2 = rotl64(h2, 28); h3 += h2;
    h0 ^= h3; h3 = rotl64(h3, 9);  h0 += h3;
    h1 ^= h0; h0 = rotl64(h0, 47); h1 += h0;
    h2 ^= h1; h1 = rotl64(h1, 54); h2 += h1;
    h3 ^= h2; h2 = rotl64(h2, 32); h3 += h2;
    h0 ^= h3; h3 = rotl64(h3, 25); h0 += h3;
    h1 ^= h0; h0 = rotl64(h0, 63); h1 += h0;
}

// Little-endian loads from an arbitrarily aligned byte pointer.
SHG_HD uint64_t ld64(const uint8_t *p) {
    uint64_t v = 0;
#pragma unroll
    for (int i = 7; i >= 0; i--) v = (v << 8) | p[i];
    return v;
}
SHG_HD uint32_t ld32(const uint8_t *p) { return (uint32_t)p[0] | (uint32_t)p[1] << 8 | (uint32_t)p[2] << 16 | (uint32_t)p[3] << 24; }

SHG_HD void spooky_short(const uint8_t *p, size_t length, uint64_t &a, uint64_t &b) {
    size_t remainder = length % 32;
    uint64_t c = kSpookyConst, d = kSpookyConst;
    if (length > 15) {
        const uint8_t *end = p + (length / 32) * 32;
        for (; p < end; p += 32) {
            c += ld64(p); d += ld64(p + 8);
            spooky_short_mix(a, b, c, d);
            a += ld64(p + 16); b += ld64(p + 24);
        }
        if (remainder >= 16) {
            c += ld64(p); d += ld64(p + 8);
            spooky_short_mix(a, b, c, d);
            p += 16;
            remainder -= 16;
        }
    }
    d += ((uint64_t)length) << 56;
    switch (remainder) {
        case 15: d += ((uint64_t)p[14]) << 48; [[fallthrough]];
        case 14: d += ((uint64_t)p[13]) << 40; [[fallthrough]];
        case 13: d += ((uint64_t)p[12]) << 32; [[fallthrough]];
        case 12: d += ld32(p + 8); c += ld64(p); break;
        case 11: d += ((uint64_t)p[10]) << 16; [[fallthrough]];
        case 10: d += ((uint64_t)p[9]) << 8; [[fallthrough]];
        case 9: d += (uint64_t)p[8]; [[fallthrough]];
        case 8: c += ld64(p); break;
        case 7: c += ((uint64_t)p[6]) << 48; [[fallthrough]];
        case 6: c += ((uint64_t)p[5]) << 40; [[fallthrough]];
        case 5: c += ((uint64_t)p[4]) << 32; [[fallthrough]];
        case 4: c += ld32(p); break;
        case 3: c += ((uint64_t)p[2]) << 16; [[fallthrough]];
        case 2: c += ((uint64_t)p[1]) << 8; [[fallthrough]];
        case 1: c += (uint64_t)p[0]; break;
        default: c += kSpookyConst; d += kSpookyConst; break;
    }
    spooky_short_end(a, b, c, d);
}

SHG_HD void spooky_mix(const uint64_t *data, uint64_t *s) {
    const int R[12] = {11, 32, 43, 31, 17, 28, 39, 57, 55, 54, 22, 46};
#pragma unroll
    for (int i = 0; i < 12; i++) {
        s[i] += data[i];
        s[(i + 2) % 12] ^= s[(i + 10) % 12];
        s[(i + 11) % 12] ^= s[i];
        s[i] = rotl64(s[i], R[i]);
        s[(i + 11) % 12] += s[(i + 1) % 12];
    }
}
SHG_HD void spooky_end_partial(uint64_t *h) {
    const int R[12] = {44, 15, 34, 21, 38, 33, 10, 13, 38, 53, 42, 54};
#pragma unroll
    for (int i = 0; i < 12; i++) {
        h[(i + 11) % 12] += h[(i + 1) % 12];
        h[(i + 2) % 12] ^= h[(i + 11) % 12];
        h[(i + 1) % 12] = rotl64(h[(i + 1) % 12], R[i]);
    }
}

// SpookyHash V2 Hash128 with both state words seeded by `seed`, returned as sux's
// hash128_t{first = hash2, second = hash1} (ShockHash.h:129 `first_hash` = spooky(k, len, 0)).
SHG_HD void spooky128(const uint8_t *msg, size_t length, uint64_t seed, uint64_t &first, uint64_t &second) {
    uint64_t h1 = seed, h2 = seed;
    if (length < 192) {
        spooky_short(msg, length, h1, h2);
    } else {
        uint64_t h[12];
        h[0] = h[3] = h[6] = h[9] = h1;
        h[1] = h[4] = h[7] = h[10] = h2;
        h[2] = h[5] = h[8] = h[11] = kSpookyConst;
        const size_t nblocks = length / 96;
        uint64_t block[12];
        for (size_t bk = 0; bk < nblocks; bk++) {
            for (int i = 0; i < 12; i++) block[i] = ld64(msg + bk * 96 + 8 * i);
            spooky_mix(block, h);
        }
        // Last partial block: the remaining bytes, zero padding, and the remainder length in the
        // block's final byte.
        const size_t rem = length - nblocks * 96;
        const uint8_t *tail = msg + nblocks * 96;
        uint8_t buf[96];
        for (int i = 0; i < 96; i++) buf[i] = 0;
        for (size_t i = 0; i < rem; i++) buf[i] = tail[i];
        buf[95] = (uint8_t)rem;
        for (int i = 0; i < 12; i++) h[i] += ld64(buf + 8 * i);
        spooky_end_partial(h);
        spooky_end_partial(h);
        spooky_end_partial(h);
        h1 = h[0];
        h2 = h[1];
    }
    first = h2;
    second = h1;
}

// 8-byte little-endian key (a uint64 given as an 8-byte string): the Short path with
// remainder 8 and no 32-byte rounds.
SHG_HD void spooky128_u64(uint64_t key, uint64_t seed, uint64_t &first, uint64_t &second) {
    uint64_t a = seed, b = seed, c = kSpookyConst + key, d = kSpookyConst + (8ULL << 56);
    spooky_short_end(a, b, c, d);
    first = b;
    second = a;
}

// ------------------------------------------------------------------ MurmurHash64A (Appleby)
// Seed of ByteHamster/Util's `MurmurHash64(ptr, len)` convenience overload (ShockHash2Flat.h:75).
// The submodule revision is not vendored; this value is the stated choice shared with the oracle.
constexpr uint64_t kMurmurSeed = 1203114875ULL;

SHG_HD uint64_t murmur64a(const uint8_t *data, size_t len, uint64_t seed) {
    const uint64_t m = 0xc6a4a7935bd1e995ULL;
    const int r = 47;
    uint64_t h = seed ^ (len * m);
    const size_t nblocks = len / 8;
    for (size_t i = 0; i < nblocks; i++) {
        uint64_t k = ld64(data + 8 * i);
        k *= m; k ^= k >> r; k *= m;
        h ^= k; h *= m;
    }
    const uint8_t *tail = data + nblocks * 8;
    switch (len & 7) {
        case 7: h ^= uint64_t(tail[6]) << 48; [[fallthrough]];
        case 6: h ^= uint64_t(tail[5]) << 40; [[fallthrough]];
        case 5: h ^= uint64_t(tail[4]) << 32; [[fallthrough]];
        case 4: h ^= uint64_t(tail[3]) << 24; [[fallthrough]];
        case 3: h ^= uint64_t(tail[2]) << 16; [[fallthrough]];
        case 2: h ^= uint64_t(tail[1]) << 8; [[fallthrough]];
        case 1: h ^= uint64_t(tail[0]); h *= m; break;
        default: break;
    }
    h ^= h >> r; h *= m; h ^= h >> r;
    return h;
}

} // namespace shg
