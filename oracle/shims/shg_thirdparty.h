// Test infrastructure only (the oracle). Nothing in the shipped library includes this file.
//
// Restatements of the third-party primitives that the ShockHash reference calls but whose
// sources are absent (the git submodules extlib/sux, extlib/util, extlib/simpleRibbon are empty
// in the reference tree and their pinned revisions are unknown). Each function restates the
// published algorithm it names; none is transcribed from the third-party sources.
//
//  * SpookyHash V2 (Bob Jenkins, 2012, public domain): 128-bit hash used by sux `spooky()`
//    (ShockHash.h:129 `first_hash`).
//  * MurmurHash64A (Austin Appleby, MurmurHash2 64-bit, public domain): ByteHamster util
//    `MurmurHash64` (ShockHash2Flat.h:75, TinyBinaryCuckooHashTable.h:24-26).
//  * Stafford "Mix13" 64-bit finalizer: `remix` (constants restated in-repo at SimdUtils.h:42-46).
//  * Lemire fast range reduction: `fastrange32/64`, sux `remap16`, `remap128`
//    (32-bit form in-repo at SimdUtils.h:48-51; 16-bit mask form at SIMDShockHash.hpp:58-71).
#pragma once
#include <cstdint>
#include <cstddef>
#include <cstring>

namespace shg_tp {

static inline uint64_t rotl64(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }

// ---------------------------------------------------------------- SpookyHash V2
static constexpr uint64_t SPOOKY_CONST = 0xdeadbeefdeadbeefULL;

static inline void spooky_short_mix(uint64_t &h0, uint64_t &h1, uint64_t &h2, uint64_t &h3) {
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

static inline void spooky_short_end(uint64_t &h0, uint64_t &h1, uint64_t &h2, uint64_t &h3) {
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

static inline uint64_t load_le64(const uint8_t *p) { uint64_t v; std::memcpy(&v, p, 8); return v; }
static inline uint32_t load_le32(const uint8_t *p) { uint32_t v; std::memcpy(&v, p, 4); return v; }

// Messages shorter than 192 bytes.
static inline void spooky_short(const uint8_t *msg, size_t length, uint64_t *hash1, uint64_t *hash2) {
    size_t remainder = length % 32;
    uint64_t a = *hash1, b = *hash2, c = SPOOKY_CONST, d = SPOOKY_CONST;
    const uint8_t *p = msg;
    if (length > 15) {
        const uint8_t *end = msg + (length / 32) * 32;
        for (; p < end; p += 32) {
            c += load_le64(p);
            d += load_le64(p + 8);
            spooky_short_mix(a, b, c, d);
            a += load_le64(p + 16);
            b += load_le64(p + 24);
        }
        if (remainder >= 16) {
            c += load_le64(p);
            d += load_le64(p + 8);
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
        case 12: d += load_le32(p + 8); c += load_le64(p); break;
        case 11: d += ((uint64_t)p[10]) << 16; [[fallthrough]];
        case 10: d += ((uint64_t)p[9]) << 8; [[fallthrough]];
        case 9: d += (uint64_t)p[8]; [[fallthrough]];
        case 8: c += load_le64(p); break;
        case 7: c += ((uint64_t)p[6]) << 48; [[fallthrough]];
        case 6: c += ((uint64_t)p[5]) << 40; [[fallthrough]];
        case 5: c += ((uint64_t)p[4]) << 32; [[fallthrough]];
        case 4: c += load_le32(p); break;
        case 3: c += ((uint64_t)p[2]) << 16; [[fallthrough]];
        case 2: c += ((uint64_t)p[1]) << 8; [[fallthrough]];
        case 1: c += (uint64_t)p[0]; break;
        case 0: c += SPOOKY_CONST; d += SPOOKY_CONST; break;
    }
    spooky_short_end(a, b, c, d);
    *hash1 = a;
    *hash2 = b;
}

static inline void spooky_mix(const uint64_t *data, uint64_t *s) {
    // s[0..11]; one 96-byte block.
    static const int R[12] = {11, 32, 43, 31, 17, 28, 39, 57, 55, 54, 22, 46};
    for (int i = 0; i < 12; i++) {
        s[i] += data[i];
        s[(i + 2) % 12] ^= s[(i + 10) % 12];
        s[(i + 11) % 12] ^= s[i];
        s[i] = rotl64(s[i], R[i]);
        s[(i + 11) % 12] += s[(i + 1) % 12];
    }
}

static inline void spooky_end_partial(uint64_t *h) {
    static const int R[12] = {44, 15, 34, 21, 38, 33, 10, 13, 38, 53, 42, 54};
    for (int i = 0; i < 12; i++) {
        h[(i + 11) % 12] += h[(i + 1) % 12];
        h[(i + 2) % 12] ^= h[(i + 11) % 12];
        h[(i + 1) % 12] = rotl64(h[(i + 1) % 12], R[i]);
    }
}

static inline void spooky_hash128(const void *message, size_t length, uint64_t *hash1, uint64_t *hash2) {
    const uint8_t *msg = (const uint8_t *)message;
    if (length < 192) {
        spooky_short(msg, length, hash1, hash2);
        return;
    }
    uint64_t h[12];
    h[0] = h[3] = h[6] = h[9] = *hash1;
    h[1] = h[4] = h[7] = h[10] = *hash2;
    h[2] = h[5] = h[8] = h[11] = SPOOKY_CONST;
    size_t nblocks = length / 96;
    uint64_t block[12];
    for (size_t b = 0; b < nblocks; b++) {
        std::memcpy(block, msg + b * 96, 96);
        spooky_mix(block, h);
    }
    size_t remainder = length - nblocks * 96;
    uint8_t buf[96];
    std::memcpy(buf, msg + nblocks * 96, remainder);
    std::memset(buf + remainder, 0, 96 - remainder);
    buf[95] = (uint8_t)remainder;
    std::memcpy(block, buf, 96);
    for (int i = 0; i < 12; i++) h[i] += block[i];
    spooky_end_partial(h);
    spooky_end_partial(h);
    spooky_end_partial(h);
    *hash1 = h[0];
    *hash2 = h[1];
}

// ---------------------------------------------------------------- MurmurHash64A
// Seed used by the `MurmurHash64(ptr, len)` convenience overload. The value in the absent
// ByteHamster/Util revision is not recoverable here; this constant is a stated choice.
static constexpr uint64_t MURMUR64_DEFAULT_SEED = 1203114875ULL;

static inline uint64_t murmur64a(const void *key, size_t len, uint64_t seed) {
    const uint64_t m = 0xc6a4a7935bd1e995ULL;
    const int r = 47;
    uint64_t h = seed ^ (len * m);
    const uint8_t *data = (const uint8_t *)key;
    size_t nblocks = len / 8;
    for (size_t i = 0; i < nblocks; i++) {
        uint64_t k = load_le64(data + 8 * i);
        k *= m;
        k ^= k >> r;
        k *= m;
        h ^= k;
        h *= m;
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
    h ^= h >> r;
    h *= m;
    h ^= h >> r;
    return h;
}

// ---------------------------------------------------------------- mixing / range reduction
static inline uint64_t remix(uint64_t z) {
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
    return z ^ (z >> 31);
}
static inline uint32_t fastrange32(uint32_t word, uint32_t p) { return (uint32_t)(((uint64_t)word * (uint64_t)p) >> 32); }
static inline uint64_t fastrange64(uint64_t word, uint64_t p) { return (uint64_t)(((__uint128_t)word * (__uint128_t)p) >> 64); }
static inline uint16_t fastrange16(uint16_t word, uint16_t p) { return (uint16_t)(((uint32_t)word * (uint32_t)p) >> 16); }
static inline uint16_t remap16(uint64_t x, uint32_t n) { return (uint16_t)(((x & 0xFFFF) * n) >> 16); }
static inline uint64_t remap128(uint64_t x, uint64_t n) { return (uint64_t)(((__uint128_t)x * (__uint128_t)n) >> 64); }

} // namespace shg_tp
