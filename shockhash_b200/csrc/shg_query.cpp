// Host-side minimal perfect hash object built from a construction result: the query path of the
// reference's operator() (ShockHash.h:199-270, ShockHash2.h:178-230) and getBits()
// (ShockHash.h:283-286, ShockHash2.h:243-246) over the arrays the device produced.
//
// The retrieval structure is an exact open-addressing map from key (hash.second) to its bit;
// the bucket accumulators are kept as plain arrays. getBits() reports those two parts with the
// same size formulas as the oracle's stand-ins for sux DoubleEF and SimpleRibbon (textbook
// Elias-Fano size; one bit per retrieval key), so bits/key compare one to one.
#include <algorithm>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <string>
#include <thread>
#include <vector>
#include "shg.h"
#include "shg_common.cuh"
#include "shg_internal.h"

using namespace shg;

extern "C" uint64_t shg_mphf_bits(const shg_mphf *f);

struct shg_mphf {
    int variant = 0, leaf = 0;
    Config cfg;
    uint64_t n = 0, nb = 0;
    std::vector<uint64_t> size_acc, pos_acc, desc;
    uint64_t ribbon_n = 0;
    // retrieval map
    std::vector<uint64_t> rkey;
    std::vector<uint8_t> rval;  // 0, 1, or 2 = empty slot
    uint64_t rmask = 0;
};

namespace {

uint64_t slot_of(uint64_t key, uint64_t mask) { return remix(key) & mask; }

// Golomb-Rice reader (RiceBitVector.h:149-213).
struct Reader {
    const uint64_t *d;
    uint64_t nw;
    uint64_t fixed_off = 0, window = 0, ptr = 0;
    int valid = 0;
    uint64_t word(uint64_t i) const { return i < nw ? d[i] : 0; }
    uint64_t next(int g) {
        uint64_t result = 0;
        if (window == 0) {
            result += valid;
            window = word(ptr++);
            valid = 64;
            while (window == 0) {
                result += 64;
                window = word(ptr++);
            }
        }
        const int pos = __builtin_ctzll(window);
        window >>= pos;
        window >>= 1;
        valid -= pos + 1;
        result += pos;
        result <<= g;
        const uint64_t lo = word(fixed_off / 64), hi = word(fixed_off / 64 + 1);
        const int sh = (int)(fixed_off % 64);
        uint64_t f = sh ? (lo >> sh) | (hi << (64 - sh)) : lo;
        if (g < 64) f &= (1ull << g) - 1;
        if (g + sh > 128) f |= 0;  // g <= 63, never reached
        result |= f;
        fixed_off += g;
        return result;
    }
    void skip(uint64_t nodes, uint64_t fixed_len) {
        uint64_t missing = nodes, cnt;
        while ((cnt = (uint64_t)__builtin_popcountll(window)) < missing) {
            window = word(ptr++);
            missing -= cnt;
            valid = 64;
        }
        uint64_t w = window;
        for (uint64_t i = 0; i + 1 < missing; i++) w &= w - 1;
        cnt = (uint64_t)__builtin_ctzll(w);
        window >>= cnt;
        window >>= 1;
        valid -= (int)cnt + 1;
        fixed_off += fixed_len;
    }
    void reset(uint64_t bit_pos, uint64_t unary_off) {
        fixed_off = bit_pos;
        const uint64_t up = bit_pos + unary_off;
        ptr = up / 64;
        window = word(ptr++) >> (up & 63);
        valid = 64 - (int)(up & 63);
    }
};

uint64_t retrieve(const shg_mphf *f, uint64_t key) {
    uint64_t s = slot_of(key, f->rmask);
    for (;;) {
        if (f->rval[s] == 2) return 0;
        if (f->rkey[s] == key) return f->rval[s];
        s = (s + 1) & f->rmask;
    }
}

uint64_t query_one(const shg_mphf *f, uint64_t first, uint64_t second) {
    const Config &c = f->cfg;
    const uint64_t bucket = remap128(first, f->nb);
    uint64_t cum = f->size_acc[bucket];
    uint32_t m = (uint32_t)(f->size_acc[bucket + 1] - cum);
    Reader rd{f->desc.data(), (uint64_t)f->desc.size()};
    rd.reset(f->pos_acc[bucket], c.skip_bits(m));
    int level = 0;
    // SIMDShockHash: its own split hash and fixed start seeds below the fanout-2 levels
    // (SIMDShockHash.hpp:785-843)
    const bool simd = is_simd(f->variant);
    auto split_hash = [simd](uint64_t z, uint32_t range) {
        return simd ? remap16(simd_split_low16(z), range) : remap16(remix(z), range);
    };
    while (m > c.upper) {
        const uint64_t d = rd.next(c.golomb(m));
        const uint32_t h = split_hash(second + d + start_seed(level), m);
        const uint32_t sp = (uint16_t(m / 2 + c.upper - 1) / c.upper) * c.upper;
        if (h < sp) {
            m = sp;
        } else {
            rd.skip(c.skip_nodes(sp), c.skip_bits(sp));
            m -= sp;
            cum += sp;
        }
        level++;
    }
    if (m > c.lower) {
        const uint64_t d = rd.next(c.golomb(m));
        const uint32_t h = split_hash(second + d + start_seed(simd ? kSimdSeedLower : level), m);
        const uint32_t part = uint16_t(h) / c.lower;
        m = std::min(c.lower, m - part * c.lower);
        cum += (uint64_t)c.lower * part;
        if (part) rd.skip((uint64_t)c.skip_nodes(c.lower) * part, (uint64_t)c.skip_bits(c.lower) * part);
        level++;
    }
    if (m > (uint32_t)c.leaf) {
        const uint64_t d = rd.next(c.golomb(m));
        const uint32_t h = split_hash(second + d + start_seed(simd ? kSimdSeedLeafAggr : level), m);
        const uint32_t part = uint16_t(h) / c.leaf;
        m = std::min((uint32_t)c.leaf, m - part * c.leaf);
        cum += (uint64_t)c.leaf * part;
        if (part) rd.skip(part, (uint64_t)c.skip_bits(c.leaf) * part);
        level++;
    }
    const uint64_t b = rd.next(c.golomb(m));
    const uint64_t ret = retrieve(f, second);
    const int leaf_seed = simd ? kSimdSeedLeaf : level;
    if (is_rotation(f->variant) && m == (uint32_t)f->leaf) {
        // rotation fitting (ShockHash.h:251-265, SIMDShockHash.hpp:826-840): code = x * L + r; set
        // B's cells rotate by r
        const uint32_t r = (uint32_t)(b % m);
        const uint64_t x = b / m + start_seed(leaf_seed);
        const uint64_t gmask = m > 32 ? 7 : 0;
        uint32_t c1, c2;
        if ((second & 1) == 0) {
            sh1_cells(second, x & ~gmask, m, c1, c2);
            return cum + (ret == 0 ? c1 : c2);
        }
        sh1_cells(second, x, m, c1, c2);
        return cum + ((ret == 0 ? c1 : c2) + r) % m;
    }
    if (is_sh1(f->variant)) {
        // hashToCell (TinyBinaryCuckooHashTable.h:116-123)
        uint32_t c1, c2;
        sh1_cells(second, b + start_seed(leaf_seed), m, c1, c2);
        return cum + (ret == 0 ? c1 : c2);
    }
    return cum + sh2_leaf_query(m, b, second, ret);
}

// Textbook Elias-Fano size of a monotone sequence (same estimate as the oracle's DoubleEF stand-in).
uint64_t ef_bits(const std::vector<uint64_t> &v) {
    if (v.empty()) return 0;
    const uint64_t n1 = v.size(), u = v.back() + 1;
    uint64_t q = u / n1, L = 0;
    while (q > 1) { q >>= 1; L++; }
    return n1 * L + n1 + (u >> L) + 1;
}

} // namespace

extern "C" {

shg_status shg_mphf_create(const shg_params *p, shg_result *r, shg_mphf **out) {
    if (!p || !r || !out) return SHG_ERR_ARG;
    auto *f = new shg_mphf();
    f->variant = p->variant;
    f->leaf = p->leaf_size;
    f->cfg = Config(p->variant, p->leaf_size);
    f->n = r->n;
    f->nb = r->nbuckets;
    f->size_acc.assign(r->bucket_size_acc, r->bucket_size_acc + r->nbuckets + 1);
    f->pos_acc.assign(r->bucket_pos_acc, r->bucket_pos_acc + r->nbuckets + 1);
    f->desc.assign(r->descriptors, r->descriptors + r->desc_words);
    f->ribbon_n = r->ribbon_n;
    uint64_t cap = 16;
    while (cap < r->ribbon_n * 3 / 2 + 1) cap <<= 1;
    f->rkey.assign(cap, 0);
    f->rval.assign(cap, 2);
    f->rmask = cap - 1;
    for (uint64_t i = 0; i < r->ribbon_n; i++) {
        uint64_t s = slot_of(r->ribbon_keys[i], f->rmask);
        while (f->rval[s] != 2 && f->rkey[s] != r->ribbon_keys[i]) s = (s + 1) & f->rmask;
        f->rkey[s] = r->ribbon_keys[i];
        f->rval[s] = r->ribbon_bits[i] & 1;
    }
    *out = f;
    return SHG_OK;
}

void shg_mphf_destroy(shg_mphf *f) { delete f; }

shg_status shg_mphf_query_hash(const shg_mphf *f, const uint64_t *first, const uint64_t *second, uint64_t n, uint64_t *out) {
    if (!f || (n && (!first || !second || !out))) return SHG_ERR_ARG;
    unsigned th = std::max(1u, std::min(32u, std::thread::hardware_concurrency()));
    if (n < 100000) th = 1;
    std::vector<std::thread> pool;
    for (unsigned t = 0; t < th; t++) {
        pool.emplace_back([=] {
            for (uint64_t i = n * t / th; i < n * (t + 1) / th; i++) out[i] = query_one(f, first[i], second[i]);
        });
    }
    for (auto &t : pool) t.join();
    return SHG_OK;
}

shg_status shg_mphf_query_strings(const shg_mphf *f, const char *bytes, const uint64_t *offsets, uint64_t n, uint64_t *out) {
    if (!f || !offsets || (n && (!bytes || !out))) return SHG_ERR_ARG;
    for (uint64_t i = 0; i < n; i++) {
        uint64_t a, b;
        spooky128((const uint8_t *)bytes + offsets[i], offsets[i + 1] - offsets[i], 0, a, b);
        out[i] = query_one(f, a, b);
    }
    return SHG_OK;
}

// getBits(): EF of the two accumulators + descriptor words + retrieval bits + the object itself
// (8 x sizeof of the reference class under the oracle's stand-in member types: 144 bytes for
// ShockHash, which also stores bucket_size, and 136 for ShockHash2).
uint64_t shg_mphf_bits(const shg_mphf *f) {
    if (!f) return 0;
    const uint64_t obj = is_sh1(f->variant) ? 144 : 136;
    return ef_bits(f->size_acc) + ef_bits(f->pos_acc) + f->desc.size() * 64 + 8 * ((f->ribbon_n + 7) / 8) + 8 * obj;
}

uint64_t shg_mphf_size(const shg_mphf *f) { return f ? f->n : 0; }

} // extern "C"

// ------------------------------------------------------------------ ShockHash2Flat<k> queries
struct shg_flat {
    uint64_t n = 0, k = 0, nbuckets = 0, layers = 0;
    std::vector<uint64_t> layer_bases, tas, free_positions;
    std::vector<std::pair<uint64_t, uint64_t>> seed_fallback;  // sorted by bucket
    FlatConsts fc;
    shg_mphf *fallback = nullptr;
    uint64_t nfallback_keys = 0;
    // retrieval map
    std::vector<uint64_t> rkey;
    std::vector<uint8_t> rval;
    uint64_t rmask = 0, ribbon_n = 0;
    ~shg_flat() {
        if (fallback) shg_mphf_destroy(fallback);
    }
};

namespace {

uint64_t flat_retrieve(const shg_flat *f, uint64_t key) {
    uint64_t s = slot_of(key, f->rmask);
    for (;;) {
        if (f->rval[s] == 2) return 0;
        if (f->rkey[s] == key) return f->rval[s];
        s = (s + 1) & f->rmask;
    }
}

// evaluateKPerfect (ShockHash2Flat.h:280-301): (bucket, seed)
std::pair<uint64_t, uint64_t> flat_eval(const shg_flat *f, uint64_t mhc) {
    const uint64_t tb = f->fc.threshold_bits, rmask = f->fc.threshold_range - 1;
    for (uint64_t layer = 0; layer < f->layers; layer++) {
        if (layer) mhc = remix(mhc);
        const uint64_t base = f->layer_bases[layer];
        const uint32_t size = (uint32_t)(f->layer_bases[layer + 1] - base);
        const uint64_t bucket = base + fastrange32((uint32_t)mhc, size);
        const uint64_t stored = f->tas[bucket];
        if ((uint32_t)(mhc >> 32) <= f->fc.mapping[stored & rmask]) return {bucket, stored >> tb};
    }
    const std::string s = std::to_string(mhc);
    const uint64_t offs[2] = {0, s.size()};
    uint64_t phf = 0;
    shg_mphf_query_strings(f->fallback, s.data(), offs, 1, &phf);
    const uint64_t bucket = phf < f->free_positions.size() ? f->free_positions[phf] : 0;  // select1(phf+1) - phf
    if (bucket >= f->nbuckets) return {bucket - f->nbuckets + f->k * f->nbuckets, 1};
    return {bucket, f->tas[bucket] >> tb};
}

// operator()(uint64_t) (ShockHash2Flat.h:266-277)
uint64_t flat_query(const shg_flat *f, uint64_t hash) {
    auto [bucket, seed] = flat_eval(f, hash);
    if (bucket >= f->nbuckets) return bucket;
    if (seed == 0) {
        auto it = std::lower_bound(f->seed_fallback.begin(), f->seed_fallback.end(), std::make_pair(bucket, (uint64_t)0));
        seed = (it != f->seed_fallback.end() && it->first == bucket) ? it->second : 0;
    }
    const uint64_t retrieved = flat_retrieve(f, hash);
    return bucket * f->k + sh2_leaf_query((uint32_t)f->k, seed, hash, retrieved, true);  // QuadSplit for every k
}

} // namespace

extern "C" {

shg_status shg_flat_create(const shg_flat_result *r, shg_flat **out) {
    if (!r || !out) return SHG_ERR_ARG;
    auto *f = new shg_flat();
    f->n = r->n;
    f->k = r->k;
    f->nbuckets = r->nbuckets;
    f->layers = r->layers;
    f->layer_bases.assign(r->layer_bases, r->layer_bases + r->layers + 1);
    f->tas.assign(r->thresholds_and_seeds, r->thresholds_and_seeds + r->nbuckets);
    f->free_positions.assign(r->free_positions, r->free_positions + r->nfree);
    for (uint64_t i = 0; i < r->nfallback_seeds; i++) f->seed_fallback.emplace_back(r->fallback_seed_buckets[i], r->fallback_seeds[i]);
    f->fc = flat_consts((uint32_t)r->k);
    f->nfallback_keys = r->nfallback_keys;
    shg_params fp{SHG_SHOCKHASH2, (int)r->k, 2000, SHG_MODE_DEFAULT, 0};
    shg_status st = shg_mphf_create(&fp, const_cast<shg_result *>(&r->fallback), &f->fallback);
    if (st) {
        delete f;
        return st;
    }
    f->ribbon_n = r->ribbon_n;
    uint64_t cap = 16;
    while (cap < r->ribbon_n * 3 / 2 + 1) cap <<= 1;
    f->rkey.assign(cap, 0);
    f->rval.assign(cap, 2);
    f->rmask = cap - 1;
    for (uint64_t i = 0; i < r->ribbon_n; i++) {
        uint64_t s = slot_of(r->ribbon_keys[i], f->rmask);
        while (f->rval[s] != 2 && f->rkey[s] != r->ribbon_keys[i]) s = (s + 1) & f->rmask;
        f->rkey[s] = r->ribbon_keys[i];
        f->rval[s] = r->ribbon_bits[i] & 1;
    }
    *out = f;
    return SHG_OK;
}

void shg_flat_destroy(shg_flat *f) { delete f; }

shg_status shg_flat_query_hash(const shg_flat *f, const uint64_t *mhc, uint64_t n, uint64_t *out) {
    if (!f || (n && (!mhc || !out))) return SHG_ERR_ARG;
    for (uint64_t i = 0; i < n; i++) out[i] = flat_query(f, mhc[i]);
    return SHG_OK;
}

shg_status shg_flat_query_strings(const shg_flat *f, const char *bytes, const uint64_t *offsets, uint64_t n, uint64_t *out) {
    if (!f || !offsets || (n && (!bytes || !out))) return SHG_ERR_ARG;
    for (uint64_t i = 0; i < n; i++)
        out[i] = flat_query(f, murmur64a((const uint8_t *)bytes + offsets[i], offsets[i + 1] - offsets[i], kMurmurSeed));
    return SHG_OK;
}

// getBits() (ShockHash2Flat.h:236-244) with the oracle's size formulas for the stand-in members:
// object (8 x 336 bytes), fallback PHF, free-position bit vector and its rank/select samples,
// retrieval bits, packed thresholds-and-seeds, 64 bits per seed-fallback entry.
uint64_t shg_flat_bits(const shg_flat *f) {
    if (!f) return 0;
    const uint64_t nfree = f->free_positions.size();
    const uint64_t bv = nfree ? nfree + f->free_positions.back() + 1 : 0;
    const uint64_t rank_select = nfree ? (bv / 512 + 1) * 8 + (nfree / 8192 + 1) * 4 : 0;
    const uint64_t w = f->fc.threshold_bits + f->fc.seed_bits;
    const uint64_t tas_bytes = ((f->nbuckets * w + 63) / 64) * 8;
    return 8 * 336 + shg_mphf_bits(f->fallback) + bv + 8 * rank_select + 8 * ((f->ribbon_n + 7) / 8) + 8 * tas_bytes +
           64 * f->seed_fallback.size();
}

} // extern "C"
