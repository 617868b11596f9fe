// Test infrastructure only (the oracle). Never linked into the shipped library.
//
// A single-threaded C++ restatement of the ShockHash construction path, written from the
// reference sources (paths relative to the reference project root) and used by the tests as the
// checker of the CUDA path, and by the benchmark as the "port" CPU baseline when the compiled
// reference (oracle/_ref) is not available. Each routine cites the reference lines it follows.
// The third-party primitives (SpookyHash V2, MurmurHash64A, remix, fastrange, remap16/128) come
// from oracle/shims/shg_thirdparty.h.
//
// Besides the products of construction it records, per search, the algorithmic work that the
// sequential reference performs up to its answer (hash evaluations, candidate pairs examined,
// pseudoforest edge operations), which is the unit of the search kernels' roofline.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <stdexcept>
#include <string>
#include <vector>
#include "../shims/shg_thirdparty.h"
#include "../keygen.h"

using namespace shg_tp;

namespace {

// ShockHash.h:47-50 (random start seed per tree depth).
const uint64_t START_SEED[20] = {
    0x106393c187cae21a, 0x6453cec3f7376937, 0x643e521ddbd2be98, 0x3740c6412f6572cb, 0x717d47562f1ce470,
    0x4cd6eb4c63befb7c, 0x9bfd8c5e18c8da73, 0x082f20e10092a9a3, 0x2ada2ce68d21defc, 0xe33cb4f3e7c6466b,
    0x3980be458c509c59, 0xc466fd9584828e8c, 0x45f0aabe1a61ede6, 0xf6e7b8b33ad9b98d, 0x4ef95e25f4b4983d,
    0x81175195173b92d3, 0x4e50927d8dd15978, 0x1ea2099d1fafae7f, 0x425c8a06fbaaa815, 0xcd4216006c74052a};

// ShockHash.h:53-61 (Rice parameter of an original-ShockHash leaf of size m).
const uint8_t BIJ_MEMO[61] = {0,  0,  0,  0,  0,  0,  1,  1,  2,  2,  2,  3,  3,  4,  4,  4,  5,  5,  6,  6,  7,
                              7,  8,  8,  9,  9,  9,  10, 10, 10, 11, 11, 12, 12, 13, 13, 13, 14, 15, 15, 15,
                              16, 16, 16, 17, 17, 18, 18, 19, 19, 19, 20, 20, 20, 21, 21, 22, 22, 23, 23, 23};
// ShockHash2.h:33-47 (Rice parameter of a bipartite leaf of size m).
const uint8_t BIJ_MEMO2[129] = {
    0,  0,  0,  0,  0,  0,  1,  3,  2,  4,  4,  6,  5,  7,  6,  8,  7,  8,  7,  9,  8,  10, 9,  11, 10, 11,
    11, 12, 11, 13, 12, 14, 13, 14, 14, 15, 14, 16, 15, 17, 16, 18, 17, 18, 17, 19, 18, 20, 19, 21, 20, 22,
    21, 22, 22, 23, 22, 24, 23, 25, 24, 26, 25, 27, 26, 27, 27, 28, 27, 29, 28, 30, 29, 31, 30, 32, 31, 33,
    32, 33, 33, 34, 33, 35, 34, 36, 35, 37, 36, 38, 37, 39, 38, 40, 38, 40, 40, 41, 40, 42, 41, 43, 42, 44,
    43, 45, 44, 45, 45, 47, 46, 47, 46, 48, 47, 49, 48, 50, 49, 51, 50, 52, 51, 53, 52, 54, 53, 54, 54};

const int MAX_BUCKET = 3000;  // ShockHash.h:33

struct Work {
    uint64_t split_evals = 0, leaf_evals = 0, pairs = 0, pairs_filtered = 0, uf_edges = 0, leaves = 0, splits = 0;
};

// Variant 5 is SIMDShockHash<l, false> (SIMDShockHash.hpp): ShockHash's tree, memo and leaves, with
// its own split hash and start seeds.
inline bool sh1_like(int variant) { return variant == 1 || variant == 5; }

// MurmurHash3's 32-bit finalizer (SIMDShockHash.hpp:76-83, remix32).
inline uint32_t fmix32(uint32_t z) {
    z ^= z >> 16;
    z *= 0x85ebca6bu;
    z ^= z >> 13;
    z *= 0xc2b2ae35u;
    z ^= z >> 16;
    return z;
}
// SIMDShockHash's split hash of z (= key + seed) onto [0, m): remixAndRemap, SIMDShockHash.hpp:762-766.
inline size_t simd_remap(uint64_t z, uint32_t m) { return remap16(fmix32(uint32_t(z >> 32) ^ uint32_t(z)), m); }

// Splitting thresholds: ShockHash.h:63-72 (variants 1, 5) and ShockHash2.h:49-56 (variant 2).
struct Config {
    int variant, leaf;
    size_t lower, upper;
    std::vector<uint64_t> memo;
    Config(int variant, int leaf) : variant(variant), leaf(leaf) {
        if (sh1_like(variant)) {
            lower = leaf * (leaf > 24 ? 4 : 2);
            upper = lower * (leaf > 24 ? 3 : 2);
        } else {
            lower = leaf * 4;
            upper = lower * 3;
        }
        memo.assign(MAX_BUCKET, 0);
        // fill_golomb_rice (ShockHash.h:121-127) / fill_golomb_rice2 (ShockHash2.h:106-115)
        size_t s = 0;
        for (; s <= (size_t)leaf; ++s) {
            uint64_t b = sh1_like(variant) ? BIJ_MEMO[s] : BIJ_MEMO2[s];
            memo[s] = b << 27 | (uint64_t)(s > 1) << 16 | b;
        }
        for (; s < (size_t)MAX_BUCKET; ++s) fill(s);
    }
    // _fill_golomb_rice (ShockHash.h:79-119) / _fill_golomb_rice2 (ShockHash2.h:63-104)
    void fill(size_t m) {
        long k[32] = {0};
        size_t fanout, unit;
        if (m > upper) {
            unit = upper * (uint16_t(m / 2 + upper - 1) / upper);
            fanout = 2;
        } else if (m > lower) {
            unit = lower;
            fanout = uint16_t(m + lower - 1) / lower;
        } else {
            unit = leaf;
            fanout = uint16_t(m + leaf - 1) / leaf;
        }
        k[fanout - 1] = m;
        for (size_t i = 0; i < fanout - 1; ++i) { k[i] = unit; k[fanout - 1] -= k[i]; }
        double sqrt_prod = 1;
        for (size_t i = 0; i < fanout; ++i) sqrt_prod *= sqrt((double)k[i]);
        const double p = sqrt((double)m) / (pow(2 * M_PI, (fanout - 1.) / 2) * sqrt_prod);
        uint64_t grl = (uint64_t)ceil(log2(-log((sqrt(5) + 1) / 2) / log1p(-p)));
        memo[m] = grl << 27;
        for (size_t i = 0; i < fanout; ++i) grl += memo[k[i]] & 0xFFFF;
        memo[m] |= grl;
        uint64_t nodes = 1;
        for (size_t i = 0; i < fanout; ++i) nodes += (memo[k[i]] >> 16) & 0x7FF;
        memo[m] |= nodes << 16;
    }
    int golomb(size_t m) const { return (int)(memo[m] >> 27); }
    size_t skip_bits(size_t m) const { return memo[m] & 0xFFFF; }
    size_t skip_nodes(size_t m) const { return (memo[m] >> 16) & 0x7FF; }
};

// Golomb-Rice bit stream, LSB first (RiceBitVector.h:67-127): per bucket, the fixed parts of all
// node codes in preorder, then their unary parts; buckets concatenated; final word count follows
// the builder's resize rule ((bits + 7) / 8 + 14) / 8.
struct BitWriter {
    std::vector<uint64_t> w;
    uint64_t bits = 0;
    void put(uint64_t v, int n) {  // n <= 64
        if (n == 0) return;
        if (n < 64) v &= (uint64_t(1) << n) - 1;
        size_t need = (bits + n + 63) / 64 + 1;
        if (w.size() < need) w.resize(need, 0);
        w[bits / 64] |= v << (bits & 63);
        if ((bits & 63) + n > 64) w[bits / 64 + 1] |= v >> (64 - (bits & 63));
        bits += n;
    }
    void unary(uint64_t u) {
        size_t need = (bits + u + 1 + 63) / 64 + 1;
        if (w.size() < need) w.resize(need, 0);
        bits += u;
        w[bits / 64] |= uint64_t(1) << (bits & 63);
        bits++;
    }
    std::vector<uint64_t> finish() {
        put(1, 1);  // sentinel, ShockHash.h:652
        size_t words = ((bits + 7) / 8 + 7 + 7) / 8;
        std::vector<uint64_t> out(words, 0);
        for (size_t i = 0; i < words && i < w.size(); i++) out[i] = w[i];
        return out;
    }
};

// ---------------------------------------------------------------- original ShockHash leaf
// TinyBinaryCuckooHashTable.h:138-149 (runtime range).
inline void cells_sh1(uint64_t key, uint64_t seed, uint32_t m, uint32_t &c1, uint32_t &c2) {
    uint64_t r = remix(key + seed);
    c1 = fastrange32((uint32_t)r, m / 2);
    c2 = fastrange32((uint32_t)(r >> 32), (m + 1) / 2) + m / 2;
}

// Cuckoo insertion with cycle detection (TinyBinaryCuckooHashTable.h:169-198); `cell` holds the
// key index occupying each cell or -1; `xr` the XOR of each key's two candidate cells.
bool cuckoo_insert(int *cell, uint32_t *xr, int e, uint32_t c1, uint32_t c2) {
    xr[e] = c1 ^ c2;
    if (cell[c1] < 0) { cell[c1] = e; return true; }
    if (cell[c2] < 0) { cell[c2] = e; return true; }
    const int orig = e;
    uint32_t cur = c1;
    const uint32_t origCell = cur;
    int entry = e;
    do {
        uint32_t alt = xr[entry] ^ cur;
        std::swap(entry, cell[alt]);
        if (entry < 0) return true;
        cur = alt;
    } while (cur != origCell || entry != orig);
    return false;
}

// ShockHash.h:404-434: smallest x >= start_seed[level] whose cells cover all m cells and whose
// ordered cuckoo insertion succeeds; retrieval bit per cell = (cell >= m/2), pushed in cell order.
uint64_t sh1_leaf(const uint64_t *keys, uint32_t m, int level, std::vector<std::pair<uint64_t, uint8_t>> &ribbon,
                  Work &work) {
    uint64_t x = START_SEED[level];
    const uint64_t all = (uint64_t(1) << m) - 1;
    std::vector<int> cell(m);
    std::vector<uint32_t> xr(m);
    for (;;) {
        for (;;) {
            uint64_t mask = 0;
            for (uint32_t i = 0; i < m; i++) {
                uint32_t c1, c2;
                cells_sh1(keys[i], x, m, c1, c2);
                mask |= (uint64_t(1) << c1) | (uint64_t(1) << c2);
            }
            work.leaf_evals += m;
            if (mask == all) break;
            x++;
        }
        std::fill(cell.begin(), cell.end(), -1);
        bool ok = true;
        for (uint32_t i = 0; i < m && ok; i++) {
            uint32_t c1, c2;
            cells_sh1(keys[i], x, m, c1, c2);
            ok = cuckoo_insert(cell.data(), xr.data(), (int)i, c1, c2);
        }
        if (ok) break;
        x++;
    }
    for (uint32_t i = 0; i < m; i++) ribbon.emplace_back(keys[cell[i]], i < m / 2 ? 0 : 1);
    work.leaves++;
    return x - START_SEED[level];
}

// ---------------------------------------------------------------- bipartite ShockHash leaf
// PairingFunction.h:47-96
inline uint64_t pair_tri(uint64_t x, uint64_t y) { return (x - 1) * x / 2 + y; }
inline void unpair_tri(uint64_t z, uint64_t &x, uint64_t &y) {
    x = (uint64_t)floor(0.5 + sqrt(0.25 + 2.0 * (double)z));
    y = z - ((x - 1) * x) / 2;
}
inline bool accurate_tri(uint64_t x, uint64_t y) {
    uint64_t a, b;
    unpair_tri(pair_tri(x, y), a, b);
    return a == x && b == y;
}
inline uint64_t pair_eleg(uint64_t x, uint64_t y) { return x < y ? y * y + x : x * x + x + y; }
inline void unpair_eleg(uint64_t z, uint64_t &x, uint64_t &y) {
    uint64_t f = (uint64_t)floor(sqrt((double)z));
    uint64_t sq = f * f;
    if (z - sq < f) { x = z - sq; y = f; } else { x = f; y = z - sq - f; }
}
inline bool accurate_eleg(uint64_t x, uint64_t y) {
    uint64_t a, b;
    unpair_eleg(pair_eleg(x, y), a, b);
    return a == x && b == y;
}

// BasicSeedCandidateFinder::hash / QuadSplitCandidateFinder::hash (ShockHash2-internal.h:100-102,
// 473-477): the half-table cell of `key` under a candidate seed.
inline uint32_t half_hash(uint64_t key, uint64_t s, uint32_t half) { return (uint32_t)fastrange64(remix(key + s), half); }
inline uint32_t cand_hash(uint64_t key, uint64_t seed, uint32_t m) {
    uint32_t half = (m + 1) / 2;
    if (m < 10) return half_hash(key, seed, half);
    uint64_t a, b;
    unpair_eleg(seed, a, b);
    return half_hash(key, (key & 1) == 0 ? a : b, half);
}

struct Cand {
    uint64_t seed;
    uint64_t iso[2];
    std::vector<uint8_t> h;
};

// calculateIsolatedVertices (ShockHash2-internal.h:34-46): key i is marked when its cell is hit by
// no other key of the same candidate.
void isolated(Cand &c, uint32_t m) {
    int hit[128] = {0};
    c.iso[0] = c.iso[1] = 0;
    for (uint32_t i = 0; i < m; i++) hit[c.h[i]]++;
    for (uint32_t i = 0; i < m; i++)
        if (hit[c.h[i]] == 1) c.iso[i >> 6] |= uint64_t(1) << (i & 63);
}

// CuckooUnionFind::unionIsStillPseudoforest (CuckooUnionFind.h:19-42).
bool cuf_union(uint32_t *cells, uint32_t c1, uint32_t c2) {
    const uint32_t EMPTY = ~0u;
    uint32_t entry = c1 ^ c2, orig = entry;
    if (cells[c1] == EMPTY) { cells[c1] = entry; return true; }
    if (cells[c2] == EMPTY) { cells[c2] = entry; return true; }
    uint32_t cur = c1, origCell = cur;
    do {
        uint32_t alt = entry ^ cur;
        std::swap(entry, cells[alt]);
        if (entry == EMPTY) return true;
        cur = alt;
    } while (cur != origCell || entry != orig);
    return false;
}

// Candidate stream. m < 10: BasicSeedCandidateFinder (ShockHash2-internal.h:68-98), every seed whose
// half hashes cover all (m+1)/2 cells, keys in given order. m >= 10: QuadSplitCandidateFinder with
// CandidateList (ShockHash2-internal.h:386-471): keys reordered into set A (even keys, in order)
// and set B (odd keys, from the back); every pair (seedA, seedB) whose combined coverage is full,
// in ascending pairElegant order.
struct Finder {
    uint32_t m, half, sizeA = 0;
    uint64_t full;
    std::vector<uint64_t> keys;  // reordered for QuadSplit
    std::vector<uint64_t> maskA, maskB;
    std::vector<Cand> pending;   // ascending seed order, front = next
    size_t pendingPos = 0;
    int64_t cur = -1;
    Work &work;
    Finder(const uint64_t *in, uint32_t m, Work &work) : m(m), half((m + 1) / 2), keys(m), work(work) {
        full = half >= 64 ? ~0ull : (uint64_t(1) << half) - 1;
        if (m < 10) {
            keys.assign(in, in + m);
        } else {
            for (uint32_t i = 0; i < m; i++) {
                if ((in[i] & 1) == 0) keys[sizeA++] = in[i];
                else keys[m - i + sizeA - 1] = in[i];
            }
        }
    }
    Cand make(uint64_t seedA, uint64_t seedB, uint64_t seed) {
        Cand c;
        c.seed = seed;
        c.h.resize(m);
        for (uint32_t i = 0; i < m; i++) c.h[i] = (uint8_t)half_hash(keys[i], i < sizeA ? seedA : seedB, half);
        work.leaf_evals += m;
        isolated(c, m);
        return c;
    }
    Cand next() {
        if (m < 10) {
            for (;;) {
                cur++;
                uint64_t taken = 0;
                for (uint32_t i = 0; i < m; i++) taken |= uint64_t(1) << half_hash(keys[i], (uint64_t)cur, half);
                work.leaf_evals += m;
                if (taken == full) return make(cur, cur, (uint64_t)cur);
            }
        }
        while (pendingPos >= pending.size()) {
            pending.clear();
            pendingPos = 0;
            cur++;
            const uint64_t s = (uint64_t)cur;
            uint64_t tA = 0, tB = 0;
            for (uint32_t i = 0; i < sizeA; i++) tA |= uint64_t(1) << half_hash(keys[i], s, half);
            for (uint32_t i = sizeA; i < m; i++) tB |= uint64_t(1) << half_hash(keys[i], s, half);
            work.leaf_evals += m;
            // earlier A masks against the new B mask: pairs (a < s, s), ascending a
            for (uint64_t a = 0; a < s; a++)
                if ((maskA[a] | tB) == full) {
                    if (accurate_eleg(a, s)) pending.push_back(make(a, s, pair_eleg(a, s)));
                }
            maskA.push_back(tA);
            maskB.push_back(tB);
            // all B masks so far (including s) against the new A mask: pairs (s, b <= s), ascending b
            for (uint64_t b = 0; b <= s; b++)
                if ((maskB[b] | tA) == full) {
                    if (accurate_eleg(s, b)) pending.push_back(make(s, b, pair_eleg(s, b)));
                }
        }
        return std::move(pending[pendingPos++]);
    }
};

// BijectionsShockHash2::findSeed (ShockHash2-internal.h:501-546) with isolatedVertexFilter=true.
uint64_t sh2_find_seed(const uint64_t *keys, uint32_t m, Work &work) {
    Finder f(keys, m, work);
    std::vector<Cand> cands;
    cands.push_back(f.next());
    std::vector<uint32_t> cells(m);
    for (;;) {
        Cand nc = f.next();
        for (const Cand &o : cands) {
            work.pairs++;
            if ((o.iso[0] & nc.iso[0]) | (o.iso[1] & nc.iso[1])) continue;
            work.pairs_filtered++;
            std::fill(cells.begin(), cells.end(), ~0u);
            uint32_t i = 0;
            for (; i < m; i++) {
                work.uf_edges++;
                if (!cuf_union(cells.data(), nc.h[i] + m / 2, o.h[i])) break;
            }
            if (i != m) continue;
            if (!accurate_tri(nc.seed, o.seed)) continue;
            return pair_tri(nc.seed, o.seed);
        }
        cands.push_back(std::move(nc));
    }
}

// BijectionsShockHash2::constructRetrieval (ShockHash2-internal.h:548-572): ordered cuckoo
// insertion of the keys in given order with cell1 = hash(seed1) + m/2, cell2 = hash(seed2); bit 1
// when the key ends up in its seed2 cell; pushed in key order.
void sh2_retrieval(const uint64_t *keys, uint32_t m, uint64_t seed, std::vector<std::pair<uint64_t, uint8_t>> &ribbon) {
    uint64_t s1, s2;
    unpair_tri(seed, s1, s2);
    std::vector<int> cell(m, -1);
    std::vector<uint32_t> xr(m);
    for (uint32_t k = 0; k < m; k++) {
        uint32_t c1 = cand_hash(keys[k], s1, m) + m / 2;
        uint32_t c2 = cand_hash(keys[k], s2, m);
        if (!cuckoo_insert(cell.data(), xr.data(), (int)k, c1, c2)) throw std::logic_error("Should be possible to construct");
    }
    for (uint32_t k = 0; k < m; k++) {
        uint32_t c2 = cand_hash(keys[k], s2, m);
        ribbon.emplace_back(keys[k], cell[c2] == (int)k ? 1 : 0);
    }
}

// BijectionsShockHash2::hash (ShockHash2-internal.h:574-584)
uint64_t sh2_query_leaf(uint32_t m, uint64_t seed, uint64_t key, uint64_t retrieved) {
    if (m <= 1) return 0;
    uint64_t s1, s2;
    unpair_tri(seed, s1, s2);
    return retrieved == 0 ? cand_hash(key, s1, m) + m / 2 : cand_hash(key, s2, m);
}

// ---------------------------------------------------------------- RecSplit tree
struct Builder {
    const Config &cfg;
    BitWriter &bw;
    std::vector<uint64_t> unary;
    std::vector<std::pair<uint64_t, uint8_t>> &ribbon;
    std::vector<uint64_t> &node_codes;  // every stored code, preorder, all buckets
    Work &work;
    std::vector<uint64_t> temp;
    Builder(const Config &cfg, BitWriter &bw, std::vector<std::pair<uint64_t, uint8_t>> &ribbon,
            std::vector<uint64_t> &node_codes, Work &work)
        : cfg(cfg), bw(bw), ribbon(ribbon), node_codes(node_codes), work(work), temp(MAX_BUCKET) {}

    void emit(uint64_t code, size_t m) {
        int g = cfg.golomb(m);
        bw.put(code, g);
        unary.push_back(code >> g);
        node_codes.push_back(code);
    }

    // Smallest x >= start_seed[level] with the exact part sizes, then the stable partition
    // (ShockHash.h:451-547 / ShockHash2.h:290-386). unit = part size, fanout parts, the last one
    // takes the rest; for the fanout-2 case the split point is `unit`.
    // Part of a key under seed x: fanout 2 splits at `unit` (h >= split goes right); otherwise
    // h / unit (the last part takes the remainder).
    // SIMDShockHash searches with its own hash (higherLevel, aggrLevel: SIMDShockHash.hpp:201-364).
    inline size_t part_of(uint64_t key, uint64_t x, size_t m, size_t unit, size_t fanout) const {
        size_t h = cfg.variant == 5 ? simd_remap(key + x, (uint32_t)m) : remap16(remix(key + x), (uint32_t)m);
        return fanout == 2 ? (h >= unit ? 1 : 0) : h / unit;
    }
    // `seed`: the index into START_SEED the search starts from (the depth, except for SIMDShockHash's
    // aggregation levels, SIMDShockHash.hpp:582, 593)
    uint64_t split(uint64_t *b, size_t m, size_t unit, size_t fanout, int seed) {
        uint64_t x = START_SEED[seed];
        size_t count[32];
        for (;;) {
            std::fill(count, count + 32, 0);
            for (size_t i = 0; i < m; i++) count[part_of(b[i], x, m, unit, fanout)]++;
            work.split_evals += m;
            bool ok = true;
            for (size_t i = 0; i + 1 < fanout; i++) ok &= count[i] == unit;
            if (ok) break;
            x++;
        }
        size_t pos[32];
        for (size_t i = 0, c = 0; i < fanout; i++, c += unit) pos[i] = c;
        for (size_t i = 0; i < m; i++) temp[pos[part_of(b[i], x, m, unit, fanout)]++] = b[i];
        std::copy(temp.begin(), temp.begin() + m, b);
        work.splits++;
        return x - START_SEED[seed];
    }

    void rec(uint64_t *b, size_t m, int level) {
        const size_t leaf = cfg.leaf;
        if (m <= leaf) {
            uint64_t code;
            if (sh1_like(cfg.variant)) {
                // SIMDShockHash's leaves start at START_SEED[19] (SIMDShockHash.hpp:411)
                code = sh1_leaf(b, (uint32_t)m, cfg.variant == 5 ? 19 : level, ribbon, work);
            } else {
                code = sh2_find_seed(b, (uint32_t)m, work);
                sh2_retrieval(b, (uint32_t)m, code, ribbon);
                work.leaves++;
            }
            emit(code, m);
            return;
        }
        if (m > cfg.upper) {
            // fanout 2: part 0 = [0, split), part 1 = the rest; remap16 < split  <=>  h / split == 0
            const size_t sp = (uint16_t(m / 2 + cfg.upper - 1) / cfg.upper) * cfg.upper;
            uint64_t x = split(b, m, sp, 2, level);
            emit(x, m);
            rec(b, sp, level + 1);
            if (m - sp > 1) rec(b + sp, m - sp, level + 1);
        } else {
            const size_t unit = m > cfg.lower ? cfg.lower : leaf;
            const size_t fanout = uint16_t(m + unit - 1) / unit;
            const int seed = cfg.variant == 5 ? (unit == leaf ? 18 : 17) : level;
            uint64_t x = split(b, m, unit, fanout, seed);
            emit(x, m);
            size_t i;
            for (i = 0; i < m - unit; i += unit) rec(b + i, unit, level + 1);
            if (m - i > 1) rec(b + i, m - i, level + 1);
        }
    }
};

struct PortResult {
    int variant, leaf;
    Config cfg;
    uint64_t n, nbuckets;
    std::vector<uint64_t> size_acc, pos_acc, desc, node_codes, sorted_keys;
    std::vector<std::pair<uint64_t, uint8_t>> ribbon;
    std::vector<std::pair<uint64_t, uint8_t>> ribbon_sorted;
    Work work;
    PortResult(int v, int l) : variant(v), leaf(l), cfg(v, l) {}
};

// hash_gen (ShockHash.h:602-654 / ShockHash2.h:441-494) with parallelPartition (Sorter.hpp:15-36):
// sort by `first` (ties by input position), bucket = remap128(first, nbuckets).
// A shard (nb_map != 0) holds the buckets [b0, b0 + nb_local) of a structure with nb_map buckets,
// built from exactly the keys that fall in them; bucket = remap128(first, nb_map) - b0.
PortResult *build(int variant, int leaf, const uint64_t *first, const uint64_t *second, uint64_t n, uint64_t bucket_size,
                  uint64_t nb_map = 0, uint64_t b0 = 0, uint64_t nb_local = 0) {
    auto *r = new PortResult(variant, leaf);
    r->n = n;
    r->nbuckets = std::max<uint64_t>(1, (n + bucket_size - 1) / bucket_size);
    if (nb_map) r->nbuckets = nb_local;
    else nb_map = r->nbuckets;
    std::vector<uint64_t> idx(n);
    for (uint64_t i = 0; i < n; i++) idx[i] = i;
    std::stable_sort(idx.begin(), idx.end(), [&](uint64_t a, uint64_t b) { return first[a] < first[b]; });
    r->sorted_keys.resize(n);
    r->size_acc.assign(r->nbuckets + 1, 0);
    {
        uint64_t i = 0;
        for (uint64_t bk = 0; bk < r->nbuckets; bk++) {
            r->size_acc[bk] = i;
            while (i < n && remap128(first[idx[i]], nb_map) - b0 == bk) { r->sorted_keys[i] = second[idx[i]]; i++; }
        }
        if (i != n) throw std::runtime_error("a key lies outside the shard's buckets");
        r->size_acc[r->nbuckets] = n;
    }
    std::vector<uint64_t> keys = r->sorted_keys;
    BitWriter bw;
    Builder bld(r->cfg, bw, r->ribbon, r->node_codes, r->work);
    r->pos_acc.assign(r->nbuckets + 1, 0);
    for (uint64_t bk = 0; bk < r->nbuckets; bk++) {
        const uint64_t s = r->size_acc[bk + 1] - r->size_acc[bk];
        if (s > (uint64_t)MAX_BUCKET - 1) throw std::runtime_error("bucket too large");
        if (s > 1) {
            bld.rec(keys.data() + r->size_acc[bk], s, 0);
            for (uint64_t u : bld.unary) bw.unary(u);
            bld.unary.clear();
        }
        r->pos_acc[bk + 1] = bw.bits;
    }
    r->desc = bw.finish();
    r->sorted_keys = keys;  // keys after all stable partitions (leaf order)
    r->ribbon_sorted = r->ribbon;
    std::sort(r->ribbon_sorted.begin(), r->ribbon_sorted.end());
    return r;
}

// ---------------------------------------------------------------- query
// RiceBitVector::Reader (RiceBitVector.h:149-213)
struct Reader {
    const std::vector<uint64_t> &d;
    size_t fixed_off = 0;
    uint64_t window = 0;
    size_t ptr = 0;
    int valid = 0;
    explicit Reader(const std::vector<uint64_t> &d) : d(d) {}
    uint64_t word(size_t i) const { return i < d.size() ? d[i] : 0; }
    uint64_t next(int g) {
        uint64_t result = 0;
        if (window == 0) {
            result += valid;
            window = word(ptr++);
            valid = 64;
            while (window == 0) { result += 64; window = word(ptr++); }
        }
        const int pos = __builtin_ctzll(window);
        window >>= pos;
        window >>= 1;
        valid -= pos + 1;
        result += pos;
        result <<= g;
        uint64_t lo = word(fixed_off / 64), hi = word(fixed_off / 64 + 1);
        unsigned __int128 f = ((unsigned __int128)hi << 64) | lo;
        result |= (uint64_t)(f >> (fixed_off % 64)) & ((uint64_t(1) << g) - 1);
        fixed_off += g;
        return result;
    }
    void skip(size_t nodes, size_t fixed_len) {
        size_t missing = nodes, cnt;
        while ((cnt = __builtin_popcountll(window)) < missing) {
            window = word(ptr++);
            missing -= cnt;
            valid = 64;
        }
        uint64_t w = window;
        for (size_t i = 0; i + 1 < missing; i++) w &= w - 1;
        cnt = __builtin_ctzll(w);
        window >>= cnt;
        window >>= 1;
        valid -= cnt + 1;
        fixed_off += fixed_len;
    }
    void reset(size_t bit_pos, size_t unary_off) {
        fixed_off = bit_pos;
        size_t up = bit_pos + unary_off;
        ptr = up / 64;
        window = word(ptr++) >> (up & 63);
        valid = 64 - (up & 63);
    }
};

uint64_t retrieve(const PortResult *r, uint64_t key) {
    auto it = std::lower_bound(r->ribbon_sorted.begin(), r->ribbon_sorted.end(), std::make_pair(key, (uint8_t)0));
    return (it != r->ribbon_sorted.end() && it->first == key) ? it->second : 0;
}

// operator() (ShockHash.h:199-270 / ShockHash2.h:178-230)
uint64_t query(const PortResult *r, uint64_t first, uint64_t second) {
    const Config &c = r->cfg;
    const uint64_t bucket = remap128(first, r->nbuckets);
    uint64_t cum = r->size_acc[bucket];
    size_t m = r->size_acc[bucket + 1] - cum;
    Reader rd(r->desc);
    rd.reset(r->pos_acc[bucket], c.skip_bits(m));
    int level = 0;
    const bool simd = r->variant == 5;  // SIMDShockHash.hpp:779-844
    auto hsplit = [simd](uint64_t z, size_t range) {
        return simd ? simd_remap(z, (uint32_t)range) : remap16(remix(z), (uint32_t)range);
    };
    while (m > c.upper) {
        uint64_t d = rd.next(c.golomb(m));
        size_t h = hsplit(second + d + START_SEED[level], m);
        const size_t sp = (uint16_t(m / 2 + c.upper - 1) / c.upper) * c.upper;
        if (h < sp) m = sp;
        else { rd.skip(c.skip_nodes(sp), c.skip_bits(sp)); m -= sp; cum += sp; }
        level++;
    }
    if (m > c.lower) {
        uint64_t d = rd.next(c.golomb(m));
        size_t h = hsplit(second + d + START_SEED[simd ? 17 : level], m);
        size_t part = uint16_t(h) / c.lower;
        m = std::min(c.lower, m - part * c.lower);
        cum += c.lower * part;
        if (part) rd.skip(c.skip_nodes(c.lower) * part, c.skip_bits(c.lower) * part);
        level++;
    }
    if (m > (size_t)c.leaf) {
        uint64_t d = rd.next(c.golomb(m));
        size_t h = hsplit(second + d + START_SEED[simd ? 18 : level], m);
        size_t part = uint16_t(h) / c.leaf;
        m = std::min((size_t)c.leaf, m - part * c.leaf);
        cum += c.leaf * part;
        if (part) rd.skip(part, c.skip_bits(c.leaf) * part);
        level++;
    }
    uint64_t b = rd.next(c.golomb(m));
    uint64_t ret = retrieve(r, second);
    if (sh1_like(r->variant)) {
        uint32_t c1, c2;
        cells_sh1(second, b + START_SEED[simd ? 19 : level], (uint32_t)m, c1, c2);
        return cum + (ret == 0 ? c1 : c2);
    }
    return cum + sh2_query_leaf((uint32_t)m, b, second, ret);
}

} // namespace

extern "C" {

void port_spooky128(const char *bytes, const uint64_t *offsets, size_t n, uint64_t *first, uint64_t *second) {
    for (size_t i = 0; i < n; i++) {
        uint64_t h0 = 0, h1 = 0;
        spooky_hash128(bytes + offsets[i], offsets[i + 1] - offsets[i], &h0, &h1);
        first[i] = h1;
        second[i] = h0;
    }
}

// The memo table (3000 entries) of variant/leaf.
void port_memo(int variant, int leaf, uint64_t *out) {
    Config c(variant, leaf);
    for (int i = 0; i < MAX_BUCKET; i++) out[i] = c.memo[i];
}

void *port_build(int variant, int leaf, const uint64_t *first, const uint64_t *second, uint64_t n, uint64_t bucket_size) {
    try {
        return build(variant, leaf, first, second, n, bucket_size);
    } catch (...) {
        return nullptr;
    }
}
void *port_build_shard(int variant, int leaf, const uint64_t *first, const uint64_t *second, uint64_t n,
                       uint64_t bucket_size, uint64_t nb_global, uint64_t b0, uint64_t b1) {
    try {
        if (b0 >= b1 || b1 > nb_global) return nullptr;
        return build(variant, leaf, first, second, n, bucket_size, nb_global, b0, b1 - b0);
    } catch (...) {
        return nullptr;
    }
}
void port_free(void *h) { delete (PortResult *)h; }
uint64_t port_nbuckets(void *h) { return ((PortResult *)h)->nbuckets; }
uint64_t port_desc_words(void *h) { return ((PortResult *)h)->desc.size(); }
void port_get_desc(void *h, uint64_t *out) {
    auto *r = (PortResult *)h;
    std::memcpy(out, r->desc.data(), r->desc.size() * 8);
}
void port_get_acc(void *h, uint64_t *size_acc, uint64_t *pos_acc) {
    auto *r = (PortResult *)h;
    std::memcpy(size_acc, r->size_acc.data(), r->size_acc.size() * 8);
    std::memcpy(pos_acc, r->pos_acc.data(), r->pos_acc.size() * 8);
}
uint64_t port_ribbon_n(void *h) { return ((PortResult *)h)->ribbon.size(); }
void port_get_ribbon(void *h, uint64_t *keys, uint8_t *bits) {
    auto &v = ((PortResult *)h)->ribbon;
    for (size_t i = 0; i < v.size(); i++) { keys[i] = v[i].first; bits[i] = v[i].second; }
}
uint64_t port_node_count(void *h) { return ((PortResult *)h)->node_codes.size(); }
void port_get_node_codes(void *h, uint64_t *out) {
    auto *r = (PortResult *)h;
    std::memcpy(out, r->node_codes.data(), r->node_codes.size() * 8);
}
void port_get_sorted_keys(void *h, uint64_t *out) {
    auto *r = (PortResult *)h;
    std::memcpy(out, r->sorted_keys.data(), r->sorted_keys.size() * 8);
}
// work[0..6] = split_evals, leaf_evals, pairs, pairs_filtered, uf_edges, leaves, splits
void port_get_work(void *h, uint64_t *w) {
    auto &k = ((PortResult *)h)->work;
    w[0] = k.split_evals; w[1] = k.leaf_evals; w[2] = k.pairs; w[3] = k.pairs_filtered;
    w[4] = k.uf_edges; w[5] = k.leaves; w[6] = k.splits;
}
void port_query_hash(void *h, const uint64_t *first, const uint64_t *second, size_t n, uint64_t *out) {
    auto *r = (PortResult *)h;
    for (size_t i = 0; i < n; i++) out[i] = query(r, first[i], second[i]);
}

// Single leaves, for the exhaustive small-leaf tests.
uint64_t port_sh2_leaf(uint32_t m, const uint64_t *keys, uint64_t *rkeys, uint8_t *rbits, uint64_t *work7) {
    Work w;
    uint64_t seed = sh2_find_seed(keys, m, w);
    std::vector<std::pair<uint64_t, uint8_t>> rb;
    sh2_retrieval(keys, m, seed, rb);
    for (size_t i = 0; i < rb.size(); i++) { rkeys[i] = rb[i].first; rbits[i] = rb[i].second; }
    if (work7) { work7[0] = w.split_evals; work7[1] = w.leaf_evals; work7[2] = w.pairs; work7[3] = w.pairs_filtered; work7[4] = w.uf_edges; }
    return seed;
}
uint64_t port_sh2_leaf_query(uint32_t m, uint64_t seed, uint64_t key, uint64_t retrieved) {
    return sh2_query_leaf(m, seed, key, retrieved);
}
uint64_t port_sh1_leaf(uint32_t m, int level, const uint64_t *keys, uint64_t *rkeys, uint8_t *rbits) {
    Work w;
    std::vector<std::pair<uint64_t, uint8_t>> rb;
    uint64_t code = sh1_leaf(keys, m, level, rb, w);
    for (size_t i = 0; i < rb.size(); i++) { rkeys[i] = rb[i].first; rbits[i] = rb[i].second; }
    return code;
}

} // extern "C"

SHG_ORACLE_KEYGEN_EXPORTS(port_)
