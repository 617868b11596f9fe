// Planning of a build: the Golomb-Rice memo of a configuration and the RecSplit tree of every
// bucket size, in preorder. The tree's shape depends only on the bucket size, so one shape per
// size is derived here (mirroring the recursion of ShockHash.h:303-555 / ShockHash2.h:259-394) and
// the device stamps it out for every bucket of that size (k_plan_expand).
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <stdexcept>
#include <mutex>
#include <vector>
#include "shg_common.cuh"
#include "shg_internal.h"

namespace shg {

// ShockHash.h:53-61
static const uint8_t kBijMemo[61] = {0,  0,  0,  0,  0,  0,  1,  1,  2,  2,  2,  3,  3,  4,  4,  4,  5,  5,  6,  6,  7,
                                     7,  8,  8,  9,  9,  9,  10, 10, 10, 11, 11, 12, 12, 13, 13, 13, 14, 15, 15, 15,
                                     16, 16, 16, 17, 17, 18, 18, 19, 19, 19, 20, 20, 20, 21, 21, 22, 22, 23, 23, 23};
// ShockHash2.h:33-47
static const uint8_t kBijMemo2[129] = {
    0,  0,  0,  0,  0,  0,  1,  3,  2,  4,  4,  6,  5,  7,  6,  8,  7,  8,  7,  9,  8,  10, 9,  11, 10, 11,
    11, 12, 11, 13, 12, 14, 13, 14, 14, 15, 14, 16, 15, 17, 16, 18, 17, 18, 17, 19, 18, 20, 19, 21, 20, 22,
    21, 22, 22, 23, 22, 24, 23, 25, 24, 26, 25, 27, 26, 27, 27, 28, 27, 29, 28, 30, 29, 31, 30, 32, 31, 33,
    32, 33, 33, 34, 33, 35, 34, 36, 35, 37, 36, 38, 37, 39, 38, 40, 38, 40, 40, 41, 40, 42, 41, 43, 42, 44,
    43, 45, 44, 45, 45, 47, 46, 47, 46, 48, 47, 49, 48, 50, 49, 51, 50, 52, 51, 53, 52, 54, 53, 54, 54};

struct ShapeCache {
    std::mutex mu;
    std::vector<Shape> cache = std::vector<Shape>(kMaxBucket);
    std::vector<char> have = std::vector<char>(kMaxBucket, 0);
};

Config::Config(int variant_, int leaf_) : variant(variant_), leaf(leaf_), shapes(std::make_shared<ShapeCache>()) {
    if (is_sh1(variant)) {
        lower = leaf * (leaf > 24 ? 4 : 2);
        upper = lower * (leaf > 24 ? 3 : 2);
    } else {
        lower = leaf * 4;
        upper = lower * 3;
    }
    memo.assign(kMaxBucket, 0);
    uint32_t s = 0;
    // fill_golomb_rice (ShockHash.h:121-127) / fill_golomb_rice2 (ShockHash2.h:106-115)
    for (; s <= (uint32_t)leaf; ++s) {
        const uint64_t b = is_sh1(variant) ? kBijMemo[s] : kBijMemo2[s];
        memo[s] = b << 27 | (uint64_t)(s > 1) << 16 | b;
    }
    // _fill_golomb_rice (ShockHash.h:79-119) / _fill_golomb_rice2 (ShockHash2.h:63-104): the Rice
    // parameter of a split is ceil(log2(-ln(phi) / ln(1 - p))) with p the probability that a
    // random seed yields the exact part sizes.
    for (; s < (uint32_t)kMaxBucket; ++s) {
        const uint32_t m = s;
        long k[32] = {0};
        uint32_t fanout, unit;
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
        for (uint32_t i = 0; i < fanout - 1; ++i) { k[i] = unit; k[fanout - 1] -= k[i]; }
        double sqrt_prod = 1;
        for (uint32_t i = 0; i < fanout; ++i) sqrt_prod *= std::sqrt((double)k[i]);
        const double p = std::sqrt((double)m) / (std::pow(2 * M_PI, (fanout - 1.) / 2) * sqrt_prod);
        uint64_t grl = (uint64_t)std::ceil(std::log2(-std::log((std::sqrt(5) + 1) / 2) / std::log1p(-p)));
        memo[m] = grl << 27;
        for (uint32_t i = 0; i < fanout; ++i) grl += memo[k[i]] & 0xFFFF;
        memo[m] |= grl;
        uint64_t nodes = 1;
        for (uint32_t i = 0; i < fanout; ++i) nodes += (memo[k[i]] >> 16) & 0x7FF;
        memo[m] |= nodes << 16;
    }
}

namespace {
struct ShapeBuilder {
    const Config &c;
    Shape &sh;
    uint32_t fixed = 0;
    void rec(uint32_t rel, uint32_t m, int level) {
        if (level >= kMaxLevels) throw std::runtime_error("tree deeper than the start-seed table");
        if (level + 1 > sh.depth) sh.depth = level + 1;
        TNode t{};
        t.rel = (uint16_t)rel;
        t.m = (uint16_t)m;
        t.level = (uint8_t)level;
        t.g = (uint8_t)c.golomb(m);
        t.fixed_off = (uint16_t)fixed;
        t.seed = (uint8_t)level;
        fixed += t.g;
        const bool simd = is_simd(c.variant);
        if (m <= (uint32_t)c.leaf) {
            t.kind = kLeaf;
            if (simd) t.seed = kSimdSeedLeaf;
            sh.nodes.push_back(t);
            return;
        }
        if (m > c.upper) {
            const uint32_t sp = (uint16_t(m / 2 + c.upper - 1) / c.upper) * c.upper;
            t.kind = kSplit2;
            t.unit = (uint16_t)sp;
            t.fanout = 2;
            sh.nodes.push_back(t);
            rec(rel, sp, level + 1);
            if (m - sp > 1) rec(rel + sp, m - sp, level + 1);
            else sh.singles.push_back((uint16_t)(rel + sp));
        } else {
            const uint32_t unit = m > c.lower ? c.lower : (uint32_t)c.leaf;
            t.kind = kSplitK;
            t.unit = (uint16_t)unit;
            if (simd) t.seed = unit == (uint32_t)c.leaf ? kSimdSeedLeafAggr : kSimdSeedLower;
            t.fanout = (uint8_t)(uint16_t(m + unit - 1) / unit);
            sh.nodes.push_back(t);
            uint32_t i;
            for (i = 0; i < m - unit; i += unit) rec(rel + i, unit, level + 1);
            if (m - i > 1) rec(rel + i, m - i, level + 1);
            else sh.singles.push_back((uint16_t)(rel + i));
        }
    }
};
} // namespace

const Shape &shape_of(const Config &c, uint32_t m, std::vector<Shape> &cache, std::vector<char> &have) {
    if (!have[m]) {
        Shape &sh = cache[m];
        sh = Shape();
        if (m == 1) sh.singles.push_back(0);
        if (m > 1) {
            ShapeBuilder b{c, sh};
            b.rec(0, m, 0);
        }
        have[m] = 1;
    }
    return cache[m];
}

void make_shape_tables(const Config &c, uint32_t rows, ShapeTables &t) {
    if (rows > (uint32_t)kMaxBucket) throw std::runtime_error("bucket size beyond MAX_BUCKET_SIZE");
    // shapes depend only on the configuration and the bucket size: reuse them across builds
    std::shared_ptr<ShapeCache> sc = c.shapes ? c.shapes : std::make_shared<ShapeCache>();
    std::lock_guard<std::mutex> lock(sc->mu);
    int depth = 0;
    for (uint32_t m = 0; m < rows; m++) depth = std::max(depth, shape_of(c, m, sc->cache, sc->have).depth);
    t.rows = rows;
    t.ncol = kColLevel0 + depth;
    t.cnt.assign((size_t)rows * t.ncol, 0);
    t.nodes.clear();
    t.singles.clear();
    t.node_off.assign(rows + 1, 0);
    t.single_off.assign(rows + 1, 0);
    for (uint32_t m = 0; m < rows; m++) {
        const Shape &sh = shape_of(c, m, sc->cache, sc->have);
        uint32_t *row = &t.cnt[(size_t)m * t.ncol];
        t.node_off[m] = (uint32_t)t.nodes.size();
        t.single_off[m] = (uint32_t)t.singles.size();
        for (const TNode &tn : sh.nodes) {
            ShapeNode n{};
            n.rel = tn.rel;
            n.m = tn.m;
            n.level = tn.level;
            n.kind = tn.kind;
            n.fanout = tn.fanout;
            n.g = tn.g;
            n.unit = tn.unit;
            n.fixed_off = tn.fixed_off;
            n.seed = tn.seed;
            const int col = tn.kind == kLeaf ? kColLeaves : kColLevel0 + tn.level;
            n.rank = (uint16_t)row[col]++;
            t.nodes.push_back(n);
        }
        row[kColNodes] = (uint32_t)sh.nodes.size();
        row[kColSingles] = (uint32_t)sh.singles.size();
        t.singles.insert(t.singles.end(), sh.singles.begin(), sh.singles.end());
    }
    t.node_off[rows] = (uint32_t)t.nodes.size();
    t.single_off[rows] = (uint32_t)t.singles.size();
}

} // namespace shg
