// Host check of the device plan's tables (no GPU): the shape tables of shg_plan.cpp, read the way
// k_plan_scan (per-column exclusive scans over buckets, computed in 1024 contiguous runs) and
// k_plan_expand (shape nodes stamped out at the bucket's offsets, node ids into launch lists by
// rank) read them, must give the node list, launch lists and size-1 positions of a direct
// per-bucket expansion of the same trees: buckets in order, preorder inside a bucket, split ids by
// level, then the leaves. Prints "ok" and exits 0 when every case agrees.
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <random>
#include <vector>
#include "shg_common.cuh"
#include "shg_internal.h"
using namespace shg;

namespace {

struct Direct {
    std::vector<Node> nodes;
    std::vector<uint16_t> fixed_off;
    std::vector<uint32_t> node_begin;
    std::vector<std::vector<uint32_t>> levels;
    std::vector<uint32_t> leaves;
    std::vector<uint64_t> singles;
};

void direct_plan(const Config &c, const std::vector<uint64_t> &acc, Direct &d) {
    std::vector<Shape> cache(kMaxBucket);
    std::vector<char> have(kMaxBucket, 0);
    const uint64_t nb = acc.size() - 1;
    uint32_t id = 0;
    d.node_begin.assign(nb + 1, 0);
    for (uint64_t b = 0; b < nb; b++) {
        d.node_begin[b] = id;
        const uint32_t m = (uint32_t)(acc[b + 1] - acc[b]);
        const Shape &sh = shape_of(c, m, cache, have);
        for (uint16_t s : sh.singles) d.singles.push_back(acc[b] + s);
        for (const TNode &t : sh.nodes) {
            Node n{};
            n.start = (uint32_t)(acc[b] + t.rel);
            n.m = t.m;
            n.level = t.level;
            n.kind = t.kind;
            n.bucket = (uint32_t)b;
            n.unit = t.unit;
            n.fanout = t.fanout;
            n.g = t.g;
            d.nodes.push_back(n);
            d.fixed_off.push_back(t.fixed_off);
            if (t.kind == kLeaf) {
                d.leaves.push_back(id);
            } else {
                if (d.levels.size() <= t.level) d.levels.resize(t.level + 1);
                d.levels[t.level].push_back(id);
            }
            id++;
        }
    }
    d.node_begin[nb] = id;
}

bool check(const Config &c, const std::vector<uint64_t> &acc, uint32_t rows) {
    const uint64_t nb = acc.size() - 1, stride = nb + 1;
    ShapeTables t;
    make_shape_tables(c, rows, t);
    const int ncol = t.ncol;
    // k_plan_scan: column by column, 1024 contiguous runs of buckets, exclusive prefix
    std::vector<uint32_t> offs((uint64_t)ncol * stride + kMaxPlanCols, 0);
    auto count_of = [&](uint64_t b, int col) -> uint32_t {
        const uint64_t m = acc[b + 1] - acc[b];
        return m < t.rows ? t.cnt[m * ncol + col] : 0u;
    };
    const uint64_t run = (nb + 1023) / 1024;
    for (int col = 0; col < ncol; col++) {
        uint32_t total = 0;
        for (int th = 0; th < 1024; th++) {
            const uint64_t lo = std::min<uint64_t>(nb, th * run), hi = std::min<uint64_t>(nb, lo + run);
            for (uint64_t b = lo; b < hi; b++) {
                offs[col * stride + b] = total;
                total += count_of(b, col);
            }
        }
        offs[col * stride + nb] = total;
        offs[(uint64_t)ncol * stride + col] = total;
    }
    const uint32_t *tot = &offs[(uint64_t)ncol * stride];
    ListOffsets lists{};
    uint64_t nids = 0;
    for (int lv = 0; lv < ncol - kColLevel0; lv++) {
        lists.level[lv] = (uint32_t)nids;
        nids += tot[kColLevel0 + lv];
    }
    lists.leaf = (uint32_t)nids;
    nids += tot[kColLeaves];
    // k_plan_expand
    std::vector<Node> nodes(tot[kColNodes]);
    std::vector<uint16_t> fixed(tot[kColNodes]);
    std::vector<uint32_t> ids(nids, 0xffffffffu);
    std::vector<uint64_t> singles(tot[kColSingles], ~0ull);
    for (uint64_t b = 0; b < nb; b++) {
        const uint64_t a0 = acc[b], m = acc[b + 1] - a0;
        if (m >= t.rows) return false;
        const uint32_t node0 = offs[kColNodes * stride + b];
        for (uint32_t j = t.node_off[m]; j < t.node_off[m + 1]; j++) {
            const ShapeNode &s = t.nodes[j];
            const uint32_t id = node0 + (j - t.node_off[m]);
            Node n{};
            n.start = (uint32_t)(a0 + s.rel);
            n.m = s.m;
            n.level = s.level;
            n.kind = s.kind;
            n.bucket = (uint32_t)b;
            n.unit = s.unit;
            n.fanout = s.fanout;
            n.g = s.g;
            nodes.at(id) = n;
            fixed.at(id) = s.fixed_off;
            if (s.kind == kLeaf)
                ids.at(lists.leaf + offs[kColLeaves * stride + b] + s.rank) = id;
            else
                ids.at(lists.level[s.level] + offs[(kColLevel0 + s.level) * stride + b] + s.rank) = id;
        }
        const uint32_t sb = offs[kColSingles * stride + b];
        for (uint32_t j = t.single_off[m]; j < t.single_off[m + 1]; j++)
            singles.at(sb + (j - t.single_off[m])) = a0 + t.singles[j];
    }
    Direct d;
    direct_plan(c, acc, d);
    std::vector<uint32_t> want;
    for (auto &l : d.levels) want.insert(want.end(), l.begin(), l.end());
    want.insert(want.end(), d.leaves.begin(), d.leaves.end());
    bool ok = d.nodes.size() == nodes.size() &&
              memcmp(d.nodes.data(), nodes.data(), nodes.size() * sizeof(Node)) == 0 && d.fixed_off == fixed &&
              d.singles == singles && want == ids;
    for (uint64_t b = 0; b <= nb; b++) ok = ok && d.node_begin[b] == offs[kColNodes * stride + b];
    for (int lv = (int)d.levels.size(); lv < ncol - kColLevel0; lv++) ok = ok && tot[kColLevel0 + lv] == 0;
    return ok;
}

} // namespace

int main() {
    struct Case { int variant, leaf; uint32_t bucket; } cases[] = {
        {2, 64, 2000}, {1, 30, 2000}, {1, 40, 2000}, {3, 8, 2000}, {2, 9, 100}, {2, 128, 2500}, {1, 2, 50}, {2, 2, 7}};
    int fails = 0;
    for (const Case &cs : cases) {
        const Config c(cs.variant, cs.leaf);
        std::mt19937_64 rng(cs.variant * 1000 + cs.leaf);
        for (int trial = 0; trial < 3; trial++) {
            const uint64_t nb = trial == 0 ? 1 : 1 + rng() % 2500;
            std::vector<uint64_t> acc(nb + 1, 0);
            std::normal_distribution<double> nd(cs.bucket, std::sqrt((double)cs.bucket));
            uint32_t maxsz = 0;
            for (uint64_t b = 0; b < nb; b++) {
                long m = (long)nd(rng);
                if (rng() % 50 == 0) m = (long)(rng() % 4);  // empty, single and tiny buckets
                if (rng() % 200 == 0) m = kMaxBucket - 1;
                m = std::max(0L, std::min<long>(m, kMaxBucket - 1));
                acc[b + 1] = acc[b] + (uint64_t)m;
                maxsz = std::max<uint32_t>(maxsz, (uint32_t)m);
            }
            // tables grown the way the engine grows them: a quarter above the largest bucket
            const uint32_t rows = std::min<uint32_t>(kMaxBucket, ((maxsz + 1 + (maxsz + 1) / 4 + 255) / 256) * 256);
            if (!check(c, acc, rows)) {
                printf("mismatch: variant %d leaf %d buckets %lu\n", cs.variant, cs.leaf, (unsigned long)nb);
                fails++;
            }
        }
    }
    if (fails) return 1;
    printf("ok\n");
    return 0;
}
