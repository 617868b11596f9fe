// Bipartite ShockHash leaf search (ShockHash2-internal.h:34-107, 386-572; ShockHash2-precompiled.cpp:24-47),
// one warp per leaf, leaves pulled from a device counter.
//
// The reference finds the first pair, in lexicographic order of (new candidate j, earlier
// candidate i), that passes the isolated-key filter and the pseudoforest test, where candidates
// arrive in ascending candidate-seed order. This kernel computes the same pair with the work laid
// out for a warp:
//   1. raw seeds are hashed 32 at a time (one seed per lane): coverage masks of set A / set B
//      (32-bit masks for leaves of up to 64 keys) and the seed's cell row (one byte per key);
//   2. the candidates whose larger raw seed lies in that block of 32 are listed in the reference's
//      order (lane L owns raw seed s0+L; its candidates (a<s, s) by a, then (s, b<=s) by b; lanes in
//      order): one scan over the earlier seeds' paired masks, the first partners kept in
//      registers, a warp prefix sum for the positions;
//   3. every new candidate's cell row and isolated-key mask are assembled from its two raw seeds'
//      rows (one candidate per lane);
//   4. all pairs (j, i) of the new batch are filtered lane-parallel in lexicographic order; the
//      survivors go through a queue, 32 pseudoforest tests at a time (one per lane, union-find with
//      a cycle flag per root over the cached cell rows); fewer than 32 wait for the next batch,
//      and the first passing survivor in queue order is the answer.
// Candidate and raw-seed state live in shared memory; indices past its capacity spill to a
// per-warp slice of global scratch, which also holds the cell rows. For leaves of more than 64
// keys, whose raw seeds run into the thousands, step 2 streams the spilled masks of earlier rounds
// through a shared-memory ring (cp.async, two chunks of 32 ahead) instead of loading them per lane.
#include <algorithm>
#include <cstdint>
#include <mutex>
#include <string>
#include <type_traits>
#include <cuda_runtime.h>
#include "shg_common.cuh"
#include "shg_internal.h"
#include "shg_split.cuh"

namespace shg {

namespace {

template <int MAXM> struct Sh2Cfg;
// A raw seed's two half-table coverage masks (keys of set A, keys of set B), adjacent so that one
// shared-memory load brings both.
template <class M> struct alignas(2 * sizeof(M)) MaskPair {
    M a, b;
};

template <> struct Sh2Cfg<64> {
    using Mask = uint32_t;            // half-table coverage: (m + 1) / 2 <= 32 cells
    static constexpr int SMS = 256;   // raw seeds whose masks stay in shared memory
    static constexpr int CMS = 128;   // candidates held in shared memory
    static constexpr int ISO_WORDS = 1;
    static constexpr uint32_t ROWS = 2048;  // candidates whose cell rows are cached in global scratch
    static constexpr uint32_t RAW_ROWS = 2048;  // raw seeds whose cell rows are cached
    static constexpr int RING = 0;  // staging buffers of 32 spilled masks (none: leaves this small rarely spill)
};
template <> struct Sh2Cfg<128> {
    using Mask = uint64_t;
    static constexpr int SMS = 128;   // 12 KB of shared memory per warp: four 4-warp blocks per SM
    static constexpr int CMS = 128;
    static constexpr int ISO_WORDS = 2;
    static constexpr uint32_t ROWS = 4096;
    static constexpr uint32_t RAW_ROWS = 1024;
    static constexpr int RING = 3;  // staging buffers of 32 spilled masks: two chunks in flight while one is tested
};

// Shared-memory ring through which a warp streams spilled raw-seed masks (R buffers of 32 pairs).
template <class M, int R> struct MaskRing {
    MaskPair<M> e[R][32];
};
template <class M> struct MaskRing<M, 0> {};

// 16-byte global -> shared copies that bypass registers and L1 (cp.async), grouped per thread.
__device__ __forceinline__ void cp_async16(void *smem_dst, const void *gsrc) {
    const uint32_t d = (uint32_t)__cvta_generic_to_shared(smem_dst);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(d), "l"(gsrc) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N> __device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

template <int MAXM> struct alignas(16) Sh2Smem {  // 16-byte aligned per warp: the masks are read 16 bytes at a time
    using C = Sh2Cfg<MAXM>;
    uint64_t keys[MAXM];  // finder order (QuadSplit: even keys in order, odd keys from the back)
    uint64_t orig[MAXM];  // leaf order
    MaskPair<typename C::Mask> mask[C::SMS];
    uint32_t csa[C::CMS], csb[C::CMS];           // raw seeds (seedA, seedB) of each candidate
    uint64_t iso[C::CMS][C::ISO_WORDS];          // isolated-key masks
    uint8_t uf[MAXM * 32];                       // per-lane union-find parents / per-lane hash rows
    uint32_t surv[64];                           // survivor queue: j << 16 | i
    uint32_t nsurv;
    uint8_t c1[MAXM], c2[MAXM];                  // retrieval cuckoo insertion
    int16_t cell[MAXM];
    uint8_t xr[MAXM];
    MaskRing<typename C::Mask, C::RING> ring;
};

// Per-warp global scratch (L2-resident in practice): what does not fit shared memory, and the
// candidates' cell rows (one byte per key, MAXM / 8 words per candidate) for the pair tests.
template <int MAXM> struct Sh2Global {
    using Mask = typename Sh2Cfg<MAXM>::Mask;
    MaskPair<Mask> *mask;  // [smax]
    uint32_t *csa, *csb;  // [cmax]
    uint64_t *iso;        // [cmax][2]
    uint64_t *rows;       // [rcap][MAXM / 8]
    uint64_t *raw;        // [rawcap][MAXM / 8]: cells of every key (finder order) under raw seed s
    uint32_t rcap, rawcap;
    // row_rows / raw_rows: candidates and raw seeds whose cell rows are cached (beyond them the
    // kernel recomputes cells from the keys)
    __device__ void carve(uint8_t *base, uint32_t smax, uint32_t cmax, uint32_t row_rows = Sh2Cfg<MAXM>::ROWS,
                          uint32_t raw_rows = Sh2Cfg<MAXM>::RAW_ROWS) {
        mask = (MaskPair<Mask> *)base;
        iso = (uint64_t *)(base + ((2ull * smax * sizeof(Mask) + 255) & ~255ull));
        csa = (uint32_t *)(iso + 2 * (uint64_t)cmax);
        csb = csa + cmax;
        rows = (uint64_t *)(csb + cmax);  // 8-byte aligned: cmax is even
        rcap = cmax < row_rows ? cmax : row_rows;
        raw = rows + (uint64_t)rcap * (MAXM / 8);
        rawcap = smax < raw_rows ? smax : raw_rows;
    }
};

// Per-lane union-find over at most MAXM vertices: parents in shared memory (byte per vertex,
// [vertex][lane]), cycle flags of roots in registers.
template <int MAXM> struct LaneUF2 {
    uint8_t *par;
    int lane;
    uint64_t cyc0, cyc1;
    __device__ __forceinline__ void init(uint32_t n) {
        for (uint32_t v = 0; v < n; v++) par[v * 32 + lane] = (uint8_t)v;
        cyc0 = cyc1 = 0;
    }
    __device__ __forceinline__ uint32_t find(uint32_t x) {
        for (;;) {
            const uint32_t p = par[x * 32 + lane];
            if (p == x) return x;
            const uint32_t gp = par[p * 32 + lane];
            par[x * 32 + lane] = (uint8_t)gp;
            x = gp;
        }
    }
    __device__ __forceinline__ bool cyc(uint32_t r) const {
        if (MAXM <= 64) return (cyc0 >> r) & 1;
        return ((r < 64 ? cyc0 : cyc1) >> (r & 63)) & 1;
    }
    __device__ __forceinline__ void set_cyc(uint32_t r) {
        if (MAXM <= 64 || r < 64) cyc0 |= 1ull << (r & 63);
        else cyc1 |= 1ull << (r & 63);
    }
    // The roots of u and of v, both paths walked (and halved) in one loop so that their
    // shared-memory loads overlap.
    __device__ __forceinline__ void find2(uint32_t u, uint32_t v, uint32_t &ru, uint32_t &rv) {
        for (;;) {
            const uint32_t pu = par[u * 32 + lane], pv = par[v * 32 + lane];
            const bool du = pu == u, dv = pv == v;
            if (du && dv) break;
            if (!du) {
                const uint32_t g = par[pu * 32 + lane];
                par[u * 32 + lane] = (uint8_t)g;
                u = g;
            }
            if (!dv) {
                const uint32_t g = par[pv * 32 + lane];
                par[v * 32 + lane] = (uint8_t)g;
                v = g;
            }
        }
        ru = u;
        rv = v;
    }
    // Adds edge (u, v); false when a component would get a second cycle.
    __device__ __forceinline__ bool add(uint32_t u, uint32_t v) {
        uint32_t ru, rv;
        find2(u, v, ru, rv);
        if (ru == rv) {
            if (cyc(ru)) return false;
            set_cyc(ru);
            return true;
        }
        const bool cu = cyc(ru), cv = cyc(rv);
        if (cu && cv) return false;
        par[ru * 32 + lane] = (uint8_t)rv;
        if (cu) set_cyc(rv);
        return true;
    }
};

__device__ bool cuckoo_insert2(int16_t *cell, uint8_t *xr, int e, uint32_t c1, uint32_t c2, int limit) {
    xr[e] = (uint8_t)(c1 ^ c2);
    if (cell[c1] < 0) { cell[c1] = (int16_t)e; return true; }
    if (cell[c2] < 0) { cell[c2] = (int16_t)e; return true; }
    uint32_t cur = c1;
    const uint32_t orig_cell = cur;
    int entry = e;
    for (int step = 0; step < limit; step++) {
        const uint32_t alt = xr[entry] ^ cur;
        const int displaced = cell[alt];
        cell[alt] = (int16_t)entry;
        entry = displaced;
        if (entry < 0) return true;
        cur = alt;
        if (cur == orig_cell && entry == e) return false;
    }
    return false;
}

template <int MAXM> struct LeafCtx {
    using Mask = typename Sh2Cfg<MAXM>::Mask;
    Sh2Smem<MAXM> &sm;
    Sh2Global<MAXM> g;
    uint32_t m, half, sizeA, smax, cmax;
    Mask full;
    bool quad;
    __device__ __forceinline__ MaskPair<Mask> &mp(uint64_t s) { return s < Sh2Cfg<MAXM>::SMS ? sm.mask[s] : g.mask[s]; }
    __device__ __forceinline__ Mask maskA(uint64_t s) { return mp(s).a; }
    __device__ __forceinline__ Mask maskB(uint64_t s) { return mp(s).b; }
    __device__ __forceinline__ uint32_t &csa(uint32_t j) { return j < Sh2Cfg<MAXM>::CMS ? sm.csa[j] : g.csa[j]; }
    __device__ __forceinline__ uint32_t &csb(uint32_t j) { return j < Sh2Cfg<MAXM>::CMS ? sm.csb[j] : g.csb[j]; }
    __device__ __forceinline__ uint64_t &iso(uint32_t j, int w) {
        return j < Sh2Cfg<MAXM>::CMS ? sm.iso[j][w] : g.iso[2 * (uint64_t)j + w];
    }
    __device__ __forceinline__ uint64_t cseed(uint32_t j) {
        const uint32_t a = csa(j), b = csb(j);
        return quad ? pair_elegant(a, b) : a;
    }
    // candidate pair test on the edges (h_j + m/2, h_i): cells from the cached rows, or
    // recomputed for candidates beyond the row cache
    __device__ __forceinline__ bool pair_ok(LaneUF2<MAXM> &uf, uint32_t j, uint32_t i, unsigned long long &edges) {
        uf.init(m);
        const uint32_t off = m / 2;
        if (j < g.rcap) {  // i < j
            constexpr uint32_t W = MAXM / 8;
            const uint64_t *rj = g.rows + (uint64_t)j * W, *ri = g.rows + (uint64_t)i * W;
            for (uint32_t w = 0; w * 8 < m; w++) {
                const uint64_t a = rj[w], b = ri[w];
                const uint32_t kend = min(8u, m - w * 8);
                for (uint32_t t = 0; t < kend; t++) {
                    edges++;
                    if (!uf.add((uint32_t)((a >> (8 * t)) & 0xFF) + off, (uint32_t)((b >> (8 * t)) & 0xFF))) return false;
                }
            }
            return true;
        }
        const uint64_t ja = csa(j), jb = csb(j), ia = csa(i), ib = csb(i);
        for (uint32_t k = 0; k < m; k++) {
            const uint64_t key = sm.keys[k];
            const bool inA = k < sizeA;
            const uint32_t u = half_hash(key, inA ? ja : jb, half) + off;
            const uint32_t v = half_hash(key, inA ? ia : ib, half);
            edges++;
            if (!uf.add(u, v)) return false;
        }
        return true;
    }
};

// Where a leaf's keys and its output seed are: the engine's planned tree nodes...
struct NodeLeaves {
    const Node *nodes;
    const uint32_t *ids;
    uint64_t *codes;
    static constexpr uint32_t kRowCache = 0;  // 0: the configuration's cell-row caches (Sh2Cfg)
    __device__ __forceinline__ bool get(uint32_t li, uint32_t &start, uint32_t &m, uint64_t *&code) const {
        const uint32_t id = ids[li];
        const Node nd = nodes[id];
        start = nd.start;
        m = nd.m;
        code = codes + id;
        return true;
    }
};
// ...or a caller's leaf offsets (leaf j = keys [offs[j], offs[j+1])), validated on the device.
template <int MAXM> struct OffsetLeaves {
    const uint64_t *offs;
    uint64_t *seeds;
    // Cell-row caches of the no-allocation entry point, which uses this source: rows of the first
    // 128 candidates and 192 raw seeds of a leaf, so that its fixed scratch array feeds about twice
    // as many warps as with the engine's caches.
    static constexpr uint32_t kRowCache = 1, kCandRows = 128, kRawRows = 192;
    __device__ __forceinline__ bool get(uint32_t li, uint32_t &start, uint32_t &m, uint64_t *&code) const {
        const uint64_t b = offs[li], e = offs[li + 1];
        if (e < b + 2 || e - b > (uint64_t)MAXM || e > 0xFFFFFFFFull) return false;
        start = (uint32_t)b;
        m = (uint32_t)(e - b);
        code = seeds + li;
        return true;
    }
};

// Work counts of one warp's leaves (summed over the warp's lanes at the end of its kernel).
struct LeafWork {
    unsigned long long evals = 0, pairs = 0, filtered = 0, edges = 0, scan = 0;
};

// One bipartite leaf, searched by the calling warp: leaf li of `src` (its keys from `keys`, its seed
// to the source's code slot, its retrieval bits to rib_bits). The warp's shared-memory state `sm`,
// global scratch `g` and union-find `uf` are reused from leaf to leaf. Errors set bits of *err.
// L2: read the leaf's keys past L1 (the work-queue kernel, where another SM's partition may have
// rewritten them after this SM cached the lines).
// SIDE_WORDS: hash whole 8-key words that lie on one side of the leaf without per-key selects
// (measured faster inside the work-queue kernel, slower in the level schedule's leaf kernel).
template <int MAXM, class Src, bool L2 = false, bool SIDE_WORDS = false>
__device__ __forceinline__ void sh2_leaf(const Src &src, uint32_t li, const uint64_t *__restrict__ keys,
                                         uint8_t *__restrict__ rib_bits, Sh2Smem<MAXM> &sm, Sh2Global<MAXM> &g,
                                         LaneUF2<MAXM> &uf, const int lane, const uint32_t smax, const uint32_t cmax,
                                         const uint32_t quad_min, uint32_t *__restrict__ err, LeafWork &lw) {
    const unsigned below = (1u << lane) - 1;
    unsigned long long &w_evals = lw.evals, &w_pairs = lw.pairs, &w_filtered = lw.filtered, &w_edges = lw.edges,
                       &w_scan = lw.scan;
    uint32_t start = 0, m_leaf = 0;
    uint64_t *code_out = nullptr;
    if (!src.get(li, start, m_leaf, code_out)) {
        if (lane == 0) atomicOr(err, kErrArg);
        return;
    }
    LeafCtx<MAXM> cx{sm, g};
    cx.m = m_leaf;
    cx.half = (cx.m + 1) / 2;
    cx.full = cx.half >= 8 * sizeof(typename LeafCtx<MAXM>::Mask) ? ~(typename LeafCtx<MAXM>::Mask)0
                                                                 : (((typename LeafCtx<MAXM>::Mask)1 << cx.half) - 1);
    cx.quad = cx.m >= quad_min;
    cx.smax = smax;
    cx.cmax = cmax;
    const uint32_t m = cx.m, half = cx.half;

    // keys in finder order (QuadSplitCandidateFinder ctor, ShockHash2-internal.h:397-407)
    {
        uint32_t evens = 0, odds = 0;
        for (uint32_t k0 = 0; k0 < m; k0 += 32) {
            const uint32_t k = k0 + lane;
            const uint64_t key = k < m ? (L2 ? __ldcg(&keys[start + k]) : keys[start + k]) : 0;
            const bool even = (key & 1) == 0;
            const unsigned be = __ballot_sync(0xffffffffu, k < m && even);
            const unsigned bo = __ballot_sync(0xffffffffu, k < m && !even);
            if (k < m) {
                sm.orig[k] = key;
                uint32_t pos = k;
                if (cx.quad) pos = even ? evens + __popc(be & below) : m - 1 - (odds + __popc(bo & below));
                sm.keys[pos] = key;
            }
            evens += __popc(be);
            odds += __popc(bo);
        }
        cx.sizeA = cx.quad ? evens : m;
    }
    if (lane == 0) sm.nsurv = 0;
    __syncwarp();

    uint32_t J = 0;             // candidates stored so far
    uint64_t S = 0;             // raw seeds hashed so far
    uint64_t answer = ~0ull;
    bool overflow = false;
    // survivor queue: run pseudoforest tests 32 at a time; returns true when a pair passed
    auto drain = [&](uint32_t upto) -> bool {
        const uint32_t cnt = min(upto, sm.nsurv);
        bool ok = false;
        uint32_t j = 0, i = 0;
        if ((uint32_t)lane < cnt) {
            const uint32_t e = sm.surv[lane];
            j = e >> 16;
            i = e & 0xFFFF;
            ok = cx.pair_ok(uf, j, i, w_edges);
        }
        unsigned pass = __ballot_sync(0xffffffffu, ok);
        while (pass) {
            const int src = __ffs(pass) - 1;
            const uint32_t jj = __shfl_sync(0xffffffffu, j, src), ii = __shfl_sync(0xffffffffu, i, src);
            const uint64_t sj = cx.cseed(jj), si = cx.cseed(ii);
            if (float_accurate_triangular(sj, si)) {
                answer = pair_triangular(sj, si);
                return true;
            }
            pass &= pass - 1;
        }
        // drop the tested entries, keep the rest in order
        const uint32_t rest = sm.nsurv - cnt;
        __syncwarp();
        uint32_t v0 = (uint32_t)lane < rest ? sm.surv[cnt + lane] : 0;
        uint32_t v1 = (uint32_t)lane + 32 < rest ? sm.surv[cnt + lane + 32] : 0;
        __syncwarp();
        if ((uint32_t)lane < rest) sm.surv[lane] = v0;
        if ((uint32_t)lane + 32 < rest) sm.surv[lane + 32] = v1;
        if (lane == 0) sm.nsurv = rest;
        __syncwarp();
        return false;
    };

    uint64_t S_proc = 0;  // raw seeds whose candidates are listed
    while (answer == ~0ull && !overflow) {
        // 1. hash raw seeds S..S+31 once the listed ones have caught up
        if (S_proc == S) {
            if (S + 32 > smax) {
                overflow = true;
                break;
            }
            const uint64_t s = S + lane;
            using Mask = typename LeafCtx<MAXM>::Mask;
            Mask tA = 0, tB = 0;
            uint64_t *rrow = s < g.rawcap ? g.raw + s * (MAXM / 8) : nullptr;
            const uint32_t sizeA = cx.sizeA;
            // eight independent hash chains per row word (keys 8w..8w+7; MAXM is a multiple of 8, so
            // sm.keys[8w + 7] is in bounds, and the cells of keys past m are dropped)
            for (uint32_t k0 = 0; k0 < m; k0 += 8) {
                uint64_t word = 0;
                if (SIDE_WORDS && k0 + 8 <= m && (k0 + 8 <= sizeA || k0 >= sizeA)) {
                    // the whole word inside the leaf and on one side (the same in every lane)
                    Mask w8 = 0;
#pragma unroll
                    for (uint32_t t = 0; t < 8; t++) {
                        const uint32_t h = half_hash(sm.keys[k0 + t], s, half);
                        w8 |= (Mask)1 << h;
                        word |= (uint64_t)h << (8 * t);
                    }
                    if (k0 + 8 <= sizeA) tA |= w8;
                    else tB |= w8;
                } else {
#pragma unroll
                    for (uint32_t t = 0; t < 8; t++) {
                        const uint32_t k = k0 + t;
                        const uint32_t h = half_hash(sm.keys[k], s, half);
                        const Mask bit = k < m ? (Mask)1 << h : (Mask)0;
                        tA |= k < sizeA ? bit : (Mask)0;
                        tB |= k < sizeA ? (Mask)0 : bit;
                        word |= k < m ? (uint64_t)h << (8 * t) : 0ull;
                    }
                }
                if (rrow) rrow[k0 >> 3] = word;
            }
            cx.mp(s) = MaskPair<typename LeafCtx<MAXM>::Mask>{tA, tB};
            w_evals += m;
            S += 32;
            __syncwarp();
        }
        // 2. candidates whose larger raw seed is s (lane L: s = S_proc + L), in the reference's order
        const uint64_t s = S_proc + lane;
        const bool live = s < S;
        uint32_t mine = 0, mineA = 0, mineB = 0;
        // each lane's partners in scan order, in the union-find area (idle until this round's pair
        // tests; [entry][lane], one column per lane): A side in entries 0..kPartners-1, B side after
        constexpr uint32_t kPartners = MAXM / 4;
        static_assert(2 * kPartners * 32 * sizeof(uint16_t) <= sizeof(sm.uf), "partner lists fit the union-find area");
        uint16_t *const plist = reinterpret_cast<uint16_t *>(sm.uf);
        if (live) w_scan += cx.quad ? s + 1 : 1;  // mask pairs this raw seed is tested against
        // one pass over the earlier raw seeds p <= s: A-side pairs (p, s) for p < s and B-side pairs
        // (s, p) for p <= s (candidatesA/B.filter, ShockHash2-internal.h:446-465), in three parts:
        // the masks in shared memory (each lane alone), the spilled masks of earlier rounds (the
        // warp streams them through a shared-memory ring), and the rest up to s (each lane alone)
        using RMask = typename LeafCtx<MAXM>::Mask;
        const MaskPair<RMask> ts = live && cx.quad ? cx.mp(s) : MaskPair<RMask>{0, 0};
        const RMask tA = ts.a, tB = ts.b;
        // a side of raw seed p pairs with s when it covers every cell s's other side leaves empty:
        // (w.a | tB) == full  <=>  (nB & ~w.a) == 0 (masks hold no bits past the half table)
        const RMask nA = ~tA & cx.full, nB = ~tB & cx.full;
        const uint32_t in_sm = (uint32_t)min(s + 1, (uint64_t)Sh2Cfg<MAXM>::SMS);
        auto visit = [&](uint64_t p, MaskPair<RMask> w) {
            if (p < s && (w.a | tB) == cx.full && float_accurate_elegant_seeds(p, s)) {
                if (mineA < kPartners) plist[mineA * 32 + lane] = (uint16_t)p;
                mineA++;
            }
            if ((w.b | tA) == cx.full && float_accurate_elegant_seeds(s, p)) {
                if (mineB < kPartners) plist[(kPartners + mineB) * 32 + lane] = (uint16_t)p;
                mineB++;
            }
        };
        if (live && cx.quad) {
            uint32_t p = 0;
            if constexpr (sizeof(typename LeafCtx<MAXM>::Mask) == 4) {
                // two raw seeds per 16-byte load; one combined test rejects the common case
                // that neither side of either seed covers the half table. A hit only
                // appends its 16-byte slot (p / 2 < 128) to a register queue of up to 8;
                // the hits are visited after the loop, in the same ascending order, so the
                // loop itself stays free of the recording path. Past 8 hits the scan
                // resumes, visiting directly, from the 9th hit's slot on.
                const uint4 *m2 = reinterpret_cast<const uint4 *>(sm.mask);
                const uint32_t full = cx.full;
                uint64_t hq = 0;
                uint32_t nh = 0, resume = 0;
                auto miss = [&](const uint4 &w) {  // 0 when a side of either seed covers the half table
                    return min(min((w.x | tB) ^ full, (w.y | tA) ^ full), min((w.z | tB) ^ full, (w.w | tA) ^ full));
                };
                auto record = [&](uint32_t slot) {
                    if (nh < 8) hq |= (uint64_t)slot << (8 * nh);
                    else if (nh == 8) resume = 2 * slot;
                    nh++;
                };
                // four 16-byte loads (eight raw seeds) in flight per step: the loads are
                // broadcasts, so latency, not bandwidth, sets this loop's speed
                for (; p + 8 <= in_sm; p += 8) {
                    const uint4 w0 = m2[(p >> 1)], w1 = m2[(p >> 1) + 1], w2 = m2[(p >> 1) + 2], w3 = m2[(p >> 1) + 3];
                    const uint32_t z0 = miss(w0), z1 = miss(w1), z2 = miss(w2), z3 = miss(w3);
                    if (min(min(z0, z1), min(z2, z3)) == 0) {
                        if (z0 == 0) record(p >> 1);
                        if (z1 == 0) record((p >> 1) + 1);
                        if (z2 == 0) record((p >> 1) + 2);
                        if (z3 == 0) record((p >> 1) + 3);
                    }
                }
                for (; p + 2 <= in_sm; p += 2)
                    if (miss(m2[p >> 1]) == 0) record(p >> 1);
                for (uint32_t h = 0; h < min(nh, 8u); h++) {
                    const uint32_t q = (uint32_t)((hq >> (8 * h)) & 0xFF) * 2;
                    const uint4 w = m2[q >> 1];
                    visit(q, MaskPair<uint32_t>{w.x, w.y});
                    visit(q + 1, MaskPair<uint32_t>{w.z, w.w});
                }
                if (nh > 8) {
                    for (uint32_t q = resume; q + 2 <= in_sm; q += 2) {
                        const uint4 w = m2[q >> 1];
                        const uint32_t z = min(min((w.x | tB) ^ full, (w.y | tA) ^ full),
                                               min((w.z | tB) ^ full, (w.w | tA) ^ full));
                        if (z == 0) {
                            visit(q, MaskPair<uint32_t>{w.x, w.y});
                            visit(q + 1, MaskPair<uint32_t>{w.z, w.w});
                        }
                    }
                }
            }
            if constexpr (sizeof(typename LeafCtx<MAXM>::Mask) == 8) {
                // one raw seed per 16-byte load, two per round; a tight scan finds the next
                // pair in which some side covers the half table, and only then records it
                for (;;) {
                    MaskPair<uint64_t> w{0, 0}, v{0, 0};
                    for (; p + 2 <= in_sm; p += 2) {
                        w = sm.mask[p];
                        v = sm.mask[p + 1];
                        if (((nB & ~w.a) == 0) | ((nA & ~w.b) == 0) | ((nB & ~v.a) == 0) | ((nA & ~v.b) == 0))
                            break;
                    }
                    if (p + 2 > in_sm) break;
                    visit(p, w);
                    visit(p + 1, v);
                    p += 2;
                }
            }
            for (; p < in_sm; p++) visit(p, sm.mask[p]);
        }
        uint64_t spill0 = in_sm;  // where each lane's own pass over the spilled masks starts
        if constexpr (Sh2Cfg<MAXM>::RING > 0) {
            constexpr int R = Sh2Cfg<MAXM>::RING;
            constexpr uint64_t lo = Sh2Cfg<MAXM>::SMS;
            if (cx.quad && S_proc > lo) {
                // raw seeds lo..S_proc-1 lie below every lane's s and their masks are in global
                // scratch: the warp copies them 32 at a time (one 16-byte pair per lane, coalesced)
                // into the ring, R - 1 chunks ahead of the one being tested, and every lane tests
                // its own seed against each pair with shared-memory broadcasts, so the loop waits on
                // no global load; hits are visited in ascending order as before
                const uint64_t hi = S_proc;
                const uint32_t nch = (uint32_t)((hi - lo + 31) / 32);
                auto issue = [&](uint32_t c) {
                    const uint64_t p = lo + 32ull * c + lane;
                    if (c < nch && p < hi) cp_async16(&sm.ring.e[c % R][lane], &g.mask[p]);
                    cp_async_commit();  // one group per chunk in every lane, empty ones included
                };
#pragma unroll
                for (int c = 0; c < R - 1; c++) issue(c);
                for (uint32_t c = 0; c < nch; c++) {
                    cp_async_wait<R - 2>();  // this lane's copies of chunk c have landed
                    __syncwarp();            // and every lane's; all are done testing chunk c - 1
                    issue(c + R - 1);        // into the buffer chunk c - 1 used
                    if (live) {
                        const MaskPair<uint64_t> *buf = sm.ring.e[c % R];
                        const uint64_t c0 = lo + 32ull * c;
                        const uint32_t cnt = (uint32_t)min((uint64_t)32, hi - c0);
                        uint32_t t = 0;
                        for (; t + 8 <= cnt; t += 8) {
                            MaskPair<uint64_t> w8[8];
#pragma unroll
                            for (int u = 0; u < 8; u++) w8[u] = buf[t + u];
                            bool any = false;
#pragma unroll
                            for (int u = 0; u < 8; u++) any |= ((nB & ~w8[u].a) == 0) | ((nA & ~w8[u].b) == 0);
                            if (any) {
#pragma unroll 1
                                for (uint32_t u = 0; u < 8; u++) visit(c0 + t + u, buf[t + u]);
                            }
                        }
                        for (; t < cnt; t++) visit(c0 + t, buf[t]);
                    }
                }
                cp_async_wait<0>();
                __syncwarp();
                spill0 = hi;
            }
        }
        if (live) {
            if (cx.quad) {
                uint64_t q = spill0;
                if constexpr (sizeof(typename LeafCtx<MAXM>::Mask) == 4) {
                    // spilled masks (raw seeds from 256 on; q is even, so the 16-byte loads are
                    // aligned): eight raw seeds' masks requested before any is tested
                    const uint4 *g2 = reinterpret_cast<const uint4 *>(g.mask);
                    const uint32_t full = cx.full;
                    for (; q + 8 <= s + 1; q += 8) {
                        uint4 w[4];
#pragma unroll
                        for (int t = 0; t < 4; t++) w[t] = g2[(q >> 1) + t];
                        uint32_t z = 0xFFFFFFFFu;
#pragma unroll
                        for (int t = 0; t < 4; t++)
                            z = min(z, min(min((w[t].x | tB) ^ full, (w[t].y | tA) ^ full),
                                           min((w[t].z | tB) ^ full, (w[t].w | tA) ^ full)));
                        if (z == 0) {  // rare: visit the eight seeds in order, reloading their masks
#pragma unroll 1
                            for (uint32_t t = 0; t < 4; t++) {
                                const uint4 v = g2[(q >> 1) + t];
                                visit(q + 2 * t, MaskPair<uint32_t>{v.x, v.y});
                                visit(q + 2 * t + 1, MaskPair<uint32_t>{v.z, v.w});
                            }
                        }
                    }
                }
                if constexpr (sizeof(typename LeafCtx<MAXM>::Mask) == 8) {  // spilled masks: same paired test
                    // eight raw seeds' masks requested before any is tested, so that eight L2 or DRAM
                    // loads are in flight per warp instead of two (these loads dominate large leaves)
                    for (; q + 8 <= s + 1; q += 8) {
                        MaskPair<uint64_t> w8[8];
#pragma unroll
                        for (int t = 0; t < 8; t++) w8[t] = g.mask[q + t];
                        bool any = false;
#pragma unroll
                        for (int t = 0; t < 8; t++) any |= ((nB & ~w8[t].a) == 0) | ((nA & ~w8[t].b) == 0);
                        if (any) {
#pragma unroll 1
                            for (uint32_t t = 0; t < 8; t++) visit(q + t, g.mask[q + t]);
                        }
                    }
                    for (; q + 2 <= s + 1; q += 2) {
                        const MaskPair<uint64_t> w = g.mask[q], v = g.mask[q + 1];
                        const bool any = ((nB & ~w.a) == 0) | ((nA & ~w.b) == 0) | ((nB & ~v.a) == 0) | ((nA & ~v.b) == 0);
                        if (any) {
                            visit(q, w);
                            visit(q + 1, v);
                        }
                    }
                }
#pragma unroll 1
                for (; q <= s; q++) visit(q, g.mask[q]);
                mine = mineA + mineB;
            } else {
                mine = cx.maskA(s) == cx.full;
            }
        }
        uint32_t incl = mine;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += y;
        }
        // take the longest prefix of raw seeds whose candidates fit the candidate capacity
        const uint32_t cap = min(cmax, 0xFFFFu);
        const unsigned fits = __ballot_sync(0xffffffffu, live && J + incl <= cap);
        const int take = fits == 0xffffffffu ? 32 : __ffs(~fits) - 1;  // fits is a prefix of lanes
        if (take == 0) {
            overflow = true;
            break;
        }
        const uint32_t T = __shfl_sync(0xffffffffu, incl, take - 1);
        if (lane < take) {
            uint32_t pos = J + incl - mine;
            if (cx.quad && mineA <= kPartners && mineB <= kPartners) {
                for (uint32_t t = 0; t < mineA; t++, pos++) {  // A side first: (a, s), a ascending
                    cx.csa(pos) = plist[t * 32 + lane];
                    cx.csb(pos) = (uint32_t)s;
                }
                for (uint32_t t = 0; t < mineB; t++, pos++) {  // then B side: (s, b), b ascending
                    cx.csa(pos) = (uint32_t)s;
                    cx.csb(pos) = plist[(kPartners + t) * 32 + lane];
                }
            } else if (cx.quad) {  // more partners on a side than the lists hold (vanishingly rare): scan again
                const auto tA = cx.maskA(s), tB = cx.maskB(s);
                for (uint64_t a = 0; a < s && mine; a++)
                    if ((cx.maskA(a) | tB) == cx.full && float_accurate_elegant_seeds(a, s)) {
                        cx.csa(pos) = (uint32_t)a;
                        cx.csb(pos) = (uint32_t)s;
                        pos++;
                    }
                for (uint64_t b = 0; b <= s && mine; b++)
                    if ((cx.maskB(b) | tA) == cx.full && float_accurate_elegant_seeds(s, b)) {
                        cx.csa(pos) = (uint32_t)s;
                        cx.csb(pos) = (uint32_t)b;
                        pos++;
                    }
            } else if (mine) {
                cx.csa(pos) = (uint32_t)s;
                cx.csb(pos) = (uint32_t)s;
            }
        }
        S_proc += take;
        __syncwarp();
        if (T == 0) continue;
        // 3. isolated-key masks of the new candidates (calculateIsolatedVertices), one per lane
        for (uint32_t c0 = J; c0 < J + T; c0 += 32) {
            const uint32_t c = c0 + lane;
            if (c < J + T && cx.csa(c) < g.rawcap && cx.csb(c) < g.rawcap) {
                // cells from the two raw seeds' rows: set-A keys under seedA, set-B keys under seedB
                const uint64_t *ra = g.raw + (uint64_t)cx.csa(c) * (MAXM / 8);
                const uint64_t *rb = g.raw + (uint64_t)cx.csb(c) * (MAXM / 8);
                uint64_t *row = c < g.rcap ? g.rows + (uint64_t)c * (MAXM / 8) : nullptr;
                const uint32_t sizeA = cx.sizeA;
                auto word_of = [&](uint32_t w) {  // cells of keys 8w..8w+7, one byte each
                    const uint32_t k0 = 8 * w;
                    uint64_t v;
                    if (k0 + 8 <= sizeA) v = ra[w];
                    else if (k0 >= sizeA) v = rb[w];
                    else {
                        const uint64_t keep = (1ull << (8 * (sizeA - k0))) - 1;
                        v = (ra[w] & keep) | (rb[w] & ~keep);
                    }
                    if (k0 + 8 > m) v &= (1ull << (8 * (m - k0))) - 1;
                    return v;
                };
                // the candidate's cell words go to its own column of the union-find area (idle until
                // the pair tests) for the second pass; the next word's loads are issued before this
                // word's stores, which would otherwise hold them back
                uint64_t *const uw = reinterpret_cast<uint64_t *>(sm.uf);  // [word][lane]
                static_assert(MAXM / 8 * 32 * sizeof(uint64_t) <= sizeof(sm.uf), "cell words fit the union-find area");
                // cells are below (m + 1) / 2: 32-bit masks for leaves of up to 64 keys
                using CMask = std::conditional_t<(MAXM <= 64), uint32_t, uint64_t>;
                CMask seen1 = 0, seen2 = 0;
                uint64_t v_next = word_of(0);
#pragma unroll 1
                for (uint32_t w = 0; 8 * w < m; w++) {
                    const uint64_t v = v_next;
                    if (8 * (w + 1) < m) v_next = word_of(w + 1);
                    uw[w * 32 + lane] = v;
                    if (row) row[w] = v;
                    const uint32_t kn = min(8u, m - 8 * w);
#pragma unroll
                    for (uint32_t t = 0; t < 8; t++) {
                        if (t < kn) {
                            const CMask bit = (CMask)1 << ((v >> (8 * t)) & 0xFF);
                            seen2 |= seen1 & bit;
                            seen1 |= bit;
                        }
                    }
                }
                const CMask single = seen1 & ~seen2;
                uint64_t iso0 = 0, iso1 = 0;
#pragma unroll 1
                for (uint32_t w = 0; 8 * w < m; w++) {
                    const uint64_t v = uw[w * 32 + lane];
                    const uint32_t kn = min(8u, m - 8 * w);
                    uint64_t b8 = 0;
#pragma unroll
                    for (uint32_t t = 0; t < 8; t++)
                        if (t < kn) b8 |= ((single >> ((v >> (8 * t)) & 0xFF)) & 1) << t;
                    const uint32_t k0 = 8 * w;
                    if (k0 < 64) iso0 |= b8 << k0; else iso1 |= b8 << (k0 - 64);
                }
                cx.iso(c, 0) = iso0;
                if (Sh2Cfg<MAXM>::ISO_WORDS > 1) cx.iso(c, 1) = iso1;
                w_evals += m;  // the reference hashes the candidate's keys here (makeCache)
            } else if (c < J + T) {
                const uint64_t sa = cx.csa(c), sb = cx.csb(c);
                uint64_t seen1 = 0, seen2 = 0, word = 0;
                uint64_t *row = c < g.rcap ? g.rows + (uint64_t)c * (MAXM / 8) : nullptr;
                for (uint32_t k = 0; k < m; k++) {
                    const uint32_t h = half_hash(sm.keys[k], k < cx.sizeA ? sa : sb, half);
                    sm.uf[k * 32 + lane] = (uint8_t)h;
                    word |= (uint64_t)h << (8 * (k & 7));
                    if ((k & 7) == 7 || k + 1 == m) {
                        if (row) row[k >> 3] = word;
                        word = 0;
                    }
                    const uint64_t bit = 1ull << h;
                    seen2 |= seen1 & bit;
                    seen1 |= bit;
                }
                const uint64_t single = seen1 & ~seen2;
                uint64_t iso0 = 0, iso1 = 0;
                for (uint32_t k = 0; k < m; k++) {
                    const uint32_t h = sm.uf[k * 32 + lane];
                    const uint64_t b = (single >> h) & 1;
                    if (k < 64) iso0 |= b << k; else iso1 |= b << (k - 64);
                }
                cx.iso(c, 0) = iso0;
                if (Sh2Cfg<MAXM>::ISO_WORDS > 1) cx.iso(c, 1) = iso1;
                w_evals += m;
            }
        }
        __syncwarp();
        // 4. all pairs (j, i), J <= j < J+T, i < j, in lexicographic order
        // pair q = j(j-1)/2 + i; lanes take 32 consecutive q, decoded by stepping from the
        // batch's first pair (jb, ib), which advances by 32 per batch
        const uint64_t q0 = (uint64_t)J * (J - 1) / 2, q1 = (uint64_t)(J + T) * (J + T - 1) / 2;
        bool done = false;
        uint32_t jb = J > 0 ? J : 1, ib = 0;
        for (uint64_t qb = q0; qb < q1 && !done; qb += 32) {
            const uint64_t q = qb + lane;
            bool filt = false;
            uint32_t j = jb, i = ib + lane;
            while (i >= j) {
                i -= j;
                j++;
            }
            for (uint32_t adv = ib + 32; ; ) {  // next batch's first pair
                if (adv < jb) {
                    ib = adv;
                    break;
                }
                adv -= jb;
                jb++;
            }
            if (q < q1) {
                uint64_t x = cx.iso(j, 0) & cx.iso(i, 0);
                if (Sh2Cfg<MAXM>::ISO_WORDS > 1) x |= cx.iso(j, 1) & cx.iso(i, 1);
                filt = x == 0;
                w_pairs++;
                w_filtered += filt;
            }
            const unsigned bal = __ballot_sync(0xffffffffu, filt);
            const uint32_t base = sm.nsurv;
            __syncwarp();
            if (filt) sm.surv[base + __popc(bal & below)] = j << 16 | i;
            __syncwarp();
            if (lane == 0) sm.nsurv = base + __popc(bal);
            __syncwarp();
            if (sm.nsurv >= 32) done = drain(32);
        }
        // Fewer than 32 survivors wait for the next round's pairs, so that pseudoforest tests
        // run with full warps; the queue stays in (j, i) order, so the first passing entry is
        // still the reference's answer.
        while (!done && sm.nsurv >= 32) done = drain(32);
        J += T;
    }
    if (answer == ~0ull) {  // the survivors still queued come before anything not yet listed
        while (answer == ~0ull && sm.nsurv > 0) drain(32);
        if (answer != ~0ull) overflow = false;
    }
    if (overflow || answer == ~0ull) {
        if (lane == 0) atomicOr(err, kErrScratch);
        return;
    }

    // Retrieval bits (constructRetrieval, ShockHash2-internal.h:548-572): ordered cuckoo
    // insertion of the leaf keys in leaf order; bit 1 when a key rests in its seed2 cell.
    uint64_t s1, s2;
    unpair_triangular(answer, s1, s2);
    for (uint32_t k = lane; k < m; k += 32) {
        sm.c1[k] = (uint8_t)(sh2_cand_hash(sm.orig[k], s1, m, cx.quad) + m / 2);
        sm.c2[k] = (uint8_t)sh2_cand_hash(sm.orig[k], s2, m, cx.quad);
        sm.cell[k] = -1;
    }
    __syncwarp();
    if (lane == 0) {
        bool okc = true;
        for (uint32_t k = 0; k < m && okc; k++) okc = cuckoo_insert2(sm.cell, sm.xr, (int)k, sm.c1[k], sm.c2[k], 8 * (int)m + 16);
        if (!okc) atomicOr(err, kErrInternal);
        *code_out = answer;
    }
    __syncwarp();
    for (uint32_t k = lane; k < m; k += 32) rib_bits[start + k] = sm.cell[sm.c2[k]] == (int16_t)k ? 1 : 0;
    __syncwarp();
}

// MINB: blocks per SM the register allocation is bounded for (a tuning parameter; any value gives
// the same results).
template <int MAXM, class Src, int MINB = (MAXM <= 64 ? 6 : 1)>
__global__ void __launch_bounds__(128, MINB) k_leaves_sh2_v2(Src src, uint32_t count, const uint64_t *__restrict__ keys,
                                                       uint8_t *__restrict__ rib_bits,
                                                       uint8_t *__restrict__ scratch, uint64_t scratch_per_warp,
                                                       uint32_t smax, uint32_t cmax, uint32_t *__restrict__ err,
                                                       unsigned long long *__restrict__ work,
                                                       unsigned int *__restrict__ next_leaf, uint32_t quad_min) {
    extern __shared__ __align__(16) uint8_t smem_raw[];
    constexpr int WPB = 4;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    Sh2Smem<MAXM> &sm = reinterpret_cast<Sh2Smem<MAXM> *>(smem_raw)[warp];
    const uint64_t gw = (uint64_t)blockIdx.x * WPB + warp;
    uint8_t *gbase = scratch + gw * scratch_per_warp;
    Sh2Global<MAXM> g;
    if constexpr (Src::kRowCache) g.carve(gbase, smax, cmax, Src::kCandRows, Src::kRawRows);
    else g.carve(gbase, smax, cmax);
    LaneUF2<MAXM> uf{sm.uf, lane, 0, 0};
    LeafWork lw;
    for (;;) {
        uint32_t li = 0;
        if (lane == 0) li = atomicAdd(next_leaf, 1u);
        li = __shfl_sync(0xffffffffu, li, 0);
        if (li >= count) break;
        sh2_leaf<MAXM, Src>(src, li, keys, rib_bits, sm, g, uf, lane, smax, cmax, quad_min, err, lw);
    }
    unsigned long long w_evals = lw.evals, w_pairs = lw.pairs, w_filtered = lw.filtered, w_edges = lw.edges,
                       w_scan = lw.scan;
    for (int o = 16; o; o >>= 1) {
        w_evals += __shfl_xor_sync(0xffffffffu, w_evals, o);
        w_pairs += __shfl_xor_sync(0xffffffffu, w_pairs, o);
        w_filtered += __shfl_xor_sync(0xffffffffu, w_filtered, o);
        w_edges += __shfl_xor_sync(0xffffffffu, w_edges, o);
        w_scan += __shfl_xor_sync(0xffffffffu, w_scan, o);
    }
    if (lane == 0) {
        atomicAdd(&work[1], w_evals);
        atomicAdd(&work[2], w_pairs);
        atomicAdd(&work[3], w_filtered);
        atomicAdd(&work[4], w_edges);
        atomicAdd(&work[5], w_scan);
    }
}

template <int MAXM, int MINB>
void launch_v2(const Node *nodes, const uint32_t *ids, uint32_t count, const uint64_t *keys, uint64_t *codes,
               uint8_t *rib_bits, uint8_t *scratch, uint64_t scratch_per_warp, uint32_t smax, uint32_t cmax,
               uint32_t *err, unsigned long long *work, unsigned int *ctr, int grid, cudaStream_t s, uint32_t quad_min) {
    const size_t smem = sizeof(Sh2Smem<MAXM>) * 4;
    // The shared-memory limit is an attribute of the kernel on the current device: set it on every
    // launch (a cheap host call), so engines on several devices and threads each get it.
    cudaFuncSetAttribute(k_leaves_sh2_v2<MAXM, NodeLeaves, MINB>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    k_leaves_sh2_v2<MAXM, NodeLeaves, MINB><<<grid, 128, smem, s>>>(NodeLeaves{nodes, ids, codes}, count, keys, rib_bits,
                                                                    scratch, scratch_per_warp, smax, cmax, err, work, ctr,
                                                                    quad_min);
}

// ------------------------------------------------------------------ work-queue schedule
// All split nodes and leaves of a ShockHash2 build (leaves of up to 64 keys) in ONE persistent
// launch. Blocks take items from one sequence: a split node (searched and partitioned by the whole
// block, split_node) or the leaves of one bucket (the block's warps take them one at a time from a
// shared counter, sh2_leaf). The sequence is staggered by bucket: time slot t holds the level-lv
// split nodes of bucket t - lv * lag for every level, then the leaves of bucket t - nlevels * lag.
// So at any moment the running blocks mix the deep split levels of some buckets, the upper levels
// of later ones and the leaves of earlier ones: the integer-bound split search and the latency-bound
// leaf search share every SM, instead of the leaves starting after the last split level.
// A node may start when its bucket's split nodes of the levels above it are done, a leaf group when
// all of its bucket's split nodes are: a per-bucket counter of finished split nodes, compared with
// the plan's counts (offs: per list column and bucket). Everything an item waits for sits earlier in
// the sequence, so it was taken by a block that is running, and the waits end; each is still
// bounded, and one that runs out sets kErrInternal (the build then fails). Keys rewritten by another
// SM's partition are read past L1.
constexpr int kQueueThreads = 256;
constexpr int kQueueWarps = kQueueThreads / 32;
constexpr uint32_t kQueueWaitLimit = 1u << 18;  // polls of at least 64 ns: a fifth of a second or more, far beyond any node

__device__ __forceinline__ uint32_t ld_acquire_gpu(const uint32_t *p) {
    uint32_t v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

// Waits until *done >= need (one thread); false when the wait ran out, or at once when another wait
// of the launch has run out already (kErrInternal in *err), so that a fault ends the launch quickly.
__device__ bool wait_done(const uint32_t *done, uint32_t need, const uint32_t *err) {
    for (uint32_t it = 0; it < kQueueWaitLimit; it++) {
        if (ld_acquire_gpu(done) >= need) return true;
        if ((it & 255) == 255 && (ld_acquire_gpu(err) & kErrInternal)) return false;
        __nanosleep(64);
    }
    return false;
}

// Split nodes of bucket b on the levels above `level` (level = nlevels: all of them).
__device__ __forceinline__ uint32_t splits_above(const uint32_t *__restrict__ offs, uint64_t stride, uint32_t b,
                                                 uint32_t level) {
    uint32_t t = 0;
    for (uint32_t lv = 0; lv < level; lv++) {
        const uint32_t *col = offs + (uint64_t)(kColLevel0 + lv) * stride;
        t += col[b + 1] - col[b];
    }
    return t;
}

// The item sequence. Items are indices into the launch lists' id array for split nodes
// (< nsplit) and nsplit + b for the leaves of bucket b (buckets without leaves have no item; with
// groups = 0 no leaf items at all: the kernel's warps then take the leaves one by one after the
// last item). cnt[t]: items of time slot t.
__global__ void k_qorder_count(const uint32_t *__restrict__ offs, uint64_t stride, uint32_t nb, uint32_t nlevels,
                               uint32_t lag, uint32_t T, uint32_t groups, uint32_t *__restrict__ cnt) {
    const uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= T) return;
    uint32_t c = 0;
    for (uint32_t lv = 0; lv < nlevels + groups; lv++) {
        const uint64_t sh = (uint64_t)lv * lag;
        if (t < sh || t - sh >= nb) continue;
        const uint64_t b = t - sh;
        if (lv < nlevels) {
            const uint32_t *col = offs + (uint64_t)(kColLevel0 + lv) * stride;
            c += col[b + 1] - col[b];
        } else {
            const uint32_t *col = offs + (uint64_t)kColLeaves * stride;
            c += col[b + 1] > col[b];
        }
    }
    cnt[t] = c;
}

// Exclusive scan of cnt[0..T) into pos, the total into pos[T] (one block: a sequential run per
// thread, then the runs' sums).
__global__ void __launch_bounds__(1024) k_qorder_scan(const uint32_t *__restrict__ cnt, uint32_t T,
                                                      uint32_t *__restrict__ pos) {
    __shared__ uint32_t part[1024];
    const uint32_t per = (T + blockDim.x - 1) / blockDim.x;
    const uint32_t lo = min(T, threadIdx.x * per), hi = min(T, lo + per);
    uint32_t sum = 0;
    for (uint32_t i = lo; i < hi; i++) sum += cnt[i];
    part[threadIdx.x] = sum;
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t run = 0;
        for (uint32_t w = 0; w < blockDim.x; w++) {
            const uint32_t v = part[w];
            part[w] = run;
            run += v;
        }
    }
    __syncthreads();
    uint32_t run = part[threadIdx.x];
    for (uint32_t i = lo; i < hi; i++) {
        pos[i] = run;
        run += cnt[i];
    }
    if (threadIdx.x == blockDim.x - 1) pos[T] = run;
}

__global__ void k_qorder_scatter(const uint32_t *__restrict__ offs, uint64_t stride, uint32_t nb, uint32_t nlevels,
                                 uint32_t lag, uint32_t T, uint32_t groups, ListOffsets lists, uint32_t nsplit,
                                 const uint32_t *__restrict__ pos, uint32_t *__restrict__ seq) {
    const uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= T) return;
    uint32_t p = pos[t];
    for (uint32_t lv = 0; lv < nlevels + groups; lv++) {
        const uint64_t sh = (uint64_t)lv * lag;
        if (t < sh || t - sh >= nb) continue;
        const uint64_t b = t - sh;
        if (lv < nlevels) {
            const uint32_t *col = offs + (uint64_t)(kColLevel0 + lv) * stride;
            for (uint32_t j = col[b]; j < col[b + 1]; j++) seq[p++] = lists.level[lv] + j;
        } else {
            const uint32_t *col = offs + (uint64_t)kColLeaves * stride;
            if (col[b + 1] > col[b]) seq[p++] = nsplit + (uint32_t)b;
        }
    }
}

// Bucket b's retrieval input (its keys in tree order and their bits, without the size-1 positions,
// which have no bit) written by the calling block to its request's compacted arrays in host-mapped
// pinned memory, once the bucket's splits and leaves are done. Size-1 positions of the batch are
// singles[] (ascending), bucket b's at singles[scol[b] .. scol[b + 1]).
__device__ void write_bucket_out(uint32_t b, const uint64_t *__restrict__ acc, const uint64_t *__restrict__ keys,
                                 const uint8_t *__restrict__ rib_bits, const uint64_t *__restrict__ singles,
                                 const uint32_t *__restrict__ scol, const QueueOut *__restrict__ out, uint32_t nreq) {
    uint32_t lo = 0, hi = nreq;  // the request of bucket b: the last with b_first <= b
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (out[mid].b_first <= b) lo = mid; else hi = mid;
    }
    const QueueOut o = out[lo];
    const uint64_t k0 = acc[b], k1 = acc[b + 1], s0 = scol[b], s1 = scol[b + 1];
    const uint64_t base = (k0 - o.key_off) - (s0 - o.single_off);  // compacted index of the bucket's first kept key
    for (uint64_t i = k0 + threadIdx.x; i < k1; i += blockDim.x) {
        uint64_t below = 0;
        bool single = false;
        for (uint64_t t = s0; t < s1; t++) {  // a bucket has few size-1 positions
            const uint64_t sp = singles[t];
            below += sp < i;
            single |= sp == i;
        }
        if (single) continue;
        const uint64_t j = base + (i - k0) - below;
        o.keys[j] = __ldcg(&keys[i]);
        o.bits[j] = rib_bits[i];
    }
}

// The queue kernel's leaf search, out of line: called once per leaf, it keeps the split loop's
// register allocation apart from the leaf search's.
__device__ __noinline__ void queue_leaf(const NodeLeaves &leaves, uint32_t li, const uint64_t *__restrict__ keys,
                                        uint8_t *__restrict__ rib_bits, Sh2Smem<64> &sm, Sh2Global<64> &g, LaneUF2<64> &uf,
                                        int lane, uint32_t smax, uint32_t cmax, uint32_t *__restrict__ err, LeafWork &lw) {
    sh2_leaf<64, NodeLeaves, true, true>(leaves, li, keys, rib_bits, sm, g, uf, lane, smax, cmax, kQuadMinRecSplit, err, lw);
}

template <int SPL, int ARITH>
__global__ void __launch_bounds__(kQueueThreads, 3)
    k_tree_queue(const Node *__restrict__ nodes, const uint32_t *__restrict__ ids, const uint32_t *__restrict__ seq,
                 const uint32_t *__restrict__ nitems_p, uint32_t nsplit, const uint32_t *__restrict__ offs, uint64_t stride, uint32_t nlevels,
                 uint32_t *__restrict__ done, uint64_t *__restrict__ keys, uint64_t *__restrict__ codes,
                 uint8_t *__restrict__ rib_bits, uint8_t *__restrict__ scratch, uint64_t scratch_per_warp, uint32_t smax,
                 uint32_t cmax, uint64_t max_trials, uint32_t *__restrict__ err, unsigned long long *__restrict__ work,
                 unsigned long long *__restrict__ kind_work, unsigned int *__restrict__ ctr, uint32_t nleaf_tail,
                 const uint64_t *__restrict__ acc, const uint64_t *__restrict__ singles,
                 const QueueOut *__restrict__ out, uint32_t nreq, int round_div, const PipeK K) {
    extern __shared__ __align__(16) uint8_t smem_raw[];
    __shared__ uint32_t item, leaf_next;
    // the block's shared memory is one SplitSmem for a split node, one Sh2Smem per warp for leaves
    SplitSmem<SPL, kQueueThreads> &ssm = *reinterpret_cast<SplitSmem<SPL, kQueueThreads> *>(smem_raw);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    Sh2Smem<64> &sm = reinterpret_cast<Sh2Smem<64> *>(smem_raw)[warp];
    Sh2Global<64> g;
    g.carve(scratch + ((uint64_t)blockIdx.x * kQueueWarps + warp) * scratch_per_warp, smax, cmax);
    LaneUF2<64> uf{sm.uf, lane, 0, 0};
    LeafWork lw;
    const NodeLeaves leaves{nodes, ids + nsplit, codes};
    const uint32_t *leaf_col = offs + (uint64_t)kColLeaves * stride;
    const uint32_t nitems = *nitems_p;
    for (;;) {
        if (threadIdx.x == 0) item = atomicAdd(&ctr[0], 1u);
        __syncthreads();
        const uint32_t i = item;
        __syncthreads();
        const uint32_t it = i < nitems ? seq[i] : 0xffffffffu;
        if (it < nsplit) {
            const uint32_t id = ids[it];
            const Node nd = nodes[id];
            if (threadIdx.x == 0 && !wait_done(&done[nd.bucket], splits_above(offs, stride, nd.bucket, nd.level), err))
                atomicOr(err, kErrInternal);
            __syncthreads();
            split_node<SPL, kQueueThreads, ARITH, true>(ssm, nd, id, keys, codes, max_trials, err, work, kind_work,
                                                        round_div, K);
            __threadfence();  // this thread's part of the partition before the bucket's counter moves
            __syncthreads();
            if (threadIdx.x == 0) atomicAdd(&done[nd.bucket], 1u);
            continue;
        }
        // leaves: the group of bucket b (the block's warps share a counter), or, once the items are
        // all taken, the leaves left out of the sequence (every warp on its own from ctr[1])
        const bool group = i < nitems;
        const uint32_t b = group ? it - nsplit : 0, end = group ? leaf_col[b + 1] : nleaf_tail;
        if (group) {
            if (threadIdx.x == 0) {
                if (!wait_done(&done[b], splits_above(offs, stride, b, nlevels), err)) atomicOr(err, kErrInternal);
                leaf_next = leaf_col[b];
            }
            __syncthreads();
        }
        for (;;) {
            uint32_t li = 0;
            if (lane == 0) li = atomicAdd(group ? &leaf_next : &ctr[1], 1u);
            li = __shfl_sync(0xffffffffu, li, 0);
            if (li >= end) break;
            if (!group) {
                const uint32_t lb = nodes[ids[nsplit + li]].bucket;
                if (lane == 0 && !wait_done(&done[lb], splits_above(offs, stride, lb, nlevels), err))
                    atomicOr(err, kErrInternal);
                __syncwarp();
            }
            queue_leaf(leaves, li, keys, rib_bits, sm, g, uf, lane, smax, cmax, err, lw);
        }
        if (!group) break;
        __syncthreads();  // every warp is done with its Sh2Smem before a split node reuses the memory
        if (out) write_bucket_out(b, acc, keys, rib_bits, singles, offs + (uint64_t)kColSingles * stride, out, nreq);
    }
    unsigned long long w[5] = {lw.evals, lw.pairs, lw.filtered, lw.edges, lw.scan};
#pragma unroll
    for (int k = 0; k < 5; k++)
        for (int o = 16; o; o >>= 1) w[k] += __shfl_xor_sync(0xffffffffu, w[k], o);
    if (lane == 0)
        for (int k = 0; k < 5; k++) atomicAdd(&work[1 + k], w[k]);
}

template <int SPL, int ARITH>
void launch_queue_t(const Node *nodes, const uint32_t *ids, const uint32_t *seq, const uint32_t *nitems, uint32_t nsplit,
                    const uint32_t *offs, uint64_t stride, uint32_t nlevels, uint32_t *done, uint64_t *keys, uint64_t *codes,
                    uint8_t *rib_bits, uint8_t *scratch, uint64_t per_warp, uint32_t smax, uint32_t cmax,
                    uint64_t max_trials, uint32_t *err, unsigned long long *work, unsigned long long *kind_work,
                    unsigned int *ctr, uint32_t nleaf_tail, const uint64_t *acc, const uint64_t *singles,
                    const QueueOut *out, uint32_t nreq, int round_div, int grid, cudaStream_t s) {
    const size_t smem = std::max(sizeof(SplitSmem<SPL, kQueueThreads>), kQueueWarps * sizeof(Sh2Smem<64>));
    cudaFuncSetAttribute(k_tree_queue<SPL, ARITH>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    const PipeK K{4u, 32u, 1u << 18, 2u};
    k_tree_queue<SPL, ARITH><<<grid, kQueueThreads, smem, s>>>(nodes, ids, seq, nitems, nsplit, offs, stride, nlevels, done,
                                                               keys, codes, rib_bits, scratch, per_warp, smax, cmax,
                                                               max_trials, err, work, kind_work, ctr, nleaf_tail, acc,
                                                               singles, out, nreq, round_div, K);
}

} // namespace

// Bytes of global scratch per warp for the given capacities (raw seeds, candidates).
// Bytes of one warp's scratch slice (Sh2Global::carve's layout); rows / raws cap the cached cell rows
// (0: the configuration's caches).
static uint64_t sh2_slice_bytes(uint32_t smax, uint32_t cmax, int max_leaf, uint32_t row_cap, uint32_t raw_cap) {
    const uint64_t rows = std::min<uint64_t>(cmax, row_cap ? row_cap : max_leaf > 64 ? Sh2Cfg<128>::ROWS : Sh2Cfg<64>::ROWS);
    const uint64_t raw = std::min<uint64_t>(smax, raw_cap ? raw_cap : max_leaf > 64 ? Sh2Cfg<128>::RAW_ROWS : Sh2Cfg<64>::RAW_ROWS);
    return 16ull * smax + 256 + 24ull * cmax + (rows + raw) * (max_leaf > 64 ? 128 : 64);
}
uint64_t sh2_scratch_bytes(uint32_t smax, uint32_t cmax, int max_leaf) { return sh2_slice_bytes(smax, cmax, max_leaf, 0, 0); }

void launch_leaves_sh2_ctr(const Node *nodes, const uint32_t *ids, uint32_t count, const uint64_t *keys, uint64_t *codes,
                           uint8_t *rib_bits, uint8_t *scratch, uint64_t scratch_per_warp, uint32_t smax, uint32_t cmax,
                           uint32_t *err, unsigned long long *work, unsigned int *ctr, int grid, cudaStream_t s,
                           int max_leaf, uint32_t quad_min, int minb) {
    if (!count) return;
    cudaMemsetAsync(ctr, 0, sizeof(unsigned int), s);
    if (max_leaf > 64)
        launch_v2<128, 4>(nodes, ids, count, keys, codes, rib_bits, scratch, scratch_per_warp, smax, cmax, err, work, ctr, grid,
                          s, quad_min);
    else if (minb == 4)
        launch_v2<64, 4>(nodes, ids, count, keys, codes, rib_bits, scratch, scratch_per_warp, smax, cmax, err, work, ctr, grid,
                         s, quad_min);
    else if (minb == 8)
        launch_v2<64, 8>(nodes, ids, count, keys, codes, rib_bits, scratch, scratch_per_warp, smax, cmax, err, work, ctr, grid,
                         s, quad_min);
    else
        launch_v2<64, 6>(nodes, ids, count, keys, codes, rib_bits, scratch, scratch_per_warp, smax, cmax, err, work, ctr, grid,
                         s, quad_min);
}

int sh2_smem_per_warp(int max_leaf) { return max_leaf <= 64 ? (int)sizeof(Sh2Smem<64>) : (int)sizeof(Sh2Smem<128>); }

int tree_queue_warps_per_block() { return kQueueWarps; }
int tree_queue_smem_per_block(int spl) {
    const size_t leaf = kQueueWarps * sizeof(Sh2Smem<64>);
    const size_t split = spl == 1 ? sizeof(SplitSmem<1, kQueueThreads>)
                                  : spl == 4 ? sizeof(SplitSmem<4, kQueueThreads>) : sizeof(SplitSmem<2, kQueueThreads>);
    return (int)std::max(leaf, split);
}

uint64_t queue_order_slots(uint64_t nb, uint32_t nlevels, uint32_t lag) { return nb + (uint64_t)nlevels * lag; }

void launch_queue_order(const uint32_t *offs, uint64_t stride, uint64_t nb, uint32_t nlevels, uint32_t lag, bool groups,
                        const ListOffsets &lists, uint32_t nsplit, uint32_t *cnt, uint32_t *pos, uint32_t *seq,
                        cudaStream_t s) {
    const uint64_t T = queue_order_slots(nb, nlevels, lag);
    if (!T) return;
    const uint32_t blocks = (uint32_t)((T + 255) / 256);
    k_qorder_count<<<blocks, 256, 0, s>>>(offs, stride, (uint32_t)nb, nlevels, lag, (uint32_t)T, groups ? 1u : 0u, cnt);
    k_qorder_scan<<<1, 1024, 0, s>>>(cnt, (uint32_t)T, pos);
    k_qorder_scatter<<<blocks, 256, 0, s>>>(offs, stride, (uint32_t)nb, nlevels, lag, (uint32_t)T, groups ? 1u : 0u, lists,
                                            nsplit, pos, seq);
}

void launch_tree_queue(const Node *nodes, const uint32_t *ids, const uint32_t *seq, const uint32_t *nitems, uint32_t nsplit,
                       const uint32_t *offs, uint64_t stride, uint32_t nlevels, uint32_t *done, uint64_t *keys,
                       uint64_t *codes, uint8_t *rib_bits, uint8_t *scratch, uint64_t per_warp, uint32_t smax, uint32_t cmax,
                       uint64_t max_trials, uint32_t *err, unsigned long long *work, unsigned long long *kind_work,
                       unsigned int *ctr, uint32_t nleaf_tail, const uint64_t *acc, const uint64_t *singles,
                       const QueueOut *out, uint32_t nreq, const SplitTuning &t, int grid, cudaStream_t s) {
#define SHG_QUEUE_CASE(SPL, AR)                                                                                          \
    if (t.spl == SPL && t.arith == AR)                                                                                  \
        return launch_queue_t<SPL, AR>(nodes, ids, seq, nitems, nsplit, offs, stride, nlevels, done, keys, codes,        \
                                       rib_bits, scratch, per_warp, smax, cmax, max_trials, err, work, kind_work, ctr,   \
                                       nleaf_tail, acc, singles, out, nreq, t.round_div, grid, s);
    SHG_QUEUE_CASE(1, 0) SHG_QUEUE_CASE(2, 0) SHG_QUEUE_CASE(4, 0) SHG_QUEUE_CASE(1, 1) SHG_QUEUE_CASE(2, 1)
    SHG_QUEUE_CASE(4, 1)
#undef SHG_QUEUE_CASE
}

// ------------------------------------------------------------------ inner-loop peaks
// The leaf search's three non-hashing inner loops run alone on register and shared-memory operands,
// with every lane busy (no divergence, no early exit): their operations per second are the
// denominators of the leaf stage's work model (the hashing loop's is k_int_peak_sh2).
//   kind 0: candidate scan, one (A, B) mask pair of an earlier raw seed against the lane's raw seed
//           (two pairs per 16-byte broadcast load, as the 64-key scan);
//   kind 1: isolated-key filter of one candidate pair (two 64-bit masks from shared memory);
//   kind 2: one pseudoforest edge of a 64-key leaf (LaneUF2::add on shared-memory parents; each
//           test initialises the parents and adds 64 edges);
//   kind 3: kind 0 for 64-bit masks with the test written as (a | t) == full, the form the scan
//           used before its complement form (~t & ~a) == 0; the faster of the two bounds the scan.
namespace {
// W = 64: the loops of leaves of up to 64 keys (32-bit half masks, two raw seeds per 16-byte load,
// one isolated-key word, 64-edge tests); W = 128: of larger leaves (64-bit half masks, one raw seed
// per 16-byte load, two isolated-key words, 100-edge tests on 100 vertices).
template <int KIND, int W>
__global__ void __launch_bounds__(256) k_sh2_op_peak(uint64_t iters, unsigned long long *sink) {
    __shared__ uint4 masks[128];
    __shared__ uint64_t iso[2][256];
    __shared__ uint8_t par[8][(W == 64 ? 64 : 128) * 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint64_t tid = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    for (int i = threadIdx.x; i < 128; i += blockDim.x) {
        const uint64_t a = remix(0x51ull * i + 7), b = remix(a);
        masks[i] = make_uint4((uint32_t)a, (uint32_t)(a >> 32), (uint32_t)b, (uint32_t)(b >> 32));
    }
    for (int i = threadIdx.x; i < 256; i += blockDim.x) {
        iso[0][i] = remix(0x93ull * i + 3) & remix(0x77ull * i + 1);
        iso[1][i] = remix(0x95ull * i + 5) & remix(0x79ull * i + 2);
    }
    __syncthreads();
    uint64_t acc = 0;
    if (KIND == 0 && W == 64) {
        const uint64_t r = remix(tid);
        const uint32_t tA = (uint32_t)r, tB = (uint32_t)(r >> 32), full = 0xFFFFFFFFu;
        uint32_t hits = 0;
        for (uint64_t i = 0; i < iters; i++) {
            const uint4 w = masks[i & 127];
            const uint32_t z = min(min((w.x | tB) ^ full, (w.y | tA) ^ full), min((w.z | tB) ^ full, (w.w | tA) ^ full));
            hits += z == 0;
        }
        acc = hits;
    } else if (KIND == 0) {
        const uint64_t tA = remix(tid), tB = remix(tA), full = (1ull << 50) - 1, nA = ~tA & full, nB = ~tB & full;
        uint32_t hits = 0;
        for (uint64_t i = 0; i < iters; i++) {
            const uint4 w = masks[i & 127];
            const uint64_t a = (uint64_t)w.y << 32 | w.x, b = (uint64_t)w.w << 32 | w.z;
            hits += ((nB & ~a) == 0) | ((nA & ~b) == 0);  // the scan's complement form
        }
        acc = hits;
    } else if (KIND == 3) {  // the same test as (a | t) == full, full a value the compiler cannot fold
        const uint64_t tA = remix(tid), tB = remix(tA), full = ~0ull >> (14 + (tid >> 62));
        uint32_t hits = 0;
        for (uint64_t i = 0; i < iters; i++) {
            const uint4 w = masks[i & 127];
            const uint64_t a = (uint64_t)w.y << 32 | w.x, b = (uint64_t)w.w << 32 | w.z;
            hits += (((a | tB) ^ full) == 0) | (((b | tA) ^ full) == 0);
        }
        acc = hits;
    } else if (KIND == 1) {
        uint32_t j = 1 + (uint32_t)(tid & 63), i = (uint32_t)(tid >> 6) % j, hits = 0;
        for (uint64_t q = 0; q < iters; q++) {
            uint64_t x = iso[0][j & 255] & iso[0][i & 255];
            if (W == 128) x |= iso[1][j & 255] & iso[1][i & 255];
            hits += x == 0;
            if (++i == j) {  // (j, i) in lexicographic order, as the pair enumeration steps
                i = 0;
                j++;
            }
        }
        acc = hits;
    } else {
        constexpr uint32_t M = W == 64 ? 64 : 100, H = W == 64 ? 32 : 50;
        LaneUF2<W> uf{par[warp], lane, 0, 0};
        uint64_t x = remix(tid), ok = 0;
        for (uint64_t t = 0; t < iters; t++) {
            uf.init(M);
            for (uint32_t k = 0; k < M; k++) {
                x = x * 0x9E3779B97F4A7C15ull + 1;
                ok += uf.add(H + (uint32_t)(((x >> 20) & 0xFFFF) * H >> 16), (uint32_t)(((x >> 40) & 0xFFFF) * H >> 16));
            }
        }
        acc = ok;
    }
    sink[tid] = acc;  // every thread's result is stored: no loop can fold
}
}  // namespace

// Operations per launch thread and iteration: kinds 0..2 for leaves of up to 64 keys (2 scan tests,
// 1 pair filter, 64 edges), kinds 3..5 for larger leaves (1 scan test, 1 pair filter, 100 edges),
// kind 6 the larger leaves' scan test in its other form (1 scan test).
int sh2_op_peak_per_iter(int kind) {
    static const int per[7] = {2, 1, 64, 1, 1, 100, 1};
    return per[kind];
}
void launch_sh2_op_peak(int kind, int blocks, uint64_t iters, unsigned long long *sink) {
    switch (kind) {
        case 0: k_sh2_op_peak<0, 64><<<blocks, 256>>>(iters, sink); break;
        case 1: k_sh2_op_peak<1, 64><<<blocks, 256>>>(iters, sink); break;
        case 2: k_sh2_op_peak<2, 64><<<blocks, 256>>>(iters, sink); break;
        case 3: k_sh2_op_peak<0, 128><<<blocks, 256>>>(iters, sink); break;
        case 4: k_sh2_op_peak<1, 128><<<blocks, 256>>>(iters, sink); break;
        case 6: k_sh2_op_peak<3, 128><<<blocks, 256>>>(iters, sink); break;
        default: k_sh2_op_peak<2, 128><<<blocks, 256>>>(iters, sink); break;
    }
}

// ------------------------------------------------------------------ no-allocation variant
// Some callers cannot allocate device memory at the moment they need leaf seeds: code running
// under a host-side allocator that forbids cudaMalloc (a memory pool owned by another framework,
// a real-time or embedded host path), or code that already owns every
// buffer it may touch. For them the bipartite leaf search also runs from a fixed scratch area that
// lives in this library's own device image: kNoAllocScratchBytes (16 MiB) per device that loads the
// library, held until the process exits. Its layout: 256 bytes of counters (error flags, the leaf
// counter, work counters), then a spill slice per warp for raw-seed masks and candidates beyond
// what fits in shared memory (512 raw seeds and 512 candidates per leaf in this variant).
constexpr uint64_t kNoAllocScratchBytes = 16ull << 20;
constexpr uint32_t kNoAllocSmax = 512, kNoAllocCmax = 512;
static __device__ __align__(256) uint8_t g_noalloc_scratch[kNoAllocScratchBytes];

struct NoAllocCounters {
    uint32_t err;
    unsigned int leaf_ctr;
    unsigned long long work[8];
};

// Device address of g_noalloc_scratch on the current device, looked up once per device.
static uint8_t *noalloc_base(int device, cudaError_t &st) {
    static std::mutex mu;
    static uint8_t *addr[64] = {};
    std::lock_guard<std::mutex> lock(mu);
    st = cudaSuccess;
    if (device < 0 || device >= 64) {
        st = cudaErrorInvalidDevice;
        return nullptr;
    }
    if (!addr[device]) {
        void *p = nullptr;
        st = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (st != cudaSuccess) return nullptr;
        addr[device] = (uint8_t *)p;
    }
    return addr[device];
}

} // namespace shg

extern "C" shg_status shg_sh2_construct_leaves_noalloc(const uint64_t *d_keys, const uint64_t *d_leaf_offsets,
                                                       uint64_t nleaves, uint64_t *d_seeds, uint8_t *d_bits,
                                                       void *stream) {
    using namespace shg;
    if (nleaves == 0) return SHG_OK;
    if (!d_keys || !d_leaf_offsets || !d_seeds || !d_bits) return shg_set_error(SHG_ERR_ARG, "null device pointer");
    if (nleaves >= (1ull << 32)) return shg_set_error(SHG_ERR_ARG, "at most 2^32 - 1 leaves per call");
    int device = 0;
    if (cudaGetDevice(&device) != cudaSuccess) return shg_set_error(SHG_ERR_NO_DEVICE, "no current CUDA device");
    cudaError_t st;
    uint8_t *base = noalloc_base(device, st);
    if (!base) return shg_set_error(SHG_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(st));
    cudaStream_t s = (cudaStream_t)stream;
    NoAllocCounters *ctr = (NoAllocCounters *)base;
    // counters start at zero on every call; the spill slices need no clearing (written before read)
    if ((st = cudaMemsetAsync(ctr, 0, sizeof(NoAllocCounters), s)) != cudaSuccess)
        return shg_set_error(SHG_ERR_CUDA, std::string("cudaMemsetAsync: ") + cudaGetErrorString(st));
    const uint64_t per_warp = (sh2_slice_bytes(kNoAllocSmax, kNoAllocCmax, 64, OffsetLeaves<64>::kCandRows,
                                               OffsetLeaves<64>::kRawRows) + 255) & ~255ull;
    const uint64_t warps = (kNoAllocScratchBytes - 256) / per_warp;
    const uint64_t blocks = std::min<uint64_t>(warps / 4, (nleaves + 3) / 4);
    const size_t smem = sizeof(Sh2Smem<64>) * 4;
    k_leaves_sh2_v2<64, OffsetLeaves<64>><<<(int)blocks, 128, smem, s>>>(
        OffsetLeaves<64>{d_leaf_offsets, d_seeds}, (uint32_t)nleaves, d_keys, d_bits, base + 256, per_warp,
        kNoAllocSmax, kNoAllocCmax, &ctr->err, ctr->work, &ctr->leaf_ctr, kQuadMinRecSplit);
    if ((st = cudaGetLastError()) != cudaSuccess)
        return shg_set_error(SHG_ERR_CUDA, std::string("leaf kernel launch: ") + cudaGetErrorString(st));
    uint32_t err = 0;
    if ((st = cudaMemcpyAsync(&err, &ctr->err, sizeof(err), cudaMemcpyDeviceToHost, s)) != cudaSuccess ||
        (st = cudaStreamSynchronize(s)) != cudaSuccess)
        return shg_set_error(SHG_ERR_CUDA, std::string("leaf kernel: ") + cudaGetErrorString(st));
    if (err & kErrArg)
        return shg_set_error(SHG_ERR_ARG, "a leaf has fewer than 2 or more than 64 keys, or keys past 2^32 - 1 "
                                          "(limits of the no-allocation entry point)");
    if (err & kErrScratch)
        return shg_set_error(SHG_ERR_TRIAL_LIMIT, "a leaf needed more than 512 raw seeds or 512 candidates (the "
                                                  "no-allocation scratch limit; duplicate keys?)");
    if (err) return shg_set_error(SHG_ERR_CUDA, "internal device error flag " + std::to_string(err));
    return SHG_OK;
}
