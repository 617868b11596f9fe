// ShockHash leaf searches, one warp per leaf, leaves pulled from a device counter.
//
// Original ShockHash (ShockHash.h:404-434): lanes take consecutive seeds x; a lane's seed passes
// when the two candidate cells of all m keys cover all m cells (64-bit OR) and the cuckoo graph
// (cells = vertices, keys = edges) is a pseudoforest. The pseudoforest test is a per-lane
// union-find with a cycle flag per root; the reference inserts into a cuckoo table instead, and
// ordered cuckoo insertion succeeds exactly when the graph is a pseudoforest, so both accept the
// same seeds. The smallest accepted seed is kept (ballot + find-first-set), then lane 0 replays
// the reference's ordered cuckoo insertion to obtain the cell of every key (the retrieval bits).
//
// Bipartite ShockHash (ShockHash2-internal.h:34-107, 386-572): candidates are produced in the
// reference's order (Basic finder below 10 keys, QuadSplit finder otherwise), each new candidate
// is tested against all earlier ones in insertion order (isolated-vertex filter, then the
// pseudoforest test on the edges (h_new + m/2, h_old)), and the first passing pair is returned as
// pairTriangular(new, old). Lanes parallelise the raw-seed hashing, the candidate scans and the
// pairwise tests; the candidate list lives in a per-warp slice of global scratch (L1/L2 resident).
#include <cstdint>
#include <cuda_runtime.h>
#include "shg_common.cuh"
#include "shg_internal.h"

namespace shg {

constexpr int kLeafWarps = 4;  // warps per block
constexpr int kMaxLeafKeys = 128;

// ------------------------------------------------------------------ per-lane union-find
// parent[v * 32 + lane] (bytes) in shared memory; cycle flags of roots in two 64-bit registers.
struct LaneUF {
    uint8_t *par;
    int lane;
    uint64_t cyc0 = 0, cyc1 = 0;
    // Root of x with path halving.
    __device__ __forceinline__ uint32_t find(uint32_t x) {
        for (;;) {
            const uint32_t p = par[x * 32 + lane];
            if (p == x) return x;
            const uint32_t gp = par[p * 32 + lane];
            par[x * 32 + lane] = (uint8_t)gp;
            x = gp;
        }
    }
    __device__ __forceinline__ bool cyc(uint32_t r) const { return ((r < 64 ? cyc0 : cyc1) >> (r & 63)) & 1; }
    __device__ __forceinline__ void set_cyc(uint32_t r) {
        if (r < 64) cyc0 |= 1ull << r; else cyc1 |= 1ull << (r & 63);
    }
    __device__ __forceinline__ void init(uint32_t n) {
        for (uint32_t v = 0; v < n; v++) par[v * 32 + lane] = (uint8_t)v;
        cyc0 = cyc1 = 0;
    }
    // Adds edge (u, v); false when a component would get a second cycle.
    __device__ __forceinline__ bool add(uint32_t u, uint32_t v) {
        const uint32_t ru = find(u), rv = find(v);
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

// Ordered cuckoo insertion with cycle detection (TinyBinaryCuckooHashTable.h:169-198), run by one
// thread. cell[c] = key index or -1; xr[e] = c1 ^ c2 of key e. Returns false when the walk returns
// to its start (insertion impossible) or exceeds `limit` steps.
__device__ bool cuckoo_insert(int16_t *cell, uint8_t *xr, int e, uint32_t c1, uint32_t c2, int limit) {
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

// ------------------------------------------------------------------ original ShockHash leaves
struct Sh1WarpSmem {
    uint64_t keys[64];
    uint8_t uf[64 * 32];
    int16_t cell[64];
    uint8_t xr[64];
};

__global__ void __launch_bounds__(kLeafWarps * 32) k_leaves_sh1(const Node *__restrict__ nodes, const uint32_t *__restrict__ ids,
                                                                uint32_t count, const uint64_t *__restrict__ keys,
                                                                uint64_t *__restrict__ codes, uint64_t *__restrict__ rib_keys,
                                                                uint8_t *__restrict__ rib_bits, uint64_t max_trials,
                                                                uint32_t *__restrict__ err, unsigned long long *__restrict__ work,
                                                                unsigned int *__restrict__ next_leaf) {
    __shared__ Sh1WarpSmem wsm[kLeafWarps];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    Sh1WarpSmem &sm = wsm[warp];
    unsigned long long evals = 0;
    for (;;) {
        uint32_t li = 0;
        if (lane == 0) li = atomicAdd(next_leaf, 1u);
        li = __shfl_sync(0xffffffffu, li, 0);
        if (li >= count) break;
        const uint32_t id = ids[li];
        const Node nd = nodes[id];
        const uint32_t m = nd.m;
        for (uint32_t k = lane; k < m; k += 32) sm.keys[k] = keys[nd.start + k];
        __syncwarp();
        const uint64_t seed0 = start_seed(nd.level);
        const uint64_t all = (1ull << m) - 1;
        // ~2^(g+1) trials are expected; 2^(g+10) is only reached by duplicate keys.
        uint64_t cap = 1ull << min(nd.g + 10, 40);
        if (max_trials && max_trials < cap) cap = max_trials;
        LaneUF uf{sm.uf, lane};
        uint64_t found = ~0ull;
        for (uint64_t base = 0; base < cap; base += 32) {
            const uint64_t x = seed0 + base + lane;
            uint64_t mask = 0;
            for (uint32_t k = 0; k < m; k++) {
                uint32_t c1, c2;
                sh1_cells(sm.keys[k], x, m, c1, c2);
                mask |= (1ull << c1) | (1ull << c2);
            }
            bool ok = mask == all;
            if (__any_sync(0xffffffffu, ok)) {
                if (ok) {
                    uf.init(m);
                    for (uint32_t k = 0; k < m && ok; k++) {
                        uint32_t c1, c2;
                        sh1_cells(sm.keys[k], x, m, c1, c2);
                        ok = uf.add(c1, c2);
                    }
                }
                const unsigned bal = __ballot_sync(0xffffffffu, ok);
                if (bal) {
                    found = base + (__ffs(bal) - 1);
                    break;
                }
            }
        }
        if (found == ~0ull) {
            if (lane == 0) atomicOr(err, kErrTrialLimit);
            continue;
        }
        // Orientation: the reference's ordered cuckoo insertion (construct, TinyBinaryCuckooHashTable.h:80-106).
        if (lane == 0) {
            const uint64_t x = seed0 + found;
            for (uint32_t c = 0; c < m; c++) sm.cell[c] = -1;
            bool okc = true;
            for (uint32_t k = 0; k < m && okc; k++) {
                uint32_t c1, c2;
                sh1_cells(sm.keys[k], x, m, c1, c2);
                okc = cuckoo_insert(sm.cell, sm.xr, (int)k, c1, c2, 8 * (int)m + 16);
            }
            if (!okc) atomicOr(err, kErrInternal);
            codes[id] = found;
            evals += (found + 1) * m;
        }
        __syncwarp();
        // Retrieval input in cell order: key in cell i, bit (i >= m/2) (ShockHash.h:425-428).
        for (uint32_t c = lane; c < m; c += 32) {
            const int e = sm.cell[c];
            rib_keys[nd.start + c] = e >= 0 ? sm.keys[e] : 0;
            rib_bits[nd.start + c] = c >= m / 2 ? 1 : 0;
        }
        __syncwarp();
    }
    if (lane == 0 && evals) atomicAdd(&work[1], evals);
}

// ------------------------------------------------------------------ bipartite ShockHash leaves
struct Sh2WarpSmem {
    uint64_t keys[kMaxLeafKeys];   // finder order (QuadSplit: set A then set B reversed)
    uint64_t orig[kMaxLeafKeys];   // leaf order
    uint8_t row[kMaxLeafKeys];     // hashes of the candidate under test
    uint8_t uf[kMaxLeafKeys * 32];
    uint32_t hist[64];
    int16_t cell[kMaxLeafKeys];
    uint8_t xr[kMaxLeafKeys];
};

struct Sh2Scratch {
    uint64_t *maskA, *maskB;  // [smax]
    uint64_t *seed;           // [cmax]
    uint64_t *iso;            // [cmax][2]
    uint8_t *rows;            // [cmax][128]
};

__device__ __forceinline__ Sh2Scratch scratch_of(uint8_t *base, uint32_t smax, uint32_t cmax) {
    Sh2Scratch s;
    s.maskA = (uint64_t *)base;
    s.maskB = s.maskA + smax;
    s.seed = s.maskB + smax;
    s.iso = s.seed + cmax;
    s.rows = (uint8_t *)(s.iso + 2 * (size_t)cmax);
    return s;
}

uint64_t sh2_scratch_bytes(uint32_t smax, uint32_t cmax) {
    return 16ull * smax + 8ull * cmax + 16ull * cmax + (uint64_t)kMaxLeafKeys * cmax;
}

// Pseudoforest test of the pair (new candidate in sm.row, old candidate `row_i`); m edges.
__device__ __forceinline__ bool pair_ok(const Sh2WarpSmem &sm, LaneUF &uf, const uint8_t *__restrict__ row_i, uint32_t m,
                                        unsigned long long &edges) {
    uf.init(m);
    const uint32_t off = m / 2;
    for (uint32_t k0 = 0; k0 < m; k0 += 16) {
        const uint4 v = *reinterpret_cast<const uint4 *>(row_i + k0);
        const uint32_t w[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
        for (int q = 0; q < 16; q++) {
            const uint32_t k = k0 + q;
            if (k >= m) return true;
            const uint32_t a = sm.row[k] + off;
            const uint32_t b = (w[q >> 2] >> (8 * (q & 3))) & 0xFF;
            edges++;
            if (!uf.add(a, b)) return false;
        }
    }
    return true;
}

__global__ void __launch_bounds__(kLeafWarps * 32) k_leaves_sh2(const Node *__restrict__ nodes, const uint32_t *__restrict__ ids,
                                                                uint32_t count, const uint64_t *__restrict__ keys,
                                                                uint64_t *__restrict__ codes, uint8_t *__restrict__ rib_bits,
                                                                uint8_t *__restrict__ scratch, uint64_t scratch_per_warp,
                                                                uint32_t smax, uint32_t cmax, uint32_t *__restrict__ err,
                                                                unsigned long long *__restrict__ work,
                                                                unsigned int *__restrict__ next_leaf) {
    extern __shared__ __align__(16) uint8_t smem_raw[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    Sh2WarpSmem &sm = reinterpret_cast<Sh2WarpSmem *>(smem_raw)[warp];
    const uint64_t gw = (uint64_t)blockIdx.x * kLeafWarps + warp;
    const Sh2Scratch scr = scratch_of(scratch + gw * scratch_per_warp, smax, cmax);
    LaneUF uf{sm.uf, lane};
    unsigned long long w_evals = 0, w_pairs = 0, w_filtered = 0, w_edges = 0;

    for (;;) {
        uint32_t li = 0;
        if (lane == 0) li = atomicAdd(next_leaf, 1u);
        li = __shfl_sync(0xffffffffu, li, 0);
        if (li >= count) break;
        const uint32_t id = ids[li];
        const Node nd = nodes[id];
        const uint32_t m = nd.m;
        const uint32_t half = (m + 1) / 2;
        const uint64_t full = half >= 64 ? ~0ull : (1ull << half) - 1;
        const bool quad = m >= 10;

        // Keys in finder order. QuadSplit: even keys first in order, odd keys from the back
        // (QuadSplitCandidateFinder ctor, ShockHash2-internal.h:397-407).
        uint32_t sizeA = m;
        {
            uint32_t evens_before = 0, odds_before = 0;
            for (uint32_t k0 = 0; k0 < m; k0 += 32) {
                const uint32_t k = k0 + lane;
                const uint64_t key = k < m ? keys[nd.start + k] : 0;
                const bool even = (key & 1) == 0;
                const unsigned be = __ballot_sync(0xffffffffu, k < m && even);
                const unsigned bo = __ballot_sync(0xffffffffu, k < m && !even);
                const unsigned below = (1u << lane) - 1;
                if (k < m) {
                    sm.orig[k] = key;
                    uint32_t pos = k;
                    if (quad) pos = even ? evens_before + __popc(be & below) : m - 1 - (odds_before + __popc(bo & below));
                    sm.keys[pos] = key;
                }
                evens_before += __popc(be);
                odds_before += __popc(bo);
            }
            if (quad) sizeA = evens_before;
        }
        __syncwarp();

        uint32_t ncand = 0;
        uint64_t s_next = 0;   // next raw seed to hash
        uint64_t answer = ~0ull;
        bool overflow = false;
        unsigned long long cands_made = 0;

        // Processes one candidate (seedA, seedB) with candidate seed `cs`; returns true when it
        // completes a pair (answer set).
        auto process = [&](uint64_t sa, uint64_t sb, uint64_t cs) -> bool {
            cands_made++;
            // hashes of this candidate, and the isolated-key mask (calculateIsolatedVertices)
            for (uint32_t c = lane; c < 64; c += 32) sm.hist[c] = 0;
            __syncwarp();
            uint32_t hk[4];
#pragma unroll
            for (int q = 0; q < 4; q++) {
                const uint32_t k = lane + 32 * q;
                hk[q] = 0;
                if (k < m) {
                    hk[q] = half_hash(sm.keys[k], k < sizeA ? sa : sb, half);
                    sm.row[k] = (uint8_t)hk[q];
                    atomicAdd(&sm.hist[hk[q]], 1u);
                }
            }
            __syncwarp();
            uint64_t iso0 = 0, iso1 = 0;
#pragma unroll
            for (int q = 0; q < 4; q++) {
                const uint32_t k = lane + 32 * q;
                const unsigned b = __ballot_sync(0xffffffffu, k < m && sm.hist[hk[q]] == 1);
                if (q == 0) iso0 |= b;
                if (q == 1) iso0 |= (uint64_t)b << 32;
                if (q == 2) iso1 |= b;
                if (q == 3) iso1 |= (uint64_t)b << 32;
            }
            // test against every earlier candidate, in insertion order
            for (uint32_t c0 = 0; c0 < ncand; c0 += 32) {
                const uint32_t i = c0 + lane;
                bool filt = false;
                if (i < ncand) {
                    const uint64_t o0 = scr.iso[2 * i], o1 = scr.iso[2 * i + 1];
                    filt = ((o0 & iso0) | (o1 & iso1)) == 0;
                }
                w_pairs += (i < ncand);
                w_filtered += filt;
                bool ok = filt && pair_ok(sm, uf, scr.rows + (size_t)i * kMaxLeafKeys, m, w_edges);
                unsigned pass = __ballot_sync(0xffffffffu, ok);
                while (pass) {
                    const uint32_t j = c0 + __ffs(pass) - 1;
                    const uint64_t other = scr.seed[j];
                    if (float_accurate_triangular(cs, other)) {
                        answer = pair_triangular(cs, other);
                        return true;
                    }
                    pass &= pass - 1;
                }
            }
            if (ncand >= cmax) {
                overflow = true;
                return true;
            }
            // append to the candidate list
            for (uint32_t k = lane * 4; k < kMaxLeafKeys; k += 128) {
                uint32_t v = 0;
                for (int q = 0; q < 4; q++) v |= (uint32_t)(k + q < m ? sm.row[k + q] : 0) << (8 * q);
                *reinterpret_cast<uint32_t *>(scr.rows + (size_t)ncand * kMaxLeafKeys + k) = v;
            }
            if (lane == 0) {
                scr.seed[ncand] = cs;
                scr.iso[2 * ncand] = iso0;
                scr.iso[2 * ncand + 1] = iso1;
            }
            ncand++;
            __syncwarp();
            return false;
        };

        for (uint64_t s = 0; answer == ~0ull && !overflow; s++) {
            if (s == s_next) {
                // hash the next 32 raw seeds: coverage masks of set A and set B per seed
                const uint64_t sl = s_next + lane;
                uint64_t tA = 0, tB = 0;
                for (uint32_t k = 0; k < m; k++) {
                    const uint64_t bit = 1ull << half_hash(sm.keys[k], sl, half);
                    if (k < sizeA) tA |= bit; else tB |= bit;
                }
                if (s_next + 32 > smax) {
                    overflow = true;
                    break;
                }
                scr.maskA[sl] = tA;
                scr.maskB[sl] = tB;
                s_next += 32;
                __syncwarp();
            }
            w_evals += m;
            const uint64_t tA = scr.maskA[s], tB = scr.maskB[s];
            if (!quad) {
                // Basic finder: seed s is a candidate when it covers all half-table cells.
                if (tA == full && process(s, s, s)) break;
                continue;
            }
            // pairs (a < s, s), ascending a (earlier A masks against the new B mask)
            bool done = false;
            for (uint64_t a0 = 0; a0 < s && !done; a0 += 32) {
                const uint64_t a = a0 + lane;
                const bool c = a < s && (scr.maskA[a] | tB) == full && float_accurate_elegant(a, s);
                unsigned bal = __ballot_sync(0xffffffffu, c);
                while (bal && !done) {
                    const uint64_t aa = a0 + __ffs(bal) - 1;
                    bal &= bal - 1;
                    done = process(aa, s, pair_elegant(aa, s));
                }
            }
            if (done) break;
            // pairs (s, b <= s), ascending b (all B masks so far against the new A mask)
            for (uint64_t b0 = 0; b0 <= s && !done; b0 += 32) {
                const uint64_t b = b0 + lane;
                const bool c = b <= s && (scr.maskB[b] | tA) == full && float_accurate_elegant(s, b);
                unsigned bal = __ballot_sync(0xffffffffu, c);
                while (bal && !done) {
                    const uint64_t bb = b0 + __ffs(bal) - 1;
                    bal &= bal - 1;
                    done = process(s, bb, pair_elegant(s, bb));
                }
            }
            if (done) break;
        }
        w_evals += cands_made * m;
        if (overflow || answer == ~0ull) {
            if (lane == 0) atomicOr(err, kErrScratch);
            continue;
        }

        // Retrieval bits (constructRetrieval, ShockHash2-internal.h:548-572): ordered cuckoo
        // insertion of the leaf keys in leaf order, bit 1 when a key rests in its seed2 cell.
        uint64_t s1, s2;
        unpair_triangular(answer, s1, s2);
        if (lane == 0) {
            for (uint32_t c = 0; c < m; c++) sm.cell[c] = -1;
            bool okc = true;
            for (uint32_t k = 0; k < m && okc; k++) {
                const uint64_t key = sm.orig[k];
                okc = cuckoo_insert(sm.cell, sm.xr, (int)k, sh2_cand_hash(key, s1, m) + m / 2, sh2_cand_hash(key, s2, m),
                                    8 * (int)m + 16);
            }
            if (!okc) atomicOr(err, kErrInternal);
            codes[id] = answer;
        }
        __syncwarp();
        for (uint32_t k = lane; k < m; k += 32) {
            const uint32_t c2 = sh2_cand_hash(sm.orig[k], s2, m);
            rib_bits[nd.start + k] = sm.cell[c2] == (int16_t)k ? 1 : 0;
        }
        __syncwarp();
    }
    // lane-summed counters
    for (int o = 16; o; o >>= 1) {
        w_pairs += __shfl_xor_sync(0xffffffffu, w_pairs, o);
        w_filtered += __shfl_xor_sync(0xffffffffu, w_filtered, o);
        w_edges += __shfl_xor_sync(0xffffffffu, w_edges, o);
    }
    if (lane == 0) {
        atomicAdd(&work[1], w_evals);
        atomicAdd(&work[2], w_pairs);
        atomicAdd(&work[3], w_filtered);
        atomicAdd(&work[4], w_edges);
    }
}

int leaves_sh2_warps_per_block() { return kLeafWarps; }
int leaves_sh1_warps_per_block() { return kLeafWarps; }

void launch_leaves_sh1_ctr(const Node *nodes, const uint32_t *ids, uint32_t count, const uint64_t *keys, uint64_t *codes,
                           uint64_t *rib_keys, uint8_t *rib_bits, uint64_t max_trials, uint32_t *err,
                           unsigned long long *work, unsigned int *ctr, int grid, cudaStream_t s) {
    if (!count) return;
    cudaMemsetAsync(ctr, 0, sizeof(unsigned int), s);
    k_leaves_sh1<<<grid, kLeafWarps * 32, 0, s>>>(nodes, ids, count, keys, codes, rib_keys, rib_bits, max_trials, err,
                                                  work, ctr);
}

void launch_leaves_sh2_ctr(const Node *nodes, const uint32_t *ids, uint32_t count, const uint64_t *keys, uint64_t *codes,
                           uint8_t *rib_bits, uint8_t *scratch, uint64_t scratch_per_warp, uint32_t smax, uint32_t cmax,
                           uint32_t *err, unsigned long long *work, unsigned int *ctr, int grid, cudaStream_t s) {
    if (!count) return;
    cudaMemsetAsync(ctr, 0, sizeof(unsigned int), s);
    const size_t smem = sizeof(Sh2WarpSmem) * kLeafWarps;
    static bool attr_set = false;
    if (!attr_set) {
        cudaFuncSetAttribute(k_leaves_sh2, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        attr_set = true;
    }
    k_leaves_sh2<<<grid, kLeafWarps * 32, smem, s>>>(nodes, ids, count, keys, codes, rib_bits, scratch, scratch_per_warp,
                                                     smax, cmax, err, work, ctr);
}

} // namespace shg
