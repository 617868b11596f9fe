// ShockHash leaf searches, one warp per leaf, leaves pulled from a device counter.
//
// Original ShockHash (ShockHash.h:404-434): lanes take consecutive seeds x (SPL per lane, x, x + 32,
// ..., per round of 32 * SPL); a lane's seed passes
// when the two candidate cells of all m keys cover all m cells (64-bit OR) and the cuckoo graph
// (cells = vertices, keys = edges) is a pseudoforest. The pseudoforest test is a per-lane
// union-find with a cycle flag per root; the reference inserts into a cuckoo table instead, and
// ordered cuckoo insertion succeeds exactly when the graph is a pseudoforest, so both accept the
// same seeds. The coverage mask is kept as two 32-bit halves (first-half and second-half cells).
// The smallest accepted seed is kept (ballot + find-first-set), then lane 0 replays
// the reference's ordered cuckoo insertion to obtain the cell of every key (the retrieval bits).
//
// The bipartite leaf search is in shg_leaves_sh2.cu.
#include <cstdint>
#include <cuda_runtime.h>
#include "shg_common.cuh"
#include "shg_internal.h"

namespace shg {

constexpr int kLeafWarps = 4;  // warps per block

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
// Seeds that pass the coverage test queue up (in seed order) until kSh1Drain of them wait, and are
// then tested for the pseudoforest property side by side, one per lane: tested one round at a
// time, a round's one or two passing seeds ran the union-find while the other lanes waited.
#ifndef SHG_SH1_DRAIN
#define SHG_SH1_DRAIN 4
#endif
constexpr uint32_t kSh1Drain = SHG_SH1_DRAIN;
constexpr uint32_t kSh1Queue = kSh1Drain + 64;  // fewer than kSh1Drain wait, plus one round's 32 x SPL (SPL <= 2)

struct Sh1WarpSmem {
    uint64_t q[kSh1Queue];  // coverage-passing seed offsets, ascending
    uint64_t keys[64];
    uint64_t fkeys[64];  // rotation fitting: even keys in order, odd keys from the back
    uint8_t uf[64 * 32];
    int16_t cell[64];
    uint8_t xr[64];
};

// Rotation of the low l bits of v by r (ShockHash.h:299-301).
__device__ __forceinline__ uint64_t rot_bits(uint64_t v, uint32_t r, uint32_t l) {
    return r ? ((v << r) | (v >> (l - r))) & ((1ull << l) - 1) : v;
}

// ShockHash<L, true>: a leaf of exactly L keys with rotation fitting (ShockHash.h:316-399). Keys
// are split into set A (even keys, in order) and set B (odd keys, from the back); for seed x, set A
// hashes with x & ~mask (mask 7 when L > 32, so eight seeds share set A's cells) and set B with x.
// For r = 0..L-1 the candidate is set B's cells rotated by r: it passes when A's cells and B's
// rotated cells cover all L cells and the cuckoo graph is a pseudoforest. The answer is the
// smallest x, then the smallest r (lanes take consecutive x, each lane tries its r in order);
// the stored code is (x - start_seed) * L + r.
__device__ bool rotation_leaf(Sh1WarpSmem &sm, uint16_t *cells, LaneUF &uf, int lane, uint32_t m, uint64_t seed0,
                              uint64_t cap_x, uint64_t &code) {
    const unsigned below = (1u << lane) - 1;
    uint32_t nA = 0, nB = 0;
    for (uint32_t k0 = 0; k0 < m; k0 += 32) {
        const uint32_t k = k0 + lane;
        const uint64_t key = k < m ? sm.keys[k] : 0;
        const bool even = (key & 1) == 0;
        const unsigned be = __ballot_sync(0xffffffffu, k < m && even), bo = __ballot_sync(0xffffffffu, k < m && !even);
        if (k < m) sm.fkeys[even ? nA + __popc(be & below) : m - 1 - (nB + __popc(bo & below))] = key;
        nA += __popc(be);
        nB += __popc(bo);
    }
    __syncwarp();
    const uint64_t gmask = m > 32 ? 7 : 0;
    const uint64_t all = (1ull << m) - 1;
    // cells[k * 32 + lane] = c1 | c2 << 8 of key k under the lane's seed, written by the coverage
    // pass; with gmask a set-A key's cells sit in the slot of the group lane that hashed it
    auto pseudoforest = [&](uint32_t r) {
        uf.init(m);
        bool ok = true;
        for (uint32_t k = 0; k < m && ok; k++) {
            uint32_t c1, c2;
            if (k < nA) {
                const uint32_t w = cells[k * 32 + (gmask ? ((lane & ~7) | (k & 7)) : lane)];
                c1 = w & 0xFF;
                c2 = w >> 8;
            } else {
                const uint32_t w = cells[k * 32 + lane];
                c1 = ((w & 0xFF) + r) % m;
                c2 = ((w >> 8) + r) % m;
            }
            ok = uf.add(c1, c2);
        }
        return ok;
    };
    // Rounds of 32 seeds start at a multiple of 8 (seeds below seed0 in the first round take no
    // part), so with gmask = 7 each aligned group of 8 lanes shares set A's seed: its lanes hash
    // every eighth set-A key and OR their masks together.
    const uint64_t x_lo = seed0 & ~7ull;
    for (uint64_t off = 0; off < cap_x + (seed0 - x_lo); off += 32) {
        const uint64_t x = x_lo + off + lane, xa = x & ~gmask;
        const bool live = x >= seed0 && x - seed0 < cap_x;
        uint64_t a = 0, b = 0;
        if (gmask) {
            for (uint32_t k = lane & 7; k < nA; k += 8) {
                uint32_t c1, c2;
                sh1_cells(sm.fkeys[k], xa, m, c1, c2);
                a |= (1ull << c1) | (1ull << c2);
                cells[k * 32 + lane] = (uint16_t)(c1 | c2 << 8);
            }
            a |= __shfl_xor_sync(0xffffffffu, a, 1);
            a |= __shfl_xor_sync(0xffffffffu, a, 2);
            a |= __shfl_xor_sync(0xffffffffu, a, 4);
        } else {
            for (uint32_t k = 0; k < nA; k++) {
                uint32_t c1, c2;
                sh1_cells(sm.fkeys[k], xa, m, c1, c2);
                a |= (1ull << c1) | (1ull << c2);
                cells[k * 32 + lane] = (uint16_t)(c1 | c2 << 8);
            }
        }
        for (uint32_t k = nA; k < m; k++) {
            uint32_t c1, c2;
            sh1_cells(sm.fkeys[k], x, m, c1, c2);
            b |= (1ull << c1) | (1ull << c2);
            cells[k * 32 + lane] = (uint16_t)(c1 | c2 << 8);
        }
        __syncwarp();
        int rr = -1;
        if (live)
            for (uint32_t r = 0; r < m; r++)
                if ((a | rot_bits(b, r, m)) == all && pseudoforest(r)) {
                    rr = (int)r;
                    break;
                }
        const unsigned bal = __ballot_sync(0xffffffffu, rr >= 0);  // also orders the cell reads before the next round's writes
        if (bal) {
            const int src = __ffs(bal) - 1;
            const uint64_t fx = x_lo + off + src - seed0;
            const int fr = __shfl_sync(0xffffffffu, rr, src);
            if (fx >= cap_x) return false;
            code = fx * m + (uint64_t)fr;
            // orientation: the reference's ordered insertion in set order, then cell order
            if (lane == 0) {
                const uint64_t xf = seed0 + fx;
                for (uint32_t c = 0; c < m; c++) sm.cell[c] = -1;
                bool okc = true;
                for (uint32_t k = 0; k < m && okc; k++) {
                    uint32_t c1, c2;
                    if (k < nA) {
                        sh1_cells(sm.fkeys[k], xf & ~gmask, m, c1, c2);
                    } else {
                        sh1_cells(sm.fkeys[k], xf, m, c1, c2);
                        c1 = (c1 + fr) % m;
                        c2 = (c2 + fr) % m;
                    }
                    okc = cuckoo_insert(sm.cell, sm.xr, (int)k, c1, c2, 8 * (int)m + 16);
                }
                if (!okc) code = ~0ull;
            }
            code = __shfl_sync(0xffffffffu, code, 0);
            return code != ~0ull;
        }
    }
    return false;
}

// SPL: seeds per lane and round (1 or 2; a tuning parameter, the same seed is found either way).
template <int SPL>
__global__ void __launch_bounds__(kLeafWarps * 32) k_leaves_sh1(const Node *__restrict__ nodes, const uint32_t *__restrict__ ids,
                                                                uint32_t count, const uint64_t *__restrict__ keys,
                                                                uint64_t *__restrict__ codes, uint64_t *__restrict__ rib_keys,
                                                                uint8_t *__restrict__ rib_bits, uint64_t max_trials,
                                                                uint32_t *__restrict__ err, unsigned long long *__restrict__ work,
                                                                unsigned int *__restrict__ next_leaf, uint32_t rot_leaf) {
    __shared__ Sh1WarpSmem wsm[kLeafWarps];
    extern __shared__ uint16_t rot_cells[];  // rotation fitting only: [warp][64 keys][32 lanes]
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
        // Coverage in two 32-bit halves: c1 < m/2 and c2 - m/2 < (m+1)/2, both <= 30 for m <= 60.
        const uint32_t h1 = m / 2, h2 = (m + 1) / 2;
        // (m = 1: fastrange32(., 0) = 0 always sets bit 0 of the empty first half; that cell is the
        // second half's cell 0, which c2 = 0 covers, so bit 0 counts as covered.)
        const uint32_t all1 = h1 ? (1u << h1) - 1 : 1u, all2 = (1u << h2) - 1;
        // ~2^(g+1) trials are expected; 2^(g+10) is only reached by duplicate keys.
        uint64_t cap = 1ull << min(nd.g + 10, 40);
        if (max_trials && max_trials < cap) cap = max_trials;
        LaneUF uf{sm.uf, lane};
        if (rot_leaf && m == rot_leaf) {
            // ~2^(g+1) codes x * L + r are expected; the cap counts seeds x
            uint64_t cap_x = (1ull << min(nd.g + 10, 40)) / m + 1;
            if (max_trials && max_trials < cap_x) cap_x = max_trials;
            uint64_t code = 0;
            const bool ok = rotation_leaf(sm, rot_cells + warp * 64 * 32, uf, lane, m, seed0, cap_x, code);
            if (!ok) {
                if (lane == 0) atomicOr(err, code == ~0ull ? kErrInternal : kErrTrialLimit);
                continue;
            }
            if (lane == 0) {
                codes[id] = code;
                evals += (code / m + 1) * m;
            }
            __syncwarp();
            // retrieval input in cell order; the bit is the unrotated cell's half (ShockHash.h:384-391)
            for (uint32_t c = lane; c < m; c += 32) {
                const int e = sm.cell[c];
                const uint64_t key = e >= 0 ? sm.fkeys[e] : 0;
                const uint32_t r = (uint32_t)(code % m);
                const uint32_t cell = (key & 1) ? (c + m - r) % m : c;
                rib_keys[nd.start + c] = key;
                rib_bits[nd.start + c] = cell < m / 2 ? 0 : 1;
            }
            __syncwarp();
            continue;
        }
        uint64_t found = ~0ull;
        // Pseudoforest test of one lane's seed (union-find with a cycle flag per root).
        auto pseudoforest = [&](uint64_t x) {
            uf.init(m);
            bool ok = true;
            for (uint32_t k = 0; k < m && ok; k++) {
                uint32_t c1, c2;
                sh1_cells(sm.keys[k], x, m, c1, c2);
                ok = uf.add(c1, c2);
            }
            return ok;
        };
        // queued survivors, tested 32 at a time in queue (= seed) order: the first passing one is
        // the smallest passing seed, as every smaller seed failed coverage or an earlier test
        const unsigned below = (1u << lane) - 1;
        uint32_t nq = 0;
        auto drain = [&]() {
            for (uint32_t q0 = 0; q0 < nq && found == ~0ull; q0 += 32) {
                const uint64_t off = q0 + lane < nq ? sm.q[q0 + lane] : ~0ull;
                const bool pass = off != ~0ull && pseudoforest(seed0 + off);
                const unsigned bal = __ballot_sync(0xffffffffu, pass);
                if (bal) found = __shfl_sync(0xffffffffu, off, __ffs(bal) - 1);
            }
            nq = 0;
            __syncwarp();  // the queue's slots are read before the next round refills them
        };
        // SPL seeds per lane (x, x + 32, ...): one shared-memory key read feeds SPL evaluations.
        for (uint64_t base = 0; base < cap && found == ~0ull; base += 32 * SPL) {
            uint32_t c1m[SPL], c2m[SPL];
#pragma unroll
            for (int t = 0; t < SPL; t++) c1m[t] = c2m[t] = 0;
            for (uint32_t k = 0; k < m; k++) {
                const uint64_t key = sm.keys[k];
#pragma unroll
                for (int t = 0; t < SPL; t++) {
                    const uint64_t r = remix(key + seed0 + base + lane + 32 * t);
                    c1m[t] |= 1u << fastrange32((uint32_t)r, h1);
                    c2m[t] |= 1u << fastrange32((uint32_t)(r >> 32), h2);
                }
            }
            bool ok[SPL], any = false;
#pragma unroll
            for (int t = 0; t < SPL; t++) {
                ok[t] = c1m[t] == all1 && c2m[t] == all2;
                any |= ok[t];
            }
            if (__any_sync(0xffffffffu, any)) {
#pragma unroll
                for (int t = 0; t < SPL; t++) {  // seeds in order: all lanes' x + 32 t before x + 32 (t + 1)
                    const unsigned bal = __ballot_sync(0xffffffffu, ok[t]);
                    if (ok[t]) sm.q[nq + __popc(bal & below)] = base + 32 * t + lane;
                    nq += __popc(bal);
                }
                __syncwarp();
                if (nq >= kSh1Drain) drain();
            }
        }
        if (found == ~0ull && nq) drain();  // the last survivors, at the trial limit
        if (found == ~0ull || found >= cap) {
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

int leaves_sh1_warps_per_block() { return kLeafWarps; }

void launch_leaves_sh1_ctr(const Node *nodes, const uint32_t *ids, uint32_t count, const uint64_t *keys, uint64_t *codes,
                           uint64_t *rib_keys, uint8_t *rib_bits, uint64_t max_trials, uint32_t *err,
                           unsigned long long *work, unsigned int *ctr, int grid, cudaStream_t s, uint32_t rot_leaf,
                           int spl) {
    if (!count) return;
    cudaMemsetAsync(ctr, 0, sizeof(unsigned int), s);
    const size_t dyn = rot_leaf ? (size_t)kLeafWarps * 64 * 32 * sizeof(uint16_t) : 0;  // 16 KB per block
    if (spl == 1)
        k_leaves_sh1<1><<<grid, kLeafWarps * 32, dyn, s>>>(nodes, ids, count, keys, codes, rib_keys, rib_bits, max_trials,
                                                           err, work, ctr, rot_leaf);
    else
        k_leaves_sh1<2><<<grid, kLeafWarps * 32, dyn, s>>>(nodes, ids, count, keys, codes, rib_keys, rib_bits, max_trials,
                                                           err, work, ctr, rot_leaf);
}

} // namespace shg
