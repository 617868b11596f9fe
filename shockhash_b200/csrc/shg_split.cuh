// RecSplit split-seed search and stable partition of one node (ShockHash.h:451-547,
// ShockHash2.h:290-386), shared by the per-level split kernel (shg_split.cu) and the work-queue
// kernel (shg_leaves_sh2.cu).
//
// One thread block per split node. The node's keys (<= 3000 x 8 B) sit in shared memory and are
// read as warp-wide broadcasts; each lane owns SPL consecutive-in-round seeds and keeps
// per-seed part counts in registers. A seed x is valid when every part but the last receives
// exactly its size under  part(k) = remap16(remix(k + x), m) / unit  (fanout 2: h >= split).
//
// The part test never multiplies: h = (r16 * m) >> 16 < K  <=>  r16 < ceil(K * 65536 / m) with
// r16 the low 16 bits of remix, so each part boundary becomes one 16-bit threshold and only the
// low 47 bits of remix's second product are needed.
//
// Rounds: the block evaluates 32*SPL*G seeds per round (SPL seeds per lane, G warp groups; a
// group's warps split the node's keys and merge counts in shared memory). G is picked from the
// node's expected trial count 1/p (the same p the Golomb-Rice memo uses) so that a round stays near
// 1/round_div of it and the overshoot past the answer stays small. The smallest valid seed of the
// first round that has one is the answer, identical to the reference's sequential `for (;;) x++`
// search, for every choice of SPL, block size and round_div (the tuning parameters).
#pragma once
#include <cmath>
#include <cstdint>
#include <cuda_runtime.h>
#include "shg_common.cuh"
#include "shg_internal.h"

namespace shg {

// The low 16 bits of a key's split hash under seed x (z = key + x): remix for ShockHash and
// ShockHash2 (arithmetic forms 0 and 1), SIMDShockHash's fmix32 fold for kSplitArithSimd.
template <int ARITH> __device__ __forceinline__ uint32_t split_r16(uint64_t z) {
    if constexpr (ARITH == kSplitArithSimd) return simd_split_low16(z);
    else return remix_low16(z);
}

template <int SPL, int THREADS> struct SplitSmem {
    static constexpr int kWarps = THREADS / 32;
    uint64_t keys[kMaxBucket];
    uint32_t part_counts[kWarps][32 * SPL][3];
    uint64_t scan[kWarps];
    uint32_t best;
};

// Counts of keys below each of NT thresholds, for SPL seeds, over keys [lo, hi).
// ARITH 1 computes the same counts with remix_lo32_pipes and multiply-add-high counting (r < T is
// the sign bit of r - T), trading integer-pipe instructions for multiply-pipe ones. ARITH
// kSplitArithSimd counts under SIMDShockHash's split hash.
template <int NT, int SPL, int ARITH>
__device__ __forceinline__ void count_range(const uint64_t *__restrict__ sk, uint32_t lo, uint32_t hi, uint64_t x0,
                                            const uint32_t T0, const uint32_t T1, const uint32_t T2,
                                            uint32_t (&c)[SPL][3], const PipeK &K) {
    const uint32_t T[3] = {T0, T1, T2};
    uint32_t i = lo;
    if constexpr (ARITH == 1) {
        for (; i < hi; i++) {
            const uint64_t k0 = sk[i];
#pragma unroll
            for (int s = 0; s < SPL; s++) {
                uint32_t a, b;
                remix_lo32_pipes(k0 + x0 + (uint64_t)(s * 32), K, a, b);
                const uint32_t r = (a ^ b) & 0xFFFFu;
#pragma unroll
                for (int t = 0; t < NT; t++) c[s][t] = add_sign_bit(c[s][t], r - T[t], K.two);
            }
        }
    } else {
        for (; i + 2 <= hi; i += 2) {
            const uint64_t k0 = sk[i], k1 = sk[i + 1];
#pragma unroll
            for (int s = 0; s < SPL; s++) {
                const uint64_t x = x0 + (uint64_t)(s * 32);
                const uint32_t r0 = split_r16<ARITH>(k0 + x);
                const uint32_t r1 = split_r16<ARITH>(k1 + x);
#pragma unroll
                for (int t = 0; t < NT; t++) c[s][t] += (r0 < T[t]) + (r1 < T[t]);
            }
        }
        for (; i < hi; i++) {
            const uint64_t k0 = sk[i];
#pragma unroll
            for (int s = 0; s < SPL; s++) {
                const uint32_t r0 = split_r16<ARITH>(k0 + x0 + (uint64_t)(s * 32));
#pragma unroll
                for (int t = 0; t < NT; t++) c[s][t] += (r0 < T[t]);
            }
        }
    }
}

// Quarter split (fanout 4 with m = 4 * unit, every full first-level node): the thresholds are
// k * 16384, so a key's part is p = r16 >> 14. Instead of three compare-and-count chains the lane
// accumulates the moments sum p, sum p^2, sum p^3 (multiply-adds); part counts (u, u, u, u) are the
// only counts with moments (6u, 14u, 36u) because the system matrix [[1,2,3],[1,4,9],[1,8,27]] is
// invertible.
template <int SPL, int ARITH>
__device__ __forceinline__ void moments_range(const uint64_t *__restrict__ sk, uint32_t lo, uint32_t hi, uint64_t x0,
                                              uint32_t (&c)[SPL][3], const PipeK &K) {
    uint32_t i = lo;
    if constexpr (ARITH == 1) {  // part p = bits 14..15 of r, taken as a multiply-high of r & 0xC000 by 2^18
        for (; i < hi; i++) {
            const uint64_t k0 = sk[i];
#pragma unroll
            for (int s = 0; s < SPL; s++) {
                uint32_t a, b;
                remix_lo32_pipes(k0 + x0 + (uint64_t)(s * 32), K, a, b);
                const uint32_t p0 = __umulhi((a ^ b) & 0xC000u, K.c18);
                const uint32_t q0 = p0 * p0;
                c[s][0] += p0;
                c[s][1] += q0;
                c[s][2] += q0 * p0;
            }
        }
    } else {
        for (; i + 2 <= hi; i += 2) {
            const uint64_t k0 = sk[i], k1 = sk[i + 1];
#pragma unroll
            for (int s = 0; s < SPL; s++) {
                const uint64_t x = x0 + (uint64_t)(s * 32);
                const uint32_t p0 = split_r16<ARITH>(k0 + x) >> 14;
                const uint32_t p1 = split_r16<ARITH>(k1 + x) >> 14;
                const uint32_t q0 = p0 * p0, q1 = p1 * p1;
                c[s][0] += p0 + p1;
                c[s][1] += q0 + q1;
                c[s][2] += q0 * p0 + q1 * p1;
            }
        }
        for (; i < hi; i++) {
            const uint64_t k0 = sk[i];
#pragma unroll
            for (int s = 0; s < SPL; s++) {
                const uint32_t p0 = split_r16<ARITH>(k0 + x0 + (uint64_t)(s * 32)) >> 14;
                c[s][0] += p0;
                c[s][1] += p0 * p0;
                c[s][2] += p0 * p0 * p0;
            }
        }
    }
}

// Smallest valid trial index (seed - seed0), or ~0 when `cap` trials were exhausted.
// NT = number of part thresholds compared (1..3); NT = 4 selects the quarter-split moments.
template <int NT, int SPL, int THREADS, int ARITH>
__device__ uint64_t search_seeds(SplitSmem<SPL, THREADS> &sm, uint32_t m, uint64_t seed0, const uint32_t T0,
                                 const uint32_t T1, const uint32_t T2, const uint32_t N0, const uint32_t N1,
                                 const uint32_t N2, int G, uint64_t cap, const PipeK &K) {
    constexpr int kWarps = THREADS / 32, kSeedsPerWarp = 32 * SPL;
    const uint32_t need[3] = {N0, N1, N2};
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int wpg = kWarps / G;  // warps per group
    const int group = warp / wpg, sub = warp % wpg;
    const uint32_t lo = (uint32_t)((uint64_t)m * sub / wpg), hi = (uint32_t)((uint64_t)m * (sub + 1) / wpg);
    const uint32_t per_round = (uint32_t)(kSeedsPerWarp * G);
    for (uint64_t base = 0; base < cap; base += per_round) {
        const uint32_t slot0 = (uint32_t)group * kSeedsPerWarp + lane;  // seed slot s is slot0 + 32 s
        uint32_t c[SPL][3] = {};
        if constexpr (NT == 4) moments_range<SPL, ARITH>(sm.keys, lo, hi, seed0 + base + slot0, c, K);
        else count_range<NT, SPL, ARITH>(sm.keys, lo, hi, seed0 + base + slot0, T0, T1, T2, c, K);
        constexpr int NC = NT == 4 ? 3 : NT;  // counters per seed
        if (wpg > 1) {
#pragma unroll
            for (int s = 0; s < SPL; s++)
#pragma unroll
                for (int t = 0; t < NC; t++) sm.part_counts[warp][s * 32 + lane][t] = c[s][t];
            __syncthreads();
            if (sub == 0) {
#pragma unroll
                for (int s = 0; s < SPL; s++)
#pragma unroll
                    for (int t = 0; t < NC; t++) {
                        uint32_t tot = 0;
                        for (int w = 0; w < wpg; w++) tot += sm.part_counts[warp + w][s * 32 + lane][t];
                        c[s][t] = tot;
                    }
            }
        }
        if (sub == 0) {
#pragma unroll
            for (int s = 0; s < SPL; s++) {
                bool ok = true;
#pragma unroll
                for (int t = 0; t < NC; t++) ok &= c[s][t] == need[t];
                if (ok) atomicMin(&sm.best, slot0 + 32u * s);
            }
        }
        __syncthreads();
        const uint32_t b = sm.best;
        if (b != 0xffffffffu) return base + b < cap ? base + b : ~0ull;  // at most `cap` seeds count
    }
    return ~0ull;
}

// One split node searched and partitioned by the whole block (THREADS threads): the smallest valid
// seed from start_seed[level] on, its code x - start_seed to codes[id], the node's keys permuted in
// place into its parts. Returns (block-uniformly) after the partition's writes are issued; a node
// whose search reaches its trial cap sets kErrTrialLimit and leaves its keys as they were.
// L2: load the node's keys past L1 (needed when another SM may have rewritten them since this SM
// last read those lines, as in the work-queue kernel; the per-level launches start with clean L1s).
template <int SPL, int THREADS, int ARITH, bool L2 = false>
__device__ __forceinline__ void split_node(SplitSmem<SPL, THREADS> &sm, const Node nd, const uint32_t id,
                                           uint64_t *__restrict__ keys, uint64_t *__restrict__ codes,
                                           const uint64_t max_trials, uint32_t *__restrict__ err,
                                           unsigned long long *__restrict__ work,
                                           unsigned long long *__restrict__ kind_work, const int round_div,
                                           const PipeK &K) {
    constexpr int kWarps = THREADS / 32, kSeedsPerWarp = 32 * SPL;
    const uint32_t m = nd.m;
    for (uint32_t i = threadIdx.x; i < m; i += blockDim.x) sm.keys[i] = L2 ? __ldcg(&keys[nd.start + i]) : keys[nd.start + i];

    // Part boundaries as thresholds on the low 16 bits of remix (see header).
    uint32_t T[3] = {65536u, 65536u, 65536u}, need[3] = {m, m, m};
    int NT;
    double p;
    if (nd.kind == kSplit2) {
        NT = 1;
        T[0] = (uint32_t)(((uint64_t)nd.unit * 65536u + m - 1) / m);
        need[0] = nd.unit;
        const double k0 = nd.unit, k1 = m - nd.unit;
        p = sqrt((double)m) / (sqrt(2 * M_PI) * sqrt(k0) * sqrt(k1));
    } else {
        NT = nd.fanout - 1;
        double sp = 1;
        for (int t = 0; t < NT; t++) {
            const uint64_t K = (uint64_t)(t + 1) * nd.unit;
            T[t] = (uint32_t)((K * 65536u + m - 1) / m);
            need[t] = (uint32_t)K;
            sp *= sqrt((double)nd.unit);
        }
        sp *= sqrt((double)(m - (uint32_t)NT * nd.unit));
        p = sqrt((double)m) / (pow(2 * M_PI, NT / 2.0) * sp);
    }
    // Warp groups: aim for a round of ~1/round_div of the expected trials.
    const double expect = 1.0 / p;
    int G = 1;
    while (G < kWarps && (double)(kSeedsPerWarp * G * 2) * (double)round_div <= expect) G <<= 1;
    if (threadIdx.x == 0) sm.best = 0xffffffffu;
    __syncthreads();

    const uint64_t seed0 = start_seed(nd.level);
    // Trial cap: 2^(g+12) is ~2000 expected searches (g ~ log2(0.48 / p)), so only duplicate keys
    // or a caller-set max_trials can reach it.
    uint64_t cap = 1ull << min(nd.g + 12, 40);
    if (max_trials && max_trials < cap) cap = max_trials;
    uint64_t trial;
    const bool quarter = nd.kind == kSplitK && nd.fanout == 4 && m == 4u * nd.unit;
    if (quarter) {
        NT = 4;  // moments: sum p = 6u, sum p^2 = 14u, sum p^3 = 36u
        need[0] = 6u * nd.unit;
        need[1] = 14u * nd.unit;
        need[2] = 36u * nd.unit;
    }
    switch (NT) {
        case 1: trial = search_seeds<1, SPL, THREADS, ARITH>(sm, m, seed0, T[0], T[1], T[2], need[0], need[1], need[2], G, cap, K); break;
        case 2: trial = search_seeds<2, SPL, THREADS, ARITH>(sm, m, seed0, T[0], T[1], T[2], need[0], need[1], need[2], G, cap, K); break;
        case 3: trial = search_seeds<3, SPL, THREADS, ARITH>(sm, m, seed0, T[0], T[1], T[2], need[0], need[1], need[2], G, cap, K); break;
        default: trial = search_seeds<4, SPL, THREADS, ARITH>(sm, m, seed0, T[0], T[1], T[2], need[0], need[1], need[2], G, cap, K); break;
    }
    if (trial == ~0ull) {
        if (threadIdx.x == 0) atomicOr(err, kErrTrialLimit);
        return;
    }
    const uint64_t x = seed0 + trial;

    // Stable partition (counting sort by part, original order inside a part). Each thread owns a
    // contiguous chunk; per-part counts are packed 16 bits per part into one 64-bit word and
    // exclusive-scanned across the block.
    const uint32_t chunk = (m + THREADS - 1) / THREADS;
    const uint32_t lo = min(m, threadIdx.x * chunk), hi = min(m, lo + chunk);
    uint64_t mine = 0;
    for (uint32_t i = lo; i < hi; i++) {
        const uint32_t r = split_r16<ARITH>(sm.keys[i] + x);
        const uint32_t part = (r >= T[0]) + (r >= T[1]) + (r >= T[2]);
        mine += 1ull << (16 * part);
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint64_t incl = mine;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint64_t y = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += y;
    }
    __syncthreads();  // sm.scan reuse
    if (lane == 31) sm.scan[warp] = incl;
    __syncthreads();
    uint64_t before = 0;
    for (int w = 0; w < warp; w++) before += sm.scan[w];
    uint64_t run = before + incl - mine;  // exclusive prefix, packed
    const uint32_t unit = nd.unit;
    for (uint32_t i = lo; i < hi; i++) {
        const uint64_t k = sm.keys[i];
        const uint32_t r = split_r16<ARITH>(k + x);
        const uint32_t part = (r >= T[0]) + (r >= T[1]) + (r >= T[2]);
        const uint32_t dest = part * unit + (uint32_t)((run >> (16 * part)) & 0xFFFF);
        run += 1ull << (16 * part);
        if (dest < m) keys[nd.start + dest] = k;
        else atomicOr(err, kErrInternal);  // unreachable for a valid seed; never write outside the node
    }
    if (threadIdx.x == 0) {
        codes[id] = trial;  // x - start_seed[level]
        atomicAdd(work, (unsigned long long)(trial + 1) * m);
        // useful evaluations by inner loop: 1, 2 or 3 compared thresholds, or quarter-split moments
        atomicAdd(&kind_work[quarter ? 3 : NT - 1], (unsigned long long)(trial + 1) * m);
    }
}

} // namespace shg
