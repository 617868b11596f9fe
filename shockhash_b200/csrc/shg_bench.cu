// Measurement utilities (not part of the reference's interface):
//  * the seeded key generators the benchmark configurations name (std::mt19937_64), shared by the
//    CPU and GPU runs so both build from the same keys;
//  * the integer-pipe peaks of the searches: the arithmetic of each search kernel's dominant inner
//    loop (split: remix to 16 bits, quarter-split part, moment sums; original leaf: remix, two
//    fastrange32 cells, half masks; bipartite leaf: remix, fastrange64, mask), two seeds per lane,
//    on register-resident operands with no memory traffic. Their evaluations per second are the
//    denominators of the search kernels' roofline fractions.
#include <algorithm>
#include <cstdint>
#include <random>
#include <thread>
#include <vector>
#include <cuda_runtime.h>
#include "shg.h"
#include "shg_common.cuh"
#include "shg_internal.h"

namespace {

constexpr int kPeakThreads = 256;

// The arithmetic of the split kernel's dominant loop (quarter splits): remix to 16 bits, part
// p = r >> 14, moments sum p, sum p^2, sum p^3; two seeds per key pair.
__global__ void __launch_bounds__(kPeakThreads) k_int_peak(uint64_t iters, uint32_t T0, uint32_t T1, uint32_t T2,
                                                           unsigned long long *sink) {
    const uint64_t tid = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    uint64_t k0 = shg::remix(tid * 0x9E3779B97F4A7C15ULL), k1 = shg::remix(k0);
    const uint64_t x0 = 0x643e521ddbd2be98ULL + tid;
    uint32_t c0 = 0, c1 = 0, c2 = 0, d0 = 0, d1 = 0, d2 = 0;
    for (uint64_t i = 0; i < iters; i++) {
        const uint32_t p0 = shg::remix_low16(k0 + x0 + i) >> 14;
        const uint32_t p1 = shg::remix_low16(k1 + x0 + i) >> 14;
        const uint32_t q0 = p0 * p0, q1 = p1 * p1;
        c0 += p0; c1 += q0; c2 += q0 * p0;
        d0 += p1; d1 += q1; d2 += q1 * p1;
    }
    sink[tid] = c0 ^ c1 ^ c2 ^ d0 ^ d1 ^ d2 ^ T0 ^ T1 ^ T2;  // every thread's result is stored: no loop can fold
}

// The arithmetic of the split kernel's compare-and-count loop (fanout-2 and uneven nodes): remix to
// 16 bits, one count per part threshold (NT of them); two seeds per key pair, as k_int_peak.
template <int NT>
__global__ void __launch_bounds__(kPeakThreads) k_int_peak_cmp(uint64_t iters, uint32_t T0, uint32_t T1, uint32_t T2,
                                                               unsigned long long *sink) {
    const uint64_t tid = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    uint64_t k0 = shg::remix(tid * 0x9E3779B97F4A7C15ULL), k1 = shg::remix(k0);
    const uint64_t x0 = 0x643e521ddbd2be98ULL + tid;
    const uint32_t T[3] = {T0, T1, T2};
    uint32_t c[2][3] = {};
    for (uint64_t i = 0; i < iters; i++) {
        const uint32_t r0 = shg::remix_low16(k0 + x0 + i);
        const uint32_t r1 = shg::remix_low16(k1 + x0 + i);
#pragma unroll
        for (int t = 0; t < NT; t++) {
            c[0][t] += r0 < T[t];
            c[1][t] += r1 < T[t];
        }
    }
    sink[tid] = c[0][0] ^ c[0][1] ^ c[0][2] ^ c[1][0] ^ c[1][1] ^ c[1][2];
}

// The same two loops with remix split between the integer and multiply pipes (the split kernel's
// arithmetic option 1): quarter moments (NT = 4) or compare-and-count against NT thresholds.
template <int NT>
__global__ void __launch_bounds__(kPeakThreads) k_int_peak_pipes(uint64_t iters, uint32_t T0, uint32_t T1, uint32_t T2,
                                                                 const shg::PipeK K, unsigned long long *sink) {
    const uint64_t tid = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    uint64_t k0 = shg::remix(tid * 0x9E3779B97F4A7C15ULL), k1 = shg::remix(k0);
    const uint64_t x0 = 0x643e521ddbd2be98ULL + tid;
    const uint32_t T[3] = {T0, T1, T2};
    uint32_t c[2][3] = {};
    for (uint64_t i = 0; i < iters; i++) {
        uint32_t a0, b0, a1, b1;
        shg::remix_lo32_pipes(k0 + x0 + i, K, a0, b0);
        shg::remix_lo32_pipes(k1 + x0 + i, K, a1, b1);
        if (NT == 4) {
            const uint32_t p0 = __umulhi((a0 ^ b0) & 0xC000u, K.c18), p1 = __umulhi((a1 ^ b1) & 0xC000u, K.c18);
            const uint32_t q0 = p0 * p0, q1 = p1 * p1;
            c[0][0] += p0; c[0][1] += q0; c[0][2] += q0 * p0;
            c[1][0] += p1; c[1][1] += q1; c[1][2] += q1 * p1;
        } else {
            const uint32_t r0 = (a0 ^ b0) & 0xFFFFu, r1 = (a1 ^ b1) & 0xFFFFu;
#pragma unroll
            for (int t = 0; t < NT; t++) {
                c[0][t] = shg::add_sign_bit(c[0][t], r0 - T[t], K.two);
                c[1][t] = shg::add_sign_bit(c[1][t], r1 - T[t], K.two);
            }
        }
    }
    sink[tid] = c[0][0] ^ c[0][1] ^ c[0][2] ^ c[1][0] ^ c[1][1] ^ c[1][2];
}

// The split loops under SIMDShockHash's split hash (fmix32 of the xor-folded halves): quarter
// moments (NT = 4) or compare-and-count against NT thresholds; two seeds per key pair.
template <int NT>
__global__ void __launch_bounds__(kPeakThreads) k_int_peak_simd(uint64_t iters, uint32_t T0, uint32_t T1, uint32_t T2,
                                                                unsigned long long *sink) {
    const uint64_t tid = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    uint64_t k0 = shg::remix(tid * 0x9E3779B97F4A7C15ULL), k1 = shg::remix(k0);
    const uint64_t x0 = 0x643e521ddbd2be98ULL + tid;
    const uint32_t T[3] = {T0, T1, T2};
    uint32_t c[2][3] = {};
    for (uint64_t i = 0; i < iters; i++) {
        const uint32_t r0 = shg::simd_split_low16(k0 + x0 + i), r1 = shg::simd_split_low16(k1 + x0 + i);
        if (NT == 4) {
            const uint32_t p0 = r0 >> 14, p1 = r1 >> 14;
            const uint32_t q0 = p0 * p0, q1 = p1 * p1;
            c[0][0] += p0; c[0][1] += q0; c[0][2] += q0 * p0;
            c[1][0] += p1; c[1][1] += q1; c[1][2] += q1 * p1;
        } else {
#pragma unroll
            for (int t = 0; t < NT; t++) {
                c[0][t] += r0 < T[t];
                c[1][t] += r1 < T[t];
            }
        }
    }
    sink[tid] = c[0][0] ^ c[0][1] ^ c[0][2] ^ c[1][0] ^ c[1][1] ^ c[1][2];
}

// The original leaf search's coverage rounds as the leaf kernel runs them, alone: a leaf of h1 + h2
// keys in shared memory, lanes on consecutive seeds, two seeds per lane per key read (full 64-bit
// remix, both cells by fastrange32 on its halves, one bit each into two 32-bit half masks), the
// masks compared after each round; no pseudoforest tests. `iters` key reads per thread, rounded up
// to whole rounds (the caller counts the rounded number).
__global__ void __launch_bounds__(kPeakThreads) k_int_peak_sh1(uint64_t iters, uint32_t h1, uint32_t h2,
                                                               unsigned long long *sink) {
    __shared__ uint64_t keys[64];
    for (int i = threadIdx.x; i < 64; i += blockDim.x) keys[i] = shg::remix(0x9E3779B97F4A7C15ULL * (i + 1) + blockIdx.x);
    __syncthreads();
    const uint32_t m = h1 + h2, lane = threadIdx.x & 31;
    const uint32_t all1 = (1u << h1) - 1, all2 = (1u << h2) - 1;
    uint64_t base = 0x643e521ddbd2be98ULL + (blockIdx.x * (uint64_t)blockDim.x + (threadIdx.x & ~31u)) * 64 * iters;
    uint32_t hits = 0;
    for (uint64_t done = 0; done < iters; done += m, base += 64) {
        uint32_t c1m[2] = {0, 0}, c2m[2] = {0, 0};
        for (uint32_t k = 0; k < m; k++) {
            const uint64_t key = keys[k];
#pragma unroll
            for (int t = 0; t < 2; t++) {
                const uint64_t r = shg::remix(key + base + lane + 32 * t);
                c1m[t] |= 1u << shg::fastrange32((uint32_t)r, h1);
                c2m[t] |= 1u << shg::fastrange32((uint32_t)(r >> 32), h2);
            }
        }
#pragma unroll
        for (int t = 0; t < 2; t++) hits += c1m[t] == all1 && c2m[t] == all2;
    }
    sink[blockIdx.x * (uint64_t)blockDim.x + threadIdx.x] = hits;
}

// The arithmetic of the bipartite leaf search's raw-seed loop: remix, fastrange64 to the half
// table (as the kernel computes it for a range below 2^32), one bit into a 64-bit mask; two seeds
// per lane.
__global__ void __launch_bounds__(kPeakThreads) k_int_peak_sh2(uint64_t iters, uint64_t half, unsigned long long *sink) {
    const uint64_t tid = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    uint64_t k0 = shg::remix(tid * 0x9E3779B97F4A7C15ULL), k1 = shg::remix(k0);
    const uint64_t x0 = 0x643e521ddbd2be98ULL + tid;
    uint64_t a0 = 0, a1 = 0;
    for (uint64_t i = 0; i < iters; i++) {
        a0 |= 1ull << shg::fastrange64_32(shg::remix(k0 + x0 + i), (uint32_t)half);
        a1 |= 1ull << shg::fastrange64_32(shg::remix(k1 + x0 + i), (uint32_t)half);
    }
    sink[tid] = a0 ^ a1;
}

} // namespace

extern "C" {

// n keys from std::mt19937_64(seed), duplicates removed by drawing replacements (the reference
// loops forever on duplicate keys), in draw order.
void shg_keys_mt19937_64(uint64_t seed, uint64_t n, uint64_t *out) {
    std::mt19937_64 rng(seed);
    for (uint64_t i = 0; i < n; i++) out[i] = rng();
    std::vector<uint64_t> sorted(out, out + n);
    std::sort(sorted.begin(), sorted.end());
    if (std::adjacent_find(sorted.begin(), sorted.end()) == sorted.end()) return;
    std::vector<uint64_t> seen;
    seen.reserve(n);
    std::vector<uint64_t> tmp(out, out + n);
    std::sort(tmp.begin(), tmp.end());
    // replace later occurrences of a duplicate by fresh draws that are not present
    std::vector<uint64_t> uniq;
    uniq.reserve(n);
    std::vector<char> keep(n, 1);
    {
        std::vector<std::pair<uint64_t, uint64_t>> vi(n);
        for (uint64_t i = 0; i < n; i++) vi[i] = {out[i], i};
        std::sort(vi.begin(), vi.end());
        for (uint64_t i = 1; i < n; i++)
            if (vi[i].first == vi[i - 1].first) keep[vi[i].second] = 0;
    }
    for (uint64_t i = 0; i < n; i++) {
        while (!keep[i]) {
            const uint64_t v = rng();
            if (!std::binary_search(tmp.begin(), tmp.end(), v)) {
                out[i] = v;
                keep[i] = 1;
                tmp.insert(std::upper_bound(tmp.begin(), tmp.end(), v), v);
            }
        }
    }
}

// Request keys of the serving stream: out[j] = remix(seed ^ (j * 0x9E3779B97F4A7C15)), j < n. Each
// step is a bijection of 64-bit words, so the n keys are distinct with no check; host threads each
// fill a contiguous range.
void shg_keys_mix(uint64_t seed, uint64_t n, uint64_t *out, int threads) {
    const uint64_t T = (uint64_t)std::max(1, std::min(threads, 64));
    const uint64_t chunk = (n + T - 1) / T;
    auto fill = [&](uint64_t a, uint64_t b) {
        for (uint64_t j = a; j < b; j++) out[j] = shg::remix(seed ^ (j * 0x9E3779B97F4A7C15ULL));
    };
    if (T == 1 || n < (1u << 16)) {
        fill(0, n);
        return;
    }
    std::vector<std::thread> pool;
    for (uint64_t t = 0; t < T; t++) {
        const uint64_t a = std::min(n, t * chunk), b = std::min(n, a + chunk);
        if (a < b) pool.emplace_back(fill, a, b);
    }
    for (auto &th : pool) th.join();
}

// Integer-pipe peak: evaluations per second of the split search arithmetic on `device`.
int shg_int_peak(int device, uint64_t iters, double *evals_per_s, double *ms_out) {
    if (cudaSetDevice(device) != cudaSuccess) return SHG_ERR_CUDA;
    cudaDeviceProp prop;
    cudaGetDeviceProperties(&prop, device);
    const int blocks = prop.multiProcessorCount * 8;
    unsigned long long *sink;
    if (cudaMalloc(&sink, (size_t)blocks * kPeakThreads * 8) != cudaSuccess) return SHG_ERR_OOM;  // one result per thread
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    const uint32_t T0 = 16384, T1 = 32768, T2 = 49152;
    k_int_peak<<<blocks, kPeakThreads>>>(iters / 16 + 1, T0, T1, T2, sink);  // warm-up
    cudaEventRecord(a);
    k_int_peak<<<blocks, kPeakThreads>>>(iters, T0, T1, T2, sink);
    cudaEventRecord(b);
    cudaEventSynchronize(b);
    float ms = 0;
    cudaEventElapsedTime(&ms, a, b);
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    cudaFree(sink);
    if (cudaGetLastError() != cudaSuccess) return SHG_ERR_CUDA;
    *evals_per_s = 2.0 * (double)iters * blocks * kPeakThreads / (ms * 1e-3);
    if (ms_out) *ms_out = ms;
    return SHG_OK;
}

// Integer-pipe peak of one search's inner loop (0 = split quarter moments, 1 = original leaf,
// 2 = bipartite leaf hashing, 3..5 = split compare-and-count with 1..3 thresholds, 6..8 = bipartite
// candidate scan, pair filter and pseudoforest edges, 9..12 = kinds 0 and 3..5 with the split
// kernel's pipe-split arithmetic, 13..15 = kinds 6..8 for leaves of more than 64 keys, 16..19 = kinds
// 0 and 3..5 under SIMDShockHash's split hash, 20 = kind 13 with the other form of the mask test).
int shg_int_peak_kind(int device, int kind, uint64_t iters, double *evals_per_s, double *ms_out) {
    if (kind == 0) return shg_int_peak(device, iters, evals_per_s, ms_out);
    if (kind < 1 || kind > 20) return SHG_ERR_ARG;
    if (cudaSetDevice(device) != cudaSuccess) return SHG_ERR_CUDA;
    cudaDeviceProp prop;
    cudaGetDeviceProperties(&prop, device);
    const int blocks = prop.multiProcessorCount * 8;
    unsigned long long *sink;
    if (cudaMalloc(&sink, (size_t)blocks * kPeakThreads * 8) != cudaSuccess) return SHG_ERR_OOM;  // one result per thread
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    for (int rep = 0; rep < 2; rep++) {  // warm-up, then the timed run
        const uint64_t it = rep ? iters : iters / 16 + 1;
        if (rep) cudaEventRecord(a);
        if (kind == 1)
            k_int_peak_sh1<<<blocks, kPeakThreads>>>(it, 20, 20, sink);
        else if (kind == 2)
            k_int_peak_sh2<<<blocks, kPeakThreads>>>(it, 32, sink);
        else if (kind == 3)
            k_int_peak_cmp<1><<<blocks, kPeakThreads>>>(it, 50331, 65536, 65536, sink);
        else if (kind == 4)
            k_int_peak_cmp<2><<<blocks, kPeakThreads>>>(it, 21846, 43691, 65536, sink);
        else if (kind == 5)
            k_int_peak_cmp<3><<<blocks, kPeakThreads>>>(it, 16384, 32768, 49152, sink);
        else if (kind <= 8)  // the bipartite leaf's scan, pair filter and pseudoforest loops (64 edges per iteration)
            shg::launch_sh2_op_peak(kind - 6, blocks, kind == 8 ? it / 64 + 1 : it, sink);
        else if (kind == 16)
            k_int_peak_simd<4><<<blocks, kPeakThreads>>>(it, 16384, 32768, 49152, sink);
        else if (kind == 17)
            k_int_peak_simd<1><<<blocks, kPeakThreads>>>(it, 50331, 65536, 65536, sink);
        else if (kind == 18)
            k_int_peak_simd<2><<<blocks, kPeakThreads>>>(it, 21846, 43691, 65536, sink);
        else if (kind == 19)
            k_int_peak_simd<3><<<blocks, kPeakThreads>>>(it, 16384, 32768, 49152, sink);
        else if (kind == 20)
            shg::launch_sh2_op_peak(6, blocks, it, sink);
        else if (kind >= 13)  // the same for leaves of more than 64 keys (100 edges per iteration)
            shg::launch_sh2_op_peak(kind - 10, blocks, kind == 15 ? it / 100 + 1 : it, sink);
        else {  // 9: quarter moments, 10..12: 1..3 thresholds, with the split kernel's pipe-split arithmetic
            const shg::PipeK K{4u, 32u, 1u << 18, 2u};
            if (kind == 9) k_int_peak_pipes<4><<<blocks, kPeakThreads>>>(it, 16384, 32768, 49152, K, sink);
            else if (kind == 10) k_int_peak_pipes<1><<<blocks, kPeakThreads>>>(it, 50331, 65536, 65536, K, sink);
            else if (kind == 11) k_int_peak_pipes<2><<<blocks, kPeakThreads>>>(it, 21846, 43691, 65536, K, sink);
            else k_int_peak_pipes<3><<<blocks, kPeakThreads>>>(it, 16384, 32768, 49152, K, sink);
        }
        if (rep) cudaEventRecord(b);
    }
    cudaEventSynchronize(b);
    float ms = 0;
    cudaEventElapsedTime(&ms, a, b);
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    cudaFree(sink);
    if (cudaGetLastError() != cudaSuccess) return SHG_ERR_CUDA;
    double per_iter = 2.0;
    uint64_t timed_iters = iters;
    if (kind >= 6 && kind <= 8) {
        per_iter = shg::sh2_op_peak_per_iter(kind - 6);
        if (kind == 8) timed_iters = iters / 64 + 1;
    } else if (kind >= 13 && kind <= 15) {
        per_iter = shg::sh2_op_peak_per_iter(kind - 10);
        if (kind == 15) timed_iters = iters / 100 + 1;
    } else if (kind == 20) {
        per_iter = shg::sh2_op_peak_per_iter(6);
    } else if (kind == 1) {
        timed_iters = (iters + 39) / 40 * 40;  // whole rounds of the 40-key leaf
    }
    *evals_per_s = per_iter * (double)timed_iters * blocks * kPeakThreads / (ms * 1e-3);
    if (ms_out) *ms_out = ms;
    return SHG_OK;
}

} // extern "C"
