// Device kernels of the construction pipeline other than the leaf searches:
//   key hashing (SpookyHash V2), bucket partition (remap128 bucketing + per-bucket sort by the
//   first hash half), RecSplit split-seed search with the stable partition, Golomb-Rice encoding.
#include <cstdint>
#include <cuda_runtime.h>
#include "shg_common.cuh"
#include "shg_internal.h"

namespace shg {

// ------------------------------------------------------------------------------ hashing
__global__ void k_spooky_u64(const uint64_t *__restrict__ keys, uint64_t n, uint64_t *__restrict__ first,
                             uint64_t *__restrict__ second) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        uint64_t f, s;
        spooky128_u64(keys[i], 0, f, s);
        first[i] = f;
        second[i] = s;
    }
}

__global__ void k_spooky_strings(const uint8_t *__restrict__ bytes, const uint64_t *__restrict__ offsets, uint64_t n,
                                 uint64_t *__restrict__ first, uint64_t *__restrict__ second) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t b = offsets[i], e = offsets[i + 1];
        uint64_t f, s;
        spooky128(bytes + b, e - b, 0, f, s);
        first[i] = f;
        second[i] = s;
    }
}

static int grid_for(uint64_t n, int threads) {
    uint64_t g = (n + threads - 1) / threads;
    if (g > 148ull * 32) g = 148ull * 32;
    return g < 1 ? 1 : (int)g;
}

void launch_spooky_u64(const uint64_t *keys, uint64_t n, uint64_t *first, uint64_t *second, cudaStream_t s) {
    if (n) k_spooky_u64<<<grid_for(n, 256), 256, 0, s>>>(keys, n, first, second);
}
void launch_spooky_strings(const uint8_t *bytes, const uint64_t *offsets, uint64_t n, uint64_t *first, uint64_t *second,
                           cudaStream_t s) {
    if (n) k_spooky_strings<<<grid_for(n, 256), 256, 0, s>>>(bytes, offsets, n, first, second);
}

// ------------------------------------------------------------------------------ partition
// Bucket of a key: remap128(first, nbuckets) (ShockHash.h:297, Sorter.hpp:248); monotone in
// `first`, so sorting by `first` globally equals bucketing followed by a sort inside each bucket.
// bucket = remap128(first, nb_map) - b0 must fall in [0, nb): a shard of a larger structure owns
// the buckets [b0, b0 + nb) of nb_map; a key outside them sets kErrArg and is skipped.
__global__ void k_bucket_count(const uint64_t *__restrict__ first, uint64_t n, uint64_t nb, uint64_t nb_map, uint64_t b0,
                               uint32_t *__restrict__ counts, uint32_t *__restrict__ err) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t b = remap128(first[i], nb_map) - b0;
        if (b >= nb) {
            atomicOr(err, kErrArg);
            continue;
        }
        atomicAdd(&counts[b], 1u);
    }
}

// Exclusive scan of the bucket counts into bucket_size_acc (one block, sequential over chunks).
__global__ void k_scan_counts(const uint32_t *__restrict__ counts, uint64_t nb, uint64_t *__restrict__ acc,
                              uint32_t *__restrict__ cursor, uint32_t *__restrict__ maxsz) {
    __shared__ uint64_t warp_sums[32];
    __shared__ uint64_t carry;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t local_max = 0;
    for (uint64_t base = 0; base < nb; base += blockDim.x) {
        const uint64_t i = base + threadIdx.x;
        const uint64_t v = i < nb ? counts[i] : 0;
        local_max = max(local_max, (uint32_t)v);
        uint64_t x = v;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            uint64_t y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += y;
        }
        if (lane == 31) warp_sums[warp] = x;
        __syncthreads();
        if (warp == 0) {
            uint64_t w = lane < (int)(blockDim.x >> 5) ? warp_sums[lane] : 0;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                uint64_t y = __shfl_up_sync(0xffffffffu, w, o);
                if (lane >= o) w += y;
            }
            warp_sums[lane] = w;
        }
        __syncthreads();
        const uint64_t excl = carry + (warp ? warp_sums[warp - 1] : 0) + x - v;
        if (i < nb) {
            acc[i] = excl;
            cursor[i] = (uint32_t)excl;
        }
        __syncthreads();
        if (threadIdx.x == blockDim.x - 1) carry = excl + v;
        __syncthreads();
    }
    if (threadIdx.x == 0) acc[nb] = carry;
    atomicMax(maxsz, local_max);
}

__global__ void k_bucket_scatter(const uint64_t *__restrict__ first, uint64_t n, uint64_t nb, uint64_t nb_map,
                                 uint64_t b0, uint32_t *__restrict__ cursor, uint64_t *__restrict__ sfirst,
                                 uint32_t *__restrict__ sidx, uint64_t idx_base) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t f = first[i];
        const uint64_t b = remap128(f, nb_map) - b0;
        if (b >= nb) continue;  // reported by k_bucket_count
        const uint32_t pos = atomicAdd(&cursor[b], 1u);
        sfirst[pos] = f;
        sidx[pos] = (uint32_t)(idx_base + i);
    }
}

// One block per bucket: bitonic sort of (first, input index) in shared memory, then gather the
// second halves in that order (Sorter.hpp:15-36 sorts by `first` and keeps `second`). Equal
// `first` values keep input order, as in the oracle's stable sort (the reference's ips2ra leaves
// their order unspecified).
constexpr int kSortThreads = 512;
constexpr int kSortCap = 4096;  // power of two >= kMaxBucket
__global__ void __launch_bounds__(kSortThreads) k_bucket_sort(const uint64_t *__restrict__ acc, uint64_t nb,
                                                              const uint64_t *__restrict__ sfirst,
                                                              const uint32_t *__restrict__ sidx,
                                                              const uint64_t *__restrict__ second,
                                                              uint64_t *__restrict__ keys) {
    extern __shared__ uint8_t smem_raw[];
    uint64_t *kf = (uint64_t *)smem_raw;
    uint32_t *ki = (uint32_t *)(kf + kSortCap);
    for (uint64_t b = blockIdx.x; b < nb; b += gridDim.x) {
        const uint64_t beg = acc[b];
        const uint32_t m = (uint32_t)(acc[b + 1] - beg);
        if (m == 0) continue;
        uint32_t cap = 1;
        while (cap < m) cap <<= 1;
        for (uint32_t i = threadIdx.x; i < cap; i += blockDim.x) {
            kf[i] = i < m ? sfirst[beg + i] : ~0ull;
            ki[i] = i < m ? sidx[beg + i] : 0xffffffffu;
        }
        __syncthreads();
        for (uint32_t k = 2; k <= cap; k <<= 1) {
            for (uint32_t j = k >> 1; j > 0; j >>= 1) {
                for (uint32_t i = threadIdx.x; i < cap; i += blockDim.x) {
                    const uint32_t p = i ^ j;
                    if (p > i) {
                        const bool up = (i & k) == 0;
                        const uint64_t a = kf[i], c = kf[p];
                        const uint32_t ai = ki[i], ci = ki[p];
                        const bool gt = a > c || (a == c && ai > ci);
                        if (gt == up) {
                            kf[i] = c; kf[p] = a;
                            ki[i] = ci; ki[p] = ai;
                        }
                    }
                }
                __syncthreads();
            }
        }
        for (uint32_t i = threadIdx.x; i < m; i += blockDim.x) keys[beg + i] = second[ki[i]];
        __syncthreads();
    }
}

// Retrieval input without the keys of size-1 children (they get no retrieval bit,
// ShockHash.h:480,514,547): out[i - #singles before i] = in[i] for every non-single position i.
__global__ void k_compact_ribbon(const uint64_t *__restrict__ keys, const uint8_t *__restrict__ bits, uint64_t n,
                                 const uint64_t *__restrict__ singles, uint64_t nsingles, uint64_t *__restrict__ out_keys,
                                 uint8_t *__restrict__ out_bits) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        uint64_t lo = 0, hi = nsingles;  // count of singles < i
        while (lo < hi) {
            const uint64_t mid = (lo + hi) >> 1;
            if (singles[mid] < i) lo = mid + 1; else hi = mid;
        }
        if (lo < nsingles && singles[lo] == i) continue;
        if (out_keys) out_keys[i - lo] = keys[i];  // either part may be compacted on its own
        if (out_bits) out_bits[i - lo] = bits[i];
    }
}

void launch_compact_ribbon(const uint64_t *keys, const uint8_t *bits, uint64_t n, const uint64_t *singles,
                           uint64_t nsingles, uint64_t *out_keys, uint8_t *out_bits, cudaStream_t s) {
    if (n) k_compact_ribbon<<<grid_for(n, 256), 256, 0, s>>>(keys, bits, n, singles, nsingles, out_keys, out_bits);
}

void launch_bucket_count(const uint64_t *first, uint64_t n, uint64_t nb, uint64_t nb_map, uint64_t b0, uint32_t *counts,
                         uint32_t *err, cudaStream_t s) {
    cudaMemsetAsync(counts, 0, nb * sizeof(uint32_t), s);
    if (n) k_bucket_count<<<grid_for(n, 256), 256, 0, s>>>(first, n, nb, nb_map, b0, counts, err);
}
void launch_scan_counts(const uint32_t *counts, uint64_t nb, uint64_t *acc, uint32_t *cursor, uint32_t *maxsz,
                        cudaStream_t s) {
    cudaMemsetAsync(maxsz, 0, sizeof(uint32_t), s);
    k_scan_counts<<<1, 1024, 0, s>>>(counts, nb, acc, cursor, maxsz);
}
void launch_bucket_scatter(const uint64_t *first, uint64_t n, uint64_t nb, uint64_t nb_map, uint64_t b0, uint32_t *cursor,
                           uint64_t *sfirst, uint32_t *sidx, uint64_t idx_base, cudaStream_t s) {
    if (n) k_bucket_scatter<<<grid_for(n, 256), 256, 0, s>>>(first, n, nb, nb_map, b0, cursor, sfirst, sidx, idx_base);
}
void launch_bucket_sort(const uint64_t *acc, uint64_t nb, const uint64_t *sfirst, const uint32_t *sidx,
                        const uint64_t *second, uint64_t *keys, cudaStream_t s) {
    const size_t smem = kSortCap * (sizeof(uint64_t) + sizeof(uint32_t));
    cudaFuncSetAttribute(k_bucket_sort, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    const uint64_t grid = nb < 148ull * 8 ? nb : 148ull * 8;
    k_bucket_sort<<<(int)grid, kSortThreads, smem, s>>>(acc, nb, sfirst, sidx, second, keys);
}

} // namespace shg
