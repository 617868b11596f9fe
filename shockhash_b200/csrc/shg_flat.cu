// ShockHash2Flat<k> construction (include/ShockHash2Flat.h:37-302) on the device.
//
//   MurmurHash64 of every key (ShockHash2Flat.h:74-79)
//   -> per threshold layer (:86-122): bucket = fastrange32(low32, buckets), threshold = high32;
//      counting sort by bucket, then a block per bucket sorts it by hash (threshold order) and
//      makes flushBucket's decision (:204-233): the compact threshold, the keys bumped to the next
//      layer and the bucket's free slots; scans then emit free positions and bumped keys in bucket
//      order. Layer 1 re-mixes the bumped keys (:96-100).
//   -> fallback ShockHash2<k> over to_string(mhc) of the keys bumped from the last layer (:124-128),
//      a nested device build; free positions of the fallback keys (:129-146)
//   -> every key's bucket (evaluateKPerfect, :280-301), keys grouped k per bucket in input order
//   -> one bipartite leaf search per bucket (:160-168, batched leaf kernel), seeds packed with the
//      thresholds (:173-185), seeds >= 2^SEED_BITS or 0 kept in a fallback map.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <map>
#include <string>
#include <vector>
#include <cuda_runtime.h>
#include "shg.h"
#include "shg_common.cuh"
#include "shg_internal.h"

namespace shg {

// ---------------------------------------------------------------- constants of ShockHash2Flat<k>
FlatConsts flat_consts(uint32_t k) {
    FlatConsts c;
    c.k = k;
    uint32_t lg = 0;
    while ((2u << lg) <= k) lg++;  // integer_log2_floor(k)
    c.threshold_bits = lg - 1;      // ShockHash2Flat.h:41
    c.threshold_range = 1u << c.threshold_bits;
    c.seed_bits = (uint32_t)std::ceil(0.442 * k - 0.2);  // :44
    // _fill_mapping (ShockHash2Flat.h:16-35)
    const uint64_t one_third = 0xFFFFFFFFull / 3;
    c.mapping.assign(c.threshold_range, 0);
    if (c.threshold_range == 2) {
        c.mapping[0] = 0;
        c.mapping[1] = 0xFFFFFFFFu;
    } else if (c.threshold_range > 2) {
        c.mapping[0] = 0;
        c.mapping[1] = (uint32_t)one_third;
        const uint64_t interp = c.threshold_range - 3;
        for (uint64_t i = 0; i < interp; i++) c.mapping[2 + i] = (uint32_t)(2 * one_third + one_third * i / interp);
        c.mapping[c.threshold_range - 1] = 0xFFFFFFFFu;
    }
    return c;
}

namespace {

constexpr int kFlatSortThreads = 256;
constexpr int kFlatSortCap = 1024;  // keys per layer bucket held in shared memory

__global__ void k_murmur_strings(const uint8_t *__restrict__ bytes, const uint64_t *__restrict__ offsets, uint64_t n,
                                 uint64_t *__restrict__ out) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        out[i] = murmur64a(bytes + offsets[i], offsets[i + 1] - offsets[i], kMurmurSeed);
}

// Layer bucket of each key (re-mixing first on layers after the first), counted.
__global__ void k_flat_count(uint64_t *__restrict__ mhc, uint64_t n, uint32_t nb, bool rehash, uint32_t *__restrict__ counts) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        uint64_t h = mhc[i];
        if (rehash) {
            h = remix(h);
            mhc[i] = h;
        }
        atomicAdd(&counts[fastrange32((uint32_t)h, nb)], 1u);
    }
}

__global__ void k_flat_scatter(const uint64_t *__restrict__ mhc, uint64_t n, uint32_t nb, uint32_t *__restrict__ cursor,
                               uint64_t *__restrict__ out) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t h = mhc[i];
        out[atomicAdd(&cursor[fastrange32((uint32_t)h, nb)], 1u)] = h;
    }
}

__device__ __forceinline__ uint32_t compact_threshold(uint32_t t, const uint32_t *mapping, uint32_t range) {
    for (uint32_t i = 0; i < range; i++)  // compact_threshold (ShockHash2Flat.h:194-202)
        if (t <= mapping[i]) return i;
    return mapping[range - 1];
}

// One block per layer bucket: sort by hash (= by threshold, then low half), then flushBucket.
__global__ void __launch_bounds__(kFlatSortThreads) k_flat_sort_flush(uint64_t *__restrict__ keys, const uint64_t *__restrict__ acc,
                                                                     uint32_t nb, uint32_t k, const uint32_t *__restrict__ mapping,
                                                                     uint32_t range, uint64_t layer_base, uint8_t *__restrict__ thr_out,
                                                                     uint64_t *__restrict__ free_cnt, uint64_t *__restrict__ bump_cnt,
                                                                     uint32_t *__restrict__ bump_first, uint32_t *__restrict__ err) {
    __shared__ uint64_t sk[kFlatSortCap];
    for (uint32_t b = blockIdx.x; b < nb; b += gridDim.x) {
        const uint64_t beg = acc[b];
        const uint32_t s = (uint32_t)(acc[b + 1] - beg);
        if (s > kFlatSortCap) {
            if (threadIdx.x == 0) atomicOr(err, kErrBucket);
            continue;
        }
        uint32_t cap = 1;
        while (cap < s) cap <<= 1;
        for (uint32_t i = threadIdx.x; i < cap; i += blockDim.x) sk[i] = i < s ? keys[beg + i] : ~0ull;
        __syncthreads();
        for (uint32_t kk = 2; kk <= cap; kk <<= 1)
            for (uint32_t j = kk >> 1; j > 0; j >>= 1) {
                for (uint32_t i = threadIdx.x; i < cap; i += blockDim.x) {
                    const uint32_t p = i ^ j;
                    if (p > i) {
                        const uint64_t a = sk[i], c = sk[p];
                        if ((a > c) == ((i & kk) == 0)) {
                            sk[i] = c;
                            sk[p] = a;
                        }
                    }
                }
                __syncthreads();
            }
        for (uint32_t i = threadIdx.x; i < s; i += blockDim.x) keys[beg + i] = sk[i];
        if (threadIdx.x == 0) {
            uint32_t t;
            uint64_t fr, bu, first;
            if (s <= k) {
                t = range - 1;
                fr = k - s;
                bu = 0;
                first = s;
            } else {
                const uint32_t last_t = compact_threshold((uint32_t)(sk[k - 1] >> 32), mapping, range);
                const uint32_t first_b = compact_threshold((uint32_t)(sk[k] >> 32), mapping, range);
                t = last_t - (first_b == last_t ? 1u : 0u);
                const uint32_t u = mapping[t];
                uint32_t p = 0;  // first key whose threshold exceeds the stored one (sorted ascending)
                while (p < s && (uint32_t)(sk[p] >> 32) <= u) p++;
                first = p;
                bu = s - p;
                fr = p < k ? k - p : 0;
            }
            thr_out[layer_base + b] = (uint8_t)t;
            free_cnt[b] = fr;
            bump_cnt[b] = bu;
            bump_first[b] = (uint32_t)first;
        }
        __syncthreads();
    }
}

// Free positions (bucket id, repeated per free slot) and bumped keys, both in bucket order.
__global__ void k_flat_emit(const uint64_t *__restrict__ keys, const uint64_t *__restrict__ acc, uint32_t nb,
                            uint64_t layer_base, const uint64_t *__restrict__ free_cnt, const uint64_t *__restrict__ free_off,
                            const uint64_t *__restrict__ bump_cnt, const uint64_t *__restrict__ bump_off,
                            const uint32_t *__restrict__ bump_first, uint64_t *__restrict__ free_out,
                            uint64_t *__restrict__ bump_out) {
    for (uint64_t b = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; b < nb; b += (uint64_t)gridDim.x * blockDim.x) {
        for (uint64_t j = 0; j < free_cnt[b]; j++) free_out[free_off[b] + j] = layer_base + b;
        const uint64_t src = acc[b] + bump_first[b];
        for (uint64_t j = 0; j < bump_cnt[b]; j++) bump_out[bump_off[b] + j] = keys[src + j];
    }
}

// evaluateKPerfect (ShockHash2Flat.h:280-301) for every key's original hash: bucket id, or a
// fallback marker together with the last layer's re-mixed hash.
__global__ void k_flat_assign(const uint64_t *__restrict__ mhc0, uint64_t n, uint32_t layers,
                              const uint64_t *__restrict__ layer_bases, const uint8_t *__restrict__ thr,
                              const uint32_t *__restrict__ mapping, uint64_t *__restrict__ bucket_out,
                              uint64_t *__restrict__ last_mhc) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        uint64_t h = mhc0[i];
        uint64_t out = ~0ull;
        for (uint32_t layer = 0; layer < layers; layer++) {
            if (layer) h = remix(h);
            const uint64_t base = layer_bases[layer];
            const uint32_t size = (uint32_t)(layer_bases[layer + 1] - base);
            const uint64_t bkt = base + fastrange32((uint32_t)h, size);
            if ((uint32_t)(h >> 32) <= mapping[thr[bkt]]) {
                out = bkt;
                break;
            }
        }
        bucket_out[i] = out;
        last_mhc[i] = h;
    }
}

// Keys grouped k per bucket, in input order inside a bucket: scatter by bucket, then a block per
// bucket sorts its input indices.
__global__ void k_flat_group_scatter(const uint64_t *__restrict__ bucket, uint64_t n, uint64_t nbuckets,
                                     uint32_t *__restrict__ cursor, uint32_t *__restrict__ slot_idx) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t b = bucket[i];
        if (b < nbuckets) slot_idx[atomicAdd(&cursor[b], 1u)] = (uint32_t)i;
    }
}

__global__ void k_flat_group_sort(uint32_t *__restrict__ slot_idx, const uint32_t *__restrict__ cursor, uint64_t nbuckets,
                                  uint32_t k, const uint64_t *__restrict__ mhc0, uint64_t *__restrict__ leaf_keys,
                                  uint32_t *__restrict__ err) {
    __shared__ uint32_t si[256];
    for (uint64_t b = blockIdx.x; b < nbuckets; b += gridDim.x) {
        const uint32_t got = cursor[b] - (uint32_t)(b * k);
        if (got != k) {
            if (threadIdx.x == 0) atomicOr(err, kErrInternal);
            continue;
        }
        for (uint32_t i = threadIdx.x; i < 256; i += blockDim.x) si[i] = i < k ? slot_idx[b * k + i] : 0xFFFFFFFFu;
        __syncthreads();
        for (uint32_t kk = 2; kk <= 256; kk <<= 1)
            for (uint32_t j = kk >> 1; j > 0; j >>= 1) {
                for (uint32_t i = threadIdx.x; i < 256; i += blockDim.x) {
                    const uint32_t p = i ^ j;
                    if (p > i) {
                        const uint32_t a = si[i], c = si[p];
                        if ((a > c) == ((i & kk) == 0)) {
                            si[i] = c;
                            si[p] = a;
                        }
                    }
                }
                __syncthreads();
            }
        for (uint32_t i = threadIdx.x; i < k; i += blockDim.x) leaf_keys[b * k + i] = mhc0[si[i]];
        __syncthreads();
    }
}

__global__ void k_flat_set_buckets(const uint64_t *__restrict__ idx, const uint64_t *__restrict__ val, uint64_t cnt,
                                   uint64_t *__restrict__ bucket) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < cnt; i += (uint64_t)gridDim.x * blockDim.x)
        bucket[idx[i]] = val[i];
}

__global__ void k_flat_gather(const uint64_t *__restrict__ idx, const uint64_t *__restrict__ src, uint64_t cnt,
                              uint64_t *__restrict__ out) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < cnt; i += (uint64_t)gridDim.x * blockDim.x)
        out[i] = src[idx[i]];
}

__global__ void k_flat_fallback_list(const uint64_t *__restrict__ bucket, uint64_t n, unsigned long long *__restrict__ count,
                                     uint64_t *__restrict__ list) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        if (bucket[i] == ~0ull) list[atomicAdd(count, 1ull)] = i;
}

__global__ void k_flat_cursor_init(uint32_t *cursor, uint64_t nbuckets, uint32_t k) {
    for (uint64_t b = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; b < nbuckets; b += (uint64_t)gridDim.x * blockDim.x)
        cursor[b] = (uint32_t)(b * k);
}

int grid_of(uint64_t n, int threads) {
    uint64_t g = (n + threads - 1) / threads;
    return (int)std::max<uint64_t>(1, std::min<uint64_t>(g, 148ull * 32));
}

} // namespace

void flat_launch_murmur(const uint8_t *bytes, const uint64_t *offsets, uint64_t n, uint64_t *out, cudaStream_t s) {
    if (n) k_murmur_strings<<<grid_of(n, 256), 256, 0, s>>>(bytes, offsets, n, out);
}
void flat_launch_count(uint64_t *mhc, uint64_t n, uint32_t nb, bool rehash, uint32_t *counts, cudaStream_t s) {
    cudaMemsetAsync(counts, 0, (size_t)nb * 4, s);
    if (n) k_flat_count<<<grid_of(n, 256), 256, 0, s>>>(mhc, n, nb, rehash, counts);
}
void flat_launch_scatter(const uint64_t *mhc, uint64_t n, uint32_t nb, uint32_t *cursor, uint64_t *out, cudaStream_t s) {
    if (n) k_flat_scatter<<<grid_of(n, 256), 256, 0, s>>>(mhc, n, nb, cursor, out);
}
void flat_launch_sort_flush(uint64_t *keys, const uint64_t *acc, uint32_t nb, uint32_t k, const uint32_t *mapping,
                            uint32_t range, uint64_t layer_base, uint8_t *thr, uint64_t *free_cnt, uint64_t *bump_cnt,
                            uint32_t *bump_first, uint32_t *err, cudaStream_t s) {
    if (nb)
        k_flat_sort_flush<<<(int)std::min<uint64_t>(nb, 148ull * 16), kFlatSortThreads, 0, s>>>(
            keys, acc, nb, k, mapping, range, layer_base, thr, free_cnt, bump_cnt, bump_first, err);
}
void flat_launch_emit(const uint64_t *keys, const uint64_t *acc, uint32_t nb, uint64_t layer_base, const uint64_t *free_cnt,
                      const uint64_t *free_off, const uint64_t *bump_cnt, const uint64_t *bump_off, const uint32_t *bump_first,
                      uint64_t *free_out, uint64_t *bump_out, cudaStream_t s) {
    if (nb)
        k_flat_emit<<<grid_of(nb, 128), 128, 0, s>>>(keys, acc, nb, layer_base, free_cnt, free_off, bump_cnt, bump_off,
                                                     bump_first, free_out, bump_out);
}
void flat_launch_assign(const uint64_t *mhc0, uint64_t n, uint32_t layers, const uint64_t *layer_bases, const uint8_t *thr,
                        const uint32_t *mapping, uint64_t *bucket, uint64_t *last_mhc, cudaStream_t s) {
    if (n) k_flat_assign<<<grid_of(n, 256), 256, 0, s>>>(mhc0, n, layers, layer_bases, thr, mapping, bucket, last_mhc);
}
void flat_launch_fallback_list(const uint64_t *bucket, uint64_t n, unsigned long long *count, uint64_t *list, cudaStream_t s) {
    cudaMemsetAsync(count, 0, 8, s);
    if (n) k_flat_fallback_list<<<grid_of(n, 256), 256, 0, s>>>(bucket, n, count, list);
}
void flat_launch_gather(const uint64_t *idx, const uint64_t *src, uint64_t cnt, uint64_t *out, cudaStream_t s) {
    if (cnt) k_flat_gather<<<grid_of(cnt, 256), 256, 0, s>>>(idx, src, cnt, out);
}
void flat_launch_set_buckets(const uint64_t *idx, const uint64_t *val, uint64_t cnt, uint64_t *bucket, cudaStream_t s) {
    if (cnt) k_flat_set_buckets<<<grid_of(cnt, 256), 256, 0, s>>>(idx, val, cnt, bucket);
}
void flat_launch_group(const uint64_t *bucket, uint64_t n, uint64_t nbuckets, uint32_t k, uint32_t *cursor,
                       uint32_t *slot_idx, const uint64_t *mhc0, uint64_t *leaf_keys, uint32_t *err, cudaStream_t s) {
    if (!nbuckets) return;
    k_flat_cursor_init<<<grid_of(nbuckets, 256), 256, 0, s>>>(cursor, nbuckets, k);
    if (n) k_flat_group_scatter<<<grid_of(n, 256), 256, 0, s>>>(bucket, n, nbuckets, cursor, slot_idx);
    k_flat_group_sort<<<(int)std::min<uint64_t>(nbuckets, 148ull * 16), 128, 0, s>>>(slot_idx, cursor, nbuckets, k, mhc0,
                                                                                     leaf_keys, err);
}

} // namespace shg
