// Device kernels of the construction pipeline other than the leaf searches:
//   key hashing (SpookyHash V2), bucket partition (remap128 bucketing + per-bucket sort by the
//   first hash half), RecSplit split-seed search with the stable partition, Golomb-Rice encoding.
#include <algorithm>
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

// The same counts with one shared-memory histogram per block (nb counters), flushed with one
// global atomic per non-empty bucket: with a few thousand buckets every counter would otherwise take
// about bucket_size contended global atomics. Each block counts a contiguous chunk of the keys.
__global__ void __launch_bounds__(1024) k_bucket_count_smem(const uint64_t *__restrict__ first, uint64_t n, uint64_t nb,
                                                            uint64_t nb_map, uint64_t b0, uint32_t *__restrict__ counts,
                                                            uint32_t *__restrict__ err) {
    extern __shared__ uint32_t hist[];
    for (uint64_t b = threadIdx.x; b < nb; b += blockDim.x) hist[b] = 0;
    __syncthreads();
    const uint64_t lo = n * blockIdx.x / gridDim.x, hi = n * (blockIdx.x + 1) / gridDim.x;
    for (uint64_t i = lo + threadIdx.x; i < hi; i += blockDim.x) {
        const uint64_t b = remap128(first[i], nb_map) - b0;
        if (b >= nb) {
            atomicOr(err, kErrArg);
            continue;
        }
        atomicAdd(&hist[b], 1u);
    }
    __syncthreads();
    for (uint64_t b = threadIdx.x; b < nb; b += blockDim.x) {
        const uint32_t c = hist[b];
        if (c) atomicAdd(&counts[b], c);
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

// The same scatter with the contention moved to shared memory: a block counts its chunk's keys per
// bucket, reserves each non-empty bucket's range with one global atomic on the cursor, then places
// its keys inside those ranges with shared-memory atomics. The order inside a bucket depends on
// atomic order here as in k_bucket_scatter; k_bucket_sort orders each bucket by (first, input
// index), so the products do not depend on it.
__global__ void __launch_bounds__(1024) k_bucket_scatter_smem(const uint64_t *__restrict__ first, uint64_t n, uint64_t nb,
                                                              uint64_t nb_map, uint64_t b0, uint32_t *__restrict__ cursor,
                                                              uint64_t *__restrict__ sfirst, uint32_t *__restrict__ sidx,
                                                              uint64_t idx_base) {
    extern __shared__ uint32_t slot[];
    for (uint64_t b = threadIdx.x; b < nb; b += blockDim.x) slot[b] = 0;
    __syncthreads();
    const uint64_t lo = n * blockIdx.x / gridDim.x, hi = n * (blockIdx.x + 1) / gridDim.x;
    for (uint64_t i = lo + threadIdx.x; i < hi; i += blockDim.x) {
        const uint64_t b = remap128(first[i], nb_map) - b0;
        if (b < nb) atomicAdd(&slot[b], 1u);  // keys outside are reported by the count kernel
    }
    __syncthreads();
    for (uint64_t b = threadIdx.x; b < nb; b += blockDim.x) {
        const uint32_t c = slot[b];
        if (c) slot[b] = atomicAdd(&cursor[b], c);  // this block's range of bucket b
    }
    __syncthreads();
    for (uint64_t i = lo + threadIdx.x; i < hi; i += blockDim.x) {
        const uint64_t f = first[i];
        const uint64_t b = remap128(f, nb_map) - b0;
        if (b >= nb) continue;
        const uint32_t pos = atomicAdd(&slot[b], 1u);
        sfirst[pos] = f;
        sidx[pos] = (uint32_t)(idx_base + i);
    }
}

// One block per bucket: sort of (first, input index) in shared memory, then gather the second
// halves in that order (Sorter.hpp:15-36 sorts by `first` and keeps `second`). Equal `first`
// values keep input order, as in the oracle's stable sort (the reference's ips2ra leaves their
// order unspecified).
//
// Within a bucket the `first` values are uniform over the bucket's range, so a counting sort on
// sub = (first - min) >> shift, with the shift leaving at most 4096 sub-ranges, places nearly every
// key; the few sub-ranges holding more than one key are finished by insertion sort on
// (first, index). sub is monotone in `first`, so the result is the sorted order.
constexpr int kSortThreads = 256;
constexpr int kSortSubs = 4096;
struct SortSmem {
    uint32_t start[kSortSubs + 1];
    uint32_t cursor[kSortSubs];
    uint64_t f[kMaxBucket];
    uint32_t idx[kMaxBucket];
    uint64_t red[2][kSortThreads / 32];
};
__global__ void __launch_bounds__(kSortThreads) k_bucket_sort(const uint64_t *__restrict__ acc, uint64_t nb,
                                                              const uint64_t *__restrict__ sfirst,
                                                              const uint32_t *__restrict__ sidx,
                                                              const uint64_t *__restrict__ second,
                                                              uint64_t *__restrict__ keys) {
    extern __shared__ __align__(16) uint8_t smem_raw[];
    SortSmem &sm = *(SortSmem *)smem_raw;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    constexpr int kPer = kSortSubs / kSortThreads;  // sub-ranges scanned per thread
    for (uint64_t b = blockIdx.x; b < nb; b += gridDim.x) {
        const uint64_t beg = acc[b];
        const uint32_t m = (uint32_t)(acc[b + 1] - beg);
        if (m < 2) {
            if (m == 1 && threadIdx.x == 0) keys[beg] = second[sidx[beg]];
            continue;
        }
        // range of `first` in the bucket
        uint64_t lo = ~0ull, hi = 0;
        for (uint32_t i = threadIdx.x; i < m; i += kSortThreads) {
            const uint64_t f = sfirst[beg + i];
            lo = min(lo, f);
            hi = max(hi, f);
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            lo = min(lo, __shfl_xor_sync(0xffffffffu, lo, o));
            hi = max(hi, __shfl_xor_sync(0xffffffffu, hi, o));
        }
        if (lane == 0) {
            sm.red[0][warp] = lo;
            sm.red[1][warp] = hi;
        }
        for (int s = threadIdx.x; s < kSortSubs; s += kSortThreads) sm.cursor[s] = 0;
        __syncthreads();
        lo = sm.red[0][0];
        hi = sm.red[1][0];
#pragma unroll
        for (int w = 1; w < kSortThreads / 32; w++) {
            lo = min(lo, sm.red[0][w]);
            hi = max(hi, sm.red[1][w]);
        }
        const uint64_t span = hi - lo;
        const int bits = span ? 64 - __clzll((long long)span) : 0;
        const int shift = bits > 12 ? bits - 12 : 0;  // (span >> shift) < 4096
        // counts per sub-range
        for (uint32_t i = threadIdx.x; i < m; i += kSortThreads)
            atomicAdd(&sm.cursor[(uint32_t)((sfirst[beg + i] - lo) >> shift)], 1u);
        __syncthreads();
        // exclusive scan of the counts: each thread owns kPer consecutive sub-ranges
        uint32_t c[kPer], sum = 0;
#pragma unroll
        for (int k = 0; k < kPer; k++) {
            c[k] = sm.cursor[threadIdx.x * kPer + k];
            sum += c[k];
        }
        uint32_t x = sum;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += y;
        }
        if (lane == 31) sm.red[0][warp] = x;  // the range reduction's reads of red ended before the counts
        __syncthreads();
        uint32_t run = x - sum;
        for (int w = 0; w < warp; w++) run += (uint32_t)sm.red[0][w];
#pragma unroll
        for (int k = 0; k < kPer; k++) {
            sm.start[threadIdx.x * kPer + k] = run;
            sm.cursor[threadIdx.x * kPer + k] = run;
            run += c[k];
        }
        if (threadIdx.x == kSortThreads - 1) sm.start[kSortSubs] = run;
        __syncthreads();
        // scatter into the sub-ranges (any order inside one)
        for (uint32_t i = threadIdx.x; i < m; i += kSortThreads) {
            const uint64_t f = sfirst[beg + i];
            const uint32_t pos = atomicAdd(&sm.cursor[(uint32_t)((f - lo) >> shift)], 1u);
            sm.f[pos] = f;
            sm.idx[pos] = sidx[beg + i];
        }
        __syncthreads();
        // sub-ranges with several keys: insertion sort by (first, index)
        for (int s = threadIdx.x; s < kSortSubs; s += kSortThreads) {
            const uint32_t a = sm.start[s], e = sm.start[s + 1];
            for (uint32_t i = a + 1; i < e; i++) {
                const uint64_t f = sm.f[i];
                const uint32_t ix = sm.idx[i];
                uint32_t j = i;
                while (j > a && (sm.f[j - 1] > f || (sm.f[j - 1] == f && sm.idx[j - 1] > ix))) {
                    sm.f[j] = sm.f[j - 1];
                    sm.idx[j] = sm.idx[j - 1];
                    j--;
                }
                sm.f[j] = f;
                sm.idx[j] = ix;
            }
        }
        __syncthreads();
        for (uint32_t i = threadIdx.x; i < m; i += kSortThreads) keys[beg + i] = second[sm.idx[i]];
        __syncthreads();
    }
}

// Retrieval input without the keys of size-1 children (they get no retrieval bit,
// ShockHash.h:480,514,547): out[i - #singles before i] = in[i] for every non-single position i.
// `singles` holds batch-wide positions in ascending order; the request starts at single_base.
__global__ void k_compact_ribbon(const uint64_t *__restrict__ keys, const uint8_t *__restrict__ bits, uint64_t n,
                                 const uint64_t *__restrict__ singles, uint64_t nsingles, uint64_t single_base,
                                 uint64_t *__restrict__ out_keys, uint8_t *__restrict__ out_bits) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t gi = single_base + i;
        uint64_t lo = 0, hi = nsingles;  // count of singles < i
        while (lo < hi) {
            const uint64_t mid = (lo + hi) >> 1;
            if (singles[mid] < gi) lo = mid + 1; else hi = mid;
        }
        if (lo < nsingles && singles[lo] == gi) continue;
        if (out_keys) out_keys[i - lo] = keys[i];  // either part may be compacted on its own
        if (out_bits) out_bits[i - lo] = bits[i];
    }
}

void launch_compact_ribbon(const uint64_t *keys, const uint8_t *bits, uint64_t n, const uint64_t *singles,
                           uint64_t nsingles, uint64_t single_base, uint64_t *out_keys, uint8_t *out_bits,
                           cudaStream_t s) {
    if (n)
        k_compact_ribbon<<<grid_for(n, 256), 256, 0, s>>>(keys, bits, n, singles, nsingles, single_base, out_keys,
                                                          out_bits);
}

// ------------------------------------------------------------------------------ plan
// The plan of a build is every bucket's tree shape (by bucket size) stamped out at the bucket's
// offsets in the node array, the launch lists and the size-1 positions. One block per column of
// the shape table: offs[col][b] = sum over buckets before b of cnt[size(b)][col], offs[col][nb] =
// the column total, also stored compactly at offs[ncol * (nb + 1) + col]. Each thread scans a
// contiguous run of buckets; a bucket of `rows` keys or more (rejected by the host afterwards)
// counts as empty.
constexpr int kPlanScanThreads = 1024;
__global__ void __launch_bounds__(kPlanScanThreads) k_plan_scan(const uint64_t *__restrict__ acc, uint64_t nb,
                                                                const uint32_t *__restrict__ cnt, uint32_t rows, int ncol,
                                                                uint32_t *__restrict__ offs) {
    __shared__ uint32_t warp_sums[kPlanScanThreads / 32];
    const int col = blockIdx.x;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint64_t run = (nb + kPlanScanThreads - 1) / kPlanScanThreads;
    const uint64_t lo = min(nb, threadIdx.x * run), hi = min(nb, lo + run);
    auto count_of = [&](uint64_t b) -> uint32_t {
        const uint64_t m = acc[b + 1] - acc[b];
        return m < rows ? cnt[m * ncol + col] : 0u;
    };
    uint32_t sum = 0;
#pragma unroll 4
    for (uint64_t b = lo; b < hi; b++) sum += count_of(b);
    uint32_t x = sum;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) warp_sums[warp] = x;
    __syncthreads();
    if (warp == 0) {
        uint32_t w = warp_sums[lane];
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= o) w += y;
        }
        warp_sums[lane] = w;
    }
    __syncthreads();
    uint32_t pos = (warp ? warp_sums[warp - 1] : 0) + x - sum;
    uint32_t *out = offs + (uint64_t)col * (nb + 1);
    for (uint64_t b = lo; b < hi; b++) {
        out[b] = pos;
        pos += count_of(b);
    }
    if (threadIdx.x == kPlanScanThreads - 1) {
        out[nb] = pos;
        offs[(uint64_t)ncol * (nb + 1) + col] = pos;
    }
}

// One warp per bucket: its shape's nodes become Node records at the bucket's node offset (ids in
// preorder, buckets in order), each node id goes to its launch list at the bucket's offset in that
// list plus the node's rank, and the size-1 positions become batch-wide key positions.
__global__ void k_plan_expand(const uint64_t *__restrict__ acc, uint64_t nb, uint32_t rows, const uint32_t *__restrict__ offs,
                              const ShapeNode *__restrict__ shape_nodes, const uint32_t *__restrict__ node_off,
                              const uint16_t *__restrict__ shape_singles, const uint32_t *__restrict__ single_off,
                              const ListOffsets lists, Node *__restrict__ nodes, uint16_t *__restrict__ fixed_off,
                              uint32_t *__restrict__ ids, uint64_t *__restrict__ singles) {
    const int lane = threadIdx.x & 31;
    const uint64_t warps = (uint64_t)gridDim.x * (blockDim.x >> 5);
    const uint64_t stride = nb + 1;
    for (uint64_t b = blockIdx.x * (uint64_t)(blockDim.x >> 5) + (threadIdx.x >> 5); b < nb; b += warps) {
        const uint64_t a0 = acc[b];
        const uint64_t m = acc[b + 1] - a0;
        if (m >= rows) continue;  // rejected by the host before this launch
        const uint32_t node0 = offs[kColNodes * stride + b];
        const uint32_t t0 = node_off[m], t1 = node_off[m + 1];
        for (uint32_t j = t0 + lane; j < t1; j += 32) {
            const ShapeNode t = shape_nodes[j];
            const uint32_t id = node0 + (j - t0);
            Node n;
            n.start = (uint32_t)(a0 + t.rel);
            n.m = t.m;
            n.level = (uint8_t)t.seed;  // start-seed index (the depth, except SIMDShockHash's fixed entries)
            n.kind = t.kind;
            n.bucket = (uint32_t)b;
            n.unit = t.unit;
            n.fanout = t.fanout;
            n.g = t.g;
            nodes[id] = n;
            fixed_off[id] = t.fixed_off;
            if (t.kind == kLeaf)
                ids[lists.leaf + offs[kColLeaves * stride + b] + t.rank] = id;
            else
                ids[lists.level[t.level] + offs[(kColLevel0 + t.level) * stride + b] + t.rank] = id;
        }
        const uint32_t s0 = single_off[m], s1 = single_off[m + 1];
        const uint32_t sb = offs[kColSingles * stride + b];
        for (uint32_t j = s0 + lane; j < s1; j += 32) singles[sb + (j - s0)] = a0 + shape_singles[j];
    }
}

void launch_plan_scan(const uint64_t *acc, uint64_t nb, const uint32_t *cnt, uint32_t rows, int ncol, uint32_t *offs,
                      cudaStream_t s) {
    k_plan_scan<<<ncol, kPlanScanThreads, 0, s>>>(acc, nb, cnt, rows, ncol, offs);
}

void launch_plan_expand(const uint64_t *acc, uint64_t nb, uint32_t rows, const uint32_t *offs, const ShapeNode *shape_nodes,
                        const uint32_t *node_off, const uint16_t *shape_singles, const uint32_t *single_off,
                        const ListOffsets &lists, Node *nodes, uint16_t *fixed_off, uint32_t *ids, uint64_t *singles,
                        cudaStream_t s) {
    if (!nb) return;
    const uint64_t blocks = std::min<uint64_t>((nb + 7) / 8, 148ull * 16);
    k_plan_expand<<<(int)blocks, 256, 0, s>>>(acc, nb, rows, offs, shape_nodes, node_off, shape_singles, single_off,
                                                lists, nodes, fixed_off, ids, singles);
}

// Blocks of the shared-memory partition kernels: two 1024-thread blocks per SM (a full SM of
// threads, which the scattered writes need), at most one per 4096 keys; 0 above 6,144 buckets, where
// the global-atomic kernels were measured faster on B200 (partition of 4M / 10M / 16M keys:
// 0.33 / 0.92 / 1.80 ms with these kernels, 0.56 / 1.04 / 1.46 ms without).
static int partition_smem_blocks(uint64_t n, uint64_t nb, size_t &smem) {
    constexpr uint64_t kMaxSmem = 6144 * sizeof(uint32_t);
    smem = (size_t)nb * sizeof(uint32_t);
    if (nb == 0 || smem > kMaxSmem) return 0;
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    return (int)std::max<uint64_t>(1, std::min<uint64_t>((uint64_t)sms * 2, (n + 4095) / 4096));
}

void launch_bucket_count(const uint64_t *first, uint64_t n, uint64_t nb, uint64_t nb_map, uint64_t b0, uint32_t *counts,
                         uint32_t *err, cudaStream_t s) {
    cudaMemsetAsync(counts, 0, nb * sizeof(uint32_t), s);
    if (!n) return;
    size_t smem = 0;
    const int blocks = partition_smem_blocks(n, nb, smem);
    if (blocks) {
        // the shared-memory limit is an attribute of the kernel on the current device: set it on every launch
        cudaFuncSetAttribute(k_bucket_count_smem, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        k_bucket_count_smem<<<blocks, 1024, smem, s>>>(first, n, nb, nb_map, b0, counts, err);
    } else {
        k_bucket_count<<<grid_for(n, 256), 256, 0, s>>>(first, n, nb, nb_map, b0, counts, err);
    }
}
void launch_scan_counts(const uint32_t *counts, uint64_t nb, uint64_t *acc, uint32_t *cursor, uint32_t *maxsz,
                        cudaStream_t s) {
    cudaMemsetAsync(maxsz, 0, sizeof(uint32_t), s);
    k_scan_counts<<<1, 1024, 0, s>>>(counts, nb, acc, cursor, maxsz);
}
void launch_bucket_scatter(const uint64_t *first, uint64_t n, uint64_t nb, uint64_t nb_map, uint64_t b0, uint32_t *cursor,
                           uint64_t *sfirst, uint32_t *sidx, uint64_t idx_base, cudaStream_t s) {
    if (!n) return;
    size_t smem = 0;
    const int blocks = partition_smem_blocks(n, nb, smem);
    if (blocks) {
        cudaFuncSetAttribute(k_bucket_scatter_smem, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        k_bucket_scatter_smem<<<blocks, 1024, smem, s>>>(first, n, nb, nb_map, b0, cursor, sfirst, sidx, idx_base);
    } else {
        k_bucket_scatter<<<grid_for(n, 256), 256, 0, s>>>(first, n, nb, nb_map, b0, cursor, sfirst, sidx, idx_base);
    }
}
void launch_bucket_sort(const uint64_t *acc, uint64_t nb, const uint64_t *sfirst, const uint32_t *sidx,
                        const uint64_t *second, uint64_t *keys, cudaStream_t s) {
    const size_t smem = sizeof(SortSmem);
    cudaFuncSetAttribute(k_bucket_sort, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    const uint64_t grid = nb < 148ull * 12 ? nb : 148ull * 12;
    k_bucket_sort<<<(int)grid, kSortThreads, smem, s>>>(acc, nb, sfirst, sidx, second, keys);
}

} // namespace shg
