// Partition of key fingerprints by owning rank, for one structure built over several GPUs.
//
// Bucket b = remap128(first, nb) is monotone in `first` (ShockHash.h:616, Sorter.hpp:15-36), and
// rank g of G owns buckets [floor(nb g / G), floor(nb (g + 1) / G)), so the owner of bucket b is
// floor(((b + 1) G - 1) / nb), the largest g whose first bucket is <= b. The partition writes every
// key's (first, second) pair in rank order, stable (input order inside a rank), plus the count per
// rank: the send buffer and split sizes of one all-to-all, after which each rank holds exactly the
// keys of its buckets in (source rank, source position) order.
//
// Device form, three launches on the engine's stream: per-chunk counts per owner (shared-memory
// atomics), one scan over (owner, chunk), then a stable scatter in which each warp ranks its keys
// among equal owners with __match_any_sync and the block adds the earlier warps' counts.
// Host form: the same order by a counting sort, for processes without a GPU.
#include <algorithm>
#include <cstdint>
#include <string>
#include <thread>
#include <vector>
#include <cuda_runtime.h>
#include "shg.h"
#include "shg_common.cuh"
#include "shg_internal.h"

namespace shg {

cudaStream_t engine_stream(shg_engine *e, int *device);
void *engine_scratch(shg_engine *e, int slot, size_t bytes, cudaError_t &err);

namespace {

constexpr int kShardThreads = 256;
constexpr int kShardChunk = 4096;  // keys per block
constexpr int kMaxWorld = 64;

SHG_HD uint32_t owner_of(uint64_t first, uint64_t nb, uint32_t world) {
    const uint64_t b = remap128(first, nb);
    const uint64_t g = ((b + 1) * world - 1) / nb;
    return (uint32_t)(g < world ? g : world - 1);
}

__global__ void __launch_bounds__(kShardThreads) k_owner_count(const uint64_t *__restrict__ first, uint64_t n, uint64_t nb,
                                                              uint32_t world, uint32_t nchunks, uint32_t *__restrict__ cnt) {
    __shared__ uint32_t c[kMaxWorld];
    for (uint32_t g = threadIdx.x; g < world; g += blockDim.x) c[g] = 0;
    __syncthreads();
    const uint64_t lo = (uint64_t)blockIdx.x * kShardChunk, hi = min(n, lo + kShardChunk);
    for (uint64_t i = lo + threadIdx.x; i < hi; i += blockDim.x) atomicAdd(&c[owner_of(first[i], nb, world)], 1u);
    __syncthreads();
    for (uint32_t g = threadIdx.x; g < world; g += blockDim.x) cnt[(uint64_t)g * nchunks + blockIdx.x] = c[g];
}

// Exclusive scan of cnt (owner-major, chunk-minor) into off; totals per owner into counts.
__global__ void __launch_bounds__(1024) k_owner_scan(const uint32_t *__restrict__ cnt, uint64_t total, uint32_t nchunks,
                                                    uint32_t world, uint64_t *__restrict__ off, uint64_t *__restrict__ counts) {
    __shared__ uint64_t part[1024];
    const uint64_t per = (total + blockDim.x - 1) / blockDim.x;
    const uint64_t lo = min(total, threadIdx.x * per), hi = min(total, lo + per);
    uint64_t s = 0;
    for (uint64_t i = lo; i < hi; i++) s += cnt[i];
    part[threadIdx.x] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        uint64_t run = 0;
        for (uint32_t t = 0; t < blockDim.x; t++) {
            const uint64_t v = part[t];
            part[t] = run;
            run += v;
        }
    }
    __syncthreads();
    uint64_t run = part[threadIdx.x];
    for (uint64_t i = lo; i < hi; i++) {
        off[i] = run;
        run += cnt[i];
    }
    __syncthreads();
    for (uint32_t g = threadIdx.x; g < world; g += blockDim.x) {
        uint64_t t = 0;
        for (uint32_t c = 0; c < nchunks; c++) t += cnt[(uint64_t)g * nchunks + c];
        counts[g] = t;
    }
}

__global__ void __launch_bounds__(kShardThreads) k_owner_scatter(const uint64_t *__restrict__ first,
                                                                const uint64_t *__restrict__ second, uint64_t n, uint64_t nb,
                                                                uint32_t world, uint32_t nchunks,
                                                                const uint64_t *__restrict__ off,
                                                                uint64_t *__restrict__ pairs) {
    constexpr int kWarps = kShardThreads / 32;
    __shared__ uint64_t run[kMaxWorld];
    __shared__ uint32_t wc[kWarps][kMaxWorld];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (uint32_t g = threadIdx.x; g < world; g += blockDim.x) run[g] = off[(uint64_t)g * nchunks + blockIdx.x];
    const uint64_t lo = (uint64_t)blockIdx.x * kShardChunk, hi = min(n, lo + kShardChunk);
    for (uint64_t base = lo; base < hi; base += kShardThreads) {
        for (uint32_t x = threadIdx.x; x < kWarps * world; x += blockDim.x) wc[x / world][x % world] = 0;
        __syncthreads();
        const uint64_t i = base + threadIdx.x;
        const bool live = i < hi;
        const uint32_t g = live ? owner_of(first[i], nb, world) : kMaxWorld;  // kMaxWorld: no owner
        const unsigned same = __match_any_sync(0xffffffffu, g);
        const uint32_t rank_in_warp = __popc(same & ((1u << lane) - 1));
        if (live && rank_in_warp == 0) wc[warp][g] = __popc(same);
        __syncthreads();
        if (live) {
            uint64_t dest = run[g] + rank_in_warp;
            for (int w = 0; w < warp; w++) dest += wc[w][g];
            pairs[2 * dest] = first[i];
            pairs[2 * dest + 1] = second[i];
        }
        __syncthreads();
        for (uint32_t x = threadIdx.x; x < world; x += blockDim.x) {
            uint64_t t = 0;
            for (int w = 0; w < kWarps; w++) t += wc[w][x];
            run[x] += t;
        }
        __syncthreads();
    }
}

} // namespace
} // namespace shg

using namespace shg;

extern "C" {

shg_status shg_shard_partition(const uint64_t *first, const uint64_t *second, uint64_t n, uint64_t nb, int world,
                               uint64_t *pairs, uint64_t *counts) {
    if (world < 1 || world > kMaxWorld || nb == 0 || nb >= (1ull << 32) || !counts || (n && (!first || !second || !pairs)))
        return shg_set_error(SHG_ERR_ARG, "shard partition: bad arguments (1 <= world <= 64, 1 <= nb < 2^32)");
    std::vector<uint32_t> own(n);
    std::vector<uint64_t> pos(world + 1, 0);
    for (int g = 0; g < world; g++) counts[g] = 0;
    for (uint64_t i = 0; i < n; i++) counts[own[i] = owner_of(first[i], nb, (uint32_t)world)]++;
    for (int g = 0; g < world; g++) pos[g + 1] = pos[g] + counts[g];
    for (uint64_t i = 0; i < n; i++) {
        const uint64_t d = pos[own[i]]++;
        pairs[2 * d] = first[i];
        pairs[2 * d + 1] = second[i];
    }
    return SHG_OK;
}

shg_status shg_hash_u64_host(const uint64_t *keys, uint64_t n, uint64_t *first, uint64_t *second, int threads) {
    if (n && (!keys || !first || !second)) return shg_set_error(SHG_ERR_ARG, "null argument");
    const uint64_t T = (uint64_t)std::max(1, std::min(threads, 64));
    const uint64_t chunk = (n + T - 1) / T;
    auto run = [&](uint64_t a, uint64_t b) {
        for (uint64_t i = a; i < b; i++) spooky128_u64(keys[i], 0, first[i], second[i]);
    };
    if (T == 1 || n < (1u << 15)) {
        run(0, n);
        return SHG_OK;
    }
    std::vector<std::thread> pool;
    for (uint64_t t = 0; t < T; t++) {
        const uint64_t a = std::min(n, t * chunk), b = std::min(n, a + chunk);
        if (a < b) pool.emplace_back(run, a, b);
    }
    for (auto &th : pool) th.join();
    return SHG_OK;
}

shg_status shg_shard_partition_device(shg_engine *e, const uint64_t *d_first, const uint64_t *d_second, uint64_t n,
                                      uint64_t nb, int world, uint64_t *d_pairs, uint64_t *counts) {
    if (!e || world < 1 || world > kMaxWorld || nb == 0 || nb >= (1ull << 32) || !counts ||
        (n && (!d_first || !d_second || !d_pairs)))
        return shg_set_error(SHG_ERR_ARG, "shard partition: bad arguments (1 <= world <= 64, 1 <= nb < 2^32)");
    int device = 0;
    cudaStream_t s = engine_stream(e, &device);
    cudaError_t err = cudaSetDevice(device);
    if (err != cudaSuccess) return shg_set_error(SHG_ERR_CUDA, cudaGetErrorString(err));
    if (!n) {
        for (int g = 0; g < world; g++) counts[g] = 0;
        return SHG_OK;
    }
    const uint64_t nchunks64 = (n + kShardChunk - 1) / kShardChunk;
    if (nchunks64 >= (1ull << 31)) return shg_set_error(SHG_ERR_ARG, "shard partition: too many keys");
    const uint32_t nchunks = (uint32_t)nchunks64;
    const uint64_t cells = (uint64_t)world * nchunks;
    // scratch: counts (u32) and offsets (u64) per (owner, chunk), then the per-owner totals
    const size_t cnt_bytes = (cells * 4 + 255) & ~(size_t)255, off_bytes = (cells * 8 + 255) & ~(size_t)255;
    uint8_t *base = (uint8_t *)engine_scratch(e, 0, cnt_bytes + off_bytes + kMaxWorld * 8, err);
    if (!base) return shg_set_error(SHG_ERR_OOM, "shard partition scratch");
    uint32_t *cnt = (uint32_t *)base;
    uint64_t *off = (uint64_t *)(base + cnt_bytes), *tot = (uint64_t *)(base + cnt_bytes + off_bytes);
    k_owner_count<<<nchunks, kShardThreads, 0, s>>>(d_first, n, nb, (uint32_t)world, nchunks, cnt);
    k_owner_scan<<<1, 1024, 0, s>>>(cnt, cells, nchunks, (uint32_t)world, off, tot);
    k_owner_scatter<<<nchunks, kShardThreads, 0, s>>>(d_first, d_second, n, nb, (uint32_t)world, nchunks, off, d_pairs);
    if ((err = cudaGetLastError()) != cudaSuccess) return shg_set_error(SHG_ERR_CUDA, cudaGetErrorString(err));
    if ((err = cudaMemcpyAsync(counts, tot, world * 8, cudaMemcpyDeviceToHost, s)) != cudaSuccess ||
        (err = cudaStreamSynchronize(s)) != cudaSuccess)
        return shg_set_error(SHG_ERR_CUDA, cudaGetErrorString(err));
    return SHG_OK;
}

shg_status shg_partition_u64(shg_engine *e, const uint64_t *keys, uint64_t n, uint64_t nb, int parts, uint64_t *pairs,
                             uint64_t *counts) {
    if (!e || parts < 1 || parts > kMaxWorld || nb == 0 || nb >= (1ull << 32) || !counts || (n && (!keys || !pairs)))
        return shg_set_error(SHG_ERR_ARG, "partition: bad arguments (1 <= parts <= 64, 1 <= nb < 2^32)");
    if (!n) {
        for (int g = 0; g < parts; g++) counts[g] = 0;
        return SHG_OK;
    }
    int device = 0;
    cudaStream_t s = engine_stream(e, &device);
    cudaError_t err = cudaSetDevice(device);
    if (err != cudaSuccess) return shg_set_error(SHG_ERR_CUDA, cudaGetErrorString(err));
    // scratch: the keys in one engine buffer, fingerprints and pairs in another (32 bytes per key)
    uint64_t *d_keys = (uint64_t *)engine_scratch(e, 1, n * 8, err);
    if (!d_keys) return shg_set_error(SHG_ERR_OOM, "partition: key buffer");
    uint64_t *d_fp = (uint64_t *)engine_scratch(e, 2, n * 32, err);
    if (!d_fp) return shg_set_error(SHG_ERR_OOM, "partition: fingerprint buffer");
    uint64_t *d_first = d_fp, *d_second = d_fp + n, *d_pairs = d_fp + 2 * n;
    if ((err = cudaMemcpyAsync(d_keys, keys, n * 8, cudaMemcpyHostToDevice, s)) != cudaSuccess)
        return shg_set_error(SHG_ERR_CUDA, cudaGetErrorString(err));
    launch_spooky_u64(d_keys, n, d_first, d_second, s);
    const shg_status st = shg_shard_partition_device(e, d_first, d_second, n, nb, parts, d_pairs, counts);
    if (st != SHG_OK) return st;
    if ((err = cudaMemcpyAsync(pairs, d_pairs, n * 16, cudaMemcpyDeviceToHost, s)) != cudaSuccess ||
        (err = cudaStreamSynchronize(s)) != cudaSuccess)
        return shg_set_error(SHG_ERR_CUDA, cudaGetErrorString(err));
    return SHG_OK;
}

} // extern "C"
