// Golomb-Rice encoding of all node codes (RiceBitVector::Builder, RiceBitVector.h:67-127, as
// driven by compute_thread/hash_gen, ShockHash.h:557-654).
//
// Per bucket the stream holds the low g bits of every node code in preorder, then every unary
// part (code >> g zeros and a one) in preorder; buckets follow each other without padding and a
// final (1,1) sentinel is appended. Bit lengths are known per node, so the encoder is a scan of
// bucket lengths followed by independent bit writes (64-bit atomic OR into zeroed words; a code
// touches at most two words).
#include <cstdint>
#include <cuda_runtime.h>
#include "shg_common.cuh"
#include "shg_internal.h"

namespace shg {

// One warp per bucket: total bits = fixed bits of the bucket (memo skip_bits) + sum (u + 1).
__global__ void k_gr_bucket_bits(const Node *__restrict__ nodes, const uint32_t *__restrict__ bnb, uint64_t nb,
                                 const uint64_t *__restrict__ acc, const uint64_t *__restrict__ codes,
                                 const uint32_t *__restrict__ skip_bits, uint64_t *__restrict__ bucket_bits) {
    const uint64_t warp = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    for (uint64_t b = warp; b < nb; b += nwarps) {
        uint64_t sum = 0;
        for (uint32_t i = bnb[b] + lane; i < bnb[b + 1]; i += 32) sum += (codes[i] >> nodes[i].g) + 1;
        for (int o = 16; o; o >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, o);
        if (lane == 0) {
            const uint32_t m = (uint32_t)(acc[b + 1] - acc[b]);
            bucket_bits[b] = sum + (bnb[b + 1] > bnb[b] ? skip_bits[m] : 0);
        }
    }
}

// Exclusive scan of n u64 values into out[0..n] (out[n] = total), one block.
__global__ void k_scan_u64(const uint64_t *__restrict__ in, uint64_t n, uint64_t *__restrict__ out) {
    __shared__ uint64_t warp_sums[32];
    __shared__ uint64_t carry;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (uint64_t base = 0; base < n; base += blockDim.x) {
        const uint64_t i = base + threadIdx.x;
        const uint64_t v = i < n ? in[i] : 0;
        uint64_t x = v;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint64_t y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += y;
        }
        if (lane == 31) warp_sums[warp] = x;
        __syncthreads();
        if (warp == 0) {
            uint64_t w = lane < (int)(blockDim.x >> 5) ? warp_sums[lane] : 0;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const uint64_t y = __shfl_up_sync(0xffffffffu, w, o);
                if (lane >= o) w += y;
            }
            warp_sums[lane] = w;
        }
        __syncthreads();
        const uint64_t excl = carry + (warp ? warp_sums[warp - 1] : 0) + x - v;
        if (i < n) out[i] = excl;
        __syncthreads();
        if (threadIdx.x == blockDim.x - 1) carry = excl + v;
        __syncthreads();
    }
    if (threadIdx.x == 0) out[n] = carry;
}

__device__ __forceinline__ void or_bits(unsigned long long *words, uint64_t pos, uint64_t v, int len) {
    if (len == 0) return;
    if (len < 64) v &= (1ull << len) - 1;
    if (v == 0) return;
    const uint64_t w = pos >> 6;
    const int sh = (int)(pos & 63);
    atomicOr(&words[w], (unsigned long long)(v << sh));
    if (sh + len > 64) atomicOr(&words[w + 1], (unsigned long long)(v >> (64 - sh)));
}

// One warp per bucket: fixed parts at their preorder offsets, unary ones after the bucket's fixed
// block at the running sum of (u + 1).
__global__ void k_gr_write(const Node *__restrict__ nodes, const uint16_t *__restrict__ fixed_off,
                           const uint32_t *__restrict__ bnb, uint64_t nb, const uint64_t *__restrict__ acc,
                           const uint64_t *__restrict__ pos_acc, const uint64_t *__restrict__ codes,
                           const uint32_t *__restrict__ skip_bits, unsigned long long *__restrict__ words) {
    const uint64_t warp = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    for (uint64_t b = warp; b < nb; b += nwarps) {
        const uint32_t n0 = bnb[b], n1 = bnb[b + 1];
        if (n0 == n1) continue;
        const uint64_t pos = pos_acc[b];
        const uint32_t m = (uint32_t)(acc[b + 1] - acc[b]);
        const uint64_t unary0 = pos + skip_bits[m];
        uint64_t carry = 0;
        for (uint32_t c0 = n0; c0 < n1; c0 += 32) {
            const uint32_t i = c0 + lane;
            uint64_t code = 0, u1 = 0;
            int g = 0;
            if (i < n1) {
                code = codes[i];
                g = nodes[i].g;
                u1 = (code >> g) + 1;
                or_bits(words, pos + fixed_off[i], code, g);
            }
            uint64_t x = u1;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const uint64_t y = __shfl_up_sync(0xffffffffu, x, o);
                if (lane >= o) x += y;
            }
            if (i < n1) {
                const uint64_t bit = unary0 + carry + x - 1;  // the terminating one of this unary code
                atomicOr(&words[bit >> 6], 1ull << (bit & 63));
            }
            carry += __shfl_sync(0xffffffffu, x, 31);
        }
    }
}

__global__ void k_set_bit(unsigned long long *words, uint64_t bit) { atomicOr(&words[bit >> 6], 1ull << (bit & 63)); }

void launch_gr_bucket_bits(const Node *nodes, const uint32_t *bnb, uint64_t nb, const uint64_t *acc, const uint64_t *codes,
                           const uint32_t *skip_bits, uint64_t *bucket_bits, cudaStream_t s) {
    const uint64_t blocks = (nb * 32 + 255) / 256;
    k_gr_bucket_bits<<<(int)(blocks < 148 * 16 ? blocks : 148 * 16), 256, 0, s>>>(nodes, bnb, nb, acc, codes, skip_bits,
                                                                                  bucket_bits);
}
void launch_scan_u64(const uint64_t *in, uint64_t n, uint64_t *out, cudaStream_t s) { k_scan_u64<<<1, 1024, 0, s>>>(in, n, out); }
void launch_gr_write(const Node *nodes, const uint16_t *fixed_off, const uint32_t *bnb, uint64_t nb, const uint64_t *acc,
                     const uint64_t *pos_acc, const uint64_t *codes, const uint32_t *skip_bits, unsigned long long *words,
                     cudaStream_t s) {
    const uint64_t blocks = (nb * 32 + 255) / 256;
    k_gr_write<<<(int)(blocks < 148 * 16 ? blocks : 148 * 16), 256, 0, s>>>(nodes, fixed_off, bnb, nb, acc, pos_acc, codes,
                                                                            skip_bits, words);
}
void launch_set_bit(unsigned long long *words, uint64_t bit, cudaStream_t s) { k_set_bit<<<1, 1, 0, s>>>(words, bit); }

} // namespace shg
