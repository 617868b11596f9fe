// Compact 1-bit retrieval built on the device: the structure the reference builds on the host with
// SimpleRibbon<1, w> from the retrieval input (ShockHash.h:152,657; ShockHash2.h:133,497) and reads
// with retrieve() in operator() (ShockHash.h:267-270, ShockHash2.h:226-229). SimpleRibbon's source
// is not part of the reference tree, so its layout is not reproduced; this structure answers the
// same question (the stored bit of every input key) in its own format:
//
//   level l (seed l): key -> h = remix(key + seed_l); bucket = fastrange64(h, B_l);
//   priority p = (h >> 8) & 127. A bucket keeps the keys with p < thr[bucket] (at most 248) and
//   stores a 256-bit vector s with parity(row(h) & s) = bit for each kept key, row(h) being four
//   remix words of h. Keys with p >= thr go to level l + 1.
//
// One warp solves one bucket: dense Gaussian elimination over GF(2) in shared memory (rows in
// word-major layout), then back substitution with the free columns at zero. The solution depends
// only on the kept set, not on the order the keys arrive in, so builds are deterministic. A kept
// set with no solution (probability ~2^-8) drops its highest priority value and is solved again.
// Space: (256 + 8) bits per bucket of ~240 keys, about 1.1 bits per key.
#include <algorithm>
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>
#include <cuda_runtime.h>
#include "shg.h"
#include "shg_common.cuh"
#include "shg_internal.h"
#include "shg_retrieval.cuh"

namespace shg {

constexpr int kRetWarps = 4;  // warps (buckets in flight) per block

__global__ void k_ret_count(const uint64_t *__restrict__ keys, uint64_t n, int level, uint64_t nb,
                            uint32_t *__restrict__ counts) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        atomicAdd(&counts[fastrange64(ret_hash(keys[i], level), nb)], 1u);
}

__global__ void k_ret_scatter(const uint64_t *__restrict__ keys, const uint8_t *__restrict__ bits, uint64_t n, int level,
                              uint64_t nb, uint32_t *__restrict__ cursor, uint64_t *__restrict__ bkeys,
                              uint8_t *__restrict__ bbits) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t k = keys[i];
        const uint32_t pos = atomicAdd(&cursor[fastrange64(ret_hash(k, level), nb)], 1u);
        bkeys[pos] = k;
        bbits[pos] = bits[i] & 1;
    }
}

struct RetWarpSmem {
    uint64_t rows[kRetWords][kRetRows];  // word-major: lane r reads rows[w][r], consecutive addresses
    uint8_t rhs[kRetRows];
    uint16_t pivot_row[kRetRows];        // per column, or 0xFFFF for a free column
    uint32_t hist[kRetPrio];
};

// Forward elimination over rows [0, n) of the warp's system; returns true when it is consistent.
__device__ bool ret_eliminate(RetWarpSmem &sm, uint32_t n, int lane) {
    uint32_t done = 0;  // per lane: its rows lane + 32k that are pivots (or beyond n)
#pragma unroll
    for (int k = 0; k < kRetRows / 32; k++)
        if ((uint32_t)(lane + 32 * k) >= n) done |= 1u << k;
#pragma unroll
    for (int w = 0; w < kRetWords; w++) {
        for (int bit = 0; bit < 64; bit++) {
            const int c = w * 64 + bit;
            uint32_t has = 0;
#pragma unroll
            for (int k = 0; k < kRetRows / 32; k++)
                if (!((done >> k) & 1) && ((sm.rows[w][lane + 32 * k] >> bit) & 1)) has |= 1u << k;
            int p = -1;
#pragma unroll
            for (int k = 0; k < kRetRows / 32; k++) {
                const uint32_t m = __ballot_sync(0xffffffffu, (has >> k) & 1);
                if (p < 0 && m) p = 32 * k + __ffs(m) - 1;
            }
            if (lane == 0) sm.pivot_row[c] = p < 0 ? 0xFFFF : (uint16_t)p;
            if (p < 0) continue;  // warp-uniform
            if ((p & 31) == lane) {
                done |= 1u << (p >> 5);
                has &= ~(1u << (p >> 5));
            }
            uint64_t piv[kRetWords];
#pragma unroll
            for (int v = w; v < kRetWords; v++) piv[v] = sm.rows[v][p];
            const uint8_t prhs = sm.rhs[p];
            __syncwarp();
#pragma unroll
            for (int k = 0; k < kRetRows / 32; k++) {
                if ((has >> k) & 1) {
                    const int r = lane + 32 * k;
#pragma unroll
                    for (int v = w; v < kRetWords; v++) sm.rows[v][r] ^= piv[v];
                    sm.rhs[r] ^= prhs;
                }
            }
            __syncwarp();
        }
    }
    bool bad = false;
#pragma unroll
    for (int k = 0; k < kRetRows / 32; k++)
        if (!((done >> k) & 1) && sm.rhs[lane + 32 * k]) bad = true;
    return !__any_sync(0xffffffffu, bad);
}

// One warp per bucket: pick the threshold, solve, store the solution, pass the rest on.
__global__ void __launch_bounds__(kRetWarps * 32) k_ret_solve(const uint64_t *__restrict__ acc, uint64_t nb, int level,
                                                              const uint64_t *__restrict__ bkeys,
                                                              const uint8_t *__restrict__ bbits, uint64_t *__restrict__ sol,
                                                              uint8_t *__restrict__ thr, uint64_t *__restrict__ next_keys,
                                                              uint8_t *__restrict__ next_bits,
                                                              unsigned long long *__restrict__ next_count,
                                                              uint32_t *__restrict__ err) {
    __shared__ RetWarpSmem smem[kRetWarps];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    RetWarpSmem &sm = smem[wib];
    const uint64_t warps = (uint64_t)gridDim.x * kRetWarps;
    for (uint64_t b = blockIdx.x * (uint64_t)kRetWarps + wib; b < nb; b += warps) {
        const uint64_t a0 = acc[b];
        const uint32_t m = (uint32_t)(acc[b + 1] - a0);
        // threshold: the largest t with #(p < t) <= kRetCap
        for (uint32_t j = lane; j < kRetPrio; j += 32) sm.hist[j] = 0;
        __syncwarp();
        for (uint32_t i = lane; i < m; i += 32) atomicAdd(&sm.hist[ret_prio(ret_hash(bkeys[a0 + i], level))], 1u);
        __syncwarp();
        uint32_t h4[4], s4 = 0;
#pragma unroll
        for (int q = 0; q < 4; q++) {
            h4[q] = sm.hist[lane * 4 + q];
            s4 += h4[q];
        }
        uint32_t incl = s4;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += y;
        }
        uint32_t run = incl - s4, t = 0;
#pragma unroll
        for (int q = 0; q < 4; q++) {
            run += h4[q];
            if (run <= kRetCap) t = lane * 4 + q + 1;
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) t = max(t, __shfl_xor_sync(0xffffffffu, t, o));
        // solve; an inconsistent kept set drops its highest priority value and is solved again
        for (;;) {
            uint32_t n = 0, pmax = 0;
            for (uint32_t base = 0; base < m; base += 32) {
                const uint32_t i = base + lane;
                uint64_t h = 0;
                uint32_t p = kRetPrio;
                if (i < m) {
                    h = ret_hash(bkeys[a0 + i], level);
                    p = ret_prio(h);
                }
                const bool keep = p < t;
                const uint32_t bal = __ballot_sync(0xffffffffu, keep);
                if (keep) {
                    const uint32_t r = n + __popc(bal & ((1u << lane) - 1));
#pragma unroll
                    for (int v = 0; v < kRetWords; v++) sm.rows[v][r] = ret_row_word(h, v);
                    sm.rhs[r] = bbits[a0 + i];
                    pmax = max(pmax, p);
                }
                n += __popc(bal);
            }
            __syncwarp();
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) pmax = max(pmax, __shfl_xor_sync(0xffffffffu, pmax, o));
            if (ret_eliminate(sm, n, lane) || n == 0) break;
            t = pmax;  // keep p < pmax: at least one key fewer
            __syncwarp();
        }
        // back substitution, free columns at zero: x_c = rhs(P_c) ^ parity(P_c & x) over columns > c
        uint64_t x[kRetWords] = {0, 0, 0, 0};
#pragma unroll
        for (int w = kRetWords - 1; w >= 0; w--) {
            for (int bit = 63; bit >= 0; bit--) {
                const uint32_t pr = sm.pivot_row[w * 64 + bit];
                if (pr == 0xFFFF) continue;
                uint32_t par = sm.rhs[pr];
#pragma unroll
                for (int v = w; v < kRetWords; v++) par += (uint32_t)__popcll(sm.rows[v][pr] & x[v]);
                if (par & 1) x[w] |= 1ull << bit;
            }
        }
        if (lane == 0) {
#pragma unroll
            for (int v = 0; v < kRetWords; v++) sol[b * kRetWords + v] = x[v];
            thr[b] = (uint8_t)t;
        }
        // keys with p >= t go on; every kept key is checked against the solution
        for (uint32_t base = 0; base < m; base += 32) {
            const uint32_t i = base + lane;
            bool bump = false;
            uint64_t k = 0;
            uint8_t bit = 0;
            if (i < m) {
                k = bkeys[a0 + i];
                bit = bbits[a0 + i];
                const uint64_t h = ret_hash(k, level);
                if (ret_prio(h) >= t)
                    bump = true;
                else if (ret_parity(h, x) != bit)
                    atomicOr(err, kErrInternal);
            }
            const uint32_t bal = __ballot_sync(0xffffffffu, bump);
            unsigned long long base_pos = 0;
            if (lane == 0 && bal) base_pos = atomicAdd(next_count, (unsigned long long)__popc(bal));
            base_pos = __shfl_sync(0xffffffffu, base_pos, 0);
            if (bump) {
                const uint64_t pos = base_pos + __popc(bal & ((1u << lane) - 1));
                next_keys[pos] = k;
                next_bits[pos] = bit;
            }
        }
        __syncwarp();
    }
}

__global__ void k_ret_query(RetLevels lv, const uint64_t *__restrict__ sol, const uint8_t *__restrict__ thr,
                            const uint64_t *__restrict__ keys, uint64_t n, uint8_t *__restrict__ out) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        out[i] = (uint8_t)ret_lookup(lv, sol, thr, keys[i]);
}

static int ret_grid(uint64_t n, int threads) {
    uint64_t g = (n + threads - 1) / threads;
    if (g > 148ull * 32) g = 148ull * 32;
    return g < 1 ? 1 : (int)g;
}

} // namespace shg

using namespace shg;

struct shg_retrieval {
    int device = 0;
    uint64_t n = 0;
    RetLevels lv{};
    std::vector<uint64_t> sol;  // kRetWords words per bucket, levels back to back
    std::vector<uint8_t> thr;
    uint64_t *d_sol = nullptr;
    uint8_t *d_thr = nullptr;
    RetLevels *d_lv = nullptr;
    float build_ms = 0.f, query_ms = 0.f;
    ~shg_retrieval() {
        if (d_sol || d_thr || d_lv) {
            int cur = 0;
            cudaGetDevice(&cur);
            cudaSetDevice(device);
            cudaFree(d_sol);
            cudaFree(d_thr);
            cudaFree(d_lv);
            cudaSetDevice(cur);
        }
    }
};

namespace shg {
void *engine_scratch(shg_engine *e, int slot, size_t bytes, cudaError_t &err);
}

namespace {

#define RCU(call)                                                                                  \
    do {                                                                                           \
        cudaError_t e_ = (call);                                                                   \
        if (e_ != cudaSuccess) {                                                                   \
            st = shg_set_error(SHG_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_));  \
            goto done;                                                                             \
        }                                                                                          \
    } while (0)

// Device copies of the concatenated levels, for device queries.
shg_status ret_upload(shg_retrieval *r) {
    shg_status st = SHG_OK;
    const size_t nbk = r->thr.size();
    RCU(cudaMalloc(&r->d_sol, std::max<size_t>(nbk, 1) * kRetWords * 8));
    RCU(cudaMalloc(&r->d_thr, std::max<size_t>(nbk, 1)));
    RCU(cudaMalloc(&r->d_lv, sizeof(RetLevels)));
    RCU(cudaMemcpy(r->d_lv, &r->lv, sizeof(RetLevels), cudaMemcpyHostToDevice));
    if (nbk) {
        RCU(cudaMemcpy(r->d_sol, r->sol.data(), nbk * kRetWords * 8, cudaMemcpyHostToDevice));
        RCU(cudaMemcpy(r->d_thr, r->thr.data(), nbk, cudaMemcpyHostToDevice));
    }
done:
    return st;
}

// The build from keys and bits already in device memory; stream-ordered on `s`, then synchronous.
// Scratch is one region, carved: the engine's reusable buffer when `e` is given, else a region
// allocated for this call.
shg_status ret_build(shg_engine *e, int device, cudaStream_t s, const uint64_t *d_keys, const uint8_t *d_bits,
                     uint64_t n, shg_retrieval **out) {
    shg_status st = SHG_OK;
    shg_retrieval *r = new shg_retrieval();
    r->device = device;
    r->n = n;
    uint64_t *ka = nullptr, *kb = nullptr, *bk = nullptr, *acc = nullptr, *dsol = nullptr;
    uint8_t *ba = nullptr, *bb = nullptr, *bbit = nullptr, *dthr = nullptr;
    uint32_t *counts = nullptr, *cursor = nullptr, *misc = nullptr;
    unsigned long long *next = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    void *own = nullptr;  // the region when no engine provides one
    const uint64_t cap_b = n / kRetLoad + 2, nn = std::max<uint64_t>(n, 1);
    const uint64_t *in_keys = d_keys;  // level 0 reads the input; later levels the bumped keys
    const uint8_t *in_bits = d_bits;
    uint64_t cur_n = n;
    int level = 0;
    {
        size_t off = 0;
        auto take = [&](size_t bytes) {
            const size_t at = off;
            off += (bytes + 255) & ~(size_t)255;
            return at;
        };
        const size_t o_ka = take(nn * 8), o_kb = take(nn * 8), o_bk = take(nn * 8), o_ba = take(nn), o_bb = take(nn),
                     o_bbit = take(nn), o_acc = take((cap_b + 1) * 8), o_cnt = take(cap_b * 4),
                     o_cur = take(cap_b * 4), o_sol = take(cap_b * kRetWords * 8), o_thr = take(cap_b),
                     o_misc = take(16), o_next = take(8);
        uint8_t *base = nullptr;
        if (e) {
            cudaError_t err = cudaSuccess;
            base = (uint8_t *)engine_scratch(e, 0, off, err);
            RCU(err);
        } else {
            RCU(cudaMalloc(&own, off));
            base = (uint8_t *)own;
        }
        ka = (uint64_t *)(base + o_ka);
        kb = (uint64_t *)(base + o_kb);
        bk = (uint64_t *)(base + o_bk);
        ba = base + o_ba;
        bb = base + o_bb;
        bbit = base + o_bbit;
        acc = (uint64_t *)(base + o_acc);
        counts = (uint32_t *)(base + o_cnt);
        cursor = (uint32_t *)(base + o_cur);
        dsol = (uint64_t *)(base + o_sol);
        dthr = base + o_thr;
        misc = (uint32_t *)(base + o_misc);
        next = (unsigned long long *)(base + o_next);
    }
    RCU(cudaEventCreate(&e0));
    RCU(cudaEventCreate(&e1));
    RCU(cudaMemsetAsync(misc, 0, 16, s));
    RCU(cudaEventRecord(e0, s));
    while (cur_n) {
        if (level == kRetMaxLevels) {
            st = shg_set_error(SHG_ERR_ARG, "retrieval input holds duplicate keys with different bits");
            goto done;
        }
        const uint64_t nb = std::max<uint64_t>(1, (cur_n + kRetLoad - 1) / kRetLoad);
        RCU(cudaMemsetAsync(counts, 0, nb * 4, s));
        k_ret_count<<<ret_grid(cur_n, 256), 256, 0, s>>>(in_keys, cur_n, level, nb, counts);
        launch_scan_counts(counts, nb, acc, cursor, misc + 1, s);
        k_ret_scatter<<<ret_grid(cur_n, 256), 256, 0, s>>>(in_keys, in_bits, cur_n, level, nb, cursor, bk, bbit);
        RCU(cudaMemsetAsync(next, 0, 8, s));
        {
            const uint64_t blocks = std::min<uint64_t>((nb + kRetWarps - 1) / kRetWarps, 148ull * 16);
            k_ret_solve<<<(int)blocks, kRetWarps * 32, 0, s>>>(acc, nb, level, bk, bbit, dsol, dthr, ka, ba, next, misc);
        }
        RCU(cudaGetLastError());
        unsigned long long bumped = 0;
        uint32_t err = 0;
        const size_t off = r->thr.size();
        r->sol.resize(off * kRetWords + nb * kRetWords);
        r->thr.resize(off + nb);
        RCU(cudaMemcpyAsync(r->sol.data() + off * kRetWords, dsol, nb * kRetWords * 8, cudaMemcpyDeviceToHost, s));
        RCU(cudaMemcpyAsync(r->thr.data() + off, dthr, nb, cudaMemcpyDeviceToHost, s));
        RCU(cudaMemcpyAsync(&bumped, next, 8, cudaMemcpyDeviceToHost, s));
        RCU(cudaMemcpyAsync(&err, misc, 4, cudaMemcpyDeviceToHost, s));
        RCU(cudaStreamSynchronize(s));
        if (err) {
            st = shg_set_error(SHG_ERR_CUDA, "retrieval solution check failed");
            goto done;
        }
        r->lv.buckets[level] = nb;
        r->lv.first[level] = off;
        r->lv.count = ++level;
        in_keys = ka;  // the bumped keys are the next level's input; the other pair takes its bumps
        in_bits = ba;
        std::swap(ka, kb);
        std::swap(ba, bb);
        cur_n = bumped;
    }
    RCU(cudaEventRecord(e1, s));
    RCU(cudaEventSynchronize(e1));
    RCU(cudaEventElapsedTime(&r->build_ms, e0, e1));
    st = ret_upload(r);
done:
    if (own) {
        cudaStreamSynchronize(s);
        cudaFree(own);
    }
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    if (st != SHG_OK) {
        delete r;
        return st;
    }
    *out = r;
    return SHG_OK;
}

} // namespace

namespace shg {
cudaStream_t engine_stream(shg_engine *e, int *device);

// For the device query: a build on another object's stream, and the structure's device arrays.
shg_status retrieval_build_on(int device, cudaStream_t s, const uint64_t *d_keys, const uint8_t *d_bits, uint64_t n,
                              shg_retrieval **out) {
    return ret_build(nullptr, device, s, d_keys, d_bits, n, out);
}
const RetLevels *retrieval_device_view(const shg_retrieval *r, const uint64_t **sol, const uint8_t **thr) {
    *sol = r->d_sol;
    *thr = r->d_thr;
    return r->d_lv;
}
} // namespace shg

extern "C" {

shg_status shg_retrieval_build(shg_engine *e, const uint64_t *keys, const uint8_t *bits, uint64_t n, shg_retrieval **out) {
    if (!e || !out || (n && (!keys || !bits))) return shg_set_error(SHG_ERR_ARG, "null argument");
    int device = 0;
    cudaStream_t s = engine_stream(e, &device);
    if (cudaSetDevice(device) != cudaSuccess) return shg_set_error(SHG_ERR_CUDA, "cudaSetDevice failed");
    uint64_t *dk = nullptr;
    uint8_t *db = nullptr;
    shg_status st = SHG_OK;
    cudaError_t err = cudaSuccess;
    dk = (uint64_t *)engine_scratch(e, 1, std::max<uint64_t>(n, 1) * 8, err);
    RCU(err);
    db = (uint8_t *)engine_scratch(e, 2, std::max<uint64_t>(n, 1), err);
    RCU(err);
    if (n) {
        RCU(cudaMemcpyAsync(dk, keys, n * 8, cudaMemcpyHostToDevice, s));
        RCU(cudaMemcpyAsync(db, bits, n, cudaMemcpyHostToDevice, s));
    }
    st = ret_build(e, device, s, dk, db, n, out);
done:
    return st;
}

shg_status shg_retrieval_build_device(shg_engine *e, const uint64_t *d_keys, const uint8_t *d_bits, uint64_t n,
                                      shg_retrieval **out) {
    if (!e || !out || (n && (!d_keys || !d_bits))) return shg_set_error(SHG_ERR_ARG, "null argument");
    int device = 0;
    cudaStream_t s = engine_stream(e, &device);
    if (cudaSetDevice(device) != cudaSuccess) return shg_set_error(SHG_ERR_CUDA, "cudaSetDevice failed");
    return ret_build(e, device, s, d_keys, d_bits, n, out);
}

shg_status shg_retrieval_load(const uint64_t *level_buckets, uint32_t levels, const uint64_t *sol, const uint8_t *thr,
                              uint64_t n, shg_retrieval **out) {
    if (!out || (levels && (!level_buckets || !sol || !thr))) return shg_set_error(SHG_ERR_ARG, "null argument");
    if (levels > (uint32_t)kRetMaxLevels) return shg_set_error(SHG_ERR_ARG, "too many retrieval levels");
    shg_retrieval *r = new shg_retrieval();
    r->device = -1;  // host queries only
    r->n = n;
    uint64_t total = 0;
    for (uint32_t l = 0; l < levels; l++) {
        if (!level_buckets[l]) {
            delete r;
            return shg_set_error(SHG_ERR_ARG, "a retrieval level has no buckets");
        }
        r->lv.buckets[l] = level_buckets[l];
        r->lv.first[l] = total;
        total += level_buckets[l];
    }
    r->lv.count = (int)levels;
    r->sol.assign(sol, sol + total * kRetWords);
    r->thr.assign(thr, thr + total);
    *out = r;
    return SHG_OK;
}

void shg_retrieval_destroy(shg_retrieval *r) { delete r; }

shg_status shg_retrieval_query(const shg_retrieval *r, const uint64_t *keys, uint64_t n, uint8_t *out) {
    if (!r || (n && (!keys || !out))) return shg_set_error(SHG_ERR_ARG, "null argument");
    for (uint64_t i = 0; i < n; i++) out[i] = (uint8_t)ret_lookup(r->lv, r->sol.data(), r->thr.data(), keys[i]);
    return SHG_OK;
}

shg_status shg_retrieval_query_device(shg_retrieval *r, const uint64_t *d_keys, uint64_t n, uint8_t *d_out) {
    if (!r || (n && (!d_keys || !d_out))) return shg_set_error(SHG_ERR_ARG, "null argument");
    if (r->device < 0 || !r->d_sol) return shg_set_error(SHG_ERR_ARG, "a loaded retrieval structure has no device copy");
    shg_status st = SHG_OK;
    cudaEvent_t a = nullptr, b = nullptr;
    RCU(cudaSetDevice(r->device));
    RCU(cudaEventCreate(&a));
    RCU(cudaEventCreate(&b));
    RCU(cudaEventRecord(a, 0));
    if (n) k_ret_query<<<ret_grid(n, 256), 256>>>(r->lv, r->d_sol, r->d_thr, d_keys, n, d_out);
    RCU(cudaGetLastError());
    RCU(cudaEventRecord(b, 0));
    RCU(cudaEventSynchronize(b));
    RCU(cudaEventElapsedTime(&r->query_ms, a, b));
done:
    if (a) cudaEventDestroy(a);
    if (b) cudaEventDestroy(b);
    return st;
}

uint32_t shg_retrieval_levels(const shg_retrieval *r) { return r ? (uint32_t)r->lv.count : 0; }
uint64_t shg_retrieval_buckets(const shg_retrieval *r, uint32_t level) {
    return r && level < (uint32_t)r->lv.count ? r->lv.buckets[level] : 0;
}
const uint64_t *shg_retrieval_solutions(const shg_retrieval *r) { return r ? r->sol.data() : nullptr; }
const uint8_t *shg_retrieval_thresholds(const shg_retrieval *r) { return r ? r->thr.data() : nullptr; }
uint64_t shg_retrieval_bits(const shg_retrieval *r) {
    if (!r) return 0;
    // per bucket 256 solution bits and an 8-bit threshold; per level a 64-bit bucket count
    return (uint64_t)r->thr.size() * (64 * kRetWords + 8) + 64ull * r->lv.count;
}
float shg_retrieval_build_ms(const shg_retrieval *r) { return r ? r->build_ms : 0.f; }
float shg_retrieval_query_ms(const shg_retrieval *r) { return r ? r->query_ms : 0.f; }

}  // extern "C"
