// Format of the device retrieval structure (shg_retrieval.cu), shared with the device query.
//
//   level l: key -> h = remix(key + 0x9E3779B97F4A7C15 * (l + 1)); bucket = fastrange64(h, B_l);
//   priority p = (h >> 8) & 127. A bucket keeps the keys with p < thr[bucket] and stores a 256-bit
//   vector s with parity(row(h) & s) = bit for each of them, row(h) being four remix words of h.
//   Keys with p >= thr go to level l + 1.
#pragma once
#include <cstdint>
#include "shg_common.cuh"

namespace shg {

constexpr int kRetWords = 4;                 // 256 columns per bucket
constexpr int kRetRows = 64 * kRetWords;     // row capacity of the solver
constexpr uint32_t kRetLoad = 240;           // mean keys per bucket
constexpr uint32_t kRetCap = 248;            // most keys a bucket keeps (8 spare columns)
constexpr uint32_t kRetPrio = 128;           // priority values
constexpr int kRetMaxLevels = 40;

SHG_HD uint64_t ret_hash(uint64_t key, int level) {
    return remix(key + 0x9E3779B97F4A7C15ull * (uint64_t)(level + 1));
}
SHG_HD uint32_t ret_prio(uint64_t h) { return (uint32_t)(h >> 8) & (kRetPrio - 1); }
SHG_HD uint64_t ret_row_word(uint64_t h, int i) { return remix(h + 0xD6E8FEB86659FD93ull * (uint64_t)(i + 1)); }
SHG_HD uint32_t ret_popc(uint64_t x) {
#ifdef __CUDA_ARCH__
    return (uint32_t)__popcll(x);
#else
    return (uint32_t)__builtin_popcountll(x);
#endif
}
SHG_HD uint32_t ret_parity(uint64_t h, const uint64_t *s) {
    uint32_t c = 0;
    for (int i = 0; i < kRetWords; i++) c += ret_popc(ret_row_word(h, i) & s[i]);
    return c & 1;
}

struct RetLevels {  // per level: bucket count and first bucket in the concatenated arrays
    uint64_t buckets[kRetMaxLevels];
    uint64_t first[kRetMaxLevels];
    int count;
};

SHG_HD uint32_t ret_lookup(const RetLevels &lv, const uint64_t *sol, const uint8_t *thr, uint64_t key) {
    for (int l = 0; l < lv.count; l++) {
        const uint64_t h = ret_hash(key, l);
        const uint64_t b = lv.first[l] + fastrange64(h, lv.buckets[l]);
        if (ret_prio(h) < thr[b]) return ret_parity(h, sol + b * kRetWords);
    }
    return 0;  // not a key of the input set
}

} // namespace shg
