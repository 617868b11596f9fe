// Test infrastructure only (the oracle): the seeded key generators of the benchmark
// configurations, compiled into the oracle libraries so that the timed reference CPU run and the
// parity tests draw their keys without loading the CUDA library.
//
// All generators draw from std::mt19937_64(seed) and never return duplicate keys (the reference
// loops forever on duplicates). Definitions:
//   * uint64 keys: n draws in order; every later occurrence of an already drawn value is replaced,
//     in index order, by the next draws of the same stream that equal no value present so far.
//     Identical, draw for draw, to the CUDA library's benchmark utility shg_keys_mt19937_64.
//   * printable strings (ShockHash<30,false> configuration): per key a length 16 + (draw % 25),
//     then one draw per byte, byte = 33 + (draw % 94).
//   * Zipf-length strings (ShockHash2Flat<100> configuration): per key a length l in [8, 200]
//     with P(l) proportional to (l - 7)^-1.1, picked as the first l whose cumulative weight exceeds
//     u * total, u = (draw >> 11) * 2^-53; then ceil(l / 8) draws whose little-endian bytes give
//     the key's bytes (NUL included), the unused high bytes of the last draw dropped.
//   Both string generators replace a later duplicate, in index order, by drawing a new key of the
//   same kind from the continuing stream until it differs from every key present.
#pragma once
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <random>
#include <set>
#include <string>
#include <vector>

namespace shg_oracle_keys {

inline void keys_u64(uint64_t seed, uint64_t n, uint64_t *out) {
    std::mt19937_64 rng(seed);
    for (uint64_t i = 0; i < n; i++) out[i] = rng();
    std::vector<std::pair<uint64_t, uint64_t>> vi(n);
    for (uint64_t i = 0; i < n; i++) vi[i] = {out[i], i};
    std::sort(vi.begin(), vi.end());
    std::vector<uint64_t> dup;  // indices of later occurrences
    for (uint64_t i = 1; i < n; i++)
        if (vi[i].first == vi[i - 1].first) dup.push_back(vi[i].second);
    if (dup.empty()) return;
    std::sort(dup.begin(), dup.end());
    std::vector<uint64_t> present(n);
    for (uint64_t i = 0; i < n; i++) present[i] = vi[i].first;
    for (uint64_t i : dup) {
        for (;;) {
            const uint64_t v = rng();
            auto it = std::lower_bound(present.begin(), present.end(), v);
            if (it != present.end() && *it == v) continue;
            present.insert(it, v);
            out[i] = v;
            break;
        }
    }
}

inline std::string draw_printable(std::mt19937_64 &rng) {
    const uint64_t len = 16 + rng() % 25;
    std::string s(len, '\0');
    for (uint64_t j = 0; j < len; j++) s[j] = (char)(33 + rng() % 94);
    return s;
}

struct ZipfLengths {
    std::vector<double> cum;  // cum[j] = sum of weights of lengths 8 .. 8 + j
    ZipfLengths() {
        double t = 0;
        for (int l = 8; l <= 200; l++) {
            t += std::pow((double)(l - 7), -1.1);
            cum.push_back(t);
        }
    }
    uint64_t draw(std::mt19937_64 &rng) const {
        const double u = (double)(rng() >> 11) * 0x1.0p-53 * cum.back();
        const size_t j = std::upper_bound(cum.begin(), cum.end(), u) - cum.begin();
        return 8 + std::min<size_t>(j, cum.size() - 1);
    }
};

inline std::string draw_zipf(std::mt19937_64 &rng, const ZipfLengths &z) {
    const uint64_t len = z.draw(rng);
    std::string s(len, '\0');
    for (uint64_t j = 0; j < len; j += 8) {
        const uint64_t w = rng();
        for (uint64_t b = 0; b < 8 && j + b < len; b++) s[j + b] = (char)((w >> (8 * b)) & 0xFF);
    }
    return s;
}

// kind 0: printable, 1: Zipf lengths. Later duplicates redrawn as described above.
inline std::vector<std::string> strings(int kind, uint64_t seed, uint64_t n) {
    std::mt19937_64 rng(seed);
    ZipfLengths z;
    std::vector<std::string> v(n);
    for (uint64_t i = 0; i < n; i++) v[i] = kind == 0 ? draw_printable(rng) : draw_zipf(rng, z);
    std::vector<uint64_t> order(n);
    for (uint64_t i = 0; i < n; i++) order[i] = i;
    std::sort(order.begin(), order.end(), [&](uint64_t a, uint64_t b) { return v[a] != v[b] ? v[a] < v[b] : a < b; });
    std::vector<uint64_t> dup;
    for (uint64_t i = 1; i < n; i++)
        if (v[order[i]] == v[order[i - 1]]) dup.push_back(order[i]);
    if (dup.empty()) return v;
    std::sort(dup.begin(), dup.end());
    std::set<std::string> present(v.begin(), v.end());
    for (uint64_t i : dup) {
        for (;;) {
            std::string s = kind == 0 ? draw_printable(rng) : draw_zipf(rng, z);
            if (present.insert(s).second) {
                v[i] = std::move(s);
                break;
            }
        }
    }
    return v;
}

// Two-call protocol for the C entry points: total byte count first (bytes == nullptr), then the
// bytes and the n + 1 offsets. Keys are regenerated on each call (deterministic).
inline uint64_t strings_packed(int kind, uint64_t seed, uint64_t n, char *bytes, uint64_t *offsets) {
    const std::vector<std::string> v = strings(kind, seed, n);
    uint64_t total = 0;
    for (const auto &s : v) total += s.size();
    if (!bytes) return total;
    uint64_t o = 0;
    for (uint64_t i = 0; i < n; i++) {
        offsets[i] = o;
        std::memcpy(bytes + o, v[i].data(), v[i].size());
        o += v[i].size();
    }
    offsets[n] = o;
    return total;
}

} // namespace shg_oracle_keys

// Exported under a library prefix (ref_ / port_).
#define SHG_ORACLE_KEYGEN_EXPORTS(P)                                                                       \
    extern "C" void P##keys_mt19937_64(uint64_t seed, uint64_t n, uint64_t *out) {                         \
        shg_oracle_keys::keys_u64(seed, n, out);                                                           \
    }                                                                                                      \
    extern "C" uint64_t P##strings_mt19937_64(int kind, uint64_t seed, uint64_t n, char *bytes,            \
                                              uint64_t *offsets) {                                         \
        return shg_oracle_keys::strings_packed(kind, seed, n, bytes, offsets);                             \
    }
