// Test infrastructure only (the oracle). Stand-in for sux/support/common.hpp (absent):
// rho (index of the lowest set bit), nu (population count), select64 (index of the k-th set bit).
#pragma once
#include <cstdint>
#include <cstddef>

namespace sux {
inline int rho(uint64_t word) { return __builtin_ctzll(word); }
inline int nu(uint64_t word) { return __builtin_popcountll(word); }
inline uint64_t select64(uint64_t x, uint64_t k) {
    // Position of the k-th (0-based) set bit, by clearing the k lowest set bits.
    for (uint64_t i = 0; i < k; i++) x &= x - 1;
    return (uint64_t)__builtin_ctzll(x);
}
} // namespace sux
