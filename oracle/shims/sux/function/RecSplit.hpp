// Test infrastructure only (the oracle). Stand-in for the parts of sux/function/RecSplit.hpp that
// the ShockHash reference uses (extlib/sux is absent): hash128_t, spooky(), remix(), remap16(),
// remap128(), MAX_LEVEL_TIME. The arithmetic is restated in shg_thirdparty.h.
#pragma once
#include <cassert>
#include <cstdint>
#include <cstddef>
#include <sux/util/Vector.hpp>
#include <sux/support/common.hpp>
#include "../../shg_thirdparty.h"

#ifndef MAX_LEVEL_TIME
#define MAX_LEVEL_TIME (20)
#endif

namespace sux::function {

using namespace sux::util;

struct hash128_t {
    uint64_t first, second;
    hash128_t() : first(0), second(0) {}
    hash128_t(const uint64_t first, const uint64_t second) : first(first), second(second) {}
    bool operator<(const hash128_t &o) const { return first < o.first || second < o.second; }
};

// sux's convenience wrapper: both SpookyHash state words start at `seed`, and the result is
// returned as {hash2, hash1}.
inline hash128_t spooky(const void *data, const size_t length, const uint64_t seed) {
    uint64_t h0 = seed, h1 = seed;
    shg_tp::spooky_hash128(data, length, &h0, &h1);
    return {h1, h0};
}

inline uint64_t remix(uint64_t z) { return shg_tp::remix(z); }
// Lets `max(1, size_t)` (ShockHash.h:616, ShockHash2.h:455) resolve under `using namespace sux`.
inline uint64_t max(uint64_t a, uint64_t b) { return a > b ? a : b; }
inline uint16_t remap16(uint64_t x, uint32_t n) { return shg_tp::remap16(x, n); }
inline uint64_t remap128(uint64_t x, uint64_t n) { return shg_tp::remap128(x, n); }

} // namespace sux::function

namespace sux {
using sux::function::remap16;
using sux::function::remap128;
using sux::function::remix;
} // namespace sux
