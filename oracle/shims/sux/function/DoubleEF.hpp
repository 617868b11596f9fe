// Test infrastructure only (the oracle). Stand-in for sux::function::DoubleEF (absent).
// Stores the two monotone sequences (cumulative bucket sizes and bucket bit positions) plainly;
// get() returns exactly what the real structure decodes. The reported bit counts use the
// textbook Elias-Fano size  (n+1)*L + (n+1) + (u >> L) + 1,  L = floor(log2(u/(n+1))),  which is
// a stated estimate, not the sux layout (parity of these two numbers with upstream is unpinned).
#pragma once
#include <cstdint>
#include <vector>
#include <sux/util/Vector.hpp>

namespace sux::function {

inline uint64_t shg_ef_bits(const std::vector<uint64_t> &v) {
    if (v.empty()) return 0;
    uint64_t n1 = v.size();
    uint64_t u = v.back() + 1;
    uint64_t q = u / n1;
    uint64_t L = 0;
    while (q > 1) { q >>= 1; L++; }
    return n1 * L + n1 + (u >> L) + 1;
}

template <util::AllocType AT = util::AllocType::MALLOC> class DoubleEF {
  public:
    std::vector<uint64_t> cum_keys, position;
    DoubleEF() {}
    DoubleEF(const std::vector<uint64_t> &cum_keys, const std::vector<uint64_t> &position)
        : cum_keys(cum_keys), position(position) {}
    void get(const size_t i, uint64_t &cum_keys_v, uint64_t &cum_keys_next, uint64_t &position_v) const {
        cum_keys_v = cum_keys[i];
        cum_keys_next = cum_keys[i + 1];
        position_v = position[i];
    }
    uint64_t bitCountCumKeys() const { return shg_ef_bits(cum_keys); }
    uint64_t bitCountPosition() const { return shg_ef_bits(position); }
};

} // namespace sux::function
