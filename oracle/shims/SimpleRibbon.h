// Test infrastructure only (the oracle). Stand-in for SimpleRibbon (extlib/simpleRibbon absent).
// An exact retrieval map: retrieve(key) returns the stored value for every key that was inserted
// (0 for absent keys), so operator() of the reference answers exactly as with a real ribbon.
// sizeBytes() reports ceil(n * bits / 8), a stated estimate (real ribbons carry a few percent of
// overhead; parity with upstream sizes is unpinned).
#pragma once
#include <cstdint>
#include <vector>
#include <algorithm>
#include <utility>

template <size_t bits, size_t coeffBits, typename ResultRow = uint8_t> class SimpleRibbon {
  public:
    std::vector<std::pair<uint64_t, uint8_t>> input;   // as given, in insertion order
    std::vector<std::pair<uint64_t, uint8_t>> sorted;  // sorted by key for lookups
    SimpleRibbon() {}
    explicit SimpleRibbon(std::vector<std::pair<uint64_t, uint8_t>> &data) : input(data), sorted(data) {
        std::sort(sorted.begin(), sorted.end());
    }
    size_t retrieve(uint64_t key) const {
        auto it = std::lower_bound(sorted.begin(), sorted.end(), std::make_pair(key, (uint8_t)0));
        if (it != sorted.end() && it->first == key) return it->second & ((1u << bits) - 1);
        return 0;
    }
    size_t sizeBytes() const { return (sorted.size() * bits + 7) / 8; }
};
