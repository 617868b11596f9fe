// Test infrastructure only (the oracle). Stand-in for ByteHamster/Util IntVector (absent):
// fixed-width integers; storage is one word per entry, size reported as if bit-packed.
#pragma once
#include <cstdint>
#include <vector>
namespace bytehamster::util {
template <size_t W> class IntVector {
    std::vector<uint64_t> v;
  public:
    void resize(size_t n) { v.resize(n, 0); }
    uint64_t at(size_t i) const { return v.at(i); }
    void set(size_t i, uint64_t x) { v.at(i) = x & ((W >= 64) ? ~0ull : ((1ull << W) - 1)); }
    size_t size() const { return v.size(); }
    size_t dataSizeBytes() const { return ((v.size() * W + 63) / 64) * 8; }
};
} // namespace bytehamster::util
