// Test infrastructure only (the oracle). The reference includes ByteHamster/Util EliasFano.h
// only to obtain pasta's bit vector with rank/select (absent). This stand-in keeps the set-bit
// positions explicitly; select1(r) returns the position of the r-th set bit (1-based).
// space_usage() reports one 64-bit sample per 512 bits plus one 32-bit sample per 8192 ones,
// a stated estimate.
#pragma once
#include <cstdint>
#include <vector>
namespace pasta {
enum class OptimizedFor { DONT_CARE, ONE_QUERIES, ZERO_QUERIES };
class BitVector {
  public:
    std::vector<uint8_t> b;
    BitVector() {}
    void resize(size_t n, bool v) { b.assign(n, v ? 1 : 0); }
    size_t size() const { return b.size(); }
    uint8_t &operator[](size_t i) { return b[i]; }
    bool operator[](size_t i) const { return b[i] != 0; }
};
template <OptimizedFor O> class FlatRankSelect {
    std::vector<uint64_t> ones;
    size_t nbits;
  public:
    explicit FlatRankSelect(const BitVector &bv) : nbits(bv.size()) {
        for (size_t i = 0; i < bv.size(); i++) if (bv.b[i]) ones.push_back(i);
    }
    size_t select1(size_t rank) const { return ones.at(rank - 1); }
    size_t space_usage() const { return (nbits / 512 + 1) * 8 + (ones.size() / 8192 + 1) * 4; }
};
} // namespace pasta
