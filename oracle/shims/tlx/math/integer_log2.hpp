// Test infrastructure only (the oracle). Stand-in for tlx integer_log2_floor (absent).
#pragma once
#include <cstdint>
namespace tlx {
template <typename T> constexpr unsigned integer_log2_floor(T i) {
    unsigned p = 0;
    while (i >= 2) { i /= 2; p++; }
    return p;
}
} // namespace tlx
