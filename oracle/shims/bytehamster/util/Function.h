// Test infrastructure only (the oracle). Stand-in for ByteHamster/Util Function.h (absent).
#pragma once
#include <cstdint>
#include "../../shg_thirdparty.h"
namespace bytehamster::util {
inline uint64_t remix(uint64_t z) { return shg_tp::remix(z); }
inline uint32_t fastrange32(uint32_t word, uint32_t p) { return shg_tp::fastrange32(word, p); }
template <uint32_t p> inline uint32_t fastrange32(uint32_t word) { return shg_tp::fastrange32(word, p); }
inline uint64_t fastrange64(uint64_t word, uint64_t p) { return shg_tp::fastrange64(word, p); }
inline uint16_t fastrange16(uint16_t word, uint16_t p) { return shg_tp::fastrange16(word, p); }
} // namespace bytehamster::util
