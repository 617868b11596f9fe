// Test infrastructure only (the oracle). Stand-in for ByteHamster/Util MurmurHash64.h (absent):
// MurmurHash64A with a fixed default seed (stated in shg_thirdparty.h).
#pragma once
#include <cstdint>
#include <string>
#include "../../shg_thirdparty.h"
namespace bytehamster::util {
inline uint64_t MurmurHash64(const void *key, size_t len) { return shg_tp::murmur64a(key, len, shg_tp::MURMUR64_DEFAULT_SEED); }
inline uint64_t MurmurHash64(const std::string &key) { return MurmurHash64(key.data(), key.size()); }
} // namespace bytehamster::util
