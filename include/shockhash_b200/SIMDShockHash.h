// Drop-in for the reference's include/SIMDShockHash.hpp: shockhash::SIMDShockHash<LEAF_SIZE,
// ROTATION_FITTING> with the same constructors from string keys, 128-bit hashes and a stream of
// keys one per line (SIMDShockHash.hpp:138, :176, :189), operator() (:776, :853), getBits() and
// printBits() (:856-866). Construction runs on the B200 through libshg (link -lshg); the structure
// is the reference's SIMD format bit for bit, which does not depend on the host's vector width.
// Differences: num_threads is ignored (the reference's output does not depend on it either), and
// no -DSIMD or vectorclass is needed to compile this header.
#pragma once
#include <fstream>
#include "detail.hpp"
#if __cplusplus >= 202002L
#include <span>
#endif

namespace shockhash {

template <size_t LEAF_SIZE, bool ROTATION_FITTING = false>
class SIMDShockHash : public shockhash_b200::RecSplitObject {
    static_assert(LEAF_SIZE >= 2 && LEAF_SIZE <= 60, "SIMDShockHash leaf sizes are 2..60 (MAX_LEAF_SIZE)");
    static constexpr int kVariant = ROTATION_FITTING ? SHG_SIMDSHOCKHASH_ROTATION : SHG_SIMDSHOCKHASH;

  public:
    SIMDShockHash() {}
#if __cplusplus >= 202002L
    SIMDShockHash(std::span<const std::string> keys, const size_t bucket_size, size_t num_threads = 1)
        : RecSplitObject(kVariant, (int)LEAF_SIZE, bucket_size) {
        (void)num_threads;
        build_strings(keys);
    }
#endif
    SIMDShockHash(const std::vector<std::string> &keys, const size_t bucket_size, size_t num_threads = 1)
        : RecSplitObject(kVariant, (int)LEAF_SIZE, bucket_size) {
        (void)num_threads;
        build_strings(keys);
    }
    template <class H, class = std::enable_if_t<shockhash_b200::is_hash128<H>::value>>
    SIMDShockHash(std::vector<H> &keys, const size_t bucket_size, size_t num_threads = 1)
        : RecSplitObject(kVariant, (int)LEAF_SIZE, bucket_size) {
        (void)num_threads;
        build_hash(keys);
    }
    SIMDShockHash(std::ifstream &input, const size_t bucket_size, size_t num_threads = 1)
        : RecSplitObject(kVariant, (int)LEAF_SIZE, bucket_size) {
        (void)num_threads;
        std::vector<std::string> keys;
        for (std::string key; std::getline(input, key);) keys.push_back(key);
        build_strings(keys);
    }
    template <class H, class = std::enable_if_t<shockhash_b200::is_hash128<H>::value>>
    size_t operator()(const H &hash) { return query_hash(hash.first, hash.second); }
    size_t operator()(const std::string &key) { return query_string(key); }
    size_t operator()(const char *key) { return query_string(std::string(key)); }
    size_t getBits() { return RecSplitObject::getBits(); }
    void printBits() { std::cout << "bits/key: " << (double)getBits() / (double)size() << std::endl; }
};

} // namespace shockhash
