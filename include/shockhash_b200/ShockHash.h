// Drop-in for the reference's include/ShockHash.h: shockhash::ShockHash<LEAF_SIZE, false> with the
// same constructors (ShockHash.h:159, :187), operator() (:199, :277), size(), getBits(),
// printBits() (:280-293). Construction runs on the B200 through libshg (link -lshg).
// ROTATION_FITTING = true selects rotation fitting for full leaves (ShockHash.h:316-399).
// Differences: the hash128_t constructor does not sort the caller's vector; num_threads is ignored
// (the reference's output does not depend on it either).
#pragma once
#include "detail.hpp"

namespace shockhash {

template <size_t LEAF_SIZE, bool ROTATION_FITTING = false>
class ShockHash : public shockhash_b200::RecSplitObject {
    static_assert(LEAF_SIZE >= 2 && LEAF_SIZE <= 60, "ShockHash leaf sizes are 2..60 (MAX_LEAF_SIZE)");

  public:
    ShockHash() {}
    ShockHash(const std::vector<std::string> &keys, const size_t bucket_size, size_t num_threads = 1)
        : RecSplitObject(ROTATION_FITTING ? SHG_SHOCKHASH_ROTATION : SHG_SHOCKHASH, (int)LEAF_SIZE, bucket_size) {
        (void)num_threads;
        build_strings(keys);
    }
    template <class H, class = std::enable_if_t<shockhash_b200::is_hash128<H>::value>>
    ShockHash(std::vector<H> &keys, const size_t bucket_size, size_t num_threads = 1)
        : RecSplitObject(ROTATION_FITTING ? SHG_SHOCKHASH_ROTATION : SHG_SHOCKHASH, (int)LEAF_SIZE, bucket_size) {
        (void)num_threads;
        build_hash(keys);
    }
    template <class H, class = std::enable_if_t<shockhash_b200::is_hash128<H>::value>>
    size_t operator()(const H &hash) { return query_hash(hash.first, hash.second); }
    size_t operator()(const std::string &key) { return query_string(key); }
    size_t operator()(const char *key) { return query_string(std::string(key)); }
    size_t size() { return RecSplitObject::size(); }
    size_t getBits() { return RecSplitObject::getBits(); }
    void printBits() { std::cout << "bits/key: " << (double)getBits() / (double)size() << std::endl; }
};

} // namespace shockhash
