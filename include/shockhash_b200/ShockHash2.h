// Drop-in for the reference's include/ShockHash2.h: shockhash::ShockHash2<LEAF_SIZE> with the same
// constructors (ShockHash2.h:140, :167), const operator() (:178, :237), size(), getBits(),
// printBits() (:239-253). Construction runs on the B200 through libshg (link -lshg).
#pragma once
#include "detail.hpp"
#if __cplusplus >= 202002L
#include <span>
#endif

namespace shockhash {

template <size_t LEAF_SIZE>
class ShockHash2 : public shockhash_b200::RecSplitObject {
    static_assert(LEAF_SIZE >= 2 && LEAF_SIZE <= 128, "ShockHash2 leaf sizes are 2..128 (MAX_LEAF_SIZE2)");

  public:
    ShockHash2() {}
#if __cplusplus >= 202002L
    ShockHash2(std::span<const std::string> keys, const size_t bucket_size, size_t num_threads = 1)
        : RecSplitObject(SHG_SHOCKHASH2, (int)LEAF_SIZE, bucket_size) {
        (void)num_threads;
        build_strings(keys);
    }
#endif
    ShockHash2(const std::vector<std::string> &keys, const size_t bucket_size, size_t num_threads = 1)
        : RecSplitObject(SHG_SHOCKHASH2, (int)LEAF_SIZE, bucket_size) {
        (void)num_threads;
        build_strings(keys);
    }
    template <class H, class = std::enable_if_t<shockhash_b200::is_hash128<H>::value>>
    ShockHash2(std::vector<H> &keys, const size_t bucket_size, size_t num_threads = 1)
        : RecSplitObject(SHG_SHOCKHASH2, (int)LEAF_SIZE, bucket_size) {
        (void)num_threads;
        build_hash(keys);
    }
    template <class H, class = std::enable_if_t<shockhash_b200::is_hash128<H>::value>>
    size_t operator()(const H &hash) const { return query_hash(hash.first, hash.second); }
    size_t operator()(const std::string &key) const { return query_string(key); }
    size_t operator()(const char *key) const { return query_string(std::string(key)); }
    void printBits() const { std::cout << "bits/key: " << (double)getBits() / (double)size() << std::endl; }
};

} // namespace shockhash
