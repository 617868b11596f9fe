// Drop-in for the reference's include/ShockHash2Flat.h: shockhash::ShockHash2Flat<k> with the same
// constructors (ShockHash2Flat.h:60-66; the two extra arguments are ignored there too),
// operator()(const string&), (const hash128_t&) using .second, (uint64_t) (:258-277) and getBits()
// (:236-244). Construction runs on the B200 through libshg (link -lshg).
#pragma once
#include "detail.hpp"
#if __cplusplus >= 202002L
#include <span>
#endif

namespace shockhash {

template <size_t k>
class ShockHash2Flat {
    static_assert(k >= 4 && k <= 128, "ShockHash2Flat needs 4 <= k <= 128");
    struct Del {
        void operator()(shg_flat *f) const { shg_flat_destroy(f); }
    };
    std::unique_ptr<shg_flat, Del> f_;
    size_t n_ = 0;

    template <class Range> void build(const Range &keys) {
        std::string bytes;
        std::vector<uint64_t> offs;
        shockhash_b200::pack(keys, bytes, offs);
        shg_flat_result r;
        shockhash_b200::check(
            shg_build_flat_strings(shockhash_b200::thread_engine(), k, bytes.data(), offs.data(), offs.size() - 1, &r));
        shg_flat *f = nullptr;
        shg_status st = shg_flat_create(&r, &f);
        n_ = r.n;
        shg_flat_result_free(&r);
        shockhash_b200::check(st);
        f_.reset(f);
    }

  public:
#if __cplusplus >= 202002L
    explicit ShockHash2Flat(std::span<const std::string> keys) { build(keys); }
    ShockHash2Flat(std::span<const std::string> keys, size_t ignore, size_t ignore2) { (void)ignore, (void)ignore2, build(keys); }
#endif
    explicit ShockHash2Flat(const std::vector<std::string> &keys) { build(keys); }
    ShockHash2Flat(const std::vector<std::string> &keys, size_t ignore, size_t ignore2) {
        (void)ignore, (void)ignore2, build(keys);
    }
    size_t operator()(const std::string &key) const {
        const uint64_t offs[2] = {0, key.size()};
        uint64_t out = 0;
        shockhash_b200::check(shg_flat_query_strings(f_.get(), key.data(), offs, 1, &out));
        return out;
    }
    size_t operator()(uint64_t hash) const {
        uint64_t out = 0;
        shockhash_b200::check(shg_flat_query_hash(f_.get(), &hash, 1, &out));
        return out;
    }
    template <class H, class = std::enable_if_t<shockhash_b200::is_hash128<H>::value>>
    size_t operator()(const H &hash) const { return operator()((uint64_t)hash.second); }
    size_t getBits() const { return (size_t)shg_flat_bits(f_.get()); }
    void printBits() const { std::cout << "bits/key: " << (double)getBits() / (double)n_ << std::endl; }
};

} // namespace shockhash
