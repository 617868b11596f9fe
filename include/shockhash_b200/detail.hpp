// Shared plumbing of the C++ drop-in classes (ShockHash.h, ShockHash2.h, ShockHash2Flat.h in this
// folder): a per-thread engine on CUDA device 0 and RAII owners of the C ABI objects (shg.h).
#pragma once
#include <cstddef>
#include <cstdint>
#include <iostream>
#include <memory>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <utility>
#include <vector>
#include "../shg.h"

namespace shockhash_b200 {

struct Error : std::runtime_error {
    shg_status status;
    Error(shg_status st, const std::string &what) : std::runtime_error(what), status(st) {}
};

// True for types with integral .first and .second (sux::function::hash128_t and the like).
template <class H, class = void> struct is_hash128 : std::false_type {};
template <class H>
struct is_hash128<H, std::void_t<decltype(uint64_t(std::declval<const H &>().first)),
                                 decltype(uint64_t(std::declval<const H &>().second))>> : std::true_type {};

inline void check(shg_status st) {
    if (st != SHG_OK) throw Error(st, std::string("shg: ") + shg_last_error());
}

// One engine per host thread (an engine owns one stream and is not thread-safe).
inline shg_engine *thread_engine() {
    struct Holder {
        shg_engine *e = nullptr;
        ~Holder() { shg_engine_destroy(e); }
    };
    thread_local Holder h;
    if (!h.e) check(shg_engine_create(0, &h.e));
    return h.e;
}

struct MphfDeleter {
    void operator()(shg_mphf *f) const { shg_mphf_destroy(f); }
};
using MphfPtr = std::unique_ptr<shg_mphf, MphfDeleter>;

// Strings -> (bytes, offsets[n+1]) as the C ABI takes them.
template <class Range> inline void pack(const Range &keys, std::string &bytes, std::vector<uint64_t> &offs) {
    offs.assign(1, 0);
    for (const auto &k : keys) {
        bytes.append(k.data(), k.size());
        offs.push_back(bytes.size());
    }
}

// A built RecSplit-framework structure (ShockHash or ShockHash2) behind its query object.
class RecSplitObject {
  protected:
    MphfPtr f_;
    shg_params p_{};
    size_t n_ = 0;

    void build_from_result(shg_result &r) {
        shg_mphf *f = nullptr;
        shg_status st = shg_mphf_create(&p_, &r, &f);
        shg_result_free(&r);
        check(st);
        f_.reset(f);
        n_ = shg_mphf_size(f);
    }
    template <class Range> void build_strings(const Range &keys) {
        std::string bytes;
        std::vector<uint64_t> offs;
        pack(keys, bytes, offs);
        shg_result r;
        check(shg_build_strings(thread_engine(), &p_, bytes.data(), offs.data(), offs.size() - 1, &r));
        build_from_result(r);
    }
    // Any element type with .first / .second (sux::function::hash128_t included).
    template <class H> void build_hash(const std::vector<H> &keys) {
        std::vector<uint64_t> a(keys.size()), b(keys.size());
        for (size_t i = 0; i < keys.size(); i++) {
            a[i] = keys[i].first;
            b[i] = keys[i].second;
        }
        shg_result r;
        check(shg_build_hash128(thread_engine(), &p_, a.data(), b.data(), keys.size(), &r));
        build_from_result(r);
    }
    size_t query_hash(uint64_t first, uint64_t second) const {
        uint64_t out = 0;
        check(shg_mphf_query_hash(f_.get(), &first, &second, 1, &out));
        return out;
    }
    size_t query_string(const std::string &key) const {
        const uint64_t offs[2] = {0, key.size()};
        uint64_t out = 0;
        check(shg_mphf_query_strings(f_.get(), key.data(), offs, 1, &out));
        return out;
    }
    RecSplitObject(int variant, int leaf, size_t bucket_size) {
        p_.variant = variant;
        p_.leaf_size = leaf;
        p_.bucket_size = bucket_size;
        p_.mode = SHG_MODE_DEFAULT;
        p_.max_trials = 0;
    }
    RecSplitObject() {}

  public:
    size_t size() const { return n_; }
    size_t getBits() const { return f_ ? (size_t)shg_mphf_bits(f_.get()) : 0; }
};

} // namespace shockhash_b200
