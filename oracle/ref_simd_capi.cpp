// Test infrastructure only (the oracle). Never linked into the shipped library.
//
// C entry points over the UNMODIFIED reference header include/SIMDShockHash.hpp (the class the
// reference's SIMD benchmark builds as its ShockHash<l>, benchmark/benchmark_construction.cpp:8-13),
// compiled with -DSIMD against the restated third-party stand-ins in oracle/shims/, vectorclass
// included (oracle/shims/vectorclass.h). The recipe builds it twice, for 4 and for 8 lanes of
// 64 bits (the AVX2 and AVX-512 widths -march=native gives), so that the tests can check that the
// format does not depend on the lane count. Entry points mirror oracle/ref_capi.cpp with the
// prefix refsimd_; `rotation` selects SIMDShockHash<leaf, true>.
//
// The private static split hash (remixAndRemap) is reached with `#define private public`, applied
// only after every standard and stand-in header has been included, so the reference sources
// themselves stay untouched.
#include <algorithm>
#include <array>
#include <cassert>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstddef>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <experimental/simd>
#include <fstream>
#include <iostream>
#include <map>
#include <memory>
#include <mutex>
#include <queue>
#include <unordered_map>
#include <utility>
#include <span>
#include <string>
#include <thread>
#include <variant>
#include <vector>
#include <vectorclass.h>
#include <sux/util/Vector.hpp>
#include <sux/support/common.hpp>
#include <sux/function/RecSplit.hpp>
#include <sux/function/DoubleEF.hpp>
#include <sux/function/RiceBitVector.hpp>
#include <SimpleRibbon.h>
#include <bytehamster/util/Function.h>
#include <bytehamster/util/MurmurHash64.h>
#include <bytehamster/util/IntVector.h>
#include <bytehamster/util/EliasFano.h>
#include <tlx/math/integer_log2.hpp>

#define private public
#include <SIMDShockHash.hpp>
#undef private

using shockhash::hash128_t;

namespace {

struct RefBase {
    virtual ~RefBase() {}
    virtual size_t desc_words() = 0;
    virtual const uint64_t *desc_data() = 0;
    virtual const std::vector<uint64_t> &size_acc() = 0;
    virtual const std::vector<uint64_t> &pos_acc() = 0;
    virtual const std::vector<std::pair<uint64_t, uint8_t>> &ribbon_input() = 0;
    virtual uint64_t query_hash(uint64_t first, uint64_t second) = 0;
    virtual uint64_t query_str(const char *p, size_t len) = 0;
    virtual uint64_t bits() = 0;
    virtual uint64_t nbuckets() = 0;
};

// SIMDShockHash's data members are private (declared before any access specifier): an explicit
// template instantiation may name private members, and it defines a friend accessor for each.
template <class Tag, typename Tag::type M> struct Rob {
    friend typename Tag::type get(Tag) { return M; }
};
template <class C, class T, int K> struct MemberTag {
    using type = T C::*;
    friend type get(MemberTag);
};
using RBV = shockhash::RiceBitVector<sux::util::AllocType::MALLOC>;
using EF = sux::function::DoubleEF<sux::util::AllocType::MALLOC>;
template <size_t L> using RibbonOf = SimpleRibbon<1, (L > 24) ? 128 : 64>;
template <class C> using DescTag = MemberTag<C, RBV, 0>;
template <class C> using EfTag = MemberTag<C, EF, 1>;
template <class C, size_t L> using RibbonTag = MemberTag<C, RibbonOf<L>, 2>;
template <class C> using NbTag = MemberTag<C, size_t, 3>;

#define SHG_ROB_CLASS(C, L)                                                   \
    template struct Rob<DescTag<C>, &C::descriptors>;                         \
    template struct Rob<EfTag<C>, &C::ef>;                                    \
    template struct Rob<RibbonTag<C, L>, &C::ribbon>;                         \
    template struct Rob<NbTag<C>, &C::nbuckets>;

template <class T, size_t L> struct RefRS : RefBase {
    T obj;
    template <class... A> explicit RefRS(A &&...a) : obj(std::forward<A>(a)...) {}
    RBV &desc() { return obj.*get(DescTag<T>()); }
    size_t desc_words() override { return desc().data.size(); }
    const uint64_t *desc_data() override { return &desc().data; }
    const std::vector<uint64_t> &size_acc() override { return (obj.*get(EfTag<T>())).cum_keys; }
    const std::vector<uint64_t> &pos_acc() override { return (obj.*get(EfTag<T>())).position; }
    const std::vector<std::pair<uint64_t, uint8_t>> &ribbon_input() override { return (obj.*get(RibbonTag<T, L>())).input; }
    uint64_t query_hash(uint64_t first, uint64_t second) override { return obj(hash128_t(first, second)); }
    uint64_t query_str(const char *p, size_t len) override { return obj(std::string(p, len)); }
    uint64_t bits() override { return obj.getBits(); }
    uint64_t nbuckets() override { return obj.*get(NbTag<T>()); }
};

#define SHG_SIMD_LEAVES(X) X(2) X(4) X(8) X(12) X(16) X(24) X(25) X(30) X(32) X(33) X(40) X(48) X(60)
#define SHG_SIMD_ROT_LEAVES(X) X(8) X(16) X(24) X(30) X(33) X(40) X(48)
#define COMMA ,
#define X(L) SHG_ROB_CLASS(shockhash::SIMDShockHash<L COMMA false>, L)
SHG_SIMD_LEAVES(X)
#undef X
#define X(L) SHG_ROB_CLASS(shockhash::SIMDShockHash<L COMMA true>, L)
SHG_SIMD_ROT_LEAVES(X)
#undef X
#undef COMMA

RefBase *make(int rotation, int leaf, std::vector<hash128_t> &keys, size_t b, size_t threads) {
    std::span<hash128_t> s(keys);
    if (rotation) {
        switch (leaf) {
#define X(L) case L: return new RefRS<shockhash::SIMDShockHash<L, true>, L>(s, b, threads);
            SHG_SIMD_ROT_LEAVES(X)
#undef X
            default: return nullptr;
        }
    }
    switch (leaf) {
#define X(L) case L: return new RefRS<shockhash::SIMDShockHash<L, false>, L>(s, b, threads);
        SHG_SIMD_LEAVES(X)
#undef X
        default: return nullptr;
    }
}

RefBase *make_str(int rotation, int leaf, const std::vector<std::string> &keys, size_t b, size_t threads) {
    std::span<const std::string> s(keys);
    if (rotation) {
        switch (leaf) {
#define X(L) case L: return new RefRS<shockhash::SIMDShockHash<L, true>, L>(s, b, threads);
            SHG_SIMD_ROT_LEAVES(X)
#undef X
            default: return nullptr;
        }
    }
    switch (leaf) {
#define X(L) case L: return new RefRS<shockhash::SIMDShockHash<L, false>, L>(s, b, threads);
        SHG_SIMD_LEAVES(X)
#undef X
        default: return nullptr;
    }
}

} // namespace

extern "C" {

// Lanes of 64 bits this build's SIMDShockHash uses (FULL_VEC_64_COUNT, SimdUtils.h:33).
uint64_t refsimd_lanes() { return shockhash::FULL_VEC_64_COUNT; }

// SIMDShockHash<leaf, rotation> over 128-bit key hashes (SIMDShockHash.hpp:175-179); the arrays
// are not modified.
void *refsimd_build_hash(int rotation, int leaf, const uint64_t *first, const uint64_t *second, size_t n,
                         size_t bucket_size, size_t threads) {
    std::vector<hash128_t> keys(n);
    for (size_t i = 0; i < n; i++) keys[i] = hash128_t(first[i], second[i]);
    return make(rotation, leaf, keys, bucket_size, threads);
}

// Same, from string keys (SIMDShockHash.hpp:138-164); offsets has n + 1 entries.
void *refsimd_build_strings(int rotation, int leaf, const char *bytes, const uint64_t *offsets, size_t n,
                            size_t bucket_size, size_t threads) {
    std::vector<std::string> keys;
    keys.reserve(n);
    for (size_t i = 0; i < n; i++) keys.emplace_back(bytes + offsets[i], offsets[i + 1] - offsets[i]);
    return make_str(rotation, leaf, keys, bucket_size, threads);
}

// refsimd_build_strings with the wall time of the constructor call alone in *seconds (the key
// strings are made before the clock starts, as benchmark/benchmark_construction.cpp:53-56 times).
void *refsimd_build_strings_timed(int rotation, int leaf, const char *bytes, const uint64_t *offsets, size_t n,
                                  size_t bucket_size, size_t threads, double *seconds) {
    std::vector<std::string> keys;
    keys.reserve(n);
    for (size_t i = 0; i < n; i++) keys.emplace_back(bytes + offsets[i], offsets[i + 1] - offsets[i]);
    const auto t0 = std::chrono::steady_clock::now();
    RefBase *r = make_str(rotation, leaf, keys, bucket_size, threads);
    *seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    return r;
}

void refsimd_free(void *h) { delete (RefBase *)h; }
uint64_t refsimd_nbuckets(void *h) { return ((RefBase *)h)->nbuckets(); }
uint64_t refsimd_desc_words(void *h) { return ((RefBase *)h)->desc_words(); }
void refsimd_get_desc(void *h, uint64_t *out) {
    auto *r = (RefBase *)h;
    std::memcpy(out, r->desc_data(), r->desc_words() * 8);
}
void refsimd_get_acc(void *h, uint64_t *size_acc, uint64_t *pos_acc) {
    auto *r = (RefBase *)h;
    std::memcpy(size_acc, r->size_acc().data(), r->size_acc().size() * 8);
    std::memcpy(pos_acc, r->pos_acc().data(), r->pos_acc().size() * 8);
}
uint64_t refsimd_ribbon_n(void *h) { return ((RefBase *)h)->ribbon_input().size(); }
void refsimd_get_ribbon(void *h, uint64_t *keys, uint8_t *bits) {
    auto &v = ((RefBase *)h)->ribbon_input();
    for (size_t i = 0; i < v.size(); i++) { keys[i] = v[i].first; bits[i] = v[i].second; }
}
void refsimd_query_hash(void *h, const uint64_t *first, const uint64_t *second, size_t n, uint64_t *out) {
    auto *r = (RefBase *)h;
    for (size_t i = 0; i < n; i++) out[i] = r->query_hash(first[i], second[i]);
}
void refsimd_query_strings(void *h, const char *bytes, const uint64_t *offsets, size_t n, uint64_t *out) {
    auto *r = (RefBase *)h;
    for (size_t i = 0; i < n; i++) out[i] = r->query_str(bytes + offsets[i], offsets[i + 1] - offsets[i]);
}
uint64_t refsimd_get_bits(void *h) { return ((RefBase *)h)->bits(); }

// The split hash of the format (SIMDShockHash.hpp:762-766, remixAndRemap) for n values.
void refsimd_remix_and_remap(const uint64_t *x, size_t n, uint32_t range, uint32_t *out) {
    using C = shockhash::SIMDShockHash<8, false>;
    for (size_t i = 0; i < n; i++) out[i] = C::remixAndRemap(x[i], range);
}

} // extern "C"
