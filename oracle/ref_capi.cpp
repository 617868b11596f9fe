// Test infrastructure only (the oracle). Never linked into the shipped library.
//
// C entry points over the UNMODIFIED reference headers (include/ShockHash.h, ShockHash2.h,
// ShockHash2Flat.h, src/ShockHash2-precompiled.cpp, src/Sorter.cpp), compiled against the
// restated third-party stand-ins in oracle/shims/. Used by the tests to pin the C restatement
// (oracle/port) and the CUDA path, to dump the construction products (Golomb-Rice words,
// bucket_size_acc, bucket_pos_acc, retrieval input) and as the timed CPU baseline.
//
// Private members are reached with `#define private public`, applied only after every standard
// and stand-in header has been included, so the reference sources themselves stay untouched.
#include <array>
#include <atomic>
#include <cassert>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstdint>
#include <cstring>
#include <experimental/simd>
#include <fstream>
#include <iostream>
#include <map>
#include <memory>
#include <mutex>
#include <span>
#include <string>
#include <thread>
#include <unordered_map>
#include <variant>
#include <vector>
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
#include "keygen.h"

#define private public
#include <ShockHash.h>
#include <ShockHash2.h>
#include <ShockHash2Flat.h>
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

// Reaching the implicitly private data members of the reference classes (declared before any
// access specifier, so `#define private public` does not cover them): an explicit template
// instantiation may name private members, and it defines a friend accessor for each.
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
using RecSplitFn = void(std::vector<uint64_t> &, std::vector<uint64_t> &, size_t, size_t, RBV::Builder &,
                        std::vector<uint32_t> &, const int, shockhash::TinyBinaryCuckooHashTable &,
                        std::vector<std::pair<uint64_t, uint8_t>> &);
template <class C> using RecSplitTag = MemberTag<C, RecSplitFn, 4>;

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

std::vector<std::string> make_strings(const char *bytes, const uint64_t *offsets, size_t n) {
    std::vector<std::string> keys;
    keys.reserve(n);
    for (size_t i = 0; i < n; i++) keys.emplace_back(bytes + offsets[i], offsets[i + 1] - offsets[i]);
    return keys;
}

#define SHG_SH1_LEAVES(X) X(2) X(3) X(4) X(5) X(6) X(7) X(8) X(10) X(12) X(13) X(16) X(20) X(24) X(25) X(30) X(32) X(33) X(40) X(48) X(60)
#define SHG_ROT_LEAVES(X) X(8) X(16) X(24) X(30) X(32) X(33) X(40) X(48)
#define SHG_SH2_LEAVES(X) X(2) X(3) X(4) X(5) X(6) X(8) X(9) X(10) X(11) X(12) X(16) X(20) X(24) X(32) X(33) X(40) X(48) X(64) X(100) X(128)

#define X(L) SHG_ROB_CLASS(shockhash::ShockHash<L COMMA false>, L) template struct Rob<RecSplitTag<shockhash::ShockHash<L COMMA false>>, &shockhash::ShockHash<L COMMA false>::recSplit>;
#define COMMA ,
SHG_SH1_LEAVES(X)
#undef X
#define X(L) SHG_ROB_CLASS(shockhash::ShockHash2<L>, L)
SHG_SH2_LEAVES(X)
#undef X
#define X(L) SHG_ROB_CLASS(shockhash::ShockHash<L COMMA true>, L)
SHG_ROT_LEAVES(X)
#undef X
#undef COMMA

RefBase *make_sh1(int leaf, std::vector<hash128_t> &keys, size_t b, size_t threads) {
    switch (leaf) {
#define X(L) case L: return new RefRS<shockhash::ShockHash<L, false>, L>(keys, b, threads);
        SHG_SH1_LEAVES(X)
#undef X
        default: return nullptr;
    }
}
RefBase *make_sh1_str(int leaf, const std::vector<std::string> &keys, size_t b, size_t threads) {
    switch (leaf) {
#define X(L) case L: return new RefRS<shockhash::ShockHash<L, false>, L>(keys, b, threads);
        SHG_SH1_LEAVES(X)
#undef X
        default: return nullptr;
    }
}
// ShockHash<leaf, true>: rotation fitting for leaves of exactly `leaf` keys (ShockHash.h:316-399).
RefBase *make_rot(int leaf, std::vector<hash128_t> &keys, size_t b, size_t threads) {
    switch (leaf) {
#define X(L) case L: return new RefRS<shockhash::ShockHash<L, true>, L>(keys, b, threads);
        SHG_ROT_LEAVES(X)
#undef X
        default: return nullptr;
    }
}
RefBase *make_rot_str(int leaf, const std::vector<std::string> &keys, size_t b, size_t threads) {
    switch (leaf) {
#define X(L) case L: return new RefRS<shockhash::ShockHash<L, true>, L>(keys, b, threads);
        SHG_ROT_LEAVES(X)
#undef X
        default: return nullptr;
    }
}
RefBase *make_sh2(int leaf, std::vector<hash128_t> &keys, size_t b, size_t threads) {
    switch (leaf) {
#define X(L) case L: return new RefRS<shockhash::ShockHash2<L>, L>(std::span<hash128_t>(keys), b, threads);
        SHG_SH2_LEAVES(X)
#undef X
        default: return nullptr;
    }
}
RefBase *make_sh2_str(int leaf, const std::vector<std::string> &keys, size_t b, size_t threads) {
    switch (leaf) {
#define X(L) case L: return new RefRS<shockhash::ShockHash2<L>, L>(std::span<const std::string>(keys), b, threads);
        SHG_SH2_LEAVES(X)
#undef X
        default: return nullptr;
    }
}

// Single original-ShockHash leaf through the reference's own recSplit leaf branch
// (ShockHash.h:404-439): returns the stored code x - start_seed[level] and the retrieval input.
template <size_t L>
uint64_t sh1_leaf(const uint64_t *keys, size_t m, int level, uint64_t *rkeys, uint8_t *rbits) {
    using C = shockhash::ShockHash<L, false>;
    C obj;
    std::vector<uint64_t> bucket(keys, keys + m), temp(shockhash::MAX_BUCKET_SIZE);
    RBV::Builder builder;
    std::vector<uint32_t> unary;
    shockhash::TinyBinaryCuckooHashTable table(L);
    std::vector<std::pair<uint64_t, uint8_t>> ribbon;
    (obj.*get(RecSplitTag<C>()))(bucket, temp, 0, m, builder, unary, level, table, ribbon);
    const int g = shockhash::bij_memo[m];
    RBV built = builder.build();
    uint64_t fixed = g ? ((&built.data)[0] & ((uint64_t(1) << g) - 1)) : 0;
    for (size_t i = 0; i < ribbon.size(); i++) { rkeys[i] = ribbon[i].first; rbits[i] = ribbon[i].second; }
    return ((uint64_t)unary.at(0) << g) | fixed;
}

// ShockHash2Flat<k> (ShockHash2Flat.h:37-302): private members reached the same way.
#define SHG_FLAT_KS(X) X(8) X(16) X(24) X(32) X(48) X(64) X(100)
template <class C> using LayerTag = MemberTag<C, std::vector<size_t>, 10>;
template <class C> using FallbackMapTag = MemberTag<C, std::map<size_t, size_t>, 11>;
template <class C, size_t K> using FallbackPhfTag = MemberTag<C, shockhash::ShockHash2<K>, 12>;
template <class C, size_t K> using FlatRibbonTag = MemberTag<C, RibbonOf<K>, 13>;
template <class C> using FreeBvTag = MemberTag<C, pasta::BitVector, 14>;
template <class C> using LayersTag = MemberTag<C, size_t, 15>;
template <class C, size_t W> using TasTag = MemberTag<C, bytehamster::util::IntVector<W>, 16>;
template <class C> using FlatNbTag = MemberTag<C, size_t, 17>;
template <size_t K> struct FlatW {
    static constexpr size_t TB = tlx::integer_log2_floor(K) - 1;
    static constexpr size_t SB = std::ceil(0.442 * K - 0.2);
    static constexpr size_t W = TB + SB;
};
#define X(K)                                                                                                            \
    template struct Rob<LayerTag<shockhash::ShockHash2Flat<K>>, &shockhash::ShockHash2Flat<K>::layerBases>;             \
    template struct Rob<FallbackMapTag<shockhash::ShockHash2Flat<K>>, &shockhash::ShockHash2Flat<K>::seedsFallback>;     \
    template struct Rob<FallbackPhfTag<shockhash::ShockHash2Flat<K>, K>, &shockhash::ShockHash2Flat<K>::fallbackPhf>;   \
    template struct Rob<FlatRibbonTag<shockhash::ShockHash2Flat<K>, K>, &shockhash::ShockHash2Flat<K>::ribbon>;         \
    template struct Rob<FreeBvTag<shockhash::ShockHash2Flat<K>>, &shockhash::ShockHash2Flat<K>::freePositionsBv>;       \
    template struct Rob<LayersTag<shockhash::ShockHash2Flat<K>>, &shockhash::ShockHash2Flat<K>::layers>;                \
    template struct Rob<FlatNbTag<shockhash::ShockHash2Flat<K>>, &shockhash::ShockHash2Flat<K>::nbuckets>;              \
    template struct Rob<TasTag<shockhash::ShockHash2Flat<K>, FlatW<K>::W>, &shockhash::ShockHash2Flat<K>::thresholdsAndSeeds>;
SHG_FLAT_KS(X)
#undef X

struct FlatBase {
    virtual ~FlatBase() {}
    virtual uint64_t query_str(const char *p, size_t len) = 0;
    virtual uint64_t bits() = 0;
    virtual void dump(std::vector<uint64_t> &layer_bases, std::vector<uint64_t> &tas, std::vector<uint64_t> &fb_buckets,
                      std::vector<uint64_t> &fb_seeds, std::vector<uint64_t> &free_positions,
                      std::vector<std::pair<uint64_t, uint8_t>> &ribbon, RefBase *&fallback, uint64_t &layers) = 0;
};
template <size_t K> struct FlatRS : FlatBase {
    using C = shockhash::ShockHash2Flat<K>;
    C obj;
    explicit FlatRS(std::span<const std::string> keys) : obj(keys) {}
    uint64_t query_str(const char *p, size_t len) override { return obj(std::string(p, len)); }
    uint64_t bits() override { return obj.getBits(); }
    void dump(std::vector<uint64_t> &layer_bases, std::vector<uint64_t> &tas, std::vector<uint64_t> &fb_buckets,
              std::vector<uint64_t> &fb_seeds, std::vector<uint64_t> &free_positions,
              std::vector<std::pair<uint64_t, uint8_t>> &ribbon, RefBase *&fallback, uint64_t &layers) override {
        for (size_t v : obj.*get(LayerTag<C>())) layer_bases.push_back(v);
        auto &iv = obj.*get(TasTag<C, FlatW<K>::W>());
        for (size_t i = 0; i < obj.*get(FlatNbTag<C>()); i++) tas.push_back(iv.at(i));
        for (auto &kv : obj.*get(FallbackMapTag<C>())) { fb_buckets.push_back(kv.first); fb_seeds.push_back(kv.second); }
        auto &bv = obj.*get(FreeBvTag<C>());
        // freePositions[i] = (position of the i-th set bit) - i  (ShockHash2Flat.h:141-144)
        for (size_t i = 0, ones = 0; i < bv.size(); i++)
            if (bv[i]) { free_positions.push_back(i - ones); ones++; }
        ribbon = (obj.*get(FlatRibbonTag<C, K>())).input;
        fallback = nullptr;
        layers = obj.*get(LayersTag<C>());
        (void)fallback;
    }
};

template <size_t L> void memo1(uint64_t *out) {
    static constexpr auto memo = shockhash::fill_golomb_rice<L>();  // evaluated at compile time, as ShockHash.h:145
    for (size_t i = 0; i < memo.size(); i++) out[i] = memo[i];
}
template <size_t L> void memo2(uint64_t *out) {
    static constexpr auto memo = shockhash::fill_golomb_rice2<L>();  // as ShockHash2.h:127
    for (size_t i = 0; i < memo.size(); i++) out[i] = memo[i];
}

} // namespace

extern "C" {

// The compile-time Golomb-Rice memo table (3000 entries) of ShockHash<leaf> (variant 1) or
// ShockHash2<leaf> (variant 2). Returns 0 when the leaf size is not instantiated here.
void *ref_flat_build_strings(int k, const char *bytes, const uint64_t *offsets, size_t n) {
    auto keys = make_strings(bytes, offsets, n);
    switch (k) {
#define X(K) case K: return new FlatRS<K>(std::span<const std::string>(keys));
        SHG_FLAT_KS(X)
#undef X
        default: return nullptr;
    }
}
void ref_flat_free(void *h) { delete (FlatBase *)h; }
uint64_t ref_flat_sizeof(int k) {
    switch (k) {
#define X(K) case K: return sizeof(shockhash::ShockHash2Flat<K>);
        SHG_FLAT_KS(X)
#undef X
        default: return 0;
    }
}
uint64_t ref_sizeof(int variant, int leaf) {
    if (variant == 1) return sizeof(shockhash::ShockHash<30, false>);
    if (variant == 3) return sizeof(shockhash::ShockHash<30, true>);
    return sizeof(shockhash::ShockHash2<64>);
}
uint64_t ref_flat_bits(void *h) { return ((FlatBase *)h)->bits(); }
void ref_flat_query_strings(void *h, const char *bytes, const uint64_t *offsets, size_t n, uint64_t *out) {
    auto *f = (FlatBase *)h;
    for (size_t i = 0; i < n; i++) out[i] = f->query_str(bytes + offsets[i], offsets[i + 1] - offsets[i]);
}
// Sizes first (sizes[0..5] = layer bases, buckets, fallback map, free positions, ribbon, layers),
// then the arrays when the pointers are non-null.
void ref_flat_dump(void *h, uint64_t *sizes, uint64_t *layer_bases, uint64_t *tas, uint64_t *fb_buckets,
                   uint64_t *fb_seeds, uint64_t *free_positions, uint64_t *rkeys, uint8_t *rbits) {
    std::vector<uint64_t> lb, t, fbb, fbs, fp;
    std::vector<std::pair<uint64_t, uint8_t>> rb;
    RefBase *fb = nullptr;
    uint64_t layers = 0;
    ((FlatBase *)h)->dump(lb, t, fbb, fbs, fp, rb, fb, layers);
    sizes[0] = lb.size(); sizes[1] = t.size(); sizes[2] = fbb.size(); sizes[3] = fp.size(); sizes[4] = rb.size();
    sizes[5] = layers;
    if (layer_bases) std::memcpy(layer_bases, lb.data(), lb.size() * 8);
    if (tas) std::memcpy(tas, t.data(), t.size() * 8);
    if (fb_buckets) std::memcpy(fb_buckets, fbb.data(), fbb.size() * 8);
    if (fb_seeds) std::memcpy(fb_seeds, fbs.data(), fbs.size() * 8);
    if (free_positions) std::memcpy(free_positions, fp.data(), fp.size() * 8);
    if (rkeys) for (size_t i = 0; i < rb.size(); i++) { rkeys[i] = rb[i].first; rbits[i] = rb[i].second; }
}

int ref_memo(int variant, int leaf, uint64_t *out) {
    if (variant == 1) {
        switch (leaf) {
#define X(L) case L: memo1<L>(out); return 1;
            SHG_SH1_LEAVES(X)
#undef X
        }
    } else {
        switch (leaf) {
#define X(L) case L: memo2<L>(out); return 1;
            SHG_SH2_LEAVES(X)
#undef X
        }
    }
    return 0;
}

// 128-bit key fingerprint as the reference computes it (ShockHash.h:129 first_hash).
void ref_spooky128(const char *bytes, const uint64_t *offsets, size_t n, uint64_t *first, uint64_t *second) {
    for (size_t i = 0; i < n; i++) {
        auto h = sux::function::spooky(bytes + offsets[i], offsets[i + 1] - offsets[i], 0);
        first[i] = h.first;
        second[i] = h.second;
    }
}

void ref_murmur64(const char *bytes, const uint64_t *offsets, size_t n, uint64_t *out) {
    for (size_t i = 0; i < n; i++) out[i] = bytehamster::util::MurmurHash64(bytes + offsets[i], offsets[i + 1] - offsets[i]);
}

// variant: 1 = ShockHash<leaf,false>, 2 = ShockHash2<leaf>. Keys given as 128-bit hashes
// (the hash128_t constructors, ShockHash.h:187 / ShockHash2.h:167; the arrays are not modified).
void *ref_build_hash(int variant, int leaf, const uint64_t *first, const uint64_t *second, size_t n,
                     size_t bucket_size, size_t threads) {
    std::vector<hash128_t> keys(n);
    for (size_t i = 0; i < n; i++) keys[i] = hash128_t(first[i], second[i]);
    if (variant == 1) return make_sh1(leaf, keys, bucket_size, threads);
    if (variant == 2) return make_sh2(leaf, keys, bucket_size, threads);
    if (variant == 3) return make_rot(leaf, keys, bucket_size, threads);
    return nullptr;
}

// Same, from string keys (ShockHash.h:159 / ShockHash2.h:140); offsets has n+1 entries.
void *ref_build_strings(int variant, int leaf, const char *bytes, const uint64_t *offsets, size_t n,
                        size_t bucket_size, size_t threads) {
    auto keys = make_strings(bytes, offsets, n);
    if (variant == 1) return make_sh1_str(leaf, keys, bucket_size, threads);
    if (variant == 2) return make_sh2_str(leaf, keys, bucket_size, threads);
    if (variant == 3) return make_rot_str(leaf, keys, bucket_size, threads);
    return nullptr;
}

// ref_build_strings with the wall time of the reference constructor alone in *seconds: the key
// strings are made before the clock starts, as the reference's own benchmark times only the
// constructor call (benchmark/benchmark_construction.cpp:53-56).
void *ref_build_strings_timed(int variant, int leaf, const char *bytes, const uint64_t *offsets, size_t n,
                              size_t bucket_size, size_t threads, double *seconds) {
    auto keys = make_strings(bytes, offsets, n);
    const auto t0 = std::chrono::steady_clock::now();
    RefBase *r = nullptr;
    if (variant == 1) r = make_sh1_str(leaf, keys, bucket_size, threads);
    if (variant == 2) r = make_sh2_str(leaf, keys, bucket_size, threads);
    if (variant == 3) r = make_rot_str(leaf, keys, bucket_size, threads);
    *seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    return r;
}

void ref_free(void *h) { delete (RefBase *)h; }
uint64_t ref_nbuckets(void *h) { return ((RefBase *)h)->nbuckets(); }
uint64_t ref_desc_words(void *h) { return ((RefBase *)h)->desc_words(); }
void ref_get_desc(void *h, uint64_t *out) {
    auto *r = (RefBase *)h;
    std::memcpy(out, r->desc_data(), r->desc_words() * 8);
}
void ref_get_acc(void *h, uint64_t *size_acc, uint64_t *pos_acc) {
    auto *r = (RefBase *)h;
    std::memcpy(size_acc, r->size_acc().data(), r->size_acc().size() * 8);
    std::memcpy(pos_acc, r->pos_acc().data(), r->pos_acc().size() * 8);
}
uint64_t ref_ribbon_n(void *h) { return ((RefBase *)h)->ribbon_input().size(); }
void ref_get_ribbon(void *h, uint64_t *keys, uint8_t *bits) {
    auto &v = ((RefBase *)h)->ribbon_input();
    for (size_t i = 0; i < v.size(); i++) { keys[i] = v[i].first; bits[i] = v[i].second; }
}
void ref_query_hash(void *h, const uint64_t *first, const uint64_t *second, size_t n, uint64_t *out) {
    auto *r = (RefBase *)h;
    for (size_t i = 0; i < n; i++) out[i] = r->query_hash(first[i], second[i]);
}
void ref_query_strings(void *h, const char *bytes, const uint64_t *offsets, size_t n, uint64_t *out) {
    auto *r = (RefBase *)h;
    for (size_t i = 0; i < n; i++) out[i] = r->query_str(bytes + offsets[i], offsets[i + 1] - offsets[i]);
}
uint64_t ref_get_bits(void *h) { return ((RefBase *)h)->bits(); }

// One bipartite leaf through the reference's plugin seam (ShockHash2-precompiled.cpp:44-47).
// Returns the leaf seed; writes m retrieval pairs in the reference's push order.
uint64_t ref_sh2_leaf(size_t m, const uint64_t *keys, uint64_t *rkeys, uint8_t *rbits) {
    std::vector<uint64_t> leaf(keys, keys + m);
    std::vector<std::pair<uint64_t, uint8_t>> ribbon;
    size_t seed = shockhash::shockhash2construct(m, leaf, ribbon);
    for (size_t i = 0; i < ribbon.size(); i++) { rkeys[i] = ribbon[i].first; rbits[i] = ribbon[i].second; }
    return seed;
}
uint64_t ref_sh2_leaf_query(size_t m, uint64_t seed, uint64_t key, uint64_t retrieved) {
    return shockhash::shockhash2query(m, seed, key, retrieved);
}

// One original-ShockHash leaf (m <= leaf) at tree depth `level`; returns the stored code.
uint64_t ref_sh1_leaf(int leaf, const uint64_t *keys, size_t m, int level, uint64_t *rkeys, uint8_t *rbits) {
    switch (leaf) {
#define X(L) case L: return sh1_leaf<L>(keys, m, level, rkeys, rbits);
        SHG_SH1_LEAVES(X)
#undef X
        default: return ~0ull;
    }
}

// Pieces of the bipartite pair test for an L-key leaf (ShockHash2-internal.h:34-44
// calculateIsolatedVertices; :510-528 the pair loop; CuckooUnionFind.h:19-42): for the hash rows of
// a new candidate `a` and an earlier one `b` (values below (L + 1) / 2), whether the isolated-vertex
// filter skips the pair and whether the union-find accepts all L edges (a[i] + L / 2, b[i]).
} // extern "C"
template <size_t L> void sh2_pair_check(const uint8_t *a, const uint8_t *b, int *skipped, int *forest) {
    shockhash::SeedCache<L, true> na, nb;
    memcpy(na.hashes, a, L);
    memcpy(nb.hashes, b, L);
    shockhash::calculateIsolatedVertices<L>(na);
    shockhash::calculateIsolatedVertices<L>(nb);
    *skipped = (na.isolatedVertices & nb.isolatedVertices) != 0;
    shockhash::CuckooUnionFind uf(L);
    uf.clear();
    size_t i = 0;
    for (; i < L; i++)
        if (!uf.unionIsStillPseudoforest((uint32_t)(a[i] + L / 2), b[i])) break;
    *forest = i == L;
}
extern "C" {
int ref_sh2_pair_check(size_t L, const uint8_t *a, const uint8_t *b, int *skipped, int *forest) {
    switch (L) {
#define X(N) case N: sh2_pair_check<N>(a, b, skipped, forest); return 1;
        X(10) X(16) X(33) X(64) X(100) X(128)
#undef X
        default: return 0;
    }
}

#ifdef STATS
// Phase times of the builds since the last call, from the reference's own STATS counters
// (ShockHash.h:37-44; ShockHash2.h:268-290, 314-388): the leaf searches and the split levels
// summed, in nanoseconds. The counters are plain globals, so builds measured this way run on one
// thread. Resets the counters to zero after reading them.
void ref_stats_times(uint64_t *leaves_ns, uint64_t *splits_ns) {
    *leaves_ns = shockhash::time_bij;
    uint64_t s = 0;
    for (int i = 0; i < MAX_LEVEL_TIME; i++) s += shockhash::time_split[i];
    *splits_ns = s;
    shockhash::time_bij = 0;
    for (int i = 0; i < MAX_LEVEL_TIME; i++) shockhash::time_split[i] = 0;
}
#endif

// The reference's ordered cuckoo insertion of m keys under one seed
// (TinyBinaryCuckooHashTable::construct / insert, TinyBinaryCuckooHashTable.h:80-106,169-198):
// 1 when every key finds a cell. Its candidate cells (getCandidateCells, :138-149) go to c1, c2.
int ref_cuckoo_construct(const uint64_t *keys, size_t m, uint64_t seed, uint32_t *c1, uint32_t *c2) {
    shockhash::TinyBinaryCuckooHashTable table(m);
    for (size_t i = 0; i < m; i++) {
        table.prepare(shockhash::HashedKey(keys[i]));
        const auto cc = shockhash::TinyBinaryCuckooHashTable::getCandidateCells(shockhash::HashedKey(keys[i]), seed, m);
        c1[i] = cc.cell1;
        c2[i] = cc.cell2;
    }
    return table.construct(seed) ? 1 : 0;
}

} // extern "C"

SHG_ORACLE_KEYGEN_EXPORTS(ref_)
