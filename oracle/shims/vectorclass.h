// Test infrastructure only (the oracle): restated stand-in for Agner Fog's vectorclass library
// (VCL, Apache-2.0). The reference's submodule extlib/vectorclass is empty here and its revision is
// unknown, so this header restates only the classes and functions that the reference's
// SIMDShockHash.hpp, shockhash/SimdUtils.h and TinyBinaryCuckooHashTable.h (under -DSIMD) use, each
// with the meaning VCL documents, on GCC vector extensions (so that, as with VCL, every operation
// compiles to one or a few AVX2 / AVX-512 instructions):
//   * VecNuq / VecNui / VecNq / VecNc: N lanes of uint64 / uint32 / int64 / int8 with wrap-around
//     arithmetic (+, -, * keep the low bits), bitwise ops, shifts by a scalar count, comparisons
//     that give a boolean vector, load/store of N lanes, extract;
//   * construction from one scalar (broadcast), from N scalars, and between vectors of the same
//     total width (a reinterpretation of the bytes, as VCL's conversion through the register type);
//   * if_add(f, a, b) = a + (f ? b : 0); blend8/blend16<i...>(a, b) picks lane i of the
//     concatenation a:b; lookup<n>(idx, table) = table[idx] for n <= N, reading one vector of N
//     entries from the table as VCL does (the reference pads its table for that,
//     SIMDShockHash.hpp:97-104); a / const_uint(d) is exact unsigned division by the constant d;
//   * horizontal_or, horizontal_find_first (-1 when no lane is set), horizontal_count and to_bits
//     (lane i to bit i) on boolean vectors.
// The two variable-shift intrinsics SimdUtils.h calls on its vectors (_mm{256,512}_{sllv,srlv}_epi64)
// are given as overloads on these classes with the instruction's meaning: a count of 64 or more
// gives 0. INSTRSET follows the compiler's target as VCL's instrset.h does (10 with AVX-512 F, BW,
// DQ and VL; 8 with AVX2), so SimdUtils.h picks 8 or 4 lanes of 64 bits as -march=native would.
#pragma once
#include <cstdint>
#include <cstring>
#include <type_traits>

#ifndef INSTRSET
#if defined(__AVX512VL__) && defined(__AVX512BW__) && defined(__AVX512DQ__)
#define INSTRSET 10
#elif defined(__AVX512F__)
#define INSTRSET 9
#elif defined(__AVX2__)
#define INSTRSET 8
#else
#define INSTRSET 2
#endif
#endif

namespace vcl_shim {

// Boolean vector of N lanes of S (a signed integer type): lane = -1 (true) or 0 (false), the
// result of a GCC vector comparison.
template <typename S, int N> struct VBool {
    typedef S M __attribute__((vector_size(sizeof(S) * N)));
    M m;
    VBool() : m{} {}
    explicit VBool(M x) : m(x) {}
    friend VBool operator&(const VBool &x, const VBool &y) { return VBool(x.m & y.m); }
    friend VBool operator|(const VBool &x, const VBool &y) { return VBool(x.m | y.m); }
    friend bool horizontal_or(const VBool &x) {
        S acc = 0;
        for (int i = 0; i < N; i++) acc |= x.m[i];
        return acc != 0;
    }
    friend int horizontal_find_first(const VBool &x) {
        for (int i = 0; i < N; i++)
            if (x.m[i]) return i;
        return -1;
    }
    friend uint32_t horizontal_count(const VBool &x) {
        uint32_t c = 0;
        for (int i = 0; i < N; i++) c += x.m[i] != 0;
        return c;
    }
    friend auto to_bits(const VBool &x) {
        using Bits = std::conditional_t<(N <= 8), uint8_t, std::conditional_t<(N <= 16), uint16_t,
                     std::conditional_t<(N <= 32), uint32_t, uint64_t>>>;
        Bits r = 0;
        for (int i = 0; i < N; i++) r |= (Bits)((Bits)(x.m[i] != 0) << i);
        return r;
    }
};

template <uint32_t d> struct Const_uint_t {};

template <typename T, int N> struct Vec {
    typedef T V __attribute__((vector_size(sizeof(T) * N)));
    using S = std::make_signed_t<T>;
    using Bool = VBool<S, N>;
    V v;

    Vec() : v{} {}
    Vec(T s) {  // broadcast
        for (int i = 0; i < N; i++) v[i] = s;
    }
    template <typename... A, typename = std::enable_if_t<(sizeof...(A) == N && N > 1)>>
    Vec(A... a) : v{(T)a...} {}
    template <typename U, int M, typename = std::enable_if_t<(sizeof(U) * M == sizeof(T) * N && !std::is_same_v<U, T>)>>
    explicit Vec(const Vec<U, M> &o) {  // same total width: reinterpret the bytes
        std::memcpy(&v, &o.v, sizeof(v));
    }
    static Vec raw(V x) {
        Vec r;
        r.v = x;
        return r;
    }

    Vec &load(const void *p) {
        std::memcpy(&v, p, sizeof(v));
        return *this;
    }
    void store(void *p) const { std::memcpy(p, &v, sizeof(v)); }
    T extract(int i) const { return v[i & (N - 1)]; }
    T operator[](int i) const { return v[i & (N - 1)]; }

#define SHG_VCL_BINOP(OP)                                                                   \
    friend Vec operator OP(const Vec &a, const Vec &b) { return raw(a.v OP b.v); }          \
    Vec &operator OP##=(const Vec &b) { return *this = *this OP b; }
    SHG_VCL_BINOP(+)
    SHG_VCL_BINOP(-)
    SHG_VCL_BINOP(*)
    SHG_VCL_BINOP(&)
    SHG_VCL_BINOP(|)
    SHG_VCL_BINOP(^)
#undef SHG_VCL_BINOP
    friend Vec operator>>(const Vec &a, int s) { return raw(a.v >> s); }
    friend Vec operator<<(const Vec &a, int s) { return raw(a.v << s); }
    Vec &operator>>=(int s) { return *this = *this >> s; }
    Vec &operator<<=(int s) { return *this = *this << s; }
#define SHG_VCL_CMP(OP)                                                                      \
    friend Bool operator OP(const Vec &a, const Vec &b) { return Bool((typename Bool::M)(a.v OP b.v)); }
    SHG_VCL_CMP(==)
    SHG_VCL_CMP(!=)
    SHG_VCL_CMP(<)
    SHG_VCL_CMP(<=)
    SHG_VCL_CMP(>)
    SHG_VCL_CMP(>=)
#undef SHG_VCL_CMP
    template <uint32_t d> friend Vec operator/(const Vec &a, Const_uint_t<d>) {
        static_assert(d != 0, "division by zero");
        return raw(a.v / (T)d);
    }
    friend Vec if_add(const Bool &f, const Vec &a, const Vec &b) { return raw(a.v + (b.v & (V)f.m)); }
};

// lane k of the result = lane I_k of the concatenation a:b
template <int... I, typename T, int N>
Vec<T, N> blend_lanes(const Vec<T, N> &a, const Vec<T, N> &b) {
    static_assert(sizeof...(I) == N, "one index per lane");
    static_assert(((I >= 0 && I < 2 * N) && ...), "lane indexes of a:b");
    return Vec<T, N>::raw(__builtin_shufflevector(a.v, b.v, I...));
}

// table[index] per lane: one vector of N table entries permuted by the index (n <= N), as VCL's
// lookup reads it; larger n gathers lane by lane
template <int n, typename T, int N> Vec<T, N> lookup(const Vec<T, N> &index, const T *table) {
    using V = typename Vec<T, N>::V;
    if constexpr (n <= N) {
        V t;
        std::memcpy(&t, table, sizeof(t));
        return Vec<T, N>::raw(__builtin_shuffle(t, index.v & (V)((T)(N - 1) + V{})));
    } else {
        Vec<T, N> r;
        for (int i = 0; i < N; i++) r.v[i] = table[index.v[i] < (T)n ? index.v[i] : (T)(n - 1)];
        return r;
    }
}

// variable shifts of 64-bit lanes: a count of 64 or more gives 0 (VPSLLVQ / VPSRLVQ)
template <int N> Vec<uint64_t, N> sllv64(const Vec<uint64_t, N> &x, const Vec<uint64_t, N> &c) {
    using V = typename Vec<uint64_t, N>::V;
    const V lim = (uint64_t)64 + V{};
    return Vec<uint64_t, N>::raw((x.v << (c.v & (lim - 1))) & (V)(c.v < lim));
}
template <int N> Vec<uint64_t, N> srlv64(const Vec<uint64_t, N> &x, const Vec<uint64_t, N> &c) {
    using V = typename Vec<uint64_t, N>::V;
    const V lim = (uint64_t)64 + V{};
    return Vec<uint64_t, N>::raw((x.v >> (c.v & (lim - 1))) & (V)(c.v < lim));
}

} // namespace vcl_shim

using vcl_shim::Const_uint_t;
using vcl_shim::lookup;
#define const_uint(x) Const_uint_t<(x)>()

using Vec4uq = vcl_shim::Vec<uint64_t, 4>;
using Vec8uq = vcl_shim::Vec<uint64_t, 8>;
using Vec4q = vcl_shim::Vec<int64_t, 4>;
using Vec8q = vcl_shim::Vec<int64_t, 8>;
using Vec8ui = vcl_shim::Vec<uint32_t, 8>;
using Vec16ui = vcl_shim::Vec<uint32_t, 16>;
using Vec32c = vcl_shim::Vec<int8_t, 32>;
using Vec64c = vcl_shim::Vec<int8_t, 64>;
using Vec8ib = Vec8ui::Bool;
using Vec16ib = Vec16ui::Bool;

template <int... I> inline Vec8ui blend8(const Vec8ui &a, const Vec8ui &b) { return vcl_shim::blend_lanes<I...>(a, b); }
template <int... I> inline Vec16ui blend16(const Vec16ui &a, const Vec16ui &b) { return vcl_shim::blend_lanes<I...>(a, b); }

// SIMDShockHash.hpp:296 evaluates min(_MAX_FANOUT, 5) with an unsigned and an int operand in a
// template argument, which std::min cannot deduce; this overload gives the smaller value.
constexpr uint32_t min(uint32_t a, int b) { return b < 0 || a < (uint32_t)b ? a : (uint32_t)b; }

inline Vec4uq _mm256_sllv_epi64(const Vec4uq &x, const Vec4uq &c) { return vcl_shim::sllv64(x, c); }
inline Vec4uq _mm256_srlv_epi64(const Vec4uq &x, const Vec4uq &c) { return vcl_shim::srlv64(x, c); }
inline Vec8uq _mm512_sllv_epi64(const Vec8uq &x, const Vec8uq &c) { return vcl_shim::sllv64(x, c); }
inline Vec8uq _mm512_srlv_epi64(const Vec8uq &x, const Vec8uq &c) { return vcl_shim::srlv64(x, c); }
