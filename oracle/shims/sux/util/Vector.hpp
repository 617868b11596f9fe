// Test infrastructure only (the oracle). Stand-in for sux::util::Vector (extlib/sux is absent).
// Semantics the reference relies on (RiceBitVector.h:53-127): `&v` yields the data pointer,
// growth zero-fills new capacity, shrinking keeps the storage, trimToFit() drops spare capacity.
#pragma once
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <iostream>
#include <algorithm>

namespace sux::util {

enum AllocType { MALLOC, SMALLPAGE, TRANSHUGEPAGE, FORCEHUGEPAGE };

template <typename T, AllocType AT = MALLOC> class Vector {
    size_t _size = 0, _capacity = 0;
    T *data = nullptr;

    void remap(size_t cap) {
        if (cap == 0) { std::free(data); data = nullptr; _capacity = 0; return; }
        T *mem = (T *)std::realloc(data, cap * sizeof(T));
        if (!mem) std::abort();
        if (cap > _capacity) std::memset((void *)(mem + _capacity), 0, (cap - _capacity) * sizeof(T));
        data = mem;
        _capacity = cap;
    }

  public:
    Vector() = default;
    explicit Vector(size_t length) { resize(length); }
    Vector(const Vector &) = delete;
    Vector &operator=(const Vector &) = delete;
    Vector(Vector &&o) noexcept : _size(o._size), _capacity(o._capacity), data(o.data) {
        o.data = nullptr; o._size = o._capacity = 0;
    }
    Vector &operator=(Vector &&o) noexcept {
        std::swap(_size, o._size); std::swap(_capacity, o._capacity); std::swap(data, o.data);
        return *this;
    }
    ~Vector() { std::free(data); }

    void resize(size_t n) {
        if (n > _capacity) remap(std::max(n, _capacity + _capacity / 2));
        _size = n;
    }
    void size(size_t n) { resize(n); }
    void reserve(size_t n) { if (n > _capacity) remap(n); }
    void trimToFit() { if (_capacity > _size) remap(_size); }
    size_t size() const { return _size; }
    size_t capacity() const { return _capacity; }
    T *p() const { return data; }
    T *operator&() const { return data; }
    T &operator[](size_t i) const { return data[i]; }
    size_t bitCount() const { return sizeof(Vector) * 8 + _capacity * sizeof(T) * 8; }

    friend std::ostream &operator<<(std::ostream &os, const Vector &v) {
        uint64_t n = v._size;
        os.write((const char *)&n, sizeof n);
        os.write((const char *)v.data, (std::streamsize)(n * sizeof(T)));
        return os;
    }
    friend std::istream &operator>>(std::istream &is, Vector &v) {
        uint64_t n = 0;
        is.read((char *)&n, sizeof n);
        v.resize(n);
        is.read((char *)v.data, (std::streamsize)(n * sizeof(T)));
        return is;
    }
};

} // namespace sux::util
