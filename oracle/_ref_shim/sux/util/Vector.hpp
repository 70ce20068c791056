/*
 * TEST INFRASTRUCTURE ONLY — used to compile the reference's own sources into oracle/_ref/.
 *
 * Stand-in for sux::util::Vector (extlib/sux, empty in this checkout), with the behaviour the
 * reference relies on (RiceBitVector.hpp, DoubleEF.hpp, AbstractParallelRecSplit.hpp):
 *
 *   - Vector(n) and size(n) make n elements; memory obtained by growing is zero-filled;
 *   - resize(n) sets the size to exactly n, growing the allocation geometrically when n is
 *     beyond it and never shrinking it (elements past the size keep their contents);
 *   - trimToFit() shrinks the allocation to the size;
 *   - operator& returns the element pointer (the reference writes through `&data + i`);
 *   - the stream format is the element count as one uint64 followed by the raw elements
 *     (the same format this project's library reads and writes).
 *
 * Only the MALLOC allocation type is implemented; the other enumerators exist so that code
 * naming them compiles.
 */
#pragma once

#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <iostream>
#include <new>
#include <utility>

namespace sux::util {

enum AllocType { MALLOC, SMALLPAGE, TRANSHUGEPAGE, FORCEHUGEPAGE };

template <typename T, AllocType AT = MALLOC> class Vector {
    size_t _size = 0, _capacity = 0;
    T *data = nullptr;

    void remap(size_t capacity) {
        if (capacity == _capacity) return;
        if (capacity == 0) {
            std::free(data);
            data = nullptr;
            _capacity = 0;
            return;
        }
        T *d = static_cast<T *>(std::realloc(data, capacity * sizeof(T)));
        if (d == nullptr) throw std::bad_alloc();
        if (capacity > _capacity) std::memset(static_cast<void *>(d + _capacity), 0, (capacity - _capacity) * sizeof(T));
        data = d;
        _capacity = capacity;
    }

  public:
    Vector() = default;
    explicit Vector(size_t length) { size(length); }
    Vector(const Vector &o) { *this = o; }
    Vector(Vector &&o) noexcept { swap(o); }
    ~Vector() { std::free(data); }

    Vector &operator=(const Vector &o) {
        if (this != &o) {
            remap(0);
            size(o._size);
            if (o._size) std::memcpy(static_cast<void *>(data), o.data, o._size * sizeof(T));
        }
        return *this;
    }
    Vector &operator=(Vector &&o) noexcept {
        swap(o);
        return *this;
    }
    void swap(Vector &o) noexcept {
        std::swap(_size, o._size);
        std::swap(_capacity, o._capacity);
        std::swap(data, o.data);
    }

    void trim(size_t capacity) {
        if (capacity >= _capacity) return;
        if (capacity < _size) capacity = _size;
        remap(capacity);
    }
    void trimToFit() { trim(_size); }
    void reserve(size_t capacity) {
        if (capacity > _capacity) remap(capacity);
    }
    void grow(size_t capacity) {
        if (capacity > _capacity) {
            const size_t g = _capacity + _capacity / 2 + 1;
            remap(capacity > g ? capacity : g);
        }
    }
    void resize(size_t size) {
        if (size > _capacity) grow(size);
        _size = size;
    }
    void size(size_t size) {
        reserve(size);
        _size = size;
    }
    size_t size() const { return _size; }
    size_t capacity() const { return _capacity; }

    T *p() const { return data; }
    T *operator&() const { return data; }
    T &operator[](size_t i) { return data[i]; }
    const T &operator[](size_t i) const { return data[i]; }

    size_t bitCount() const { return sizeof(Vector) * 8 + _capacity * sizeof(T) * 8; }

    friend std::ostream &operator<<(std::ostream &os, const Vector &v) {
        const uint64_t n = v._size;
        os.write(reinterpret_cast<const char *>(&n), sizeof(n));
        if (n) os.write(reinterpret_cast<const char *>(v.data), n * sizeof(T));
        return os;
    }
    friend std::istream &operator>>(std::istream &is, Vector &v) {
        uint64_t n = 0;
        is.read(reinterpret_cast<char *>(&n), sizeof(n));
        v.size(n);
        if (n) is.read(reinterpret_cast<char *>(v.data), n * sizeof(T));
        return is;
    }
};

}  // namespace sux::util
