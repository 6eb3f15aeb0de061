#pragma once
// Oracle build shim (test infrastructure only).
//
// The reference's lib/kernels.cpp and lib/loki/math.hpp include <xsimd/xsimd.hpp>
// for the Fourier-domain helpers only; the time-domain FP32 path never touches
// SIMD types. xsimd is not installed on this machine, so this header supplies a
// width-1 scalar stand-in with the same names so those translation units build.
// Every operation has plain scalar semantics (a batch holds exactly one value).

#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdint>
#include <limits>
#include <mutex>
#include <cstddef>
#include <cstdlib>
#include <new>
#include <type_traits>
#include <utility>

namespace xsimd {

template <class T> struct batch {
    using value_type          = T;
    static constexpr std::size_t size = 1;
    T v{};

    batch() = default;
    batch(T x) : v(x) {} // NOLINT: implicit broadcast, as xsimd allows

    static batch load_unaligned(const T* p) { return batch(*p); }
    static batch load_aligned(const T* p) { return batch(*p); }
    void store_unaligned(T* p) const { *p = v; }
    void store_aligned(T* p) const { *p = v; }
    T get(std::size_t) const { return v; }

    batch& operator+=(const batch& o) { v += o.v; return *this; }
    batch& operator-=(const batch& o) { v -= o.v; return *this; }
    batch& operator*=(const batch& o) { v *= o.v; return *this; }
    batch& operator/=(const batch& o) { v /= o.v; return *this; }
    batch operator-() const { return batch(-v); }
};

template <class T> batch<T> operator+(batch<T> a, const batch<T>& b) { return a += b; }
template <class T> batch<T> operator-(batch<T> a, const batch<T>& b) { return a -= b; }
template <class T> batch<T> operator*(batch<T> a, const batch<T>& b) { return a *= b; }
template <class T> batch<T> operator/(batch<T> a, const batch<T>& b) { return a /= b; }

template <class T> batch<T> operator+(const T& a, const batch<T>& b) { return batch<T>(a) + b; }
template <class T> batch<T> operator-(const T& a, const batch<T>& b) { return batch<T>(a) - b; }
template <class T> batch<T> operator*(const T& a, const batch<T>& b) { return batch<T>(a) * b; }
template <class T> batch<T> operator/(const T& a, const batch<T>& b) { return batch<T>(a) / b; }
template <class T> batch<T> operator+(batch<T> a, const T& b) { return a += batch<T>(b); }
template <class T> batch<T> operator-(batch<T> a, const T& b) { return a -= batch<T>(b); }
template <class T> batch<T> operator*(batch<T> a, const T& b) { return a *= batch<T>(b); }
template <class T> batch<T> operator/(batch<T> a, const T& b) { return a /= batch<T>(b); }

template <class T> batch<T> load_unaligned(const T* p) { return batch<T>(*p); }
template <class T> batch<T> load_aligned(const T* p) { return batch<T>(*p); }
template <class T> batch<T> broadcast(T x) { return batch<T>(x); }

template <class T> batch<T> fma(const batch<T>& a, const batch<T>& b, const batch<T>& c) {
    return batch<T>(a.v * b.v + c.v);
}
template <class T> batch<T> fms(const batch<T>& a, const batch<T>& b, const batch<T>& c) {
    return batch<T>(a.v * b.v - c.v);
}
template <class T> T reduce_add(const batch<T>& a) { return a.v; }

template <class T> batch<T> remainder(const batch<T>& a, const batch<T>& b) {
    return batch<T>(std::remainder(a.v, b.v));
}
template <class T> std::pair<batch<T>, batch<T>> sincos(const batch<T>& a) {
    return {batch<T>(std::sin(a.v)), batch<T>(std::cos(a.v))};
}
template <class T> batch<T> sqrt(const batch<T>& a) { return batch<T>(std::sqrt(a.v)); }
template <class T> batch<T> abs(const batch<T>& a) { return batch<T>(std::abs(a.v)); }
template <class T> batch<T> max(const batch<T>& a, const batch<T>& b) {
    return batch<T>(a.v > b.v ? a.v : b.v);
}
template <class T> batch<T> min(const batch<T>& a, const batch<T>& b) {
    return batch<T>(a.v < b.v ? a.v : b.v);
}

// Allocator with 64-byte alignment, the only property the callers rely on.
template <class T> struct aligned_allocator {
    using value_type = T;
    aligned_allocator() noexcept = default;
    template <class U> aligned_allocator(const aligned_allocator<U>&) noexcept {}
    T* allocate(std::size_t n) {
        void* p = ::operator new(n * sizeof(T), std::align_val_t(64));
        return static_cast<T*>(p);
    }
    void deallocate(T* p, std::size_t) noexcept {
        ::operator delete(p, std::align_val_t(64));
    }
    template <class U> struct rebind { using other = aligned_allocator<U>; };
};
template <class T, class U>
bool operator==(const aligned_allocator<T>&, const aligned_allocator<U>&) { return true; }
template <class T, class U>
bool operator!=(const aligned_allocator<T>&, const aligned_allocator<U>&) { return false; }

} // namespace xsimd
