#pragma once
// Oracle build shim (test infrastructure only).
//
// The reference's lib/loki/math.hpp includes four Boost.Math headers. On the
// time-domain FP32 path only integer factorials and binomial coefficients can
// be reached; the distributions feed the Monte-Carlo threshold tables and the
// Fourier paths. Boost is not installed here, so this header provides:
//   * factorial<T>(n) and binomial_coefficient<T>(n, k): exact products from
//     the definitions (exact in double for the small arguments used);
//   * normal / chi-squared distribution types whose quantile/cdf throw, so a
//     call from an out-of-scope path fails loudly instead of returning junk.

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <limits>
#include <mutex>
#include <stdexcept>
#include <string>

namespace boost::math {

template <class T> T factorial(unsigned n) {
    double r = 1.0;
    for (unsigned i = 2; i <= n; ++i) {
        r *= static_cast<double>(i);
    }
    return static_cast<T>(r);
}

template <class T> T binomial_coefficient(unsigned n, unsigned k) {
    if (k > n) {
        return static_cast<T>(0);
    }
    if (k > n - k) {
        k = n - k;
    }
    double r = 1.0;
    for (unsigned i = 1; i <= k; ++i) {
        r = r * static_cast<double>(n - k + i) / static_cast<double>(i);
    }
    return static_cast<T>(r);
}

template <class T = double> class normal_distribution {
public:
    explicit normal_distribution(T mean = 0, T sd = 1) : m_mean(mean), m_sd(sd) {}
    T mean() const { return m_mean; }
    T standard_deviation() const { return m_sd; }

private:
    T m_mean;
    T m_sd;
};

template <class T = double> class chi_squared_distribution {
public:
    explicit chi_squared_distribution(T df) : m_df(df) {}
    T degrees_of_freedom() const { return m_df; }

private:
    T m_df;
};

template <class Dist, class T> struct complemented_shim {
    Dist dist;
    T x;
};

template <class Dist, class T> complemented_shim<Dist, T> complement(const Dist& d, const T& x) {
    return {d, x};
}

[[noreturn]] inline void oracle_shim_unavailable(const char* what) {
    throw std::logic_error(std::string("oracle shim: boost::math::") + what +
                           " is not available (off the time-domain FP32 path)");
}

template <class Dist, class T> T quantile(const Dist&, const T&) {
    oracle_shim_unavailable("quantile");
}
template <class Dist, class T> T quantile(const complemented_shim<Dist, T>&) {
    oracle_shim_unavailable("quantile(complement)");
}
template <class Dist, class T> T cdf(const Dist&, const T&) {
    oracle_shim_unavailable("cdf");
}
template <class Dist, class T> T cdf(const complemented_shim<Dist, T>&) {
    oracle_shim_unavailable("cdf(complement)");
}

} // namespace boost::math
