/*
 * TEST INFRASTRUCTURE ONLY — used to compile the reference's own sources into oracle/_ref/.
 *
 * Stand-in for the constexpr math library gcem (extlib/gcem, empty in this checkout). The
 * reference evaluates at compile time only ceil() (SplittingStrategy::lower_aggr/upper_aggr,
 * AbstractParallelRecSplit.hpp:133,135) and ceil(2.6 * sqrt(s)) (fill_bij_midstop,
 * SIMDRecSplit.hpp:127-132, which only prunes the search). The other functions are named by
 * templates that are not instantiated here (the Golomb-Rice table comes from
 * golombRiceMemo.hpp); they are implemented from their series so that the header is complete.
 */
#pragma once

#include <cstdint>
#include <limits>
#include <type_traits>

namespace gcem {

template <class T> constexpr double to_double(T x) { return static_cast<double>(x); }

// Smallest integer value not less than x.
template <class T> constexpr double ceil(T xin) {
    const double x = to_double(xin);
    if (x != x) return x;
    if (x >= 4503599627370496.0 || x <= -4503599627370496.0) return x;  // |x| >= 2^52: integral
    const double t = static_cast<double>(static_cast<int64_t>(x));      // toward zero
    return t < x ? t + 1.0 : t;
}

template <class T> constexpr double floor(T xin) {
    const double x = to_double(xin);
    const double c = ceil(x);
    return c > x ? c - 1.0 : c;
}

// Square root by Newton's iteration from a power-of-two starting point (exact for the small
// perfect squares the reference uses; at most one ulp from the true root otherwise).
template <class T> constexpr double sqrt(T xin) {
    const double x = to_double(xin);
    if (x < 0 || x != x) return std::numeric_limits<double>::quiet_NaN();
    if (x == 0 || x == std::numeric_limits<double>::infinity()) return x;
    double g = 1.0;
    while (g * g < x) g *= 2.0;
    while ((g / 2) * (g / 2) > x) g /= 2.0;
    for (int i = 0; i < 200; i++) {
        const double n = 0.5 * (g + x / g);
        if (n == g) break;
        g = n;
    }
    return g;
}

// Natural logarithm: x = m * 2^e with m in [1, 2), log(m) = 2 atanh((m - 1) / (m + 1)).
template <class T> constexpr double log(T xin) {
    const double x = to_double(xin);
    if (x < 0 || x != x) return std::numeric_limits<double>::quiet_NaN();
    if (x == 0) return -std::numeric_limits<double>::infinity();
    double m = x;
    int e = 0;
    while (m >= 2.0) { m /= 2.0; e++; }
    while (m < 1.0) { m *= 2.0; e--; }
    const double z = (m - 1.0) / (m + 1.0), z2 = z * z;
    double term = z, sum = 0.0;
    for (int k = 1; k < 200; k += 2) {
        sum += term / k;
        term *= z2;
    }
    return 2.0 * sum + e * 0.69314718055994530942;
}

template <class T> constexpr double log2(T x) { return log(x) / 0.69314718055994530942; }

// log(1 + x); the direct form is adequate away from x = 0, the series near it.
template <class T> constexpr double log1p(T xin) {
    const double x = to_double(xin);
    if (x > -1e-4 && x < 1e-4) {
        double term = x, sum = 0.0;
        for (int k = 1; k < 12; k++) {
            sum += term / k;
            term *= -x;
        }
        return sum;
    }
    return log(1.0 + x);
}

template <class T> constexpr double exp(T xin) {
    const double x = to_double(xin);
    int e = 0;
    double r = x;
    while (r > 0.5) { r -= 0.69314718055994530942; e++; }
    while (r < -0.5) { r += 0.69314718055994530942; e--; }
    double term = 1.0, sum = 1.0;
    for (int k = 1; k < 40; k++) {
        term *= r / k;
        sum += term;
    }
    while (e > 0) { sum *= 2.0; e--; }
    while (e < 0) { sum /= 2.0; e++; }
    return sum;
}

template <class T1, class T2> constexpr double pow(T1 b, T2 e) {
    if constexpr (std::is_integral_v<T2>) {
        double r = 1.0, bb = to_double(b);
        long long n = static_cast<long long>(e);
        const bool neg = n < 0;
        if (neg) n = -n;
        while (n) {
            if (n & 1) r *= bb;
            bb *= bb;
            n >>= 1;
        }
        return neg ? 1.0 / r : r;
    } else {
        return exp(to_double(e) * log(b));
    }
}

}  // namespace gcem
