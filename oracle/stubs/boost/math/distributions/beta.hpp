// Test-infrastructure stand-in for boost/math/distributions/beta.hpp (boost is not
// installed in this image). It provides only what the reference's Clopper-Pearson
// bounds use (include/state.h:134-151): beta_distribution<double>(a, b) and
// quantile(dist, p).
//
// The quantile is found by plain bisection on the regularized incomplete beta
// function I_x(a, b), which is evaluated with the continued fraction of
// Abramowitz & Stegun 26.5.8 (modified Lentz evaluation). It is deliberately a
// different method from the product's own Newton/bisection solver so that the two
// can be cross-checked; both are pinned against scipy.stats.beta.ppf in tests.
#pragma once

#include <cmath>

namespace boost
{
namespace math
{
template <typename T> struct beta_distribution
{
    T a, b;
    beta_distribution(T a_, T b_) : a(a_), b(b_) {}
};

namespace detail
{
inline double betacf(double a, double b, double x)
{
    const double tiny = 1e-300;
    double qab = a + b, qap = a + 1.0, qam = a - 1.0;
    double c = 1.0, d = 1.0 - qab * x / qap;
    if (std::fabs(d) < tiny)
        d = tiny;
    d = 1.0 / d;
    double h = d;
    for (int m = 1; m <= 10000; m++)
    {
        int m2 = 2 * m;
        double aa = m * (b - m) * x / ((qam + m2) * (a + m2));
        d = 1.0 + aa * d;
        if (std::fabs(d) < tiny)
            d = tiny;
        c = 1.0 + aa / c;
        if (std::fabs(c) < tiny)
            c = tiny;
        d = 1.0 / d;
        h *= d * c;
        aa = -(a + m) * (qab + m) * x / ((a + m2) * (qap + m2));
        d = 1.0 + aa * d;
        if (std::fabs(d) < tiny)
            d = tiny;
        c = 1.0 + aa / c;
        if (std::fabs(c) < tiny)
            c = tiny;
        d = 1.0 / d;
        double del = d * c;
        h *= del;
        if (std::fabs(del - 1.0) < 1e-16)
            break;
    }
    return h;
}

inline double ibeta(double a, double b, double x)
{
    if (x <= 0.0)
        return 0.0;
    if (x >= 1.0)
        return 1.0;
    double lbt = std::lgamma(a + b) - std::lgamma(a) - std::lgamma(b) + a * std::log(x) + b * std::log1p(-x);
    double bt = std::exp(lbt);
    if (x < (a + 1.0) / (a + b + 2.0))
        return bt * betacf(a, b, x) / a;
    return 1.0 - bt * betacf(b, a, 1.0 - x) / b;
}
} // namespace detail

template <typename T> T quantile(const beta_distribution<T>& dist, T p)
{
    if (p <= 0)
        return 0;
    if (p >= 1)
        return 1;
    double lo = 0.0, hi = 1.0;
    for (int it = 0; it < 200; it++)
    {
        double mid = 0.5 * (lo + hi);
        if (detail::ibeta((double)dist.a, (double)dist.b, mid) < (double)p)
            lo = mid;
        else
            hi = mid;
        if (hi - lo < 1e-17)
            break;
    }
    return (T)(0.5 * (lo + hi));
}
} // namespace math
} // namespace boost
