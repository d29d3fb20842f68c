// Clopper-Pearson binomial confidence bounds (reference: include/state.h:134-151,
// which calls boost::math::quantile of a beta distribution).
//
// The beta quantile is computed here from its definition: the regularized incomplete
// beta function I_x(a, b) is evaluated with its continued fraction (Abramowitz &
// Stegun 26.5.8, modified Lentz evaluation) and inverted by Newton steps safeguarded by
// bisection. The k = 0 upper bound and the k = n lower bound have closed forms. Results
// are memoised per (k, n, alpha) because the certified-loss scan asks for the same
// cumulative counts again and again.
#pragma once

#include <cmath>
#include <cstdint>
#include <cstring>
#include <unordered_map>

#if defined(__CUDACC__)
#define DR_HD __host__ __device__
#else
#define DR_HD
#endif

namespace dr
{

// The quantile functions below compile for the host (the host tail of the control step)
// and for the device (the device tail, finish_kernels.cu); both use the C math library's
// double-precision functions by their global names.
namespace cpdetail
{
DR_HD inline double betacf(double a, double b, double x)
{
    const double tiny = 1e-300;
    double qab = a + b, qap = a + 1.0, qam = a - 1.0;
    double c = 1.0, d = 1.0 - qab * x / qap;
    if (::fabs(d) < tiny)
        d = tiny;
    d = 1.0 / d;
    double h = d;
    for (int m = 1; m <= 20000; m++)
    {
        int m2 = 2 * m;
        double aa = m * (b - m) * x / ((qam + m2) * (a + m2));
        d = 1.0 + aa * d;
        if (::fabs(d) < tiny)
            d = tiny;
        c = 1.0 + aa / c;
        if (::fabs(c) < tiny)
            c = tiny;
        d = 1.0 / d;
        h *= d * c;
        aa = -(a + m) * (qab + m) * x / ((a + m2) * (qap + m2));
        d = 1.0 + aa * d;
        if (::fabs(d) < tiny)
            d = tiny;
        c = 1.0 + aa / c;
        if (::fabs(c) < tiny)
            c = tiny;
        d = 1.0 / d;
        double del = d * c;
        h *= del;
        if (::fabs(del - 1.0) < 1e-16)
            break;
    }
    return h;
}

DR_HD inline double lbeta(double a, double b)
{
    return ::lgamma(a) + ::lgamma(b) - ::lgamma(a + b);
}

// I_x(a, b)
DR_HD inline double ibeta(double a, double b, double x)
{
    if (x <= 0.0)
        return 0.0;
    if (x >= 1.0)
        return 1.0;
    double bt = ::exp(a * ::log(x) + b * ::log1p(-x) - lbeta(a, b));
    if (x < (a + 1.0) / (a + b + 2.0))
        return bt * betacf(a, b, x) / a;
    return 1.0 - bt * betacf(b, a, 1.0 - x) / b;
}

// x with I_x(a, b) = p
DR_HD inline double ibeta_inv(double a, double b, double p)
{
    if (p <= 0.0)
        return 0.0;
    if (p >= 1.0)
        return 1.0;
    double lo = 0.0, hi = 1.0;
    double x = a / (a + b);
    const double lb = lbeta(a, b);
    for (int it = 0; it < 200; it++)
    {
        double f = ibeta(a, b, x) - p;
        if (f == 0.0)
            return x;
        if (f < 0.0)
            lo = x;
        else
            hi = x;
        double logpdf = (a - 1.0) * ::log(x) + (b - 1.0) * ::log1p(-x) - lb;
        double pdf = ::exp(logpdf);
        double xn = (pdf > 0.0 && isfinite(pdf)) ? x - f / pdf : -1.0;
        if (!(xn > lo && xn < hi))
            xn = 0.5 * (lo + hi);
        if (::fabs(xn - x) <= 1e-16 * ::fmax(x, 1e-300) || hi - lo <= 1e-17)
            return xn;
        x = xn;
    }
    return x;
}
// quantile(beta(k, n-k+1), alpha), 0 for k == 0 (state.h:134-141)
DR_HD inline double cpLower(uint32_t k, uint32_t n, double alpha)
{
    if (k == 0)
        return 0.0;
    if (k == n)
        return ::pow(alpha, 1.0 / (double)n);
    return ibeta_inv((double)k, (double)(n - k + 1), alpha);
}

// quantile(beta(k+1, n-k), 1-alpha), 1 for k == n (state.h:144-151)
DR_HD inline double cpUpper(uint32_t k, uint32_t n, double alpha)
{
    if (k == n)
        return 1.0;
    if (k == 0)
        return -::expm1(::log(alpha) / (double)n);
    return ibeta_inv((double)(k + 1), (double)(n - k), 1.0 - alpha);
}
} // namespace cpdetail

class ClopperPearson
{
  public:
    // quantile(beta(k, n-k+1), alpha), 0 for k == 0 (state.h:134-141)
    double lower(uint32_t k, uint32_t n, double alpha)
    {
        if (k == 0)
            return 0.0;
        return memo(0, k, n, alpha, [&] { return cpdetail::cpLower(k, n, alpha); });
    }
    // quantile(beta(k+1, n-k), 1-alpha), 1 for k == n (state.h:144-151)
    double upper(uint32_t k, uint32_t n, double alpha)
    {
        if (k == n)
            return 1.0;
        return memo(1, k, n, alpha, [&] { return cpdetail::cpUpper(k, n, alpha); });
    }

  private:
    template <typename F> double memo(int which, uint32_t k, uint32_t n, double alpha, F f)
    {
        uint64_t ab;
        std::memcpy(&ab, &alpha, 8);
        uint64_t key = ((uint64_t)which << 63) ^ ((uint64_t)k << 32) ^ (uint64_t)n ^ (ab * 0x9E3779B97F4A7C15ull);
        auto it = cache_.find(key);
        if (it != cache_.end() && it->second.k == k && it->second.n == n && it->second.alpha == alpha && it->second.which == which)
            return it->second.v;
        double v = f();
        if (cache_.size() > 65536)
            cache_.clear();
        cache_[key] = Entry{k, n, alpha, which, v};
        return v;
    }
    struct Entry
    {
        uint32_t k, n;
        double alpha;
        int which;
        double v;
    };
    std::unordered_map<uint64_t, Entry> cache_;
};

} // namespace dr
