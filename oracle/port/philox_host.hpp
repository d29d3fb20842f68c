// TEST INFRASTRUCTURE (oracle). Host restatement of the Philox4x32-10 counter-based
// generator (Salmon, Moraes, Dror, Shaw, "Parallel random numbers: as easy as 1, 2, 3",
// SC'11) and of the normal variate the product draws from it. The product's device
// implementation must reproduce these bits exactly; tests check that.
//
// Normal variate: inverse normal CDF by P. J. Acklam's rational approximation
// (2003, published coefficients), evaluated in float with explicit fused
// multiply-adds; the natural log in its tails is computed from the atanh series
// log(m) = 2*atanh((m-1)/(m+1)) after an exponent split. Every float operation is
// a correctly rounded IEEE operation, so host and device agree bit for bit.
#pragma once

#include <cmath>
#include <cstdint>
#include <cstring>

namespace orc
{

struct Philox4
{
    uint32_t v[4];
};

inline Philox4 philox4x32_10(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3, uint32_t k0, uint32_t k1)
{
    const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u;
    const uint32_t W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
    for (int r = 0; r < 10; r++)
    {
        uint64_t p0 = (uint64_t)M0 * c0;
        uint64_t p1 = (uint64_t)M1 * c2;
        uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
        uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
        uint32_t n0 = hi1 ^ c1 ^ k0;
        uint32_t n1 = lo1;
        uint32_t n2 = hi0 ^ c3 ^ k1;
        uint32_t n3 = lo0;
        c0 = n0;
        c1 = n1;
        c2 = n2;
        c3 = n3;
        k0 += W0;
        k1 += W1;
    }
    return Philox4{{c0, c1, c2, c3}};
}

// Stream identifiers (the high byte of counter word 3).
enum Stream : uint32_t
{
    S_MPPI_EPS = 1,
    S_MPPI_ROLL_ENV = 2,
    S_VERIF_THETA = 3,
    S_VERIF_ENV = 4,
    S_PR_EPS = 5,
    S_PR_THETA = 6,
    S_PR_ROLL_ENV = 7,
    S_PR_CAND_ENV = 8,
    S_PR_SAFE_ENV = 9,
    S_ENV_STEP = 10,
};

inline float bits_to_float(uint32_t b)
{
    float f;
    std::memcpy(&f, &b, 4);
    return f;
}
inline uint32_t float_to_bits(float f)
{
    uint32_t b;
    std::memcpy(&b, &f, 4);
    return b;
}

// u in (0,1): (2*(w>>9)+1) * 2^-24, exact.
inline float uniform_from_word(uint32_t w)
{
    return (float)(2u * (w >> 9) + 1u) * 5.9604644775390625e-08f;
}

// log(x) for normal positive floats.
inline float series_logf(float x)
{
    uint32_t b = float_to_bits(x);
    int e = (int)(b >> 23) - 127;
    float m = bits_to_float((b & 0x007fffffu) | 0x3f800000u);
    if (m > 1.41421356f)
    {
        m = m * 0.5f;
        e += 1;
    }
    float f = m - 1.0f;
    float den = m + 1.0f;
    float z = f / den;
    float z2 = z * z;
    float p = std::fmaf(std::fmaf(std::fmaf(std::fmaf(0.0909090936f, z2, 0.111111112f), z2, 0.142857149f), z2, 0.200000003f), z2,
                        0.333333343f);
    float zz = z + z;
    float zz3 = zz * z2;
    float lm = std::fmaf(zz3, p, zz);
    return std::fmaf((float)e, 0.693147182f, lm);
}

inline float acklam_tail(float q)
{
    float num = std::fmaf(std::fmaf(std::fmaf(std::fmaf(std::fmaf(-7.784894002430293e-03f, q, -3.223964580411365e-01f), q, -2.400758277161838e+00f), q,
                                              -2.549732539343734e+00f),
                                    q, 4.374664141464968e+00f),
                          q, 2.938163982698783e+00f);
    float den = std::fmaf(std::fmaf(std::fmaf(std::fmaf(7.784695709041462e-03f, q, 3.224671290700398e-01f), q, 2.445134137142996e+00f), q,
                                    3.754408661907416e+00f),
                          q, 1.0f);
    return num / den;
}

inline float normal_from_uniform(float u)
{
    const float plow = 0.02425f;
    if (u < plow)
    {
        float q = std::sqrt(-2.0f * series_logf(u));
        return acklam_tail(q);
    }
    if (u > 1.0f - plow)
    {
        float q = std::sqrt(-2.0f * series_logf(1.0f - u));
        return -acklam_tail(q);
    }
    float q = u - 0.5f;
    float r = q * q;
    float num = std::fmaf(std::fmaf(std::fmaf(std::fmaf(std::fmaf(-3.969683028665376e+01f, r, 2.209460984245205e+02f), r, -2.759285104469687e+02f), r,
                                              1.383577518672690e+02f),
                                    r, -3.066479806614716e+01f),
                          r, 2.506628277459239e+00f);
    float den = std::fmaf(std::fmaf(std::fmaf(std::fmaf(std::fmaf(-5.447609879822406e+01f, r, 1.615858368580409e+02f), r, -1.556989798598866e+02f), r,
                                              6.680131188771972e+01f),
                                    r, -1.328068155288572e+01f),
                          r, 1.0f);
    float nq = num * q;
    return nq / den;
}

struct Key
{
    uint32_t k0, k1;
    explicit Key(uint64_t seed) : k0((uint32_t)seed), k1((uint32_t)(seed >> 32)) {}
};

inline Philox4 draw(const Key& key, uint32_t c0, uint32_t c1, uint64_t step, uint32_t stream, uint32_t sub)
{
    return philox4x32_10(c0, c1, (uint32_t)step, (stream << 24) | (sub & 0x00ffffffu), key.k0, key.k1);
}

// Sequential normal source for the in-rollout environment noise: normal j of a
// rollout step uses word (j & 3) of counter sub-index (j >> 2).
struct EnvNoise
{
    Key key;
    uint32_t c0, c1base;
    uint64_t step;
    uint32_t stream;
    uint32_t t = 0;
    int j = 0;
    Philox4 cur{};
    EnvNoise(uint64_t seed, uint32_t c0_, uint32_t c1base_, uint64_t step_, uint32_t stream_) : key(seed), c0(c0_), c1base(c1base_), step(step_), stream(stream_) {}
    void begin_step(uint32_t t_)
    {
        t = t_;
        j = 0;
    }
    float next()
    {
        if ((j & 3) == 0)
            cur = draw(key, c0, c1base | t, step, stream, (uint32_t)(j >> 2));
        float z = normal_from_uniform(uniform_from_word(cur.v[j & 3]));
        j++;
        return z;
    }
};

} // namespace orc
