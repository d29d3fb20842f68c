// Counter-based random streams of the control step.
//
// Philox4x32-10 (Salmon, Moraes, Dror, Shaw, "Parallel random numbers: as easy as
// 1, 2, 3", SC'11): 10 rounds of two 32x32->64 multiplies keyed by a Weyl sequence.
// A normal variate is the inverse normal CDF of a 23-bit uniform in (0,1), by
// P. J. Acklam's published rational approximation; the log in its tails is taken
// from the series log(m) = 2*atanh((m-1)/(m+1)) after an exponent split. Every float
// operation is an explicitly rounded IEEE operation (__fmaf_rn, __fmul_rn, ...), so
// the values are reproducible bit for bit by a host implementation of the same
// recipe; nothing here calls CUDA's math library.
//
// Stream layout (counter = c0, c1, step, stream << 24 | sub; key = seed):
//   MPPI perturbation        c0 = sample, c1 = branch * M + knot, words 0..1 = dims
//   MPPI rollout env noise   c0 = sample, c1 = theta << 16 | t, normal j: sub j>>2, word j&3
//   verification theta draw  c0 = sample, c1 = plan, word 0 (uniform)
//   verification env noise   c0 = sample, c1 = plan << 16 | t
//     (fast flavour)         c0 = sample, c1 = plan << 16, sub = 0x400000 | block (FastNoise)
//   PR-MPPI perturbation     c0 = sample, c1 = t, words 0..1
//   PR-MPPI theta draw       c0 = p, c1 = 0, word 0 (uniform)
//   PR-MPPI rollout env      c0 = sample, c1 = ((robust << 8 | p) << 16) | t
//   PR-MPPI candidate env    c0 = p, c1 = cand << 16 | t   (safety re-check: own stream)
//   environment step         c0 = 0, c1 = 0
#pragma once

#include <cstdint>

namespace dr
{

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

struct U4
{
    uint32_t x, y, z, w;
};

__device__ __forceinline__ U4 philox(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3, uint32_t k0, uint32_t k1)
{
#pragma unroll
    for (int r = 0; r < 10; r++)
    {
        uint32_t lo0 = 0xD2511F53u * c0;
        uint32_t hi0 = __umulhi(0xD2511F53u, c0);
        uint32_t lo1 = 0xCD9E8D57u * c2;
        uint32_t hi1 = __umulhi(0xCD9E8D57u, c2);
        uint32_t n0 = hi1 ^ c1 ^ k0;
        uint32_t n2 = hi0 ^ c3 ^ k1;
        c0 = n0;
        c1 = lo1;
        c2 = n2;
        c3 = lo0;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
    return U4{c0, c1, c2, c3};
}

__device__ __forceinline__ U4 draw(uint32_t k0, uint32_t k1, uint32_t c0, uint32_t c1, uint32_t step, uint32_t stream, uint32_t sub)
{
    return philox(c0, c1, step, (stream << 24) | (sub & 0x00ffffffu), k0, k1);
}

__device__ __forceinline__ float uniform_from_word(uint32_t w)
{
    return __fmul_rn(__uint2float_rn(2u * (w >> 9) + 1u), 5.9604644775390625e-08f);
}

__device__ __forceinline__ float series_logf(float x)
{
    uint32_t b = __float_as_uint(x);
    int e = (int)(b >> 23) - 127;
    float m = __uint_as_float((b & 0x007fffffu) | 0x3f800000u);
    if (m > 1.41421356f)
    {
        m = __fmul_rn(m, 0.5f);
        e += 1;
    }
    float f = __fsub_rn(m, 1.0f);
    float den = __fadd_rn(m, 1.0f);
    float z = __fdiv_rn(f, den);
    float z2 = __fmul_rn(z, z);
    float p = __fmaf_rn(__fmaf_rn(__fmaf_rn(__fmaf_rn(0.0909090936f, z2, 0.111111112f), z2, 0.142857149f), z2, 0.200000003f), z2, 0.333333343f);
    float zz = __fadd_rn(z, z);
    float zz3 = __fmul_rn(zz, z2);
    float lm = __fmaf_rn(zz3, p, zz);
    return __fmaf_rn(__int2float_rn(e), 0.693147182f, lm);
}

__device__ __forceinline__ float acklam_tail(float q)
{
    float num = __fmaf_rn(__fmaf_rn(__fmaf_rn(__fmaf_rn(__fmaf_rn(-7.784894002430293e-03f, q, -3.223964580411365e-01f), q, -2.400758277161838e+00f), q,
                                              -2.549732539343734e+00f),
                                    q, 4.374664141464968e+00f),
                          q, 2.938163982698783e+00f);
    float den = __fmaf_rn(__fmaf_rn(__fmaf_rn(__fmaf_rn(7.784695709041462e-03f, q, 3.224671290700398e-01f), q, 2.445134137142996e+00f), q,
                                    3.754408661907416e+00f),
                          q, 1.0f);
    return __fdiv_rn(num, den);
}

__device__ __forceinline__ float normal_from_uniform(float u)
{
    const float plow = 0.02425f;
    if (u < plow)
    {
        float q = __fsqrt_rn(__fmul_rn(-2.0f, series_logf(u)));
        return acklam_tail(q);
    }
    if (u > __fsub_rn(1.0f, plow))
    {
        float q = __fsqrt_rn(__fmul_rn(-2.0f, series_logf(__fsub_rn(1.0f, u))));
        return -acklam_tail(q);
    }
    float q = __fsub_rn(u, 0.5f);
    float r = __fmul_rn(q, q);
    float num = __fmaf_rn(__fmaf_rn(__fmaf_rn(__fmaf_rn(__fmaf_rn(-3.969683028665376e+01f, r, 2.209460984245205e+02f), r, -2.759285104469687e+02f), r,
                                              1.383577518672690e+02f),
                                    r, -3.066479806614716e+01f),
                          r, 2.506628277459239e+00f);
    float den = __fmaf_rn(__fmaf_rn(__fmaf_rn(__fmaf_rn(__fmaf_rn(-5.447609879822406e+01f, r, 1.615858368580409e+02f), r, -1.556989798598866e+02f), r,
                                              6.680131188771972e+01f),
                                    r, -1.328068155288572e+01f),
                          r, 1.0f);
    return __fdiv_rn(__fmul_rn(num, q), den);
}

__device__ __forceinline__ float normal_from_word(uint32_t w)
{
    return normal_from_uniform(uniform_from_word(w));
}

// A perturbation entry sigma * N(0,1), rounded on its own (the reference stores the
// perturbation tensor and adds it to the nominal afterwards; letting the compiler fuse
// the product into that addition would change the last bit).
__device__ __forceinline__ float scaled_normal(float sigma, uint32_t w)
{
    return __fmul_rn(sigma, normal_from_word(w));
}

// Sequential normal source for the environment noise of one rollout step.
// Out-of-line copies for the environment-step noise. An environment step has up to 14
// noise sites (opponent action noise, action noise per agent and axis, position and
// velocity noise); most are switched off in a given configuration but all are compiled.
// Inlining a Philox block and the inverse CDF at each of them multiplies the size of the
// step's code, and the instruction-cache misses that follow cost more than two calls.
// The arithmetic is the same either way (every operation is rounded explicitly).
static __device__ __noinline__ U4 draw_ool(uint32_t k0, uint32_t k1, uint32_t c0, uint32_t c1, uint32_t step, uint32_t stream, uint32_t sub)
{
    return draw(k0, k1, c0, c1, step, stream, sub);
}

static __device__ __noinline__ float normal_from_word_ool(uint32_t w)
{
    return normal_from_word(w);
}

static __device__ __noinline__ float2 normal_pair_ool(uint32_t w0, uint32_t w1)
{
    return make_float2(normal_from_word(w0), normal_from_word(w1));
}

struct EnvNoise
{
    uint32_t k0, k1, c0, c1base, step, stream, t;
    int j;
    U4 cur;
    EnvNoise() = default; // for arrays of streams, assigned before use
    __device__ __forceinline__ EnvNoise(uint32_t k0_, uint32_t k1_, uint32_t c0_, uint32_t c1base_, uint32_t step_, uint32_t stream_)
        : k0(k0_), k1(k1_), c0(c0_), c1base(c1base_), step(step_), stream(stream_), t(0), j(0), cur{0, 0, 0, 0}
    {
    }
    __device__ __forceinline__ void begin_step(uint32_t t_)
    {
        t = t_;
        j = 0;
    }
    __device__ __forceinline__ float next()
    {
        if ((j & 3) == 0)
            cur = draw_ool(k0, k1, c0, c1base | t, step, stream, (uint32_t)(j >> 2));
        uint32_t w = (j & 3) == 0 ? cur.x : (j & 3) == 1 ? cur.y : (j & 3) == 2 ? cur.z : cur.w;
        j++;
        return normal_from_word_ool(w);
    }
    // The next two normals (words j and j+1 of the stream; j is even, so both come from
    // the same Philox block). The block is drawn inline: this is the one noise site that
    // runs every step in the default configuration (opponent action noise).
    __device__ __forceinline__ float2 next2()
    {
        if ((j & 3) == 0)
            cur = draw(k0, k1, c0, c1base | t, step, stream, (uint32_t)(j >> 2));
        const bool lo = (j & 3) == 0;
        const uint32_t w0 = lo ? cur.x : cur.z, w1 = lo ? cur.y : cur.w;
        j += 2;
        return normal_pair_ool(w0, w1);
    }
};

// A pair of normal variates from two Philox words by the Box-Muller transform (Box and
// Muller, "A note on the generation of random normal deviates", 1958):
// r = sqrt(-2 ln u1), (r cos 2 pi u2, r sin 2 pi u2), with the hardware's approximate
// log, square root, sine and cosine (the angle is taken in (-pi, pi), where the
// approximate sine and cosine are accurate). u1 is at least 2^-24, so |z| < 5.8.
__device__ __forceinline__ float2 box_muller_fast(uint32_t w0, uint32_t w1)
{
    const float u1 = uniform_from_word(w0);
    const float u2 = uniform_from_word(w1);
    // the approximate log of a u1 just below 1 may come out just above 0
    float r2 = fmaxf(-2.0f * __logf(u1), 0.0f);
    float r;
    asm("sqrt.approx.f32 %0, %1;" : "=f"(r) : "f"(r2));
    float sn, cs;
    __sincosf(6.28318531f * (u2 - 0.5f), &sn, &cs);
    return make_float2(r * cs, r * sn);
}

// Philox4x32 with 7 rounds instead of 10: the same round function and key schedule.
// Salmon, Moraes, Dror and Shaw ("Parallel random numbers: as easy as 1, 2, 3", SC 2011)
// report that Philox4x32 passes the TestU01 BigCrush battery from 7 rounds on, the 10 of
// the default being a safety margin; the fast verification's noise uses 7.
__device__ __forceinline__ U4 philox7(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3, uint32_t k0, uint32_t k1)
{
#pragma unroll
    for (int r = 0; r < 7; r++)
    {
        uint32_t lo0 = 0xD2511F53u * c0;
        uint32_t hi0 = __umulhi(0xD2511F53u, c0);
        uint32_t lo1 = 0xCD9E8D57u * c2;
        uint32_t hi1 = __umulhi(0xCD9E8D57u, c2);
        uint32_t n0 = hi1 ^ c1 ^ k0;
        uint32_t n2 = hi0 ^ c3 ^ k1;
        c0 = n0;
        c1 = lo1;
        c2 = n2;
        c3 = lo0;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
    return U4{c0, c1, c2, c3};
}

// Normal source of the Monte-Carlo verification's fast flavour: Box-Muller pairs from
// the words of one 7-round Philox stream per sample, taken in sequence across its steps (a
// block of four words gives two pairs: one returned at once, one kept for the next call),
// counter = (c0, c1, step, stream << 24 | 0x400000 | block). Its draws differ from
// EnvNoise's; the distribution is the same.
struct FastNoise
{
    uint32_t k0, k1, c0, c1, step, stream;
    uint32_t block; // next Philox block
    bool have;      // spare holds the second pair of the last block
    float2 spare;
    __device__ __forceinline__ FastNoise(uint32_t k0_, uint32_t k1_, uint32_t c0_, uint32_t c1_, uint32_t step_, uint32_t stream_)
        : k0(k0_), k1(k1_), c0(c0_), c1(c1_), step(step_), stream(stream_), block(0), have(false), spare{0.f, 0.f}
    {
    }
    __device__ __forceinline__ void begin_step(uint32_t)
    {
    }
    __device__ __forceinline__ float2 next2()
    {
        if (have)
        {
            have = false;
            return spare;
        }
        const U4 r = philox7(c0, c1, step, (stream << 24) | ((0x400000u | block) & 0x00ffffffu), k0, k1);
        block++;
        spare = box_muller_fast(r.z, r.w);
        have = true;
        return box_muller_fast(r.x, r.y);
    }
    __device__ __forceinline__ float next()
    {
        return next2().x;
    }
};

} // namespace dr
