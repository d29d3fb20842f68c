// Device model of the StratRace environment: dynamics, opponent policy, belief update
// and costs, as evaluated inside every rollout step.
//
// Semantics follow the reference (include/environments/env_stratrace.h:33-894,
// include/costs.cuh:7-86, include/state.h:93-228) expression by expression, so that
// on identical inputs the FP32 results agree with the reference kernels. The work is
// organised for the GPU: the track quantities of each agent at the start of a step
// (unit tangent, curvature, ds/dt, centre point) are computed once and shared by
// every opponent-hypothesis evaluation and by the arc-length update, where the
// reference recomputes them per call; the hypothesis-independent part of the opponent
// policy is likewise evaluated once per step. The track grids live in shared memory.
#pragma once

#include <cmath>
#include <cstddef>
#include <cstdint>

#include "philox.cuh"

namespace dr
{

// Arithmetic of the model in two flavours. The exact flavour (F = false) is IEEE division
// and square root and the CUDA math library's expf, the operations the reference's
// kernels evaluate, so that results agree with them bit for bit. The fast flavour
// (F = true) takes the hardware approximations (div.approx, sqrt.approx, rsqrt, ex2;
// about 2 ulp): the Monte-Carlo verification uses it, whose agreement with the reference
// is statistical because the reference draws its hypotheses and noise from curand.
template <bool F> __device__ __forceinline__ float mdiv(float a, float b)
{
    if constexpr (F)
        return __fdividef(a, b);
    else
        return a / b;
}

template <bool F> __device__ __forceinline__ float msqrt(float x)
{
    if constexpr (F)
    {
        float r;
        asm("sqrt.approx.f32 %0, %1;" : "=f"(r) : "f"(x));
        return r;
    }
    else
        return sqrtf(x);
}

// a / sqrt(x)
template <bool F> __device__ __forceinline__ float mdivsqrt(float a, float x)
{
    if constexpr (F)
        return a * rsqrtf(x);
    else
        return a / sqrtf(x);
}

template <bool F> __device__ __forceinline__ float mexp(float x)
{
    if constexpr (F)
        return __expf(x);
    else
        return expf(x);
}

constexpr int NTS = 512;       // N_TRACK_SAMPLES (env_stratrace_defs.h:11)
static_assert((NTS & (NTS - 1)) == 0, "the track sample count is a power of two");
// x % NTS for x >= 0, which every track index taken modulo NTS here is (one AND instead of
// the signed remainder's sequence)
__host__ __device__ __forceinline__ int wrapNts(int x)
{
    return x & (NTS - 1);
}
constexpr int WIN = 10;        // WINDOW_SIZE (env_stratrace_defs.h:40)
constexpr float DECAY = 0.97f; // include/config.h:30
constexpr float MIN_COEFF = 0.01f; // MIN_COEFF_THRESHOLD, include/config.h:29
// Track grids in one buffer (offsets in floats, each of a sample index 0):
//   p      centreline points, interleaved (x, y), with GRID_PAD wrapped samples on each
//          side (p[j] for j in [-16, 528)), so that the projection window needs no modulo;
//   t      unit tangent [513][2] and kappa curvature [513] (sample 512 = sample 0);
//   px, py the padded centreline again as separate x and y rows (8-byte aligned at even
//          indices), read two samples at a time by the projection window;
//   cert   [512] per sample c, the squared radius within which a local minimum at c of the
//          squared distances to the samples is their minimum over every window holding c
//          (projectionCertificate, computed with the grids on the host).
constexpr int GRID_PAD = 16;
constexpr int GRID_ROW = NTS + 2 * GRID_PAD; // padded centreline samples
constexpr int GRID_P = GRID_PAD * 2, GRID_T = GRID_ROW * 2, GRID_K = GRID_T + (NTS + 1) * 2;
constexpr int GRID_PX = GRID_K + NTS + 1 + 1 + GRID_PAD, GRID_PY = GRID_PX + GRID_ROW;
constexpr int GRID_CERT = GRID_PY - GRID_PAD + GRID_ROW;
constexpr int GRID_FLOATS = GRID_CERT + NTS;
static_assert(GRID_FLOATS % 4 == 0 && GRID_PX % 2 == 0 && GRID_PY % 2 == 0 && GRID_PAD > WIN + 1, "grid layout");

enum Term
{
    TERM_NONE = 0,
    TERM_LOSE = 1,
    TERM_WIN = 2,
    TERM_OPP_WIN = 3
};

// Environment parameters (EnvironmentConfig minus the grid pointers).
struct EnvParams
{
    float dt, droneRadius, posNoise, speedNoise, actionNoiseLevel;
    float maxSpeed[4], maxAccel[4];
    float trackWidth;
    int nWinLaps;
    float kP, kV, maxOppLatDistFact, trackLength;
    float s1[8][3], s2[8][3], s3[8][3], speedScale[8][3], actionNoise[8][3];
    // Filled on the device by envDeviceTerms (never copied from the host):
    // logf(0.2^2 + actionNoise^2), the per-hypothesis constant of the belief update's
    // log-likelihood (env_stratrace.h:199-203), evaluated once per launch instead of
    // once per step with the same device logf.
    float logSqSigma[8][3];
    // the fast flavour's Gaussian log-likelihood of an action error e: |e|^2 llScale + llConst,
    // llScale = -1 / (2 sigma^2), llConst = -log(2 pi) - log(sigma^2) (two action dimensions)
    float llScale[8][3], llConst[8][3];
    // 1 / trackLength and 1 / dt (the fast flavour multiplies by them)
    float invTrackLength, invDt;
    // Hypotheses that give opponent o the same action as an earlier one: dupAll[th][o] is
    // the first hypothesis j < th with the same s1, s2, s3 and speedScale (else -1), so
    // j's action is th's whatever the state; dupNoBlock[th][o] the first j < th with the
    // same s1, s2 and speedScale, so j's action is th's whenever the opponent blocks no
    // one (s3 is read only by the blocking term, env_stratrace.h:357-372).
    signed char dupAll[8][3], dupNoBlock[8][3];
    // hypothesis th gives opponent o's action the noise level of hypothesis 0 (so the two
    // have the same likelihood constants)
    bool noiseAs0[8][3];
};

constexpr int ENV_HOST_WORDS = (int)(offsetof(EnvParams, logSqSigma) / 4);
constexpr float BELIEF_SIGMA_ENV = 0.2f; // sigmaEnv of updateBelief (env_stratrace.h:170)

__device__ __forceinline__ float beliefSqSigma(float an)
{
    return BELIEF_SIGMA_ENV * BELIEF_SIGMA_ENV + an * an;
}

// Device-computed terms of EnvParams from the host-filled fields of `src`; thread `tid`
// of `n` fills its share of `dst`.
__device__ __forceinline__ void envDeviceTerms(EnvParams& dst, const EnvParams& src, int tid, int n)
{
    for (int i = tid; i < 8 * 3; i += n)
    {
        const int th = i / 3, o = i % 3;
        dst.logSqSigma[th][o] = logf(beliefSqSigma(src.actionNoise[th][o]));
        dst.llScale[th][o] = -0.5f / beliefSqSigma(src.actionNoise[th][o]);
        dst.llConst[th][o] = -logf(2.0f * M_PIf32) - dst.logSqSigma[th][o];
        int all = -1, noBlock = -1;
        for (int j = th - 1; j >= 0; j--)
        {
            const bool base = src.s1[j][o] == src.s1[th][o] && src.s2[j][o] == src.s2[th][o] && src.speedScale[j][o] == src.speedScale[th][o];
            if (base)
                noBlock = j;
            if (base && src.s3[j][o] == src.s3[th][o])
                all = j;
        }
        dst.dupAll[th][o] = (signed char)all;
        dst.dupNoBlock[th][o] = (signed char)noBlock;
        dst.noiseAs0[th][o] = src.actionNoise[th][o] == src.actionNoise[0][o];
    }
    if (tid == 0)
    {
        dst.invTrackLength = 1.0f / src.trackLength;
        dst.invDt = 1.0f / src.dt;
    }
}

// Position on the sampled track (sampleTrackArray, env_stratrace.h:53-67, split into its
// index computation and its interpolation): sample index below s and the weight of the
// next sample.
struct TrackPos
{
    int i0;
    float w;
};

__device__ __forceinline__ TrackPos trackPos(float s, float L)
{
    s /= L;
    s = s - floorf(s);
    float idx_f = s * NTS;
    int idx0 = (int)idx_f;
    return TrackPos{idx0, idx_f - idx0};
}

// trackPos in either flavour (the fast one multiplies by 1 / L)
template <bool F> __device__ __forceinline__ TrackPos trackPosT(float s, float L, float invL)
{
    if constexpr (F)
    {
        s *= invL;
        s = s - floorf(s);
        float idx_f = s * NTS;
        int idx0 = min((int)idx_f, NTS - 1);
        return TrackPos{idx0, idx_f - idx0};
    }
    else
        return trackPos(s, L);
}

template <int NA> struct DState
{
    float pos[2 * NA];
    float vel[2 * NA];
    float S[NA];
    float lat[NA];
    int laps[NA];
    // trackPos(S[a]): computed by the projection that produced S[a] (or by locate() for a
    // loaded state) and reused by the next step's track lookups at the same S[a]
    TrackPos tp[NA];

    __device__ __forceinline__ void locate(float L)
    {
#pragma unroll
        for (int a = 0; a < NA; a++)
            tp[a] = trackPos(S[a], L);
    }
};

template <int NTH> struct BState
{
    float belief[NTH];
    int predTheta;
    int branchingTime;
};

struct Track
{
    const float* p;  // [-16, 528)[2]
    const float* t;  // [513][2]
    const float* k;  // [513]
    const float* px; // [-16, 528)
    const float* py; // [-16, 528)
    const float* cert; // [512]
};

__device__ __forceinline__ Track trackIn(const float* grids)
{
    return Track{grids + GRID_P, grids + GRID_T, grids + GRID_K, grids + GRID_PX, grids + GRID_PY, grids + GRID_CERT};
}

// ---- track sampling (env_stratrace.h:44-85) ------------------------------------------

__device__ __forceinline__ void sampleAt2(const float* __restrict__ arr, TrackPos q, float& o0, float& o1)
{
    const int idx0 = q.i0;
    const int idx1 = wrapNts(idx0 + 1);
    const float t = q.w;
    o0 = (1.0f - t) * arr[idx0 * 2 + 0] + t * arr[idx1 * 2 + 0];
    o1 = (1.0f - t) * arr[idx0 * 2 + 1] + t * arr[idx1 * 2 + 1];
}

__device__ __forceinline__ float sampleAt1(const float* __restrict__ arr, TrackPos q)
{
    const int idx0 = q.i0;
    const int idx1 = wrapNts(idx0 + 1);
    const float t = q.w;
    return (1.0f - t) * arr[idx0] + t * arr[idx1];
}

__device__ __forceinline__ float sqNorm(float x, float y)
{
    return x * x + y * y;
}

template <bool F> __device__ __forceinline__ void normalizedSpeed(const Track& tr, TrackPos q, float& o0, float& o1)
{
    sampleAt2(tr.t, q, o0, o1);
    float invNorm = mdivsqrt<F>(1.0f, sqNorm(o0, o1));
    o0 *= invNorm;
    o1 *= invNorm;
}

// The part of fastProjectOnTrack after the window scan: exact projection onto the two
// segments at the nearest sample bestJ, then the signed lateral distance.
template <bool F>
__device__ __forceinline__ float projectSegments(const Track& tr, float L, float invL, float px, float py, int bestJ, float& latDist, TrackPos& tpS)
{
    const float2* __restrict__ P2 = reinterpret_cast<const float2*>(tr.p);
    const int bestInd = wrapNts(bestJ + NTS); // bestJ >= -WIN
    float bestSegSqDist = INFINITY;
    float bestS = 0.0f;
    float closestX = 0.0f, closestY = 0.0f;
#pragma unroll
    for (int seg = -1; seg <= 0; ++seg)
    {
        const int aj = bestInd + seg;  // -1 .. 511; the padded grid holds p[-1] and p[512]
        const int a = aj < 0 ? aj + NTS : aj;
        const float2 qa = P2[aj], qb = P2[aj + 1];
        float ax = qa.x, ay = qa.y;
        float abx = qb.x - ax;
        float aby = qb.y - ay;
        float sqAB = sqNorm(abx, aby);
        float t = 0.0f;
        if (sqAB > 1e-12f) // the reference compares with the double 1e-12; for floats the two tests agree
        {
            t = mdiv<F>((px - ax) * abx + (py - ay) * aby, sqAB);
            t = fmaxf(0.0f, fminf(t, 1.0f));
        }
        float projx = ax + t * abx;
        float projy = ay + t * aby;
        float sqDist = sqNorm(px - projx, py - projy);
        if (sqDist < bestSegSqDist)
        {
            bestSegSqDist = sqDist;
            bestS = ((float)a + t) / NTS * L;
            closestX = projx;
            closestY = projy;
        }
    }
    float tg0, tg1;
    tpS = trackPosT<F>(bestS, L, invL);
    sampleAt2(tr.t, tpS, tg0, tg1);
    float cross = -tg1 * (px - closestX) + tg0 * (py - closestY);
    latDist = copysignf(msqrt<F>(bestSegSqDist), cross);
    return bestS;
}

// Squared distance from (px, py) to window sample j0 + k, rounded like each lane of the
// packed window scans below (sub, mul, then fma).
__device__ __forceinline__ float windowSqDist(const Track& tr, int j0, int k, float px, float py)
{
    const int j = j0 + k;
    const float d0 = __fsub_rn(tr.px[j], px), d1 = __fsub_rn(tr.py[j], py);
    return __fmaf_rn(d1, d1, __fmul_rn(d0, d0));
}

// Key of window place k for the search of flavour F. Fast: the squared distance with its
// low five mantissa bits dropped, then the place, as one unsigned word (the smaller key is
// the nearer sample, at equal truncated distances the earlier one). Exact: the squared
// distance itself, compared as the reference's scan compares it (strict '<' in increasing
// place order: at equal distances the earlier place wins).
template <bool F> struct WindowKey;
template <> struct WindowKey<true>
{
    uint32_t v;
    __device__ __forceinline__ WindowKey(const Track& tr, int j0, int k, float px, float py)
    {
        v = (__float_as_uint(windowSqDist(tr, j0, k, px, py)) & ~31u) | (uint32_t)k;
    }
    // this key (place k) before the key of place k + 1 / after the one of place k - 1
    __device__ __forceinline__ bool beatsNext(const WindowKey& o) const { return v < o.v; }
    __device__ __forceinline__ bool beatsPrev(const WindowKey& o) const { return v < o.v; }
    __device__ __forceinline__ float dist() const { return __uint_as_float(v & ~31u); }
};
template <> struct WindowKey<false>
{
    float v;
    __device__ __forceinline__ WindowKey(const Track& tr, int j0, int k, float px, float py) { v = windowSqDist(tr, j0, k, px, py); }
    __device__ __forceinline__ bool beatsNext(const WindowKey& o) const { return v <= o.v; }
    __device__ __forceinline__ bool beatsPrev(const WindowKey& o) const { return v < o.v; }
    __device__ __forceinline__ float dist() const { return v; }
};

// The local search of the projection window: from the window's centre (the previous
// position's sample), step to the neighbour whose key wins against the current one while
// there is one. The sample it stops at is a local minimum of the keys and is the window's
// first minimum when the point lies within the sample's certified radius (tr.cert: every
// other sample of any window holding it is then farther by more than 1e-3 m^2, far above
// the keys' truncation and the distances' rounding) and is not at the window's edge;
// returns -1 otherwise, and the caller scans the whole window.
template <bool F>
__device__ __forceinline__ int windowLocalSearch(const Track& tr, int j0, float px, float py)
{
    using Key = WindowKey<F>;
    int c = WIN;
    Key kc(tr, j0, c, px, py);
    Key kl(tr, j0, c - 1, px, py);
    if (kl.beatsNext(kc))
    {
        for (int it = 0; it < WIN; it++) // down the window
        {
            c--;
            kc = kl;
            if (c == 0)
                break;
            kl = Key(tr, j0, c - 1, px, py);
            if (!kl.beatsNext(kc))
                break;
        }
    }
    else
    {
        Key kr(tr, j0, c + 1, px, py);
        for (int it = 0; it < WIN && kr.beatsPrev(kc); it++) // up the window
        {
            c++;
            kc = kr;
            if (c == 2 * WIN)
                break;
            kr = Key(tr, j0, c + 1, px, py);
        }
    }
    const bool certified = c > 0 && c < 2 * WIN && kc.dist() <= tr.cert[wrapNts(j0 + c + NTS)];
    return certified ? c : -1;
}

// fastProjectOnTrack<false> (env_stratrace.h:88-162): returns S, writes latDist and the
// track position of S. The fast flavour takes the window's minimum on keys that pack the
// squared distance (its low five mantissa bits dropped) with the sample's place in the
// window (WindowKey), so one unsigned minimum per sample finds the first of the nearest
// samples; two distances within 2^-18 relative of each other count as equal there. With
// LOCAL (the default, both flavours) it first runs the certified local search
// (windowLocalSearch), which evaluates three samples where the point moved less than a
// sample's spacing, and scans the window only where that search cannot certify its
// result; both give the same sample, in the exact flavour the reference's.
template <bool F, bool LOCAL = true>
__device__ __forceinline__ float projectOnTrack(const Track& tr, float L, float invL, float px, float py, float prevS, float& latDist, TrackPos& tpS)
{
    if constexpr (F)
        prevS *= invL;
    else
        prevS /= L;
    prevS = prevS - floorf(prevS);
    int idxPrev = (int)(prevS * NTS); // 512 when prevS rounds to 1: the padded grid holds that window
    const float* __restrict__ P = tr.p;
    const float2* __restrict__ P2 = reinterpret_cast<const float2*>(P);
    // Window idxPrev-10 .. idxPrev+10, first minimum of the squared distance wins (the
    // reference scans it in increasing index order with a strict '<'). Samples are taken
    // in pairs of consecutive indices from the separate x / y rows with packed FP32x2
    // arithmetic (each lane rounds exactly like the scalar sub, mul and fma), then the
    // one sample left over; the window of 21 has 10 pairs starting at an even index and
    // one single sample, either its first (odd start) or its last (even start).
    const int j0 = idxPrev - WIN;
    const int jp = (j0 + 1) & ~1;
    const int js = (j0 & 1) ? j0 : j0 + 2 * WIN;
    const uint64_t* __restrict__ PX2 = reinterpret_cast<const uint64_t*>(tr.px);
    const uint64_t* __restrict__ PY2 = reinterpret_cast<const uint64_t*>(tr.py);
    uint64_t pxx, pyy;
    asm("mov.b64 %0, {%1, %1};" : "=l"(pxx) : "f"(px));
    asm("mov.b64 %0, {%1, %1};" : "=l"(pyy) : "f"(py));
    int local = -1;
    if constexpr (LOCAL)
        local = windowLocalSearch<F>(tr, j0, px, py);
    int bestJ = j0 + local;
    if (F && local < 0)
    {
        uint32_t best = 0xffffffffu;
        const uint32_t off = (uint32_t)(jp - j0); // place of the first pair's first sample
#pragma unroll 5
        for (int q = 0; q < WIN; q++)
        {
            const int j = jp + 2 * q;
            float sqA, sqB;
            asm("{\n\t.reg .b64 d0, d1, s;\n\t"
                "sub.rn.f32x2 d0, %2, %4;\n\t"
                "sub.rn.f32x2 d1, %3, %5;\n\t"
                "mul.rn.f32x2 s, d0, d0;\n\t"
                "fma.rn.f32x2 s, d1, d1, s;\n\t"
                "mov.b64 {%0, %1}, s;\n\t}"
                : "=f"(sqA), "=f"(sqB)
                : "l"(PX2[j >> 1]), "l"(PY2[j >> 1]), "l"(pxx), "l"(pyy));
            best = min(best, (__float_as_uint(sqA) & ~31u) | (off + 2u * q));
            best = min(best, (__float_as_uint(sqB) & ~31u) | (off + 2u * q + 1u));
        }
        {
            // rounded like each lane of the pairs above
            float2 qs = P2[js];
            float d0 = __fsub_rn(qs.x, px), d1 = __fsub_rn(qs.y, py);
            float sq = __fmaf_rn(d1, d1, __fmul_rn(d0, d0));
            best = min(best, (__float_as_uint(sq) & ~31u) | (uint32_t)(js - j0));
        }
        bestJ = j0 + (int)(best & 31u);
    }
    else if (!F && local < 0)
    {
        bestJ = j0;
        float bestSqDist = INFINITY;
#pragma unroll 5
        for (int q = 0; q < WIN; q++)
        {
            const int j = jp + 2 * q;
            float sqA, sqB;
            asm("{\n\t.reg .b64 d0, d1, s;\n\t"
                "sub.rn.f32x2 d0, %2, %4;\n\t"
                "sub.rn.f32x2 d1, %3, %5;\n\t"
                "mul.rn.f32x2 s, d0, d0;\n\t"
                "fma.rn.f32x2 s, d1, d1, s;\n\t"
                "mov.b64 {%0, %1}, s;\n\t}"
                : "=f"(sqA), "=f"(sqB)
                : "l"(PX2[j >> 1]), "l"(PY2[j >> 1]), "l"(pxx), "l"(pyy));
            if (sqA < bestSqDist)
            {
                bestSqDist = sqA;
                bestJ = j;
            }
            if (sqB < bestSqDist)
            {
                bestSqDist = sqB;
                bestJ = j + 1;
            }
        }
        {
            float2 qs = P2[js];
            float sq = 0.f;
            float d0 = qs.x - px;
            sq += d0 * d0;
            float d1 = qs.y - py;
            sq += d1 * d1;
            if (sq < bestSqDist || (sq == bestSqDist && js < bestJ))
                bestJ = js;
        }
    }
    return projectSegments<F>(tr, L, invL, px, py, bestJ, latDist, tpS);
}

// projectOnTrack<true> with the window scan spread over the 32 lanes of a warp, all of
// which hold the same position and take part: lane j < 21 evaluates window sample j and one
// warp-wide unsigned minimum of the packed (squared distance, place) keys finds the nearest;
// every lane returns projectOnTrack<true>'s result.
__device__ __forceinline__ float projectOnTrackWarp(const Track& tr, float L, float invL, float px, float py, float prevS, float& latDist, TrackPos& tpS)
{
    prevS *= invL;
    prevS = prevS - floorf(prevS);
    const int idxPrev = (int)(prevS * NTS);
    const int j0 = idxPrev - WIN;
    const uint32_t lane = threadIdx.x & 31u;
    uint32_t key = 0xffffffffu;
    if (lane <= 2 * WIN)
    {
        const int j = j0 + (int)lane;
        const float d0 = __fsub_rn(tr.px[j], px), d1 = __fsub_rn(tr.py[j], py);
        const float sq = __fmaf_rn(d1, d1, __fmul_rn(d0, d0));
        key = (__float_as_uint(sq) & ~31u) | lane;
    }
    key = __reduce_min_sync(0xffffffffu, key);
    return projectSegments<true>(tr, L, invL, px, py, j0 + (int)(key & 31u), latDist, tpS);
}

// ---- per-step agent quantities -------------------------------------------------------

template <int NA> struct AgentGeo
{
    float tn0[NA], tn1[NA]; // unit tangent at S[a]
    float kap[NA];          // curvature at S[a]
    float sdot[NA];         // computeSdot(a) (env_stratrace.h:302-315)
};

template <int NA, bool F = false, int A0 = 0>
__device__ __forceinline__ void agentGeometry(const Track& tr, const EnvParams& E, const DState<NA>& s, AgentGeo<NA>& g)
{
#pragma unroll
    for (int a = A0; a < NA; a++)
    {
        normalizedSpeed<F>(tr, s.tp[a], g.tn0[a], g.tn1[a]);
        g.kap[a] = sampleAt1(tr.k, s.tp[a]);
        float metric = 1 - g.kap[a] * s.lat[a];
        if (fabsf(metric) < 1e-12f)
            metric = copysignf(1e-12f, metric);
        g.sdot[a] = mdiv<F>(g.tn0[a] * s.vel[2 * a] + g.tn1[a] * s.vel[2 * a + 1], metric);
    }
}

// Hypothesis-independent part of the opponent policy for opponent iOpp
// (env_stratrace.h:318-461 and 611-706).
struct OppCommon
{
    // computeOppTargetLatDist, k = 0 (behind) and 1 (ahead)
    int j[2];
    float deltaS[2], deltaE[2], latJ[2], sdotJ[2], blockTol[2], oppLong[2];
    bool shouldBlock[2], fasterThanJ[2];
    float sdot_i, maxLatDis;
    // computeOpponentAction
    float tang0, tang1, norm0, norm1, kappa, e_n, v_t, v_n, e_n_max, metric_actual, a_centripetal, a_lat_max, distPos, distNeg, maxAccel;
    // maxAccel^2 rounded on its own: the reference evaluates the policy under every
    // hypothesis, so this hypothesis-independent product is shared and never fused into
    // maxAccel^2 - a_n^2 (env_stratrace.h:691); fusing it would change the last bit
    float maxAccelSq;
    bool brakePos, brakeNeg;
};

template <int NOPP, bool F = false>
__device__ __forceinline__ void oppCommon(int iOpp, const Track& tr, const EnvParams& E, const DState<NOPP + 1>& s, const AgentGeo<NOPP + 1>& g,
                                          OppCommon& c)
{
    const float L = E.trackLength;
    int iAhead = 0;
    float deltaSAhead = s.S[0] - s.S[iOpp];
    if (deltaSAhead < 0.0f)
        deltaSAhead += L;
#pragma unroll
    for (int j = 1; j <= NOPP; j++)
        if (j != iOpp)
        {
            float deltaS = s.S[j] - s.S[iOpp];
            if (deltaS < 0.0f)
                deltaS += L;
            if (deltaS < deltaSAhead)
            {
                deltaSAhead = deltaS;
                iAhead = j;
            }
        }
    int iBehind = 0;
    float deltaSBehind = s.S[0] - s.S[iOpp];
    if (deltaSBehind > 0.0f)
        deltaSBehind -= L;
#pragma unroll
    for (int j = 1; j <= NOPP; j++)
        if (j != iOpp)
        {
            float deltaS = s.S[j] - s.S[iOpp];
            if (deltaS > 0.0f)
                deltaS -= L;
            if (deltaS > deltaSBehind)
            {
                deltaSBehind = deltaS;
                iBehind = j;
            }
        }
    c.sdot_i = g.sdot[iOpp];
#pragma unroll
    for (int k = 0; k <= 1; k++)
    {
        int j = k ? iAhead : iBehind;
        float deltaS = k ? deltaSAhead : deltaSBehind;
        // runtime agent index j -> select from the unrolled arrays
        float latJ = s.lat[0], S_unused = 0.f, tj0 = g.tn0[0], tj1 = g.tn1[0], sdj = g.sdot[0], vj0 = s.vel[0], vj1 = s.vel[1], msj = E.maxSpeed[0];
#pragma unroll
        for (int a = 1; a <= NOPP; a++)
            if (a == j)
            {
                latJ = s.lat[a];
                tj0 = g.tn0[a];
                tj1 = g.tn1[a];
                sdj = g.sdot[a];
                vj0 = s.vel[2 * a];
                vj1 = s.vel[2 * a + 1];
                msj = E.maxSpeed[a];
            }
        (void)S_unused;
        c.j[k] = j;
        c.deltaS[k] = deltaS;
        c.deltaE[k] = latJ - s.lat[iOpp];
        c.latJ[k] = latJ;
        c.sdotJ[k] = sdj;
        // loop-invariant in the reference (hoisted, rounded on its own before the additions)
        c.blockTol[k] = __fmul_rn(msj, 0.3f);
        c.shouldBlock[k] = (deltaS < 0.0f) && (deltaS > -L * 0.25f) && (sdj + c.blockTol[k] > c.sdot_i);
        c.fasterThanJ[k] = c.sdot_i > sdj;
        c.oppLong[k] = vj0 * tj0 + vj1 * tj1;
    }
    c.maxLatDis = E.trackWidth - E.droneRadius * E.maxOppLatDistFact;

    c.maxAccel = E.maxAccel[iOpp];
    c.maxAccelSq = __fmul_rn(c.maxAccel, c.maxAccel);
    float pc0, pc1;
    sampleAt2(tr.p, s.tp[iOpp], pc0, pc1);
    c.tang0 = g.tn0[iOpp];
    c.tang1 = g.tn1[iOpp];
    c.kappa = g.kap[iOpp];
    c.norm0 = -c.tang1;
    c.norm1 = c.tang0;
    float pos0 = s.pos[iOpp * 2], pos1 = s.pos[iOpp * 2 + 1];
    float vel0 = s.vel[iOpp * 2], vel1 = s.vel[iOpp * 2 + 1];
    c.e_n = (pos0 - pc0) * c.norm0 + (pos1 - pc1) * c.norm1;
    c.v_t = vel0 * c.tang0 + vel1 * c.tang1;
    c.v_n = vel0 * c.norm0 + vel1 * c.norm1;
    c.e_n_max = E.trackWidth - E.droneRadius * 1.2f;
    float metric_actual = 1.0f - c.kappa * c.e_n;
    if (fabsf(metric_actual) < 1e-6f)
        metric_actual = copysignf(1e-6f, metric_actual);
    c.metric_actual = metric_actual;
    c.a_centripetal = mdiv<F>(c.v_t * c.v_t * c.kappa, metric_actual);
    c.a_lat_max = fmaxf(c.maxAccel - fabsf(c.a_centripetal), c.maxAccel * 0.2f);
    c.distPos = fmaxf(c.e_n_max - c.e_n, 0.001f);
    c.distNeg = fmaxf(c.e_n_max + c.e_n, 0.001f);
    c.brakePos = c.v_n > 0.0f && c.v_n * c.v_n > 1.8f * c.a_lat_max * c.distPos;
    c.brakeNeg = c.v_n < 0.0f && c.v_n * c.v_n > 1.8f * c.a_lat_max * c.distNeg;
}

// Hypothesis-dependent part: target lateral offset / speed goal and the resulting
// acceleration of opponent iOpp under hypothesis th.
template <bool F = false>
__device__ __forceinline__ void oppAction(int iOpp, int th, const EnvParams& E, const OppCommon& c, float& out0, float& out1)
{
    const float s1 = E.s1[th][iOpp - 1], s2 = E.s2[th][iOpp - 1], s3 = E.s3[th][iOpp - 1];
    float latDis = 0.0f;
    float baseSpeed = E.speedScale[th][iOpp - 1] * E.maxSpeed[iOpp];
    float speedGoal = baseSpeed;
#pragma unroll
    for (int k = 0; k <= 1; k++)
    {
        float deltaS = c.deltaS[k];
        float deltaE = c.deltaE[k];
        bool shouldOvertake = c.fasterThanJ[k] && (fabsf(deltaE) < s1);
        if (!c.shouldBlock[k] && !shouldOvertake)
            continue; // neither term uses the proximity factor
        float factor = mexp<F>(-s2 * deltaS * deltaS);
        if (c.shouldBlock[k])
        {
            float blockTerm = c.latJ[k] * (1 - mexp<F>(-s3 * (c.sdotJ[k] + c.blockTol[k] - c.sdot_i))) * factor;
            latDis += blockTerm;
        }
        if (shouldOvertake)
        {
            float overtakeTerm = (c.latJ[k] - copysignf(s1, deltaE)) * factor;
            latDis += overtakeTerm;
            float oppLongSpeed = c.oppLong[k];
            if (deltaS < 3 * E.droneRadius)
                speedGoal = fminf(speedGoal, 0.7f * oppLongSpeed);
            else if (deltaS < 6 * E.droneRadius && s1 > 1e-6f) // double 1e-6 in the reference; same test for floats
            {
                float latFactor = mdiv<F>(fabsf(deltaE), s1);
                speedGoal = fminf(speedGoal, latFactor * oppLongSpeed + (1.0f - latFactor) * baseSpeed);
            }
        }
    }
    float latDisRaw = fmaxf(-c.maxLatDis, fminf(c.maxLatDis, latDis));

    const float maxAccel = c.maxAccel, a_lat_max = c.a_lat_max, v_n = c.v_n, dt = E.dt;
    float latDisC = fmaxf(-c.e_n_max, fminf(c.e_n_max, latDisRaw));
    float e_error = latDisC - c.e_n;
    float a_n_cmd;
    if (c.brakePos)
        a_n_cmd = -a_lat_max;
    else if (c.brakeNeg)
        a_n_cmd = a_lat_max;
    else if (fabsf(e_error) < 0.02f)
    {
        float kp = F ? a_lat_max * 50.0f : a_lat_max / 0.02f;
        a_n_cmd = kp * e_error - 2.0f * msqrt<F>(kp) * v_n;
        a_n_cmd = fmaxf(-a_lat_max, fminf(a_lat_max, a_n_cmd));
    }
    else
    {
        float stopping_dist = mdiv<F>(v_n * v_n, 2.0f * a_lat_max);
        bool v_toward = (e_error > 0.0f && v_n > 0.0f) || (e_error < 0.0f && v_n < 0.0f);
        bool decel_phase = v_toward && stopping_dist >= fabsf(e_error) * 0.95f;
        a_n_cmd = (e_error > 0.0f) ? a_lat_max : -a_lat_max;
        if (decel_phase)
            a_n_cmd = -a_n_cmd;
        float v_n_next = v_n + a_n_cmd * dt;
        if (v_n_next > 0.0f)
        {
            float v_safe = msqrt<F>(2.0f * a_lat_max * c.distPos);
            if (v_n_next > v_safe)
                a_n_cmd = F ? (v_safe - v_n) * E.invDt : (v_safe - v_n) / dt;
        }
        else
        {
            float v_safe = msqrt<F>(2.0f * a_lat_max * c.distNeg);
            if (-v_n_next > v_safe)
                a_n_cmd = F ? (-v_safe - v_n) * E.invDt : (-v_safe - v_n) / dt;
        }
    }
    float a_n_total = fmaxf(-maxAccel, fminf(maxAccel, a_n_cmd + c.a_centripetal));
    float a_t_max = msqrt<F>(fmaxf(c.maxAccelSq - a_n_total * a_n_total, 0.0f));
    float kappa = c.kappa;
    float kappa_eff = mdiv<F>(kappa, 1.0f - kappa * latDisC + 1e-6f);
    float pathSpeed = fminf(speedGoal, msqrt<F>(mdiv<F>(maxAccel, fmaxf(fabsf(kappa_eff), 1e-12f))));
    if (fabsf(a_n_cmd) > a_lat_max * 0.5f)
        pathSpeed *= fmaxf(0.4f, 1.5f - mdiv<F>(fabsf(a_n_cmd), a_lat_max));
    float a_t_cmd = E.kV * (pathSpeed - c.v_t) - mdiv<F>(v_n * kappa * c.v_t, c.metric_actual);
    a_t_cmd = fmaxf(-a_t_max, fminf(a_t_max, a_t_cmd));
    out0 = a_t_cmd * c.tang0 + a_n_total * c.norm0;
    out1 = a_t_cmd * c.tang1 + a_n_total * c.norm1;
}

// findConfident (state.h:93-115) for one parameter factor.
template <int NTH> __device__ __forceinline__ int findConfident(const float (&belief)[NTH], float threshold)
{
    int pt = 0;
#pragma unroll
    for (int th = NTH - 1; th >= 0; th--)
        if (belief[th] > threshold)
            pt = th + 1;
    return pt;
}

// One step of the ego (agent 0) as the environment step moves it: its geometry before the
// step (unit tangent, ds/dt) and its state after it. The ego's motion depends on its own
// action only (the opponents enter its costs and terminal tests, not its dynamics), so when
// the ego draws no noise every Monte-Carlo verification sample that has taken the same
// branch at the same step moves the ego identically; mppi_ego_table computes these rows once
// per plan, and envStep<..., EGO = true> reads them instead of moving the ego itself.
struct __align__(16) EgoRow
{
    float tn0, tn1, sdot;       // before the step
    float pos0, pos1, vel0, vel1; // after the step
    float S, lat, w;            // after the step: arc length, lateral offset, TrackPos weight
    int laps, i0;               // after the step: laps, TrackPos index
};

// The ego's part of envStep (geometry, clamp, position, arc length, velocity, speed cap,
// projection, laps; the same expressions), for an ego that draws no noise. WARP (fast
// flavour only): all 32 lanes of the warp hold the same ego and share the projection's scan.
template <bool F, bool WARP = false>
__device__ __forceinline__ void egoStep(const Track& tr, const EnvParams& E, float ego0, float ego1, DState<1>& s, EgoRow& row)
{
    AgentGeo<1> g;
    agentGeometry<1, F>(tr, E, s, g);
    row.tn0 = g.tn0[0];
    row.tn1 = g.tn1[0];
    row.sdot = g.sdot[0];
    const float prevS = s.S[0];
    float sq = 0.0f;
    sq += ego0 * ego0;
    sq += ego1 * ego1;
    float factor = 1.0f;
    float maxSq = E.maxAccel[0] * E.maxAccel[0];
    if (sq > maxSq)
        factor = mdivsqrt<F>(E.maxAccel[0], sq);
    ego0 *= factor;
    ego1 *= factor;
    s.pos[0] += E.dt * s.vel[0];
    s.pos[1] += E.dt * s.vel[1];
    s.S[0] += E.dt * g.sdot[0];
    s.vel[0] += E.dt * ego0;
    s.vel[1] += E.dt * ego1;
    float sqSpd = sqNorm(s.vel[0], s.vel[1]);
    if (sqSpd > E.maxSpeed[0] * E.maxSpeed[0])
    {
        float sc = mdivsqrt<F>(E.maxSpeed[0], sqSpd);
        s.vel[0] *= sc;
        s.vel[1] *= sc;
    }
    if constexpr (WARP)
        s.S[0] = projectOnTrackWarp(tr, E.trackLength, E.invTrackLength, s.pos[0], s.pos[1], s.S[0], s.lat[0], s.tp[0]);
    else
        s.S[0] = projectOnTrack<F>(tr, E.trackLength, E.invTrackLength, s.pos[0], s.pos[1], s.S[0], s.lat[0], s.tp[0]);
    if (s.S[0] < prevS - E.trackLength * 0.5f)
        s.laps[0]++;
    if (s.S[0] > prevS + E.trackLength * 0.5f)
        s.laps[0]--;
    row.pos0 = s.pos[0];
    row.pos1 = s.pos[1];
    row.vel0 = s.vel[0];
    row.vel1 = s.vel[1];
    row.S = s.S[0];
    row.lat = s.lat[0];
    row.w = s.tp[0].w;
    row.laps = s.laps[0];
    row.i0 = s.tp[0].i0;
}

// The environment noise of every agent is off: no draw of envStep moves the ego.
__device__ __forceinline__ bool egoNoiseFree(const EnvParams& E)
{
    return E.actionNoiseLevel == 0.0f && E.posNoise == 0.0f && E.speedNoise == 0.0f;
}

struct StepOut
{
    int term;
    float bdRaw;  // trackBoundaryDist without the opponent-win shortcut
    bool oppWon;  // isOppWinner
    bool winner;  // isWinner
};

// environmentStep (env_stratrace.h:711-894).
//   UPD: shouldUpdateBelief, BR: considerBranching, LOSE: loseOnOppWin,
//   ALLTH: evaluate the opponent policy under every hypothesis (needed by the belief
//   update) or only under the true one (the result is the same when UPD is false),
//   F: the arithmetic flavour (exact or fast, see mdiv), RNG: the noise source,
//   EGO: the ego's geometry and its move come from *ego (an EgoRow; only for an ego that
//   draws no noise, egoNoiseFree), the step computes the opponents only.
// Work whose result cannot change the step's outputs is not done:
//   * a hypothesis whose policy parameters equal an earlier one's on every term the step
//     evaluates (EnvParams::dupAll / dupNoBlock) takes that one's action;
//   * with BR, once the sample has committed to a branch (predTheta != 0) its belief is
//     read by nothing any more (the branch test runs only while predTheta == 0; the
//     callers with BR return costs, branch records and failure times, never the belief),
//     so the belief update and the other hypotheses' actions it needs are skipped.
template <int NOPP, int NTH, bool UPD, bool BR, bool LOSE, bool ALLTH, bool F = false, class RNG = EnvNoise, bool EGO = false>
__device__ __forceinline__ StepOut envStep(int t, int trueTheta, const Track& tr, const EnvParams& E, float ego0, float ego1, DState<NOPP + 1>& s,
                                           BState<NTH>& bs, bool& branched, float minConf, RNG& rng, const EgoRow* ego = nullptr)
{
    constexpr int NA = NOPP + 1;
    constexpr int A0 = EGO ? 1 : 0; // first agent this step moves itself
    float prevS[NA];
#pragma unroll
    for (int a = 0; a < NA; a++)
        prevS[a] = s.S[a];
    const bool live = !BR || bs.predTheta == 0; // the belief is still read after this step

    AgentGeo<NA> g;
    if constexpr (EGO)
    {
        g.tn0[0] = ego->tn0;
        g.tn1[0] = ego->tn1;
        g.sdot[0] = ego->sdot;
        g.kap[0] = 0.0f; // read by nothing for the ego
    }
    agentGeometry<NA, F, A0>(tr, E, s, g);

    float act0[NA], act1[NA];
    act0[0] = ego0;
    act1[0] = ego1;
    float nom0[ALLTH ? NTH : 1][NOPP], nom1[ALLTH ? NTH : 1][NOPP];
    // every hypothesis took hypothesis 0's action for every opponent, at its noise level:
    // then their likelihoods are equal and the belief update only renormalises the belief
    bool likeAs0 = true;
#pragma unroll
    for (int o = 1; o <= NOPP; o++)
    {
        OppCommon c;
        oppCommon<NOPP, F>(o, tr, E, s, g, c);
        float u0 = 0.f, u1 = 0.f;
        if constexpr (ALLTH)
        {
            const bool blocks = c.shouldBlock[0] || c.shouldBlock[1];
#pragma unroll
            for (int th = 0; th < NTH; th++)
            {
                if (!live && th != trueTheta)
                    continue;
                // an earlier hypothesis with the same action (all of them are evaluated
                // while the belief is live, so that one's action is at hand)
                const int src = live ? (blocks ? E.dupAll[th][o - 1] : E.dupNoBlock[th][o - 1]) : -1;
                if (th > 0 && !(src == 0 && E.noiseAs0[th][o - 1]))
                    likeAs0 = false;
                bool copied = false;
#pragma unroll
                for (int j = 0; j < th; j++)
                    if (src == j)
                    {
                        nom0[th][o - 1] = nom0[j][o - 1];
                        nom1[th][o - 1] = nom1[j][o - 1];
                        copied = true;
                    }
                if (!copied)
                    oppAction<F>(o, th, E, c, nom0[th][o - 1], nom1[th][o - 1]);
                if (th == trueTheta)
                {
                    u0 = nom0[th][o - 1];
                    u1 = nom1[th][o - 1];
                }
            }
        }
        else
        {
            oppAction<F>(o, trueTheta, E, c, nom0[0][o - 1], nom1[0][o - 1]);
            u0 = nom0[0][o - 1];
            u1 = nom1[0][o - 1];
        }
        float an = E.actionNoise[trueTheta][o - 1];
        if (an != 0.0f)
        {
            const float2 nn = rng.next2(); // the stream's next two words, as next() twice
            u0 += an * nn.x;
            u1 += an * nn.y;
        }
        act0[o] = u0;
        act1[o] = u1;
    }
    // 2. clamp + action noise
#pragma unroll
    for (int a = A0; a < NA; a++)
    {
        float sq = 0.0f;
        sq += act0[a] * act0[a];
        sq += act1[a] * act1[a];
        float factor = 1.0f;
        float maxSq = E.maxAccel[a] * E.maxAccel[a];
        if (sq > maxSq)
            factor = mdivsqrt<F>(E.maxAccel[a], sq);
        act0[a] *= factor;
        if (E.actionNoiseLevel != 0.0f)
            act0[a] += rng.next() * E.actionNoiseLevel;
        act1[a] *= factor;
        if (E.actionNoiseLevel != 0.0f)
            act1[a] += rng.next() * E.actionNoiseLevel;
    }
    // 3. position
#pragma unroll
    for (int a = A0; a < NA; a++)
    {
        s.pos[2 * a] += E.dt * s.vel[2 * a];
        s.pos[2 * a + 1] += E.dt * s.vel[2 * a + 1];
    }
    // 4. arc length (ds/dt of the pre-step state)
#pragma unroll
    for (int a = A0; a < NA; a++)
        s.S[a] += E.dt * g.sdot[a];
    // 5. velocity
#pragma unroll
    for (int a = A0; a < NA; a++)
    {
        s.vel[2 * a] += E.dt * act0[a];
        s.vel[2 * a + 1] += E.dt * act1[a];
    }
    // 6. speed cap
#pragma unroll
    for (int a = A0; a < NA; a++)
    {
        float sqSpd = sqNorm(s.vel[2 * a], s.vel[2 * a + 1]);
        if (sqSpd > E.maxSpeed[a] * E.maxSpeed[a])
        {
            float sc = mdivsqrt<F>(E.maxSpeed[a], sqSpd);
            s.vel[2 * a] *= sc;
            s.vel[2 * a + 1] *= sc;
        }
    }
    // 7. state noise
    if (E.posNoise != 0.0f || E.speedNoise != 0.0f)
    {
#pragma unroll
        for (int a = A0; a < NA; a++)
#pragma unroll
            for (int d = 0; d < 2; d++)
            {
                if (E.posNoise != 0.0f)
                    s.pos[a * 2 + d] += rng.next() * E.posNoise;
                if (E.speedNoise != 0.0f)
                    s.vel[a * 2 + d] += rng.next() * E.speedNoise;
            }
    }
    // 8. projection
#pragma unroll
    for (int a = A0; a < NA; a++)
        s.S[a] = projectOnTrack<F>(tr, E.trackLength, E.invTrackLength, s.pos[2 * a], s.pos[2 * a + 1], s.S[a], s.lat[a], s.tp[a]);
    // 9. laps
#pragma unroll
    for (int a = A0; a < NA; a++)
    {
        if (s.S[a] < prevS[a] - E.trackLength * 0.5f)
            s.laps[a]++;
        if (s.S[a] > prevS[a] + E.trackLength * 0.5f)
            s.laps[a]--;
    }
    if constexpr (EGO)
    {
        s.pos[0] = ego->pos0;
        s.pos[1] = ego->pos1;
        s.vel[0] = ego->vel0;
        s.vel[1] = ego->vel1;
        s.S[0] = ego->S;
        s.lat[0] = ego->lat;
        s.laps[0] = ego->laps;
        s.tp[0] = TrackPos{ego->i0, ego->w};
    }
    // 10. belief update (env_stratrace.h:166-222)
    if constexpr (UPD)
    {
        // The fast flavour skips the update when the likelihoods are equal (ALLTH: every
        // hypothesis' action is at hand), leaving the belief as it was where the update
        // would renormalise it (a change of rounding only; the verification's results
        // are checked in distribution).
        if (live && !(F && ALLTH && likeAs0))
        {
            float sum = 0.0f;
#pragma unroll
            for (int th = 0; th < NTH; th++)
            {
                float logLikelihood = 0.0f;
#pragma unroll
                for (int o = 0; o < NOPP; o++)
                {
                    float n0 = nom0[th][o], n1 = nom1[th][o];
                    float sqAccel = 0.0f;
                    sqAccel += n0 * n0;
                    sqAccel += n1 * n1;
                    float scale = 1.0f;
                    if (sqAccel > E.maxAccel[o + 1] * E.maxAccel[o + 1])
                        scale = mdivsqrt<F>(E.maxAccel[o + 1], sqAccel);
                    float sqDist = 0.0f;
                    float dx0 = act0[o + 1] - n0 * scale;
                    sqDist += dx0 * dx0;
                    float dx1 = act1[o + 1] - n1 * scale;
                    sqDist += dx1 * dx1;
                    float an = E.actionNoise[th][o];
                    if constexpr (F)
                        logLikelihood += __fmaf_rn(sqDist, E.llScale[th][o], E.llConst[th][o]); // the same terms, constants folded
                    else
                    {
                        float sqSigma = beliefSqSigma(an);
                        logLikelihood += mdiv<F>(-0.5f * sqDist, sqSigma) - (float)2 * 0.5f * logf(2.0f * M_PIf32) - (float)2 * 0.5f * E.logSqSigma[th][o];
                    }
                }
                bs.belief[th] *= mexp<F>(logLikelihood);
                sum += bs.belief[th];
            }
            if (sum < 1e-20f)
            {
                float uniform = 1.0f / NTH;
#pragma unroll
                for (int th = 0; th < NTH; ++th)
                    bs.belief[th] = uniform;
            }
            else
            {
#pragma unroll
                for (int th = 0; th < NTH; th++)
                    bs.belief[th] = mdiv<F>(bs.belief[th], sum);
            }
        }
    }
    if constexpr (BR)
    {
        int np = findConfident<NTH>(bs.belief, minConf);
        if (bs.predTheta == 0 && np != 0)
        {
            bs.predTheta = np;
            bs.branchingTime = t + 1;
            branched = true;
        }
    }
    // terminal checks (trackBoundaryDist / isOutside / isWinner, env_stratrace.h:226-274)
    StepOut r;
    bool oppWon = false;
#pragma unroll
    for (int o = 1; o <= NOPP; o++)
        if (s.laps[o] >= E.nWinLaps)
            oppWon = true;
    float minSq = INFINITY;
#pragma unroll
    for (int o = 1; o <= NOPP; o++)
        minSq = fminf(minSq, sqNorm(s.pos[2 * o] - s.pos[0], s.pos[2 * o + 1] - s.pos[1]));
    float bdRaw = fminf(msqrt<F>(minSq) - E.droneRadius, E.trackWidth - fabsf(s.lat[0]));
    bool winner = s.laps[0] >= E.nWinLaps;
#pragma unroll
    for (int o = 1; o <= NOPP; o++)
        if (fabsf(s.lat[o]) > E.trackWidth - E.droneRadius)
            winner = true;
    float bdTerm = (LOSE && oppWon) ? -1.0f : bdRaw;
    int term = TERM_NONE;
    if (bdTerm < E.droneRadius)
        term = TERM_LOSE;
    else if (winner)
        term = TERM_WIN;
    else if (!LOSE && (oppWon ? -1.0f : bdRaw) < E.droneRadius)
        term = TERM_OPP_WIN;
    r.term = term;
    r.bdRaw = bdRaw;
    r.oppWon = oppWon;
    r.winner = winner;
    return r;
}

struct MppiCostW
{
    float collDistFactor, boundaryCost, boundaryThresholdFactor, outsideCost, winCost, oppWinCost, finalAdvWeight, finalOppAdvWeight;
};

// stateCost (costs.cuh:7-28) from the step's boundary distance.
__device__ __forceinline__ float stateCost(const StepOut& o, const EnvParams& E, const MppiCostW& w)
{
    float cost = 0.0f;
    float bd = o.bdRaw;
    float danger = w.boundaryThresholdFactor * E.droneRadius;
    if (bd < danger)
        cost += w.boundaryCost * powf(bd / E.droneRadius, 2.0f);
    if (bd < E.droneRadius * w.collDistFactor)
        cost += w.outsideCost;
    if (o.oppWon)
        cost += w.oppWinCost;
    if (o.winner)
        cost -= w.winCost;
    return cost;
}

// PRMPPIstateCost (costs.cuh:44-63).
__device__ __forceinline__ float prStateCost(const StepOut& o, const EnvParams& E, float boundaryThresholdFactor, float boundaryCost, float winCost,
                                             float oppWinCost)
{
    float cost = 0.0f;
    float bd = o.oppWon ? -1.0f : o.bdRaw;
    float danger = boundaryThresholdFactor * E.droneRadius;
    if (bd < danger)
        cost += boundaryCost * powf(bd / E.droneRadius, 2.0f);
    if (o.winner)
        cost -= winCost;
    if (o.oppWon)
        cost += oppWinCost;
    return cost;
}

// PRMPPIsafetyCost (costs.cuh:78-86).
// droneRadius * collDistFactor - bd with one rounding: in the reference both factors
// are kernel parameters used in place, and the product is fused into the subtraction
// (measured against PRMPPIfullRolloutKernel); computing the product once before the
// loop here would otherwise round it separately.
struct SafetyMargin
{
    float r, cdf;
};

__device__ __forceinline__ SafetyMargin safetyMargin(const EnvParams& E, float collDistFactor)
{
    return SafetyMargin{E.droneRadius, collDistFactor};
}

__device__ __forceinline__ float prSafetyCost(const StepOut& o, SafetyMargin m)
{
    return __fmaf_rn(m.r, m.cdf, -o.bdRaw);
}

// finalCost / PRMPPIfinalCost (costs.cuh:31-39, 66-74).
template <int NOPP> __device__ __forceinline__ float finalCost(const DState<NOPP + 1>& s, const EnvParams& E, float finalAdvWeight, float finalOppAdvWeight)
{
    float cost = -finalAdvWeight * (s.S[0] / E.trackLength + s.laps[0]);
    if (finalOppAdvWeight != 0.0f)
    {
        float mx = -INFINITY;
#pragma unroll
        for (int o = 1; o <= NOPP; o++)
            mx = fmaxf(mx, s.S[o] / E.trackLength + s.laps[o]);
        cost += finalOppAdvWeight * mx;
    }
    return cost;
}

} // namespace dr
