// Differentiable restatement of the strategic race model for the gradient path
// (gradient-refined MPPI): the dynamics, opponent policy, projection, belief update and
// costs of model.cuh (env_stratrace.h:33-894, costs.cuh:7-39, state.h:93-115), with the
// in-rollout noise sources off, evaluated on a value-and-tangent scalar `Dv`.
//
// Each value is computed with explicitly rounded intrinsics (no contraction), so a
// value-only evaluation of a step and a value-and-tangent evaluation of the same step
// produce the same values and take the same discrete decisions: the projection window's
// nearest sample, the action and speed clamps, the branches of the opponent policy, the
// belief threshold and the terminal tests. Division, square root and exponential use the
// hardware approximations (reciprocal, reciprocal square root, exp2; about 2 ulp): the
// gradient path is not held to bit parity with the reference, and these shorten the
// dependent chain of a step, which bounds its latency. The tangent is the directional derivative of
// the piecewise-smooth step along the seeded input direction with every discrete
// decision held. Where only values are used the tangent arithmetic is dead code and the
// compiler removes it.
#pragma once

#include "model.cuh"

namespace dr
{
namespace grad
{

struct Dv
{
    float v, d;
};

__device__ __forceinline__ Dv cst(float x)
{
    return Dv{x, 0.0f};
}

__device__ __forceinline__ Dv operator+(Dv a, Dv b)
{
    return Dv{__fadd_rn(a.v, b.v), a.d + b.d};
}
__device__ __forceinline__ Dv operator-(Dv a, Dv b)
{
    return Dv{__fsub_rn(a.v, b.v), a.d - b.d};
}
__device__ __forceinline__ Dv operator-(Dv a)
{
    return Dv{-a.v, -a.d};
}
__device__ __forceinline__ Dv operator*(Dv a, Dv b)
{
    return Dv{__fmul_rn(a.v, b.v), a.d * b.v + a.v * b.d};
}
__device__ __forceinline__ float rcp(float x)
{
    return __fdividef(1.0f, x);
}
__device__ __forceinline__ Dv operator/(Dv a, Dv b)
{
    const float r = rcp(b.v);
    const float q = __fmul_rn(a.v, r);
    return Dv{q, (a.d - q * b.d) * r};
}
__device__ __forceinline__ Dv operator+(Dv a, float b)
{
    return Dv{__fadd_rn(a.v, b), a.d};
}
__device__ __forceinline__ Dv operator+(float a, Dv b)
{
    return Dv{__fadd_rn(a, b.v), b.d};
}
__device__ __forceinline__ Dv operator-(Dv a, float b)
{
    return Dv{__fsub_rn(a.v, b), a.d};
}
__device__ __forceinline__ Dv operator-(float a, Dv b)
{
    return Dv{__fsub_rn(a, b.v), -b.d};
}
__device__ __forceinline__ Dv operator*(Dv a, float b)
{
    return Dv{__fmul_rn(a.v, b), a.d * b};
}
__device__ __forceinline__ Dv operator*(float a, Dv b)
{
    return Dv{__fmul_rn(a, b.v), a * b.d};
}
__device__ __forceinline__ Dv operator/(Dv a, float b)
{
    const float r = rcp(b);
    return Dv{__fmul_rn(a.v, r), a.d * r};
}
__device__ __forceinline__ Dv operator/(float a, Dv b)
{
    const float r = rcp(b.v);
    const float q = __fmul_rn(a, r);
    return Dv{q, -q * b.d * r};
}
__device__ __forceinline__ Dv& operator+=(Dv& a, Dv b)
{
    return a = a + b;
}
__device__ __forceinline__ Dv& operator-=(Dv& a, Dv b)
{
    return a = a - b;
}
__device__ __forceinline__ Dv& operator*=(Dv& a, Dv b)
{
    return a = a * b;
}
__device__ __forceinline__ Dv& operator*=(Dv& a, float b)
{
    return a = a * b;
}
__device__ __forceinline__ Dv& operator/=(Dv& a, Dv b)
{
    return a = a / b;
}

__device__ __forceinline__ Dv dsqrt(Dv a)
{
    if (!(a.v > 0.0f))
        return Dv{0.0f, 0.0f};
    const float rs = rsqrtf(a.v);
    return Dv{__fmul_rn(a.v, rs), a.d * 0.5f * rs};
}
__device__ __forceinline__ Dv dexp(Dv a)
{
    const float e = __expf(a.v);
    return Dv{e, a.d * e};
}
__device__ __forceinline__ Dv dabs(Dv a)
{
    return Dv{fabsf(a.v), a.v < 0.0f ? -a.d : a.d};
}
__device__ __forceinline__ Dv dmin(Dv a, Dv b)
{
    return Dv{fminf(a.v, b.v), a.v <= b.v ? a.d : b.d};
}
__device__ __forceinline__ Dv dmax(Dv a, Dv b)
{
    return Dv{fmaxf(a.v, b.v), a.v >= b.v ? a.d : b.d};
}
__device__ __forceinline__ Dv dfloor(Dv a)
{
    return Dv{floorf(a.v), 0.0f};
}
// copysignf(a, sign of s)
__device__ __forceinline__ Dv dcopysign(Dv a, float s)
{
    const float r = copysignf(a.v, s);
    return Dv{r, (signbit(r) != signbit(a.v)) ? -a.d : a.d};
}
__device__ __forceinline__ Dv sq2(Dv x, Dv y)
{
    return x * x + y * y;
}

// ---- state -------------------------------------------------------------------------------

// Continuous state of a step's input and output, in the canonical order used for seeding,
// tangents and adjoints: pos[2 NA] | vel[2 NA] | S[NA] | lat[NA] | belief[NTH].
template <int NA, int NTH> struct XState
{
    static constexpr int NX = 6 * NA + NTH;
    Dv pos[2 * NA], vel[2 * NA], S[NA], lat[NA], belief[NTH];
    int laps[NA];
    int predTheta, branchingTime;
};

// Sets the tangent of input j (state component j < NX, ego action component NX + d) to 1
// and every other tangent to 0.
template <int NA, int NTH> __device__ __forceinline__ void seed(XState<NA, NTH>& s, Dv& u0, Dv& u1, int j)
{
    int i = 0;
#pragma unroll
    for (int k = 0; k < 2 * NA; k++)
        s.pos[k].d = (i++ == j) ? 1.0f : 0.0f;
#pragma unroll
    for (int k = 0; k < 2 * NA; k++)
        s.vel[k].d = (i++ == j) ? 1.0f : 0.0f;
#pragma unroll
    for (int k = 0; k < NA; k++)
        s.S[k].d = (i++ == j) ? 1.0f : 0.0f;
#pragma unroll
    for (int k = 0; k < NA; k++)
        s.lat[k].d = (i++ == j) ? 1.0f : 0.0f;
#pragma unroll
    for (int k = 0; k < NTH; k++)
        s.belief[k].d = (i++ == j) ? 1.0f : 0.0f;
    u0.d = (i++ == j) ? 1.0f : 0.0f;
    u1.d = (i == j) ? 1.0f : 0.0f;
}

// sum_i mu[i] * tangent of state component i
template <int NA, int NTH> __device__ __forceinline__ float dotTangent(const XState<NA, NTH>& s, const float* mu)
{
    float r = 0.0f;
    int i = 0;
#pragma unroll
    for (int k = 0; k < 2 * NA; k++)
        r += mu[i++] * s.pos[k].d;
#pragma unroll
    for (int k = 0; k < 2 * NA; k++)
        r += mu[i++] * s.vel[k].d;
#pragma unroll
    for (int k = 0; k < NA; k++)
        r += mu[i++] * s.S[k].d;
#pragma unroll
    for (int k = 0; k < NA; k++)
        r += mu[i++] * s.lat[k].d;
#pragma unroll
    for (int k = 0; k < NTH; k++)
        r += mu[i++] * s.belief[k].d;
    return r;
}

// Record of a state in shared memory: NX values, laps[NA], predTheta, branchingTime, and
// two words for the caller (the branch origin of the plan time and the discount).
template <int NA, int NTH> constexpr int recWords()
{
    return XState<NA, NTH>::NX + NA + 4;
}

template <int NA, int NTH> __device__ __forceinline__ void storeRec(float* r, const XState<NA, NTH>& s, int tOrigin, float decay)
{
    int i = 0;
#pragma unroll
    for (int k = 0; k < 2 * NA; k++)
        r[i++] = s.pos[k].v;
#pragma unroll
    for (int k = 0; k < 2 * NA; k++)
        r[i++] = s.vel[k].v;
#pragma unroll
    for (int k = 0; k < NA; k++)
        r[i++] = s.S[k].v;
#pragma unroll
    for (int k = 0; k < NA; k++)
        r[i++] = s.lat[k].v;
#pragma unroll
    for (int k = 0; k < NTH; k++)
        r[i++] = s.belief[k].v;
#pragma unroll
    for (int k = 0; k < NA; k++)
        r[i++] = __int_as_float(s.laps[k]);
    r[i++] = __int_as_float(s.predTheta);
    r[i++] = __int_as_float(s.branchingTime);
    r[i++] = __int_as_float(tOrigin);
    r[i] = decay;
}

template <int NA, int NTH> __device__ __forceinline__ void loadRec(const float* r, XState<NA, NTH>& s, int& tOrigin, float& decay)
{
    int i = 0;
#pragma unroll
    for (int k = 0; k < 2 * NA; k++)
        s.pos[k] = cst(r[i++]);
#pragma unroll
    for (int k = 0; k < 2 * NA; k++)
        s.vel[k] = cst(r[i++]);
#pragma unroll
    for (int k = 0; k < NA; k++)
        s.S[k] = cst(r[i++]);
#pragma unroll
    for (int k = 0; k < NA; k++)
        s.lat[k] = cst(r[i++]);
#pragma unroll
    for (int k = 0; k < NTH; k++)
        s.belief[k] = cst(r[i++]);
#pragma unroll
    for (int k = 0; k < NA; k++)
        s.laps[k] = __float_as_int(r[i++]);
    s.predTheta = __float_as_int(r[i++]);
    s.branchingTime = __float_as_int(r[i++]);
    tOrigin = __float_as_int(r[i++]);
    decay = r[i];
}

// ---- track sampling (env_stratrace.h:44-85) ------------------------------------------

struct GPos
{
    int i0;
    Dv w;
};

__device__ __forceinline__ GPos gpos(Dv s, float L)
{
    s = s / L;
    s = s - dfloor(s);
    Dv idx = s * (float)NTS;
    const int i0 = (int)idx.v;
    return GPos{i0, idx - (float)i0};
}

__device__ __forceinline__ void gsample2(const float* __restrict__ arr, GPos q, Dv& o0, Dv& o1)
{
    const int i0 = q.i0, i1 = wrapNts(i0 + 1);
    const Dv om = 1.0f - q.w;
    o0 = om * arr[i0 * 2 + 0] + q.w * arr[i1 * 2 + 0];
    o1 = om * arr[i0 * 2 + 1] + q.w * arr[i1 * 2 + 1];
}

__device__ __forceinline__ Dv gsample1(const float* __restrict__ arr, GPos q)
{
    const int i0 = q.i0, i1 = wrapNts(i0 + 1);
    return (1.0f - q.w) * arr[i0] + q.w * arr[i1];
}

// fastProjectOnTrack<false> (env_stratrace.h:88-162): nearest centreline sample in the
// window around prevS (by value; first minimum in increasing index order), then the
// nearest point of its two adjacent segments. Returns S, writes the signed lateral
// distance.
__device__ __forceinline__ Dv gproject(const Track& tr, float L, Dv px, Dv py, float prevS, Dv& lat)
{
    prevS = __fmul_rn(prevS, rcp(L));
    prevS = __fsub_rn(prevS, floorf(prevS));
    const int idxPrev = (int)__fmul_rn(prevS, (float)NTS);
    float best = INFINITY;
    int bestJ = idxPrev - WIN;
    for (int j = idxPrev - WIN; j <= idxPrev + WIN; j++)
    {
        const float d0 = __fsub_rn(tr.p[j * 2 + 0], px.v), d1 = __fsub_rn(tr.p[j * 2 + 1], py.v);
        const float sq = __fadd_rn(__fmul_rn(d0, d0), __fmul_rn(d1, d1));
        if (sq < best)
        {
            best = sq;
            bestJ = j;
        }
    }
    const int bestInd = wrapNts(bestJ + NTS); // bestJ >= -WIN
    Dv bestSq = cst(INFINITY), bestS = cst(0.0f), cx = cst(0.0f), cy = cst(0.0f);
#pragma unroll
    for (int seg = -1; seg <= 0; ++seg)
    {
        const int aj = bestInd + seg; // -1 .. 511 (the padded grid holds p[-1] and p[512])
        const int a = aj < 0 ? aj + NTS : aj;
        const float ax = tr.p[aj * 2], ay = tr.p[aj * 2 + 1];
        const float abx = __fsub_rn(tr.p[aj * 2 + 2], ax), aby = __fsub_rn(tr.p[aj * 2 + 3], ay);
        const float sqAB = __fadd_rn(__fmul_rn(abx, abx), __fmul_rn(aby, aby));
        Dv t = cst(0.0f);
        if (sqAB > 1e-12f)
        {
            t = ((px - ax) * abx + (py - ay) * aby) / sqAB;
            t = dmax(cst(0.0f), dmin(t, cst(1.0f)));
        }
        const Dv projx = ax + t * abx, projy = ay + t * aby;
        const Dv sqDist = sq2(px - projx, py - projy);
        if (sqDist.v < bestSq.v)
        {
            bestSq = sqDist;
            bestS = ((float)a + t) / (float)NTS * L;
            cx = projx;
            cy = projy;
        }
    }
    Dv tg0, tg1;
    gsample2(tr.t, gpos(bestS, L), tg0, tg1);
    const Dv cross = (-tg1) * (px - cx) + tg0 * (py - cy);
    lat = dcopysign(dsqrt(bestSq), cross.v);
    return bestS;
}

// ---- per-step agent quantities -------------------------------------------------------

template <int NA> struct GGeo
{
    Dv tn0[NA], tn1[NA], kap[NA], sdot[NA];
    GPos tp[NA];
};

template <int NA, int NTH> __device__ __forceinline__ void ggeometry(const Track& tr, const EnvParams& E, const XState<NA, NTH>& s, GGeo<NA>& g)
{
#pragma unroll
    for (int a = 0; a < NA; a++)
    {
        g.tp[a] = gpos(s.S[a], E.trackLength);
        Dv t0, t1;
        gsample2(tr.t, g.tp[a], t0, t1);
        const Dv inv = 1.0f / dsqrt(sq2(t0, t1));
        g.tn0[a] = t0 * inv;
        g.tn1[a] = t1 * inv;
        g.kap[a] = gsample1(tr.k, g.tp[a]);
        Dv metric = 1.0f - g.kap[a] * s.lat[a];
        if (fabsf(metric.v) < 1e-12f)
            metric = cst(copysignf(1e-12f, metric.v));
        g.sdot[a] = (g.tn0[a] * s.vel[2 * a] + g.tn1[a] * s.vel[2 * a + 1]) / metric;
    }
}

// Hypothesis-independent part of the opponent policy (env_stratrace.h:318-461, 611-706).
struct GOpp
{
    Dv deltaS[2], deltaE[2], latJ[2], sdotJ[2], oppLong[2];
    float blockTol[2];
    bool shouldBlock[2], fasterThanJ[2];
    Dv sdot_i;
    float maxLatDis, e_n_max, maxAccel, maxAccelSq;
    Dv tang0, tang1, norm0, norm1, kappa, e_n, v_t, v_n, metric_actual, a_centripetal, a_lat_max, distPos, distNeg;
    bool brakePos, brakeNeg;
};

template <int NOPP, int NTH>
__device__ __forceinline__ void goppCommon(int iOpp, const Track& tr, const EnvParams& E, const XState<NOPP + 1, NTH>& s, const GGeo<NOPP + 1>& g,
                                           GOpp& c)
{
    const float L = E.trackLength;
    int iAhead = 0;
    Dv dAhead = s.S[0] - s.S[iOpp];
    if (dAhead.v < 0.0f)
        dAhead = dAhead + L;
#pragma unroll
    for (int j = 1; j <= NOPP; j++)
        if (j != iOpp)
        {
            Dv d = s.S[j] - s.S[iOpp];
            if (d.v < 0.0f)
                d = d + L;
            if (d.v < dAhead.v)
            {
                dAhead = d;
                iAhead = j;
            }
        }
    int iBehind = 0;
    Dv dBehind = s.S[0] - s.S[iOpp];
    if (dBehind.v > 0.0f)
        dBehind = dBehind - L;
#pragma unroll
    for (int j = 1; j <= NOPP; j++)
        if (j != iOpp)
        {
            Dv d = s.S[j] - s.S[iOpp];
            if (d.v > 0.0f)
                d = d - L;
            if (d.v > dBehind.v)
            {
                dBehind = d;
                iBehind = j;
            }
        }
    c.sdot_i = g.sdot[iOpp];
#pragma unroll
    for (int k = 0; k <= 1; k++)
    {
        const int j = k ? iAhead : iBehind;
        const Dv deltaS = k ? dAhead : dBehind;
        Dv latJ = s.lat[0], tj0 = g.tn0[0], tj1 = g.tn1[0], sdj = g.sdot[0], vj0 = s.vel[0], vj1 = s.vel[1];
        float msj = E.maxSpeed[0];
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
        c.deltaS[k] = deltaS;
        c.deltaE[k] = latJ - s.lat[iOpp];
        c.latJ[k] = latJ;
        c.sdotJ[k] = sdj;
        c.blockTol[k] = __fmul_rn(msj, 0.3f);
        c.shouldBlock[k] = (deltaS.v < 0.0f) && (deltaS.v > -L * 0.25f) && (__fadd_rn(sdj.v, c.blockTol[k]) > c.sdot_i.v);
        c.fasterThanJ[k] = c.sdot_i.v > sdj.v;
        c.oppLong[k] = vj0 * tj0 + vj1 * tj1;
    }
    c.maxLatDis = __fsub_rn(E.trackWidth, __fmul_rn(E.droneRadius, E.maxOppLatDistFact));
    c.maxAccel = E.maxAccel[iOpp];
    c.maxAccelSq = __fmul_rn(c.maxAccel, c.maxAccel);
    Dv pc0, pc1;
    gsample2(tr.p, g.tp[iOpp], pc0, pc1);
    c.tang0 = g.tn0[iOpp];
    c.tang1 = g.tn1[iOpp];
    c.kappa = g.kap[iOpp];
    c.norm0 = -c.tang1;
    c.norm1 = c.tang0;
    const Dv pos0 = s.pos[iOpp * 2], pos1 = s.pos[iOpp * 2 + 1];
    const Dv vel0 = s.vel[iOpp * 2], vel1 = s.vel[iOpp * 2 + 1];
    c.e_n = (pos0 - pc0) * c.norm0 + (pos1 - pc1) * c.norm1;
    c.v_t = vel0 * c.tang0 + vel1 * c.tang1;
    c.v_n = vel0 * c.norm0 + vel1 * c.norm1;
    c.e_n_max = __fsub_rn(E.trackWidth, __fmul_rn(E.droneRadius, 1.2f));
    Dv metric_actual = 1.0f - c.kappa * c.e_n;
    if (fabsf(metric_actual.v) < 1e-6f)
        metric_actual = cst(copysignf(1e-6f, metric_actual.v));
    c.metric_actual = metric_actual;
    c.a_centripetal = c.v_t * c.v_t * c.kappa / metric_actual;
    c.a_lat_max = dmax(c.maxAccel - dabs(c.a_centripetal), cst(__fmul_rn(c.maxAccel, 0.2f)));
    c.distPos = dmax(c.e_n_max - c.e_n, cst(0.001f));
    c.distNeg = dmax(c.e_n_max + c.e_n, cst(0.001f));
    c.brakePos = c.v_n.v > 0.0f && (c.v_n * c.v_n).v > (1.8f * c.a_lat_max * c.distPos).v;
    c.brakeNeg = c.v_n.v < 0.0f && (c.v_n * c.v_n).v > (1.8f * c.a_lat_max * c.distNeg).v;
}

// Hypothesis-dependent part: target lateral offset, speed goal and the resulting
// acceleration of opponent iOpp under hypothesis th.
__device__ __forceinline__ void goppAction(int iOpp, int th, const EnvParams& E, const GOpp& c, Dv& out0, Dv& out1)
{
    const float s1 = E.s1[th][iOpp - 1], s2 = E.s2[th][iOpp - 1], s3 = E.s3[th][iOpp - 1];
    Dv latDis = cst(0.0f);
    const float baseSpeed = __fmul_rn(E.speedScale[th][iOpp - 1], E.maxSpeed[iOpp]);
    Dv speedGoal = cst(baseSpeed);
#pragma unroll
    for (int k = 0; k <= 1; k++)
    {
        const Dv deltaS = c.deltaS[k], deltaE = c.deltaE[k];
        const bool shouldOvertake = c.fasterThanJ[k] && (fabsf(deltaE.v) < s1);
        if (!c.shouldBlock[k] && !shouldOvertake)
            continue;
        const Dv factor = dexp((-s2) * deltaS * deltaS);
        if (c.shouldBlock[k])
            latDis += c.latJ[k] * (1.0f - dexp((-s3) * (c.sdotJ[k] + c.blockTol[k] - c.sdot_i))) * factor;
        if (shouldOvertake)
        {
            latDis += (c.latJ[k] - copysignf(s1, deltaE.v)) * factor;
            const Dv oppLongSpeed = c.oppLong[k];
            if (deltaS.v < 3 * E.droneRadius)
                speedGoal = dmin(speedGoal, 0.7f * oppLongSpeed);
            else if (deltaS.v < 6 * E.droneRadius && s1 > 1e-6f)
            {
                const Dv latFactor = dabs(deltaE) / s1;
                speedGoal = dmin(speedGoal, latFactor * oppLongSpeed + (1.0f - latFactor) * baseSpeed);
            }
        }
    }
    const Dv latDisRaw = dmax(cst(-c.maxLatDis), dmin(cst(c.maxLatDis), latDis));
    const float maxAccel = c.maxAccel, dt = E.dt;
    const Dv a_lat_max = c.a_lat_max, v_n = c.v_n;
    const Dv latDisC = dmax(cst(-c.e_n_max), dmin(cst(c.e_n_max), latDisRaw));
    const Dv e_error = latDisC - c.e_n;
    Dv a_n_cmd;
    if (c.brakePos)
        a_n_cmd = -a_lat_max;
    else if (c.brakeNeg)
        a_n_cmd = a_lat_max;
    else if (fabsf(e_error.v) < 0.02f)
    {
        const Dv kp = a_lat_max / 0.02f;
        a_n_cmd = kp * e_error - 2.0f * dsqrt(kp) * v_n;
        a_n_cmd = dmax(-a_lat_max, dmin(a_lat_max, a_n_cmd));
    }
    else
    {
        const Dv stopping = v_n * v_n / (2.0f * a_lat_max);
        const bool toward = (e_error.v > 0.0f && v_n.v > 0.0f) || (e_error.v < 0.0f && v_n.v < 0.0f);
        const bool decel = toward && stopping.v >= __fmul_rn(fabsf(e_error.v), 0.95f);
        a_n_cmd = (e_error.v > 0.0f) ? a_lat_max : -a_lat_max;
        if (decel)
            a_n_cmd = -a_n_cmd;
        const Dv v_next = v_n + a_n_cmd * dt;
        if (v_next.v > 0.0f)
        {
            const Dv v_safe = dsqrt(2.0f * a_lat_max * c.distPos);
            if (v_next.v > v_safe.v)
                a_n_cmd = (v_safe - v_n) / dt;
        }
        else
        {
            const Dv v_safe = dsqrt(2.0f * a_lat_max * c.distNeg);
            if ((-v_next).v > v_safe.v)
                a_n_cmd = (-v_safe - v_n) / dt;
        }
    }
    const Dv a_n_total = dmax(cst(-maxAccel), dmin(cst(maxAccel), a_n_cmd + c.a_centripetal));
    const Dv a_t_max = dsqrt(dmax(c.maxAccelSq - a_n_total * a_n_total, cst(0.0f)));
    const Dv kappa = c.kappa;
    const Dv kappa_eff = kappa / (1.0f - kappa * latDisC + 1e-6f);
    Dv pathSpeed = dmin(speedGoal, dsqrt(maxAccel / dmax(dabs(kappa_eff), cst(1e-12f))));
    if (fabsf(a_n_cmd.v) > __fmul_rn(a_lat_max.v, 0.5f))
        pathSpeed *= dmax(cst(0.4f), 1.5f - dabs(a_n_cmd) / a_lat_max);
    Dv a_t_cmd = E.kV * (pathSpeed - c.v_t) - v_n * kappa * c.v_t / c.metric_actual;
    a_t_cmd = dmax(-a_t_max, dmin(a_t_max, a_t_cmd));
    out0 = a_t_cmd * c.tang0 + a_n_total * c.norm0;
    out1 = a_t_cmd * c.tang1 + a_n_total * c.norm1;
}

// Per-step quantities the costs need.
struct GOut
{
    int term;
    Dv bdRaw;
    bool oppWon, winner;
};

// environmentStep<true, true, loseOnOppWin = true> (env_stratrace.h:711-894) with the
// noise sources off; `branched` reports a new commitment (state.h:93-115).
template <int NOPP, int NTH>
__device__ __forceinline__ GOut gstep(int t, int trueTheta, const Track& tr, const EnvParams& E, Dv ego0, Dv ego1, XState<NOPP + 1, NTH>& s,
                                      float minConf, bool& branched)
{
    constexpr int NA = NOPP + 1;
    const float L = E.trackLength;
    float prevS[NA];
#pragma unroll
    for (int a = 0; a < NA; a++)
        prevS[a] = s.S[a].v;
    GGeo<NA> g;
    ggeometry<NA, NTH>(tr, E, s, g);

    Dv act0[NA], act1[NA];
    act0[0] = ego0;
    act1[0] = ego1;
    Dv nom0[NTH][NOPP], nom1[NTH][NOPP];
#pragma unroll
    for (int o = 1; o <= NOPP; o++)
    {
        GOpp c;
        goppCommon<NOPP, NTH>(o, tr, E, s, g, c);
        Dv u0 = cst(0.0f), u1 = cst(0.0f);
#pragma unroll
        for (int th = 0; th < NTH; th++)
        {
            goppAction(o, th, E, c, nom0[th][o - 1], nom1[th][o - 1]);
            if (th == trueTheta)
            {
                u0 = nom0[th][o - 1];
                u1 = nom1[th][o - 1];
            }
        }
        act0[o] = u0;
        act1[o] = u1;
    }
    // clamp to the acceleration limit
#pragma unroll
    for (int a = 0; a < NA; a++)
    {
        const Dv sq = sq2(act0[a], act1[a]);
        if (sq.v > __fmul_rn(E.maxAccel[a], E.maxAccel[a]))
        {
            const Dv f = E.maxAccel[a] / dsqrt(sq);
            act0[a] *= f;
            act1[a] *= f;
        }
    }
    // integrate (position with the pre-step velocity, arc length with the pre-step ds/dt)
    Dv Sint[NA];
#pragma unroll
    for (int a = 0; a < NA; a++)
    {
        s.pos[2 * a] += E.dt * s.vel[2 * a];
        s.pos[2 * a + 1] += E.dt * s.vel[2 * a + 1];
        Sint[a] = s.S[a] + E.dt * g.sdot[a];
        s.vel[2 * a] += E.dt * act0[a];
        s.vel[2 * a + 1] += E.dt * act1[a];
        const Dv sqSpd = sq2(s.vel[2 * a], s.vel[2 * a + 1]);
        if (sqSpd.v > __fmul_rn(E.maxSpeed[a], E.maxSpeed[a]))
        {
            const Dv sc = E.maxSpeed[a] / dsqrt(sqSpd);
            s.vel[2 * a] *= sc;
            s.vel[2 * a + 1] *= sc;
        }
    }
    // projection and laps
#pragma unroll
    for (int a = 0; a < NA; a++)
    {
        s.S[a] = gproject(tr, L, s.pos[2 * a], s.pos[2 * a + 1], Sint[a].v, s.lat[a]);
        if (s.S[a].v < __fsub_rn(prevS[a], __fmul_rn(L, 0.5f)))
            s.laps[a]++;
        if (s.S[a].v > __fadd_rn(prevS[a], __fmul_rn(L, 0.5f)))
            s.laps[a]--;
    }
    // belief update (env_stratrace.h:166-222)
    Dv sum = cst(0.0f);
#pragma unroll
    for (int th = 0; th < NTH; th++)
    {
        Dv ll = cst(0.0f);
#pragma unroll
        for (int o = 0; o < NOPP; o++)
        {
            const Dv n0 = nom0[th][o], n1 = nom1[th][o];
            const Dv sqA = sq2(n0, n1);
            Dv scale = cst(1.0f);
            if (sqA.v > __fmul_rn(E.maxAccel[o + 1], E.maxAccel[o + 1]))
                scale = E.maxAccel[o + 1] / dsqrt(sqA);
            const Dv sqDist = sq2(act0[o + 1] - n0 * scale, act1[o + 1] - n1 * scale);
            const float sqSigma = beliefSqSigma(E.actionNoise[th][o]);
            ll = ll + ((-0.5f) * sqDist / sqSigma - logf(2.0f * M_PIf32) - E.logSqSigma[th][o]);
        }
        s.belief[th] *= dexp(ll);
        sum += s.belief[th];
    }
    if (sum.v < 1e-20f)
    {
#pragma unroll
        for (int th = 0; th < NTH; th++)
            s.belief[th] = cst(1.0f / NTH);
    }
    else
    {
#pragma unroll
        for (int th = 0; th < NTH; th++)
            s.belief[th] /= sum;
    }
    // branching (findConfident, state.h:93-115)
    int np = 0;
#pragma unroll
    for (int th = NTH - 1; th >= 0; th--)
        if (s.belief[th].v > minConf)
            np = th + 1;
    branched = false;
    if (s.predTheta == 0 && np != 0)
    {
        s.predTheta = np;
        s.branchingTime = t + 1;
        branched = true;
    }
    // terminal tests (trackBoundaryDist / isOutside / isWinner, env_stratrace.h:226-274)
    GOut r;
    bool oppWon = false;
#pragma unroll
    for (int o = 1; o <= NOPP; o++)
        if (s.laps[o] >= E.nWinLaps)
            oppWon = true;
    Dv minSq = cst(INFINITY);
#pragma unroll
    for (int o = 1; o <= NOPP; o++)
        minSq = dmin(minSq, sq2(s.pos[2 * o] - s.pos[0], s.pos[2 * o + 1] - s.pos[1]));
    const Dv bdRaw = dmin(dsqrt(minSq) - E.droneRadius, E.trackWidth - dabs(s.lat[0]));
    bool winner = s.laps[0] >= E.nWinLaps;
#pragma unroll
    for (int o = 1; o <= NOPP; o++)
        if (fabsf(s.lat[o].v) > __fsub_rn(E.trackWidth, E.droneRadius))
            winner = true;
    const float bdTerm = oppWon ? -1.0f : bdRaw.v;
    r.term = TERM_NONE;
    if (bdTerm < E.droneRadius)
        r.term = TERM_LOSE;
    else if (winner)
        r.term = TERM_WIN;
    r.bdRaw = bdRaw;
    r.oppWon = oppWon;
    r.winner = winner;
    return r;
}

// The cost weights the gradient is taken with respect to, in this order.
enum WeightIndex
{
    W_BOUNDARY = 0,
    W_OUTSIDE = 1,
    W_WIN = 2,
    W_OPP_WIN = 3,
    W_FINAL_ADV = 4,
    W_FINAL_OPP_ADV = 5,
    N_WEIGHTS = 6
};

// stateCost (costs.cuh:7-28); feat[i] += d cost / d weight i (the weights enter linearly).
__device__ __forceinline__ Dv gcost(const GOut& o, const EnvParams& E, const MppiCostW& w, float* feat)
{
    Dv c = cst(0.0f);
    const Dv bd = o.bdRaw;
    const float r = E.droneRadius;
    if (bd.v < __fmul_rn(w.boundaryThresholdFactor, r))
    {
        const Dv q = bd / r;
        const Dv q2 = q * q;
        c += w.boundaryCost * q2;
        feat[W_BOUNDARY] = q2.v;
    }
    if (bd.v < __fmul_rn(r, w.collDistFactor))
    {
        c = c + w.outsideCost;
        feat[W_OUTSIDE] = 1.0f;
    }
    if (o.oppWon)
    {
        c = c + w.oppWinCost;
        feat[W_OPP_WIN] = 1.0f;
    }
    if (o.winner)
    {
        c = c - w.winCost;
        feat[W_WIN] = -1.0f;
    }
    return c;
}

// finalCost (costs.cuh:31-39); feat as for gcost.
template <int NA, int NTH> __device__ __forceinline__ Dv gfinal(const XState<NA, NTH>& s, const EnvParams& E, const MppiCostW& w, float* feat)
{
    const float L = E.trackLength;
    const Dv adv = s.S[0] / L + (float)s.laps[0];
    Dv c = (-w.finalAdvWeight) * adv;
    feat[W_FINAL_ADV] = -adv.v;
    Dv mx = cst(-INFINITY);
#pragma unroll
    for (int o = 1; o < NA; o++)
        mx = dmax(mx, s.S[o] / L + (float)s.laps[o]);
    feat[W_FINAL_OPP_ADV] = mx.v;
    if (w.finalOppAdvWeight != 0.0f)
        c += w.finalOppAdvWeight * mx;
    return c;
}

} // namespace grad
} // namespace dr
