// Device model of the gate race: the reference's EnvDroneRace
// (include/environments/env_dronerace.h) with the costs of include/costs.cuh.
// Two agents (ego at iMppi, one PID opponent), gates crossed in order, racelines the
// PID opponents follow. Expression order follows the reference so that nvcc contracts
// the same multiply-adds and the results are bit-identical to the reference's kernels
// on the same inputs; each function cites the lines it follows. Per-hypothesis terms
// of the belief update that do not change within a launch are evaluated once per CTA
// with the same device functions (GateParams::beliefSig2 / beliefNorm).
#pragma once

#include <cstddef>
#include <cstdint>

#include "../../include/drmppi.h"
#include "model.cuh"

namespace dr
{

constexpr int G_NA = DR_GATE_AGENTS;    // env_dronerace_defs.h:8
constexpr int G_NR = DR_GATE_RACELINES; // env_dronerace_defs.h:17
constexpr int G_MAXG = DR_GATE_MAX_GATES;
constexpr int G_MAXO = DR_GATE_MAX_OBSTACLES;
// Track buffer: the racelines [G_NR][NTS][2] plus the sample read when s wraps to exactly
// 1.0f (the last raceline's first sample), padded to 16 bytes; then every raceline again as
// a row of x and a row of y with G_RPAD wrapped samples on each side (samples -G_RPAD ..
// NTS + G_RPAD - 1, 8-byte aligned at even samples), read two samples at a time by the
// raceline walk's margin scan; then per raceline the squared radii [NTS] of the
// projection certificate (projectionCertificate, computed on the host with the track).
constexpr int G_RPAD = 16;
constexpr int G_ROW = NTS + 2 * G_RPAD;
constexpr int GATE_INTERLEAVED_FLOATS = G_NR * NTS * 2 + 4;
constexpr int GATE_CERT = GATE_INTERLEAVED_FLOATS + G_NR * 2 * G_ROW;
constexpr int GATE_TRACK_FLOATS = GATE_CERT + G_NR * NTS;
static_assert(GATE_TRACK_FLOATS % 4 == 0 && G_ROW % 2 == 0 && G_RPAD % 2 == 0 && G_RPAD > 10, "gate track layout");

// raceline r's x row at its sample 0 (the y row follows at + G_ROW)
__host__ __device__ __forceinline__ const float* gateRowX(const float* track, int r)
{
    return track + GATE_INTERLEAVED_FLOATS + 2 * r * G_ROW + G_RPAD;
}

// raceline r's certified squared radii [NTS]
__host__ __device__ __forceinline__ const float* gateCert(const float* track, int r)
{
    return track + GATE_CERT + r * NTS;
}

struct GateParams
{
    float arenaMin[2], arenaMax[2];
    float dt, droneRadius, posNoise, speedNoise, actionNoiseLevel;
    float maxSpeed[G_NA], maxAccel[G_NA];
    int nWinLaps;
    float targetDistance;
    int nGates, nObs, nRound, iMppi;
    float gateCenters[G_MAXG * 2], gateVectors[G_MAXG * 2], gateRadius[G_MAXG];
    float obstacles[G_MAXO * 4], roundCenters[G_MAXO * 2], roundRadius[G_MAXO];
    float pidKp[DR_MAX_THETA], pidKd[DR_MAX_THETA], pidRepF[DR_MAX_THETA], pidRepP[DR_MAX_THETA], pidRepD[DR_MAX_THETA], pidNoise[DR_MAX_THETA];
    int pidRaceline[DR_MAX_THETA];
    // filled on the device by gateDeviceTerms (never copied from the host)
    float beliefSig2[DR_MAX_THETA]; // sigma * sigma, sigma = sqrtf(0.2^2 + actionNoise^2) (env_dronerace.h:242)
    float beliefNorm[DR_MAX_THETA]; // powf(2 pi, DIM / 2) * powf(sigma, DIM) (env_dronerace.h:247)
};

constexpr int GATE_HOST_WORDS = (int)(offsetof(GateParams, beliefSig2) / 4);

__device__ __forceinline__ void gateDeviceTerms(GateParams& dst, const GateParams& src, int tid, int n)
{
    for (int th = tid; th < DR_MAX_THETA; th += n)
    {
        const float sigmaEnv = 0.2f;
        float an = src.pidNoise[th];
        float sigma = sqrtf(sigmaEnv * sigmaEnv + an * an);
        dst.beliefSig2[th] = sigma * sigma;
        dst.beliefNorm[th] = powf(2.0f * M_PIf32, (float)2 / 2.0f) * powf(sigma, (float)2);
    }
}

// SimState (env_dronerace_defs.h:95-103) in registers.
struct GState
{
    float pos[G_NA * 2];
    float vel[G_NA * 2];
    float S[G_NA * G_NR];
    int laps[G_NA];
    int gates[G_NA];
};

__device__ __forceinline__ void loadGState(GState& g, const dr_gate_state& s)
{
#pragma unroll
    for (int i = 0; i < G_NA * 2; i++)
    {
        g.pos[i] = s.pos[i];
        g.vel[i] = s.vel[i];
    }
#pragma unroll
    for (int i = 0; i < G_NA * G_NR; i++)
        g.S[i] = s.S[i];
#pragma unroll
    for (int a = 0; a < G_NA; a++)
    {
        g.laps[a] = s.laps[a];
        g.gates[a] = s.gates[a];
    }
}

__device__ __forceinline__ void storeGState(dr_gate_state& s, const GState& g)
{
    for (int i = 0; i < G_NA * 2; i++)
    {
        s.pos[i] = g.pos[i];
        s.vel[i] = g.vel[i];
    }
    for (int i = 0; i < G_NA * G_NR; i++)
        s.S[i] = g.S[i];
    for (int a = 0; a < G_NA; a++)
    {
        s.laps[a] = g.laps[a];
        s.gates[a] = g.gates[a];
    }
}

// sampleCenterline, env_dronerace.h:55-64. The interpolation (1 - t) p0 + t p1 has two
// products, and the compiler fuses one of them into the addition. The reference's PR-MPPI
// kernels (prmppi_kernels.cu, built for the gate race) fuse the first,
// fma(1 - t, p0, t p1): FUSE_FIRST states that explicitly (found by tracing one
// PRMPPIfullRolloutKernel sample step by step: the PID target, and from it the opponent's
// velocity, differed in the last bits from the other fusion). Without it the expression
// is left to the compiler, which then evaluates it as the reference's MPPI kernels do.
template <bool FUSE_FIRST = false>
__device__ __forceinline__ void sampleCenterline(const float* __restrict__ tp, float s, float& o0, float& o1)
{
    s = s - floorf(s);
    float idx_f = s * NTS;
    int idx0 = (int)idx_f;
    int idx1 = wrapNts(idx0 + 1);
    float t = idx_f - idx0;
    if constexpr (FUSE_FIRST)
    {
        const float omt = 1.0f - t;
        o0 = __fmaf_rn(omt, tp[idx0 * 2 + 0], __fmul_rn(t, tp[idx1 * 2 + 0]));
        o1 = __fmaf_rn(omt, tp[idx0 * 2 + 1], __fmul_rn(t, tp[idx1 * 2 + 1]));
    }
    else
    {
        o0 = (1.0f - t) * tp[idx0 * 2 + 0] + t * tp[idx1 * 2 + 0];
        o1 = (1.0f - t) * tp[idx0 * 2 + 1] + t * tp[idx1 * 2 + 1];
    }
}

// (g + 1) % n for a gate index g >= 0: the remainder only when the index wraps, which a
// gate index in [0, n) does at the last gate
__device__ __forceinline__ int nextGateIndex(int g, int n)
{
    const int next = g + 1;
    return next < n ? next : next % n;
}

// sqDistToSample, :96-102
__device__ __forceinline__ float sqDistToSample(const float* __restrict__ tp, int i, float px, float py)
{
    float sq = 0.f;
    sq += (tp[i * 2 + 0] - px) * (tp[i * 2 + 0] - px);
    sq += (tp[i * 2 + 1] - py) * (tp[i * 2 + 1] - py);
    return sq;
}

// projectOnTrack (full scan), :69-93; reached only for a raceline whose S is negative
// while the agent's first raceline is tracked, so kept out of line
static __device__ __noinline__ float projectFull(const float* __restrict__ tp, float px, float py)
{
    float bestS = 0.0f;
    float bestD2 = __FLT_MAX__;
    float sStep = 1.0f / NTS;
    for (int i = 0; i < NTS; i++)
    {
        float d2 = 0.0f;
        float dx = tp[i * 2 + 0] - px;
        d2 += dx * dx;
        dx = tp[i * 2 + 1] - py;
        d2 += dx * dx;
        if (d2 < bestD2)
        {
            bestD2 = d2;
            bestS = i * sStep;
        }
    }
    return bestS;
}

// findMinAlongDirection, :105-140. The walk ends within NTS samples (the distance
// decreases strictly along it); the bound only makes that explicit. The margin's ten
// samples (the walk's stop and the nine after it) are evaluated as pairs of consecutive
// samples from the padded x / y rows with packed FP32x2 arithmetic (each lane rounds as
// sqDistToSample's scalar sub, mul and fma do), then compared in the walk's order.
//
// walkStop is the walk (moves: the samples it advanced), walkMargin the margin scan from
// the walk's stop bestI, which it may replace.
template <int DELTA>
__device__ __forceinline__ int walkStop(const float* __restrict__ tp, int i0, float px, float py, float baseSq, float& bestSq, int& moves)
{
    int bestI = i0;
    bestSq = baseSq;
    moves = 0;
    int cur = wrapNts(i0 + DELTA + NTS);
    float curSq = sqDistToSample(tp, cur, px, py);
    for (int n = 0; curSq < bestSq && n < NTS; n++)
    {
        bestI = cur;
        bestSq = curSq;
        moves++;
        cur = wrapNts(cur + DELTA + NTS);
        curSq = sqDistToSample(tp, cur, px, py);
    }
    return bestI;
}

template <int DELTA>
__device__ __forceinline__ int walkMargin(const float* __restrict__ rowX, int bestI, float px, float py, float& bestSq)
{
    const int cur = wrapNts(bestI + DELTA + NTS);
    float curSq;
    // samples cur + k DELTA, k = 0..9, lie in [lo, lo + 11] with lo even, inside the rows'
    // padding (cur - 9 >= -9, cur + 9 <= 520)
    const int lo = (DELTA > 0 ? cur : cur - 9) & ~1;
    const int off = cur - lo; // DELTA > 0: 0 or 1; DELTA < 0: 9 or 10
    // from sample -G_RPAD of the raceline's rows
    const uint64_t* __restrict__ X2 = reinterpret_cast<const uint64_t*>(rowX - G_RPAD);
    const uint64_t* __restrict__ Y2 = reinterpret_cast<const uint64_t*>(rowX - G_RPAD + G_ROW);
    uint64_t pxx, pyy;
    asm("mov.b64 %0, {%1, %1};" : "=l"(pxx) : "f"(px));
    asm("mov.b64 %0, {%1, %1};" : "=l"(pyy) : "f"(py));
    float d[12];
#pragma unroll
    for (int q = 0; q < 6; q++)
    {
        const int pi = (lo + G_RPAD) / 2 + q;
        asm("{\n\t.reg .b64 d0, d1, s;\n\t"
            "sub.rn.f32x2 d0, %2, %4;\n\t"
            "sub.rn.f32x2 d1, %3, %5;\n\t"
            "mul.rn.f32x2 s, d0, d0;\n\t"
            "fma.rn.f32x2 s, d1, d1, s;\n\t"
            "mov.b64 {%0, %1}, s;\n\t}"
            : "=f"(d[2 * q]), "=f"(d[2 * q + 1])
            : "l"(X2[pi]), "l"(Y2[pi]), "l"(pxx), "l"(pyy));
    }
#pragma unroll
    for (int k = 0; k < 10; k++)
    {
        // the distance of sample cur + k DELTA: d[off + k DELTA], off taken from its two values
        const int a = DELTA > 0 ? k : 9 - k;
        curSq = (DELTA > 0 ? (off & 1) : (off == 10)) ? d[a + 1] : d[a];
        if (curSq < bestSq)
        {
            bestI = wrapNts(cur + k * DELTA + NTS);
            bestSq = curSq;
        }
    }
    return bestI;
}

// fastProjectOnTrack, :143-209 (its distance output is unused on the path); tp the
// raceline's interleaved samples, rowX its padded x row (gateRowX)
__device__ __forceinline__ float projectGreedy(const float* __restrict__ tp, const float* __restrict__ rowX, const float* __restrict__ cert, float px, float py,
                                              float prevS)
{
    if (prevS < 0)
        return projectFull(tp, px, py);
    int baseI = wrapNts((int)(prevS * NTS + 0.5f)); // prevS >= 0
    float baseSq = sqDistToSample(tp, baseI, px, py);
    float bSq, fSq;
    int nb, nf;
    int bI = walkStop<-1>(tp, baseI, px, py, baseSq, bSq, nb);
    int fI = walkStop<+1>(tp, baseI, px, py, baseSq, fSq, nf);
    // The better stop c is a local minimum of the distances (the walks stopped on either
    // side of it, or descended into it). Within its certified radius every other sample
    // within 20 of it is farther by more than 1e-3 m^2, so no margin sample can win when
    // both margins (bI - 10 .. bI - 1, fI + 1 .. fI + 10) lie within 20 of c.
    const bool back = !(fSq < bSq);
    const int c = back ? bI : fI;
    if (nb + nf <= 10 && (back ? bSq : fSq) <= cert[c])
        return ((float)c) / NTS;
    bI = walkMargin<-1>(rowX, bI, px, py, bSq);
    fI = walkMargin<+1>(rowX, fI, px, py, fSq);
    if (fSq < bSq)
        return ((float)fI) / NTS;
    return ((float)bI) / NTS;
}

// computePIDAction, :473-541, for hypothesis th. The agent is a template parameter and
// the raceline's arc length is selected, so that the state stays in registers. PRK: as the
// reference's PR-MPPI kernels evaluate it (sampleCenterline<true>).
template <int AGENT, bool PRK = false, bool F = false>
__device__ __forceinline__ void pidAction(const GState& s, const GateParams& G, const float* __restrict__ track, int th, float& out0, float& out1)
{
    constexpr int agent = AGENT;
    static_assert(G_NR == 2, "two racelines");
    const int rl = G.pidRaceline[th];
    const float sRl = rl == 0 ? s.S[agent * G_NR] : s.S[agent * G_NR + 1];
    float tx, ty;
    sampleCenterline<PRK>(track + rl * NTS * 2, sRl + G.targetDistance, tx, ty);
    const float cx = s.pos[agent * 2], cy = s.pos[agent * 2 + 1];
    const float vx = s.vel[agent * 2], vy = s.vel[agent * 2 + 1];
    float sqError = 0.0f;
    {
        float e = tx - cx;
        sqError += e * e;
        e = ty - cy;
        sqError += e * e;
    }
    float invDist = mdivsqrt<F>(1.0f, sqError + 1e-5f);
    float vParallelMag = 0.0f;
    {
        float dir = (tx - cx) * invDist;
        vParallelMag += vx * dir;
        dir = (ty - cy) * invDist;
        vParallelMag += vy * dir;
    }
    const float kp = G.pidKp[th], kd = G.pidKd[th];
    {
        float error = (tx - cx) * invDist;
        float latVelError = vx - vParallelMag * error;
        out0 = kp * error + kd * (-latVelError);
        error = (ty - cy) * invDist;
        latVelError = vy - vParallelMag * error;
        out1 = kp * error + kd * (-latVelError);
    }
    const float repF = G.pidRepF[th];
    if (repF != 0.0f)
    {
        constexpr int other = 1 - agent;
        float d0 = s.pos[other * 2] - cx, d1 = s.pos[other * 2 + 1] - cy;
        float dist2 = 0.0f;
        dist2 += d0 * d0;
        dist2 += d1 * d1;
        float dist = msqrt<F>(dist2) + 1e-8f;
        if (dist < G.pidRepD[th] * G.droneRadius * 2.0f)
        {
            float scale = mdiv<F>(repF, powf(dist * 0.5f / G.droneRadius, G.pidRepP[th] + 1.0f));
            out0 -= scale * d0;
            out1 -= scale * d1;
        }
    }
    float sqAccel = 0.0f;
    sqAccel += out0 * out0;
    sqAccel += out1 * out1;
    const float ma = G.maxAccel[agent];
    if (sqAccel > ma * ma)
    {
        float fact = mdivsqrt<F>(ma, sqAccel);
        out0 *= fact;
        out1 *= fact;
    }
}

// updateGates<addMargin>, :412-470
template <bool ADDMARGIN, bool F = false>
__device__ __forceinline__ void updateGates(const GateParams& G, const float* __restrict__ track, GState& s, const float* prevPos, float margin)
{
#pragma unroll
    for (int a = 0; a < G_NA; a++)
    {
        const float px = s.pos[a * 2], py = s.pos[a * 2 + 1];
        if (s.S[a * G_NR] >= 0.0f)
#pragma unroll
            for (int r = 0; r < G_NR; r++)
                s.S[a * G_NR + r] = projectGreedy(track + r * NTS * 2, gateRowX(track, r), gateCert(track, r), px, py, s.S[a * G_NR + r]);
        const int next = nextGateIndex(s.gates[a], G.nGates);
        const float gc0 = G.gateCenters[next * 2], gc1 = G.gateCenters[next * 2 + 1];
        const float gv0 = G.gateVectors[next * 2], gv1 = G.gateVectors[next * 2 + 1];
        const float pp0 = prevPos[a * 2], pp1 = prevPos[a * 2 + 1];
        float num = 0.f, denom = 0.f;
        num += gv0 * (gc0 - pp0);
        denom += gv0 * (px - pp0);
        num += gv1 * (gc1 - pp1);
        denom += gv1 * (py - pp1);
        if (fabsf(denom) < 1e-10f)
            continue;
        float lambda = mdiv<F>(num, denom);
        if (lambda < 0.f || lambda > 1.f)
            continue;
        float sqDist = 0.f;
        float dx = (1.f - lambda) * pp0 + lambda * px - gc0;
        sqDist += dx * dx;
        dx = (1.f - lambda) * pp1 + lambda * py - gc1;
        sqDist += dx * dx;
        float rad = G.gateRadius[next] * G.gateRadius[next];
        if constexpr (ADDMARGIN)
            rad *= margin * margin;
        if (sqDist <= rad)
        {
            s.gates[a]++;
            if (s.gates[a] == G.nGates)
            {
                s.gates[a] = 0;
                s.laps[a]++;
            }
        }
    }
}

// trackBoundaryDist<false>, :262-307 (the opponent-win shortcut is applied by callers);
// ME is the ego's index (envConfig.iMppi)
template <int ME, bool F = false> __device__ __forceinline__ float gateBoundaryDist(const GState& s, const GateParams& G)
{
    constexpr int me = ME;
    const float c0 = s.pos[me * 2], c1 = s.pos[me * 2 + 1];
    float minDist = INFINITY;
    minDist = fminf(minDist, fminf(c0 - G.arenaMin[0], G.arenaMax[0] - c0));
    minDist = fminf(minDist, fminf(c1 - G.arenaMin[1], G.arenaMax[1] - c1));
    for (int i = 0; i < G.nObs; i++)
    {
        float sqDist = 0.0f;
        float dist = fmaxf(0.0f, fmaxf(G.obstacles[i * 4 + 0] - c0, c0 - G.obstacles[(i * 2 + 1) * 2 + 0]));
        sqDist += dist * dist;
        dist = fmaxf(0.0f, fmaxf(G.obstacles[i * 4 + 1] - c1, c1 - G.obstacles[(i * 2 + 1) * 2 + 1]));
        sqDist += dist * dist;
        minDist = fminf(minDist, msqrt<F>(sqDist));
    }
    for (int i = 0; i < G.nRound; i++)
    {
        float sqDist = 0.0f;
        float dx = c0 - G.roundCenters[i * 2];
        sqDist += dx * dx;
        dx = c1 - G.roundCenters[i * 2 + 1];
        sqDist += dx * dx;
        minDist = fminf(minDist, msqrt<F>(sqDist) - G.roundRadius[i]);
    }
    float sqDist = 0.0f;
    float dx = s.pos[0] - s.pos[2];
    sqDist += dx * dx;
    dx = s.pos[1] - s.pos[3];
    sqDist += dx * dx;
    minDist = fminf(minDist, msqrt<F>(sqDist) - G.droneRadius);
    return minDist;
}

// isWinner, :316-360 (the upper arena test adds the radius, as the reference does)
template <int ME> __device__ __forceinline__ bool gateIsWinner(const GState& s, const GateParams& G)
{
    if (s.laps[ME] >= G.nWinLaps)
        return true;
    constexpr int o = 1 - ME;
    const float c0 = s.pos[o * 2], c1 = s.pos[o * 2 + 1];
    const float radius = G.droneRadius;
    if (c0 < G.arenaMin[0] + radius || c0 > G.arenaMax[0] + radius)
        return true;
    if (c1 < G.arenaMin[1] + radius || c1 > G.arenaMax[1] + radius)
        return true;
    for (int i = 0; i < G.nObs; i++)
    {
        float sqDist = 0.0f;
        float dist = fmaxf(0.0f, fmaxf(G.obstacles[i * 4 + 0] - c0, c0 - G.obstacles[(i * 2 + 1) * 2 + 0]));
        sqDist += dist * dist;
        dist = fmaxf(0.0f, fmaxf(G.obstacles[i * 4 + 1] - c1, c1 - G.obstacles[(i * 2 + 1) * 2 + 1]));
        sqDist += dist * dist;
        if (sqDist < radius * radius)
            return true;
    }
    for (int i = 0; i < G.nRound; i++)
    {
        float sqDist = 0.0f;
        float dx = c0 - G.roundCenters[i * 2];
        sqDist += dx * dx;
        dx = c1 - G.roundCenters[i * 2 + 1];
        sqDist += dx * dx;
        if (sqDist < (radius + G.roundRadius[i]) * (radius + G.roundRadius[i]))
            return true;
    }
    return false;
}

// getAnyAdvance, :374-394
template <int AGENT> __device__ __forceinline__ float gateAdvance(const GState& s, const GateParams& G)
{
    constexpr int agent = AGENT;
    float sqGateDist = 0.0f, sqConsGateDist = 0.0f;
    int nextGate = nextGateIndex(s.gates[agent], G.nGates);
    float scale = 0.8f;
    const float* prevC = G.gateCenters + s.gates[agent] * 2;
    const float* nextC = G.gateCenters + nextGate * 2;
    const float p0 = s.pos[agent * 2], p1 = s.pos[agent * 2 + 1];
    sqGateDist += (nextC[0] - p0) * (nextC[0] - p0);
    sqConsGateDist += (nextC[0] - prevC[0]) * (nextC[0] - prevC[0]);
    sqGateDist += (nextC[1] - p1) * (nextC[1] - p1);
    sqConsGateDist += (nextC[1] - prevC[1]) * (nextC[1] - prevC[1]);
    return s.gates[agent] + G.nGates * s.laps[agent] + scale * (1.0f - sqrtf(sqGateDist / sqConsGateDist));
}

// environmentStep<UPD, BR, ADDMARGIN, LOSE>, :546-680. The ego's action is (ego0, ego1);
// the returned StepOut carries what the running cost needs. PRK: the PR-MPPI kernels'
// evaluation of the PID target (sampleCenterline). With BR, once the sample has committed
// to a branch (predTheta != 0) its belief is read by nothing any more (the branch test
// runs only while predTheta == 0, and the callers with BR return costs, branch records
// and failure times, never the belief), so the belief update and the other hypotheses'
// PID actions it needs are skipped; no output changes.
template <int NTH, bool UPD, bool BR, bool ADDMARGIN, bool LOSE, int ME, bool PRK = false, bool F = false, class RNG = EnvNoise>
__device__ __forceinline__ StepOut gateStep(int t, int trueTheta, const float* __restrict__ track, const GateParams& G, float ego0, float ego1,
                                            GState& s, BState<NTH>& bs, bool& branched, float minConf, RNG& rng, float gateMargin)
{
    constexpr int me = ME, opp = 1 - ME;
    const bool live = !BR || bs.predTheta == 0; // the belief is still read after this step
    float prevPos[G_NA * 2];
#pragma unroll
    for (int i = 0; i < G_NA * 2; i++)
        prevPos[i] = s.pos[i];
    // 2. actions: the PID nominal action of every hypothesis (the reference computes all
    // of them; without the belief update only the true one is used)
    float nom0[UPD ? NTH : 1], nom1[UPD ? NTH : 1];
    float u0, u1;
    if (UPD && live)
    {
#pragma unroll
        for (int th = 0; th < (UPD ? NTH : 1); th++)
            pidAction<opp, PRK, F>(s, G, track, th, nom0[th], nom1[th]);
        u0 = nom0[0];
        u1 = nom1[0];
#pragma unroll
        for (int th = 1; th < (UPD ? NTH : 1); th++)
            if (th == trueTheta)
            {
                u0 = nom0[th];
                u1 = nom1[th];
            }
    }
    else
        pidAction<opp, PRK, F>(s, G, track, trueTheta, u0, u1);
    {
        float an = G.pidNoise[trueTheta];
        if (an != 0.0f)
        {
            const float2 nn = rng.next2();
            u0 += an * nn.x;
            u1 += an * nn.y;
        }
    }
    // the actions by agent; the ego is agent `me` (0 or 1), selected without indexing
    float a00 = me == 0 ? ego0 : u0, a01 = me == 0 ? ego1 : u1;
    float a10 = me == 0 ? u0 : ego0, a11 = me == 0 ? u1 : ego1;
    float act[G_NA * 2] = {a00, a01, a10, a11};
    // 3. clamp + action noise
#pragma unroll
    for (int a = 0; a < G_NA; a++)
    {
        float sqNorm = 0.0f;
        sqNorm += act[a * 2] * act[a * 2];
        sqNorm += act[a * 2 + 1] * act[a * 2 + 1];
        float factor = 1.0f;
        float maxSq = G.maxAccel[a] * G.maxAccel[a];
        if (sqNorm > maxSq)
            factor = mdivsqrt<F>(G.maxAccel[a], sqNorm);
#pragma unroll
        for (int d = 0; d < 2; d++)
        {
            act[a * 2 + d] *= factor;
            if (G.actionNoiseLevel != 0.0f)
                act[a * 2 + d] += rng.next() * G.actionNoiseLevel;
        }
    }
    // 4. position, 5. velocity
#pragma unroll
    for (int i = 0; i < G_NA * 2; i++)
        s.pos[i] += G.dt * s.vel[i];
#pragma unroll
    for (int i = 0; i < G_NA * 2; i++)
        s.vel[i] += G.dt * act[i];
    // 6. speed cap (agentSpeed, :43-52)
#pragma unroll
    for (int a = 0; a < G_NA; a++)
    {
        float sq = 0.0f;
        sq += s.vel[a * 2] * s.vel[a * 2];
        sq += s.vel[a * 2 + 1] * s.vel[a * 2 + 1];
        float spd = msqrt<F>(sq);
        if (spd > G.maxSpeed[a])
        {
            float sc = mdiv<F>(G.maxSpeed[a], spd);
            s.vel[a * 2] *= sc;
            s.vel[a * 2 + 1] *= sc;
        }
    }
    // 7. state noise
    if (G.posNoise != 0.0f || G.speedNoise != 0.0f)
    {
#pragma unroll
        for (int i = 0; i < G_NA * 2; i++)
        {
            if (G.posNoise != 0.0f)
                s.pos[i] += rng.next() * G.posNoise;
            if (G.speedNoise != 0.0f)
                s.vel[i] += rng.next() * G.speedNoise;
        }
    }
    // 8. gates
    updateGates<ADDMARGIN, F>(G, track, s, prevPos, gateMargin);
    // 9. belief (updateBelief, :212-258)
    if constexpr (UPD)
    {
        if (live)
        {
            const float maxPIDaccel = G.maxAccel[opp];
            const float oa0 = me == 0 ? act[2] : act[0], oa1 = me == 0 ? act[3] : act[1];
            float sum = 0.0f;
#pragma unroll
            for (int th = 0; th < NTH; th++)
            {
                float sqAccel = 0.f;
                sqAccel += nom0[th] * nom0[th];
                sqAccel += nom1[th] * nom1[th];
                float scale = 1.0f;
                if (sqAccel > maxPIDaccel * maxPIDaccel)
                    scale = mdivsqrt<F>(maxPIDaccel, sqAccel);
                float sqDist = 0.f;
                float dx = oa0 - nom0[th] * scale;
                sqDist += dx * dx;
                dx = oa1 - nom1[th] * scale;
                sqDist += dx * dx;
                bs.belief[th] *= mdiv<F>(mexp<F>(mdiv<F>(-0.5f * sqDist, G.beliefSig2[th])), G.beliefNorm[th]);
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
    // terminal checks (:672-679)
    StepOut r;
    bool oppWon = s.laps[opp] >= G.nWinLaps;
    float bdRaw = gateBoundaryDist<ME, F>(s, G);
    bool winner = gateIsWinner<ME>(s, G);
    float bdTerm = (LOSE && oppWon) ? -1.0f : bdRaw;
    int term = TERM_NONE;
    if (bdTerm < G.droneRadius)
        term = TERM_LOSE;
    else if (winner)
        term = TERM_WIN;
    else if (!LOSE && (oppWon || bdRaw < G.droneRadius))
        term = TERM_OPP_WIN;
    r.term = term;
    r.bdRaw = bdRaw;
    r.oppWon = oppWon;
    r.winner = winner;
    return r;
}

// stateCost (costs.cuh:7-28) from the step's outputs.
__device__ __forceinline__ float gateStateCost(const StepOut& o, const GateParams& G, const MppiCostW& w)
{
    float cost = 0.0f;
    float bd = o.bdRaw;
    float danger = w.boundaryThresholdFactor * G.droneRadius;
    if (bd < danger)
        cost += w.boundaryCost * powf(bd / G.droneRadius, 2.0f);
    if (bd < G.droneRadius * w.collDistFactor)
        cost += w.outsideCost;
    if (o.oppWon)
        cost += w.oppWinCost;
    if (o.winner)
        cost -= w.winCost;
    return cost;
}

// finalCost (costs.cuh:31-39)
template <int ME>
__device__ __forceinline__ float gateFinalCost(const GState& s, const GateParams& G, float finalAdvWeight, float finalOppAdvWeight)
{
    float cost = -finalAdvWeight * gateAdvance<ME>(s, G);
    if (finalOppAdvWeight != 0.0f)
        cost += finalOppAdvWeight * gateAdvance<1 - ME>(s, G);
    return cost;
}

} // namespace dr
