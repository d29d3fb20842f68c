// TEST INFRASTRUCTURE (oracle). Not part of the product: only tests/, the smoke
// check and bench.py's CPU-baseline leg load this code, and only as the checker.
//
// CPU restatement of the reference's StratRace model (include/environments/
// env_stratrace.h), costs (include/costs.cuh) and branch bookkeeping
// (include/state.h), templated on the scalar type R so that the same text gives
// the FP32 oracle (R = float, reference arithmetic) and the FP64 transcription
// (R = double). Expression order follows the reference line by line; each function
// cites the lines it restates.
#pragma once

#include <cmath>
#include <cstdint>
#include <vector>

#include "../../include/drmppi.h"
#include "philox_host.hpp"

namespace orc
{

using std::copysign;
using std::exp;
using std::fabs;
using std::floor;
using std::fmax;
using std::fmin;
using std::isfinite;
using std::isinf;
using std::log;
using std::pow;
using std::sqrt;

constexpr int DIM = 2;
constexpr int NTS = DR_N_TRACK_SAMPLES;
constexpr int WINDOW_SIZE = 10; // env_stratrace_defs.h:40
constexpr float DECAY = 0.97f;  // include/config.h:30
constexpr float MIN_COEFF_THRESHOLD = 0.01f; // include/config.h:29

enum Term
{
    TERM_NONE = 0,
    TERM_LOSE = 1,
    TERM_WIN = 2,
    TERM_OPP_WIN = 3
}; // include/config.h:78-84

template <typename R> inline R rsqrt_div(R x)
{
    return R(1) / sqrt(x);
}

// Environment parameters converted to R, plus the track grids padded with one
// wrap-around sample (index 512 == index 0) so that the reference's edge case
// idx0 == N_TRACK_SAMPLES (a wrap of s/L to exactly 1.0f) reads the wrapped value.
template <typename R> struct Env
{
    int nopp, nth;
    R dt, droneRadius, posNoise, speedNoise, actionNoiseLevel;
    R maxSpeed[DR_MAX_AGENTS], maxAccel[DR_MAX_AGENTS];
    R trackWidth;
    int nWinLaps;
    R kP, kV, maxOppLatDistFact, trackLength;
    R s1[DR_MAX_THETA][DR_MAX_OPP], s2[DR_MAX_THETA][DR_MAX_OPP], s3[DR_MAX_THETA][DR_MAX_OPP], speedScale[DR_MAX_THETA][DR_MAX_OPP],
        actionNoise[DR_MAX_THETA][DR_MAX_OPP];
    std::vector<R> p, t, kappa;

    explicit Env(const dr_env_config& c)
    {
        nopp = c.n_opp;
        nth = c.n_theta;
        dt = c.dt;
        droneRadius = c.drone_radius;
        posNoise = c.pos_noise_level;
        speedNoise = c.speed_noise_level;
        actionNoiseLevel = c.action_noise_level;
        for (int a = 0; a < DR_MAX_AGENTS; a++)
        {
            maxSpeed[a] = c.max_speed[a];
            maxAccel[a] = c.max_accel[a];
        }
        trackWidth = c.track_width;
        nWinLaps = c.n_win_laps;
        kP = c.kP;
        kV = c.kV;
        maxOppLatDistFact = c.max_opp_lat_dist_fact;
        trackLength = c.track_length;
        for (int th = 0; th < DR_MAX_THETA; th++)
            for (int o = 0; o < DR_MAX_OPP; o++)
            {
                s1[th][o] = c.opp_configs[th].s1[o];
                s2[th][o] = c.opp_configs[th].s2[o];
                s3[th][o] = c.opp_configs[th].s3[o];
                speedScale[th][o] = c.opp_configs[th].speed_scale[o];
                actionNoise[th][o] = c.opp_configs[th].action_noise[o];
            }
        p.resize((NTS + 1) * DIM);
        t.resize((NTS + 1) * DIM);
        kappa.resize(NTS + 1);
        for (int i = 0; i <= NTS; i++)
        {
            int k = i % NTS;
            for (int d = 0; d < DIM; d++)
            {
                p[i * DIM + d] = c.p_grid[k * DIM + d];
                t[i * DIM + d] = c.t_grid[k * DIM + d];
            }
            kappa[i] = c.kappa_grid[k];
        }
    }
};

template <typename R> struct State
{
    R pos[DR_MAX_AGENTS * DIM];
    R vel[DR_MAX_AGENTS * DIM];
    R S[DR_MAX_AGENTS];
    R lat[DR_MAX_AGENTS];
    int laps[DR_MAX_AGENTS];

    static State from(const dr_sim_state& s)
    {
        State r;
        for (int i = 0; i < DR_MAX_AGENTS * DIM; i++)
        {
            r.pos[i] = s.pos[i];
            r.vel[i] = s.vel[i];
        }
        for (int a = 0; a < DR_MAX_AGENTS; a++)
        {
            r.S[a] = s.S[a];
            r.lat[a] = s.lat_dist[a];
            r.laps[a] = s.laps[a];
        }
        return r;
    }
    void to(dr_sim_state& s) const
    {
        for (int i = 0; i < DR_MAX_AGENTS * DIM; i++)
        {
            s.pos[i] = (float)pos[i];
            s.vel[i] = (float)vel[i];
        }
        for (int a = 0; a < DR_MAX_AGENTS; a++)
        {
            s.S[a] = (float)S[a];
            s.lat_dist[a] = (float)lat[a];
            s.laps[a] = laps[a];
        }
    }
};

// BranchState for one parameter factor (include/config.h:86-92).
template <typename R> struct Branch
{
    R belief[DR_MAX_THETA];
    int predTheta;
    int branchingTime;
};

// ---- include/state.h -------------------------------------------------------------

// findConfident, state.h:93-115 (one factor: the marginal is the belief itself).
template <typename R> inline int findConfident(const R* belief, int nth, R threshold)
{
    for (int th = 0; th < nth; th++)
        if (belief[th] > threshold)
            return th + 1;
    return 0;
}

// initBranchState, state.h:154-163.
template <typename R> inline void initBranchState(Branch<R>& b, const R* initBelief, int nth, R threshold)
{
    for (int th = 0; th < nth; th++)
        b.belief[th] = initBelief[th];
    b.predTheta = findConfident(b.belief, nth, threshold);
    b.branchingTime = b.predTheta == 0 ? -1 : 0;
}

// localBranchTimeOrigin, state.h:166-174.
inline int localBranchTimeOrigin(int branch, int branchTime)
{
    int mx = 0;
    if (branch != 0 && branchTime > mx)
        mx = branchTime;
    return mx;
}

// branchCompatibleWithModel, state.h:178-185 (predTheta 0 = uncommitted).
inline bool branchCompatibleWithModel(int predTheta, int theta)
{
    return !(predTheta != 0 && predTheta != theta + 1);
}

// branchCompatibleWithInitialModel, state.h:189-196.
inline bool branchCompatibleWithInitialModel(int branch, int initPredTheta)
{
    return !(initPredTheta != 0 && initPredTheta != branch);
}

// sampleContributed, state.h:203-219.
inline bool sampleContributed(int branch, int tLocal, int sampleBranchTime, int samplePredTheta, int T)
{
    int tGlobal = tLocal + localBranchTimeOrigin(branch, sampleBranchTime);
    if (tGlobal >= T)
        return false;
    if ((branch != 0 && branch != samplePredTheta) || (branch == 0 && samplePredTheta != 0 && tGlobal >= sampleBranchTime))
        return false;
    return true;
}

// splineSampleContributed, state.h:222-228.
inline bool splineSampleContributed(int branch, int m, int sampleBranchTime, int samplePredTheta, int T, int M, const int* knots)
{
    return ((m > 0 && sampleContributed(branch, knots[m - 1], sampleBranchTime, samplePredTheta, T)) ||
            sampleContributed(branch, knots[m], sampleBranchTime, samplePredTheta, T) ||
            (m < M - 1 && sampleContributed(branch, knots[m + 1], sampleBranchTime, samplePredTheta, T)));
}

// ---- include/environments/env_stratrace.h ----------------------------------------

template <typename R> inline R sqNorm(R x, R y) // :33-36
{
    return x * x + y * y;
}

// sampleTrackArray<true>, :53-67
template <typename R> inline void sampleTrackArray2(const R* arr, R s, R* out, R L)
{
    s /= L;
    s = s - floor(s);
    R idx_f = s * NTS;
    int idx0 = (int)idx_f;
    int idx1 = (idx0 + 1) % NTS;
    R t = idx_f - idx0;
    for (int d = 0; d < DIM; d++)
        out[d] = (R(1) - t) * arr[idx0 * DIM + d] + t * arr[idx1 * DIM + d];
}

// sampleTrackArray<false>, :53-67
template <typename R> inline R sampleTrackArray1(const R* arr, R s, R L)
{
    s /= L;
    s = s - floor(s);
    R idx_f = s * NTS;
    int idx0 = (int)idx_f;
    int idx1 = (idx0 + 1) % NTS;
    R t = idx_f - idx0;
    return (R(1) - t) * arr[idx0] + t * arr[idx1];
}

// sampleNormalizedSpeed, :69-76
template <typename R> inline void sampleNormalizedSpeed(const R* t_grid, R s, R* out, R L)
{
    sampleTrackArray2(t_grid, s, out, L);
    R invNorm = R(1) / sqrt(sqNorm(out[0], out[1]));
    out[0] *= invNorm;
    out[1] *= invNorm;
}

// sqDistToSample, :79-85
template <typename R> inline R sqDistToSample(const R* p_grid, int i, const R* pos)
{
    R sq = R(0);
    for (int d = 0; d < DIM; d++)
        sq += (p_grid[i * DIM + d] - pos[d]) * (p_grid[i * DIM + d] - pos[d]);
    return sq;
}

// Operation counting only (opcount.cpp): with `local` set, the projections count the
// searches the CUDA kernels run where their certificate holds (the local search of the
// window from its centre; the gate race's walks without the margin scans) and take their
// result from the searches as written below, evaluated with counting paused by `pause`.
struct SearchCount
{
    bool local = false;
    void (*pause)(bool) = nullptr;
};
inline thread_local SearchCount g_searchCount;

// The kernels' local search of the window idxPrev -+ WINDOW_SIZE (windowLocalSearch in
// model.cuh): from the centre, to the neighbour at no greater (below) or smaller (above)
// distance while there is one; returns the sample it stops at.
template <typename R> inline int localWindowSearch(const Env<R>& env, int idxPrev, const R* pos)
{
    auto f = [&](int k) { return sqDistToSample(env.p.data(), (idxPrev + k - WINDOW_SIZE + NTS) % NTS, pos); };
    int c = WINDOW_SIZE;
    R fc = f(c), fl = f(c - 1);
    if (fl <= fc)
    {
        for (int it = 0; it < WINDOW_SIZE; it++)
        {
            c--;
            fc = fl;
            if (c == 0)
                break;
            fl = f(c - 1);
            if (!(fl <= fc))
                break;
        }
    }
    else
    {
        R fr = f(c + 1);
        for (int it = 0; it < WINDOW_SIZE && fr < fc; it++)
        {
            c++;
            fc = fr;
            if (c == 2 * WINDOW_SIZE)
                break;
            fr = f(c + 1);
        }
    }
    return (idxPrev + c - WINDOW_SIZE + NTS) % NTS;
}

// fastProjectOnTrack<false>, :88-162. Returns S, writes latDist.
template <typename R> inline R fastProjectOnTrack(const Env<R>& env, const R* pos, R prevS, R& latDist)
{
    prevS /= env.trackLength;
    prevS = prevS - floor(prevS);
    int idxPrev = (int)(prevS * NTS);
    if (g_searchCount.local)
    {
        localWindowSearch(env, idxPrev, pos);
        g_searchCount.pause(true);
    }

    int bestInd = (idxPrev - WINDOW_SIZE + NTS) % NTS;
    R bestSqDist = sqDistToSample(env.p.data(), bestInd, pos);

    for (int offset = NTS - WINDOW_SIZE + 1; offset <= NTS + WINDOW_SIZE; offset++)
    {
        R sqDist = sqDistToSample(env.p.data(), (idxPrev + offset) % NTS, pos);
        if (sqDist < bestSqDist)
        {
            bestSqDist = sqDist;
            bestInd = (idxPrev + offset) % NTS;
        }
    }
    if (g_searchCount.local)
        g_searchCount.pause(false);

    R bestSegSqDist = INFINITY;
    R bestS = R(0);
    R closestX = R(0), closestY = R(0);
    const R* P = env.p.data();
    for (int seg = -1; seg <= 0; ++seg)
    {
        int a = (bestInd + seg + NTS) % NTS;
        int b = (a + 1) % NTS;
        R abx = P[2 * b] - P[2 * a];
        R aby = P[2 * b + 1] - P[2 * a + 1];
        R sqAB = sqNorm(abx, aby);
        R t = R(0);
        if ((double)sqAB > 1e-12) // float compared with a double literal, as in the reference
        {
            t = ((pos[0] - P[2 * a]) * abx + (pos[1] - P[2 * a + 1]) * aby) / sqAB;
            t = fmax(R(0), fmin(t, R(1)));
        }
        R projx = P[2 * a] + t * abx;
        R projy = P[2 * a + 1] + t * aby;
        R sqDist = sqNorm(pos[0] - projx, pos[1] - projy);
        if (sqDist < bestSegSqDist)
        {
            bestSegSqDist = sqDist;
            bestS = ((R)a + t) / NTS * env.trackLength;
            closestX = projx;
            closestY = projy;
        }
    }
    R tang[2];
    sampleTrackArray2(env.t.data(), bestS, tang, env.trackLength);
    R cross = -tang[1] * (pos[0] - closestX) + tang[0] * (pos[1] - closestY);
    latDist = copysign(sqrt(bestSegSqDist), cross);
    return bestS;
}

// updateBelief, :166-222 (nomAction laid out [theta][opp][dim]).
template <typename R> inline void updateBelief(const Env<R>& env, R* belief, const R* oppAction, const R* nomAction)
{
    R sum = R(0);
    const R sigmaEnv = R(0.2);
    const R pi = sizeof(R) == 4 ? R(3.14159265358979323846f) : R(3.14159265358979323846);
    for (int th = 0; th < env.nth; th++)
    {
        R logLikelihood = R(0);
        for (int o = 0; o < env.nopp; o++)
        {
            const R* nom = &nomAction[(th * env.nopp + o) * DIM];
            const R* obs = &oppAction[o * DIM];
            R sqAccel = R(0);
            for (int d = 0; d < DIM; d++)
                sqAccel += nom[d] * nom[d];
            R scale = R(1);
            if (sqAccel > env.maxAccel[o + 1] * env.maxAccel[o + 1])
                scale = env.maxAccel[o + 1] / sqrt(sqAccel);
            R sqDist = R(0);
            for (int d = 0; d < DIM; d++)
            {
                R dx = obs[d] - nom[d] * scale;
                sqDist += dx * dx;
            }
            R an = env.actionNoise[th][o];
            R sqSigma = sigmaEnv * sigmaEnv + an * an;
            logLikelihood += R(-0.5) * sqDist / sqSigma - (R)DIM * R(0.5) * log(R(2) * pi) - (R)DIM * R(0.5) * log(sqSigma);
        }
        belief[th] *= exp(logLikelihood);
        sum += belief[th];
    }
    if (sum < R(1e-20))
    {
        R uniform = R(1) / env.nth;
        for (int th = 0; th < env.nth; ++th)
            belief[th] = uniform;
    }
    else
    {
        for (int th = 0; th < env.nth; th++)
            belief[th] /= sum;
    }
}

// trackBoundaryDist<loseOnOppWin>, :226-244
template <typename R> inline R trackBoundaryDist(const State<R>& s, const Env<R>& env, bool loseOnOppWin)
{
    if (loseOnOppWin)
        for (int o = 1; o <= env.nopp; o++)
            if (s.laps[o] >= env.nWinLaps)
                return R(-1);
    R minSq = INFINITY;
    for (int o = 1; o <= env.nopp; o++)
        minSq = fmin(minSq, sqNorm(s.pos[2 * o] - s.pos[0], s.pos[2 * o + 1] - s.pos[1]));
    return fmin(sqrt(minSq) - env.droneRadius, env.trackWidth - fabs(s.lat[0]));
}

template <typename R> inline bool isOutside(const State<R>& s, const Env<R>& env, R radius, bool loseOnOppWin) // :246-250
{
    return trackBoundaryDist(s, env, loseOnOppWin) < radius;
}

template <typename R> inline bool isWinner(const State<R>& s, const Env<R>& env) // :252-265
{
    if (s.laps[0] >= env.nWinLaps)
        return true;
    for (int o = 1; o <= env.nopp; o++)
        if (fabs(s.lat[o]) > env.trackWidth - env.droneRadius)
            return true;
    return false;
}

template <typename R> inline bool isOppWinner(const State<R>& s, const Env<R>& env) // :267-274
{
    for (int o = 1; o <= env.nopp; o++)
        if (s.laps[o] >= env.nWinLaps)
            return true;
    return false;
}

template <typename R> inline R getAnyAdvance(const State<R>& s, const Env<R>& env, int a) // :277-280
{
    return s.S[a] / env.trackLength + s.laps[a];
}

template <typename R> inline R getOppAdvance(const State<R>& s, const Env<R>& env) // :287-293
{
    R mx = -INFINITY;
    for (int o = 1; o <= env.nopp; o++)
        mx = fmax(mx, getAnyAdvance(s, env, o));
    return mx;
}

// computeSdot, :302-315
template <typename R> inline R computeSdot(int i, const State<R>& s, const Env<R>& env)
{
    R tang_i[2];
    sampleNormalizedSpeed(env.t.data(), s.S[i], tang_i, env.trackLength);
    R kappa_current = sampleTrackArray1(env.kappa.data(), s.S[i], env.trackLength);
    R metric = 1 - kappa_current * s.lat[i];
    if (fabs(metric) < R(1e-12))
        metric = copysign(R(1e-12), metric);
    return (tang_i[0] * s.vel[2 * i] + tang_i[1] * s.vel[2 * i + 1]) / metric;
}

// computeOppTargetLatDist, :318-461 (returns latDis, writes speedGoal)
template <typename R> inline R computeOppTargetLatDist(int iOpp, const State<R>& s, const Env<R>& env, int th, R& speedGoalOut)
{
    R L = env.trackLength;
    int iAhead = 0;
    R deltaSAhead = s.S[0] - s.S[iOpp];
    if (deltaSAhead < R(0))
        deltaSAhead += L;
    for (int j = 1; j <= env.nopp; j++)
        if (j != iOpp)
        {
            R deltaS = s.S[j] - s.S[iOpp];
            if (deltaS < R(0))
                deltaS += L;
            if (deltaS < deltaSAhead)
            {
                deltaSAhead = deltaS;
                iAhead = j;
            }
        }
    int iBehind = 0;
    R deltaSBehind = s.S[0] - s.S[iOpp];
    if (deltaSBehind > R(0))
        deltaSBehind -= L;
    for (int j = 1; j <= env.nopp; j++)
        if (j != iOpp)
        {
            R deltaS = s.S[j] - s.S[iOpp];
            if (deltaS > R(0))
                deltaS -= L;
            if (deltaS > deltaSBehind)
            {
                deltaSBehind = deltaS;
                iBehind = j;
            }
        }

    R latDis = R(0);
    R tang_i[2];
    sampleNormalizedSpeed(env.t.data(), s.S[iOpp], tang_i, L);
    R sdot_i = computeSdot(iOpp, s, env);
    R baseSpeed = env.speedScale[th][iOpp - 1] * env.maxSpeed[iOpp];
    R speedGoal = baseSpeed;
    const R s1 = env.s1[th][iOpp - 1], s2 = env.s2[th][iOpp - 1], s3 = env.s3[th][iOpp - 1];

    for (int k = 0; k <= 1; k++)
    {
        int j = k ? iAhead : iBehind;
        R deltaS = k ? deltaSAhead : deltaSBehind;
        R deltaE = s.lat[j] - s.lat[iOpp];
        R tang_j[2];
        sampleNormalizedSpeed(env.t.data(), s.S[j], tang_j, env.trackLength);
        R sdot_j = computeSdot(j, s, env);
        R blockTolerance = env.maxSpeed[j] * R(0.3);
        bool shouldBlock = (deltaS < R(0)) && (deltaS > -env.trackLength * R(0.25)) && (sdot_j + blockTolerance > sdot_i);
        bool shouldOvertake = (sdot_i > sdot_j) && (fabs(deltaE) < s1);
        R factor = exp(-s2 * deltaS * deltaS);
        if (shouldBlock)
        {
            R blockTerm = s.lat[j] * (1 - exp(-s3 * (sdot_j + blockTolerance - sdot_i))) * factor;
            latDis += blockTerm;
        }
        if (shouldOvertake)
        {
            R overtakeTerm = (s.lat[j] - copysign(s1, deltaE)) * factor;
            latDis += overtakeTerm;
            R oppLongSpeed = s.vel[2 * j] * tang_j[0] + s.vel[2 * j + 1] * tang_j[1];
            if (deltaS < 3 * env.droneRadius)
                speedGoal = fmin(speedGoal, R(0.7) * oppLongSpeed);
            else if (deltaS < 6 * env.droneRadius && (double)s1 > 1e-6) // double literal, as in the reference
            {
                R latFactor = fabs(deltaE) / s1;
                speedGoal = fmin(speedGoal, latFactor * oppLongSpeed + (R(1) - latFactor) * baseSpeed);
            }
        }
    }
    R maxLatDis = env.trackWidth - env.droneRadius * env.maxOppLatDistFact;
    latDis = fmax(-maxLatDis, fmin(maxLatDis, latDis));
    speedGoalOut = speedGoal;
    return latDis;
}

// computeOpponentAction ("second try"), :611-706
template <typename R> inline void computeOpponentAction(int iOpp, const State<R>& s, const Env<R>& env, R* out, int th)
{
    R L = env.trackLength;
    R maxAccel = env.maxAccel[iOpp];
    R dt = env.dt;
    R speedGoal;
    R latDisRaw = computeOppTargetLatDist(iOpp, s, env, th, speedGoal);

    R s_now = s.S[iOpp];
    R pos_i[2] = {s.pos[iOpp * 2], s.pos[iOpp * 2 + 1]};
    R vel_i[2] = {s.vel[iOpp * 2], s.vel[iOpp * 2 + 1]};
    R p_center[2], tang[2];
    sampleTrackArray2(env.p.data(), s_now, p_center, L);
    sampleNormalizedSpeed(env.t.data(), s_now, tang, L);
    R kappa = sampleTrackArray1(env.kappa.data(), s_now, L);

    R norm[2] = {-tang[1], tang[0]};
    R e_n = (pos_i[0] - p_center[0]) * norm[0] + (pos_i[1] - p_center[1]) * norm[1];
    R v_t = vel_i[0] * tang[0] + vel_i[1] * tang[1];
    R v_n = vel_i[0] * norm[0] + vel_i[1] * norm[1];

    R e_n_max = env.trackWidth - env.droneRadius * R(1.2);
    R metric_actual = R(1) - kappa * e_n;
    if (fabs(metric_actual) < R(1e-6))
        metric_actual = copysign(R(1e-6), metric_actual);
    R a_centripetal = v_t * v_t * kappa / metric_actual;
    R a_lat_max = fmax(maxAccel - fabs(a_centripetal), maxAccel * R(0.2));

    R latDis = fmax(-e_n_max, fmin(e_n_max, latDisRaw));
    R e_error = latDis - e_n;
    R dist_to_pos_wall = fmax(e_n_max - e_n, R(0.001));
    R dist_to_neg_wall = fmax(e_n_max + e_n, R(0.001));

    R a_n_cmd;
    if (v_n > R(0) && v_n * v_n > R(1.8) * a_lat_max * dist_to_pos_wall)
        a_n_cmd = -a_lat_max;
    else if (v_n < R(0) && v_n * v_n > R(1.8) * a_lat_max * dist_to_neg_wall)
        a_n_cmd = a_lat_max;
    else if (fabs(e_error) < R(0.02))
    {
        R kp = a_lat_max / R(0.02);
        a_n_cmd = kp * e_error - R(2) * sqrt(kp) * v_n;
        a_n_cmd = fmax(-a_lat_max, fmin(a_lat_max, a_n_cmd));
    }
    else
    {
        R stopping_dist = v_n * v_n / (R(2) * a_lat_max);
        bool v_toward = (e_error > R(0) && v_n > R(0)) || (e_error < R(0) && v_n < R(0));
        bool decel_phase = v_toward && stopping_dist >= fabs(e_error) * R(0.95);
        a_n_cmd = (e_error > R(0)) ? a_lat_max : -a_lat_max;
        if (decel_phase)
            a_n_cmd = -a_n_cmd;
        R v_n_next = v_n + a_n_cmd * dt;
        if (v_n_next > R(0))
        {
            R v_safe = sqrt(R(2) * a_lat_max * dist_to_pos_wall);
            if (v_n_next > v_safe)
                a_n_cmd = (v_safe - v_n) / dt;
        }
        else
        {
            R v_safe = sqrt(R(2) * a_lat_max * dist_to_neg_wall);
            if (-v_n_next > v_safe)
                a_n_cmd = (-v_safe - v_n) / dt;
        }
    }
    R a_n_total = fmax(-maxAccel, fmin(maxAccel, a_n_cmd + a_centripetal));
    R a_t_max = sqrt(fmax(maxAccel * maxAccel - a_n_total * a_n_total, R(0)));
    R kappa_eff = kappa / (R(1) - kappa * latDis + R(1e-6));
    R pathSpeed = fmin(speedGoal, sqrt(maxAccel / fmax(fabs(kappa_eff), R(1e-12))));
    if (fabs(a_n_cmd) > a_lat_max * R(0.5))
        pathSpeed *= fmax(R(0.4), R(1.5) - fabs(a_n_cmd) / a_lat_max);
    R a_t_cmd = env.kV * (pathSpeed - v_t) - v_n * kappa * v_t / metric_actual;
    a_t_cmd = fmax(-a_t_max, fmin(a_t_max, a_t_cmd));
    out[0] = a_t_cmd * tang[0] + a_n_total * norm[0];
    out[1] = a_t_cmd * tang[1] + a_n_total * norm[1];
}

struct StepFlags
{
    bool updateBelief;
    bool considerBranching;
    bool loseOnOppWin;
    bool applyNoise;
    bool allThetaOppActions; // compute the nominal opponent action for every theta (reference), or only the true one
    // operation counting only: with considerBranching, skip the belief update and the other
    // hypotheses' actions once the sample has committed (nothing reads that belief any more)
    bool skipDeadBelief = false;
};

// environmentStep, :711-894. The noise source is any object with next().
template <typename R, typename RNG>
inline int environmentStep(int t, int trueTheta, const Env<R>& env, const R* egoAction, const StepFlags& f, State<R>& s, Branch<R>& bs,
                           bool& branched, R minConfidence, RNG& rng)
{
    const int NA = env.nopp + 1;
    R prevS[DR_MAX_AGENTS];
    for (int a = 0; a < NA; a++)
        prevS[a] = s.S[a];

    R actions[DR_MAX_AGENTS * DIM];
    R nomOpp[DR_MAX_THETA * DR_MAX_OPP * DIM];
    for (int d = 0; d < DIM; d++)
        actions[d] = egoAction[d];
    const bool dead = f.skipDeadBelief && f.considerBranching && bs.predTheta != 0;
    for (int o = 1; o <= env.nopp; o++)
    {
        for (int th = 0; th < env.nth; th++)
            if ((f.allThetaOppActions && !dead) || th == trueTheta)
                computeOpponentAction(o, s, env, &nomOpp[(th * env.nopp + o - 1) * DIM], th);
        for (int d = 0; d < DIM; d++)
        {
            R u = nomOpp[(trueTheta * env.nopp + o - 1) * DIM + d];
            R an = env.actionNoise[trueTheta][o - 1];
            if (f.applyNoise && an != R(0))
                u += an * (R)rng.next();
            actions[o * DIM + d] = u;
        }
    }
    for (int a = 0; a < NA; a++)
    {
        R sq = R(0);
        for (int d = 0; d < DIM; d++)
            sq += actions[a * DIM + d] * actions[a * DIM + d];
        R factor = R(1);
        R maxSq = env.maxAccel[a] * env.maxAccel[a];
        if (sq > maxSq)
            factor = env.maxAccel[a] / sqrt(sq);
        for (int d = 0; d < DIM; d++)
        {
            R& v = actions[a * DIM + d];
            v *= factor;
            if (env.actionNoiseLevel != R(0) && f.applyNoise)
                v += (R)rng.next() * env.actionNoiseLevel;
        }
    }
    for (int a = 0; a < NA; a++)
        for (int d = 0; d < DIM; d++)
            s.pos[a * DIM + d] += env.dt * s.vel[a * DIM + d];
    for (int a = 0; a < NA; a++)
    {
        R sdot = computeSdot(a, s, env);
        s.S[a] += env.dt * sdot;
    }
    for (int a = 0; a < NA; a++)
        for (int d = 0; d < DIM; d++)
            s.vel[a * DIM + d] += env.dt * actions[a * DIM + d];
    for (int a = 0; a < NA; a++)
    {
        R sqSpd = sqNorm(s.vel[2 * a], s.vel[2 * a + 1]);
        if (sqSpd > env.maxSpeed[a] * env.maxSpeed[a])
        {
            R sc = env.maxSpeed[a] / sqrt(sqSpd);
            for (int d = 0; d < DIM; d++)
                s.vel[a * DIM + d] *= sc;
        }
    }
    if ((env.posNoise != R(0) || env.speedNoise != R(0)) && f.applyNoise)
    {
        for (int a = 0; a < NA; a++)
            for (int d = 0; d < DIM; d++)
            {
                if (env.posNoise != R(0))
                    s.pos[a * DIM + d] += (R)rng.next() * env.posNoise;
                if (env.speedNoise != R(0))
                    s.vel[a * DIM + d] += (R)rng.next() * env.speedNoise;
            }
    }
    for (int a = 0; a < NA; a++)
        s.S[a] = fastProjectOnTrack(env, s.pos + a * DIM, s.S[a], s.lat[a]);
    for (int a = 0; a < NA; a++)
    {
        if (s.S[a] < prevS[a] - env.trackLength * R(0.5))
            s.laps[a]++;
        if (s.S[a] > prevS[a] + env.trackLength * R(0.5))
            s.laps[a]--;
    }
    if (f.updateBelief && !dead)
        updateBelief(env, bs.belief, actions + DIM, nomOpp);
    if (f.considerBranching)
    {
        int np = findConfident(bs.belief, env.nth, minConfidence);
        if (bs.predTheta == 0 && np != 0)
        {
            bs.predTheta = np;
            bs.branchingTime = t + 1;
            branched = true;
        }
    }
    if (isOutside(s, env, env.droneRadius, f.loseOnOppWin))
        return TERM_LOSE;
    if (isWinner(s, env))
        return TERM_WIN;
    if (!f.loseOnOppWin)
        if (isOutside(s, env, env.droneRadius, true))
            return TERM_OPP_WIN;
    return TERM_NONE;
}

// ---- include/costs.cuh -----------------------------------------------------------

template <typename R> struct MppiCosts
{
    R collDistFactor, boundaryCost, boundaryThresholdFactor, outsideCost, winCost, oppWinCost, finalAdvWeight, finalOppAdvWeight;
};

template <typename R> struct PrCosts
{
    R collDistFactor, boundaryCost, boundaryThresholdFactor, winCost, oppWinCost, finalAdvWeight, finalOppAdvWeight, safetyWeight;
};

template <typename R> inline R powi2(R x)
{
    return pow(x, R(2));
}

// stateCost, costs.cuh:7-28
template <typename R> inline R stateCost(const State<R>& s, const Env<R>& env, const MppiCosts<R>& mc)
{
    R cost = R(0);
    R bd = trackBoundaryDist(s, env, false);
    R danger = mc.boundaryThresholdFactor * env.droneRadius;
    if (bd < danger)
        cost += mc.boundaryCost * powi2(bd / env.droneRadius);
    if (bd < env.droneRadius * mc.collDistFactor)
        cost += mc.outsideCost;
    if (isOppWinner(s, env))
        cost += mc.oppWinCost;
    if (isWinner(s, env))
        cost -= mc.winCost;
    return cost;
}

// finalCost, costs.cuh:31-39
template <typename R> inline R finalCost(const State<R>& s, const Env<R>& env, R finalAdvWeight, R finalOppAdvWeight)
{
    R cost = -finalAdvWeight * getAnyAdvance(s, env, 0);
    if (finalOppAdvWeight != R(0))
        cost += finalOppAdvWeight * getOppAdvance(s, env);
    return cost;
}

// PRMPPIstateCost, costs.cuh:44-63
template <typename R> inline R prStateCost(const State<R>& s, const Env<R>& env, const PrCosts<R>& mc)
{
    R cost = R(0);
    R bd = trackBoundaryDist(s, env, true);
    R danger = mc.boundaryThresholdFactor * env.droneRadius;
    if (bd < danger)
        cost += mc.boundaryCost * powi2(bd / env.droneRadius);
    if (isWinner(s, env))
        cost -= mc.winCost;
    if (isOppWinner(s, env))
        cost += mc.oppWinCost;
    return cost;
}

// PRMPPIsafetyCost, costs.cuh:78-86
template <typename R> inline R prSafetyCost(const State<R>& s, const Env<R>& env, const PrCosts<R>& mc)
{
    return env.droneRadius * mc.collDistFactor - trackBoundaryDist(s, env, false);
}

} // namespace orc
