// TEST INFRASTRUCTURE (oracle). Not part of the product: only tests/, the smoke
// check and bench.py's CPU-baseline leg load this code, and only as the checker.
//
// CPU restatement of the reference's gate-race model, EnvDroneRace
// (include/environments/env_dronerace.h) with the costs of include/costs.cuh,
// templated on the scalar type R like model.hpp (R = float: the reference's
// arithmetic; R = double: the transcription). Expression order follows the
// reference line by line; each function cites the lines it restates. The functions
// share their names with the strategic-race ones in model.hpp and are found by
// argument-dependent lookup on gate::Env / gate::State, so that the rollout and
// verification loops of port.cpp serve both models.
#pragma once

#include <cfloat>
#include <cmath>
#include <cstdint>
#include <vector>

#include "model.hpp"

namespace orc
{
namespace gate
{

constexpr int NA = DR_GATE_AGENTS;    // env_dronerace_defs.h:8
constexpr int NR = DR_GATE_RACELINES; // env_dronerace_defs.h:17

template <typename R> struct Pid
{
    R kp, kd, repulsionFactor, repulsionPower, repulsionDistFact;
    int raceline;
    R actionNoise;
};

// EnvironmentConfig (env_dronerace_defs.h:60-93). The racelines are stored one after the
// other with one extra sample at the end (the first sample of the last raceline): the
// reference's sampleCenterline reads sample 512 when s wraps to exactly 1.0f, which for
// raceline r < NR-1 is the next raceline's first sample and for the last one lies past
// the reference's buffer.
template <typename R> struct Env
{
    int nth, nGates, nObs, nRound, iMppi, nWinLaps;
    R arenaMin[DIM], arenaMax[DIM];
    R dt, droneRadius, posNoise, speedNoise, actionNoiseLevel;
    R maxSpeed[NA], maxAccel[NA];
    R targetDistance;
    R gateCenters[DR_GATE_MAX_GATES * DIM], gateVectors[DR_GATE_MAX_GATES * DIM], gateRadius[DR_GATE_MAX_GATES];
    R obstacles[DR_GATE_MAX_OBSTACLES * DIM * 2], roundCenters[DR_GATE_MAX_OBSTACLES * DIM], roundRadius[DR_GATE_MAX_OBSTACLES];
    Pid<R> pid[DR_MAX_THETA];
    std::vector<R> track;

    explicit Env(const dr_gate_env_config& c)
    {
        nth = c.n_theta;
        nGates = c.n_gates;
        nObs = c.n_obstacles;
        nRound = c.n_round_obstacles;
        iMppi = c.i_mppi;
        nWinLaps = c.n_win_laps;
        for (int d = 0; d < DIM; d++)
        {
            arenaMin[d] = c.arena_min[d];
            arenaMax[d] = c.arena_max[d];
        }
        dt = c.dt;
        droneRadius = c.drone_radius;
        posNoise = c.pos_noise_level;
        speedNoise = c.speed_noise_level;
        actionNoiseLevel = c.action_noise_level;
        for (int a = 0; a < NA; a++)
        {
            maxSpeed[a] = c.max_speed[a];
            maxAccel[a] = c.max_accel[a];
        }
        targetDistance = c.target_distance;
        for (int i = 0; i < DR_GATE_MAX_GATES * DIM; i++)
        {
            gateCenters[i] = c.gate_centers[i];
            gateVectors[i] = c.gate_vectors[i];
        }
        for (int i = 0; i < DR_GATE_MAX_GATES; i++)
            gateRadius[i] = c.gate_radius[i];
        for (int i = 0; i < DR_GATE_MAX_OBSTACLES * DIM * 2; i++)
            obstacles[i] = c.obstacles[i];
        for (int i = 0; i < DR_GATE_MAX_OBSTACLES * DIM; i++)
            roundCenters[i] = c.round_obs_centers[i];
        for (int i = 0; i < DR_GATE_MAX_OBSTACLES; i++)
            roundRadius[i] = c.round_obs_radius[i];
        for (int th = 0; th < DR_MAX_THETA; th++)
        {
            const dr_pid_config& p = c.opp_pid[th];
            pid[th] = Pid<R>{p.kp, p.kd, p.repulsion_factor, p.repulsion_power, p.repulsion_dist_fact, p.raceline_index, p.action_noise};
        }
        track.resize((size_t)NR * NTS * DIM + DIM);
        for (size_t i = 0; i < (size_t)NR * NTS * DIM; i++)
            track[i] = c.track_points[i];
        for (int d = 0; d < DIM; d++)
            track[(size_t)NR * NTS * DIM + d] = c.track_points[(size_t)(NR - 1) * NTS * DIM + d];
    }
    const R* raceline(int r) const
    {
        return track.data() + (size_t)r * NTS * DIM;
    }
};

// SimState (env_dronerace_defs.h:95-103).
template <typename R> struct State
{
    R pos[NA * DIM];
    R vel[NA * DIM];
    R S[NA * NR];
    int laps[NA];
    int gates[NA];

    static State from(const dr_gate_state& s)
    {
        State r;
        for (int i = 0; i < NA * DIM; i++)
        {
            r.pos[i] = s.pos[i];
            r.vel[i] = s.vel[i];
        }
        for (int i = 0; i < NA * NR; i++)
            r.S[i] = s.S[i];
        for (int a = 0; a < NA; a++)
        {
            r.laps[a] = s.laps[a];
            r.gates[a] = s.gates[a];
        }
        return r;
    }
    void to(dr_gate_state& s) const
    {
        for (int i = 0; i < NA * DIM; i++)
        {
            s.pos[i] = (float)pos[i];
            s.vel[i] = (float)vel[i];
        }
        for (int i = 0; i < NA * NR; i++)
            s.S[i] = (float)S[i];
        for (int a = 0; a < NA; a++)
        {
            s.laps[a] = laps[a];
            s.gates[a] = gates[a];
        }
    }
};

struct Flags
{
    bool updateBelief;
    bool considerBranching;
    bool addMargin;
    bool loseOnOppWin;
    bool applyNoise;
    float gateMargin;
    // operation counting only: with considerBranching, skip the belief update and the other
    // hypotheses' PID actions once the sample has committed (nothing reads that belief)
    bool skipDeadBelief = false;
};

// agentSpeed, env_dronerace.h:43-52
template <typename R> inline R agentSpeed(const R* vel, int a)
{
    R s = R(0);
    for (int d = 0; d < DIM; d++)
    {
        R v = vel[a * DIM + d];
        s += v * v;
    }
    return sqrt(s);
}

// sampleCenterline, :55-64
template <typename R> inline void sampleCenterline(const R* tp, R s, R* out)
{
    s = s - floor(s);
    R idx_f = s * (R)NTS;
    int idx0 = (int)idx_f;
    int idx1 = (idx0 + 1) % NTS;
    R t = idx_f - (R)idx0;
    for (int d = 0; d < DIM; d++)
        out[d] = (R(1) - t) * tp[idx0 * DIM + d] + t * tp[idx1 * DIM + d];
}

// projectOnTrack (full scan), :69-93
template <typename R> inline R projectFull(const R* tp, const R* pos)
{
    R bestS = R(0);
    R bestD2 = (R)FLT_MAX;
    const R sStep = R(1) / (R)NTS;
    for (int i = 0; i < NTS; i++)
    {
        R d2 = R(0);
        for (int d = 0; d < DIM; d++)
        {
            R dx = tp[i * DIM + d] - pos[d];
            d2 += dx * dx;
        }
        if (d2 < bestD2)
        {
            bestD2 = d2;
            bestS = (R)i * sStep;
        }
    }
    return bestS;
}

// sqDistToSample, :96-102
template <typename R> inline R sqDistToSample(const R* tp, int i, const R* pos)
{
    R sq = R(0);
    for (int d = 0; d < DIM; d++)
        sq += (tp[i * DIM + d] - pos[d]) * (tp[i * DIM + d] - pos[d]);
    return sq;
}

// findMinAlongDirection, :105-140: walk while the distance decreases, then 10 more
// samples (the first of them the one that stopped the walk)
template <typename R> inline int walkMin(const R* tp, int i0, const R* pos, int delta, R baseSq, R& bestSq)
{
    const int margin = 10;
    int bestI = i0;
    bestSq = baseSq;
    int cur = (i0 + delta + NTS) % NTS;
    R curSq = gate::sqDistToSample(tp, cur, pos);
    while (curSq < bestSq)
    {
        bestI = cur;
        bestSq = curSq;
        cur = (cur + delta + NTS) % NTS;
        curSq = gate::sqDistToSample(tp, cur, pos);
    }
    for (int i = 0; i < margin; i++)
    {
        curSq = gate::sqDistToSample(tp, cur, pos);
        if (curSq < bestSq)
        {
            bestI = cur;
            bestSq = curSq;
        }
        cur = (cur + delta + NTS) % NTS;
    }
    return bestI;
}

// fastProjectOnTrack, :143-209 (the distance output is unused on the path)
template <typename R> inline R projectGreedy(const R* tp, const R* pos, R prevS)
{
    if (prevS < R(0))
        return projectFull(tp, pos);
    int baseI = (int)(prevS * (R)NTS + R(0.5)) % NTS;
    R baseSq = gate::sqDistToSample(tp, baseI, pos);
    if (g_searchCount.local)
    {
        // counting only: the kernels' walks (walkStop in gate_model.cuh); their margin
        // scans are skipped where the walks advanced at most 10 samples together
        int moves = 0;
        for (int delta = -1; delta <= 1; delta += 2)
        {
            R best = baseSq;
            int cur = (baseI + delta + NTS) % NTS;
            R curSq = gate::sqDistToSample(tp, cur, pos);
            while (curSq < best)
            {
                best = curSq;
                moves++;
                cur = (cur + delta + NTS) % NTS;
                curSq = gate::sqDistToSample(tp, cur, pos);
            }
        }
        g_searchCount.pause(moves <= 10);
    }
    R bSq, fSq;
    int bI = walkMin(tp, baseI, pos, -1, baseSq, bSq);
    int fI = walkMin(tp, baseI, pos, +1, baseSq, fSq);
    if (g_searchCount.local)
        g_searchCount.pause(false);
    if (fSq < bSq)
        return (R)fI / (R)NTS;
    return (R)bI / (R)NTS;
}

// updateBelief, :212-258
template <typename R> inline void updateBelief(const Env<R>& env, R* belief, const R* oppAction, const R* nomAction, R maxPidAccel)
{
    R sum = R(0);
    const R sigmaEnv = R(0.2f);
    for (int th = 0; th < env.nth; th++)
    {
        R sqAccel = R(0);
        for (int d = 0; d < DIM; d++)
            sqAccel += nomAction[th * DIM + d] * nomAction[th * DIM + d];
        R scale = R(1);
        if (sqAccel > maxPidAccel * maxPidAccel)
            scale = maxPidAccel / sqrt(sqAccel);
        R sqDist = R(0);
        for (int d = 0; d < DIM; d++)
        {
            R dx = oppAction[d] - nomAction[th * DIM + d] * scale;
            sqDist += dx * dx;
        }
        R an = env.pid[th].actionNoise;
        R sigma = sqrt(sigmaEnv * sigmaEnv + an * an);
        belief[th] *= exp(R(-0.5f) * sqDist / (sigma * sigma)) / (pow(R(2.0f) * (R)M_PIf32, (R)DIM / R(2)) * pow(sigma, (R)DIM));
        sum += belief[th];
    }
    if (sum < R(1e-20f))
    {
        R uniform = R(1) / (R)env.nth;
        for (int th = 0; th < env.nth; th++)
            belief[th] = uniform;
    }
    else
        for (int th = 0; th < env.nth; th++)
            belief[th] /= sum;
}

// trackBoundaryDist, :262-307
template <typename R> inline R trackBoundaryDist(const State<R>& s, const Env<R>& env, bool loseOnOppWin)
{
    if (loseOnOppWin && s.laps[1 - env.iMppi] >= env.nWinLaps)
        return R(-1);
    const R* cur = s.pos + env.iMppi * DIM;
    R minDist = (R)INFINITY;
    for (int d = 0; d < DIM; d++)
        minDist = fmin(minDist, fmin(cur[d] - env.arenaMin[d], env.arenaMax[d] - cur[d]));
    for (int i = 0; i < env.nObs; i++)
    {
        R sq = R(0);
        for (int d = 0; d < DIM; d++)
        {
            R dist = fmax(R(0), fmax(env.obstacles[i * 2 * DIM + d] - cur[d], cur[d] - env.obstacles[(i * 2 + 1) * DIM + d]));
            sq += dist * dist;
        }
        minDist = fmin(minDist, sqrt(sq));
    }
    for (int i = 0; i < env.nRound; i++)
    {
        R sq = R(0);
        for (int d = 0; d < DIM; d++)
        {
            R dx = cur[d] - env.roundCenters[i * DIM + d];
            sq += dx * dx;
        }
        minDist = fmin(minDist, sqrt(sq) - env.roundRadius[i]);
    }
    R sq = R(0);
    for (int d = 0; d < DIM; d++)
    {
        R dx = s.pos[d] - s.pos[d + DIM];
        sq += dx * dx;
    }
    minDist = fmin(minDist, sqrt(sq) - env.droneRadius);
    return minDist;
}

template <typename R> inline bool isOutside(const State<R>& s, const Env<R>& env, R radius, bool loseOnOppWin) // :310-314
{
    return trackBoundaryDist(s, env, loseOnOppWin) < radius;
}

// isWinner, :316-360 (the upper arena test adds the radius, as the reference does)
template <typename R> inline bool isWinner(const State<R>& s, const Env<R>& env)
{
    if (s.laps[env.iMppi] >= env.nWinLaps)
        return true;
    const R* cur = s.pos + (1 - env.iMppi) * DIM;
    const R radius = env.droneRadius;
    for (int d = 0; d < DIM; d++)
        if (cur[d] < env.arenaMin[d] + radius || cur[d] > env.arenaMax[d] + radius)
            return true;
    for (int i = 0; i < env.nObs; i++)
    {
        R sq = R(0);
        for (int d = 0; d < DIM; d++)
        {
            R dist = fmax(R(0), fmax(env.obstacles[i * 2 * DIM + d] - cur[d], cur[d] - env.obstacles[(i * 2 + 1) * DIM + d]));
            sq += dist * dist;
        }
        if (sq < radius * radius)
            return true;
    }
    for (int i = 0; i < env.nRound; i++)
    {
        R sq = R(0);
        for (int d = 0; d < DIM; d++)
        {
            R dx = cur[d] - env.roundCenters[i * DIM + d];
            sq += dx * dx;
        }
        if (sq < (radius + env.roundRadius[i]) * (radius + env.roundRadius[i]))
            return true;
    }
    return false;
}

template <typename R> inline bool isOppWinner(const State<R>& s, const Env<R>& env) // :362-370
{
    for (int a = 0; a < NA; a++)
        if (a != env.iMppi && s.laps[a] >= env.nWinLaps)
            return true;
    return false;
}

// getAnyAdvance, :374-394
template <typename R> inline R getAnyAdvance(const State<R>& s, const Env<R>& env, int a)
{
    R sqGate = R(0), sqCons = R(0);
    int next = (s.gates[a] + 1) % env.nGates;
    const R scale = R(0.8f);
    const R* prevC = env.gateCenters + s.gates[a] * DIM;
    const R* nextC = env.gateCenters + next * DIM;
    const R* pos = s.pos + a * DIM;
    for (int d = 0; d < DIM; d++)
    {
        sqGate += (nextC[d] - pos[d]) * (nextC[d] - pos[d]);
        sqCons += (nextC[d] - prevC[d]) * (nextC[d] - prevC[d]);
    }
    return (R)(s.gates[a] + env.nGates * s.laps[a]) + scale * (R(1) - sqrt(sqGate / sqCons));
}

// updateGates, :412-470
template <typename R> inline void updateGates(const Env<R>& env, State<R>& s, const R* prevPos, bool addMargin, R margin)
{
    for (int a = 0; a < NA; a++)
    {
        if (s.S[a * NR] >= R(0))
            for (int r = 0; r < NR; r++)
                s.S[a * NR + r] = projectGreedy(env.raceline(r), s.pos + a * DIM, s.S[a * NR + r]);
        int next = (s.gates[a] + 1) % env.nGates;
        R num = R(0), den = R(0);
        for (int d = 0; d < DIM; d++)
        {
            num += env.gateVectors[next * DIM + d] * (env.gateCenters[next * DIM + d] - prevPos[a * DIM + d]);
            den += env.gateVectors[next * DIM + d] * (s.pos[a * DIM + d] - prevPos[a * DIM + d]);
        }
        if (fabs(den) < R(1e-10f))
            continue;
        R lambda = num / den;
        if (lambda < R(0) || lambda > R(1))
            continue;
        R sq = R(0);
        for (int d = 0; d < DIM; d++)
        {
            R dx = (R(1) - lambda) * prevPos[a * DIM + d] + lambda * s.pos[a * DIM + d] - env.gateCenters[next * DIM + d];
            sq += dx * dx;
        }
        R rad = env.gateRadius[next] * env.gateRadius[next];
        if (addMargin)
            rad *= margin * margin;
        if (sq <= rad)
        {
            s.gates[a]++;
            if (s.gates[a] == env.nGates)
            {
                s.gates[a] = 0;
                s.laps[a]++;
            }
        }
    }
}

// computePIDAction, :473-541
template <typename R> inline void pidAction(int agent, const State<R>& s, const Env<R>& env, const Pid<R>& pid, R* out)
{
    R target[DIM] = {};
    sampleCenterline(env.raceline(pid.raceline), s.S[agent * NR + pid.raceline] + env.targetDistance, target);
    const R* cur = s.pos + agent * DIM;
    const R* vel = s.vel + agent * DIM;
    R sqError = R(0);
    for (int d = 0; d < DIM; d++)
    {
        R e = target[d] - cur[d];
        sqError += e * e;
    }
    R invDist = R(1) / sqrt(sqError + R(1e-5f));
    R vPar = R(0);
    for (int d = 0; d < DIM; d++)
    {
        R dir = (target[d] - cur[d]) * invDist;
        vPar += vel[d] * dir;
    }
    for (int d = 0; d < DIM; d++)
    {
        R error = (target[d] - cur[d]) * invDist;
        R latVelError = vel[d] - vPar * error;
        out[d] = pid.kp * error + pid.kd * (-latVelError);
    }
    if (pid.repulsionFactor != R(0))
        for (int other = 0; other < NA; other++)
        {
            if (other == agent)
                continue;
            R diff[DIM];
            R dist2 = R(0);
            for (int d = 0; d < DIM; d++)
            {
                diff[d] = s.pos[other * DIM + d] - cur[d];
                dist2 += diff[d] * diff[d];
            }
            R dist = sqrt(dist2) + R(1e-8f);
            if (dist < pid.repulsionDistFact * env.droneRadius * R(2))
            {
                R scale = pid.repulsionFactor / pow(dist * R(0.5f) / env.droneRadius, pid.repulsionPower + R(1));
                for (int d = 0; d < DIM; d++)
                    out[d] -= scale * diff[d];
            }
        }
    R sqAccel = R(0);
    for (int d = 0; d < DIM; d++)
        sqAccel += out[d] * out[d];
    if (sqAccel > env.maxAccel[agent] * env.maxAccel[agent])
    {
        R fact = env.maxAccel[agent] / sqrt(sqAccel);
        for (int d = 0; d < DIM; d++)
            out[d] *= fact;
    }
}

// environmentStep, :546-680. The noise source is any object with next().
template <typename R, typename RNG>
inline int environmentStep(int t, int trueTheta, const Env<R>& env, const R* egoAction, const Flags& f, State<R>& s, Branch<R>& bs, bool& branched,
                           R minConfidence, RNG& rng)
{
    R prevPos[NA * DIM];
    for (int i = 0; i < NA * DIM; i++)
        prevPos[i] = s.pos[i];
    R actions[NA * DIM];
    R nomPid[DR_MAX_THETA * DIM];
    for (int a = 0; a < NA; a++)
    {
        if (a == env.iMppi)
            for (int d = 0; d < DIM; d++)
                actions[a * DIM + d] = egoAction[d];
        else
        {
            const bool dead = f.skipDeadBelief && f.considerBranching && bs.predTheta != 0;
            for (int th = 0; th < env.nth; th++)
                if (!dead || th == trueTheta)
                    pidAction(a, s, env, env.pid[th], nomPid + th * DIM);
            for (int d = 0; d < DIM; d++)
            {
                R u = nomPid[trueTheta * DIM + d];
                if (f.applyNoise && env.pid[trueTheta].actionNoise != R(0))
                    u += env.pid[trueTheta].actionNoise * (R)rng.next();
                actions[a * DIM + d] = u;
            }
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
        for (int d = 0; d < DIM; d++)
            s.vel[a * DIM + d] += env.dt * actions[a * DIM + d];
    for (int a = 0; a < NA; a++)
    {
        R spd = agentSpeed(s.vel, a);
        if (spd > env.maxSpeed[a])
        {
            R sc = env.maxSpeed[a] / spd;
            for (int d = 0; d < DIM; d++)
                s.vel[a * DIM + d] *= sc;
        }
    }
    if ((env.posNoise != R(0) || env.speedNoise != R(0)) && f.applyNoise)
        for (int a = 0; a < NA; a++)
            for (int d = 0; d < DIM; d++)
            {
                if (env.posNoise != R(0))
                    s.pos[a * DIM + d] += (R)rng.next() * env.posNoise;
                if (env.speedNoise != R(0))
                    s.vel[a * DIM + d] += (R)rng.next() * env.speedNoise;
            }
    updateGates(env, s, prevPos, f.addMargin, (R)f.gateMargin);
    const int opp = 1 - env.iMppi;
    if (f.updateBelief && !(f.skipDeadBelief && f.considerBranching && bs.predTheta != 0))
        updateBelief(env, bs.belief, actions + opp * DIM, nomPid, env.maxAccel[opp]);
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

// ---- include/costs.cuh on the gate race ---------------------------------------------

template <typename R> inline R stateCost(const State<R>& s, const Env<R>& env, const MppiCosts<R>& mc) // costs.cuh:7-28
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

template <typename R> inline R finalCost(const State<R>& s, const Env<R>& env, R finalAdvWeight, R finalOppAdvWeight) // costs.cuh:31-39
{
    R cost = -finalAdvWeight * getAnyAdvance(s, env, env.iMppi);
    if (finalOppAdvWeight != R(0))
        cost += finalOppAdvWeight * getAnyAdvance(s, env, 1 - env.iMppi);
    return cost;
}

} // namespace gate
} // namespace orc
