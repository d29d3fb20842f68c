// TEST INFRASTRUCTURE (oracle). Not part of the product.
//
// Glue around the reference implementation, compiled against the reference's own
// headers and kernels (include/, src/kernels.cu, src/prmppi_kernels.cu,
// src/mppi_controller.cu, src/prmppi_controller.cu) by oracle/Makefile into
// oracle/_ref/. Two faces:
//   refh_*  host loops over the reference's __host__ __device__ model functions
//           (environmentStep, stateCost, ... as src/engine.cpp uses them on the host):
//           the reference's CPU path, and the FP32 reference for the oracle port.
//           The bodies of the reference's __global__ kernels are restated as loops.
//   refc_*  launches of the reference's own CUDA kernels on injected inputs (GPU box
//           only), and timing of its getControl.
// Environment noise inside refh_* rollouts comes from the product's Philox streams
// (via an RNG type that environmentStep's sampleNormal(rng) finds by argument-
// dependent lookup); refc_* kernels draw it from curand, so parity runs set every
// environment noise level to zero there.
#include "config.h"
#include "controllers.h"
#include "costs.cuh"
#include "kernels.cuh"
#include "state.h"

#include <chrono>
#include <cstdio>
#include <cstring>
#include <fcntl.h>
#include <iostream>
#include <memory>
#include <unistd.h>
#include <vector>

#include "../../include/drmppi.h"
#include "../port/philox_host.hpp"

// The C-ABI environment and state the exported functions take: the strategic race's
// (dr_env_config / dr_sim_state), or the gate race's when the reference is compiled with
// USE_ENV_DRONERACE (dr_gate_env_config / dr_gate_state).
#ifdef USE_ENV_DRONERACE
typedef dr_gate_env_config CEnv;
typedef dr_gate_state CState;
#else
typedef dr_env_config CEnv;
typedef dr_sim_state CState;
#endif

// RNG whose normals come from the Philox environment-noise stream.
struct PhiloxRefRNG
{
    orc::EnvNoise* n;
};
__host__ inline float sampleNormal(PhiloxRefRNG& r)
{
    return r.n->next();
}

namespace
{

constexpr int NTS = Env::N_TRACK_SAMPLES;
constexpr int NBP = N_BRANCH_PLANS;
constexpr int NTH = N_TRUE_MODELS;
constexpr int DIMR = ACTION_DIM;

#ifdef USE_ENV_DRONERACE
struct HostGrids
{
    std::vector<float> track;
};

// EnvironmentConfig of the gate race (env_dronerace_defs.h:60-93) from the C-ABI struct;
// the counts the reference fixes at compile time must match.
bool toRefEnv(const CEnv& c, EnvironmentConfig& e, HostGrids& g)
{
    if (c.n_theta != NTH || c.n_gates != Env::N_GATES || c.n_obstacles != Env::N_OBSTACLES || c.n_round_obstacles != Env::N_ROUND_OBSTACLES)
        return false;
    for (int d = 0; d < 2; d++)
    {
        e.arenaMin[d] = c.arena_min[d];
        e.arenaMax[d] = c.arena_max[d];
    }
    e.dt = c.dt;
    e.sendStates = c.send_states != 0;
    e.droneRadius = c.drone_radius;
    e.posNoiseLevel = c.pos_noise_level;
    e.speedNoiseLevel = c.speed_noise_level;
    e.actionNoiseLevel = c.action_noise_level;
    for (int a = 0; a < Env::N_AGENTS; a++)
    {
        e.maxSpeed[a] = c.max_speed[a];
        e.maxAccel[a] = c.max_accel[a];
    }
    e.nWinLaps = c.n_win_laps;
    e.targetDistance = c.target_distance;
    for (int i = 0; i < Env::N_GATES * 2; i++)
    {
        e.gateCenters[i] = c.gate_centers[i];
        e.gateVectors[i] = c.gate_vectors[i];
    }
    for (int i = 0; i < Env::N_GATES; i++)
        e.gateRadius[i] = c.gate_radius[i];
    for (int i = 0; i < Env::N_OBSTACLES * 4; i++)
        e.obstacles[i] = c.obstacles[i];
    for (int i = 0; i < Env::N_ROUND_OBSTACLES * 2; i++)
        e.roundObsCenters[i] = c.round_obs_centers[i];
    for (int i = 0; i < Env::N_ROUND_OBSTACLES; i++)
        e.roundObsRadius[i] = c.round_obs_radius[i];
    for (int th = 0; th < NTH; th++)
    {
        e.initBelief[th] = c.init_belief[th];
        const dr_pid_config& p = c.opp_pid[th];
        e.oppPid[th].kp = p.kp;
        e.oppPid[th].kd = p.kd;
        e.oppPid[th].repulsionFactor = p.repulsion_factor;
        e.oppPid[th].repulsionPower = p.repulsion_power;
        e.oppPid[th].repulsionDistFact = p.repulsion_dist_fact;
        e.oppPid[th].racelineIndex = p.raceline_index;
        e.oppPid[th].actionNoise = p.action_noise;
    }
    e.iMppi = c.i_mppi;
    // the racelines plus one sample (the last raceline's first) read when s wraps to 1.0f
    const size_t n = (size_t)Env::N_RACELINES * NTS * 2;
    g.track.assign(c.track_points, c.track_points + n);
    g.track.push_back(c.track_points[(size_t)(Env::N_RACELINES - 1) * NTS * 2]);
    g.track.push_back(c.track_points[(size_t)(Env::N_RACELINES - 1) * NTS * 2 + 1]);
    e.trackPoints = g.track.data();
    return true;
}

SimState toRefState(const CState& s)
{
    SimState r;
    for (int i = 0; i < Env::N_AGENTS * 2; i++)
    {
        r.pos[i] = s.pos[i];
        r.vel[i] = s.vel[i];
    }
    for (int i = 0; i < Env::N_AGENTS * Env::N_RACELINES; i++)
        r.S[i] = s.S[i];
    for (int a = 0; a < Env::N_AGENTS; a++)
    {
        r.laps[a] = s.laps[a];
        r.gates[a] = s.gates[a];
    }
    return r;
}

void fromRefState(const SimState& r, CState& s)
{
    for (int i = 0; i < Env::N_AGENTS * 2; i++)
    {
        s.pos[i] = r.pos[i];
        s.vel[i] = r.vel[i];
    }
    for (int i = 0; i < Env::N_AGENTS * Env::N_RACELINES; i++)
        s.S[i] = r.S[i];
    for (int a = 0; a < Env::N_AGENTS; a++)
    {
        s.laps[a] = r.laps[a];
        s.gates[a] = r.gates[a];
    }
}

#else
struct HostGrids
{
    std::vector<float> p, dp, t, kappa;
};

// EnvironmentConfig (env_stratrace_defs.h:53-86) from the C-ABI struct. Grids are
// padded with one wrap-around sample (see oracle/port/model.hpp).
bool toRefEnv(const CEnv& c, EnvironmentConfig& e, HostGrids& g)
{
    if (c.n_opp != Env::N_OPP || c.n_theta != NTH)
        return false;
    for (int d = 0; d < 2; d++)
    {
        e.arenaMin[d] = c.arena_min[d];
        e.arenaMax[d] = c.arena_max[d];
    }
    e.dt = c.dt;
    e.sendStates = c.send_states != 0;
    e.droneRadius = c.drone_radius;
    e.posNoiseLevel = c.pos_noise_level;
    e.speedNoiseLevel = c.speed_noise_level;
    e.actionNoiseLevel = c.action_noise_level;
    for (int a = 0; a < Env::N_AGENTS; a++)
    {
        e.maxSpeed[a] = c.max_speed[a];
        e.maxAccel[a] = c.max_accel[a];
    }
    e.trackWidth = c.track_width;
    e.nWinLaps = c.n_win_laps;
    for (int th = 0; th < NTH; th++)
    {
        e.initBelief[th] = c.init_belief[th];
        for (int o = 0; o < Env::N_OPP; o++)
        {
            e.oppConfigs[th].s1[o] = c.opp_configs[th].s1[o];
            e.oppConfigs[th].s2[o] = c.opp_configs[th].s2[o];
            e.oppConfigs[th].s3[o] = c.opp_configs[th].s3[o];
            e.oppConfigs[th].speedScale[o] = c.opp_configs[th].speed_scale[o];
            e.oppConfigs[th].actionNoise[o] = c.opp_configs[th].action_noise[o];
        }
    }
    e.kP = c.kP;
    e.kV = c.kV;
    e.maxOppLatDistFact = c.max_opp_lat_dist_fact;
    e.trackLength = c.track_length;
    g.p.resize((NTS + 1) * 2);
    g.dp.resize((NTS + 1) * 2);
    g.t.resize((NTS + 1) * 2);
    g.kappa.resize(NTS + 1);
    for (int i = 0; i <= NTS; i++)
    {
        int k = i % NTS;
        for (int d = 0; d < 2; d++)
        {
            g.p[i * 2 + d] = c.p_grid[k * 2 + d];
            g.dp[i * 2 + d] = c.dp_grid[k * 2 + d];
            g.t[i * 2 + d] = c.t_grid[k * 2 + d];
        }
        g.kappa[i] = c.kappa_grid[k];
    }
    e.p_grid = g.p.data();
    e.dp_grid = g.dp.data();
    e.t_grid = g.t.data();
    e.kappa_grid = g.kappa.data();
    return true;
}

SimState toRefState(const CState& s)
{
    SimState r;
    for (int i = 0; i < Env::N_AGENTS * 2; i++)
    {
        r.pos[i] = s.pos[i];
        r.vel[i] = s.vel[i];
    }
    for (int a = 0; a < Env::N_AGENTS; a++)
    {
        r.S[a] = s.S[a];
        r.latDist[a] = s.lat_dist[a];
        r.laps[a] = s.laps[a];
    }
    return r;
}

void fromRefState(const SimState& r, CState& s)
{
    for (int i = 0; i < Env::N_AGENTS * 2; i++)
    {
        s.pos[i] = r.pos[i];
        s.vel[i] = r.vel[i];
    }
    for (int a = 0; a < Env::N_AGENTS; a++)
    {
        s.S[a] = r.S[a];
        s.lat_dist[a] = r.latDist[a];
        s.laps[a] = r.laps[a];
    }
}

#endif

MPPIConfig toRefMppi(const dr_mppi_config& c)
{
    MPPIConfig m;
    m.nSamples = c.n_samples;
    m.nTimesteps = c.n_timesteps;
    m.nKnots = USE_SPLINES ? c.n_knots : c.n_timesteps; // config.cpp:252-253
    for (int i = 0; i < MAX_N_KNOTS; i++)
        m.knots[i] = i < DR_MAX_KNOTS ? c.knots[i] : 0;
    m.invTemperature = c.inv_temperature;
    m.samplingNoise = c.sampling_noise;
    m.gateTraversalMargin = c.gate_traversal_margin;
    m.collDistFactor = c.coll_dist_factor;
    m.boundaryCost = c.boundary_cost;
    m.boundaryThresholdFactor = c.boundary_threshold_factor;
    m.outsideCost = c.outside_cost;
    m.winCost = c.win_cost;
    m.oppWinCost = c.opp_win_cost;
    m.finalAdvWeight = c.final_adv_weight;
    m.finalOppAdvWeight = c.final_opp_adv_weight;
    m.minConfidence = c.min_confidence;
    m.nVerifSamples = c.n_verif_samples;
    m.beta = c.beta;
    m.verifHorizon = c.verif_horizon;
    m.maxVerifEps = c.max_verif_eps;
    return m;
}

PRMPPIConfig toRefPr(const dr_prmppi_config& c)
{
    PRMPPIConfig m;
    m.nSamples = c.n_samples;
    m.nTimesteps = c.n_timesteps;
    m.invTemperature = c.inv_temperature;
    m.samplingNoise = c.sampling_noise;
    m.gateTraversalMargin = c.gate_traversal_margin;
    m.collDistFactor = c.coll_dist_factor;
    m.boundaryCost = c.boundary_cost;
    m.boundaryThresholdFactor = c.boundary_threshold_factor;
    m.winCost = c.win_cost;
    m.oppWinCost = c.opp_win_cost;
    m.finalAdvWeight = c.final_adv_weight;
    m.finalOppAdvWeight = c.final_opp_adv_weight;
    m.safetyWeight = c.safety_weight;
    m.minSafeDist = c.min_safe_dist;
    m.delta = c.delta;
    m.P = (float)c.P;
    return m;
}

int MK(const MPPIConfig& mc)
{
    return USE_SPLINES ? mc.nKnots : mc.nTimesteps;
}

// Body of fullRolloutKernel (src/kernels.cu:34-171) for one sample.
void rolloutSample(int s, const EnvironmentConfig& envConfig, const MPPIConfig& mc, const SimState& initState, const float* initBelief,
                   const float* nominal, const float* noise, const float* B, uint64_t seed, uint64_t step, double* costsTrue, int* branchUsed,
                   int* branchTime)
{
    SimState state;
    BranchState branchState;
    float egoAction[ACTION_DIM];
    ScratchEnvBuffer buffer;
    BranchState firstBranchState;
    initBranchState(firstBranchState, initBelief, mc.minConfidence);
    const int N = mc.nSamples;
    for (int theta = 0; theta < NTH; theta++)
    {
        costsTrue[theta * N + s] = INFINITY;
        branchUsed[theta * N + s] = firstBranchState.predTheta[0];
        branchTime[theta * N + s] = firstBranchState.branchingTime[0];
    }
    int trueTheta[N_MODEL_FACTORS];
    for (int trueThetaFlat = 0; trueThetaFlat < NTH; trueThetaFlat++)
    {
        unflattenTrueModelIndex(trueThetaFlat, trueTheta);
        if (!branchCompatibleWithModel(firstBranchState.predTheta.data(), trueTheta))
            continue;
        state = initState;
        branchState = firstBranchState;
        float cost = 0.0f;
        bool stop = false;
        float decay = 1.0f;
        int tOrigin = 0;
        orc::EnvNoise en(seed, (uint32_t)s, (uint32_t)trueThetaFlat << 16, step, orc::S_MPPI_ROLL_ENV);
        PhiloxRefRNG rng{&en};
        for (int t = 0; t < mc.nTimesteps && !stop; t++)
        {
            en.begin_step((uint32_t)t);
            int local_time = t - tOrigin;
            int flatBranch = flattenBranchIndex(branchState.predTheta.data());
            if (USE_SPLINES)
            {
                const float* B_row = B + local_time * mc.nKnots;
                for (int d = 0; d < ACTION_DIM; d++)
                {
                    float sum = 0.0f;
                    for (int m = 0; m < mc.nKnots; m++)
                    {
                        float nom = nominal[(flatBranch * mc.nKnots + m) * ACTION_DIM + d];
                        float noisef = noise[((size_t)(flatBranch * mc.nKnots + m) * mc.nSamples + s) * ACTION_DIM + d];
                        sum += B_row[m] * (nom + noisef);
                    }
                    egoAction[d] = sum;
                }
            }
            else
                for (int d = 0; d < ACTION_DIM; d++)
                {
                    float nom = nominal[(flatBranch * mc.nTimesteps + local_time) * ACTION_DIM + d];
                    float noisef = noise[((size_t)(flatBranch * mc.nTimesteps + local_time) * mc.nSamples + s) * ACTION_DIM + d];
                    egoAction[d] = nom + noisef;
                }
            bool branched = false;
            TerminalType term = environmentStep<true, true, false>(t, trueThetaFlat, envConfig, egoAction, true, state, branchState, branched,
                                                                   mc.minConfidence, buffer, rng, mc.gateTraversalMargin);
            if (branched)
                tOrigin = t + 1;
            stop = (term != TERM_NONE);
            cost += stateCost(state, t, envConfig, mc, trueThetaFlat) * decay;
            decay *= DECAY;
        }
        cost += finalCost(state, envConfig, mc, trueThetaFlat);
        costsTrue[trueThetaFlat * N + s] = cost;
        branchTime[trueThetaFlat * N + s] = branchState.branchingTime[0];
        branchUsed[trueThetaFlat * N + s] = branchState.predTheta[0];
    }
}

// Eligibility coefficient of kernels.cu:252-279 / 349-372.
float sampleCoeffRef(const MPPIConfig& mc, const float* belief, int branchPlan, int tLocal, int s, const int* branchUsed, const int* branchTime)
{
    int branchTuple[N_MODEL_FACTORS];
    int thetaTuple[N_MODEL_FACTORS];
    unflattenBranchIndex(branchPlan, branchTuple);
    const int N = mc.nSamples, T = mc.nTimesteps, M = mc.nKnots;
    float coeff = 0.0f;
    for (int trueTheta = 0; trueTheta < NTH; trueTheta++)
    {
        if (belief[trueTheta] <= 0.0f)
            continue;
        unflattenTrueModelIndex(trueTheta, thetaTuple);
        if (!branchCompatibleWithModel(branchTuple, thetaTuple))
            continue;
        const int* samplePredTheta = branchUsed + (trueTheta * N + s) * N_MODEL_FACTORS;
        const int* sampleBranchTime = branchTime + (trueTheta * N + s) * N_MODEL_FACTORS;
        if (USE_SPLINES)
        {
            if (splineSampleContributed(branchTuple, tLocal, sampleBranchTime, samplePredTheta, T, M, mc.knots.data()))
                coeff += belief[trueTheta];
        }
        else if (sampleContributed(branchTuple, tLocal, sampleBranchTime, samplePredTheta, T))
            coeff += belief[trueTheta];
    }
    return coeff;
}

struct DevBuf
{
    void* p = nullptr;
    DevBuf(size_t n)
    {
        if (cudaMalloc(&p, n ? n : 4) != cudaSuccess)
            p = nullptr;
    }
    ~DevBuf()
    {
        if (p)
            cudaFree(p);
    }
    template <typename T> T* as()
    {
        return (T*)p;
    }
};

#ifdef USE_ENV_DRONERACE
// Device copy of the racelines in an EnvironmentConfig.
struct DevEnv
{
    EnvironmentConfig e;
    DevBuf track;
    DevEnv(const EnvironmentConfig& host) : e(host), track(((size_t)Env::N_RACELINES * NTS + 1) * 2 * 4)
    {
        cudaMemcpy(track.p, host.trackPoints, ((size_t)Env::N_RACELINES * NTS + 1) * 2 * 4, cudaMemcpyHostToDevice);
        e.trackPoints = track.as<float>();
    }
};

#else
// Device copy of the (padded) track grids in an EnvironmentConfig.
struct DevEnv
{
    EnvironmentConfig e;
    DevBuf p, dp, t, k;
    DevEnv(const EnvironmentConfig& host)
        : e(host), p((NTS + 1) * 2 * 4), dp((NTS + 1) * 2 * 4), t((NTS + 1) * 2 * 4), k((NTS + 1) * 4)
    {
        cudaMemcpy(p.p, host.p_grid, (NTS + 1) * 2 * 4, cudaMemcpyHostToDevice);
        cudaMemcpy(dp.p, host.dp_grid, (NTS + 1) * 2 * 4, cudaMemcpyHostToDevice);
        cudaMemcpy(t.p, host.t_grid, (NTS + 1) * 2 * 4, cudaMemcpyHostToDevice);
        cudaMemcpy(k.p, host.kappa_grid, (NTS + 1) * 4, cudaMemcpyHostToDevice);
        e.p_grid = p.as<float>();
        e.dp_grid = dp.as<float>();
        e.t_grid = t.as<float>();
        e.kappa_grid = k.as<float>();
    }
};

#endif

int cudaStatus()
{
    cudaError_t err = cudaDeviceSynchronize();
    if (err == cudaSuccess)
        err = cudaGetLastError();
    if (err != cudaSuccess)
    {
        fprintf(stderr, "reference CUDA error: %s\n", cudaGetErrorString(err));
        return 3;
    }
    return 0;
}

// Silences std::cout / stdout of the reference controllers while in scope.
struct Quiet
{
    int saved = -1;
    Quiet()
    {
        fflush(stdout);
        std::cout.flush();
        saved = dup(1);
        int fd = open("/dev/null", O_WRONLY);
        dup2(fd, 1);
        close(fd);
    }
    ~Quiet()
    {
        fflush(stdout);
        std::cout.flush();
        dup2(saved, 1);
        close(saved);
    }
};

} // namespace

extern "C" {

int ref_n_theta()
{
    return NTH;
}
int ref_n_opp()
{
#ifdef USE_ENV_DRONERACE
    return Env::N_AGENTS - 1;
#else
    return Env::N_OPP;
#endif
}
int ref_use_splines()
{
    return USE_SPLINES ? 1 : 0;
}
void ref_sizes(int* out)
{
    out[0] = (int)sizeof(EnvironmentConfig);
    out[1] = (int)sizeof(SimState);
    out[2] = (int)sizeof(MPPIConfig);
    out[3] = (int)sizeof(PRMPPIConfig);
}

// ==== host face ==============================================================================

int refh_mppi_rollout(const CEnv* ec, const dr_mppi_config* c, const CState* s0, const float* belief, const float* nominal,
                      const float* noise, const float* B, uint64_t seed, uint64_t step, double* costsTrue, int* branchUsed, int* branchTime,
                      int nthreads)
{
    EnvironmentConfig env;
    HostGrids g;
    if (!toRefEnv(*ec, env, g))
        return 2;
    MPPIConfig mc = toRefMppi(*c);
    SimState init = toRefState(*s0);
    const int N = mc.nSamples;
#pragma omp parallel for schedule(dynamic, 16) num_threads(nthreads > 0 ? nthreads : 1)
    for (int s = 0; s < N; s++)
        rolloutSample(s, env, mc, init, belief, nominal, noise, B, seed, step, costsTrue, branchUsed, branchTime);
    return 0;
}

// aggregate (kernels.cu:175-217), masked min (221-301), weighted average (307-408,
// sums in 256-thread block order), interpolation (411-431), clamp (434-456).
int refh_mppi_update(const CEnv* ec, const dr_mppi_config* c, const float* belief, const double* costsTrueIn, const int* branchUsed,
                     const int* branchTime, const float* noise, const float* B, float* splineOrDense, float* denseOut, float* minCosts, float* nu,
                     float* costsOut, int nthreads)
{
    EnvironmentConfig env;
    HostGrids g;
    if (!toRefEnv(*ec, env, g))
        return 2;
    MPPIConfig mc = toRefMppi(*c);
    const int N = mc.nSamples, T = mc.nTimesteps, M = MK(mc);
    std::vector<float> costsTrue((size_t)NTH * N), costs((size_t)NBP * N);
    for (size_t i = 0; i < costsTrue.size(); i++)
        costsTrue[i] = (float)costsTrueIn[i];
    for (int branchPlan = 0; branchPlan < NBP; branchPlan++)
        for (int s = 0; s < N; s++)
        {
            int branchTuple[N_MODEL_FACTORS], thetaTuple[N_MODEL_FACTORS];
            unflattenBranchIndex(branchPlan, branchTuple);
            float num = 0.0f, den = 0.0f;
            for (int m = 0; m < NTH; m++)
            {
                unflattenTrueModelIndex(m, thetaTuple);
                if (!branchCompatibleWithModel(branchTuple, thetaTuple))
                    continue;
                float cv = costsTrue[m * N + s];
                if (!isfinite(cv))
                    continue;
                float w = belief[m];
                num += w * cv;
                den += w;
            }
            costs[branchPlan * N + s] = (den > 1e-30f) ? (num / den) : INFINITY;
        }
    if (costsOut)
        std::memcpy(costsOut, costs.data(), costs.size() * 4);
    int initPredTheta[N_MODEL_FACTORS];
    findConfident(belief, mc.minConfidence, initPredTheta);
#pragma omp parallel for num_threads(nthreads > 0 ? nthreads : 1)
    for (int bt = 0; bt < NBP * M; bt++)
    {
        int tLocal = bt % M, branchPlan = bt / M;
        int branchTuple[N_MODEL_FACTORS];
        unflattenBranchIndex(branchPlan, branchTuple);
        float mn = INFINITY;
        if (branchCompatibleWithInitialModel(branchTuple, initPredTheta))
            for (int s = 0; s < N; s++)
            {
                float coeff = sampleCoeffRef(mc, belief, branchPlan, tLocal, s, branchUsed, branchTime);
                if (coeff > MIN_COEFF_THRESHOLD)
                {
                    float cv = costs[branchPlan * N + s];
                    if (cv < mn)
                        mn = cv;
                }
            }
        minCosts[branchPlan * M + tLocal] = mn;
    }
#pragma omp parallel for num_threads(nthreads > 0 ? nthreads : 1)
    for (int btd = 0; btd < NBP * M * ACTION_DIM; btd++)
    {
        int d = btd % ACTION_DIM;
        int rest = btd / ACTION_DIM;
        int tLocal = rest % M, branchPlan = rest / M;
        const int NT = 256;
        float s_num[NT], s_den[NT];
        float minC = minCosts[branchPlan * M + tLocal];
        for (int i = 0; i < NT; i++)
        {
            float num = 0.0f, den = 0.0f;
            if (!isinf(minC))
                for (int s = i; s < N; s += NT)
                {
                    float coeff = sampleCoeffRef(mc, belief, branchPlan, tLocal, s, branchUsed, branchTime);
                    if (coeff > MIN_COEFF_THRESHOLD)
                    {
                        float cost = costs[branchPlan * N + s];
                        float w = expf(-(cost - minC) / mc.invTemperature);
                        float eps = noise[((size_t)(branchPlan * M + tLocal) * N + s) * ACTION_DIM + d];
                        num += w * coeff * eps;
                        den += w * coeff;
                    }
                }
            s_num[i] = num;
            s_den[i] = den;
        }
        for (int stride = NT / 2; stride > 0; stride >>= 1)
            for (int i = 0; i < stride; i++)
            {
                s_num[i] += s_num[i + stride];
                s_den[i] += s_den[i + stride];
            }
        if (s_den[0] > 1e-30f)
            splineOrDense[(branchPlan * M + tLocal) * ACTION_DIM + d] += s_num[0] / s_den[0];
        if (tLocal == 0 && d == 0)
            nu[branchPlan] = s_den[0];
    }
    if (USE_SPLINES)
        for (int idx = 0; idx < NBP * T * ACTION_DIM; idx++)
        {
            int dim = idx % ACTION_DIM, r = idx / ACTION_DIM, t = r % T, branch = r / T;
            float sum = 0.0f;
            for (int m = 0; m < M; m++)
                sum += B[t * M + m] * splineOrDense[(branch * M + m) * ACTION_DIM + dim];
            denseOut[(branch * T + t) * ACTION_DIM + dim] = sum;
        }
    float maxAccel = Env::getMaxAccel(env);
    for (int idx = 0; idx < NBP * M; idx++)
    {
        float sq = 0.0f;
        int base = idx * ACTION_DIM;
        for (int d = 0; d < ACTION_DIM; ++d)
        {
            float v = splineOrDense[base + d];
            sq += v * v;
        }
        float maxSq = maxAccel * maxAccel;
        if (sq > maxSq)
        {
            float scale = maxAccel / sqrtf(sq);
            for (int d = 0; d < ACTION_DIM; ++d)
                splineOrDense[base + d] *= scale;
        }
    }
    if (!USE_SPLINES)
        std::memcpy(denseOut, splineOrDense, (size_t)NBP * T * ACTION_DIM * 4);
    return 0;
}

// verifyNominalFailureKernel (kernels.cu:488-551) with the theta draw and the
// environment noise from the Philox streams.
int refh_mppi_verify(const CEnv* ec, const dr_mppi_config* c, const CState* s0, const float* belief, const float* plan, uint64_t seed,
                     uint64_t step, int planId, unsigned* failCount, int* failTime, int nthreads)
{
    EnvironmentConfig envConfig;
    HostGrids g;
    if (!toRefEnv(*ec, envConfig, g))
        return 2;
    MPPIConfig mc = toRefMppi(*c);
    SimState initState = toRefState(*s0);
    const int V = mc.nVerifSamples;
    std::vector<int> ft(V, -1);
    const orc::Key key(seed);
#pragma omp parallel for schedule(dynamic, 64) num_threads(nthreads > 0 ? nthreads : 1)
    for (int s = 0; s < V; s++)
    {
        SimState state = initState;
        BranchState branchState;
        initBranchState(branchState, belief, mc.minConfidence);
        ScratchEnvBuffer buffer;
        float egoAction[ACTION_DIM];
        float u = orc::uniform_from_word(orc::draw(key, (uint32_t)s, (uint32_t)planId, step, orc::S_VERIF_THETA, 0).v[0]);
        // sampleModelFromBelief, state.h:118-131
        int theta = NTH - 1;
        float cdf = 0.0f;
        for (int k = 0; k < NTH; k++)
        {
            cdf += branchState.belief[k];
            if (u <= cdf)
            {
                theta = k;
                break;
            }
        }
        orc::EnvNoise en(seed, (uint32_t)s, (uint32_t)planId << 16, step, orc::S_VERIF_ENV);
        PhiloxRefRNG rng{&en};
        int tOrigin = 0, t = 0;
        bool failed = false;
        for (; t < mc.verifHorizon; t++)
        {
            en.begin_step((uint32_t)t);
            int local_time = t - tOrigin;
            int flatBranch = flattenBranchIndex(branchState.predTheta.data());
            for (int d = 0; d < ACTION_DIM; d++)
                egoAction[d] = plan[(flatBranch * mc.nTimesteps + local_time) * ACTION_DIM + d];
            bool branched = false;
            TerminalType term =
                environmentStep<true, true, false, false>(t, theta, envConfig, egoAction, true, state, branchState, branched, mc.minConfidence, buffer, rng);
            if (branched)
                tOrigin = t + 1;
            if (term == TERM_LOSE)
            {
                failed = true;
                break;
            }
            else if (term == TERM_WIN || term == TERM_OPP_WIN)
                break;
        }
        if (failed)
            ft[s] = t;
    }
    for (int t = 0; t < mc.nTimesteps; t++)
        failCount[t] = 0;
    for (int s = 0; s < V; s++)
    {
        if (ft[s] >= 0)
            failCount[ft[s]]++;
        if (failTime)
            failTime[s] = ft[s];
    }
    return 0;
}

// MPPIController::buildSplineMatrix (src/mppi_controller.cu:56-141), the reference's own code.
int refh_spline_matrix(const CEnv* ec, const dr_mppi_config* c, float* Bout)
{
    EnvironmentConfig env;
    HostGrids g;
    if (!toRefEnv(*ec, env, g))
        return 2;
    Quiet q;
    MPPIController ctl(env, toRefMppi(*c), 0);
    std::vector<float> B = ctl.buildSplineMatrix();
    std::memcpy(Bout, B.data(), B.size() * sizeof(float));
    return 0;
}

// clopperPearson bounds (include/state.h:134-151).
double refh_cp_lower(unsigned k, unsigned n, double alpha)
{
    return clopperPearsonLowerBound(k, n, alpha);
}
double refh_cp_upper(unsigned k, unsigned n, double alpha)
{
    return clopperPearsonUpperBound(k, n, alpha);
}

// PRMPPIfullRolloutKernel (prmppi_kernels.cu:55-130).
int refh_pr_rollout(const CEnv* ec, const dr_prmppi_config* c, const CState* s0, const float* nom_nominal, const float* rob_nominal,
                    const float* noise, const int* thetas, uint64_t seed, uint64_t step, double* cost_nom, double* cost_rob, int nthreads)
{
    EnvironmentConfig envConfig;
    HostGrids g;
    if (!toRefEnv(*ec, envConfig, g))
        return 2;
    PRMPPIConfig mppiConfig = toRefPr(*c);
    SimState initState = toRefState(*s0);
    const int N = mppiConfig.nSamples, T = mppiConfig.nTimesteps, P = (int)mppiConfig.P;
    const long total = (long)N * P;
#pragma omp parallel for schedule(dynamic, 16) num_threads(nthreads > 0 ? nthreads : 1)
    for (long tid = 0; tid < 2 * total; tid++)
    {
        bool robust = tid >= total;
        long idx = robust ? tid - total : tid;
        int p = (int)(idx / N), s = (int)(idx % N);
        SimState state = initState;
        BranchState branchState;
        ScratchEnvBuffer buffer;
        float egoAction[ACTION_DIM];
        orc::EnvNoise en(seed, (uint32_t)s, ((((uint32_t)robust << 8) | (uint32_t)p) << 16), step, orc::S_PR_ROLL_ENV);
        PhiloxRefRNG rng{&en};
        const float* nominal = robust ? rob_nominal : nom_nominal;
        int theta = thetas[p];
        float runningCost = 0.0f, safeCost = -INFINITY, decay = 1.0f;
        bool stop = false;
        for (int t = 0; t < T && !stop; t++)
        {
            en.begin_step((uint32_t)t);
            for (int d = 0; d < ACTION_DIM; d++)
                egoAction[d] = nominal[t * ACTION_DIM + d] + noise[((size_t)t * N + s) * ACTION_DIM + d];
            bool branched = false;
            TerminalType term = environmentStep<false, false, true>(t, theta, envConfig, egoAction, true, state, branchState, branched, 0.0f, buffer,
                                                                    rng, mppiConfig.gateTraversalMargin);
            stop = (term != TERM_NONE);
            runningCost += decay * PRMPPIstateCost(state, t, envConfig, mppiConfig, theta);
            safeCost = fmaxf(safeCost, PRMPPIsafetyCost(state, t, envConfig, mppiConfig, theta));
            decay *= DECAY;
        }
        runningCost += PRMPPIfinalCost(state, envConfig, mppiConfig, theta);
        double* out = robust ? cost_rob : cost_nom;
        out[idx * 2 + 0] = runningCost;
        out[idx * 2 + 1] = safeCost;
    }
    return 0;
}

// PRMPPIcomputeCandidateCostKernel (prmppi_kernels.cu:285-347) and the rollout of
// PRMPPIcomputeSafeCostKernel (350-393), for both candidates, noise stream `stream`.
int refh_pr_candidates(const CEnv* ec, const dr_prmppi_config* c, const CState* s0, const float* cand1, const float* cand2,
                       const int* thetas, uint64_t seed, uint64_t step, int stream, double* fullCost, double* safeCostOut)
{
    EnvironmentConfig envConfig;
    HostGrids g;
    if (!toRefEnv(*ec, envConfig, g))
        return 2;
    PRMPPIConfig mppiConfig = toRefPr(*c);
    SimState initState = toRefState(*s0);
    const int P = (int)mppiConfig.P;
    for (int tid = 0; tid < 2 * P; tid++)
    {
        bool second = tid >= P;
        int p = second ? tid - P : tid;
        const float* nominal = second ? cand2 : cand1;
        SimState state = initState;
        BranchState branchState;
        ScratchEnvBuffer buffer;
        float egoAction[ACTION_DIM];
        orc::EnvNoise en(seed, (uint32_t)p, (uint32_t)second << 16, step, (uint32_t)stream);
        PhiloxRefRNG rng{&en};
        float cost = 0.0f, safeCost = -INFINITY, decay = 1.0f;
        bool stop = false;
        for (int t = 0; t < mppiConfig.nTimesteps && !stop; ++t)
        {
            en.begin_step((uint32_t)t);
            for (int d = 0; d < ACTION_DIM; ++d)
                egoAction[d] = nominal[t * ACTION_DIM + d];
            bool branched = false;
            TerminalType term = environmentStep<false, false, true>(t, thetas[p], envConfig, egoAction, true, state, branchState, branched, 0.0f,
                                                                    buffer, rng, mppiConfig.gateTraversalMargin);
            stop = (term != TERM_NONE);
            cost += decay * PRMPPIstateCost(state, t, envConfig, mppiConfig, thetas[p]);
            decay *= DECAY;
            safeCost = fmaxf(safeCost, PRMPPIsafetyCost(state, t, envConfig, mppiConfig, thetas[p]));
        }
        cost += PRMPPIfinalCost(state, envConfig, mppiConfig, thetas[p]);
        if (safeCost > 0.0f)
            cost += mppiConfig.safetyWeight;
        fullCost[tid] = cost;
        safeCostOut[tid] = safeCost;
    }
    return 0;
}

// One environment step with the reference's own environmentStep (engine.cpp:286-312).
int refh_env_step(const CEnv* ec, int trueTheta, const float* action, CState* st, float* belief, int updateBelief, int considerBranching,
                  float minConfidence, int loseOnOppWin, int applyNoise, uint64_t seed, uint64_t step, int t)
{
    EnvironmentConfig envConfig;
    HostGrids g;
    if (!toRefEnv(*ec, envConfig, g))
        return -2;
    SimState state = toRefState(*st);
    BranchState bs;
    initBranchState(bs, belief, minConfidence);
    ScratchEnvBuffer buffer;
    orc::EnvNoise en(seed, 0u, 0u, step, orc::S_ENV_STEP);
    en.begin_step(0);
    PhiloxRefRNG rng{&en};
    bool branched = false;
    TerminalType term;
    bool n = applyNoise != 0;
    if (updateBelief && considerBranching && loseOnOppWin)
        term = environmentStep<true, true, false, true>(t, trueTheta, envConfig, action, n, state, bs, branched, minConfidence, buffer, rng);
    else if (updateBelief && considerBranching)
        term = environmentStep<true, true, false, false>(t, trueTheta, envConfig, action, n, state, bs, branched, minConfidence, buffer, rng);
    else if (updateBelief && loseOnOppWin)
        term = environmentStep<true, false, false, true>(t, trueTheta, envConfig, action, n, state, bs, branched, minConfidence, buffer, rng);
    else if (updateBelief)
        term = environmentStep<true, false, false, false>(t, trueTheta, envConfig, action, n, state, bs, branched, minConfidence, buffer, rng);
    else if (loseOnOppWin)
        term = environmentStep<false, false, true, true>(t, trueTheta, envConfig, action, n, state, bs, branched, minConfidence, buffer, rng);
    else
        term = environmentStep<false, false, true, false>(t, trueTheta, envConfig, action, n, state, bs, branched, minConfidence, buffer, rng);
    fromRefState(state, *st);
    for (int th = 0; th < NTH; th++)
        belief[th] = bs.belief[th];
    return (int)term;
}

void refh_costs(const CEnv* ec, const dr_mppi_config* c, const dr_prmppi_config* pc, const CState* s, float* out4)
{
    EnvironmentConfig envConfig;
    HostGrids g;
    if (!toRefEnv(*ec, envConfig, g))
        return;
    MPPIConfig mc = toRefMppi(*c);
    PRMPPIConfig prc = toRefPr(*pc);
    SimState state = toRefState(*s);
    out4[0] = stateCost(state, 0, envConfig, mc, 0);
    out4[1] = PRMPPIstateCost(state, 0, envConfig, prc, 0);
    out4[2] = PRMPPIsafetyCost(state, 0, envConfig, prc, 0);
    out4[3] = finalCost(state, envConfig, mc, 0);
}

// ==== CUDA face (GPU box only) ==============================================================

int refc_device_count()
{
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess)
        return 0;
    return n;
}

// fullRolloutKernel on injected noise (mppi_controller.cu:290-291 launch shape).
int refc_mppi_rollout(const CEnv* ec, const dr_mppi_config* c, const CState* s0, const float* belief, const float* nominal,
                      const float* noise, const float* B, uint64_t seed, float* costsTrue, int* branchUsed, int* branchTime)
{
    EnvironmentConfig env;
    HostGrids g;
    if (!toRefEnv(*ec, env, g))
        return 2;
    DevEnv de(env);
    MPPIConfig mc = toRefMppi(*c);
    SimState init = toRefState(*s0);
    const int N = mc.nSamples, T = mc.nTimesteps, M = MK(mc);
    DevBuf dBelief(NTH * 4), dNom((size_t)NBP * M * 2 * 4), dNoise((size_t)NBP * M * N * 2 * 4), dB((size_t)T * M * 4), dCT((size_t)NTH * N * 4),
        dBU((size_t)NTH * N * 4), dBT((size_t)NTH * N * 4), dRng((size_t)N * sizeof(curandState));
    cudaMemcpy(dBelief.p, belief, NTH * 4, cudaMemcpyHostToDevice);
    cudaMemcpy(dNom.p, nominal, (size_t)NBP * M * 2 * 4, cudaMemcpyHostToDevice);
    cudaMemcpy(dNoise.p, noise, (size_t)NBP * M * N * 2 * 4, cudaMemcpyHostToDevice);
    if (USE_SPLINES)
        cudaMemcpy(dB.p, B, (size_t)T * M * 4, cudaMemcpyHostToDevice);
    int blk = 256, grd = (N + blk - 1) / blk;
    initRNGKernel<<<grd, blk>>>(dRng.as<curandState>(), seed, N);
    fullRolloutKernel<<<grd, blk>>>(de.e, mc, init, dBelief.as<float>(), dNom.as<float>(), dNoise.as<float>(), dB.as<float>(), dCT.as<float>(),
                                    dBU.as<int>(), dBT.as<int>(), dRng.as<curandState>());
    int st = cudaStatus();
    cudaMemcpy(costsTrue, dCT.p, (size_t)NTH * N * 4, cudaMemcpyDeviceToHost);
    cudaMemcpy(branchUsed, dBU.p, (size_t)NTH * N * 4, cudaMemcpyDeviceToHost);
    cudaMemcpy(branchTime, dBT.p, (size_t)NTH * N * 4, cudaMemcpyDeviceToHost);
    return st;
}

// aggregate + masked min + weighted average + interpolate + clamp, the reference
// kernels in the launch order of mppi_controller.cu:299-345.
int refc_mppi_update(const CEnv* ec, const dr_mppi_config* c, const float* belief, const float* costsTrue, const int* branchUsed,
                     const int* branchTime, const float* noise, const float* B, float* splineOrDense, float* denseOut, float* minCosts, float* nu,
                     float* costsOut)
{
    EnvironmentConfig env;
    HostGrids g;
    if (!toRefEnv(*ec, env, g))
        return 2;
    MPPIConfig mc = toRefMppi(*c);
    const int N = mc.nSamples, T = mc.nTimesteps, M = MK(mc);
    DevBuf dBelief(NTH * 4), dCT((size_t)NTH * N * 4), dBU((size_t)NTH * N * 4), dBT((size_t)NTH * N * 4), dCosts((size_t)NBP * N * 4),
        dNoise((size_t)NBP * M * N * 2 * 4), dB((size_t)T * M * 4), dSpl((size_t)NBP * M * 2 * 4), dDense((size_t)NBP * T * 2 * 4), dMin((size_t)NBP * M * 4),
        dNu(NBP * 4);
    cudaMemcpy(dBelief.p, belief, NTH * 4, cudaMemcpyHostToDevice);
    cudaMemcpy(dCT.p, costsTrue, (size_t)NTH * N * 4, cudaMemcpyHostToDevice);
    cudaMemcpy(dBU.p, branchUsed, (size_t)NTH * N * 4, cudaMemcpyHostToDevice);
    cudaMemcpy(dBT.p, branchTime, (size_t)NTH * N * 4, cudaMemcpyHostToDevice);
    cudaMemcpy(dNoise.p, noise, (size_t)NBP * M * N * 2 * 4, cudaMemcpyHostToDevice);
    if (USE_SPLINES)
        cudaMemcpy(dB.p, B, (size_t)T * M * 4, cudaMemcpyHostToDevice);
    cudaMemcpy(dSpl.p, splineOrDense, (size_t)NBP * M * 2 * 4, cudaMemcpyHostToDevice);
    cudaMemset(dNu.p, 0, NBP * 4);
    int blk = 256;
    aggregateBranchCostsKernel<<<(NBP * N + blk - 1) / blk, blk>>>(dCT.as<float>(), dBelief.as<float>(), dCosts.as<float>(), N);
    computeMaskedMinCostsKernel<<<NBP * M, blk, blk * sizeof(float)>>>(dCosts.as<float>(), dBU.as<int>(), dBT.as<int>(), dBelief.as<float>(),
                                                                      dMin.as<float>(), mc);
    weightedAverageKernelUnified<<<NBP * M * ACTION_DIM, blk, 2 * blk * sizeof(float)>>>(dCosts.as<float>(), dMin.as<float>(), dNoise.as<float>(),
                                                                                          dBU.as<int>(), dBT.as<int>(), dBelief.as<float>(),
                                                                                          dSpl.as<float>(), mc, dNu.as<float>());
    if (USE_SPLINES)
        interpolateSplineKernel<<<(NBP * T * ACTION_DIM + blk - 1) / blk, blk>>>(dSpl.as<float>(), dDense.as<float>(), dB.as<float>(), T, M);
    clampNominalKernel<<<(NBP * M + blk - 1) / blk, blk>>>(dSpl.as<float>(), Env::getMaxAccel(env), M);
    int st = cudaStatus();
    cudaMemcpy(splineOrDense, dSpl.p, (size_t)NBP * M * 2 * 4, cudaMemcpyDeviceToHost);
    if (USE_SPLINES)
        cudaMemcpy(denseOut, dDense.p, (size_t)NBP * T * 2 * 4, cudaMemcpyDeviceToHost);
    else
        cudaMemcpy(denseOut, dSpl.p, (size_t)NBP * T * 2 * 4, cudaMemcpyDeviceToHost);
    cudaMemcpy(minCosts, dMin.p, (size_t)NBP * M * 4, cudaMemcpyDeviceToHost);
    cudaMemcpy(nu, dNu.p, NBP * 4, cudaMemcpyDeviceToHost);
    if (costsOut)
        cudaMemcpy(costsOut, dCosts.p, (size_t)NBP * N * 4, cudaMemcpyDeviceToHost);
    return st;
}

// verifyNominalFailureKernel with its curand streams (statistical comparison only).
int refc_mppi_verify(const CEnv* ec, const dr_mppi_config* c, const CState* s0, const float* belief, const float* plan, uint64_t seed,
                     unsigned* failCount)
{
    EnvironmentConfig env;
    HostGrids g;
    if (!toRefEnv(*ec, env, g))
        return 2;
    DevEnv de(env);
    MPPIConfig mc = toRefMppi(*c);
    if (mc.verifHorizon > mc.nTimesteps)
        return 1; // the reference kernel indexes failCount[t] with t < verifHorizon
    SimState init = toRefState(*s0);
    const int V = mc.nVerifSamples, T = mc.nTimesteps;
    DevBuf dBelief(NTH * 4), dPlan((size_t)NBP * T * 2 * 4), dFc((size_t)T * 4), dRng((size_t)V * sizeof(curandState));
    cudaMemcpy(dBelief.p, belief, NTH * 4, cudaMemcpyHostToDevice);
    cudaMemcpy(dPlan.p, plan, (size_t)NBP * T * 2 * 4, cudaMemcpyHostToDevice);
    cudaMemset(dFc.p, 0, (size_t)T * 4);
    int blk = 256, grd = (V + blk - 1) / blk;
    initRNGKernel<<<grd, blk>>>(dRng.as<curandState>(), seed + 1, V);
    verifyNominalFailureKernel<<<grd, blk>>>(de.e, mc, init, dBelief.as<float>(), dPlan.as<float>(), dRng.as<curandState>(), dFc.as<unsigned>());
    int st = cudaStatus();
    cudaMemcpy(failCount, dFc.p, (size_t)T * 4, cudaMemcpyDeviceToHost);
    return st;
}

// PRMPPIfullRolloutKernel on injected noise and thetas.
int refc_pr_rollout(const CEnv* ec, const dr_prmppi_config* c, const CState* s0, const float* nom, const float* rob, const float* noise,
                    const int* thetas, uint64_t seed, float* cost_nom, float* cost_rob)
{
    EnvironmentConfig env;
    HostGrids g;
    if (!toRefEnv(*ec, env, g))
        return 2;
    DevEnv de(env);
    PRMPPIConfig pc = toRefPr(*c);
    SimState init = toRefState(*s0);
    const int N = pc.nSamples, T = pc.nTimesteps, P = (int)pc.P;
    DevBuf dNom((size_t)T * 2 * 4), dRob((size_t)T * 2 * 4), dNoise((size_t)T * N * 2 * 4), dCN((size_t)P * N * 2 * 4), dCR((size_t)P * N * 2 * 4),
        dTh((size_t)P * 4), dRng((size_t)P * N * sizeof(curandState));
    cudaMemcpy(dNom.p, nom, (size_t)T * 2 * 4, cudaMemcpyHostToDevice);
    cudaMemcpy(dRob.p, rob, (size_t)T * 2 * 4, cudaMemcpyHostToDevice);
    cudaMemcpy(dNoise.p, noise, (size_t)T * N * 2 * 4, cudaMemcpyHostToDevice);
    cudaMemcpy(dTh.p, thetas, (size_t)P * 4, cudaMemcpyHostToDevice);
    int blk = 256;
    initRNGKernel<<<(P * N + blk - 1) / blk, blk>>>(dRng.as<curandState>(), seed, P * N);
    PRMPPIfullRolloutKernel<<<(2 * N * P + blk - 1) / blk, blk>>>(de.e, pc, init, dNom.as<float>(), dRob.as<float>(), dNoise.as<float>(), dCN.as<float>(),
                                                                  dCR.as<float>(), dTh.as<int>(), dRng.as<curandState>());
    int st = cudaStatus();
    cudaMemcpy(cost_nom, dCN.p, (size_t)P * N * 2 * 4, cudaMemcpyDeviceToHost);
    cudaMemcpy(cost_rob, dCR.p, (size_t)P * N * 2 * 4, cudaMemcpyDeviceToHost);
    return st;
}

// PRMPPIcostAvgKernel + PRMPPIcomputeMinCostsKernel + PRMPPIWeightedAverageKernel.
int refc_pr_update(const dr_prmppi_config* c, float* cost_nom, float* cost_rob, const float* noise, const float* nom, const float* rob,
                   const float* invTemps, float* minCosts, float* cand1, float* cand2, float* newRob, float* nu)
{
    PRMPPIConfig pc = toRefPr(*c);
    const int N = pc.nSamples, T = pc.nTimesteps, P = (int)pc.P;
    DevBuf dNom((size_t)T * 2 * 4), dRob((size_t)T * 2 * 4), dNoise((size_t)T * N * 2 * 4), dCN((size_t)P * N * 2 * 4), dCR((size_t)P * N * 2 * 4),
        dMin(3 * 4), dC1((size_t)T * 2 * 4), dC2((size_t)T * 2 * 4), dNR((size_t)T * 2 * 4), dNu(3 * 4);
    cudaMemcpy(dNom.p, nom, (size_t)T * 2 * 4, cudaMemcpyHostToDevice);
    cudaMemcpy(dRob.p, rob, (size_t)T * 2 * 4, cudaMemcpyHostToDevice);
    cudaMemcpy(dNoise.p, noise, (size_t)T * N * 2 * 4, cudaMemcpyHostToDevice);
    cudaMemcpy(dCN.p, cost_nom, (size_t)P * N * 2 * 4, cudaMemcpyHostToDevice);
    cudaMemcpy(dCR.p, cost_rob, (size_t)P * N * 2 * 4, cudaMemcpyHostToDevice);
    cudaMemset(dNu.p, 0, 3 * 4);
    int blk = 256;
    PRMPPIcostAvgKernel<<<(2 * N + blk - 1) / blk, blk>>>(dCN.as<float>(), dCR.as<float>(), N, P, pc.safetyWeight);
    PRMPPIcomputeMinCostsKernel<<<3, blk, blk * sizeof(float)>>>(dCN.as<float>(), dCR.as<float>(), dMin.as<float>(), N);
    PRMPPIWeightedAverageKernel<<<3 * T * ACTION_DIM, blk, 2 * blk * sizeof(float)>>>(dNom.as<float>(), dRob.as<float>(), dNoise.as<float>(), dCN.as<float>(),
                                                                                      dCR.as<float>(), dMin.as<float>(), dC1.as<float>(), dC2.as<float>(),
                                                                                      dNR.as<float>(), N, T, invTemps[0], invTemps[1], invTemps[2],
                                                                                      dNu.as<float>());
    int st = cudaStatus();
    cudaMemcpy(cost_nom, dCN.p, (size_t)P * N * 2 * 4, cudaMemcpyDeviceToHost);
    cudaMemcpy(cost_rob, dCR.p, (size_t)P * N * 2 * 4, cudaMemcpyDeviceToHost);
    cudaMemcpy(minCosts, dMin.p, 3 * 4, cudaMemcpyDeviceToHost);
    cudaMemcpy(cand1, dC1.p, (size_t)T * 2 * 4, cudaMemcpyDeviceToHost);
    cudaMemcpy(cand2, dC2.p, (size_t)T * 2 * 4, cudaMemcpyDeviceToHost);
    cudaMemcpy(newRob, dNR.p, (size_t)T * 2 * 4, cudaMemcpyDeviceToHost);
    cudaMemcpy(nu, dNu.p, 3 * 4, cudaMemcpyDeviceToHost);
    return st;
}

// PRMPPIcomputeCandidateCostKernel and PRMPPIcomputeSafeCostKernel (noise-free configs).
int refc_pr_candidates(const CEnv* ec, const dr_prmppi_config* c, const CState* s0, const float* cand1, const float* cand2,
                       const float* chosen, const int* thetas, uint64_t seed, float* candCosts, float* safeCosts)
{
    EnvironmentConfig env;
    HostGrids g;
    if (!toRefEnv(*ec, env, g))
        return 2;
    DevEnv de(env);
    PRMPPIConfig pc = toRefPr(*c);
    SimState init = toRefState(*s0);
    const int T = pc.nTimesteps, P = (int)pc.P;
    DevBuf dC1((size_t)T * 2 * 4), dC2((size_t)T * 2 * 4), dCh((size_t)T * 2 * 4), dTh((size_t)P * 4), dCC((size_t)2 * P * 4), dSC((size_t)P * 4),
        dRng((size_t)2 * P * sizeof(curandState));
    cudaMemcpy(dC1.p, cand1, (size_t)T * 2 * 4, cudaMemcpyHostToDevice);
    cudaMemcpy(dC2.p, cand2, (size_t)T * 2 * 4, cudaMemcpyHostToDevice);
    cudaMemcpy(dCh.p, chosen, (size_t)T * 2 * 4, cudaMemcpyHostToDevice);
    cudaMemcpy(dTh.p, thetas, (size_t)P * 4, cudaMemcpyHostToDevice);
    int blk = 256;
    initRNGKernel<<<(2 * P + blk - 1) / blk, blk>>>(dRng.as<curandState>(), seed, 2 * P);
    PRMPPIcomputeCandidateCostKernel<<<(2 * P + blk - 1) / blk, blk>>>(de.e, pc, init, dC1.as<float>(), dC2.as<float>(), dTh.as<int>(), dCC.as<float>(),
                                                                       dRng.as<curandState>());
    PRMPPIcomputeSafeCostKernel<<<(P + blk - 1) / blk, blk>>>(de.e, pc, init, dCh.as<float>(), dTh.as<int>(), dSC.as<float>(), dRng.as<curandState>());
    int st = cudaStatus();
    cudaMemcpy(candCosts, dCC.p, (size_t)2 * P * 4, cudaMemcpyDeviceToHost);
    cudaMemcpy(safeCosts, dSC.p, (size_t)P * 4, cudaMemcpyDeviceToHost);
    return st;
}

// Timing of the reference CUDA path on a GPU, two figures:
//  out[0] = kernels-only ms per control step (noise generation .. clamp, CUDA events,
//           mppi_controller.cu:282-345, injected initial state, no host copies),
//  out[1] = full MPPIController::getControl wall ms per step (stdout silenced).
// nAgents controllers are stepped one after the other per control step.
int refc_mppi_time(const CEnv* ec, const dr_mppi_config* c, const CState* s0, int nAgents, int warmup, int steps, double* out)
{
    EnvironmentConfig env;
    HostGrids g;
    if (!toRefEnv(*ec, env, g))
        return 2;
    DevEnv de(env);
    MPPIConfig mc = toRefMppi(*c);
    SimState init = toRefState(*s0);
    const int N = mc.nSamples, T = mc.nTimesteps, M = MK(mc);
    {
        // kernels-only sequence
        DevBuf dBelief(NTH * 4), dNom((size_t)NBP * M * 2 * 4), dDense((size_t)NBP * T * 2 * 4), dNoise((size_t)NBP * M * N * 2 * 4), dB((size_t)T * M * 4),
            dCT((size_t)NTH * N * 4), dBU((size_t)NTH * N * 4), dBT((size_t)NTH * N * 4), dCosts((size_t)NBP * N * 4), dMin((size_t)NBP * M * 4), dNu(NBP * 4),
            dRng((size_t)N * sizeof(curandState));
        std::vector<float> bel(NTH);
        for (int i = 0; i < NTH; i++)
            bel[i] = env.initBelief[i];
        cudaMemcpy(dBelief.p, bel.data(), NTH * 4, cudaMemcpyHostToDevice);
        cudaMemset(dNom.p, 0, (size_t)NBP * M * 2 * 4);
        cudaMemset(dB.p, 0, (size_t)T * M * 4);
        int blk = 256, grd = (N + blk - 1) / blk;
        initRNGKernel<<<grd, blk>>>(dRng.as<curandState>(), 1234, N);
        cudaEvent_t e0, e1;
        cudaEventCreate(&e0);
        cudaEventCreate(&e1);
        auto seq = [&]()
        {
            generateNoiseKernel<<<grd, blk>>>(dNoise.as<float>(), dRng.as<curandState>(), mc.samplingNoise, M, N);
            fullRolloutKernel<<<grd, blk>>>(de.e, mc, init, dBelief.as<float>(), dNom.as<float>(), dNoise.as<float>(), dB.as<float>(), dCT.as<float>(),
                                            dBU.as<int>(), dBT.as<int>(), dRng.as<curandState>());
            aggregateBranchCostsKernel<<<(NBP * N + blk - 1) / blk, blk>>>(dCT.as<float>(), dBelief.as<float>(), dCosts.as<float>(), N);
            computeMaskedMinCostsKernel<<<NBP * M, blk, blk * sizeof(float)>>>(dCosts.as<float>(), dBU.as<int>(), dBT.as<int>(), dBelief.as<float>(),
                                                                              dMin.as<float>(), mc);
            weightedAverageKernelUnified<<<NBP * M * ACTION_DIM, blk, 2 * blk * sizeof(float)>>>(
                dCosts.as<float>(), dMin.as<float>(), dNoise.as<float>(), dBU.as<int>(), dBT.as<int>(), dBelief.as<float>(), dNom.as<float>(), mc,
                dNu.as<float>());
            if (USE_SPLINES)
                interpolateSplineKernel<<<(NBP * T * ACTION_DIM + blk - 1) / blk, blk>>>(dNom.as<float>(), dDense.as<float>(), dB.as<float>(), T, M);
            clampNominalKernel<<<(NBP * M + blk - 1) / blk, blk>>>(dNom.as<float>(), Env::getMaxAccel(env), M);
        };
        for (int i = 0; i < warmup; i++)
            for (int a = 0; a < nAgents; a++)
                seq();
        cudaEventRecord(e0);
        for (int i = 0; i < steps; i++)
            for (int a = 0; a < nAgents; a++)
                seq();
        cudaEventRecord(e1);
        cudaEventSynchronize(e1);
        float ms = 0;
        cudaEventElapsedTime(&ms, e0, e1);
        out[0] = ms / steps;
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        int st = cudaStatus();
        if (st)
            return st;
    }
    {
        // full getControl
        Quiet q;
        std::vector<std::unique_ptr<MPPIController>> ctl;
        for (int a = 0; a < nAgents; a++)
        {
            ctl.emplace_back(new MPPIController(de.e, mc, 42 + a));
            ctl.back()->engine = reinterpret_cast<SimulationEngine*>(ctl.back().get()); // only tested for nullptr (mppi_controller.cu:252)
        }
        float act[2];
        for (int i = 0; i < warmup; i++)
            for (int a = 0; a < nAgents; a++)
                ctl[a]->getControl(init, act);
        cudaDeviceSynchronize();
        auto t0 = std::chrono::steady_clock::now();
        for (int i = 0; i < steps; i++)
            for (int a = 0; a < nAgents; a++)
                ctl[a]->getControl(init, act);
        cudaDeviceSynchronize();
        auto t1 = std::chrono::steady_clock::now();
        out[1] = std::chrono::duration<double, std::milli>(t1 - t0).count() / steps;
    }
    return cudaStatus();
}

// Full PRMPPIController::getControl wall ms per control step (nAgents controllers).
int refc_prmppi_time(const CEnv* ec, const dr_prmppi_config* c, const CState* s0, int nAgents, int warmup, int steps, double* out)
{
    EnvironmentConfig env;
    HostGrids g;
    if (!toRefEnv(*ec, env, g))
        return 2;
    DevEnv de(env);
    PRMPPIConfig pc = toRefPr(*c);
    SimState init = toRefState(*s0);
    Quiet q;
    std::vector<std::unique_ptr<PRMPPIController>> ctl;
    for (int a = 0; a < nAgents; a++)
    {
        ctl.emplace_back(new PRMPPIController(de.e, pc, 42 + a));
        ctl.back()->engine = reinterpret_cast<SimulationEngine*>(ctl.back().get());
    }
    float act[2];
    for (int i = 0; i < warmup; i++)
        for (int a = 0; a < nAgents; a++)
            ctl[a]->getControl(init, act);
    cudaDeviceSynchronize();
    auto t0 = std::chrono::steady_clock::now();
    for (int i = 0; i < steps; i++)
        for (int a = 0; a < nAgents; a++)
            ctl[a]->getControl(init, act);
    cudaDeviceSynchronize();
    auto t1 = std::chrono::steady_clock::now();
    out[0] = std::chrono::duration<double, std::milli>(t1 - t0).count() / steps;
    return cudaStatus();
}

} // extern "C"
