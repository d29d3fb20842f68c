// MPPIController / PRMPPIController of the reference's controller interface
// (include/controllers.h), implemented over the C ABI of libdrmppi (include/drmppi.h).
// A maintainer builds this file in place of src/mppi_controller.cu,
// src/prmppi_controller.cu, src/kernels.cu and src/prmppi_kernels.cu, with the
// controllers.h next to it, and links libdrmppi.so.
//
// Semantics kept from the reference: the constructor stores the configuration
// (mppi_controller.cu:15-49, prmppi_controller.cu:14-40) and validates the size of a
// given nominal; device state is created on the first getControl; getControl throws
// std::runtime_error when engine is unset (mppi_controller.cu:252-253) and fills the
// public fields the engine reads; mppiConfig.invTemperature follows the temperature
// adaptation (mppi_controller.cu:413-424). CUDA and configuration errors surface as
// std::runtime_error with the library's message (the reference ignores CUDA errors in
// release builds, include/common.h:20).
#include "controllers.h"

#include <cuda_runtime.h>

#include <cstring>
#include <format>
#include <stdexcept>

namespace
{

void check(int status, const char* what)
{
    if (status != DR_OK)
        throw std::runtime_error(std::format("{}: {} ({})", what, dr_status_string(status), dr_last_error()));
}

// a host copy of n floats at p, which may be device memory (the engine passes the device
// copy of the environment, engine.cpp:26,37,42)
void hostCopy(const float* p, size_t n, float* out)
{
    cudaPointerAttributes attr{};
    bool dev = cudaPointerGetAttributes(&attr, p) == cudaSuccess && attr.type == cudaMemoryTypeDevice;
    cudaGetLastError();
    if (dev)
    {
        if (cudaMemcpy(out, p, n * sizeof(float), cudaMemcpyDeviceToHost) != cudaSuccess)
            throw std::runtime_error("copying the track from the device failed");
    }
    else
        std::memcpy(out, p, n * sizeof(float));
}

#ifdef USE_ENV_DRONERACE
// dr_gate_env_config from the gate race's EnvironmentConfig (env_dronerace_defs.h:60-93)
void envFromRef(const EnvironmentConfig& c, dr_gate_env_config& e, std::vector<float>& track)
{
    constexpr int NTS = DR_N_TRACK_SAMPLES;
    static_assert(Env::N_RACELINES == DR_GATE_RACELINES && Env::N_AGENTS == DR_GATE_AGENTS, "gate race sizes");
    static_assert(Env::N_GATES <= DR_GATE_MAX_GATES && Env::N_OBSTACLES <= DR_GATE_MAX_OBSTACLES && Env::N_ROUND_OBSTACLES <= DR_GATE_MAX_OBSTACLES,
                  "gate race sizes");
    std::memset(&e, 0, sizeof(e));
    e.n_theta = N_TRUE_MODELS;
    for (int d = 0; d < DR_DIM; d++)
    {
        e.arena_min[d] = c.arenaMin[d];
        e.arena_max[d] = c.arenaMax[d];
    }
    e.dt = c.dt;
    e.send_states = c.sendStates ? 1 : 0;
    e.drone_radius = c.droneRadius;
    e.pos_noise_level = c.posNoiseLevel;
    e.speed_noise_level = c.speedNoiseLevel;
    e.action_noise_level = c.actionNoiseLevel;
    for (int a = 0; a < Env::N_AGENTS; a++)
    {
        e.max_speed[a] = c.maxSpeed[a];
        e.max_accel[a] = c.maxAccel[a];
    }
    e.n_win_laps = c.nWinLaps;
    e.target_distance = c.targetDistance;
    e.n_gates = Env::N_GATES;
    for (int i = 0; i < Env::N_GATES * DR_DIM; i++)
    {
        e.gate_centers[i] = c.gateCenters[i];
        e.gate_vectors[i] = c.gateVectors[i];
    }
    for (int i = 0; i < Env::N_GATES; i++)
        e.gate_radius[i] = c.gateRadius[i];
    e.n_obstacles = Env::N_OBSTACLES;
    for (int i = 0; i < Env::N_OBSTACLES * DR_DIM * 2; i++)
        e.obstacles[i] = c.obstacles[i];
    e.n_round_obstacles = Env::N_ROUND_OBSTACLES;
    for (int i = 0; i < Env::N_ROUND_OBSTACLES * DR_DIM; i++)
        e.round_obs_centers[i] = c.roundObsCenters[i];
    for (int i = 0; i < Env::N_ROUND_OBSTACLES; i++)
        e.round_obs_radius[i] = c.roundObsRadius[i];
    for (int th = 0; th < N_TRUE_MODELS; th++)
    {
        e.init_belief[th] = c.initBelief[th];
        const auto& p = c.oppPid[th];
        e.opp_pid[th] = dr_pid_config{p.kp, p.kd, p.repulsionFactor, p.repulsionPower, p.repulsionDistFact, p.racelineIndex, p.actionNoise};
    }
    e.i_mppi = c.iMppi;
    track.assign((size_t)Env::N_RACELINES * NTS * DR_DIM, 0.0f);
    hostCopy(c.trackPoints, track.size(), track.data());
    e.track_points = track.data();
}

dr_gate_state stateFromRef(const SimState& s)
{
    dr_gate_state r;
    std::memset(&r, 0, sizeof(r));
    for (int i = 0; i < Env::N_AGENTS * DR_DIM; i++)
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

int createMppi(const dr_gate_env_config* e, const dr_mppi_config* c, uint64_t seed, const float* nominal, int dev, dr_mppi** h)
{
    return dr_gate_mppi_create(e, c, seed, nominal, dev, nullptr, h);
}

int stepMppi(dr_mppi* h, const dr_gate_state* s, const float* belief, float* out, dr_mppi_info* info)
{
    return dr_gate_mppi_step(h, s, belief, out, info);
}
#else
// dr_env_config from the reference's EnvironmentConfig, whose grid pointers are device
// pointers here (the engine passes the device copy, engine.cpp:26,37,42).
void envFromRef(const EnvironmentConfig& c, dr_env_config& e, std::vector<float>& grids)
{
    constexpr int NTS = DR_N_TRACK_SAMPLES;
    std::memset(&e, 0, sizeof(e));
    e.n_opp = Env::N_OPP;
    e.n_theta = N_TRUE_MODELS;
    for (int d = 0; d < DR_DIM; d++)
    {
        e.arena_min[d] = c.arenaMin[d];
        e.arena_max[d] = c.arenaMax[d];
    }
    e.dt = c.dt;
    e.send_states = c.sendStates ? 1 : 0;
    e.drone_radius = c.droneRadius;
    e.pos_noise_level = c.posNoiseLevel;
    e.speed_noise_level = c.speedNoiseLevel;
    e.action_noise_level = c.actionNoiseLevel;
    for (int a = 0; a < Env::N_AGENTS; a++)
    {
        e.max_speed[a] = c.maxSpeed[a];
        e.max_accel[a] = c.maxAccel[a];
    }
    e.track_width = c.trackWidth;
    e.n_win_laps = c.nWinLaps;
    for (int th = 0; th < N_TRUE_MODELS; th++)
    {
        e.init_belief[th] = c.initBelief[th];
        for (int o = 0; o < Env::N_OPP; o++)
        {
            e.opp_configs[th].s1[o] = c.oppConfigs[th].s1[o];
            e.opp_configs[th].s2[o] = c.oppConfigs[th].s2[o];
            e.opp_configs[th].s3[o] = c.oppConfigs[th].s3[o];
            e.opp_configs[th].speed_scale[o] = c.oppConfigs[th].speedScale[o];
            e.opp_configs[th].action_noise[o] = c.oppConfigs[th].actionNoise[o];
        }
    }
    e.kP = c.kP;
    e.kV = c.kV;
    e.max_opp_lat_dist_fact = c.maxOppLatDistFact;
    e.track_length = c.trackLength;
    grids.assign(NTS * 7, 0.0f);
    const float* src[4] = {c.p_grid, c.dp_grid, c.t_grid, c.kappa_grid};
    const size_t n[4] = {NTS * 2, NTS * 2, NTS * 2, NTS};
    size_t off = 0;
    for (int i = 0; i < 4; i++)
    {
        hostCopy(src[i], n[i], grids.data() + off);
        off += n[i];
    }
    e.p_grid = grids.data();
    e.dp_grid = grids.data() + NTS * 2;
    e.t_grid = grids.data() + NTS * 4;
    e.kappa_grid = grids.data() + NTS * 6;
}

dr_sim_state stateFromRef(const SimState& s)
{
    dr_sim_state r;
    std::memset(&r, 0, sizeof(r));
    for (int i = 0; i < Env::N_AGENTS * DR_DIM; i++)
    {
        r.pos[i] = s.pos[i];
        r.vel[i] = s.vel[i];
    }
    for (int a = 0; a < Env::N_AGENTS; a++)
    {
        r.S[a] = s.S[a];
        r.lat_dist[a] = s.latDist[a];
        r.laps[a] = s.laps[a];
    }
    return r;
}

int createMppi(const dr_env_config* e, const dr_mppi_config* c, uint64_t seed, const float* nominal, int dev, dr_mppi** h)
{
    return dr_mppi_create(e, c, seed, nominal, dev, nullptr, h);
}

int stepMppi(dr_mppi* h, const dr_sim_state* s, const float* belief, float* out, dr_mppi_info* info)
{
    return dr_mppi_step(h, s, belief, out, info);
}
#endif

} // namespace

// ---- MPPI ------------------------------------------------------------------------------

MPPIController::MPPIController(const EnvironmentConfig& c, const MPPIConfig& mc, int s, std::optional<std::vector<float>> nominal)
{
    mppiConfig = mc;
    seed = s;
    std::copy(c.initBelief.begin(), c.initBelief.end(), h_belief.begin());
    if (nominal)
    {
        if ((int)nominal->size() != N_BRANCH_PLANS * mc.nTimesteps * ACTION_DIM)
            throw std::runtime_error(std::format("Invalid MPPI construction: expected nominal size {}, got {}", N_BRANCH_PLANS * mc.nTimesteps * ACTION_DIM,
                                                 nominal->size()));
        h_nominal = nominal.value();
    }
    else
        h_nominal.assign(N_BRANCH_PLANS * mc.nTimesteps * ACTION_DIM, 0.0f);
    failCountNew.assign(mc.nTimesteps, 0u);
    failCountOld.assign(mc.nTimesteps, 0u);
    failCount.assign(mc.nTimesteps, 0u);
    envFromRef(c, envC, grids);
    std::memset(&cfgC, 0, sizeof(cfgC));
    cfgC.n_samples = mc.nSamples;
    cfgC.n_timesteps = mc.nTimesteps;
    cfgC.n_knots = USE_SPLINES ? mc.nKnots : mc.nTimesteps;
    for (int i = 0; i < DR_MAX_KNOTS && i < MAX_N_KNOTS; i++)
        cfgC.knots[i] = mc.knots[i];
    cfgC.use_splines = USE_SPLINES ? 1 : 0;
    cfgC.inv_temperature = mc.invTemperature;
    cfgC.sampling_noise = mc.samplingNoise;
    cfgC.gate_traversal_margin = mc.gateTraversalMargin;
    cfgC.coll_dist_factor = mc.collDistFactor;
    cfgC.boundary_cost = mc.boundaryCost;
    cfgC.boundary_threshold_factor = mc.boundaryThresholdFactor;
    cfgC.outside_cost = mc.outsideCost;
    cfgC.win_cost = mc.winCost;
    cfgC.opp_win_cost = mc.oppWinCost;
    cfgC.final_adv_weight = mc.finalAdvWeight;
    cfgC.final_opp_adv_weight = mc.finalOppAdvWeight;
    cfgC.min_confidence = mc.minConfidence;
    cfgC.n_verif_samples = mc.nVerifSamples;
    cfgC.beta = mc.beta;
    cfgC.verif_horizon = mc.verifHorizon;
    cfgC.max_verif_eps = mc.maxVerifEps;
    cfgC.min_nu = min_nu;
    cfgC.max_nu = max_nu;
    cfgC.verify = 1;
}

MPPIController::~MPPIController()
{
    dr_mppi_destroy(h);
}

std::vector<float> MPPIController::buildSplineMatrix()
{
    std::vector<float> B((size_t)mppiConfig.nTimesteps * mppiConfig.nKnots);
    check(dr_spline_matrix(mppiConfig.nTimesteps, mppiConfig.nKnots, mppiConfig.knots.data(), B.data()), "dr_spline_matrix");
    return B;
}

void MPPIController::getControl(const SimState& state, float* outAction)
{
    if (!engine)
        throw std::runtime_error("MPPI: engine not set");
    if (!h)
    {
        int dev = 0;
        cudaGetDevice(&dev);
        check(createMppi(&envC, &cfgC, (uint64_t)seed, h_nominal.data(), dev, &h), "dr_mppi_create");
    }
    auto s = stateFromRef(state);
    dr_mppi_info info{};
    check(stepMppi(h, &s, h_belief.data(), outAction, &info), "dr_mppi_step");
    check(dr_mppi_get_fail_counts(h, failCountNew.data(), failCountOld.data(), failCount.data(), failCount.size()), "dr_mppi_get_fail_counts");
    check(dr_mppi_get_nominal(h, h_nominal.data(), h_nominal.size()), "dr_mppi_get_nominal");
    epsilon = info.epsilon;
    epsilonPartial = info.epsilon_partial;
    certifiedLoss = info.certified_loss;
    useNewPlan = info.use_new_plan != 0;
    mppiConfig.invTemperature = info.inv_temperature;
}

// ---- PR-MPPI ---------------------------------------------------------------------------

PRMPPIController::PRMPPIController(const EnvironmentConfig& c, const PRMPPIConfig& mc, int s, std::optional<std::vector<float>> nominal)
{
    mppiConfig = mc;
    seed = s;
    std::copy(c.initBelief.begin(), c.initBelief.end(), h_belief.begin());
    if (nominal)
    {
        if ((int)nominal->size() != mc.nTimesteps * ACTION_DIM)
            throw std::runtime_error(std::format("Invalid PRMPPI construction: expected nominal size {}, got {}", mc.nTimesteps * ACTION_DIM, nominal->size()));
        h_nom_nominal = nominal.value();
        h_rob_nominal = nominal.value();
    }
    else
    {
        h_nom_nominal.assign(mc.nTimesteps * ACTION_DIM, 0.0f);
        h_rob_nominal.assign(mc.nTimesteps * ACTION_DIM, 0.0f);
    }
    resetNom = false;
    useNomPlan = true;
    envFromRef(c, envC, grids);
    std::memset(&cfgC, 0, sizeof(cfgC));
    cfgC.n_samples = mc.nSamples;
    cfgC.n_timesteps = mc.nTimesteps;
    cfgC.inv_temperature = mc.invTemperature;
    cfgC.sampling_noise = mc.samplingNoise;
    cfgC.gate_traversal_margin = mc.gateTraversalMargin;
    cfgC.coll_dist_factor = mc.collDistFactor;
    cfgC.boundary_cost = mc.boundaryCost;
    cfgC.boundary_threshold_factor = mc.boundaryThresholdFactor;
    cfgC.win_cost = mc.winCost;
    cfgC.opp_win_cost = mc.oppWinCost;
    cfgC.final_adv_weight = mc.finalAdvWeight;
    cfgC.final_opp_adv_weight = mc.finalOppAdvWeight;
    cfgC.safety_weight = mc.safetyWeight;
    cfgC.min_safe_dist = mc.minSafeDist;
    cfgC.delta = mc.delta;
    cfgC.P = (int)mc.P;
    cfgC.min_nu = min_nu;
    cfgC.max_nu = max_nu;
}

PRMPPIController::~PRMPPIController()
{
    dr_prmppi_destroy(h);
}

void PRMPPIController::getControl(const SimState& state, float* outAction)
{
    if (!engine)
        throw std::runtime_error("PRMPPI: engine not set");
#ifdef USE_ENV_DRONERACE
    (void)state;
    (void)outAction;
    throw std::runtime_error("PRMPPI: libdrmppi provides PR-MPPI on the strategic race only");
#else
    if (!h)
    {
        int dev = 0;
        cudaGetDevice(&dev);
        check(dr_prmppi_create(&envC, &cfgC, (uint64_t)seed, h_nom_nominal.data(), dev, nullptr, &h), "dr_prmppi_create");
    }
    dr_sim_state s = stateFromRef(state);
    dr_prmppi_info info{};
    check(dr_prmppi_step(h, &s, h_belief.data(), outAction, &info), "dr_prmppi_step");
    check(dr_prmppi_get_nominals(h, h_nom_nominal.data(), h_rob_nominal.data(), h_nom_nominal.size()), "dr_prmppi_get_nominals");
    resetNom = info.reset_nom != 0;
    useNomPlan = info.use_nom_plan != 0;
#endif
}
