// TEST INFRASTRUCTURE (oracle). Not part of the product.
//
// Drives the C++ drop-in adapter (drone-race_b200/adapter) built against the reference's
// headers with USE_ENV_DRONERACE: the reference's MPPIController interface on the gate
// race, over libdrmppi. The reference's engine does not build for the gate race (it
// names the strategic race directly, src/engine.cpp:233), so this driver stands in for
// it: it builds the reference's EnvironmentConfig / MPPIConfig / SimState from the C-ABI
// structs, constructs the controller and calls getControl like the engine does.
#include "config.h"
#include "controllers.h"

#include <cstring>
#include <exception>
#include <vector>

extern "C" int adapter_gate_run(const dr_gate_env_config* c, const dr_mppi_config* m, int seed, const dr_gate_state* s0, int nsteps, float* actions,
                                float* nominals)
{
    try
    {
        EnvironmentConfig e;
        for (int d = 0; d < 2; d++)
        {
            e.arenaMin[d] = c->arena_min[d];
            e.arenaMax[d] = c->arena_max[d];
        }
        e.dt = c->dt;
        e.sendStates = c->send_states != 0;
        e.droneRadius = c->drone_radius;
        e.posNoiseLevel = c->pos_noise_level;
        e.speedNoiseLevel = c->speed_noise_level;
        e.actionNoiseLevel = c->action_noise_level;
        for (int a = 0; a < Env::N_AGENTS; a++)
        {
            e.maxSpeed[a] = c->max_speed[a];
            e.maxAccel[a] = c->max_accel[a];
        }
        e.nWinLaps = c->n_win_laps;
        e.targetDistance = c->target_distance;
        for (int i = 0; i < Env::N_GATES * 2; i++)
        {
            e.gateCenters[i] = c->gate_centers[i];
            e.gateVectors[i] = c->gate_vectors[i];
        }
        for (int i = 0; i < Env::N_GATES; i++)
            e.gateRadius[i] = c->gate_radius[i];
        std::vector<float> track(c->track_points, c->track_points + (size_t)Env::N_RACELINES * Env::N_TRACK_SAMPLES * 2);
        e.trackPoints = track.data();
        for (int th = 0; th < N_TRUE_MODELS; th++)
        {
            e.initBelief[th] = c->init_belief[th];
            const dr_pid_config& p = c->opp_pid[th];
            e.oppPid[th].kp = p.kp;
            e.oppPid[th].kd = p.kd;
            e.oppPid[th].repulsionFactor = p.repulsion_factor;
            e.oppPid[th].repulsionPower = p.repulsion_power;
            e.oppPid[th].repulsionDistFact = p.repulsion_dist_fact;
            e.oppPid[th].racelineIndex = p.raceline_index;
            e.oppPid[th].actionNoise = p.action_noise;
        }
        e.iMppi = c->i_mppi;
        MPPIConfig mc;
        mc.nSamples = m->n_samples;
        mc.nTimesteps = m->n_timesteps;
        mc.nKnots = USE_SPLINES ? m->n_knots : m->n_timesteps;
        for (int i = 0; i < MAX_N_KNOTS; i++)
            mc.knots[i] = i < DR_MAX_KNOTS ? m->knots[i] : 0;
        mc.invTemperature = m->inv_temperature;
        mc.samplingNoise = m->sampling_noise;
        mc.gateTraversalMargin = m->gate_traversal_margin;
        mc.collDistFactor = m->coll_dist_factor;
        mc.boundaryCost = m->boundary_cost;
        mc.boundaryThresholdFactor = m->boundary_threshold_factor;
        mc.outsideCost = m->outside_cost;
        mc.winCost = m->win_cost;
        mc.oppWinCost = m->opp_win_cost;
        mc.finalAdvWeight = m->final_adv_weight;
        mc.finalOppAdvWeight = m->final_opp_adv_weight;
        mc.minConfidence = m->min_confidence;
        mc.nVerifSamples = m->n_verif_samples;
        mc.beta = m->beta;
        mc.verifHorizon = m->verif_horizon;
        mc.maxVerifEps = m->max_verif_eps;
        SimState st;
        for (int i = 0; i < Env::N_AGENTS * 2; i++)
        {
            st.pos[i] = s0->pos[i];
            st.vel[i] = s0->vel[i];
        }
        for (int i = 0; i < Env::N_AGENTS * Env::N_RACELINES; i++)
            st.S[i] = s0->S[i];
        for (int a = 0; a < Env::N_AGENTS; a++)
        {
            st.laps[a] = s0->laps[a];
            st.gates[a] = s0->gates[a];
        }
        MPPIController ctl(e, mc, seed);
        ctl.engine = reinterpret_cast<SimulationEngine*>(&ctl); // only tested for nullptr
        const size_t nn = ctl.h_nominal.size();
        for (int k = 0; k < nsteps; k++)
        {
            ctl.getControl(st, actions + 2 * k);
            std::memcpy(nominals + k * nn, ctl.h_nominal.data(), nn * sizeof(float));
        }
        return 0;
    }
    catch (const std::exception&)
    {
        return 1;
    }
}
