// C ABI of the PR-MPPI controller (reference PRMPPIController, src/prmppi_controller.cu)
// and of the device environment step (reference SimulationEngine::dynStep,
// src/engine.cpp:286-312).
#include <algorithm>
#include <memory>
#include <vector>
#include <cmath>
#include <cstring>
#include <map>
#include <mutex>
#include <type_traits>

#include <cuda_runtime.h>

#include "../../include/drmppi.h"
#include "common.cuh"
#include "hostutil.hpp"
#include "instance.cuh"
#include "launch.h"

using namespace dr;

struct dr_prmppi
{
    int device = 0;
    cudaStream_t stream = nullptr;
    bool ownStream = false;
    dr_env_config env{};
    dr_prmppi_config cfg{};
    uint64_t seed = 0;
    int nth = 0, nopp = 0, K = 0, T = 0, P = 0;
    Arena arena;
    PrDev desc{};
    unsigned char* hRes = nullptr;
    std::vector<float> hNom, hRob;
    bool useNomPlan = true, resetNom = false;
    float lambda[3] = {1, 1, 1}; // invTempNomFull, invTempRobFull, invTempRobSafe
    uint64_t step = 0;
    dr_prmppi_batch* self = nullptr;
    // sample sharding across processes (dr_prmppi_set_shard): this process's samples
    int shardWorld = 1;
    int sLo = 0, sHi = 0;
    int envKind = 0, iMppi = 0; // 1: the gate race, with the ego at index iMppi
    DevScratch predBuf;         // dr_prmppi_predict's inputs and outputs on the device

    PrIn input(const dr_gate_state& s, const float* belief) const
    {
        PrIn in = input(dr_sim_state{}, belief);
        in.gstate = s;
        return in;
    }

    PrIn input(const dr_sim_state& s, const float* belief) const
    {
        PrIn in{};
        in.state = s;
        for (int i = 0; i < DR_MAX_THETA; i++)
            in.belief[i] = i < nth ? belief[i] : 0.0f;
        for (int i = 0; i < 3; i++)
            in.lambda[i] = lambda[i];
        in.step = (uint32_t)step;
        return in;
    }

    template <typename T_> const T_* at(const void* devPtr) const
    {
        return (const T_*)(hRes + ((const unsigned char*)devPtr - (const unsigned char*)desc.nom));
    }

    // host tail of PRMPPIController::getControl (prmppi_controller.cu:268-346); the
    // candidate choice and the safety decision were taken on the device.
    int lastTimeouts = 0; // staging waits that gave up in the last finished step

    void finish(float* outAction, dr_prmppi_info* info)
    {
        const float* nom = at<float>(desc.nom);
        const float* rob = at<float>(desc.rob);
        const float* mins = at<float>(desc.minCosts);
        const float* nu = at<float>(desc.nu);
        const float* full = at<float>(desc.candFull);
        const int* dec = at<int>(desc.decision);
        const int* stats = at<int>(desc.stats);
        lastTimeouts = stats[1];
        resetNom = dec[0] != 0;
        useNomPlan = dec[1] != 0;
        hNom.assign(nom, nom + (size_t)T * 2);
        hRob.assign(rob, rob + (size_t)T * 2);
        const float* first = useNomPlan ? nom : rob;
        outAction[0] = first[0];
        outAction[1] = first[1];
        for (int w = 0; w < 3; w++)
        {
            // adaptTemperature (prmppi_controller.cu:328-342)
            float& invTemp = lambda[w];
            if (nu[w] > cfg.max_nu * (float)K && invTemp > 0.01f)
                invTemp *= 0.9f;
            else if (nu[w] < cfg.min_nu * (float)K && invTemp < 100.0f)
                invTemp *= 1.2f;
        }
        step++;
        if (info)
        {
            info->use_nom_plan = useNomPlan;
            info->reset_nom = resetNom;
            float c1 = 0.0f, c2 = 0.0f;
            for (int p = 0; p < P; p++)
            {
                c1 += full[p];
                c2 += full[P + p];
            }
            info->cand_cost[0] = c1 / (float)P;
            info->cand_cost[1] = c2 / (float)P;
            for (int w = 0; w < 3; w++)
            {
                info->min_costs[w] = mins[w];
                info->nu[w] = nu[w];
                info->inv_temperature[w] = lambda[w];
            }
            info->nonfinite_costs = stats[0];
        }
    }
};

// Hypothesis slots per PR-MPPI rollout thread by default (dr_prmppi_batch_set_rollout_slots).
constexpr int DEFAULT_PR_SLOTS = 1;

struct dr_prmppi_batch
{
    std::vector<dr_prmppi*> hs;
    int device = 0;
    cudaStream_t stream = nullptr;
    bool ownStream = false;
    int nopp = 0, nth = 0, maxT = 0, maxP = 0;
    int envKind = 0, iMppi = 0;
    PrDev* dDesc = nullptr;
    PrIn* dIn = nullptr;
    PrIn* hIn = nullptr;
    Tile *dRoll = nullptr, *dWa = nullptr;
    int nRoll = 0, nWa = 0;
    size_t rollSmem = 0;
    bool useGraph = true;
    bool profiling = false;
    Timer timer;
    int runs = 0;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t graphExec = nullptr;
    // dr_prmppi_batch_step_dev: the device-input step as one graph, per (states, beliefs)
    cudaGraph_t devGraph = nullptr;
    cudaGraphExec_t devGraphExec = nullptr;
    const void* devKey[2] = {nullptr, nullptr};

    // hypothesis slots per rollout thread (dr_prmppi_batch_set_rollout_slots)
    int prSlots = DEFAULT_PR_SLOTS;

    // the slots a rollout thread may take: several only where every controller's ego
    // draws no noise (its moves are then shared by the slots) and P is a multiple
    int slotsFor(int want) const
    {
        if (envKind != 0 || want <= 1)
            return 1;
        for (auto* h : hs)
            if (h->env.action_noise_level != 0.0f || h->env.pos_noise_level != 0.0f || h->env.speed_noise_level != 0.0f || h->P % want != 0)
                return 1;
        return want;
    }

    LaunchArgs args(const Tile* tiles, int n, const PrIn* in) const
    {
        LaunchArgs a;
        a.stream = stream;
        a.pr = dDesc;
        a.prIn = in;
        a.tiles = tiles;
        a.nTiles = n;
        a.prSlots = slotsFor(prSlots);
        return a;
    }

    int launchAll(const PrIn* in, bool profile, Timer* timer)
    {
        const int n = (int)hs.size();
        if (profile)
        {
            timer->begin();
            timer->mark("prologue", stream);
        }
        CK(launchPrPrologue(args(nullptr, 0, in), n));
        if (profile)
            timer->mark("rollout", stream);
        CK(envKind ? launchGatePrRollout(args(dRoll, nRoll, in), nth, iMppi, rollSmem) : launchPrRollout(args(dRoll, nRoll, in), nopp, nth, rollSmem));
        if (profile)
            timer->mark("weighted", stream);
        CK(launchPrReduce(args(dWa, nWa, in)));
        if (profile)
            timer->mark("candidates", stream);
        CK(envKind ? launchGatePrCandidates(args(nullptr, 0, in), nth, iMppi, n, maxT) : launchPrCandidates(args(nullptr, 0, in), nopp, nth, n, maxT, 0));
        if (profile)
        {
            timer->mark("end", stream);
            timer->end();
        }
        return DR_OK;
    }

    int copyResults()
    {
        for (auto* h : hs)
            CK(cudaMemcpyAsync(h->hRes, h->desc.nom, h->desc.resBytes, cudaMemcpyDeviceToHost, stream));
        return DR_OK;
    }

    int enqueue(bool profile)
    {
        const int n = (int)hs.size();
        if (profile || !useGraph || runs == 0)
        {
            CK(cudaMemcpyAsync(dIn, hIn, sizeof(PrIn) * n, cudaMemcpyHostToDevice, stream));
            int rc = launchAll(dIn, profile, &timer);
            if (rc)
                return rc;
            rc = copyResults();
            runs++;
            return rc;
        }
        if (!graphExec)
        {
            CK(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
            cudaMemcpyAsync(dIn, hIn, sizeof(PrIn) * n, cudaMemcpyHostToDevice, stream);
            int rc = launchAll(dIn, false, nullptr);
            if (rc == DR_OK)
                rc = copyResults();
            cudaGraph_t g = nullptr;
            cudaError_t e = cudaStreamEndCapture(stream, &g);
            if (rc)
                return rc;
            CK(e);
            graph = g;
            CK(cudaGraphInstantiate(&graphExec, graph, 0));
        }
        CK(cudaGraphLaunch(graphExec, stream));
        runs++;
        return DR_OK;
    }

    template <typename St> int step(const St* states, const float* beliefs, int stride, float* actions, dr_prmppi_info* infos)
    {
        const int n = (int)hs.size();
        CK(cudaSetDevice(device));
        for (int i = 0; i < n; i++)
            hIn[i] = hs[i]->input(states[i], beliefs + (size_t)i * stride);
        bool profile = profiling;
        int rc = enqueue(profile);
        if (rc)
            return rc;
        CK(cudaStreamSynchronize(stream));
        int timeouts = 0;
        for (int i = 0; i < n; i++)
        {
            hs[i]->finish(actions + 2 * i, infos ? infos + i : nullptr);
            timeouts += hs[i]->lastTimeouts;
        }
        return timeouts ? timedOut(timeouts) : DR_OK;
    }

    // A step whose kernels gave up a bounded wait is reported, not returned as valid.
    static int timedOut(int n)
    {
        return fail(DR_ERR_TIMEOUT, "a bounded device wait gave up in " + std::to_string(n) + " CTA(s); the step's results are not valid");
    }

    // ---- sample-sharded step of a batch of one (dr_prmppi_shard_*) ----
    // Begin only enqueues work; the caller's all-gather follows on the same stream.
    DevScratch shardBuf; // merged minima and sums

    int shardWords() const
    {
        return 3 + 9 * hs[0]->T;
    }

    int shardBegin(const PrIn& hin, float* partial)
    {
        CK(cudaSetDevice(device));
        hIn[0] = hin;
        CK(cudaMemcpyAsync(dIn, hIn, sizeof(PrIn), cudaMemcpyHostToDevice, stream));
        CK(launchPrPrologue(args(nullptr, 0, dIn), 1));
        CK(launchPrRollout(args(dRoll, nRoll, dIn), nopp, nth, rollSmem));
        CK(launchPrShardMin(stream, dDesc, partial));
        CK(launchPrShardSums(stream, dDesc, dIn, hs[0]->T, partial, partial + 3));
        return DR_OK;
    }

    int shardFinish(const float* gathered, int world, float* action, dr_prmppi_info* info)
    {
        CK(cudaSetDevice(device));
        CK(shardBuf.reserve((size_t)shardWords() * sizeof(float)));
        float* mins = (float*)shardBuf.p;
        float* sums = mins + 3;
        CK(launchPrShardMerge(stream, dDesc, dIn, gathered, shardWords(), world, mins, sums));
        CK(launchPrShardApply(stream, dDesc, mins, sums));
        CK(launchPrCandidates(args(nullptr, 0, dIn), nopp, nth, 1, maxT, 0));
        int rc = copyResults();
        if (rc)
            return rc;
        CK(cudaStreamSynchronize(stream));
        hs[0]->finish(action, info);
        return hs[0]->lastTimeouts ? timedOut(hs[0]->lastTimeouts) : DR_OK;
    }

    void dropGraph()
    {
        if (graphExec)
            cudaGraphExecDestroy(graphExec);
        if (graph)
            cudaGraphDestroy(graph);
        graphExec = nullptr;
        graph = nullptr;
    }

    void dropDevGraph()
    {
        if (devGraphExec)
            cudaGraphExecDestroy(devGraphExec);
        if (devGraph)
            cudaGraphDestroy(devGraph);
        devGraphExec = nullptr;
        devGraph = nullptr;
    }

    // The step from device-resident states and beliefs (dr_prmppi_batch_step_dev): the
    // input records (filled on the host with the controllers' temperatures and step
    // counters, which this step does not advance) and the per-controller state and belief
    // copies, then the kernels; replayed from a graph unless profiling.
    int stepDev(const dr_sim_state* states, const float* beliefs)
    {
        const int n = (int)hs.size();
        CK(cudaSetDevice(device));
        std::vector<float> zero(DR_MAX_THETA, 0.0f);
        for (int i = 0; i < n; i++)
            hIn[i] = hs[i]->input(dr_sim_state{}, zero.data());
        auto body = [&](bool profile) -> int {
            CK(cudaMemcpyAsync(dIn, hIn, sizeof(PrIn) * n, cudaMemcpyHostToDevice, stream));
            for (int i = 0; i < n; i++)
            {
                CK(cudaMemcpyAsync(&dIn[i].state, states + i, sizeof(dr_sim_state), cudaMemcpyDeviceToDevice, stream));
                CK(cudaMemcpyAsync(&dIn[i].belief, beliefs + (size_t)i * DR_MAX_THETA, DR_MAX_THETA * 4, cudaMemcpyDeviceToDevice, stream));
            }
            return launchAll(dIn, profile, &timer);
        };
        if (profiling || !useGraph)
            return body(profiling);
        const void* key[2] = {states, beliefs};
        if (devGraphExec && std::memcmp(key, devKey, sizeof(key)) != 0)
            dropDevGraph();
        if (!devGraphExec)
        {
            CK(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
            int rc = body(false);
            cudaGraph_t g = nullptr;
            cudaError_t e = cudaStreamEndCapture(stream, &g);
            if (rc)
                return rc;
            CK(e);
            devGraph = g;
            CK(cudaGraphInstantiate(&devGraphExec, devGraph, 0));
            std::memcpy(devKey, key, sizeof(key));
        }
        CK(cudaGraphLaunch(devGraphExec, stream));
        return DR_OK;
    }

    void release()
    {
        dropDevGraph();
        shardBuf.release();
        if (graphExec)
            cudaGraphExecDestroy(graphExec);
        if (graph)
            cudaGraphDestroy(graph);
        graphExec = nullptr;
        graph = nullptr;
        cudaFree(dDesc);
        cudaFree(dIn);
        cudaFree(dRoll);
        cudaFree(dWa);
        if (hIn)
            cudaFreeHost(hIn);
        if (ownStream && stream)
            cudaStreamDestroy(stream);
    }
};

namespace
{

int buildPrBatch(dr_prmppi* const* hs, int n, cudaStream_t stream, bool ownStream, dr_prmppi_batch** out)
{
    if (n <= 0 || !hs)
        return fail(DR_ERR_INVALID_ARG, "empty batch");
    auto b = std::make_unique<dr_prmppi_batch>();
    b->hs.assign(hs, hs + n);
    b->device = hs[0]->device;
    b->nopp = hs[0]->nopp;
    b->nth = hs[0]->nth;
    b->envKind = hs[0]->envKind;
    b->iMppi = hs[0]->iMppi;
    for (int i = 0; i < n; i++)
        if (!hs[i] || hs[i]->device != b->device || hs[i]->nopp != b->nopp || hs[i]->nth != b->nth || hs[i]->envKind != b->envKind ||
            hs[i]->iMppi != b->iMppi)
            return fail(DR_ERR_INVALID_ARG, "a batch needs controllers on one device with equal environment kind, ego index, n_opp and n_theta");
    CK(cudaSetDevice(b->device));
    b->stream = stream;
    b->ownStream = ownStream;
    std::vector<PrDev> descs;
    std::vector<Tile> roll, wa;
    for (int i = 0; i < n; i++)
    {
        dr_prmppi* h = hs[i];
        descs.push_back(h->desc);
        const int spb = (h->envKind ? gatePrRolloutSamplesPerBlock() : prRolloutSamplesPerBlock()) / h->P;
        for (int nr = 0; nr < 2; nr++)
            for (int s0 = h->sLo; s0 < h->sHi; s0 += spb)
                roll.push_back(Tile{i, s0, std::min(spb, h->sHi - s0), nr});
        for (int w = 0; w < 3 * h->T; w++)
            wa.push_back(Tile{i, w, 0, 0});
        b->maxT = std::max(b->maxT, h->T);
        b->maxP = std::max(b->maxP, h->P);
        b->rollSmem = std::max(b->rollSmem, h->envKind ? gatePrRolloutSmem(h->T) : prRolloutSmem(h->T));
    }
    b->nRoll = (int)roll.size();
    b->nWa = (int)wa.size();
    CK(cudaMalloc(&b->dDesc, sizeof(PrDev) * n));
    CK(cudaMemcpy(b->dDesc, descs.data(), sizeof(PrDev) * n, cudaMemcpyHostToDevice));
    CK(cudaMalloc(&b->dIn, sizeof(PrIn) * n));
    CK(cudaMallocHost(&b->hIn, sizeof(PrIn) * n));
    CK(cudaMalloc(&b->dRoll, sizeof(Tile) * roll.size()));
    CK(cudaMemcpy(b->dRoll, roll.data(), sizeof(Tile) * roll.size(), cudaMemcpyHostToDevice));
    CK(cudaMalloc(&b->dWa, sizeof(Tile) * wa.size()));
    CK(cudaMemcpy(b->dWa, wa.data(), sizeof(Tile) * wa.size(), cudaMemcpyHostToDevice));
    *out = b.release();
    return DR_OK;
}

} // namespace

extern "C" {

// one of env (strategic race) / genv (gate race) is given
static int prCreate(const dr_env_config* env, const dr_gate_env_config* genv, const dr_prmppi_config* cfg, uint64_t seed, const float* nominal, int device,
                    void* stream, dr_prmppi** out)
{
    if (!out)
        return fail(DR_ERR_INVALID_ARG, "out is NULL");
    *out = nullptr;
    int rc = env ? checkEnv(env) : checkGateEnv(genv);
    if (rc)
        return rc;
    if (!cfg)
        return fail(DR_ERR_INVALID_ARG, "cfg is NULL");
    if (cfg->n_samples < 1 || cfg->n_samples > (1 << 22))
        return fail(DR_ERR_INVALID_ARG, "n_samples must be in [1, 2^22]");
    if (cfg->n_timesteps < 2 || cfg->n_timesteps > DR_MAX_T)
        return fail(DR_ERR_INVALID_ARG, "n_timesteps must be in [2, 256]");
    if (cfg->P < 1 || cfg->P > 32)
        return fail(DR_ERR_INVALID_ARG, "P must be in [1, 32]");
    for (int i = 0; i < 3; i++)
        if (!(cfg->inv_temperature > 0.0f))
            return fail(DR_ERR_INVALID_ARG, "inv_temperature must be positive");
    if (env ? !prSupported(env->n_opp, env->n_theta) : !gateSupported(genv->n_theta))
        return fail(DR_ERR_UNSUPPORTED, "(n_opp, n_theta) combination not compiled in");
    rc = selectDevice(device);
    if (rc)
        return rc;
    auto h = std::make_unique<dr_prmppi>();
    h->device = device;
    if (env)
    {
        h->env = *env;
        h->env.p_grid = h->env.dp_grid = h->env.t_grid = h->env.kappa_grid = nullptr;
    }
    else
    {
        h->envKind = 1;
        h->iMppi = genv->i_mppi;
    }
    h->cfg = *cfg;
    if (h->cfg.min_nu == 0.0f && h->cfg.max_nu == 0.0f)
    {
        h->cfg.min_nu = 0.0005f; // controllers.h:135-136
        h->cfg.max_nu = 0.001f;
    }
    h->seed = seed;
    h->nth = env ? env->n_theta : genv->n_theta;
    h->nopp = env ? env->n_opp : 1;
    h->K = cfg->n_samples;
    h->T = cfg->n_timesteps;
    h->P = cfg->P;
    for (int i = 0; i < 3; i++)
        h->lambda[i] = cfg->inv_temperature; // prmppi_controller.cu:39
    const int K = h->K, T = h->T, P = h->P;
    PrDev& D = h->desc;
    if (env)
        D.env = toEnvParams(*env);
    D.cfg.gateMargin = cfg->gate_traversal_margin;
    D.cfg.K = K;
    D.cfg.T = T;
    D.cfg.P = P;
    D.cfg.nth = h->nth;
    D.cfg.nopp = h->nopp;
    float s0 = cfg->sampling_noise_dim[0], s1 = cfg->sampling_noise_dim[1];
    if (s0 == 0.0f && s1 == 0.0f)
        s0 = s1 = cfg->sampling_noise;
    D.cfg.sigma0 = s0;
    D.cfg.sigma1 = s1;
    D.cfg.collDistFactor = cfg->coll_dist_factor;
    D.cfg.boundaryCost = cfg->boundary_cost;
    D.cfg.boundaryThresholdFactor = cfg->boundary_threshold_factor;
    D.cfg.winCost = cfg->win_cost;
    D.cfg.oppWinCost = cfg->opp_win_cost;
    D.cfg.finalAdvWeight = cfg->final_adv_weight;
    D.cfg.finalOppAdvWeight = cfg->final_opp_adv_weight;
    D.cfg.safetyWeight = cfg->safety_weight;
    D.cfg.k0 = (uint32_t)seed;
    D.cfg.k1 = (uint32_t)(seed >> 32);
    h->sLo = 0;
    h->sHi = K;
    D.cfg.sLo = 0;
    D.cfg.sHi = K;

    float *grids = nullptr, *costNom, *costRob, *avg, *robWork, *gtrack = nullptr;
    GateParams* gp = nullptr;
    unsigned* counter;
    Arena& A = h->arena;
    if (env)
        A.add(grids, GRID_FLOATS * 4);
    else
    {
        A.add(gp, sizeof(GateParams));
        A.add(gtrack, GATE_TRACK_FLOATS * 4);
    }
    A.add(costNom, (size_t)P * K * 2 * 4);
    A.add(costRob, (size_t)P * K * 2 * 4);
    A.add(avg, (size_t)2 * K * 2 * 4);
    A.add(robWork, a16((size_t)T * 2 * 4));
    A.add(counter, 16);
    const size_t tb = a16((size_t)T * 2 * 4);
    size_t oNom = 0, oRob = tb, oC1 = 2 * tb, oC2 = 3 * tb, oMin = 4 * tb, oNu = oMin + 16, oFull = oNu + 16, oSafe = oFull + a16((size_t)2 * P * 4),
           oTh = oSafe + a16((size_t)2 * P * 4), oDec = oTh + a16((size_t)P * 4), oStats = oDec + 16, resBytes = oStats + 16;
    unsigned char* res;
    A.add(res, resBytes);
    CK(A.alloc());
    D.grids = grids;
    D.gate = gp;
    D.gtrack = gtrack;
    D.costNom = costNom;
    D.costRob = costRob;
    D.avg = avg;
    D.robWork = robWork;
    D.nomWork = nullptr;
    D.counter = counter;
    D.nom = (float*)(res + oNom);
    D.rob = (float*)(res + oRob);
    D.cand1 = (float*)(res + oC1);
    D.cand2 = (float*)(res + oC2);
    D.minCosts = (float*)(res + oMin);
    D.nu = (float*)(res + oNu);
    D.candFull = (float*)(res + oFull);
    D.candSafe = (float*)(res + oSafe);
    D.thetas = (int*)(res + oTh);
    D.decision = (int*)(res + oDec);
    D.stats = (int*)(res + oStats);
    D.resBytes = resBytes;
    if (env)
    {
        std::vector<float> g = packGrids(*env);
        CK(cudaMemcpy(grids, g.data(), g.size() * 4, cudaMemcpyHostToDevice));
    }
    else
    {
        GateParams hp = toGateParams(*genv);
        CK(cudaMemcpy(gp, &hp, sizeof(GateParams), cudaMemcpyHostToDevice));
        std::vector<float> t = packGateTrack(*genv);
        CK(cudaMemcpy(gtrack, t.data(), t.size() * 4, cudaMemcpyHostToDevice));
    }
    h->hNom.assign((size_t)T * 2, 0.0f);
    if (nominal)
        std::memcpy(h->hNom.data(), nominal, h->hNom.size() * 4);
    h->hRob = h->hNom;
    CK(cudaMemcpy(D.nom, h->hNom.data(), h->hNom.size() * 4, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(D.rob, h->hRob.data(), h->hRob.size() * 4, cudaMemcpyHostToDevice));
    CK(cudaMallocHost(&h->hRes, resBytes));
    cudaStream_t s = (cudaStream_t)stream;
    bool own = false;
    if (!s)
    {
        CK(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
        own = true;
    }
    h->stream = s;
    h->ownStream = own;
    dr_prmppi* raw = h.get();
    rc = buildPrBatch(&raw, 1, s, false, &h->self);
    if (rc)
        return rc;
    *out = h.release();
    return DR_OK;
}

int dr_prmppi_create(const dr_env_config* env, const dr_prmppi_config* cfg, uint64_t seed, const float* nominal, int device, void* stream,
                     dr_prmppi** out)
{
    if (!env)
        return fail(DR_ERR_INVALID_ARG, "env is NULL");
    return prCreate(env, nullptr, cfg, seed, nominal, device, stream, out);
}

int dr_gate_prmppi_create(const dr_gate_env_config* env, const dr_prmppi_config* cfg, uint64_t seed, const float* nominal, int device, void* stream,
                          dr_prmppi** out)
{
    if (!env)
        return fail(DR_ERR_INVALID_ARG, "env is NULL");
    return prCreate(nullptr, env, cfg, seed, nominal, device, stream, out);
}

int dr_prmppi_destroy(dr_prmppi* h)
{
    if (!h)
        return DR_OK;
    cudaSetDevice(h->device);
    if (h->stream)
        cudaStreamSynchronize(h->stream);
    if (h->self)
    {
        h->self->release();
        delete h->self;
    }
    h->predBuf.release();
    h->arena.release();
    if (h->hRes)
        cudaFreeHost(h->hRes);
    if (h->ownStream && h->stream)
        cudaStreamDestroy(h->stream);
    delete h;
    return DR_OK;
}

int dr_prmppi_predict(dr_prmppi* h, const dr_sim_state* prev_state, float* positions, float* actions, int32_t* records, float* costs)
{
    if (!h || !prev_state || !positions || !actions || !records || !costs)
        return fail(DR_ERR_INVALID_ARG, "NULL argument");
    if (h->envKind != 0)
        return fail(DR_ERR_UNSUPPORTED, "predictions are built for the strategic race");
    CK(cudaSetDevice(h->device));
    const int rows = h->nth + 1, T = h->T, na = h->nopp + 1;
    const size_t nPos = (size_t)rows * T * 2 * na, nAct = (size_t)rows * T * 2, nRec = (size_t)rows * PREDICT_RECORD;
    const size_t oSt = 0, oPos = a256(sizeof(dr_sim_state)), oAct = oPos + a256(nPos * 4), oRec = oAct + a256(nAct * 4),
                 oCost = oRec + a256(nRec * 4), total = oCost + a256((size_t)rows * 4);
    CK(h->predBuf.reserve(total));
    unsigned char* base = (unsigned char*)h->predBuf.p;
    CK(cudaMemcpyAsync(base + oSt, prev_state, sizeof(dr_sim_state), cudaMemcpyHostToDevice, h->stream));
    PredictOut out{(float*)(base + oPos), (float*)(base + oAct), (int*)(base + oRec), (float*)(base + oCost), T};
    CK(launchPrPredict(h->stream, h->nopp, h->nth, h->self->dDesc, (const dr_sim_state*)(base + oSt), out, 1));
    CK(cudaMemcpyAsync(positions, base + oPos, nPos * 4, cudaMemcpyDeviceToHost, h->stream));
    CK(cudaMemcpyAsync(actions, base + oAct, nAct * 4, cudaMemcpyDeviceToHost, h->stream));
    CK(cudaMemcpyAsync(records, base + oRec, nRec * 4, cudaMemcpyDeviceToHost, h->stream));
    CK(cudaMemcpyAsync(costs, base + oCost, (size_t)rows * 4, cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    return DR_OK;
}

int dr_prmppi_step(dr_prmppi* h, const dr_sim_state* state, const float* belief, float* out_action, dr_prmppi_info* info)
{
    if (!h || !state || !belief || !out_action)
        return fail(DR_ERR_INVALID_ARG, "NULL argument");
    if (h->shardWorld > 1)
        return fail(DR_ERR_STATE, "a sharded controller steps through dr_prmppi_shard_*");
    if (h->envKind != 0)
        return fail(DR_ERR_INVALID_ARG, "a gate-race controller steps through dr_gate_prmppi_step");
    return h->self->step(state, belief, h->nth, out_action, info);
}

int dr_gate_prmppi_step(dr_prmppi* h, const dr_gate_state* state, const float* belief, float* out_action, dr_prmppi_info* info)
{
    if (!h || !state || !belief || !out_action)
        return fail(DR_ERR_INVALID_ARG, "NULL argument");
    if (h->envKind != 1)
        return fail(DR_ERR_INVALID_ARG, "a strategic-race controller steps through dr_prmppi_step");
    return h->self->step(state, belief, h->nth, out_action, info);
}

int dr_prmppi_set_shard(dr_prmppi* h, int rank, int world)
{
    if (!h)
        return fail(DR_ERR_INVALID_ARG, "NULL handle");
    if (h->envKind != 0)
        return fail(DR_ERR_UNSUPPORTED, "sample sharding is built for the strategic race");
    if (world < 1 || rank < 0 || rank >= world || world > h->K)
        return fail(DR_ERR_INVALID_ARG, "need 0 <= rank < world <= n_samples");
    h->shardWorld = world;
    h->sLo = (int)((int64_t)h->K * rank / world);
    h->sHi = (int)((int64_t)h->K * (rank + 1) / world);
    h->desc.cfg.sLo = h->sLo;
    h->desc.cfg.sHi = h->sHi;
    CK(cudaSetDevice(h->device));
    CK(cudaStreamSynchronize(h->stream));
    if (h->self)
    {
        h->self->release();
        delete h->self;
        h->self = nullptr;
    }
    dr_prmppi* raw = h;
    return buildPrBatch(&raw, 1, h->stream, false, &h->self);
}

int dr_prmppi_shard_words(const dr_prmppi* h, size_t* words)
{
    if (!h || !words)
        return fail(DR_ERR_INVALID_ARG, "NULL argument");
    *words = (size_t)h->self->shardWords();
    return DR_OK;
}

int dr_prmppi_shard_begin(dr_prmppi* h, const dr_sim_state* state, const float* belief, float* partial_dev)
{
    if (!h || !state || !belief || !partial_dev)
        return fail(DR_ERR_INVALID_ARG, "NULL argument");
    return h->self->shardBegin(h->input(*state, belief), partial_dev);
}

int dr_prmppi_shard_finish(dr_prmppi* h, const float* gathered_dev, int world, float* out_action, dr_prmppi_info* info)
{
    if (!h || !gathered_dev || !out_action)
        return fail(DR_ERR_INVALID_ARG, "NULL argument");
    if (world != h->shardWorld)
        return fail(DR_ERR_INVALID_ARG, "world differs from dr_prmppi_set_shard's");
    return h->self->shardFinish(gathered_dev, world, out_action, info);
}

int dr_prmppi_get_nominals(const dr_prmppi* h, float* nom, float* rob, size_t n)
{
    if (!h || n < h->hNom.size())
        return fail(DR_ERR_INVALID_ARG, "output too small");
    if (nom)
        std::memcpy(nom, h->hNom.data(), h->hNom.size() * 4);
    if (rob)
        std::memcpy(rob, h->hRob.data(), h->hRob.size() * 4);
    return DR_OK;
}

uint64_t dr_prmppi_get_step(const dr_prmppi* h)
{
    return h ? h->step : 0;
}

int dr_prmppi_io_bytes(const dr_prmppi* h, size_t* h2d, size_t* d2h)
{
    if (!h)
        return fail(DR_ERR_INVALID_ARG, "NULL handle");
    if (h2d)
        *h2d = sizeof(PrIn);
    if (d2h)
        *d2h = h->desc.resBytes;
    return DR_OK;
}

int dr_prmppi_set_step(dr_prmppi* h, uint64_t step)
{
    if (!h)
        return fail(DR_ERR_INVALID_ARG, "NULL handle");
    h->step = step;
    return DR_OK;
}

int dr_prmppi_set_profiling(dr_prmppi* h, int on)
{
    if (!h)
        return fail(DR_ERR_INVALID_ARG, "NULL handle");
    h->self->profiling = on != 0;
    h->self->timer.reset();
    return DR_OK;
}

int dr_prmppi_get_kernel_times(dr_prmppi* h, const char** names, float* ms, int n, int* count)
{
    if (!h)
        return fail(DR_ERR_INVALID_ARG, "NULL handle");
    return kernelTimes(h->self->timer, names, ms, n, count);
}

int dr_prmppi_batch_create(dr_prmppi* const* hs, int n, void* stream, dr_prmppi_batch** out)
{
    if (!out)
        return fail(DR_ERR_INVALID_ARG, "out is NULL");
    *out = nullptr;
    if (n <= 0 || !hs || !hs[0])
        return fail(DR_ERR_INVALID_ARG, "empty batch");
    CK(cudaSetDevice(hs[0]->device));
    cudaStream_t s = (cudaStream_t)stream;
    bool own = false;
    if (!s)
    {
        CK(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
        own = true;
    }
    return buildPrBatch(hs, n, s, own, out);
}

int dr_prmppi_batch_destroy(dr_prmppi_batch* b)
{
    if (!b)
        return DR_OK;
    cudaSetDevice(b->device);
    cudaStreamSynchronize(b->stream);
    b->release();
    delete b;
    return DR_OK;
}

int dr_prmppi_batch_step(dr_prmppi_batch* b, const dr_sim_state* states, const float* beliefs, float* out_actions, dr_prmppi_info* infos)
{
    if (!b || !states || !beliefs || !out_actions)
        return fail(DR_ERR_INVALID_ARG, "NULL argument");
    return b->step(states, beliefs, DR_MAX_THETA, out_actions, infos);
}

int dr_prmppi_batch_step_dev(dr_prmppi_batch* b, const dr_sim_state* states_dev, const float* beliefs_dev)
{
    if (!b || !states_dev || !beliefs_dev)
        return fail(DR_ERR_INVALID_ARG, "NULL argument");
    return b->stepDev(states_dev, beliefs_dev);
}

int dr_prmppi_debug_noise(dr_prmppi* h, const float* belief, float* noise, size_t n, int32_t* thetas)
{
    size_t need = (size_t)h->T * h->K * 2;
    if (!h || !belief || (noise && n < need))
        return fail(DR_ERR_INVALID_ARG, "bad argument");
    CK(cudaSetDevice(h->device));
    dr_prmppi_batch* b = h->self;
    b->hIn[0] = h->input(dr_sim_state{}, belief);
    CK(cudaMemcpyAsync(b->dIn, b->hIn, sizeof(PrIn), cudaMemcpyHostToDevice, h->stream));
    if (noise)
    {
        float* d = nullptr;
        CK(cudaMalloc(&d, need * 4));
        cudaError_t e = launchPrNoise(b->args(nullptr, 0, b->dIn), need / 2, d);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(noise, d, need * 4, cudaMemcpyDeviceToHost, h->stream);
        if (e == cudaSuccess)
            e = cudaStreamSynchronize(h->stream);
        cudaFree(d);
        CK(e);
    }
    if (thetas)
    {
        // theta draw of the prologue, on a scratch copy of the nominals
        std::vector<float> nom(h->hNom.size()), rob(h->hRob.size());
        CK(cudaMemcpyAsync(nom.data(), h->desc.nom, nom.size() * 4, cudaMemcpyDeviceToHost, h->stream));
        CK(cudaMemcpyAsync(rob.data(), h->desc.rob, rob.size() * 4, cudaMemcpyDeviceToHost, h->stream));
        CK(launchPrPrologue(b->args(nullptr, 0, b->dIn), 1));
        CK(cudaMemcpyAsync(thetas, h->desc.thetas, h->P * 4, cudaMemcpyDeviceToHost, h->stream));
        CK(cudaStreamSynchronize(h->stream));
        CK(cudaMemcpy(h->desc.nom, nom.data(), nom.size() * 4, cudaMemcpyHostToDevice));
        CK(cudaMemcpy(h->desc.rob, rob.data(), rob.size() * 4, cudaMemcpyHostToDevice));
    }
    return DR_OK;
}

} // extern "C"

template <typename St> static int prDebugRollout(dr_prmppi* h, const St* state, const float* belief, float* cost_nom, float* cost_rob)
{
    if (!h || !state || !belief)
        return fail(DR_ERR_INVALID_ARG, "NULL argument");
    if (h->envKind != (std::is_same<St, dr_gate_state>::value ? 1 : 0))
        return fail(DR_ERR_INVALID_ARG, "state type does not match the controller's environment");
    CK(cudaSetDevice(h->device));
    dr_prmppi_batch* b = h->self;
    std::vector<float> nom(h->hNom.size()), rob(h->hRob.size());
    CK(cudaMemcpyAsync(nom.data(), h->desc.nom, nom.size() * 4, cudaMemcpyDeviceToHost, h->stream));
    CK(cudaMemcpyAsync(rob.data(), h->desc.rob, rob.size() * 4, cudaMemcpyDeviceToHost, h->stream));
    b->hIn[0] = h->input(*state, belief);
    CK(cudaMemcpyAsync(b->dIn, b->hIn, sizeof(PrIn), cudaMemcpyHostToDevice, h->stream));
    CK(launchPrPrologue(b->args(nullptr, 0, b->dIn), 1));
    CK(h->envKind ? launchGatePrRollout(b->args(b->dRoll, b->nRoll, b->dIn), h->nth, h->iMppi, b->rollSmem)
                  : launchPrRollout(b->args(b->dRoll, b->nRoll, b->dIn), h->nopp, h->nth, b->rollSmem));
    size_t nb = (size_t)h->P * h->K * 2 * 4;
    if (cost_nom)
        CK(cudaMemcpyAsync(cost_nom, h->desc.costNom, nb, cudaMemcpyDeviceToHost, h->stream));
    if (cost_rob)
        CK(cudaMemcpyAsync(cost_rob, h->desc.costRob, nb, cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    // restore the unshifted nominals: the next step shifts them itself
    CK(cudaMemcpy(h->desc.nom, nom.data(), nom.size() * 4, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(h->desc.rob, rob.data(), rob.size() * 4, cudaMemcpyHostToDevice));
    return DR_OK;
}

extern "C" {

int dr_prmppi_debug_rollout(dr_prmppi* h, const dr_sim_state* state, const float* belief, float* cost_nom, float* cost_rob)
{
    return prDebugRollout(h, state, belief, cost_nom, cost_rob);
}

int dr_gate_prmppi_debug_rollout(dr_prmppi* h, const dr_gate_state* state, const float* belief, float* cost_nom, float* cost_rob)
{
    return prDebugRollout(h, state, belief, cost_nom, cost_rob);
}

} // extern "C"

// ---- device environment step -------------------------------------------------------------------

template <int NOPP, int NTH>
__global__ void env_step_kernel(EnvParams Eh, const float* __restrict__ grids, int trueTheta, float a0, float a1, dr_sim_state* st, float* belief,
                                int updateBelief, uint32_t k0, uint32_t k1, uint32_t step, int* term)
{
    __shared__ float sg[GRID_FLOATS];
    __shared__ EnvParams sE;
    for (int i = threadIdx.x; i < GRID_FLOATS; i += blockDim.x)
        sg[i] = grids[i];
    if (threadIdx.x == 0)
    {
        sE = Eh;
        envDeviceTerms(sE, Eh, 0, 1);
    }
    __syncthreads();
    const EnvParams& E = sE;
    if (threadIdx.x != 0)
        return;
    constexpr int NA = NOPP + 1;
    DState<NA> s;
    for (int a = 0; a < NA; a++)
    {
        s.pos[2 * a] = st->pos[2 * a];
        s.pos[2 * a + 1] = st->pos[2 * a + 1];
        s.vel[2 * a] = st->vel[2 * a];
        s.vel[2 * a + 1] = st->vel[2 * a + 1];
        s.S[a] = st->S[a];
        s.lat[a] = st->lat_dist[a];
        s.laps[a] = st->laps[a];
    }
    s.locate(E.trackLength);
    BState<NTH> bs;
    for (int i = 0; i < NTH; i++)
        bs.belief[i] = belief[i];
    bs.predTheta = 0;
    bs.branchingTime = -1;
    const Track tr = trackIn(sg);
    EnvNoise rng(k0, k1, 0u, 0u, step, S_ENV_STEP);
    rng.begin_step(0);
    bool branched = false;
    StepOut o;
    if (updateBelief)
        o = envStep<NOPP, NTH, true, false, false, true>(0, trueTheta, tr, E, a0, a1, s, bs, branched, 2.0f, rng);
    else
        o = envStep<NOPP, NTH, false, false, false, false>(0, trueTheta, tr, E, a0, a1, s, bs, branched, 2.0f, rng);
    for (int a = 0; a < NA; a++)
    {
        st->pos[2 * a] = s.pos[2 * a];
        st->pos[2 * a + 1] = s.pos[2 * a + 1];
        st->vel[2 * a] = s.vel[2 * a];
        st->vel[2 * a + 1] = s.vel[2 * a + 1];
        st->S[a] = s.S[a];
        st->lat_dist[a] = s.lat[a];
        st->laps[a] = s.laps[a];
    }
    for (int i = 0; i < NTH; i++)
        belief[i] = bs.belief[i];
    *term = o.term;
}

namespace
{
// Device scratch of the single environment steps (dr_env_step, dr_gate_env_step): one
// block per device, allocated on first use and kept for the process; the calls of a
// process share it under a mutex (each call is synchronous).
// Layout: [parameters / grids / racelines] | [state record | belief | terminal type].
constexpr size_t ENV_SCRATCH_PARAMS = 48 * 1024, ENV_SCRATCH_IO = 1024;
std::mutex g_envMu;
std::map<int, unsigned char*> g_envScratch;

cudaError_t envScratch(int dev, unsigned char** out)
{
    auto it = g_envScratch.find(dev);
    if (it != g_envScratch.end())
    {
        *out = it->second;
        return cudaSuccess;
    }
    unsigned char* p = nullptr;
    cudaError_t e = cudaMalloc(&p, ENV_SCRATCH_PARAMS + ENV_SCRATCH_IO);
    if (e == cudaSuccess)
        g_envScratch[dev] = p;
    *out = p;
    return e;
}

// host image of the io part: state record, belief, terminal type
template <class St> struct EnvIo
{
    St state;
    float belief[DR_MAX_THETA];
    int term;
};
static_assert(sizeof(EnvIo<dr_sim_state>) <= ENV_SCRATCH_IO && sizeof(EnvIo<dr_gate_state>) <= ENV_SCRATCH_IO, "env step scratch");
} // namespace

extern "C" int dr_env_step(const dr_env_config* env, int true_theta, const float* action, dr_sim_state* state, float* belief, int update_belief,
                           uint64_t seed, uint64_t step, int* term)
{
    int rc = checkEnv(env);
    if (rc)
        return rc;
    if (!action || !state || !belief || true_theta < 0 || true_theta >= env->n_theta)
        return fail(DR_ERR_INVALID_ARG, "bad argument");
    if (!prSupported(env->n_opp, env->n_theta))
        return fail(DR_ERR_UNSUPPORTED, "(n_opp, n_theta) combination not compiled in");
    int dev = 0;
    CK(cudaGetDevice(&dev));
    std::vector<float> g = packGrids(*env);
    EnvParams E = toEnvParams(*env);
    std::lock_guard<std::mutex> lock(g_envMu);
    unsigned char* base = nullptr;
    CK(envScratch(dev, &base));
    float* dg = (float*)base;
    EnvIo<dr_sim_state>* dio = (EnvIo<dr_sim_state>*)(base + ENV_SCRATCH_PARAMS);
    EnvIo<dr_sim_state> io{};
    io.state = *state;
    for (int i = 0; i < env->n_theta; i++)
        io.belief[i] = belief[i];
    CK(cudaMemcpy(dg, g.data(), GRID_FLOATS * 4, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(dio, &io, sizeof(io), cudaMemcpyHostToDevice));
    uint32_t k0 = (uint32_t)seed, k1 = (uint32_t)(seed >> 32);
    switch (env->n_opp * 16 + env->n_theta)
    {
    case 17: env_step_kernel<1, 1><<<1, 128>>>(E, dg, true_theta, action[0], action[1], &dio->state, dio->belief, update_belief, k0, k1, (uint32_t)step, &dio->term); break;
    case 18: env_step_kernel<1, 2><<<1, 128>>>(E, dg, true_theta, action[0], action[1], &dio->state, dio->belief, update_belief, k0, k1, (uint32_t)step, &dio->term); break;
    case 20: env_step_kernel<1, 4><<<1, 128>>>(E, dg, true_theta, action[0], action[1], &dio->state, dio->belief, update_belief, k0, k1, (uint32_t)step, &dio->term); break;
    case 24: env_step_kernel<1, 8><<<1, 128>>>(E, dg, true_theta, action[0], action[1], &dio->state, dio->belief, update_belief, k0, k1, (uint32_t)step, &dio->term); break;
    case 34: env_step_kernel<2, 2><<<1, 128>>>(E, dg, true_theta, action[0], action[1], &dio->state, dio->belief, update_belief, k0, k1, (uint32_t)step, &dio->term); break;
    default: break;
    }
    CK(cudaGetLastError());
    CK(cudaMemcpy(&io, dio, sizeof(io), cudaMemcpyDeviceToHost));
    *state = io.state;
    for (int i = 0; i < env->n_theta; i++)
        belief[i] = io.belief[i];
    if (term)
        *term = io.term;
    return DR_OK;
}

// Test hook kernel of dr_debug_project: one point per thread.
template <int MODE>
__global__ void __launch_bounds__(256) debug_project_kernel(const float* __restrict__ grids, float L, float invL, const float* __restrict__ xy,
                                                            const float* __restrict__ prevS, int n, float* __restrict__ outS, float* __restrict__ outLat,
                                                            int* __restrict__ outIdx)
{
    __shared__ __align__(16) float sg[GRID_FLOATS];
    for (int i = threadIdx.x; i < GRID_FLOATS; i += blockDim.x)
        sg[i] = grids[i];
    __syncthreads();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    const Track tr = trackIn(sg);
    float lat = 0.0f;
    TrackPos tp{0, 0.0f};
    float S;
    if constexpr (MODE == 0)
        S = projectOnTrack<true, true>(tr, L, invL, xy[2 * i], xy[2 * i + 1], prevS[i], lat, tp);
    else if constexpr (MODE == 1)
        S = projectOnTrack<true, false>(tr, L, invL, xy[2 * i], xy[2 * i + 1], prevS[i], lat, tp);
    else if constexpr (MODE == 2)
        S = projectOnTrack<false, true>(tr, L, invL, xy[2 * i], xy[2 * i + 1], prevS[i], lat, tp);
    else
        S = projectOnTrack<false, false>(tr, L, invL, xy[2 * i], xy[2 * i + 1], prevS[i], lat, tp);
    outS[i] = S;
    outLat[i] = lat;
    outIdx[i] = tp.i0;
}

extern "C" int dr_debug_project(const dr_env_config* env, const float* xy, const float* prev_s, int n, int mode, float* s_out, float* lat_out,
                                int32_t* idx_out)
{
    int rc = checkEnv(env);
    if (rc)
        return rc;
    if (n < 0 || mode < 0 || mode > 3 || (n > 0 && (!xy || !prev_s || !s_out || !lat_out || !idx_out)))
        return fail(DR_ERR_INVALID_ARG, "bad argument");
    if (n == 0)
        return DR_OK;
    const std::vector<float> g = packGrids(*env);
    const float L = env->track_length, invL = 1.0f / env->track_length;
    float *dg = nullptr, *dxy = nullptr, *dps = nullptr, *dS = nullptr, *dLat = nullptr;
    int* dIdx = nullptr;
    auto release = [&]() {
        cudaFree(dg);
        cudaFree(dxy);
        cudaFree(dps);
        cudaFree(dS);
        cudaFree(dLat);
        cudaFree(dIdx);
    };
    const size_t nb = (size_t)n * 4;
    cudaError_t e = cudaSuccess;
    for (auto [ptr, bytes] : {std::pair<void**, size_t>{(void**)&dg, GRID_FLOATS * 4}, {(void**)&dxy, 2 * nb}, {(void**)&dps, nb}, {(void**)&dS, nb},
                              {(void**)&dLat, nb}, {(void**)&dIdx, nb}})
        if (e == cudaSuccess)
            e = cudaMalloc(ptr, bytes);
    if (e == cudaSuccess)
        e = cudaMemcpy(dg, g.data(), GRID_FLOATS * 4, cudaMemcpyHostToDevice);
    if (e == cudaSuccess)
        e = cudaMemcpy(dxy, xy, 2 * nb, cudaMemcpyHostToDevice);
    if (e == cudaSuccess)
        e = cudaMemcpy(dps, prev_s, nb, cudaMemcpyHostToDevice);
    if (e == cudaSuccess)
    {
        const int blocks = (n + 255) / 256;
        if (mode == 0)
            debug_project_kernel<0><<<blocks, 256>>>(dg, L, invL, dxy, dps, n, dS, dLat, dIdx);
        else if (mode == 1)
            debug_project_kernel<1><<<blocks, 256>>>(dg, L, invL, dxy, dps, n, dS, dLat, dIdx);
        else if (mode == 2)
            debug_project_kernel<2><<<blocks, 256>>>(dg, L, invL, dxy, dps, n, dS, dLat, dIdx);
        else
            debug_project_kernel<3><<<blocks, 256>>>(dg, L, invL, dxy, dps, n, dS, dLat, dIdx);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess)
        e = cudaMemcpy(s_out, dS, nb, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess)
        e = cudaMemcpy(lat_out, dLat, nb, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess)
        e = cudaMemcpy(idx_out, dIdx, nb, cudaMemcpyDeviceToHost);
    release();
    if (e != cudaSuccess)
        return fail(DR_ERR_CUDA, std::string("dr_debug_project: ") + cudaGetErrorString(e));
    return DR_OK;
}

extern "C" int dr_projection_certificate(const float* p_grid, float* cert)
{
    if (!p_grid || !cert)
        return fail(DR_ERR_INVALID_ARG, "NULL argument");
    for (int i = 0; i < 2 * NTS; i++)
        if (!std::isfinite(p_grid[i]))
            return fail(DR_ERR_INVALID_ARG, "track grids must be finite");
    for (int c = 0; c < NTS; c++)
        cert[c] = projectionCertificate(p_grid, c);
    return DR_OK;
}

extern "C" int dr_track_grids(const double* q, int n_tracks, float* p_grid, float* dp_grid, float* t_grid, float* kappa_grid, float* track_length)
{
    if (!q || n_tracks < 1 || !p_grid || !dp_grid || !t_grid || !kappa_grid || !track_length)
        return fail(DR_ERR_INVALID_ARG, "bad argument");
    for (size_t i = 0; i < (size_t)n_tracks * DR_N_TRACK_SAMPLES * 2; i++)
        if (!std::isfinite(q[i]))
            return fail(DR_ERR_INVALID_ARG, "track samples must be finite");
    // the spline parameter (cumulative chord length) must increase strictly, as scipy's
    // CubicSpline requires of the reference's knots
    for (int r = 0; r < n_tracks; r++)
        for (int k = 0; k < DR_N_TRACK_SAMPLES; k++)
        {
            const double* a = q + ((size_t)r * DR_N_TRACK_SAMPLES + k) * 2;
            const double* b = q + ((size_t)r * DR_N_TRACK_SAMPLES + (k + 1) % DR_N_TRACK_SAMPLES) * 2;
            if (a[0] == b[0] && a[1] == b[1])
                return fail(DR_ERR_INVALID_ARG, "consecutive track samples must differ");
        }
    const int NS = DR_N_TRACK_SAMPLES;
    const size_t perTrack = (size_t)NS * 7;
    double* dq = nullptr;
    float* dout = nullptr;
    float* dlen = nullptr;
    cudaError_t e = cudaMalloc(&dq, sizeof(double) * n_tracks * NS * 2);
    if (e == cudaSuccess)
        e = cudaMalloc(&dout, sizeof(float) * perTrack * n_tracks);
    if (e == cudaSuccess)
        e = cudaMalloc(&dlen, sizeof(float) * n_tracks);
    if (e == cudaSuccess)
        e = cudaMemcpy(dq, q, sizeof(double) * n_tracks * NS * 2, cudaMemcpyHostToDevice);
    if (e == cudaSuccess)
        e = launchTrackGrids(nullptr, dq, n_tracks, dout, dlen);
    std::vector<float> out;
    if (e == cudaSuccess)
    {
        out.resize(perTrack * n_tracks);
        e = cudaMemcpy(out.data(), dout, sizeof(float) * out.size(), cudaMemcpyDeviceToHost);
    }
    if (e == cudaSuccess)
        e = cudaMemcpy(track_length, dlen, sizeof(float) * n_tracks, cudaMemcpyDeviceToHost);
    cudaFree(dq);
    cudaFree(dout);
    cudaFree(dlen);
    CK(e);
    for (int r = 0; r < n_tracks; r++)
    {
        const float* o = out.data() + perTrack * r;
        std::memcpy(p_grid + (size_t)r * NS * 2, o, sizeof(float) * NS * 2);
        std::memcpy(dp_grid + (size_t)r * NS * 2, o + NS * 2, sizeof(float) * NS * 2);
        std::memcpy(t_grid + (size_t)r * NS * 2, o + NS * 4, sizeof(float) * NS * 2);
        std::memcpy(kappa_grid + (size_t)r * NS, o + NS * 6, sizeof(float) * NS);
    }
    return DR_OK;
}

extern "C" int dr_gate_env_step(const dr_gate_env_config* env, int true_theta, const float* action, dr_gate_state* state, float* belief,
                                int update_belief, uint64_t seed, uint64_t step, int* term)
{
    int rc = checkGateEnv(env);
    if (rc)
        return rc;
    if (!action || !state || !belief || true_theta < 0 || true_theta >= env->n_theta)
        return fail(DR_ERR_INVALID_ARG, "bad argument");
    if (!gateSupported(env->n_theta))
        return fail(DR_ERR_UNSUPPORTED, "n_theta not compiled in for the gate race");
    int dev = 0;
    CK(cudaGetDevice(&dev));
    GateParams hp = toGateParams(*env);
    std::vector<float> tr = packGateTrack(*env);
    const size_t trOff = (sizeof(GateParams) + 255) & ~(size_t)255;
    if (trOff + tr.size() * 4 > ENV_SCRATCH_PARAMS)
        return fail(DR_ERR_INVALID_ARG, "gate parameters too large");
    std::lock_guard<std::mutex> lock(g_envMu);
    unsigned char* base = nullptr;
    CK(envScratch(dev, &base));
    GateParams* dgp = (GateParams*)base;
    float* dtr = (float*)(base + trOff);
    EnvIo<dr_gate_state>* dio = (EnvIo<dr_gate_state>*)(base + ENV_SCRATCH_PARAMS);
    EnvIo<dr_gate_state> io{};
    io.state = *state;
    for (int i = 0; i < env->n_theta; i++)
        io.belief[i] = belief[i];
    CK(cudaMemcpy(dgp, &hp, sizeof(GateParams), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(dtr, tr.data(), tr.size() * 4, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(dio, &io, sizeof(io), cudaMemcpyHostToDevice));
    CK(launchGateEnvStep(nullptr, env->n_theta, env->i_mppi, dgp, dtr, true_theta, action[0], action[1], &dio->state, dio->belief, update_belief,
                         (uint32_t)seed, (uint32_t)(seed >> 32), (uint32_t)step, &dio->term));
    CK(cudaMemcpy(&io, dio, sizeof(io), cudaMemcpyDeviceToHost));
    *state = io.state;
    for (int i = 0; i < env->n_theta; i++)
        belief[i] = io.belief[i];
    if (term)
        *term = io.term;
    return DR_OK;
}

extern "C" int dr_prmppi_batch_set_rollout_slots(dr_prmppi_batch* b, int slots)
{
    if (!b)
        return fail(DR_ERR_INVALID_ARG, "NULL batch");
    if (slots != 1 && slots != 2 && slots != 4)
        return fail(DR_ERR_INVALID_ARG, "slots must be 1, 2 or 4");
    CK(cudaSetDevice(b->device));
    CK(cudaStreamSynchronize(b->stream));
    b->dropGraph();
    b->dropDevGraph();
    b->prSlots = slots;
    return DR_OK;
}

extern "C" int dr_prmppi_batch_set_profiling(dr_prmppi_batch* b, int on)
{
    if (!b)
        return fail(DR_ERR_INVALID_ARG, "NULL batch");
    b->profiling = on != 0;
    b->timer.reset();
    return DR_OK;
}

extern "C" int dr_prmppi_batch_get_kernel_times(dr_prmppi_batch* b, const char** names, float* ms, int n, int* count)
{
    if (!b)
        return fail(DR_ERR_INVALID_ARG, "NULL batch");
    CK(cudaSetDevice(b->device));
    return kernelTimes(b->timer, names, ms, n, count);
}
