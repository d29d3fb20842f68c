// C ABI of the control step (include/drmppi.h): controller objects, device memory,
// batched launches, CUDA-graph replay and the host tails of the reference controllers
// (src/mppi_controller.cu:363-466, src/prmppi_controller.cu:232-349).
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <numeric>
#include <string>
#include <type_traits>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/drmppi.h"
#include "cp.hpp"
#include "hostutil.hpp"
#include "instance.cuh"
#include "launch.h"

using namespace dr;

namespace dr
{
std::string& lastError()
{
    static thread_local std::string e;
    return e;
}
} // namespace dr


// ============================================================================================
// MPPI controller
// ============================================================================================
struct dr_mppi
{
    int envKind = 0; // 0 strategic race, 1 gate race
    int iMppi = 0;   // gate race: the ego's agent index
    int device = 0;
    cudaStream_t stream = nullptr;
    bool ownStream = false;
    dr_env_config env{};
    dr_mppi_config cfg{};
    uint64_t seed = 0;
    int nth = 0, nopp = 0, K = 0, T = 0, M = 0, nbp = 0, V = 0, H = 0;
    bool spl = false;
    // verification flavour: exact (per-sample parity with the oracle) or fast (default)
    bool exactVerify = false;
    bool egoTableOn = true; // dr_mppi_set_ego_table

    // The fast verification takes the ego's moves from the ego tables: they exist, are
    // switched on and no noise of the environment moves the ego.
    bool egoTableUsable() const
    {
        return !exactVerify && egoTableOn && desc.egoTab && env.action_noise_level == 0.0f && env.pos_noise_level == 0.0f &&
               env.speed_noise_level == 0.0f;
    }
    DevScratch predBuf; // dr_mppi_predict's inputs and outputs on the device
    Arena arena;
    MppiDev desc{};
    unsigned char* hRes = nullptr; // pinned copy of the result block
    // host mirrors of the reference controller's public fields
    std::vector<float> hNominal;
    std::vector<uint32_t> fcNew, fcOld, fc;
    double epsilon = 0, epsilonPartial = 0, certifiedLoss = -1;
    bool useNewPlan = true;
    float lambda = 1.0f;
    uint64_t step = 0;
    int pendBranch = -1, pendUseNew = 0;
    ClopperPearson cp;
    dr_mppi_batch* self = nullptr; // batch of one used by dr_mppi_step
    // gradient refinement after the update (dr_mppi_set_grad_refine)
    int gradSteps = 0, gradCkpt = 1;
    double cpBeta = 0.0; // beta of the shared Clopper-Pearson table this controller holds
    float gradAlpha = 0.05f;
    // sample sharding across processes (dr_mppi_set_shard): this process's samples and
    // verification samples
    int shardRank = 0, shardWorld = 1;
    int sLo = 0, sHi = 0, vLo = 0, vHi = 0;
    // dr_mppi_nominal_grad: device input record and job table
    MppiIn* dGradIn = nullptr;
    GradJob* dGradJobs = nullptr;
    int gradJobsCap = 0;

    MppiIn input(const dr_sim_state& s, const float* belief) const
    {
        MppiIn in{};
        in.state = s;
        fillInput(in, belief);
        return in;
    }

    MppiIn input(const dr_gate_state& s, const float* belief) const
    {
        MppiIn in{};
        in.gstate = s;
        fillInput(in, belief);
        return in;
    }

    void fillInput(MppiIn& in, const float* belief) const
    {
        for (int i = 0; i < DR_MAX_THETA; i++)
            in.belief[i] = i < nth ? belief[i] : 0.0f;
        in.lambda = lambda;
        in.step = (uint32_t)step;
        in.pendBranch = pendBranch;
        in.pendUseNew = pendUseNew;
    }

    // host tail of MPPIController::getControl (mppi_controller.cu:363-456)
    int lastTimeouts = 0; // staging waits that gave up in the last finished step

    void finish(const float* belief, float* outAction, dr_mppi_info* info)
    {
        const unsigned char* r = hRes;
        const uint32_t* fail = (const uint32_t*)(r + ((const unsigned char*)desc.fail - (const unsigned char*)desc.fail));
        const float* dense = (const float*)(r + ((const unsigned char*)desc.dense - (const unsigned char*)desc.fail));
        const float* prevDense = (const float*)(r + ((const unsigned char*)desc.prevDense - (const unsigned char*)desc.fail));
        const float* nu = (const float*)(r + ((const unsigned char*)desc.nu - (const unsigned char*)desc.fail));
        const float* minCosts = (const float*)(r + ((const unsigned char*)desc.minCosts - (const unsigned char*)desc.fail));
        const int* stats = (const int*)(r + ((const unsigned char*)desc.stats - (const unsigned char*)desc.fail));
        lastTimeouts = stats[1];
        fcNew.assign(fail, fail + T);
        fcOld.assign(fail + T, fail + 2 * T);
        if (cfg.verify)
        {
            // computeCertifiedLoss (mppi_controller.cu:468-501)
            certifiedLoss = -1.0;
            uint32_t totOld = 0, totNew = 0;
            for (int t = 0; t < T; t++)
            {
                totOld += fcOld[t];
                totNew += fcNew[t];
                double eps1 = cp.upper(totNew, (uint32_t)V, cfg.beta / 2.0);
                double eps2 = cp.lower(totOld, (uint32_t)V, cfg.beta / 2.0);
                if (eps1 - eps2 > certifiedLoss)
                    certifiedLoss = eps1 - eps2;
            }
            useNewPlan = certifiedLoss < cfg.max_verif_eps;
        }
        else
        {
            certifiedLoss = -1.0;
            useNewPlan = true;
        }
        fc = useNewPlan ? fcNew : fcOld;
        // computeEpsilon (mppi_controller.cu:503-514)
        uint32_t totFail = std::accumulate(fc.begin(), fc.end(), 0u);
        epsilonPartial = cp.upper(totFail, (uint32_t)std::max(V, 1), cfg.beta);
        epsilon = epsilonPartial + (float)(cfg.verif_horizon * cfg.max_verif_eps);
        const float* chosen = useNewPlan ? dense : prevDense;
        hNominal.assign(chosen, chosen + (size_t)nbp * T * 2);
        int branchIdx = findConfidentHost(belief, nth, cfg.min_confidence);
        for (int d = 0; d < 2; d++)
            outAction[d] = hNominal[(size_t)branchIdx * T * 2 + d];
        float usedNu = nu[branchIdx];
        float before = lambda;
        if (usedNu > cfg.max_nu * (float)K)
            lambda *= 0.9f;
        else if (usedNu < cfg.min_nu * (float)K)
            lambda *= 1.2f;
        (void)before;
        // shift the chosen branch (mppi_controller.cu:430-436)
        size_t base = (size_t)branchIdx * T * 2;
        for (int t = 0; t < T - 1; t++)
            for (int d = 0; d < 2; d++)
                hNominal[base + t * 2 + d] = hNominal[base + (t + 1) * 2 + d];
        for (int d = 0; d < 2; d++)
            hNominal[base + (T - 1) * 2 + d] = 0.0f;
        pendBranch = branchIdx;
        pendUseNew = useNewPlan ? 1 : 0;
        step++;
        if (info)
        {
            info->fail_count_total = totFail;
            info->use_new_plan = useNewPlan ? 1 : 0;
            info->epsilon = epsilon;
            info->epsilon_partial = epsilonPartial;
            info->certified_loss = certifiedLoss;
            info->branch_idx = branchIdx;
            info->min_cost = minCosts[branchIdx * M];
            info->nu = usedNu;
            info->inv_temperature = lambda;
            info->nonfinite_costs = stats[0];
            info->verif_timeouts = stats[1];
            const float* gstat = (const float*)(r + ((const unsigned char*)desc.gstat - (const unsigned char*)desc.fail));
            if (gradSteps > 0)
            {
                const int bestIt = std::min(std::max((int)gstat[DR_GRAD_MAX_STEPS + 1], 0), DR_GRAD_MAX_STEPS);
                info->grad_cost_plain = gstat[0];
                info->grad_cost_refined = gstat[bestIt];
                info->grad_best_step = bestIt;
            }
            else
            {
                info->grad_cost_plain = 0.0f;
                info->grad_cost_refined = 0.0f;
                info->grad_best_step = -1;
            }
        }
    }
};

struct dr_mppi_batch
{
    std::vector<dr_mppi*> hs;
    int envKind = 0;
    int iMppi = 0;
    int device = 0;
    cudaStream_t stream = nullptr;
    bool ownStream = false;
    int nopp = 0, nth = 0;
    bool spl = false, verify = true;
    MppiDev* dDesc = nullptr;
    MppiIn* dIn = nullptr;
    MppiIn* hIn = nullptr;
    Tile *dRoll = nullptr, *dUpd = nullptr, *dVer = nullptr, *dVerNew = nullptr, *dVerOld = nullptr;
    int nRoll = 0, nUpd = 0, nVer = 0, nVerNew = 0, nVerOld = 0;
    GradJob* dGrad = nullptr; // gradient refinement jobs (controllers with it on)
    int nGrad = 0;
    size_t gradSmemB = 0;
    // device-resident stepping: the controller state lives in dIn while devCtl is set
    bool devCtl = false;
    cudaGraph_t devGraph = nullptr;
    cudaGraphExec_t devGraphExec = nullptr;
    const void* devKey[4] = {nullptr, nullptr, nullptr, nullptr};
    size_t rollSmem = 0, verSmem = 0, proSmem = 0;
    bool overlap = true;                 // previous-plan verification on sideStream
    // The critical path of a step (prologue, rollout, update, refinement, new-plan
    // verification, tail) runs on hiStream, created with the device's highest stream
    // priority, and the previous plan's verification on sideStream, with the lowest: when
    // the update is launched, its CTAs are dispatched ahead of the side verification's
    // waiting CTAs instead of behind them.
    bool prio = true;
    cudaStream_t hiStream = nullptr;
    cudaStream_t execStream = nullptr; // stream the kernels of launchAll go to (hiStream or stream)
    cudaEvent_t evIn = nullptr, evOut = nullptr;
    cudaStream_t sideStream = nullptr;
    cudaEvent_t evFork = nullptr, evJoin = nullptr;
    Timer timerSide;
    bool useGraph = true;
    bool profiling = false;
    Timer timer;
    int runs = 0;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t graphExec = nullptr;
    const MppiIn* graphIn = nullptr;

    LaunchArgs args(const Tile* tiles, int n, const MppiIn* in) const
    {
        LaunchArgs a;
        a.stream = execStream ? execStream : stream;
        a.mppi = dDesc;
        a.mppiIn = in;
        a.tiles = tiles;
        a.nTiles = n;
        a.exactVerify = hs[0]->exactVerify ? 1 : 0; // equal across the batch (dr_mppi_batch_create)
        a.egoTable = egoTable() ? 1 : 0;
        return a;
    }

    // every controller's verification reads its ego tables (filled before each verification)
    bool egoTable() const
    {
        if (envKind != 0 || !verify)
            return false;
        for (auto* h : hs)
            if (!h->egoTableUsable())
                return false;
        return true;
    }

    cudaError_t launchEgo(cudaStream_t s, const MppiIn* in, int plans) const
    {
        if (!egoTable())
            return cudaSuccess;
        int maxH = 1;
        for (auto* h : hs)
            maxH = std::max(maxH, h->H);
        return launchEgoTable(s, nopp, nth, dDesc, in, (int)hs.size(), plans, maxH);
    }

    cudaError_t launchRollout(const LaunchArgs& a) const
    {
        return envKind ? launchGateRollout(a, nth, iMppi, spl, rollSmem) : launchMppiRollout(a, nopp, nth, spl, rollSmem);
    }

    cudaError_t launchVerify(const LaunchArgs& a) const
    {
        return envKind ? launchGateVerify(a, nth, iMppi, verSmem, nullptr, nullptr) : launchMppiVerify(a, nopp, nth, verSmem, nullptr, nullptr);
    }

    // Persistent launches of the rollout and the verification: perSm CTAs per SM take the
    // tiles from a device work queue (a ticket counter, zeroed by a memset node before
    // each launch) until the table is exhausted; the tables list the longest tiles first.
    // perSm 0 launches one CTA per tile.
    enum QueueSlot
    {
        Q_ROLL = 0,
        Q_VER_NEW = 1,
        Q_VER_OLD = 2,
        Q_VER_ALL = 3
    };
    unsigned* dQueue = nullptr;
    int numSms = 0;
    int rollPerSm = 0, verPerSm = 0;
    int rollLock = 0; // rollout threads of a CTA step through the horizon together
    // Shape of the previous plan's verification when it runs beside the critical path:
    // 0 (default) one CTA per tile, or a persistent grid of sidePerSm CTAs per SM. One
    // persistent CTA per SM leaves room for the rollout and the update (the update drops
    // from 0.26 to 0.13 ms on the 4 x 4096 x 64 step), but verifies more slowly while it
    // runs alone, and the step takes 2.88 ms against 2.82 ms with one CTA per tile.
    int sidePerSm = 0;
    // update and new-plan verification launched as programmatic dependents (0, default:
    // measured on the 4 x 4096 x 64 step, 354.6 against 354.5 control steps/s device-
    // resident and 343.6 against 354.5 through the C ABI, so plain launches)
    int pdl = 0;

    LaunchArgs qargs(const Tile* tiles, int n, const MppiIn* in, QueueSlot slot, int perSm, cudaStream_t s, int lock = -1) const
    {
        LaunchArgs a = args(tiles, n, in);
        a.stream = s;
        a.lockstep = lock < 0 ? rollLock : lock;
        if (perSm > 0 && envKind == 0 && dQueue)
        {
            a.queue = dQueue + slot;
            a.grid = perSm * numSms;
        }
        return a;
    }

    cudaError_t launchQueued(const LaunchArgs& a, bool verification) const
    {
        if (a.queue)
        {
            cudaError_t e = cudaMemsetAsync(a.queue, 0, sizeof(unsigned), a.stream);
            if (e != cudaSuccess)
                return e;
        }
        return verification ? launchVerify(a) : launchRollout(a);
    }

    // kernels of one control step, reading inputs from `in` (device)
    // finish != null: the device tail after the kernels (fully device-resident steps)
    int launchAll(const MppiIn* in, bool profile, Timer* timer, MppiIn* finishIn = nullptr, float* actions = nullptr, dr_mppi_info* infos = nullptr)
    {
        const int n = (int)hs.size();
        cudaStream_t ex = prio && hiStream ? hiStream : stream;
        if (ex != stream)
        {
            CK(cudaEventRecord(evIn, stream));
            CK(cudaStreamWaitEvent(ex, evIn, 0));
        }
        execStream = ex;
        struct Restore
        {
            cudaStream_t& s;
            ~Restore() { s = nullptr; }
        } restore{execStream};
        if (profile)
        {
            timer->begin();
            timer->mark("prologue", ex);
        }
        CK(launchMppiPrologue(args(nullptr, 0, in), n, proSmem));
        // The previous plan's verification needs only the prologue's shifted plan and that
        // plan's ego table, so it runs on a second stream while the rollout (a few warps per
        // SM) and the update run on the first; the new plan's verification follows the
        // update. The previous plan's table is computed here, on the critical stream, before
        // the fork: alone on the device it takes a few tens of microseconds, beside the
        // rollout several times longer (its single warp per table row issues behind the
        // rollout's warps), and the side verification could not start before it ends.
        bool side = verify && overlap && nVerOld > 0;
        if (side)
        {
            if (egoTable())
            {
                if (profile)
                    timer->mark("ego_table_old", ex);
                CK(launchEgo(ex, in, 1));
            }
            CK(cudaEventRecord(evFork, ex)); // the side verification depends on the prologue and the table
        }
        if (profile)
            timer->mark("rollout", ex);
        // the rollout is enqueued (captured) before the side verification, so that its
        // CTAs are dispatched first when both become ready after the prologue
        CK(launchQueued(qargs(dRoll, nRoll, in, Q_ROLL, rollPerSm, ex), false));
        if (side)
        {
            CK(cudaStreamWaitEvent(sideStream, evFork, 0));
            if (profile)
            {
                timerSide.begin();
                timerSide.mark("verify_old", sideStream);
            }
            CK(launchQueued(qargs(dVerOld, nVerOld, in, Q_VER_OLD, sidePerSm, sideStream), true));
            if (profile)
            {
                timerSide.mark("end", sideStream);
                timerSide.end();
            }
            CK(cudaEventRecord(evJoin, sideStream));
        }
        if (profile)
            timer->mark("update", ex);
        {
            // programmatic dependents of the kernel before them: their CTAs are dispatched
            // (at the critical path's priority) as SM slots free up, instead of after the
            // side verification's pending CTAs, and wait in the kernel for its results
            LaunchArgs ua = args(dUpd, nUpd, in);
            ua.pdl = pdl;
            CK(launchMppiUpdate(ua, nth));
        }
        if (nGrad > 0)
        {
            if (profile)
                timer->mark("grad_refine", ex);
            CK(launchGradNominal(ex, dGrad, nGrad, nopp, nth, spl, gradSmemB));
        }
        if (verify && nVerNew > 0)
        {
            if (profile)
                timer->mark("ego_table", ex);
            CK(launchEgo(ex, in, side ? 0 : 2));
            if (profile)
                timer->mark(side ? "verify_new" : "verify", ex);
            LaunchArgs va = side ? qargs(dVerNew, nVerNew, in, Q_VER_NEW, verPerSm, ex) : qargs(dVer, nVer, in, Q_VER_ALL, verPerSm, ex);
            va.pdl = pdl;
            CK(launchQueued(va, true));
        }
        if (finishIn)
        {
            if (side)
                CK(cudaStreamWaitEvent(ex, evJoin, 0));
            if (profile)
                timer->mark("finish", ex);
            CK(launchMppiFinish(ex, dDesc, finishIn, actions, infos, n));
            side = false;
        }
        if (profile)
        {
            timer->mark("end", ex);
            timer->end();
        }
        if (side)
            CK(cudaStreamWaitEvent(stream, evJoin, 0));
        if (ex != stream)
        {
            CK(cudaEventRecord(evOut, ex));
            CK(cudaStreamWaitEvent(stream, evOut, 0));
        }
        return DR_OK;
    }

    int copyResults()
    {
        for (auto* h : hs)
            CK(cudaMemcpyAsync(h->hRes, h->desc.fail, h->desc.resBytes, cudaMemcpyDeviceToHost, stream));
        return DR_OK;
    }

    // H2D inputs + kernels + D2H results, replayed from a CUDA graph after the first run
    int enqueue(bool profile)
    {
        const int n = (int)hs.size();
        if (profile || !useGraph || runs == 0)
        {
            CK(cudaMemcpyAsync(dIn, hIn, sizeof(MppiIn) * n, cudaMemcpyHostToDevice, stream));
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
            cudaMemcpyAsync(dIn, hIn, sizeof(MppiIn) * n, cudaMemcpyHostToDevice, stream);
            int rc = launchAll(dIn, false, nullptr);
            if (rc == DR_OK)
                rc = copyResults();
            cudaGraph_t g = nullptr;
            cudaError_t e = cudaStreamEndCapture(stream, &g);
            if (rc)
                return rc;
            CK(e);
            graph = g;
            CK(cudaGraphInstantiate(&graphExec, graph, cudaGraphInstantiateFlagUseNodePriority));
        }
        CK(cudaGraphLaunch(graphExec, stream));
        runs++;
        return DR_OK;
    }

    template <class St> int step(const St* states, const float* beliefs, int beliefStride, float* actions, dr_mppi_info* infos)
    {
        const int n = (int)hs.size();
        if (envKind != (std::is_same<St, dr_gate_state>::value ? 1 : 0))
            return fail(DR_ERR_INVALID_ARG, envKind ? "gate-race controllers: step them with the dr_gate_* functions"
                                                    : "strategic-race controllers: step them with dr_mppi_step / dr_mppi_batch_step");
        CK(cudaSetDevice(device));
        int prc = pullDeviceControl();
        if (prc)
            return prc;
        for (int i = 0; i < n; i++)
            hIn[i] = hs[i]->input(states[i], beliefs + (size_t)i * beliefStride);
        bool profile = profiling;
        int rc = enqueue(profile);
        if (rc)
            return rc;
        CK(cudaStreamSynchronize(stream));
        int timeouts = 0;
        for (int i = 0; i < n; i++)
        {
            hs[i]->finish(beliefs + (size_t)i * beliefStride, actions + 2 * i, infos ? infos + i : nullptr);
            timeouts += hs[i]->lastTimeouts;
        }
        return timeouts ? timedOut(timeouts) : DR_OK;
    }

    // A step whose kernels gave up a bounded wait has run to its end on defined values
    // (timed-out rollout tiles cost infinity, timed-out verification tiles count no
    // failures), but its result is not the control step's: report it.
    static int timedOut(int n)
    {
        return fail(DR_ERR_TIMEOUT, "a bounded device wait gave up in " + std::to_string(n) + " CTA(s); the step's results are not valid");
    }

    // ---- sample-sharded step of a batch of one (dr_mppi_shard_*) ----
    // The phases only enqueue work on the stream; the caller's collectives order after
    // them on the same stream, and only the tail synchronises.
    DevScratch shardBuf; // merged minima and sums of the update

    int shardWords() const
    {
        const dr_mppi* h = hs[0];
        return h->nbp * h->M * 4 + h->T;
    }

    int shardBegin(const MppiIn& hin, float* partial)
    {
        CK(cudaSetDevice(device));
        dr_mppi* h = hs[0];
        hIn[0] = hin;
        CK(cudaMemcpyAsync(dIn, hIn, sizeof(MppiIn), cudaMemcpyHostToDevice, stream));
        CK(launchMppiPrologue(args(nullptr, 0, dIn), 1, proSmem));
        if (verify && nVerOld > 0)
        {
            CK(launchEgo(stream, dIn, 1));
            CK(launchVerify(args(dVerOld, nVerOld, dIn)));
        }
        CK(launchRollout(args(dRoll, nRoll, dIn)));
        CK(launchShardLocal(args(dUpd, nUpd, dIn), nth, partial));
        // the previous plan's failure histogram of this process's verification samples
        CK(cudaMemcpyAsync(partial + (size_t)h->nbp * h->M * 4, h->desc.fail + h->T, sizeof(uint32_t) * h->T, cudaMemcpyDeviceToDevice, stream));
        return DR_OK;
    }

    int shardUpdate(const float* gathered, int world, uint32_t* hist)
    {
        CK(cudaSetDevice(device));
        dr_mppi* h = hs[0];
        const size_t nv = (size_t)h->nbp * h->M;
        CK(shardBuf.reserve(nv * 4 * sizeof(float)));
        float* mins = (float*)shardBuf.p;
        float* sums = mins + nv;
        CK(launchShardMerge(stream, dDesc, dIn, gathered, shardWords(), world, mins, sums));
        CK(launchShardApply(stream, dDesc, 1, nth, mins, sums));
        if (nGrad > 0)
            CK(launchGradNominal(stream, dGrad, nGrad, nopp, nth, spl, gradSmemB));
        if (verify && nVerNew > 0)
        {
            CK(launchEgo(stream, dIn, 0));
            CK(launchVerify(args(dVerNew, nVerNew, dIn)));
        }
        CK(cudaMemcpyAsync(hist, h->desc.fail, sizeof(uint32_t) * h->T, cudaMemcpyDeviceToDevice, stream));
        return DR_OK;
    }

    int shardFinish(const uint32_t* hist, const float* belief, float* action, dr_mppi_info* info)
    {
        CK(cudaSetDevice(device));
        CK(cudaMemcpyAsync(hs[0]->desc.fail, hist, sizeof(uint32_t) * hs[0]->T, cudaMemcpyDeviceToDevice, stream));
        int rc = copyResults();
        if (rc)
            return rc;
        CK(cudaStreamSynchronize(stream));
        hs[0]->finish(belief, action, info);
        return hs[0]->lastTimeouts ? timedOut(hs[0]->lastTimeouts) : DR_OK;
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

    // Fully device-resident step: state and belief from device memory, the device tail
    // writes actions and infos to device memory and carries the controller state (the
    // input records' temperature, step counter and warm-start shift) to the next step.
    int stepDevice(const void* states, const float* beliefs, float* actions, dr_mppi_info* infos)
    {
        const int n = (int)hs.size();
        CK(cudaSetDevice(device));
        if (!devCtl)
        {
            // the controllers' host state, once; from here on it lives in the device records
            dropDevGraph();
            std::vector<float> zero(DR_MAX_THETA, 0.0f);
            for (int i = 0; i < n; i++)
                hIn[i] = envKind ? hs[i]->input(dr_gate_state{}, zero.data()) : hs[i]->input(dr_sim_state{}, zero.data());
            CK(cudaMemcpyAsync(dIn, hIn, sizeof(MppiIn) * n, cudaMemcpyHostToDevice, stream));
            CK(cudaStreamSynchronize(stream));
            devCtl = true;
        }
        const size_t stBytes = envKind ? sizeof(dr_gate_state) : sizeof(dr_sim_state);
        auto body = [&](bool profile) -> int {
            for (int i = 0; i < n; i++)
            {
                CK(cudaMemcpyAsync(&dIn[i].state, (const unsigned char*)states + i * stBytes, stBytes, cudaMemcpyDeviceToDevice, stream));
                CK(cudaMemcpyAsync(&dIn[i].belief, beliefs + (size_t)i * DR_MAX_THETA, DR_MAX_THETA * 4, cudaMemcpyDeviceToDevice, stream));
            }
            return launchAll(dIn, profile, &timer, dIn, actions, infos);
        };
        if (profiling || !useGraph)
            return body(profiling);
        const void* key[4] = {states, beliefs, actions, infos};
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
            CK(cudaGraphInstantiate(&devGraphExec, devGraph, cudaGraphInstantiateFlagUseNodePriority));
            std::memcpy(devKey, key, sizeof(key));
        }
        CK(cudaGraphLaunch(devGraphExec, stream));
        return DR_OK;
    }

    // Copies the controller state carried by the device records back to the controllers
    // (after device-resident steps, before a host step).
    int pullDeviceControl()
    {
        if (!devCtl)
            return DR_OK;
        const int n = (int)hs.size();
        std::vector<MppiIn> tmp((size_t)n);
        CK(cudaStreamSynchronize(stream));
        CK(cudaMemcpy(tmp.data(), dIn, sizeof(MppiIn) * n, cudaMemcpyDeviceToHost));
        for (int i = 0; i < n; i++)
        {
            dr_mppi* h = hs[i];
            h->lambda = tmp[i].lambda;
            // the device record carries the low 32 bits of the step counter
            const uint64_t prev = h->step;
            uint64_t next = (prev & ~(uint64_t)0xffffffffu) | tmp[i].step;
            if (next < prev)
                next += (uint64_t)1 << 32;
            h->step = next;
            h->pendBranch = tmp[i].pendBranch;
            h->pendUseNew = tmp[i].pendUseNew;
        }
        devCtl = false;
        return DR_OK;
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

    // Copies the controllers' device descriptors (host copies in dr_mppi::desc) to the
    // batch's descriptor table; the caller has synchronised the stream.
    int uploadDescs()
    {
        std::vector<MppiDev> descs;
        for (auto* h : hs)
            descs.push_back(h->desc);
        CK(cudaMemcpy(dDesc, descs.data(), sizeof(MppiDev) * descs.size(), cudaMemcpyHostToDevice));
        return DR_OK;
    }

    // (Re)builds the gradient refinement job table from the controllers' settings.
    int setupGrad()
    {
        CK(cudaSetDevice(device));
        CK(cudaStreamSynchronize(stream));
        dropGraph();
        dropDevGraph();
        {
            int rc = uploadDescs();
            if (rc)
                return rc;
        }
        std::vector<GradJob> jobs;
        gradSmemB = 0;
        for (size_t i = 0; i < hs.size(); i++)
        {
            dr_mppi* h = hs[i];
            if (h->gradSteps <= 0)
                continue;
            GradJob j{};
            j.D = dDesc + i;
            j.in = dIn + i;
            j.J = h->desc.gstat;
            j.stats = h->desc.gstat + DR_GRAD_MAX_STEPS + 1;
            j.iters = h->gradSteps;
            j.ckpt = h->gradCkpt;
            j.alpha = h->gradAlpha;
            j.write = 1;
            jobs.push_back(j);
            gradSmemB = std::max(gradSmemB, gradSmem(nopp, nth, h->T, h->M, h->gradCkpt, spl));
        }
        if (dGrad)
            CK(cudaFree(dGrad));
        dGrad = nullptr;
        nGrad = (int)jobs.size();
        if (nGrad > 0)
        {
            CK(cudaMalloc(&dGrad, sizeof(GradJob) * jobs.size()));
            CK(cudaMemcpy(dGrad, jobs.data(), sizeof(GradJob) * jobs.size(), cudaMemcpyHostToDevice));
        }
        return DR_OK;
    }

    void release()
    {
        dropGraph();
        dropDevGraph();
        shardBuf.release();
        cudaFree(dGrad);
        dGrad = nullptr;
        cudaFree(dDesc);
        cudaFree(dIn);
        cudaFree(dRoll);
        cudaFree(dUpd);
        cudaFree(dVer);
        cudaFree(dQueue);
        dQueue = nullptr;
        if (hIn)
            cudaFreeHost(hIn);
        if (sideStream)
        {
            cudaStreamSynchronize(sideStream);
            cudaStreamDestroy(sideStream);
        }
        if (evFork)
            cudaEventDestroy(evFork);
        if (evJoin)
            cudaEventDestroy(evJoin);
        if (evIn)
            cudaEventDestroy(evIn);
        if (evOut)
            cudaEventDestroy(evOut);
        if (hiStream)
        {
            cudaStreamSynchronize(hiStream);
            cudaStreamDestroy(hiStream);
        }
        if (ownStream && stream)
            cudaStreamDestroy(stream);
    }
};

namespace
{

int buildMppiBatch(dr_mppi* const* hs, int n, cudaStream_t stream, bool ownStream, dr_mppi_batch** out)
{
    if (n <= 0 || !hs)
        return fail(DR_ERR_INVALID_ARG, "empty batch");
    auto b = std::make_unique<dr_mppi_batch>();
    b->hs.assign(hs, hs + n);
    b->device = hs[0]->device;
    b->nopp = hs[0]->nopp;
    b->nth = hs[0]->nth;
    b->spl = hs[0]->spl;
    b->verify = hs[0]->cfg.verify != 0;
    b->envKind = hs[0]->envKind;
    b->iMppi = hs[0]->iMppi;
    for (int i = 0; i < n; i++)
        if (!hs[i] || hs[i]->device != b->device || hs[i]->nopp != b->nopp || hs[i]->nth != b->nth || hs[i]->spl != b->spl ||
            (hs[i]->cfg.verify != 0) != b->verify || hs[i]->envKind != b->envKind || hs[i]->iMppi != b->iMppi ||
            hs[i]->exactVerify != hs[0]->exactVerify)
            return fail(DR_ERR_INVALID_ARG, "a batch needs controllers on one device with equal environment kind, ego index, n_opp, n_theta, "
                                            "use_splines, verify and verification flavour");
    CK(cudaSetDevice(b->device));
    b->stream = stream;
    b->ownStream = ownStream;
    std::vector<MppiDev> descs;
    std::vector<Tile> roll, upd, ver, verOld;
    const int spb = b->envKind ? gateRolloutSamplesPerBlock(b->nth) : rolloutSamplesPerBlock(b->nth);
    int maxT = 0, maxM = 0, maxNbpT = 0;
    for (int i = 0; i < n; i++)
    {
        dr_mppi* h = hs[i];
        descs.push_back(h->desc);
        for (int s0 = h->sLo; s0 < h->sHi; s0 += spb)
            roll.push_back(Tile{i, s0, std::min(spb, h->sHi - s0), 0});
        for (int bk = 0; bk < h->nbp * h->M; bk++)
            upd.push_back(Tile{i, bk, 0, 0});
        if (b->verify)
            for (int plan = 0; plan < 2; plan++)
                for (int v0 = h->vLo; v0 < h->vHi; v0 += VERIFY_TILE)
                    (plan == 0 ? ver : verOld).push_back(Tile{i, v0, std::min(VERIFY_TILE, h->vHi - v0), plan});
        maxT = std::max(maxT, h->T);
        maxM = std::max(maxM, h->M);
        maxNbpT = std::max(maxNbpT, h->nbp * h->T);
    }
    // longest tiles first (stable, so equal tiles keep controller order): a persistent
    // launch takes them in this order, and a static grid is dispatched roughly in it
    auto byWork = [&](std::vector<Tile>& v, bool verification) {
        std::stable_sort(v.begin(), v.end(), [&](const Tile& x, const Tile& y) {
            const long long wx = (long long)x.count * (verification ? hs[x.inst]->H : hs[x.inst]->T);
            const long long wy = (long long)y.count * (verification ? hs[y.inst]->H : hs[y.inst]->T);
            return wx > wy;
        });
    };
    byWork(roll, false);
    byWork(ver, true);
    byWork(verOld, true);
    // tile table: new-plan tiles first, then previous-plan tiles
    b->nVerNew = (int)ver.size();
    b->nVerOld = (int)verOld.size();
    ver.insert(ver.end(), verOld.begin(), verOld.end());
    for (int i = 0; i < n; i++)
    {
        b->rollSmem = std::max(b->rollSmem, b->envKind ? gateRolloutSmem(b->nth, hs[i]->T, hs[i]->M, b->spl) : mppiRolloutSmem(b->nth, hs[i]->T, hs[i]->M, b->spl));
        b->verSmem = std::max(b->verSmem, b->envKind ? gateVerifySmem(b->nth, hs[i]->T) : mppiVerifySmem(b->nth, hs[i]->T));
    }
    b->proSmem = ((size_t)maxNbpT * 2 + (size_t)maxM * 2) * 4;
    if (b->rollSmem > 227 * 1024)
        return fail(DR_ERR_INVALID_ARG, "horizon x knots too large for shared memory");
    b->nRoll = (int)roll.size();
    b->nUpd = (int)upd.size();
    b->nVer = (int)ver.size();
    CK(cudaMalloc(&b->dDesc, sizeof(MppiDev) * n));
    CK(cudaMemcpy(b->dDesc, descs.data(), sizeof(MppiDev) * n, cudaMemcpyHostToDevice));
    CK(cudaMalloc(&b->dIn, sizeof(MppiIn) * n));
    CK(cudaMallocHost(&b->hIn, sizeof(MppiIn) * n));
    CK(cudaMalloc(&b->dRoll, sizeof(Tile) * std::max<size_t>(roll.size(), 1)));
    CK(cudaMemcpy(b->dRoll, roll.data(), sizeof(Tile) * roll.size(), cudaMemcpyHostToDevice));
    CK(cudaMalloc(&b->dUpd, sizeof(Tile) * std::max<size_t>(upd.size(), 1)));
    CK(cudaMemcpy(b->dUpd, upd.data(), sizeof(Tile) * upd.size(), cudaMemcpyHostToDevice));
    CK(cudaMalloc(&b->dVer, sizeof(Tile) * std::max<size_t>(ver.size(), 1)));
    if (!ver.empty())
        CK(cudaMemcpy(b->dVer, ver.data(), sizeof(Tile) * ver.size(), cudaMemcpyHostToDevice));
    b->dVerNew = b->dVer;
    b->dVerOld = b->dVer + b->nVerNew;
    CK(cudaMalloc(&b->dQueue, sizeof(unsigned) * 4));
    CK(cudaMemset(b->dQueue, 0, sizeof(unsigned) * 4));
    CK(cudaDeviceGetAttribute(&b->numSms, cudaDevAttrMultiProcessorCount, b->device));
    {
        int least = 0, greatest = 0;
        CK(cudaDeviceGetStreamPriorityRange(&least, &greatest));
        CK(cudaStreamCreateWithPriority(&b->sideStream, cudaStreamNonBlocking, least));
        CK(cudaStreamCreateWithPriority(&b->hiStream, cudaStreamNonBlocking, greatest));
    }
    CK(cudaEventCreateWithFlags(&b->evFork, cudaEventDisableTiming));
    CK(cudaEventCreateWithFlags(&b->evJoin, cudaEventDisableTiming));
    CK(cudaEventCreateWithFlags(&b->evIn, cudaEventDisableTiming));
    CK(cudaEventCreateWithFlags(&b->evOut, cudaEventDisableTiming));
    int rc = b->setupGrad();
    if (rc)
        return rc;
    *out = b.release();
    return DR_OK;
}

int checkMppiCfg(const dr_env_config* env, const dr_mppi_config* c)
{
    if (!c)
        return fail(DR_ERR_INVALID_ARG, "cfg is NULL");
    if (c->n_samples < 1 || c->n_samples > (1 << 24))
        return fail(DR_ERR_INVALID_ARG, "n_samples must be in [1, 2^24]");
    if (c->n_timesteps < 2 || c->n_timesteps > DR_MAX_T)
        return fail(DR_ERR_INVALID_ARG, "n_timesteps must be in [2, 256]");
    if (c->use_splines)
    {
        if (c->n_knots < 2 || c->n_knots > DR_MAX_KNOTS)
            return fail(DR_ERR_INVALID_ARG, "n_knots must be in [2, 64]");
        for (int i = 0; i < c->n_knots; i++)
        {
            if (c->knots[i] < 0 || c->knots[i] > c->n_timesteps - 2)
                return fail(DR_ERR_INVALID_ARG, "knots must lie in [0, T-2]");
            if (i > 0 && c->knots[i] <= c->knots[i - 1])
                return fail(DR_ERR_INVALID_ARG, "knots must be strictly increasing");
        }
    }
    if (c->verify)
    {
        if (c->n_verif_samples < 1)
            return fail(DR_ERR_INVALID_ARG, "n_verif_samples must be positive");
        if (c->verif_horizon < 1 || c->verif_horizon > c->n_timesteps)
            return fail(DR_ERR_INVALID_ARG, "verif_horizon must be in [1, n_timesteps]");
    }
    if (!(c->inv_temperature > 0.0f) || !std::isfinite(c->inv_temperature))
        return fail(DR_ERR_INVALID_ARG, "inv_temperature must be positive");
    if (!mppiSupported(env->n_opp, env->n_theta))
        return fail(DR_ERR_UNSUPPORTED, "(n_opp, n_theta) combination not compiled in");
    return DR_OK;
}

} // namespace

extern "C" {

int dr_abi_version(void)
{
    return DR_ABI_VERSION;
}

int dr_supported(int n_opp, int n_theta)
{
    return mppiSupported(n_opp, n_theta) && prSupported(n_opp, n_theta);
}

const char* dr_last_error(void)
{
    return lastError().c_str();
}

const char* dr_status_string(int s)
{
    switch (s)
    {
    case DR_OK: return "ok";
    case DR_ERR_INVALID_ARG: return "invalid argument";
    case DR_ERR_UNSUPPORTED: return "unsupported configuration";
    case DR_ERR_CUDA: return "CUDA error";
    case DR_ERR_OOM: return "out of device memory";
    case DR_ERR_NO_DEVICE: return "no CUDA device";
    case DR_ERR_TIMEOUT: return "device wait timed out";
    case DR_ERR_STATE: return "invalid state";
    default: return "unknown";
    }
}

} // extern "C"

// MPPIController construction for either environment: the strategic race (env) or the
// gate race (genv); exactly one of the two is given.
static int createMppi(const dr_env_config* env, const dr_gate_env_config* genv, const dr_mppi_config* cfg, uint64_t seed, const float* nominal,
                      int device, void* stream, dr_mppi** out)
{
    if (!out)
        return fail(DR_ERR_INVALID_ARG, "out is NULL");
    *out = nullptr;
    int rc = env ? checkEnv(env) : checkGateEnv(genv);
    if (rc)
        return rc;
    if (env)
        rc = checkMppiCfg(env, cfg);
    else
    {
        dr_env_config probe{};
        probe.n_opp = 1;
        probe.n_theta = genv->n_theta;
        rc = checkMppiCfg(&probe, cfg);
        if (!rc && !gateSupported(genv->n_theta))
            rc = fail(DR_ERR_UNSUPPORTED, "n_theta not compiled in for the gate race");
    }
    if (rc)
        return rc;
    rc = selectDevice(device);
    if (rc)
        return rc;
    auto h = std::make_unique<dr_mppi>();
    h->envKind = env ? 0 : 1;
    h->iMppi = env ? 0 : genv->i_mppi;
    h->device = device;
    if (env)
    {
        h->env = *env;
        h->env.p_grid = h->env.dp_grid = h->env.t_grid = h->env.kappa_grid = nullptr;
    }
    h->cfg = *cfg;
    h->seed = seed;
    h->nth = env ? env->n_theta : genv->n_theta;
    h->nopp = env ? env->n_opp : 1;
    h->K = cfg->n_samples;
    h->T = cfg->n_timesteps;
    h->spl = cfg->use_splines != 0;
    h->M = h->spl ? cfg->n_knots : h->T;
    if (!h->spl)
        for (int i = 0; i < DR_MAX_KNOTS; i++)
            h->cfg.knots[i] = i; // unused in dense mode
    h->nbp = h->nth + 1;
    h->V = cfg->verify ? cfg->n_verif_samples : 0;
    h->H = cfg->verif_horizon;
    h->lambda = cfg->inv_temperature;
    const int K = h->K, T = h->T, M = h->M, nbp = h->nbp, nth = h->nth;
    MppiDev& D = h->desc;
    if (env)
        D.env = toEnvParams(*env);
    else
        D.env.maxAccel[0] = genv->max_accel[genv->i_mppi]; // Env::getMaxAccel, the update's clamp (mppi_controller.cu:345)
    D.cfg.K = K;
    D.cfg.T = T;
    D.cfg.M = M;
    D.cfg.useSplines = h->spl ? 1 : 0;
    D.cfg.V = h->V;
    D.cfg.H = h->H;
    D.cfg.nth = nth;
    D.cfg.nopp = h->nopp;
    for (int i = 0; i < DR_MAX_KNOTS; i++)
        D.cfg.knots[i] = h->cfg.knots[i];
    float s0 = cfg->sampling_noise_dim[0], s1 = cfg->sampling_noise_dim[1];
    if (s0 == 0.0f && s1 == 0.0f)
        s0 = s1 = cfg->sampling_noise;
    D.cfg.sigma0 = s0;
    D.cfg.sigma1 = s1;
    D.cfg.minConf = cfg->min_confidence;
    D.cfg.gateMargin = cfg->gate_traversal_margin;
    D.cfg.w = MppiCostW{cfg->coll_dist_factor, cfg->boundary_cost, cfg->boundary_threshold_factor, cfg->outside_cost,
                        cfg->win_cost,         cfg->opp_win_cost,  cfg->final_adv_weight,          cfg->final_opp_adv_weight};
    D.cfg.k0 = (uint32_t)seed;
    D.cfg.k1 = (uint32_t)(seed >> 32);
    if (h->cfg.min_nu == 0.0f && h->cfg.max_nu == 0.0f)
    {
        h->cfg.min_nu = 0.0005f; // controllers.h:47-48
        h->cfg.max_nu = 0.001f;
    }
    D.cfg.beta = cfg->beta;
    D.cfg.maxVerifEps = cfg->max_verif_eps;
    D.cfg.minNu = h->cfg.min_nu;
    D.cfg.maxNu = h->cfg.max_nu;
    D.cfg.verify = cfg->verify ? 1 : 0;
    D.cfg.gradSteps = 0;
    D.cfg.sLo = 0;
    D.cfg.sHi = K;
    h->sHi = K;
    h->vHi = h->V;

    // device memory
    float *grids, *B, *knots, *costsTrue, *costs, *dense, *prevDense, *nu, *minCosts;
    int *binfo, *stats;
    unsigned *counter, *failc;
    Arena& A = h->arena;
    GateParams* gp = nullptr;
    float* gtrack = nullptr;
    if (env)
        A.add(grids, GRID_FLOATS * 4);
    else
    {
        A.add(gp, a16(sizeof(GateParams)));
        A.add(gtrack, GATE_TRACK_FLOATS * 4);
    }
    A.add(B, a16((size_t)T * M * 4));
    A.add(knots, a16((size_t)nbp * M * 2 * 4));
    A.add(costsTrue, (size_t)nth * K * 4);
    A.add(binfo, (size_t)nth * K * 4);
    A.add(costs, (size_t)nbp * K * 4);
    A.add(counter, 16);
    double* cpTab;
    A.add(cpTab, sizeof(double) * 3 * CP_TAB);
    // the ego tables of the fast verification (strategic race), when they stay small
    EgoRow* egoTab = nullptr;
    const size_t egoBytes = (size_t)2 * egoRows(nth, h->H) * h->H * sizeof(EgoRow);
    if (env && cfg->verify && egoBytes <= EGO_TABLE_MAX_BYTES)
        A.add(egoTab, egoBytes);

    // result block, one contiguous range
    size_t oFail = 0, oDense = a16(oFail + (size_t)2 * T * 4), oPrev = oDense + a16((size_t)nbp * T * 2 * 4), oNu = oPrev + a16((size_t)nbp * T * 2 * 4),
           oMin = oNu + a16((size_t)nbp * 4), oStats = oMin + a16((size_t)nbp * M * 4), oGrad = oStats + 16,
           resBytes = oGrad + a16((DR_GRAD_MAX_STEPS + 3) * 4);
    unsigned char* res;
    A.add(res, resBytes);
    CK(A.alloc());
    failc = (unsigned*)(res + oFail);
    dense = (float*)(res + oDense);
    prevDense = (float*)(res + oPrev);
    nu = (float*)(res + oNu);
    minCosts = (float*)(res + oMin);
    stats = (int*)(res + oStats);
    D.gstat = (float*)(res + oGrad);
    D.cpTab = cpTab;
    D.cpFull = nullptr;
    if (cfg->verify)
    {
        // failure counts of CP_TAB and more (plans that fail often) read the shared table
        h->cpBeta = (double)cfg->beta;
        if (!acquireCpTable(h->device, (uint32_t)h->V, h->cpBeta, &D.cpFull))
            return fail(DR_ERR_CUDA, "Clopper-Pearson table: " + std::string(cudaGetErrorString(cudaGetLastError())));
    }
    D.grids = env ? grids : nullptr;
    D.gate = gp;
    D.gtrack = gtrack;
    D.B = B;
    D.knots = knots;
    D.costsTrue = costsTrue;
    D.binfo = binfo;
    D.costs = costs;
    D.counter = counter;
    D.fail = failc;
    D.dense = dense;
    D.prevDense = prevDense;
    D.nu = nu;
    D.minCosts = minCosts;
    D.stats = stats;
    D.egoTab = egoTab;
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
    if (h->spl)
    {
        std::vector<float> Bm = splineMatrix(T, M, h->cfg.knots);
        CK(cudaMemcpy(B, Bm.data(), Bm.size() * 4, cudaMemcpyHostToDevice));
    }
    {
        // the device tail's Clopper-Pearson table (counts below CP_TAB)
        std::vector<double> tab(3 * (size_t)CP_TAB);
        const uint32_t Vv = (uint32_t)h->V, V1 = (uint32_t)std::max(h->V, 1);
        const double beta = (double)cfg->beta;
        for (int k = 0; k < CP_TAB; k++)
        {
            tab[k] = (uint32_t)k <= Vv && Vv > 0 ? h->cp.upper((uint32_t)k, Vv, beta / 2.0) : 1.0;
            tab[CP_TAB + k] = (uint32_t)k <= Vv && Vv > 0 ? h->cp.lower((uint32_t)k, Vv, beta / 2.0) : 0.0;
            tab[2 * CP_TAB + k] = (uint32_t)k <= V1 ? h->cp.upper((uint32_t)k, V1, beta) : 1.0;
        }
        CK(cudaMemcpy(cpTab, tab.data(), tab.size() * sizeof(double), cudaMemcpyHostToDevice));
    }
    h->hNominal.assign((size_t)nbp * T * 2, 0.0f);
    if (nominal)
        std::memcpy(h->hNominal.data(), nominal, h->hNominal.size() * 4);
    CK(cudaMemcpy(dense, h->hNominal.data(), h->hNominal.size() * 4, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(prevDense, h->hNominal.data(), h->hNominal.size() * 4, cudaMemcpyHostToDevice));
    if (!h->spl)
        CK(cudaMemcpy(knots, h->hNominal.data(), h->hNominal.size() * 4, cudaMemcpyHostToDevice)); // spline knots start at 0 (mppi_controller.cu:205)
    CK(cudaMallocHost(&h->hRes, resBytes));
    h->fcNew.assign(T, 0u);
    h->fcOld.assign(T, 0u);
    h->fc.assign(T, 0u);
    cudaStream_t s = (cudaStream_t)stream;
    bool own = false;
    if (!s)
    {
        CK(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
        own = true;
    }
    h->stream = s;
    h->ownStream = own;
    dr_mppi* raw = h.get();
    rc = buildMppiBatch(&raw, 1, s, false, &h->self);
    if (rc)
        return rc;
    *out = h.release();
    return DR_OK;
}

extern "C" {

int dr_mppi_create(const dr_env_config* env, const dr_mppi_config* cfg, uint64_t seed, const float* nominal, int device, void* stream, dr_mppi** out)
{
    if (!env)
        return fail(DR_ERR_INVALID_ARG, "env is NULL");
    return createMppi(env, nullptr, cfg, seed, nominal, device, stream, out);
}

int dr_gate_mppi_create(const dr_gate_env_config* env, const dr_mppi_config* cfg, uint64_t seed, const float* nominal, int device, void* stream,
                        dr_mppi** out)
{
    if (!env)
        return fail(DR_ERR_INVALID_ARG, "env is NULL");
    return createMppi(nullptr, env, cfg, seed, nominal, device, stream, out);
}

int dr_mppi_destroy(dr_mppi* h)
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
    cudaFree(h->dGradIn);
    cudaFree(h->dGradJobs);
    h->predBuf.release();
    if (h->desc.cpFull)
        releaseCpTable(h->device, (uint32_t)h->V, h->cpBeta);
    h->arena.release();
    if (h->hRes)
        cudaFreeHost(h->hRes);
    if (h->ownStream && h->stream)
        cudaStreamDestroy(h->stream);
    delete h;
    return DR_OK;
}

int dr_mppi_step(dr_mppi* h, const dr_sim_state* state, const float* belief, float* out_action, dr_mppi_info* info)
{
    if (!h || !state || !belief || !out_action)
        return fail(DR_ERR_INVALID_ARG, "NULL argument");
    if (h->shardWorld > 1)
        return fail(DR_ERR_STATE, "a sample-sharded controller steps through dr_mppi_shard_*");
    return h->self->step(state, belief, h->nth, out_action, info);
}

int dr_gate_mppi_step(dr_mppi* h, const dr_gate_state* state, const float* belief, float* out_action, dr_mppi_info* info)
{
    if (!h || !state || !belief || !out_action)
        return fail(DR_ERR_INVALID_ARG, "NULL argument");
    return h->self->step(state, belief, h->nth, out_action, info);
}

int dr_mppi_get_nominal(const dr_mppi* h, float* out, size_t n)
{
    if (!h || !out || n < h->hNominal.size())
        return fail(DR_ERR_INVALID_ARG, "output too small");
    std::memcpy(out, h->hNominal.data(), h->hNominal.size() * 4);
    return DR_OK;
}

int dr_mppi_get_knots(dr_mppi* h, float* out, size_t n)
{
    size_t need = (size_t)h->nbp * h->M * 2;
    if (!h || !out || n < need)
        return fail(DR_ERR_INVALID_ARG, "output too small");
    CK(cudaSetDevice(h->device));
    CK(cudaStreamSynchronize(h->stream));
    CK(cudaMemcpy(out, h->desc.knots, need * 4, cudaMemcpyDeviceToHost));
    return DR_OK;
}

int dr_mppi_get_fail_counts(const dr_mppi* h, uint32_t* a, uint32_t* b, uint32_t* c, size_t n)
{
    if (!h || n < (size_t)h->T)
        return fail(DR_ERR_INVALID_ARG, "output too small");
    if (a)
        std::memcpy(a, h->fcNew.data(), h->T * 4);
    if (b)
        std::memcpy(b, h->fcOld.data(), h->T * 4);
    if (c)
        std::memcpy(c, h->fc.data(), h->T * 4);
    return DR_OK;
}

float dr_mppi_get_temperature(const dr_mppi* h)
{
    return h ? h->lambda : NAN;
}

int dr_mppi_set_temperature(dr_mppi* h, float v)
{
    if (!h || !(v > 0.0f))
        return fail(DR_ERR_INVALID_ARG, "temperature must be positive");
    h->lambda = v;
    return DR_OK;
}

uint64_t dr_mppi_get_step(const dr_mppi* h)
{
    return h ? h->step : 0;
}

int dr_mppi_io_bytes(const dr_mppi* h, size_t* h2d, size_t* d2h)
{
    if (!h)
        return fail(DR_ERR_INVALID_ARG, "NULL handle");
    if (h2d)
        *h2d = sizeof(MppiIn);
    if (d2h)
        *d2h = h->desc.resBytes;
    return DR_OK;
}

int dr_mppi_set_shard(dr_mppi* h, int rank, int world)
{
    if (!h)
        return fail(DR_ERR_INVALID_ARG, "NULL handle");
    if (h->envKind != 0)
        return fail(DR_ERR_UNSUPPORTED, "sample sharding is built for the strategic race");
    if (world < 1 || rank < 0 || rank >= world || world > h->K)
        return fail(DR_ERR_INVALID_ARG, "need 0 <= rank < world <= n_samples");
    h->shardRank = rank;
    h->shardWorld = world;
    h->sLo = (int)((int64_t)h->K * rank / world);
    h->sHi = (int)((int64_t)h->K * (rank + 1) / world);
    h->vLo = (int)((int64_t)h->V * rank / world);
    h->vHi = (int)((int64_t)h->V * (rank + 1) / world);
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
    dr_mppi* raw = h;
    return buildMppiBatch(&raw, 1, h->stream, false, &h->self);
}

int dr_mppi_shard_words(const dr_mppi* h, size_t* words)
{
    if (!h || !words)
        return fail(DR_ERR_INVALID_ARG, "NULL argument");
    *words = (size_t)h->self->shardWords();
    return DR_OK;
}

int dr_mppi_shard_begin(dr_mppi* h, const dr_sim_state* state, const float* belief, float* partial_dev)
{
    if (!h || !state || !belief || !partial_dev)
        return fail(DR_ERR_INVALID_ARG, "NULL argument");
    if (h->envKind != 0)
        return fail(DR_ERR_UNSUPPORTED, "sample sharding is built for the strategic race");
    return h->self->shardBegin(h->input(*state, belief), partial_dev);
}

int dr_mppi_shard_update(dr_mppi* h, const float* gathered_dev, int world, uint32_t* hist_dev)
{
    if (!h || !gathered_dev || !hist_dev)
        return fail(DR_ERR_INVALID_ARG, "NULL argument");
    if (world != h->shardWorld)
        return fail(DR_ERR_INVALID_ARG, "world differs from dr_mppi_set_shard's");
    return h->self->shardUpdate(gathered_dev, world, hist_dev);
}

int dr_mppi_shard_finish(dr_mppi* h, const uint32_t* hist_dev, const float* belief, float* out_action, dr_mppi_info* info)
{
    if (!h || !hist_dev || !belief || !out_action)
        return fail(DR_ERR_INVALID_ARG, "NULL argument");
    return h->self->shardFinish(hist_dev, belief, out_action, info);
}

int dr_mppi_set_grad_refine(dr_mppi* h, int steps, float step_size, int ckpt_stride)
{
    if (!h)
        return fail(DR_ERR_INVALID_ARG, "NULL handle");
    if (h->envKind != 0)
        return fail(DR_ERR_UNSUPPORTED, "the gradient path is built for the strategic race");
    if (steps < 0 || steps > DR_GRAD_MAX_STEPS)
        return fail(DR_ERR_INVALID_ARG, "steps must be in [0, DR_GRAD_MAX_STEPS]");
    if (steps > 0 && !(step_size > 0.0f && std::isfinite(step_size)))
        return fail(DR_ERR_INVALID_ARG, "step_size must be positive");
    if (ckpt_stride < 0 || ckpt_stride > h->T)
        return fail(DR_ERR_INVALID_ARG, "ckpt_stride must be in [0, n_timesteps]");
    const int ck = ckpt_stride ? ckpt_stride : gradDefaultStride(h->nopp, h->nth, h->T, h->M, h->spl);
    if (steps > 0 && gradSmem(h->nopp, h->nth, h->T, h->M, ck, h->spl) > 227 * 1024)
        return fail(DR_ERR_INVALID_ARG, "checkpoint stride x horizon too large for shared memory");
    h->gradSteps = steps;
    h->gradAlpha = step_size;
    h->gradCkpt = ck;
    h->desc.cfg.gradSteps = steps;
    return h->self->setupGrad();
}

int dr_mppi_nominal_grad(dr_mppi* h, const dr_sim_state* state, const float* belief, int n, const float* knots_dev, const float* weights_dev,
                         float* cost_dev, float* d_knots_dev, float* d_weights_dev, int ckpt_stride, void* stream)
{
    if (!h || !state || !belief || !knots_dev || !cost_dev)
        return fail(DR_ERR_INVALID_ARG, "NULL argument");
    if (h->envKind != 0)
        return fail(DR_ERR_UNSUPPORTED, "the gradient path is built for the strategic race");
    if (n < 1 || n > 65535)
        return fail(DR_ERR_INVALID_ARG, "n must be in [1, 65535]");
    if (ckpt_stride < 0 || ckpt_stride > h->T)
        return fail(DR_ERR_INVALID_ARG, "ckpt_stride must be in [0, n_timesteps]");
    const int ck = ckpt_stride ? ckpt_stride : gradDefaultStride(h->nopp, h->nth, h->T, h->M, h->spl);
    const size_t smem = gradSmem(h->nopp, h->nth, h->T, h->M, ck, h->spl);
    if (smem > 227 * 1024)
        return fail(DR_ERR_INVALID_ARG, "checkpoint stride x horizon too large for shared memory");
    CK(cudaSetDevice(h->device));
    cudaStream_t s = (cudaStream_t)stream;
    if (!h->dGradIn)
        CK(cudaMalloc(&h->dGradIn, sizeof(MppiIn)));
    if (h->gradJobsCap < n)
    {
        CK(cudaStreamSynchronize(s));
        cudaFree(h->dGradJobs);
        h->dGradJobs = nullptr;
        h->gradJobsCap = 0;
        CK(cudaMalloc(&h->dGradJobs, sizeof(GradJob) * (size_t)n));
        h->gradJobsCap = n;
    }
    const MppiIn in = h->input(*state, belief);
    const size_t nU = (size_t)h->nbp * h->M * 2;
    std::vector<GradJob> jobs((size_t)n);
    for (int i = 0; i < n; i++)
    {
        GradJob& j = jobs[(size_t)i];
        j = GradJob{};
        j.D = h->self->dDesc;
        j.in = h->dGradIn;
        j.U = knots_dev + nU * (size_t)i;
        j.w6 = weights_dev ? weights_dev + (size_t)DR_GRAD_WEIGHTS * i : nullptr;
        j.J = cost_dev + i;
        j.gU = d_knots_dev ? d_knots_dev + nU * (size_t)i : nullptr;
        j.gW = d_weights_dev ? d_weights_dev + (size_t)DR_GRAD_WEIGHTS * i : nullptr;
        j.iters = 0;
        j.ckpt = ck;
    }
    // pageable sources: both copies are staged before the calls return
    CK(cudaMemcpyAsync(h->dGradIn, &in, sizeof(MppiIn), cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(h->dGradJobs, jobs.data(), sizeof(GradJob) * jobs.size(), cudaMemcpyHostToDevice, s));
    CK(launchGradNominal(s, h->dGradJobs, n, h->nopp, h->nth, h->spl, smem));
    return DR_OK;
}

int dr_mppi_set_step(dr_mppi* h, uint64_t step)
{
    if (!h)
        return fail(DR_ERR_INVALID_ARG, "NULL handle");
    h->step = step;
    return DR_OK;
}

int dr_mppi_set_profiling(dr_mppi* h, int on)
{
    if (!h)
        return fail(DR_ERR_INVALID_ARG, "NULL handle");
    h->self->profiling = on != 0;
    h->self->timer.reset();
    h->self->timerSide.reset();
    return DR_OK;
}

int dr_mppi_get_kernel_times(dr_mppi* h, const char** names, float* ms, int n, int* count)
{
    if (!h)
        return fail(DR_ERR_INVALID_ARG, "NULL handle");
    return kernelTimes(h->self->timer, names, ms, n, count, &h->self->timerSide);
}

int dr_mppi_batch_create(dr_mppi* const* hs, int n, void* stream, dr_mppi_batch** out)
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
    return buildMppiBatch(hs, n, s, own, out);
}

int dr_mppi_batch_destroy(dr_mppi_batch* b)
{
    if (!b)
        return DR_OK;
    cudaSetDevice(b->device);
    cudaStreamSynchronize(b->stream);
    b->release();
    delete b;
    return DR_OK;
}

int dr_mppi_batch_step(dr_mppi_batch* b, const dr_sim_state* states, const float* beliefs, float* out_actions, dr_mppi_info* infos)
{
    if (!b || !states || !beliefs || !out_actions)
        return fail(DR_ERR_INVALID_ARG, "NULL argument");
    return b->step(states, beliefs, DR_MAX_THETA, out_actions, infos);
}

int dr_gate_mppi_batch_step(dr_mppi_batch* b, const dr_gate_state* states, const float* beliefs, float* out_actions, dr_mppi_info* infos)
{
    if (!b || !states || !beliefs || !out_actions)
        return fail(DR_ERR_INVALID_ARG, "NULL argument");
    return b->step(states, beliefs, DR_MAX_THETA, out_actions, infos);
}

int dr_mppi_batch_set_graph(dr_mppi_batch* b, int use_graph)
{
    if (!b)
        return fail(DR_ERR_INVALID_ARG, "NULL batch");
    b->useGraph = use_graph != 0;
    return DR_OK;
}

// Device-resident step for throughput measurement: inputs are MppiIn-compatible states
// and beliefs already on the device; the controllers' host state (temperature, shift
// decision, step counter) is not advanced and no results are copied back.
int dr_mppi_batch_step_dev(dr_mppi_batch* b, const dr_sim_state* states_dev, const float* beliefs_dev)
{
    if (!b || !states_dev || !beliefs_dev)
        return fail(DR_ERR_INVALID_ARG, "NULL argument");
    CK(cudaSetDevice(b->device));
    int prc = b->pullDeviceControl();
    if (prc)
        return prc;
    const int n = (int)b->hs.size();
    for (int i = 0; i < n; i++)
    {
        MppiIn tmp = b->hs[i]->input(dr_sim_state{}, std::vector<float>(DR_MAX_THETA, 0.0f).data());
        b->hIn[i] = tmp;
    }
    // a gate-race batch takes dr_gate_state records
    const size_t stBytes = b->envKind ? sizeof(dr_gate_state) : sizeof(dr_sim_state);
    // host part of the record (temperature, step, pending shift), then state and belief device-to-device
    CK(cudaMemcpyAsync(b->dIn, b->hIn, sizeof(MppiIn) * n, cudaMemcpyHostToDevice, b->stream));
    for (int i = 0; i < n; i++)
    {
        CK(cudaMemcpyAsync(&b->dIn[i].state, (const unsigned char*)states_dev + i * stBytes, stBytes, cudaMemcpyDeviceToDevice, b->stream));
        CK(cudaMemcpyAsync(&b->dIn[i].belief, beliefs_dev + (size_t)i * DR_MAX_THETA, DR_MAX_THETA * 4, cudaMemcpyDeviceToDevice, b->stream));
    }
    return b->launchAll(b->dIn, b->profiling, &b->timer);
}

int dr_mppi_batch_step_device(dr_mppi_batch* b, const void* states_dev, const float* beliefs_dev, float* actions_dev, dr_mppi_info* infos_dev)
{
    if (!b || !states_dev || !beliefs_dev || !actions_dev || !infos_dev)
        return fail(DR_ERR_INVALID_ARG, "NULL argument");
    return b->stepDevice(states_dev, beliefs_dev, actions_dev, infos_dev);
}

int dr_mppi_batch_predict_device(dr_mppi_batch* b, const void* states_dev, const float* beliefs_dev, float* positions_dev, float* actions_dev,
                                 int32_t* records_dev, float* costs_dev, int t_stride)
{
    if (!b || !states_dev || !beliefs_dev || !positions_dev || !actions_dev || !records_dev || !costs_dev)
        return fail(DR_ERR_INVALID_ARG, "NULL argument");
    if (b->envKind != 0)
        return fail(DR_ERR_UNSUPPORTED, "predictions are built for the strategic race");
    for (auto* h : b->hs)
        if (h->T > t_stride)
            return fail(DR_ERR_INVALID_ARG, "t_stride is below a controller's horizon");
    if (!b->devCtl)
        return fail(DR_ERR_STATE, "the batch's device records hold no step yet: step it with dr_mppi_batch_step_device first");
    CK(cudaSetDevice(b->device));
    PredictOut out{positions_dev, actions_dev, records_dev, costs_dev, t_stride};
    CK(launchMppiPredict(b->stream, b->nopp, b->nth, b->dDesc, b->dIn, (const dr_sim_state*)states_dev, beliefs_dev, DR_MAX_THETA, out,
                         (int)b->hs.size()));
    return DR_OK;
}

int dr_mppi_batch_env_step_device(dr_mppi_batch* b, const int32_t* true_theta_dev, const float* actions_dev, void* states_dev, float* beliefs_dev,
                                  int update_belief, uint64_t seed, int32_t* terms_dev)
{
    if (!b || !true_theta_dev || !actions_dev || !states_dev || !beliefs_dev || !terms_dev)
        return fail(DR_ERR_INVALID_ARG, "NULL argument");
    if (!b->devCtl)
        return fail(DR_ERR_STATE, "step the batch with dr_mppi_batch_step_device first");
    CK(cudaSetDevice(b->device));
    const uint32_t k0 = (uint32_t)seed, k1 = (uint32_t)(seed >> 32);
    const int n = (int)b->hs.size();
    if (b->envKind)
        CK(launchGateBatchEnvStep(b->stream, b->nth, b->iMppi, b->dDesc, b->dIn, n, true_theta_dev, actions_dev, (dr_gate_state*)states_dev, beliefs_dev,
                                  update_belief, k0, k1, terms_dev));
    else
        CK(launchBatchEnvStep(b->stream, b->nopp, b->nth, b->dDesc, b->dIn, n, true_theta_dev, actions_dev, (dr_sim_state*)states_dev, beliefs_dev,
                              update_belief, k0, k1, terms_dev));
    return DR_OK;
}

int dr_debug_cp(const uint32_t* k, int n, uint32_t N, double alpha, int upper, double* out)
{
    if (!k || !out || n < 1)
        return fail(DR_ERR_INVALID_ARG, "bad argument");
    uint32_t* dk = nullptr;
    double* dout = nullptr;
    cudaError_t e = cudaMalloc(&dk, sizeof(uint32_t) * n);
    if (e == cudaSuccess)
        e = cudaMalloc(&dout, sizeof(double) * n);
    if (e == cudaSuccess)
        e = cudaMemcpy(dk, k, sizeof(uint32_t) * n, cudaMemcpyHostToDevice);
    if (e == cudaSuccess)
        e = launchCp(nullptr, dk, n, N, alpha, upper, dout);
    if (e == cudaSuccess)
        e = cudaMemcpy(out, dout, sizeof(double) * n, cudaMemcpyDeviceToHost);
    cudaFree(dk);
    cudaFree(dout);
    CK(e);
    return DR_OK;
}

int dr_debug_cp_host(const uint32_t* k, int n, uint32_t N, double alpha, int upper, double* out)
{
    if (!k || !out || n < 1)
        return fail(DR_ERR_INVALID_ARG, "bad argument");
    ClopperPearson cp;
    for (int i = 0; i < n; i++)
        out[i] = upper ? cp.upper(k[i], N, alpha) : cp.lower(k[i], N, alpha);
    return DR_OK;
}

// ---- test hooks -------------------------------------------------------------------------------

int dr_mppi_debug_noise(dr_mppi* h, float* noise, size_t n)
{
    size_t need = (size_t)h->nbp * h->M * h->K * 2;
    if (!h || !noise || n < need)
        return fail(DR_ERR_INVALID_ARG, "output too small");
    CK(cudaSetDevice(h->device));
    dr_mppi_batch* b = h->self;
    b->hIn[0] = h->input(dr_sim_state{}, std::vector<float>(DR_MAX_THETA, 0.0f).data());
    float* d = nullptr;
    CK(cudaMalloc(&d, need * 4));
    cudaMemcpyAsync(b->dIn, b->hIn, sizeof(MppiIn), cudaMemcpyHostToDevice, h->stream);
    LaunchArgs a = b->args(nullptr, 0, b->dIn);
    cudaError_t e = launchMppiNoise(a, need / 2, d);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(noise, d, need * 4, cudaMemcpyDeviceToHost, h->stream);
    if (e == cudaSuccess)
        e = cudaStreamSynchronize(h->stream);
    cudaFree(d);
    CK(e);
    return DR_OK;
}

extern "C++" {
template <class St> static int applyPending(dr_mppi* h, const St* state, const float* belief)
{
    dr_mppi_batch* b = h->self;
    b->hIn[0] = h->input(*state, belief);
    CK(cudaMemcpyAsync(b->dIn, b->hIn, sizeof(MppiIn), cudaMemcpyHostToDevice, h->stream));
    CK(launchMppiPrologue(b->args(nullptr, 0, b->dIn), 1, b->proSmem));
    // the shift is now applied; the next step must not apply it again
    h->pendBranch = -1;
    b->hIn[0].pendBranch = -1;
    CK(cudaMemcpyAsync(b->dIn, b->hIn, sizeof(MppiIn), cudaMemcpyHostToDevice, h->stream));
    return DR_OK;
}
} // extern "C++"

extern "C++" {
template <class St>
static int debugRollout(dr_mppi* h, const St* state, const float* belief, float* costs_true, int32_t* branch_used, int32_t* branch_time, float* costs)
{
    if (!h || !state || !belief)
        return fail(DR_ERR_INVALID_ARG, "NULL argument");
    if (h->envKind != (std::is_same<St, dr_gate_state>::value ? 1 : 0))
        return fail(DR_ERR_INVALID_ARG, "state type does not match the controller's environment");
    CK(cudaSetDevice(h->device));
    int rc = applyPending(h, state, belief);
    if (rc)
        return rc;
    dr_mppi_batch* b = h->self;
    CK(b->launchRollout(b->args(b->dRoll, b->nRoll, b->dIn)));
    const size_t nk = (size_t)h->nth * h->K;
    std::vector<int> info(nk);
    if (costs_true)
        CK(cudaMemcpyAsync(costs_true, h->desc.costsTrue, nk * 4, cudaMemcpyDeviceToHost, h->stream));
    CK(cudaMemcpyAsync(info.data(), h->desc.binfo, nk * 4, cudaMemcpyDeviceToHost, h->stream));
    if (costs)
        CK(cudaMemcpyAsync(costs, h->desc.costs, (size_t)h->nbp * h->K * 4, cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    for (size_t i = 0; i < nk; i++)
    {
        if (branch_used)
            branch_used[i] = info[i] >> 16;
        if (branch_time)
            branch_time[i] = (int)(short)(info[i] & 0xffff);
    }
    return DR_OK;
}
} // extern "C++"

int dr_mppi_debug_rollout(dr_mppi* h, const dr_sim_state* state, const float* belief, float* costs_true, int32_t* branch_used, int32_t* branch_time,
                          float* costs)
{
    return debugRollout(h, state, belief, costs_true, branch_used, branch_time, costs);
}

int dr_gate_mppi_debug_rollout(dr_mppi* h, const dr_gate_state* state, const float* belief, float* costs_true, int32_t* branch_used,
                               int32_t* branch_time, float* costs)
{
    return debugRollout(h, state, belief, costs_true, branch_used, branch_time, costs);
}

int dr_mppi_debug_update(dr_mppi* h, const float* belief, const float* costs_true, const int32_t* branch_used, const int32_t* branch_time,
                         float* dense_nominal, float* min_costs, float* nu)
{
    if (!h || !belief || !costs_true || !branch_used || !branch_time)
        return fail(DR_ERR_INVALID_ARG, "NULL argument");
    CK(cudaSetDevice(h->device));
    dr_sim_state st{};
    int rc = applyPending(h, &st, belief);
    if (rc)
        return rc;
    dr_mppi_batch* b = h->self;
    const size_t nk = (size_t)h->nth * h->K;
    std::vector<int> info(nk);
    for (size_t i = 0; i < nk; i++)
        info[i] = (branch_used[i] << 16) | (branch_time[i] & 0xffff);
    CK(cudaMemcpyAsync(h->desc.costsTrue, costs_true, nk * 4, cudaMemcpyHostToDevice, h->stream));
    CK(cudaMemcpyAsync(h->desc.binfo, info.data(), nk * 4, cudaMemcpyHostToDevice, h->stream));
    CK(launchMppiAggregate(b->args(nullptr, 0, b->dIn), h->nth, h->K));
    CK(launchMppiUpdate(b->args(b->dUpd, b->nUpd, b->dIn), h->nth));
    if (dense_nominal)
        CK(cudaMemcpyAsync(dense_nominal, h->desc.dense, (size_t)h->nbp * h->T * 2 * 4, cudaMemcpyDeviceToHost, h->stream));
    if (min_costs)
        CK(cudaMemcpyAsync(min_costs, h->desc.minCosts, (size_t)h->nbp * h->M * 4, cudaMemcpyDeviceToHost, h->stream));
    if (nu)
        CK(cudaMemcpyAsync(nu, h->desc.nu, (size_t)h->nbp * 4, cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    return DR_OK;
}

extern "C++" {
template <class St>
static int debugVerify(dr_mppi* h, const St* state, const float* belief, const float* dense_plan, int plan, uint32_t* fail_count, int32_t* fail_time,
                       int32_t* thetas)
{
    if (!h || !state || !belief || !dense_plan || plan < 0 || plan > 1 || h->V <= 0)
        return fail(DR_ERR_INVALID_ARG, "bad argument (verification disabled?)");
    if (h->envKind != (std::is_same<St, dr_gate_state>::value ? 1 : 0))
        return fail(DR_ERR_INVALID_ARG, "state type does not match the controller's environment");
    CK(cudaSetDevice(h->device));
    const int V = h->V, T = h->T;
    // a private copy of the instance with its own plan and histogram buffers
    MppiDev D = h->desc;
    float* dPlan = nullptr;
    unsigned* dFail = nullptr;
    int *dFt = nullptr, *dTh = nullptr, *dStats = nullptr;
    MppiDev* dD = nullptr;
    MppiIn* dIn = nullptr;
    Tile* dT = nullptr;
    std::vector<Tile> tiles;
    for (int v0 = 0; v0 < V; v0 += VERIFY_TILE)
        tiles.push_back(Tile{0, v0, std::min(VERIFY_TILE, V - v0), plan});
    size_t planBytes = a16((size_t)h->nbp * T * 2 * 4);
    cudaError_t e = cudaMalloc(&dPlan, planBytes);
    if (e == cudaSuccess)
        e = cudaMalloc(&dFail, 2 * T * 4);
    if (e == cudaSuccess)
        e = cudaMalloc(&dFt, V * 4);
    if (e == cudaSuccess)
        e = cudaMalloc(&dTh, V * 4);
    if (e == cudaSuccess)
        e = cudaMalloc(&dStats, 16);
    if (e == cudaSuccess)
        e = cudaMalloc(&dD, sizeof(MppiDev));
    if (e == cudaSuccess)
        e = cudaMalloc(&dIn, sizeof(MppiIn));
    if (e == cudaSuccess)
        e = cudaMalloc(&dT, sizeof(Tile) * tiles.size());
    if (e == cudaSuccess)
    {
        D.dense = dPlan;
        D.prevDense = dPlan;
        D.fail = dFail;
        D.stats = dStats;
        MppiIn in = h->input(*state, belief);
        cudaMemsetAsync(dFail, 0, 2 * T * 4, h->stream);
        cudaMemsetAsync(dStats, 0, 16, h->stream);
        cudaMemcpyAsync(dPlan, dense_plan, (size_t)h->nbp * T * 2 * 4, cudaMemcpyHostToDevice, h->stream);
        cudaMemcpyAsync(dD, &D, sizeof(MppiDev), cudaMemcpyHostToDevice, h->stream);
        cudaMemcpyAsync(dIn, &in, sizeof(MppiIn), cudaMemcpyHostToDevice, h->stream);
        cudaMemcpyAsync(dT, tiles.data(), sizeof(Tile) * tiles.size(), cudaMemcpyHostToDevice, h->stream);
        LaunchArgs a;
        a.stream = h->stream;
        a.mppi = dD;
        a.mppiIn = dIn;
        a.tiles = dT;
        a.nTiles = (int)tiles.size();
        a.exactVerify = h->exactVerify ? 1 : 0;
        a.egoTable = h->envKind == 0 && h->egoTableUsable() ? 1 : 0;
        if (a.egoTable)
            e = launchEgoTable(h->stream, h->nopp, h->nth, dD, dIn, 1, plan, h->H);
        if (e == cudaSuccess)
            e = h->envKind ? launchGateVerify(a, h->nth, h->iMppi, gateVerifySmem(h->nth, T), dFt, dTh)
                       : launchMppiVerify(a, h->nopp, h->nth, mppiVerifySmem(h->nth, T), dFt, dTh);
        std::vector<unsigned> fc(2 * T);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(fc.data(), dFail, 2 * T * 4, cudaMemcpyDeviceToHost, h->stream);
        if (e == cudaSuccess && fail_time)
            e = cudaMemcpyAsync(fail_time, dFt, V * 4, cudaMemcpyDeviceToHost, h->stream);
        if (e == cudaSuccess && thetas)
            e = cudaMemcpyAsync(thetas, dTh, V * 4, cudaMemcpyDeviceToHost, h->stream);
        if (e == cudaSuccess)
            e = cudaStreamSynchronize(h->stream);
        if (e == cudaSuccess && fail_count)
            std::memcpy(fail_count, fc.data() + plan * T, T * 4);
    }
    cudaFree(dPlan);
    cudaFree(dFail);
    cudaFree(dFt);
    cudaFree(dTh);
    cudaFree(dStats);
    cudaFree(dD);
    cudaFree(dIn);
    cudaFree(dT);
    CK(e);
    return DR_OK;
}
} // extern "C++"

int dr_mppi_debug_verify(dr_mppi* h, const dr_sim_state* state, const float* belief, const float* dense_plan, int plan, uint32_t* fail_count,
                         int32_t* fail_time, int32_t* thetas)
{
    return debugVerify(h, state, belief, dense_plan, plan, fail_count, fail_time, thetas);
}

int dr_mppi_predict(dr_mppi* h, const dr_sim_state* state, const float* belief, float* positions, float* actions, int32_t* records, float* costs)
{
    if (!h || !state || !belief || !positions || !actions || !records || !costs)
        return fail(DR_ERR_INVALID_ARG, "NULL argument");
    if (h->envKind != 0)
        return fail(DR_ERR_UNSUPPORTED, "predictions are built for the strategic race");
    CK(cudaSetDevice(h->device));
    const int nth = h->nth, T = h->T, na = h->nopp + 1;
    const size_t nPos = (size_t)nth * T * 2 * na, nAct = (size_t)nth * T * 2, nRec = (size_t)nth * PREDICT_RECORD;
    const size_t oIn = 0, oSt = a256(sizeof(MppiIn)), oBel = oSt + a256(sizeof(dr_sim_state)), oPos = oBel + a256(DR_MAX_THETA * 4),
                 oAct = oPos + a256(nPos * 4), oRec = oAct + a256(nAct * 4), oCost = oRec + a256(nRec * 4), total = oCost + a256((size_t)nth * 4);
    CK(h->predBuf.reserve(total));
    unsigned char* base = (unsigned char*)h->predBuf.p;
    // the record carries the pending warm-start shift that the engine's h_nominal holds
    MppiIn in = h->input(*state, belief);
    float bel[DR_MAX_THETA] = {};
    for (int i = 0; i < nth; i++)
        bel[i] = belief[i];
    CK(cudaMemcpyAsync(base + oIn, &in, sizeof(MppiIn), cudaMemcpyHostToDevice, h->stream));
    CK(cudaMemcpyAsync(base + oSt, state, sizeof(dr_sim_state), cudaMemcpyHostToDevice, h->stream));
    CK(cudaMemcpyAsync(base + oBel, bel, sizeof(bel), cudaMemcpyHostToDevice, h->stream));
    PredictOut out{(float*)(base + oPos), (float*)(base + oAct), (int*)(base + oRec), (float*)(base + oCost), T};
    CK(launchMppiPredict(h->stream, h->nopp, nth, h->self->dDesc, (const MppiIn*)(base + oIn), (const dr_sim_state*)(base + oSt),
                         (const float*)(base + oBel), DR_MAX_THETA, out, 1));
    CK(cudaMemcpyAsync(positions, base + oPos, nPos * 4, cudaMemcpyDeviceToHost, h->stream));
    CK(cudaMemcpyAsync(actions, base + oAct, nAct * 4, cudaMemcpyDeviceToHost, h->stream));
    CK(cudaMemcpyAsync(records, base + oRec, nRec * 4, cudaMemcpyDeviceToHost, h->stream));
    CK(cudaMemcpyAsync(costs, base + oCost, (size_t)nth * 4, cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    return DR_OK;
}

int dr_mppi_set_verify_exact(dr_mppi* h, int on)
{
    if (!h)
        return fail(DR_ERR_INVALID_ARG, "NULL handle");
    CK(cudaSetDevice(h->device));
    CK(cudaStreamSynchronize(h->stream));
    h->exactVerify = on != 0;
    // the controller's own batch of one captured its verification kernels in its graphs
    h->self->dropGraph();
    h->self->dropDevGraph();
    return DR_OK;
}

int dr_mppi_set_ego_table(dr_mppi* h, int on)
{
    if (!h)
        return fail(DR_ERR_INVALID_ARG, "NULL handle");
    CK(cudaSetDevice(h->device));
    CK(cudaStreamSynchronize(h->stream));
    h->egoTableOn = on != 0;
    h->self->dropGraph();
    h->self->dropDevGraph();
    return DR_OK;
}

int dr_mppi_debug_stage_timeout(dr_mppi* h, int on, int polls)
{
    if (!h)
        return fail(DR_ERR_INVALID_ARG, "NULL handle");
    CK(cudaSetDevice(h->device));
    CK(cudaStreamSynchronize(h->stream));
    h->desc.cfg.dbgNoStage = on ? 1 : 0;
    h->desc.cfg.waitPolls = polls > 0 ? polls : 0;
    // the controller's own batch of one: re-upload its descriptor; its captured graph
    // keeps pointers only, so it needs no rebuild
    return h->self->uploadDescs();
}

int dr_gate_mppi_debug_verify(dr_mppi* h, const dr_gate_state* state, const float* belief, const float* dense_plan, int plan, uint32_t* fail_count,
                              int32_t* fail_time, int32_t* thetas)
{
    return debugVerify(h, state, belief, dense_plan, plan, fail_count, fail_time, thetas);
}

} // extern "C"

extern "C" int dr_mppi_batch_set_profiling(dr_mppi_batch* b, int on)
{
    if (!b)
        return fail(DR_ERR_INVALID_ARG, "NULL batch");
    b->profiling = on != 0;
    b->timer.reset();
    b->timerSide.reset();
    return DR_OK;
}

extern "C" int dr_mppi_batch_get_kernel_times(dr_mppi_batch* b, const char** names, float* ms, int n, int* count)
{
    if (!b)
        return fail(DR_ERR_INVALID_ARG, "NULL batch");
    CK(cudaSetDevice(b->device));
    return kernelTimes(b->timer, names, ms, n, count, &b->timerSide);
}

extern "C" int dr_mppi_batch_get_kernel_timeline(dr_mppi_batch* b, const char** names, float* start_ms, float* end_ms, int n, int* count)
{
    if (!b)
        return fail(DR_ERR_INVALID_ARG, "NULL batch");
    CK(cudaSetDevice(b->device));
    return kernelTimeline(b->timer, names, start_ms, end_ms, n, count, &b->timerSide);
}

extern "C" int dr_mppi_batch_set_overlap(dr_mppi_batch* b, int on)
{
    if (!b)
        return fail(DR_ERR_INVALID_ARG, "NULL batch");
    CK(cudaSetDevice(b->device));
    CK(cudaStreamSynchronize(b->stream));
    b->dropGraph();
    b->dropDevGraph();
    b->overlap = on != 0;
    return DR_OK;
}

extern "C" int dr_mppi_batch_set_priority(dr_mppi_batch* b, int on)
{
    if (!b)
        return fail(DR_ERR_INVALID_ARG, "NULL batch");
    CK(cudaSetDevice(b->device));
    CK(cudaStreamSynchronize(b->stream));
    b->dropGraph();
    b->dropDevGraph();
    b->prio = on != 0;
    return DR_OK;
}

namespace
{
// Resolves a requested CTAs-per-SM count for a persistent launch: -1 = as many as fit.
int resolvePerSm(const dr_mppi_batch* b, int req, bool verification, int* out)
{
    if (req == 0)
    {
        *out = 0;
        return DR_OK;
    }
    const int fit = mppiResident(b->nopp, b->nth, verification, b->spl, verification ? b->verSmem : b->rollSmem);
    if (fit <= 0)
        return fail(DR_ERR_CUDA, "persistent launch: no CTA of this kernel fits on an SM");
    if (req < 0)
        req = fit;
    if (req > fit)
        return fail(DR_ERR_INVALID_ARG, "persistent launch: " + std::to_string(req) + " CTAs per SM requested, " + std::to_string(fit) + " fit");
    *out = req;
    return DR_OK;
}

// A candidate launch shape replaces the current choice only when it is faster by more
// than 2 %; the default shape is timed first.
constexpr float TUNE_MARGIN = 0.98f;

// Median device time of `reps` runs of `launch` on `s` (after one untimed run).
template <typename F> int timeLaunch(cudaStream_t s, int reps, F launch, float* ms)
{
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    std::vector<float> t;
    int rc = DR_OK;
    for (int r = -1; r < reps && rc == DR_OK; r++)
    {
        cudaError_t e = cudaEventRecord(e0, s);
        if (e == cudaSuccess)
            e = launch();
        if (e == cudaSuccess)
            e = cudaEventRecord(e1, s);
        if (e == cudaSuccess)
            e = cudaEventSynchronize(e1);
        float x = 0.0f;
        if (e == cudaSuccess)
            e = cudaEventElapsedTime(&x, e0, e1);
        if (e != cudaSuccess)
            rc = fail(DR_ERR_CUDA, std::string("autotune: ") + cudaGetErrorString(e));
        else if (r >= 0)
            t.push_back(x);
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (rc)
        return rc;
    std::sort(t.begin(), t.end());
    *ms = t[t.size() / 2];
    return DR_OK;
}
} // namespace

extern "C" int dr_mppi_batch_set_persistent(dr_mppi_batch* b, int rollout_ctas_per_sm, int verify_ctas_per_sm, int rollout_lockstep)
{
    if (!b)
        return fail(DR_ERR_INVALID_ARG, "NULL batch");
    if (b->envKind != 0 && (rollout_ctas_per_sm != 0 || verify_ctas_per_sm != 0 || rollout_lockstep != 0))
        return fail(DR_ERR_UNSUPPORTED, "persistent launches are built for the strategic race");
    CK(cudaSetDevice(b->device));
    int r = 0, v = 0;
    int rc = resolvePerSm(b, rollout_ctas_per_sm, false, &r);
    if (rc)
        return rc;
    rc = resolvePerSm(b, verify_ctas_per_sm, true, &v);
    if (rc)
        return rc;
    CK(cudaStreamSynchronize(b->stream));
    b->dropGraph();
    b->dropDevGraph();
    b->rollPerSm = r;
    b->verPerSm = v;
    b->rollLock = rollout_lockstep != 0;
    return DR_OK;
}

extern "C" int dr_mppi_batch_set_pdl(dr_mppi_batch* b, int on)
{
    if (!b)
        return fail(DR_ERR_INVALID_ARG, "NULL batch");
    CK(cudaSetDevice(b->device));
    CK(cudaStreamSynchronize(b->stream));
    b->dropGraph();
    b->dropDevGraph();
    b->pdl = on != 0;
    return DR_OK;
}

extern "C" int dr_mppi_batch_set_side_verify(dr_mppi_batch* b, int ctas_per_sm)
{
    if (!b)
        return fail(DR_ERR_INVALID_ARG, "NULL batch");
    if (b->envKind != 0 && ctas_per_sm != 0)
        return fail(DR_ERR_UNSUPPORTED, "persistent launches are built for the strategic race");
    CK(cudaSetDevice(b->device));
    int v = 0;
    int rc = resolvePerSm(b, ctas_per_sm, true, &v);
    if (rc)
        return rc;
    CK(cudaStreamSynchronize(b->stream));
    b->dropGraph();
    b->dropDevGraph();
    b->sidePerSm = v;
    return DR_OK;
}

extern "C" int dr_mppi_batch_autotune(dr_mppi_batch* b, int reps, dr_tune_report* out)
{
    if (!b)
        return fail(DR_ERR_INVALID_ARG, "NULL batch");
    if (reps < 1 || reps > 1000)
        return fail(DR_ERR_INVALID_ARG, "reps must be in 1..1000");
    if (b->runs == 0 && !b->devCtl)
        return fail(DR_ERR_STATE, "autotune needs one completed step of the batch");
    CK(cudaSetDevice(b->device));
    CK(cudaStreamSynchronize(b->stream));
    dr_tune_report rep{};
    cudaStream_t s = b->stream;
    const bool persistOk = b->envKind == 0;
    // rollout grid (one CTA per tile, or the two fullest persistent grids) x lockstep
    {
        std::vector<int> cand{0};
        const int fit = persistOk ? mppiResident(b->nopp, b->nth, false, b->spl, b->rollSmem) : 0;
        for (int c : {fit - 1, fit})
            if (c >= 1 && std::find(cand.begin(), cand.end(), c) == cand.end())
                cand.push_back(c);
        float best = INFINITY;
        for (int lock = 0; lock < 2; lock++)
            for (int c : cand)
            {
                if (rep.n_rollout >= DR_TUNE_MAX_CANDIDATES)
                    break;
                float ms = 0.0f;
                int rc = timeLaunch(
                    s, reps, [&] { return b->launchQueued(b->qargs(b->dRoll, b->nRoll, b->dIn, dr_mppi_batch::Q_ROLL, c, s, lock), false); }, &ms);
                if (rc)
                    return rc;
                rep.rollout_cand[rep.n_rollout] = c;
                rep.rollout_lock[rep.n_rollout] = lock;
                rep.rollout_ms[rep.n_rollout++] = ms;
                // the first candidate is the default shape; another replaces it only when
                // faster by more than the tuner's margin (launch-to-launch spread)
                if (rep.n_rollout == 1 ? true : ms < best * TUNE_MARGIN)
                {
                    best = ms;
                    rep.rollout_ctas_per_sm = c;
                    rep.rollout_lockstep = lock;
                }
            }
    }
    // verification grid (both plans in one launch)
    if (b->verify && b->nVer > 0)
    {
        std::vector<int> cand{0};
        const int fit = persistOk ? mppiResident(b->nopp, b->nth, true, b->spl, b->verSmem) : 0;
        for (int c = 1; c <= fit && (int)cand.size() < DR_TUNE_MAX_CANDIDATES; c++)
            cand.push_back(c);
        float best = INFINITY;
        for (int c : cand)
        {
            float ms = 0.0f;
            int rc = timeLaunch(s, reps, [&] { return b->launchQueued(b->qargs(b->dVer, b->nVer, b->dIn, dr_mppi_batch::Q_VER_ALL, c, s), true); }, &ms);
            if (rc)
                return rc;
            rep.verify_cand[rep.n_verify] = c;
            rep.verify_ms[rep.n_verify++] = ms;
            if (rep.n_verify == 1 ? true : ms < best * TUNE_MARGIN)
            {
                best = ms;
                rep.verify_ctas_per_sm = c;
            }
        }
    }
    // checkpoint stride of the gradient refinement, timed without writing the plans
    if (b->nGrad > 0)
    {
        std::vector<int> cand{0};
        int maxT = 0;
        for (auto* h : b->hs)
            if (h->gradSteps > 0)
                maxT = std::max(maxT, h->T);
        const int sq = (int)std::ceil(std::sqrt((double)maxT));
        for (int c : {1, sq, 2 * sq})
            if (c >= 1 && c <= maxT && std::find(cand.begin(), cand.end(), c) == cand.end())
                cand.push_back(c);
        std::vector<GradJob> base(b->nGrad);
        CK(cudaMemcpy(base.data(), b->dGrad, sizeof(GradJob) * b->nGrad, cudaMemcpyDeviceToHost));
        GradJob* dJobs = nullptr;
        CK(cudaMalloc(&dJobs, sizeof(GradJob) * b->nGrad));
        float best = INFINITY;
        int rc = DR_OK;
        for (int c : cand)
        {
            std::vector<GradJob> jobs = base;
            size_t smem = 0;
            bool fits = true;
            for (auto& j : jobs)
            {
                const dr_mppi* h = nullptr;
                for (size_t i = 0; i < b->hs.size(); i++)
                    if (j.D == b->dDesc + i)
                        h = b->hs[i];
                if (!h)
                    continue;
                j.write = 0;
                j.ckpt = c > 0 ? std::min(c, h->T) : gradDefaultStride(b->nopp, b->nth, h->T, h->M, b->spl);
                const size_t need = gradSmem(b->nopp, b->nth, h->T, h->M, j.ckpt, b->spl);
                if (need > 227 * 1024)
                    fits = false;
                smem = std::max(smem, need);
            }
            if (!fits)
                continue;
            if (cudaMemcpy(dJobs, jobs.data(), sizeof(GradJob) * jobs.size(), cudaMemcpyHostToDevice) != cudaSuccess)
            {
                rc = fail(DR_ERR_CUDA, "autotune: job copy failed");
                break;
            }
            float ms = 0.0f;
            rc = timeLaunch(s, reps, [&] { return launchGradNominal(s, dJobs, b->nGrad, b->nopp, b->nth, b->spl, smem); }, &ms);
            if (rc)
                break;
            rep.grad_cand[rep.n_grad] = c;
            rep.grad_ms[rep.n_grad++] = ms;
            if (rep.n_grad == 1 ? true : ms < best * TUNE_MARGIN)
            {
                best = ms;
                rep.grad_ckpt = c;
            }
        }
        cudaFree(dJobs);
        if (rc)
            return rc;
        for (auto* h : b->hs)
            if (h->gradSteps > 0)
                h->gradCkpt = rep.grad_ckpt > 0 ? std::min(rep.grad_ckpt, h->T) : gradDefaultStride(b->nopp, b->nth, h->T, h->M, b->spl);
        rc = b->setupGrad();
        if (rc)
            return rc;
    }
    b->dropGraph();
    b->dropDevGraph();
    b->rollPerSm = rep.rollout_ctas_per_sm;
    b->rollLock = rep.rollout_lockstep;
    b->verPerSm = rep.verify_ctas_per_sm;
    if (out)
        *out = rep;
    return DR_OK;
}

extern "C" int dr_spline_matrix(int T, int M, const int32_t* knots, float* out)
{
    if (T < 2 || M < 2 || M > DR_MAX_KNOTS || !knots || !out)
        return fail(DR_ERR_INVALID_ARG, "bad spline size or NULL pointer");
    for (int i = 0; i < M; i++)
        if (knots[i] < 0 || knots[i] >= T || (i > 0 && knots[i] <= knots[i - 1]))
            return fail(DR_ERR_INVALID_ARG, "knots must be strictly increasing inside [0, T)");
    std::vector<float> B = splineMatrix(T, M, knots);
    std::memcpy(out, B.data(), B.size() * sizeof(float));
    return DR_OK;
}
