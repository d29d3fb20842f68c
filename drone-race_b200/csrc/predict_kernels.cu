// Prediction streaming of the simulation engine on the device: the re-simulation that
// SimulationEngine::sendState (src/engine.cpp:55-264) runs on the host after every closed-
// loop step to show where the controller's plan leads, for every controller of a batch in
// one launch.
//
//   mppi_predict   MPPI (engine.cpp:73-166): from the state after the step, under every
//                  hypothesis theta, the controller's plan (its chosen plan with the
//                  warm-start shift the next step will apply, the engine's h_nominal) is
//                  rolled out for the horizon with the belief update and branching on
//                  (environmentStep<true, true, false>), noise off: the initial branch, the
//                  positions of every agent at every step (repeated after a terminal step),
//                  the ego actions taken, the branch taken and when, why and when it
//                  stopped, and the discounted running + terminal cost (the engine prints
//                  it, engine.cpp:139-141).
//   pr_predict     PR-MPPI (engine.cpp:167-240): from the state before the step, the new
//                  nominal plan under every hypothesis and the robust plan under the last
//                  one (environmentStep<false, false, false>), noise off, with the running,
//                  safety and terminal cost of PRMPPIstateCost / PRMPPIsafetyCost /
//                  PRMPPIfinalCost evaluated on the predicted states (the engine evaluates
//                  them on the unchanged current state, engine.cpp:221-222, and only prints
//                  them).
// One CTA per controller stages the track grids in shared memory; thread r computes row r
// (a hypothesis, or the robust plan).
#include <cstdio>

#include "common.cuh"
#include "instance.cuh"
#include "launch.h"

namespace dr
{

namespace
{

// The engine re-simulates with applyNoise = false: no draws, every noise term zero.
struct NoNoise
{
    __device__ __forceinline__ void begin_step(uint32_t)
    {
    }
    __device__ __forceinline__ float next()
    {
        return 0.0f;
    }
    __device__ __forceinline__ float2 next2()
    {
        return make_float2(0.0f, 0.0f);
    }
};

// EventType of the reference (include/protocol.h:17-23) for a terminal step (parseTerm,
// engine.cpp:365-380)
__device__ __forceinline__ int eventOf(int term)
{
    return term == TERM_LOSE ? 0 : term == TERM_WIN ? 1 : 2;
}
constexpr int EVT_TRUNCATED = 3;

__device__ __forceinline__ void stageTrack(float* sg, EnvParams& sE, const float* grids, const EnvParams& env)
{
    for (int i = threadIdx.x; i < GRID_FLOATS; i += blockDim.x)
        sg[i] = grids[i];
    for (int i = threadIdx.x; i < ENV_HOST_WORDS; i += blockDim.x)
        ((float*)&sE)[i] = ((const float*)&env)[i];
    envDeviceTerms(sE, env, threadIdx.x, blockDim.x);
}

template <int NA> __device__ __forceinline__ void loadPredState(DState<NA>& s, const dr_sim_state& st, float L)
{
#pragma unroll
    for (int a = 0; a < NA; a++)
    {
        s.pos[2 * a] = st.pos[2 * a];
        s.pos[2 * a + 1] = st.pos[2 * a + 1];
        s.vel[2 * a] = st.vel[2 * a];
        s.vel[2 * a + 1] = st.vel[2 * a + 1];
        s.S[a] = st.S[a];
        s.lat[a] = st.lat_dist[a];
        s.laps[a] = st.laps[a];
    }
    s.locate(L);
}

template <int NA> __device__ __forceinline__ void putPositions(float* out, const DState<NA>& s)
{
#pragma unroll
    for (int k = 0; k < 2 * NA; k++)
        out[k] = s.pos[k];
}

} // namespace

template <int NOPP, int NTH>
__global__ void __launch_bounds__(128) mppi_predict(const MppiDev* __restrict__ insts, const MppiIn* __restrict__ in,
                                                    const dr_sim_state* __restrict__ states, const float* __restrict__ beliefs, int beliefStride,
                                                    PredictOut out, int nInst)
{
    constexpr int NA = NOPP + 1;
    __shared__ float sg[GRID_FLOATS];
    __shared__ EnvParams sE;
    const int inst = blockIdx.x;
    if (inst >= nInst)
        return;
    const MppiDev& D = insts[inst];
    const MppiIn& I = in[inst];
    stageTrack(sg, sE, D.grids, D.env);
    __syncthreads();
    const int th = threadIdx.x;
    if (th >= NTH)
        return;
    const EnvParams& E = sE;
    const Track tr = trackIn(sg);
    const int T = D.cfg.T, nbp = NTH + 1;
    const size_t row = (size_t)inst * NTH + th;
    float* pos = out.pos + row * out.tStride * 2 * NA;
    float* act = out.act + row * out.tStride * 2;
    int* rec = out.rec + row * PREDICT_RECORD;
    // the controller's plan as the engine holds it: the chosen plan with the pending
    // warm-start shift of branch pendBranch (mppi_controller.cu:430-436)
    const float* plan = (I.pendBranch >= 0 && !I.pendUseNew) ? D.prevDense : D.dense;
    const int shiftB = (I.pendBranch >= 0 && I.pendBranch < nbp) ? I.pendBranch : -1;

    DState<NA> s;
    loadPredState<NA>(s, states[inst], E.trackLength);
    BState<NTH> bs;
    const float* belief = beliefs + (size_t)inst * beliefStride;
#pragma unroll
    for (int i = 0; i < NTH; i++)
        bs.belief[i] = belief[i];
    // initBranchState (state.h:154-163)
    bs.predTheta = findConfident<NTH>(bs.belief, D.cfg.minConf);
    bs.branchingTime = bs.predTheta == 0 ? -1 : 0;
    rec[0] = bs.predTheta;
    NoNoise rng;
    float cost = 0.0f, decay = 1.0f;
    int tOrigin = 0, stopTime = -1, stopReason = EVT_TRUNCATED;
    int t = 0;
    for (; t < T; t++)
    {
        const int b = bs.predTheta, local = t - tOrigin;
        float e0 = 0.0f, e1 = 0.0f;
        if (b == shiftB)
        {
            if (local + 1 < T)
            {
                e0 = plan[(b * T + local + 1) * 2];
                e1 = plan[(b * T + local + 1) * 2 + 1];
            }
        }
        else
        {
            e0 = plan[(b * T + local) * 2];
            e1 = plan[(b * T + local) * 2 + 1];
        }
        act[t * 2] = e0;
        act[t * 2 + 1] = e1;
        bool branched = false;
        StepOut o = envStep<NOPP, NTH, true, true, false, true>(t, th, tr, E, e0, e1, s, bs, branched, D.cfg.minConf, rng);
        if (branched)
            tOrigin = t + 1;
        putPositions<NA>(pos + (size_t)t * 2 * NA, s);
        cost += stateCost(o, E, D.cfg.w) * decay;
        decay *= DECAY;
        if (o.term != TERM_NONE)
        {
            stopTime = t;
            stopReason = eventOf(o.term);
            break;
        }
    }
    // after a terminal step the engine repeats the last state and leaves the actions zero
    for (int u = t + 1; u < T; u++)
    {
        putPositions<NA>(pos + (size_t)u * 2 * NA, s);
        act[u * 2] = 0.0f;
        act[u * 2 + 1] = 0.0f;
    }
    cost += finalCost<NOPP>(s, E, D.cfg.w.finalAdvWeight, D.cfg.w.finalOppAdvWeight);
    rec[1] = bs.branchingTime;
    rec[2] = bs.predTheta;
    rec[3] = stopReason;
    rec[4] = stopTime;
    out.cost[row] = cost;
}

template <int NOPP, int NTH>
__global__ void __launch_bounds__(128) pr_predict(const PrDev* __restrict__ insts, const dr_sim_state* __restrict__ prevStates, PredictOut out, int nInst)
{
    constexpr int NA = NOPP + 1;
    constexpr int ROWS = NTH + 1;
    __shared__ float sg[GRID_FLOATS];
    __shared__ EnvParams sE;
    const int inst = blockIdx.x;
    if (inst >= nInst)
        return;
    const PrDev& D = insts[inst];
    stageTrack(sg, sE, D.grids, D.env);
    __syncthreads();
    const int j = threadIdx.x;
    if (j >= ROWS)
        return;
    const EnvParams& E = sE;
    const Track tr = trackIn(sg);
    const int T = D.cfg.T;
    const int theta = j < NTH ? j : NTH - 1;
    const float* plan = j < NTH ? D.nom : D.rob;
    const size_t row = (size_t)inst * ROWS + j;
    float* pos = out.pos + row * out.tStride * 2 * NA;
    float* act = out.act + row * out.tStride * 2;
    int* rec = out.rec + row * PREDICT_RECORD;

    DState<NA> s;
    loadPredState<NA>(s, prevStates[inst], E.trackLength);
    BState<NTH> bs{};
    NoNoise rng;
    const SafetyMargin margin = safetyMargin(E, D.cfg.collDistFactor);
    float cost = 0.0f, safe = -INFINITY, decay = 1.0f;
    int stopTime = -1, stopReason = EVT_TRUNCATED;
    int t = 0;
    for (; t < T; t++)
    {
        const float e0 = plan[t * 2], e1 = plan[t * 2 + 1];
        act[t * 2] = e0;
        act[t * 2 + 1] = e1;
        bool branched = false;
        StepOut o = envStep<NOPP, NTH, false, false, false, false>(t, theta, tr, E, e0, e1, s, bs, branched, 0.0f, rng);
        safe = fmaxf(safe, prSafetyCost(o, margin));
        cost += prStateCost(o, E, D.cfg.boundaryThresholdFactor, D.cfg.boundaryCost, D.cfg.winCost, D.cfg.oppWinCost) * decay;
        decay *= DECAY;
        putPositions<NA>(pos + (size_t)t * 2 * NA, s);
        if (o.term != TERM_NONE)
        {
            stopTime = t;
            stopReason = eventOf(o.term);
            break;
        }
    }
    for (int u = t + 1; u < T; u++)
    {
        putPositions<NA>(pos + (size_t)u * 2 * NA, s);
        act[u * 2] = 0.0f;
        act[u * 2 + 1] = 0.0f;
    }
    cost += finalCost<NOPP>(s, E, D.cfg.finalAdvWeight, D.cfg.finalOppAdvWeight);
    rec[0] = 0;
    rec[1] = -1;
    rec[2] = 0;
    rec[3] = stopReason;
    rec[4] = stopTime;
    out.cost[row] = cost + (safe > 0.0f ? D.cfg.safetyWeight : 0.0f);
}

#define DR_PRED_DISPATCH(NOPP_, NTH_, CALL)                                                                                                          \
    switch (NOPP_ * 16 + NTH_)                                                                                                                       \
    {                                                                                                                                                \
    case 1 * 16 + 1: CALL(1, 1); break;                                                                                                              \
    case 1 * 16 + 2: CALL(1, 2); break;                                                                                                              \
    case 1 * 16 + 4: CALL(1, 4); break;                                                                                                              \
    case 1 * 16 + 8: CALL(1, 8); break;                                                                                                              \
    case 2 * 16 + 2: CALL(2, 2); break;                                                                                                              \
    default: return cudaErrorInvalidValue;                                                                                                           \
    }

cudaError_t launchMppiPredict(cudaStream_t stream, int nopp, int nth, const MppiDev* insts, const MppiIn* in, const dr_sim_state* states,
                              const float* beliefs, int beliefStride, const PredictOut& out, int nInst)
{
#define CALL(P, Q) mppi_predict<P, Q><<<nInst, 128, 0, stream>>>(insts, in, states, beliefs, beliefStride, out, nInst)
    DR_PRED_DISPATCH(nopp, nth, CALL)
#undef CALL
    return cudaGetLastError();
}

cudaError_t launchPrPredict(cudaStream_t stream, int nopp, int nth, const PrDev* insts, const dr_sim_state* prevStates, const PredictOut& out, int nInst)
{
#define CALL(P, Q) pr_predict<P, Q><<<nInst, 128, 0, stream>>>(insts, prevStates, out, nInst)
    DR_PRED_DISPATCH(nopp, nth, CALL)
#undef CALL
    return cudaGetLastError();
}

} // namespace dr
