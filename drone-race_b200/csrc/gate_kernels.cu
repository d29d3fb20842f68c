// MPPI kernels of the gate race (the reference's kernels.cu compiled with
// USE_ENV_DRONERACE): the rollout with per-branch cost aggregation and the plan
// verification, built like mppi_rollout / mppi_verify (one thread per (sample,
// hypothesis), resp. per verification sample; state in registers; racelines in shared
// memory, staged by a bulk copy; gate parameters copied to shared memory; perturbations
// from Philox) on the model of gate_model.cuh. The prologue and the update kernels of
// mppi_kernels.cu serve both environments (they see only costs, bookkeeping and plans).
#include <cstdio>

#include <type_traits>

#include "common.cuh"
#include "gate_model.cuh"
#include "instance.cuh"
#include "launch.h"

namespace dr
{

namespace
{

constexpr int GRB = 128; // rollout block size

__host__ __device__ __forceinline__ size_t ga16(size_t x)
{
    return (x + 15) & ~(size_t)15;
}

__device__ __forceinline__ int gPackInfo(int pt, int bt)
{
    return (pt << 16) | (bt & 0xffff);
}

__device__ __forceinline__ void copyGate(GateParams* dst, const GateParams* src)
{
    for (int i = threadIdx.x; i < GATE_HOST_WORDS; i += blockDim.x)
        ((float*)dst)[i] = ((const float*)src)[i];
    gateDeviceTerms(*dst, *src, threadIdx.x, blockDim.x);
}

struct GateSmem
{
    size_t gp, track, knots, B, vbuf, red, total;
};

__host__ __device__ inline GateSmem gateRolloutLayout(int nbp, int T, int M, bool spl)
{
    GateSmem L;
    size_t off = 16; // mbarrier
    L.gp = off;
    off = ga16(off + sizeof(GateParams));
    L.track = off;
    off = ga16(off + GATE_TRACK_FLOATS * 4);
    L.knots = off;
    off = ga16(off + (size_t)nbp * M * 2 * 4);
    L.B = off;
    if (spl)
        off = ga16(off + (size_t)T * M * 4);
    L.vbuf = off;
    if (spl)
        off = ga16(off + (size_t)M * 2 * GRB * 4);
    L.red = off;
    off = ga16(off + GRB * 4);
    L.total = off;
    return L;
}

} // namespace

// fullRolloutKernel (kernels.cu:34-171) + aggregateBranchCostsKernel (175-217) on the
// gate race: environmentStep<true, true, false> (kernels.cu:141-143).
template <int NTH, bool SPL, int ME>
__global__ void __launch_bounds__(GRB) gate_rollout(const MppiDev* __restrict__ insts, const MppiIn* __restrict__ in, const Tile* __restrict__ tiles)
{
    constexpr int NBP = NTH + 1;
    extern __shared__ __align__(128) unsigned char smraw[];
    const Tile tile = tiles[blockIdx.x];
    const MppiDev& D = insts[tile.inst];
    const MppiIn& I = in[tile.inst];
    const int K = D.cfg.K, T = D.cfg.T, M = D.cfg.M;
    const GateSmem L = gateRolloutLayout(NBP, T, M, SPL);
    uint64_t* bar = (uint64_t*)smraw;
    GateParams* sG = (GateParams*)(smraw + L.gp);
    float* sTrack = (float*)(smraw + L.track);
    float* sKn = (float*)(smraw + L.knots);
    float* sB = (float*)(smraw + L.B);
    float* vbuf = (float*)(smraw + L.vbuf);
    float* red = (float*)(smraw + L.red);
    const uint32_t knBytes = (uint32_t)ga16((size_t)NBP * M * 2 * 4);
    const uint32_t bBytes = SPL ? (uint32_t)ga16((size_t)T * M * 4) : 0u;
    if (threadIdx.x == 0)
    {
        mbar_init(bar, 1);
        mbar_expect_tx(bar, GATE_TRACK_FLOATS * 4 + knBytes + bBytes);
        if (!D.cfg.dbgNoStage)
        {
            bulk_g2s(sTrack, D.gtrack, GATE_TRACK_FLOATS * 4, bar);
            bulk_g2s(sKn, D.knots, knBytes, bar);
            if (SPL)
                bulk_g2s(sB, D.B, bBytes, bar);
        }
    }
    copyGate(sG, D.gate);
    __syncthreads();
    if (!__syncthreads_and(mbar_wait(bar, 0, D.cfg.waitPolls)))
    {
        rolloutTileTimedOut<NTH>(D, I, tile, K);
        if (threadIdx.x == 0)
            atomicAdd(&D.stats[1], 1);
        return;
    }
    const GateParams& G = *sG;
    const int th = threadIdx.x % NTH;
    const int sl = threadIdx.x / NTH;
    const int s = tile.s0 + sl;
    const bool valid = sl < tile.count;
    const float minConf = D.cfg.minConf;
    const uint32_t k0 = D.cfg.k0, k1 = D.cfg.k1, step = I.step;
    const float sig0 = D.cfg.sigma0, sig1 = D.cfg.sigma1;
    const float gateMargin = D.cfg.gateMargin;

    float belief0[NTH];
#pragma unroll
    for (int i = 0; i < NTH; i++)
        belief0[i] = I.belief[i];
    const int pt0 = findConfident<NTH>(belief0, minConf);
    const int bt0 = pt0 == 0 ? -1 : 0;
    const bool compatible = (pt0 == 0 || pt0 == th + 1);

    float cost = INFINITY;
    int pt = pt0, bt = bt0;
    if (valid && compatible)
    {
        GState st;
        loadGState(st, I.gstate);
        BState<NTH> bs;
#pragma unroll
        for (int i = 0; i < NTH; i++)
            bs.belief[i] = belief0[i];
        bs.predTheta = pt0;
        bs.branchingTime = bt0;
        cost = 0.0f;
        bool stop = false;
        float decay = 1.0f;
        int tOrigin = 0;
        EnvNoise rng(k0, k1, (uint32_t)s, (uint32_t)th << 16, step, S_MPPI_ROLL_ENV);
        int curB = -1;
        for (int t = 0; t < T && !stop; t++)
        {
            rng.begin_step((uint32_t)t);
            const int local = t - tOrigin;
            const int b = bs.predTheta;
            float ego0, ego1;
            if constexpr (SPL)
            {
                if (b != curB)
                {
                    for (int m = 0; m < M; m++)
                    {
                        U4 r = draw(k0, k1, (uint32_t)s, (uint32_t)(b * M + m), step, S_MPPI_EPS, 0);
                        float e0 = scaled_normal(sig0, r.x);
                        float e1 = scaled_normal(sig1, r.y);
                        vbuf[(m * 2 + 0) * GRB + threadIdx.x] = sKn[(b * M + m) * 2 + 0] + e0;
                        vbuf[(m * 2 + 1) * GRB + threadIdx.x] = sKn[(b * M + m) * 2 + 1] + e1;
                    }
                    curB = b;
                }
                const float* Brow = sB + local * M;
                float sum = 0.0f;
                for (int m = 0; m < M; m++)
                    sum += Brow[m] * vbuf[(m * 2 + 0) * GRB + threadIdx.x];
                ego0 = sum;
                sum = 0.0f;
                for (int m = 0; m < M; m++)
                    sum += Brow[m] * vbuf[(m * 2 + 1) * GRB + threadIdx.x];
                ego1 = sum;
            }
            else
            {
                U4 r = draw(k0, k1, (uint32_t)s, (uint32_t)(b * T + local), step, S_MPPI_EPS, 0);
                float e0 = scaled_normal(sig0, r.x);
                float e1 = scaled_normal(sig1, r.y);
                ego0 = sKn[(b * T + local) * 2 + 0] + e0;
                ego1 = sKn[(b * T + local) * 2 + 1] + e1;
            }
            bool branched = false;
            StepOut o = gateStep<NTH, true, true, false, true, ME>(t, th, sTrack, G, ego0, ego1, st, bs, branched, minConf, rng, gateMargin);
            if (branched)
                tOrigin = t + 1;
            stop = (o.term != TERM_NONE);
            cost += gateStateCost(o, G, D.cfg.w) * decay;
            decay *= DECAY;
        }
        cost += gateFinalCost<ME>(st, G, D.cfg.w.finalAdvWeight, D.cfg.w.finalOppAdvWeight);
        pt = bs.predTheta;
        bt = bs.branchingTime;
    }
    if (valid)
    {
        D.costsTrue[th * K + s] = cost;
        D.binfo[th * K + s] = gPackInfo(pt, bt);
        if (compatible && !isfinite(cost))
            atomicAdd(&D.stats[0], 1);
    }
    red[threadIdx.x] = cost;
    __syncthreads();
    // aggregateBranchCostsKernel (kernels.cu:175-217): costs[b][s] = E_belief[cost | b]
    if (valid)
    {
        const float* c = red + sl * NTH;
        if (th == 0)
        {
            float num = 0.0f, den = 0.0f;
#pragma unroll
            for (int m = 0; m < NTH; m++)
            {
                float cv = c[m];
                if (!isfinite(cv))
                    continue;
                float w = belief0[m];
                num += w * cv;
                den += w;
            }
            D.costs[s] = (den > 1e-30f) ? (num / den) : INFINITY;
        }
        {
            float num = 0.0f, den = 0.0f;
            float cv = c[th];
            if (isfinite(cv))
            {
                float w = belief0[th];
                num += w * cv;
                den += w;
            }
            D.costs[(size_t)(th + 1) * K + s] = (den > 1e-30f) ? (num / den) : INFINITY;
        }
    }
}

// verifyNominalFailureKernel (kernels.cu:488-551) on the gate race:
// environmentStep<true, true, false, false>; one thread per sample, both plans in one
// grid, the CTA's warps in step (a barrier per step) as in mppi_verify.
// Two 512-thread CTAs per SM (64 registers a thread, ~20 bytes spilled) for up to four
// hypotheses: measured on the 4 x 2 x 2^17 x 40 gate verification (B200, 1965 MHz)
// 2.66 ms against 3.42 ms with one CTA per SM (128 registers, no spills).
#ifndef GATE_VERIFY_MIN_BLOCKS
#define GATE_VERIFY_MIN_BLOCKS 2
#endif
template <int NTH> constexpr int gateVerifyMinBlocks()
{
    return NTH <= 4 ? GATE_VERIFY_MIN_BLOCKS : 1;
}
// FAST: the verification's fast arithmetic flavour and noise source (the default; the
// exact flavour reproduces the oracle's per-sample results and serves parity tests), as
// in the strategic race's mppi_verify; its warps step without a CTA barrier.
template <int NTH, int ME, bool FAST>
__global__ void __launch_bounds__(VERIFY_TILE, (gateVerifyMinBlocks<NTH>())) gate_verify(const MppiDev* __restrict__ insts, const MppiIn* __restrict__ in, const Tile* __restrict__ tiles,
                                                             int* __restrict__ dbgFailTime, int* __restrict__ dbgTheta)
{
    constexpr int NBP = NTH + 1;
    extern __shared__ __align__(128) unsigned char smraw[];
    const Tile tile = tiles[blockIdx.x];
    const MppiDev& D = insts[tile.inst];
    const MppiIn& I = in[tile.inst];
    const int T = D.cfg.T, H = D.cfg.H;
    const int plan = tile.aux;
    uint64_t* bar = (uint64_t*)smraw;
    GateParams* sG = (GateParams*)(smraw + 16);
    const size_t offT = ga16(16 + sizeof(GateParams));
    float* sTrack = (float*)(smraw + offT);
    float* sPlan = (float*)(smraw + offT + GATE_TRACK_FLOATS * 4);
    const uint32_t planBytes = (uint32_t)ga16((size_t)NBP * T * 2 * 4);
    unsigned* hist = (unsigned*)(smraw + offT + GATE_TRACK_FLOATS * 4 + planBytes);
    if (threadIdx.x == 0)
    {
        mbar_init(bar, 1);
        mbar_expect_tx(bar, GATE_TRACK_FLOATS * 4 + planBytes);
        if (!D.cfg.dbgNoStage)
        {
            bulk_g2s(sTrack, D.gtrack, GATE_TRACK_FLOATS * 4, bar);
            bulk_g2s(sPlan, plan == 0 ? D.dense : D.prevDense, planBytes, bar);
        }
    }
    copyGate(sG, D.gate);
    for (int i = threadIdx.x; i < T; i += blockDim.x)
        hist[i] = 0u;
    __syncthreads();
    if (!__syncthreads_and(mbar_wait(bar, 0, D.cfg.waitPolls)))
    {
        if (threadIdx.x == 0)
            atomicAdd(&D.stats[1], 1);
        return;
    }
    const GateParams& G = *sG;
    const int v = tile.s0 + threadIdx.x;
    bool active = threadIdx.x < tile.count; // idle lanes of a partial tile still take the barriers
    {
        const float minConf = D.cfg.minConf;
        const float gateMargin = D.cfg.gateMargin;
        GState st;
        loadGState(st, I.gstate);
        BState<NTH> bs;
#pragma unroll
        for (int i = 0; i < NTH; i++)
            bs.belief[i] = I.belief[i];
        bs.predTheta = findConfident<NTH>(bs.belief, minConf);
        bs.branchingTime = bs.predTheta == 0 ? -1 : 0;
        // sampleModelFromBelief (state.h:118-131) on a Philox uniform
        const uint32_t k0 = D.cfg.k0, k1 = D.cfg.k1, step = I.step;
        float u = uniform_from_word(draw(k0, k1, (uint32_t)v, (uint32_t)plan, step, S_VERIF_THETA, 0).x);
        int theta = NTH - 1;
        {
            float cdf = 0.0f;
            bool found = false;
#pragma unroll
            for (int kk = 0; kk < NTH; kk++)
            {
                cdf += bs.belief[kk];
                if (!found && u <= cdf)
                {
                    theta = kk;
                    found = true;
                }
            }
        }
        using Noise = typename std::conditional<FAST, FastNoise, EnvNoise>::type;
        Noise rng(k0, k1, (uint32_t)v, (uint32_t)plan << 16, step, S_VERIF_ENV);
        int tOrigin = 0, tEnd = H;
        bool failed = false;
        for (int t = 0; t < H; t++)
        {
            // exact flavour: every thread takes this barrier once per step (H is uniform),
            // which keeps the warps on the same step, where they fetch the same
            // instructions, and ends the loop once all samples of the CTA are done; fast
            // flavour: a warp leaves once its samples are done
            if constexpr (FAST)
            {
                if (!__any_sync(0xffffffffu, active))
                    break;
            }
            else if (!__syncthreads_or(active))
                break;
            if (!active)
                continue;
            rng.begin_step((uint32_t)t);
            int local = t - tOrigin;
            int b = bs.predTheta;
            float e0 = sPlan[(b * T + local) * 2], e1 = sPlan[(b * T + local) * 2 + 1];
            bool branched = false;
            StepOut o = gateStep<NTH, true, true, false, false, ME, false, FAST, Noise>(t, theta, sTrack, G, e0, e1, st, bs, branched, minConf, rng, gateMargin);
            if (branched)
                tOrigin = t + 1;
            if (o.term == TERM_LOSE)
            {
                failed = true;
                active = false;
                tEnd = t;
            }
            else if (o.term == TERM_WIN || o.term == TERM_OPP_WIN)
            {
                active = false;
                tEnd = t;
            }
        }
        if (failed)
            atomicAdd(&hist[tEnd], 1u);
        if (threadIdx.x < tile.count)
        {
            if (dbgFailTime)
                dbgFailTime[v] = failed ? tEnd : -1;
            if (dbgTheta)
                dbgTheta[v] = theta;
        }
    }
    __syncthreads();
    for (int i = threadIdx.x; i < T; i += blockDim.x)
        if (hist[i])
            atomicAdd(&D.fail[plan * T + i], hist[i]);
}

// One true-dynamics step (environmentStep with noise, as the engine's dynStep).
template <int NTH, int ME>
__global__ void gate_env_step_kernel(const GateParams* __restrict__ gp, const float* __restrict__ track, int trueTheta, float a0, float a1,
                                     dr_gate_state* st, float* belief, int updateBelief, uint32_t k0, uint32_t k1, uint32_t step, int* term)
{
    __shared__ GateParams sG;
    if (threadIdx.x == 0)
    {
        sG = *gp;
        gateDeviceTerms(sG, *gp, 0, 1);
    }
    __syncthreads();
    if (threadIdx.x != 0)
        return;
    GState s;
    loadGState(s, *st);
    BState<NTH> bs;
    for (int i = 0; i < NTH; i++)
        bs.belief[i] = belief[i];
    bs.predTheta = 0;
    bs.branchingTime = -1;
    EnvNoise rng(k0, k1, 0u, 0u, step, S_ENV_STEP);
    rng.begin_step(0);
    bool branched = false;
    StepOut o;
    if (updateBelief)
        o = gateStep<NTH, true, false, false, true, ME>(0, trueTheta, track, sG, a0, a1, s, bs, branched, 2.0f, rng, 0.0f);
    else
        o = gateStep<NTH, false, false, false, true, ME>(0, trueTheta, track, sG, a0, a1, s, bs, branched, 2.0f, rng, 0.0f);
    storeGState(*st, s);
    for (int i = 0; i < NTH; i++)
        belief[i] = bs.belief[i];
    *term = o.term;
}

// The same for every controller of a batch (dr_mppi_batch_env_step_device): one CTA per
// controller, its gate parameters and racelines, the action it sent, the noise stream of
// its step counter.
template <int NTH, int ME>
__global__ void gate_batch_env_step(const MppiDev* __restrict__ insts, const MppiIn* __restrict__ in, const int* __restrict__ trueTheta,
                                    const float* __restrict__ actions, dr_gate_state* __restrict__ states, float* __restrict__ beliefs, int updateBelief,
                                    uint32_t k0, uint32_t k1, int* __restrict__ terms)
{
    __shared__ GateParams sG;
    const int inst = blockIdx.x;
    const MppiDev& D = insts[inst];
    if (threadIdx.x == 0)
    {
        sG = *D.gate;
        gateDeviceTerms(sG, *D.gate, 0, 1);
    }
    __syncthreads();
    if (threadIdx.x != 0)
        return;
    GState s;
    loadGState(s, states[inst]);
    float* belief = beliefs + (size_t)inst * DR_MAX_THETA;
    BState<NTH> bs;
    for (int i = 0; i < NTH; i++)
        bs.belief[i] = belief[i];
    bs.predTheta = 0;
    bs.branchingTime = -1;
    EnvNoise rng(k0, k1, 0u, 0u, in[inst].step, S_ENV_STEP);
    rng.begin_step(0);
    bool branched = false;
    const float a0 = actions[inst * 2], a1 = actions[inst * 2 + 1];
    StepOut o;
    if (updateBelief)
        o = gateStep<NTH, true, false, false, true, ME>(0, trueTheta[inst], D.gtrack, sG, a0, a1, s, bs, branched, 2.0f, rng, 0.0f);
    else
        o = gateStep<NTH, false, false, false, true, ME>(0, trueTheta[inst], D.gtrack, sG, a0, a1, s, bs, branched, 2.0f, rng, 0.0f);
    storeGState(states[inst], s);
    for (int i = 0; i < NTH; i++)
        belief[i] = bs.belief[i];
    terms[inst] = o.term;
}

// ---------------------------------------------------------------------------------------
// launchers
// ---------------------------------------------------------------------------------------
bool gateSupported(int nth)
{
    return nth == 1 || nth == 2 || nth == 4 || nth == 8;
}

size_t gateRolloutSmem(int nth, int T, int M, bool spl)
{
    return gateRolloutLayout(nth + 1, T, M, spl).total;
}

size_t gateVerifySmem(int nth, int T)
{
    return ga16(16 + sizeof(GateParams)) + GATE_TRACK_FLOATS * 4 + ga16((size_t)(nth + 1) * T * 2 * 4) + (size_t)T * 4;
}

int gateRolloutSamplesPerBlock(int nth)
{
    return GRB / nth;
}

template <int NTH, int ME> static cudaError_t launchGateRolloutT(const LaunchArgs& a, bool spl, size_t smem)
{
    if (spl)
    {
        auto k = gate_rollout<NTH, true, ME>;
        ensureSmem(k, smem);
        k<<<a.nTiles, GRB, smem, a.stream>>>(a.mppi, a.mppiIn, a.tiles);
    }
    else
    {
        auto k = gate_rollout<NTH, false, ME>;
        ensureSmem(k, smem);
        k<<<a.nTiles, GRB, smem, a.stream>>>(a.mppi, a.mppiIn, a.tiles);
    }
    return cudaGetLastError();
}

template <int NTH, int ME> static cudaError_t launchGateVerifyT(const LaunchArgs& a, size_t smem, int* ft, int* th)
{
    auto k = a.exactVerify ? gate_verify<NTH, ME, false> : gate_verify<NTH, ME, true>;
    ensureSmem(k, smem);
    k<<<a.nTiles, VERIFY_TILE, smem, a.stream>>>(a.mppi, a.mppiIn, a.tiles, ft, th);
    return cudaGetLastError();
}

// (n_theta, ego index) -> instantiation
#define GATE_DISPATCH(NTH_, ME_, CALL)                                                                                                                \
    switch ((NTH_) * 2 + (ME_))                                                                                                                      \
    {                                                                                                                                                \
    case 1 * 2 + 0: return CALL(1, 0);                                                                                                              \
    case 1 * 2 + 1: return CALL(1, 1);                                                                                                              \
    case 2 * 2 + 0: return CALL(2, 0);                                                                                                              \
    case 2 * 2 + 1: return CALL(2, 1);                                                                                                              \
    case 4 * 2 + 0: return CALL(4, 0);                                                                                                              \
    case 4 * 2 + 1: return CALL(4, 1);                                                                                                              \
    case 8 * 2 + 0: return CALL(8, 0);                                                                                                              \
    case 8 * 2 + 1: return CALL(8, 1);                                                                                                              \
    default: return cudaErrorInvalidValue;                                                                                                           \
    }

cudaError_t launchGateRollout(const LaunchArgs& a, int nth, int me, bool spl, size_t smem)
{
#define CALL(P, Q) launchGateRolloutT<P, Q>(a, spl, smem)
    GATE_DISPATCH(nth, me, CALL)
#undef CALL
}

cudaError_t launchGateVerify(const LaunchArgs& a, int nth, int me, size_t smem, int* dbgFailTime, int* dbgTheta)
{
#define CALL(P, Q) launchGateVerifyT<P, Q>(a, smem, dbgFailTime, dbgTheta)
    GATE_DISPATCH(nth, me, CALL)
#undef CALL
}

template <int NTH, int ME>
static cudaError_t launchGateEnvStepT(cudaStream_t stream, const GateParams* gp, const float* track, int trueTheta, float a0, float a1, dr_gate_state* st,
                                      float* belief, int updateBelief, uint32_t k0, uint32_t k1, uint32_t step, int* term)
{
    gate_env_step_kernel<NTH, ME><<<1, 32, 0, stream>>>(gp, track, trueTheta, a0, a1, st, belief, updateBelief, k0, k1, step, term);
    return cudaGetLastError();
}

template <int NTH, int ME>
static cudaError_t launchGateBatchEnvStepT(cudaStream_t stream, const MppiDev* insts, const MppiIn* in, int nInst, const int* trueTheta, const float* actions,
                                           dr_gate_state* states, float* beliefs, int updateBelief, uint32_t k0, uint32_t k1, int* terms)
{
    gate_batch_env_step<NTH, ME><<<nInst, 32, 0, stream>>>(insts, in, trueTheta, actions, states, beliefs, updateBelief, k0, k1, terms);
    return cudaGetLastError();
}

cudaError_t launchGateBatchEnvStep(cudaStream_t stream, int nth, int me, const MppiDev* insts, const MppiIn* in, int nInst, const int* trueTheta,
                                   const float* actions, dr_gate_state* states, float* beliefs, int updateBelief, uint32_t k0, uint32_t k1, int* terms)
{
#define CALL(P, Q) launchGateBatchEnvStepT<P, Q>(stream, insts, in, nInst, trueTheta, actions, states, beliefs, updateBelief, k0, k1, terms)
    GATE_DISPATCH(nth, me, CALL)
#undef CALL
}

cudaError_t launchGateEnvStep(cudaStream_t stream, int nth, int me, const GateParams* gp, const float* track, int trueTheta, float a0, float a1,
                              dr_gate_state* st, float* belief, int updateBelief, uint32_t k0, uint32_t k1, uint32_t step, int* term)
{
#define CALL(P, Q) launchGateEnvStepT<P, Q>(stream, gp, track, trueTheta, a0, a1, st, belief, updateBelief, k0, k1, step, term)
    GATE_DISPATCH(nth, me, CALL)
#undef CALL
}

} // namespace dr
