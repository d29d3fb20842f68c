// PR-MPPI on the gate race: the reference's PR-MPPI kernels (src/prmppi_kernels.cu)
// compiled with USE_ENV_DRONERACE, whose cost functions (include/costs.cuh:44-86) call the
// gate race's trackBoundaryDist / isWinner / isOppWinner / getAdvance
// (include/environments/env_dronerace.h:262-401). The step is the gate model's
// environment step (gate_model.cuh, gateStep<UPD = false, BR = false, ADDMARGIN = true,
// LOSE = true>), as PRMPPIfullRolloutKernel calls environmentStep<false, false, true>.
//
//   gate_pr_rollout      PRMPPIfullRolloutKernel (:55-130) with the per-sample average
//                        over hypotheses (PRMPPIcostAvgKernel, :134-166) in its epilogue;
//                        512-thread CTAs whose warps take a barrier every step
//   gate_pr_candidates   PRMPPIcomputeCandidateCostKernel (:285-347), the safety re-check
//                        (PRMPPIcomputeSafeCostKernel, :350-393) for both candidates, and
//                        the choice (prmppi_controller.cu:232-304)
// The prologue (shift, hypothesis draw) and the weighted averages do not depend on the
// environment and are the strategic race's kernels.
#include "common.cuh"
#include "gate_model.cuh"
#include "instance.cuh"
#include "launch.h"

namespace dr
{

namespace
{
constexpr int GPR_TILE = 512;
constexpr int GPR_CAND = 128;

template <int NTH> constexpr int gatePrMinBlocks()
{
    return NTH <= 4 ? 2 : 1;
}

__host__ __device__ __forceinline__ size_t gp16(size_t x)
{
    return (x + 15) & ~(size_t)15;
}

__device__ __forceinline__ void copyGateP(GateParams* dst, const GateParams* src)
{
    for (int i = threadIdx.x; i < GATE_HOST_WORDS; i += blockDim.x)
        ((float*)dst)[i] = ((const float*)src)[i];
    gateDeviceTerms(*dst, *src, threadIdx.x, blockDim.x);
}

// PRMPPIstateCost (costs.cuh:44-63) on the gate race: trackBoundaryDist<true> is -1 once
// the opponent has won.
__device__ __forceinline__ float gatePrStateCost(const StepOut& o, const GateParams& G, const PrCfgDev& c)
{
    float cost = 0.0f;
    float bd = o.oppWon ? -1.0f : o.bdRaw;
    float danger = c.boundaryThresholdFactor * G.droneRadius;
    if (bd < danger)
        cost += c.boundaryCost * powf(bd / G.droneRadius, 2.0f);
    if (o.winner)
        cost -= c.winCost;
    if (o.oppWon)
        cost += c.oppWinCost;
    return cost;
}

// PRMPPIsafetyCost (costs.cuh:78-86): droneRadius * collDistFactor - trackBoundaryDist<false>,
// the product fused into the subtraction as in the strategic race's kernel
__device__ __forceinline__ float gatePrSafetyCost(const StepOut& o, const GateParams& G, float collDistFactor)
{
    return __fmaf_rn(G.droneRadius, collDistFactor, -o.bdRaw);
}

struct GatePrSmem
{
    size_t gp, track, nom, red, total;
};

__host__ __device__ inline GatePrSmem gatePrLayout(int T)
{
    GatePrSmem L;
    size_t off = 16; // mbarrier
    L.gp = off;
    off = gp16(off + sizeof(GateParams));
    L.track = off;
    off = gp16(off + GATE_TRACK_FLOATS * 4);
    L.nom = off;
    off = gp16(off + (size_t)T * 2 * 4);
    L.red = off;
    off = gp16(off + (size_t)GPR_TILE * 2 * 4);
    L.total = off;
    return L;
}
} // namespace

// tile: inst, s0 (first sample), count (samples), aux (0 nominal / 1 robust)
template <int NTH, int ME>
__global__ void __launch_bounds__(GPR_TILE, gatePrMinBlocks<NTH>()) gate_pr_rollout(const PrDev* __restrict__ insts, const PrIn* __restrict__ in,
                                                                                const Tile* __restrict__ tiles)
{
    extern __shared__ __align__(128) unsigned char smraw[];
    const Tile tile = tiles[blockIdx.x];
    const PrDev& D = insts[tile.inst];
    const PrIn& I = in[tile.inst];
    const int K = D.cfg.K, T = D.cfg.T, P = D.cfg.P;
    const int robust = tile.aux;
    const GatePrSmem L = gatePrLayout(T);
    uint64_t* bar = (uint64_t*)smraw;
    GateParams* sG = (GateParams*)(smraw + L.gp);
    float* sTrack = (float*)(smraw + L.track);
    float* sNom = (float*)(smraw + L.nom);
    float* red = (float*)(smraw + L.red);
    const uint32_t nomBytes = (uint32_t)gp16((size_t)T * 2 * 4);
    if (threadIdx.x == 0)
    {
        mbar_init(bar, 1);
        mbar_expect_tx(bar, GATE_TRACK_FLOATS * 4 + nomBytes);
        bulk_g2s(sTrack, D.gtrack, GATE_TRACK_FLOATS * 4, bar);
        bulk_g2s(sNom, robust ? D.rob : D.nom, nomBytes, bar);
    }
    copyGateP(sG, D.gate);
    __syncthreads();
    if (!__syncthreads_and(mbar_wait(bar, 0)))
    {
        if (threadIdx.x == 0)
            atomicAdd(&D.stats[1], 1);
        return;
    }
    const GateParams& G = *sG;
    const int spb = GPR_TILE / P;
    const int sl = threadIdx.x / P, p = threadIdx.x % P;
    const int s = tile.s0 + sl;
    const bool valid = sl < spb && sl < tile.count;
    float running = 0.0f, safe = -INFINITY;
    {
        const int theta = D.thetas[p];
        GState st;
        loadGState(st, I.gstate);
        BState<NTH> bs{};
        const uint32_t k0 = D.cfg.k0, k1 = D.cfg.k1, step = I.step;
        EnvNoise rng(k0, k1, (uint32_t)s, ((((uint32_t)robust << 8) | (uint32_t)p) << 16), step, S_PR_ROLL_ENV);
        float decay = 1.0f;
        bool active = valid;
        for (int t = 0; t < T; t++)
        {
            // every thread of the CTA takes this barrier once per step (T is uniform)
            if (!__syncthreads_or(active))
                break;
            if (!active)
                continue;
            rng.begin_step((uint32_t)t);
            U4 r = draw(k0, k1, (uint32_t)s, (uint32_t)t, step, S_PR_EPS, 0);
            float ego0 = sNom[t * 2] + scaled_normal(D.cfg.sigma0, r.x);
            float ego1 = sNom[t * 2 + 1] + scaled_normal(D.cfg.sigma1, r.y);
            bool branched = false;
            StepOut o = gateStep<NTH, false, false, true, true, ME, true>(t, theta, sTrack, G, ego0, ego1, st, bs, branched, 0.0f, rng, D.cfg.gateMargin);
            if (o.term != TERM_NONE)
                active = false;
            running += decay * gatePrStateCost(o, G, D.cfg);
            safe = fmaxf(safe, gatePrSafetyCost(o, G, D.cfg.collDistFactor));
            decay *= DECAY;
        }
        if (valid)
        {
            running += gateFinalCost<ME>(st, G, D.cfg.finalAdvWeight, D.cfg.finalOppAdvWeight);
            float* out = robust ? D.costRob : D.costNom;
            out[((size_t)p * K + s) * 2 + 0] = running;
            out[((size_t)p * K + s) * 2 + 1] = safe;
        }
    }
    red[threadIdx.x * 2] = running;
    red[threadIdx.x * 2 + 1] = safe;
    __syncthreads();
    // PRMPPIcostAvgKernel (prmppi_kernels.cu:134-166)
    if (valid && p == 0)
    {
        float avg = 0.0f, maxSafe = -INFINITY;
        for (int q = 0; q < P; q++)
        {
            avg += red[(sl * P + q) * 2];
            maxSafe = fmaxf(maxSafe, red[(sl * P + q) * 2 + 1]);
        }
        avg /= (float)P;
        float full = avg + ((maxSafe > 0.0f) ? D.cfg.safetyWeight : 0.0f);
        D.avg[((size_t)robust * K + s) * 2 + 0] = full;
        D.avg[((size_t)robust * K + s) * 2 + 1] = maxSafe;
        if (!isfinite(full))
            atomicAdd(&D.stats[0], 1);
    }
}

// one block per instance: threads (kind, cand, p), kind 0 = full cost, 1 = safety re-check
template <int NTH, int ME>
__global__ void __launch_bounds__(GPR_CAND) gate_pr_candidates(const PrDev* __restrict__ insts, const PrIn* __restrict__ in, int nInst)
{
    extern __shared__ __align__(128) unsigned char smraw[];
    __shared__ int sChosen;
    const int inst = blockIdx.x;
    if (inst >= nInst)
        return;
    const PrDev& D = insts[inst];
    const PrIn& I = in[inst];
    const int T = D.cfg.T, P = D.cfg.P;
    uint64_t* bar = (uint64_t*)smraw;
    GateParams* sG = (GateParams*)(smraw + 16);
    const size_t offT = gp16(16 + sizeof(GateParams));
    float* sTrack = (float*)(smraw + offT);
    float* sC1 = (float*)(smraw + offT + GATE_TRACK_FLOATS * 4);
    const uint32_t cb = (uint32_t)gp16((size_t)T * 2 * 4);
    float* sC2 = (float*)((unsigned char*)sC1 + cb);
    if (threadIdx.x == 0)
    {
        mbar_init(bar, 1);
        mbar_expect_tx(bar, GATE_TRACK_FLOATS * 4 + 2 * cb);
        bulk_g2s(sTrack, D.gtrack, GATE_TRACK_FLOATS * 4, bar);
        bulk_g2s(sC1, D.cand1, cb, bar);
        bulk_g2s(sC2, D.cand2, cb, bar);
    }
    copyGateP(sG, D.gate);
    __syncthreads();
    if (!__syncthreads_and(mbar_wait(bar, 0)))
    {
        if (threadIdx.x == 0)
            atomicAdd(&D.stats[1], 1);
        return;
    }
    const GateParams& G = *sG;
    const uint32_t k0 = D.cfg.k0, k1 = D.cfg.k1, step = I.step;
    for (int task = threadIdx.x; task < 4 * P; task += blockDim.x)
    {
        const int kind = task / (2 * P);
        const int tid = task % (2 * P);
        const int second = tid >= P;
        const int p = second ? tid - P : tid;
        const float* nominal = second ? sC2 : sC1;
        const int theta = D.thetas[p];
        GState st;
        loadGState(st, I.gstate);
        BState<NTH> bs{};
        EnvNoise rng(k0, k1, (uint32_t)p, (uint32_t)second << 16, step, kind ? S_PR_SAFE_ENV : S_PR_CAND_ENV);
        float cost = 0.0f, safeCost = -INFINITY, decay = 1.0f;
        bool stop = false;
        for (int t = 0; t < T && !stop; ++t)
        {
            rng.begin_step((uint32_t)t);
            bool branched = false;
            StepOut o = gateStep<NTH, false, false, true, true, ME, true>(t, theta, sTrack, G, nominal[t * 2], nominal[t * 2 + 1], st, bs, branched, 0.0f,
                                                                          rng, D.cfg.gateMargin);
            stop = (o.term != TERM_NONE);
            cost += decay * gatePrStateCost(o, G, D.cfg);
            decay *= DECAY;
            safeCost = fmaxf(safeCost, gatePrSafetyCost(o, G, D.cfg.collDistFactor));
        }
        cost += gateFinalCost<ME>(st, G, D.cfg.finalAdvWeight, D.cfg.finalOppAdvWeight);
        if (safeCost > 0.0f)
            cost += D.cfg.safetyWeight;
        if (kind == 0)
            D.candFull[tid] = cost;
        else
            D.candSafe[tid] = safeCost;
    }
    __syncthreads();
    // candidate choice (prmppi_controller.cu:236-256) and safety decision (:264-275)
    if (threadIdx.x == 0)
    {
        float c1 = 0.0f, c2 = 0.0f;
        for (int p = 0; p < P; ++p)
        {
            c1 += D.candFull[p];
            c2 += D.candFull[P + p];
        }
        c1 /= (float)P;
        c2 /= (float)P;
        D.decision[0] = c2 < c1; // resetNom
        int chosen = (c1 <= c2) ? 0 : 1;
        int useNom = 1;
        for (int p = 0; p < P; p++)
            if (D.candSafe[chosen * P + p] > 0.0f)
            {
                useNom = 0;
                break;
            }
        D.decision[1] = useNom;
        D.decision[2] = chosen;
        sChosen = chosen;
    }
    __syncthreads();
    const float* ch = sChosen ? sC2 : sC1;
    for (int i = threadIdx.x; i < T * 2; i += blockDim.x)
    {
        D.nom[i] = ch[i];
        D.rob[i] = D.robWork[i];
    }
}

size_t gatePrRolloutSmem(int T)
{
    return gatePrLayout(T).total;
}

int gatePrRolloutSamplesPerBlock()
{
    return GPR_TILE;
}

template <int NTH, int ME> static cudaError_t gatePrRollT(const LaunchArgs& a, size_t smem)
{
    auto k = gate_pr_rollout<NTH, ME>;
    ensureSmem(k, smem);
    k<<<a.nTiles, GPR_TILE, smem, a.stream>>>(a.pr, a.prIn, a.tiles);
    return cudaGetLastError();
}

template <int NTH, int ME> static cudaError_t gatePrCandT(const LaunchArgs& a, int nInst, int maxT)
{
    const size_t smem = gp16(16 + sizeof(GateParams)) + GATE_TRACK_FLOATS * 4 + 2 * gp16((size_t)maxT * 2 * 4);
    auto k = gate_pr_candidates<NTH, ME>;
    ensureSmem(k, smem);
    k<<<nInst, GPR_CAND, smem, a.stream>>>(a.pr, a.prIn, nInst);
    return cudaGetLastError();
}

#define GPR_DISPATCH(NTH_, ME_, CALL)                                                                                                                 \
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

cudaError_t launchGatePrRollout(const LaunchArgs& a, int nth, int me, size_t smem)
{
#define CALL(P_, Q_) gatePrRollT<P_, Q_>(a, smem)
    GPR_DISPATCH(nth, me, CALL)
#undef CALL
}

cudaError_t launchGatePrCandidates(const LaunchArgs& a, int nth, int me, int nInst, int maxT)
{
#define CALL(P_, Q_) gatePrCandT<P_, Q_>(a, nInst, maxT)
    GPR_DISPATCH(nth, me, CALL)
#undef CALL
}

} // namespace dr
