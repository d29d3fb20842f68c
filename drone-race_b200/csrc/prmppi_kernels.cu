// PR-MPPI control-step kernels (reference: src/prmppi_kernels.cu; host sequence
// src/prmppi_controller.cu:142-349).
//
//   pr_prologue    shifts both nominals by one step (prmppi_controller.cu:163-175) and
//                  draws the P hypotheses from the belief (PRMPPIsampleThetaValues,
//                  prmppi_kernels.cu:23-51).
//   pr_rollout     one thread per (nominal/robust, sample, hypothesis): rollout of
//                  nominal + Philox perturbation under theta_p with running and safety cost
//                  (PRMPPIfullRolloutKernel, :55-130); the hypotheses of a sample sit in
//                  neighbouring threads, so the per-sample average over p and the safety
//                  indicator (PRMPPIcostAvgKernel, :134-166) are done in the epilogue.
//   pr_weighted    per (which, t): minimum of the averaged cost (PRMPPIcomputeMinCosts-
//                  Kernel, :169-199), exponential weights and the weighted average of the
//                  absolute perturbed controls (PRMPPIWeightedAverageKernel, :204-282),
//                  with the perturbation regenerated and the sums in the reference's order.
//   pr_candidates  full cost of both candidates under every theta_p (PRMPPIcompute-
//                  CandidateCostKernel, :285-347) and, speculatively for both, the safety
//                  re-check of the one that will be chosen (PRMPPIcomputeSafeCostKernel,
//                  :350-393); then the choice itself (prmppi_controller.cu:232-304) so
//                  that the host needs one synchronisation per step.
#include "common.cuh"
#include "instance.cuh"
#include "launch.h"

namespace dr
{

constexpr int PRB = 128;
// Rollout CTA: 448 threads (56 samples x 8 hypotheses), two CTAs per SM (72 registers a
// thread), whose warps take a barrier every step (`__syncthreads_or` on the still-running
// samples) so the warps that share an SM sub-partition fetch the same instructions; the
// benchmark's 4 x 2 x 8 x 2048 rollouts are then 296 CTAs, two on every SM in one wave
// (with 512 threads they were 256 CTAs, which left 40 SMs with one: 0.53 against 0.49 ms).
#ifndef PR_ROLL_TILE
#define PR_ROLL_TILE 448
#endif
// two CTAs a SM where one opponent keeps the state in 64 registers; one with two opponents
template <int NOPP>
constexpr int prRollMinBlocks()
{
    return NOPP <= 1 ? 2 : 1;
}
constexpr int PUB = 256;

__host__ __device__ __forceinline__ size_t pa16(size_t x)
{
    return (x + 15) & ~(size_t)15;
}

// Copies the host-filled part of EnvParams to shared memory and computes the
// device-filled part; the caller's next __syncthreads publishes both.
__device__ __forceinline__ void copyEnvP(EnvParams* dst, const EnvParams* src)
{
    for (int i = threadIdx.x; i < ENV_HOST_WORDS; i += blockDim.x)
        ((float*)dst)[i] = ((const float*)src)[i];
    envDeviceTerms(*dst, *src, threadIdx.x, blockDim.x);
}

template <int NA> __device__ __forceinline__ void loadState(DState<NA>& st, const dr_sim_state& s)
{
#pragma unroll
    for (int a = 0; a < NA; a++)
    {
        st.pos[2 * a] = s.pos[2 * a];
        st.pos[2 * a + 1] = s.pos[2 * a + 1];
        st.vel[2 * a] = s.vel[2 * a];
        st.vel[2 * a + 1] = s.vel[2 * a + 1];
        st.S[a] = s.S[a];
        st.lat[a] = s.lat_dist[a];
        st.laps[a] = s.laps[a];
    }
}

__global__ void __launch_bounds__(256) pr_prologue(const PrDev* __restrict__ insts, const PrIn* __restrict__ in, int nInst)
{
    __shared__ float sh[2 * DR_MAX_T * 2];
    const int inst = blockIdx.x;
    if (inst >= nInst)
        return;
    const PrDev& D = insts[inst];
    const PrIn& I = in[inst];
    const int T = D.cfg.T, P = D.cfg.P, nth = D.cfg.nth;
    for (int i = threadIdx.x; i < T * 2; i += blockDim.x)
    {
        sh[i] = D.nom[i];
        sh[T * 2 + i] = D.rob[i];
    }
    if (threadIdx.x < 4)
        D.stats[threadIdx.x] = 0;
    __syncthreads();
    for (int i = threadIdx.x; i < T * 2; i += blockDim.x)
    {
        int t = i >> 1, d = i & 1;
        D.nom[i] = (t < T - 1) ? sh[(t + 1) * 2 + d] : 0.0f;
        D.rob[i] = (t < T - 1) ? sh[T * 2 + (t + 1) * 2 + d] : 0.0f;
    }
    for (int p = threadIdx.x; p < P; p += blockDim.x)
    {
        float u = uniform_from_word(draw(D.cfg.k0, D.cfg.k1, (uint32_t)p, 0u, I.step, S_PR_THETA, 0).x);
        float accum = 0.0f;
        int theta = nth - 1;
        for (int i = 0; i < nth; i++)
        {
            accum += I.belief[i];
            if (u <= accum)
            {
                theta = i;
                break;
            }
        }
        D.thetas[p] = theta;
    }
}

struct PrRollSmem
{
    size_t env, grids, nom, red, total;
};

__host__ __device__ inline PrRollSmem prLayout(int T)
{
    auto a16 = [](size_t x) { return (x + 15) & ~(size_t)15; };
    PrRollSmem L;
    size_t off = 16;
    L.env = off;
    off = a16(off + sizeof(EnvParams));
    L.grids = off;
    off = a16(off + GRID_FLOATS * 4);
    L.nom = off;
    off = a16(off + (size_t)T * 2 * 4);
    L.red = off;
    off = a16(off + (size_t)PR_ROLL_TILE * 2 * 4);
    L.total = off;
    return L;
}

// pr_rollout's body for HPT > 1 slots per thread (see pr_rollout): thread i rolls out
// slots pg HPT .. pg HPT + HPT - 1 of sample i / (P / HPT), pg = i % (P / HPT).
template <int NOPP, int NTH, int HPT>
__device__ __forceinline__ void prRolloutShared(const PrDev& D, const PrIn& I, const Tile& tile, const EnvParams& E, const Track& tr, const float* sNom,
                                                float* red, int K, int T, int P, int robust, int spb)
{
    constexpr int NA = NOPP + 1;
    const int G = P / HPT;
    const int sl = threadIdx.x / G, pg = threadIdx.x % G;
    const int s = tile.s0 + sl;
    const bool valid = sl < spb && sl < tile.count;
    const uint32_t k0 = D.cfg.k0, k1 = D.cfg.k1, step = I.step;
    const SafetyMargin margin = safetyMargin(E, D.cfg.collDistFactor);
    float running[HPT], safe[HPT];
    bool active[HPT];
    int theta[HPT];
    DState<NA> st[HPT];
    EnvNoise rng[HPT];
    DState<1> ego;
    {
        DState<NA> s0;
        loadState<NA>(s0, I.state);
        s0.locate(E.trackLength);
        ego.pos[0] = s0.pos[0];
        ego.pos[1] = s0.pos[1];
        ego.vel[0] = s0.vel[0];
        ego.vel[1] = s0.vel[1];
        ego.S[0] = s0.S[0];
        ego.lat[0] = s0.lat[0];
        ego.laps[0] = s0.laps[0];
        ego.tp[0] = s0.tp[0];
#pragma unroll
        for (int h = 0; h < HPT; h++)
        {
            const int p = pg * HPT + h;
            running[h] = 0.0f;
            safe[h] = -INFINITY;
            active[h] = valid;
            theta[h] = D.thetas[p];
            st[h] = s0;
            rng[h] = EnvNoise(k0, k1, (uint32_t)s, ((((uint32_t)robust << 8) | (uint32_t)p) << 16), step, S_PR_ROLL_ENV);
        }
    }
    BState<NTH> bs{};
    float decay = 1.0f;
    for (int t = 0; t < T; t++)
    {
        bool any = false;
#pragma unroll
        for (int h = 0; h < HPT; h++)
            any = any || active[h];
        // every thread of the CTA takes this barrier once per step (T is uniform)
        if (!__syncthreads_or(any))
            break;
        if (!any)
            continue;
        U4 r = draw(k0, k1, (uint32_t)s, (uint32_t)t, step, S_PR_EPS, 0);
        float ego0 = sNom[t * 2] + scaled_normal(D.cfg.sigma0, r.x);
        float ego1 = sNom[t * 2 + 1] + scaled_normal(D.cfg.sigma1, r.y);
        EgoRow row;
        egoStep<false>(tr, E, ego0, ego1, ego, row);
#pragma unroll
        for (int h = 0; h < HPT; h++)
        {
            if (!active[h])
                continue;
            rng[h].begin_step((uint32_t)t);
            bool branched = false;
            StepOut o = envStep<NOPP, NTH, false, false, true, false, false, EnvNoise, true>(t, theta[h], tr, E, ego0, ego1, st[h], bs, branched, 0.0f,
                                                                                           rng[h], &row);
            if (o.term != TERM_NONE)
                active[h] = false;
            running[h] += decay * prStateCost(o, E, D.cfg.boundaryThresholdFactor, D.cfg.boundaryCost, D.cfg.winCost, D.cfg.oppWinCost);
            safe[h] = fmaxf(safe[h], prSafetyCost(o, margin));
        }
        decay *= DECAY;
    }
#pragma unroll
    for (int h = 0; h < HPT; h++)
    {
        const int p = pg * HPT + h;
        if (valid)
        {
            running[h] += finalCost<NOPP>(st[h], E, D.cfg.finalAdvWeight, D.cfg.finalOppAdvWeight);
            float* out = robust ? D.costRob : D.costNom;
            out[((size_t)p * K + s) * 2 + 0] = running[h];
            out[((size_t)p * K + s) * 2 + 1] = safe[h];
        }
        red[(sl * P + p) * 2] = running[h];
        red[(sl * P + p) * 2 + 1] = safe[h];
    }
    __syncthreads();
    // PRMPPIcostAvgKernel (prmppi_kernels.cu:134-166)
    if (valid && pg == 0)
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

// tile: inst, s0 (first sample), count (samples), aux (0 nominal / 1 robust)
// HPT hypothesis slots per thread (PR_ROLL_TILE / HPT threads a CTA, the same PR_ROLL_TILE slots):
// with HPT > 1 a thread rolls out HPT of its sample's slots side by side and moves the
// ego once for them (egoStep; envStep<..., EGO = true> then steps the opponents of each
// slot): the ego's motion depends on its own action only, the sample's perturbed plan,
// shared by every slot, so the costs are those of HPT = 1 bit for bit. Only for an ego
// that draws no noise (egoNoiseFree on every instance of the launch).
template <int NOPP, int NTH, int HPT = 1>
__global__ void __launch_bounds__(PR_ROLL_TILE / HPT, prRollMinBlocks<NOPP>()) pr_rollout(const PrDev* __restrict__ insts, const PrIn* __restrict__ in,
                                                                                    const Tile* __restrict__ tiles)
{
    constexpr int NA = NOPP + 1;
    extern __shared__ __align__(128) unsigned char smraw[];
    const Tile tile = tiles[blockIdx.x];
    const PrDev& D = insts[tile.inst];
    const PrIn& I = in[tile.inst];
    const int K = D.cfg.K, T = D.cfg.T, P = D.cfg.P;
    const int robust = tile.aux;
    const PrRollSmem L = prLayout(T);
    uint64_t* bar = (uint64_t*)smraw;
    EnvParams* sE = (EnvParams*)(smraw + L.env);
    float* sGrid = (float*)(smraw + L.grids);
    float* sNom = (float*)(smraw + L.nom);
    float* red = (float*)(smraw + L.red);
    const uint32_t nomBytes = (uint32_t)pa16((size_t)T * 2 * 4);
    if (threadIdx.x == 0)
    {
        mbar_init(bar, 1);
        mbar_expect_tx(bar, GRID_FLOATS * 4 + nomBytes);
        bulk_g2s(sGrid, D.grids, GRID_FLOATS * 4, bar);
        bulk_g2s(sNom, robust ? D.rob : D.nom, nomBytes, bar);
    }
    copyEnvP(sE, &D.env);
    __syncthreads();
    if (!__syncthreads_and(mbar_wait(bar, 0)))
    {
        if (threadIdx.x == 0)
            atomicAdd(&D.stats[1], 1);
        return;
    }
    const EnvParams& E = *sE;
    const Track tr = trackIn(sGrid);
    const int spb = PR_ROLL_TILE / P;
    if constexpr (HPT > 1)
    {
        prRolloutShared<NOPP, NTH, HPT>(D, I, tile, E, tr, sNom, red, K, T, P, robust, spb);
        return;
    }
    const int sl = threadIdx.x / P, p = threadIdx.x % P;
    const int s = tile.s0 + sl;
    const bool valid = sl < spb && sl < tile.count;
    float running = 0.0f, safe = -INFINITY;
    {
        const int theta = D.thetas[p];
        DState<NA> st;
        loadState<NA>(st, I.state);
        st.locate(E.trackLength);
        BState<NTH> bs{};
        const uint32_t k0 = D.cfg.k0, k1 = D.cfg.k1, step = I.step;
        EnvNoise rng(k0, k1, (uint32_t)s, ((((uint32_t)robust << 8) | (uint32_t)p) << 16), step, S_PR_ROLL_ENV);
        float decay = 1.0f;
        const SafetyMargin margin = safetyMargin(E, D.cfg.collDistFactor);
        bool active = valid;
        for (int t = 0; t < T; t++)
        {
            // every thread of the CTA takes this barrier once per step (T is uniform); it
            // keeps the warps on the same step and ends the loop once all samples are done
            if (!__syncthreads_or(active))
                break;
            if (!active)
                continue;
            rng.begin_step((uint32_t)t);
            U4 r = draw(k0, k1, (uint32_t)s, (uint32_t)t, step, S_PR_EPS, 0);
            float ego0 = sNom[t * 2] + scaled_normal(D.cfg.sigma0, r.x);
            float ego1 = sNom[t * 2 + 1] + scaled_normal(D.cfg.sigma1, r.y);
            bool branched = false;
            StepOut o = envStep<NOPP, NTH, false, false, true, false>(t, theta, tr, E, ego0, ego1, st, bs, branched, 0.0f, rng);
            if (o.term != TERM_NONE)
                active = false;
            running += decay * prStateCost(o, E, D.cfg.boundaryThresholdFactor, D.cfg.boundaryCost, D.cfg.winCost, D.cfg.oppWinCost);
            safe = fmaxf(safe, prSafetyCost(o, margin));
            decay *= DECAY;
        }
        if (valid)
        {
            running += finalCost<NOPP>(st, E, D.cfg.finalAdvWeight, D.cfg.finalOppAdvWeight);
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

// block per (inst, which, t); tile.s0 = which * T + t
__global__ void __launch_bounds__(PUB) pr_weighted(const PrDev* __restrict__ insts, const PrIn* __restrict__ in, const Tile* __restrict__ tiles)
{
    __shared__ float sA[PUB], sB[PUB], sC[PUB];
    __shared__ float sMin[PUB / 32];
    const Tile tile = tiles[blockIdx.x];
    const PrDev& D = insts[tile.inst];
    const PrIn& I = in[tile.inst];
    const int K = D.cfg.K, T = D.cfg.T;
    const int which = tile.s0 / T, t = tile.s0 % T;
    const int tid = threadIdx.x;
    // which 0: nominal + full cost; 1: robust + full cost; 2: robust + safety cost
    const float* arr = D.avg + (size_t)(which == 0 ? 0 : K) * 2 + (which == 2 ? 1 : 0);
    const float* nominal = which == 0 ? D.nom : D.rob;
    float mn = INFINITY;
    for (int s = tid; s < K; s += PUB)
        mn = fminf(mn, arr[(size_t)s * 2]);
    mn = warp_min(mn);
    if ((tid & 31) == 0)
        sMin[tid >> 5] = mn;
    __syncthreads();
    float minCost = sMin[0];
#pragma unroll
    for (int w = 1; w < PUB / 32; w++)
        minCost = fminf(minCost, sMin[w]);
    const float invTemp = I.lambda[which];
    const float nom0 = nominal[t * 2], nom1 = nominal[t * 2 + 1];
    const uint32_t k0 = D.cfg.k0, k1 = D.cfg.k1, step = I.step;
    float num0 = 0.0f, num1 = 0.0f, den = 0.0f;
    for (int s = tid; s < K; s += PUB)
    {
        float cost = arr[(size_t)s * 2];
        float w = expf(-(cost - minCost) / invTemp);
        U4 r = draw(k0, k1, (uint32_t)s, (uint32_t)t, step, S_PR_EPS, 0);
        float u0 = nom0 + scaled_normal(D.cfg.sigma0, r.x);
        float u1 = nom1 + scaled_normal(D.cfg.sigma1, r.y);
        num0 += w * u0;
        num1 += w * u1;
        den += w;
    }
    sA[tid] = num0;
    sB[tid] = num1;
    sC[tid] = den;
    __syncthreads();
#pragma unroll
    for (int stride = PUB / 2; stride >= 32; stride >>= 1)
    {
        if (tid < stride)
        {
            sA[tid] += sA[tid + stride];
            sB[tid] += sB[tid + stride];
            sC[tid] += sC[tid + stride];
        }
        __syncthreads();
    }
    if (tid < 32)
    {
        float a0 = sA[tid], a1 = sB[tid], dd = sC[tid];
#pragma unroll
        for (int stride = 16; stride > 0; stride >>= 1)
        {
            a0 += __shfl_down_sync(0xffffffffu, a0, stride);
            a1 += __shfl_down_sync(0xffffffffu, a1, stride);
            dd += __shfl_down_sync(0xffffffffu, dd, stride);
        }
        if (tid == 0)
        {
            float* out = which == 0 ? D.cand1 : (which == 1 ? D.cand2 : D.robWork);
            out[t * 2] = (dd > 1e-30f) ? a0 / dd : nom0;
            out[t * 2 + 1] = (dd > 1e-30f) ? a1 / dd : nom1;
            if (t == 0)
            {
                D.nu[which] = dd;
                D.minCosts[which] = minCost;
            }
        }
    }
}

// ---------------------------------------------------------------------------------------
// sample-sharded update of one controller (dr_prmppi_shard_*): this process holds samples
// [sLo, sHi) of every hypothesis. pr_shard_min: the three minima (nominal + full cost,
// robust + full cost, robust + safety cost) over its samples; pr_shard_sums: its weighted
// sums of the absolute controls with those local minima (per (which, t): sum w u0,
// sum w u1, sum w); the processes all-gather both (one exchange), and pr_shard_merge takes
// the global minima and rescales every process's sums to them by exp(-(m_r - m) / lambda);
// pr_shard_apply: the weighted averages from the merged sums, as pr_weighted writes them.
// ---------------------------------------------------------------------------------------
__device__ __forceinline__ const float* prArr(const PrDev& D, int which)
{
    return D.avg + (size_t)(which == 0 ? 0 : D.cfg.K) * 2 + (which == 2 ? 1 : 0);
}

__global__ void __launch_bounds__(PUB) pr_shard_min(const PrDev* __restrict__ insts, float* __restrict__ mins)
{
    __shared__ float sMin[PUB / 32];
    const PrDev& D = insts[0];
    const int which = blockIdx.x, tid = threadIdx.x;
    const float* arr = prArr(D, which);
    float mn = INFINITY;
    for (int s = D.cfg.sLo + tid; s < D.cfg.sHi; s += PUB)
        mn = fminf(mn, arr[(size_t)s * 2]);
    mn = warp_min(mn);
    if ((tid & 31) == 0)
        sMin[tid >> 5] = mn;
    __syncthreads();
    if (tid == 0)
    {
        float m = sMin[0];
#pragma unroll
        for (int w = 1; w < PUB / 32; w++)
            m = fminf(m, sMin[w]);
        mins[which] = m;
    }
}

// block per (which, t)
__global__ void __launch_bounds__(PUB) pr_shard_sums(const PrDev* __restrict__ insts, const PrIn* __restrict__ in, const float* __restrict__ mins,
                                                     float* __restrict__ sums)
{
    __shared__ float sA[PUB], sB[PUB], sC[PUB];
    const PrDev& D = insts[0];
    const PrIn& I = in[0];
    const int T = D.cfg.T;
    const int which = blockIdx.x / T, t = blockIdx.x % T, tid = threadIdx.x;
    const float* arr = prArr(D, which);
    const float* nominal = which == 0 ? D.nom : D.rob;
    const float minCost = mins[which];
    const float invTemp = I.lambda[which];
    const float nom0 = nominal[t * 2], nom1 = nominal[t * 2 + 1];
    const uint32_t k0 = D.cfg.k0, k1 = D.cfg.k1, step = I.step;
    float num0 = 0.0f, num1 = 0.0f, den = 0.0f;
    for (int s = D.cfg.sLo + tid; s < D.cfg.sHi; s += PUB)
    {
        float cost = arr[(size_t)s * 2];
        float w = expf(-(cost - minCost) / invTemp);
        U4 r = draw(k0, k1, (uint32_t)s, (uint32_t)t, step, S_PR_EPS, 0);
        float u0 = nom0 + scaled_normal(D.cfg.sigma0, r.x);
        float u1 = nom1 + scaled_normal(D.cfg.sigma1, r.y);
        num0 += w * u0;
        num1 += w * u1;
        den += w;
    }
    sA[tid] = num0;
    sB[tid] = num1;
    sC[tid] = den;
    __syncthreads();
#pragma unroll
    for (int stride = PUB / 2; stride >= 32; stride >>= 1)
    {
        if (tid < stride)
        {
            sA[tid] += sA[tid + stride];
            sB[tid] += sB[tid + stride];
            sC[tid] += sC[tid + stride];
        }
        __syncthreads();
    }
    if (tid < 32)
    {
        float a0 = sA[tid], a1 = sB[tid], dd = sC[tid];
#pragma unroll
        for (int stride = 16; stride > 0; stride >>= 1)
        {
            a0 += __shfl_down_sync(0xffffffffu, a0, stride);
            a1 += __shfl_down_sync(0xffffffffu, a1, stride);
            dd += __shfl_down_sync(0xffffffffu, dd, stride);
        }
        if (tid == 0)
        {
            float* o = sums + ((size_t)which * T + t) * 3;
            o[0] = a0;
            o[1] = a1;
            o[2] = dd;
        }
    }
}

__global__ void __launch_bounds__(PUB) pr_shard_apply(const PrDev* __restrict__ insts, const float* __restrict__ mins, const float* __restrict__ sums)
{
    const PrDev& D = insts[0];
    const int T = D.cfg.T;
    for (int i = threadIdx.x; i < 3 * T; i += blockDim.x)
    {
        const int which = i / T, t = i % T;
        const float* nominal = which == 0 ? D.nom : D.rob;
        const float* sm = sums + (size_t)i * 3;
        const float dd = sm[2];
        float* out = which == 0 ? D.cand1 : (which == 1 ? D.cand2 : D.robWork);
        out[t * 2] = (dd > 1e-30f) ? sm[0] / dd : nominal[t * 2];
        out[t * 2 + 1] = (dd > 1e-30f) ? sm[1] / dd : nominal[t * 2 + 1];
        if (t == 0)
        {
            D.nu[which] = dd;
            D.minCosts[which] = mins[which];
        }
    }
}

// gathered[r * words + ...] = process r's (3 minima, 3 x T x 3 sums), rank order
__global__ void __launch_bounds__(PUB) pr_shard_merge(const PrDev* __restrict__ insts, const PrIn* __restrict__ in, const float* __restrict__ gathered,
                                                      int words, int world, float* __restrict__ mins, float* __restrict__ sums)
{
    const PrDev& D = insts[0];
    const int T = D.cfg.T;
    __shared__ float sMin[3];
    if (threadIdx.x < 3)
    {
        float m = INFINITY;
        for (int r = 0; r < world; r++)
            m = fminf(m, gathered[(size_t)r * words + threadIdx.x]);
        sMin[threadIdx.x] = m;
        mins[threadIdx.x] = m;
    }
    __syncthreads();
    for (int i = threadIdx.x; i < 3 * T; i += blockDim.x)
    {
        const int which = i / T;
        const float m = sMin[which], invTemp = in[0].lambda[which];
        float a0 = 0.0f, a1 = 0.0f, dd = 0.0f;
        if (!isinf(m))
            for (int r = 0; r < world; r++)
            {
                const float* g = gathered + (size_t)r * words;
                if (isinf(g[which]))
                    continue;
                const float f = expf(-(g[which] - m) / invTemp);
                const float* p = g + 3 + (size_t)i * 3;
                a0 += p[0] * f;
                a1 += p[1] * f;
                dd += p[2] * f;
            }
        sums[i * 3] = a0;
        sums[i * 3 + 1] = a1;
        sums[i * 3 + 2] = dd;
    }
}

cudaError_t launchPrShardMerge(cudaStream_t stream, const PrDev* insts, const PrIn* in, const float* gathered, int words, int world, float* mins,
                               float* sums)
{
    pr_shard_merge<<<1, PUB, 0, stream>>>(insts, in, gathered, words, world, mins, sums);
    return cudaGetLastError();
}

cudaError_t launchPrShardMin(cudaStream_t stream, const PrDev* insts, float* mins)
{
    pr_shard_min<<<3, PUB, 0, stream>>>(insts, mins);
    return cudaGetLastError();
}

cudaError_t launchPrShardSums(cudaStream_t stream, const PrDev* insts, const PrIn* in, int T, const float* mins, float* sums)
{
    pr_shard_sums<<<3 * T, PUB, 0, stream>>>(insts, in, mins, sums);
    return cudaGetLastError();
}

cudaError_t launchPrShardApply(cudaStream_t stream, const PrDev* insts, const float* mins, const float* sums)
{
    pr_shard_apply<<<1, PUB, 0, stream>>>(insts, mins, sums);
    return cudaGetLastError();
}

// one block per instance: threads (kind, cand, p), kind 0 = full cost, 1 = safety re-check
template <int NOPP, int NTH>
__global__ void __launch_bounds__(PRB) pr_candidates(const PrDev* __restrict__ insts, const PrIn* __restrict__ in, int nInst)
{
    constexpr int NA = NOPP + 1;
    extern __shared__ __align__(128) unsigned char smraw[];
    __shared__ int sChosen;
    const int inst = blockIdx.x;
    if (inst >= nInst)
        return;
    const PrDev& D = insts[inst];
    const PrIn& I = in[inst];
    const int T = D.cfg.T, P = D.cfg.P;
    uint64_t* bar = (uint64_t*)smraw;
    EnvParams* sE = (EnvParams*)(smraw + 16);
    const size_t offG = pa16(16 + sizeof(EnvParams));
    float* sGrid = (float*)(smraw + offG);
    float* sC1 = (float*)(smraw + offG + GRID_FLOATS * 4);
    const uint32_t cb = (uint32_t)pa16((size_t)T * 2 * 4);
    float* sC2 = (float*)((unsigned char*)sC1 + cb);
    if (threadIdx.x == 0)
    {
        mbar_init(bar, 1);
        mbar_expect_tx(bar, GRID_FLOATS * 4 + 2 * cb);
        bulk_g2s(sGrid, D.grids, GRID_FLOATS * 4, bar);
        bulk_g2s(sC1, D.cand1, cb, bar);
        bulk_g2s(sC2, D.cand2, cb, bar);
    }
    copyEnvP(sE, &D.env);
    __syncthreads();
    if (!__syncthreads_and(mbar_wait(bar, 0)))
    {
        if (threadIdx.x == 0)
            atomicAdd(&D.stats[1], 1);
        return;
    }
    const EnvParams& E = *sE;
    const Track tr = trackIn(sGrid);
    const uint32_t k0 = D.cfg.k0, k1 = D.cfg.k1, step = I.step;
    for (int task = threadIdx.x; task < 4 * P; task += blockDim.x)
    {
        const int kind = task / (2 * P);
        const int tid = task % (2 * P);
        const int second = tid >= P;
        const int p = second ? tid - P : tid;
        const float* nominal = second ? sC2 : sC1;
        const int theta = D.thetas[p];
        DState<NA> st;
        loadState<NA>(st, I.state);
        st.locate(E.trackLength);
        BState<NTH> bs{};
        EnvNoise rng(k0, k1, (uint32_t)p, (uint32_t)second << 16, step, kind ? S_PR_SAFE_ENV : S_PR_CAND_ENV);
        float cost = 0.0f, safeCost = -INFINITY, decay = 1.0f;
        const SafetyMargin margin = safetyMargin(E, D.cfg.collDistFactor);
        bool stop = false;
        for (int t = 0; t < T && !stop; ++t)
        {
            rng.begin_step((uint32_t)t);
            bool branched = false;
            StepOut o = envStep<NOPP, NTH, false, false, true, false>(t, theta, tr, E, nominal[t * 2], nominal[t * 2 + 1], st, bs, branched, 0.0f, rng);
            stop = (o.term != TERM_NONE);
            cost += decay * prStateCost(o, E, D.cfg.boundaryThresholdFactor, D.cfg.boundaryCost, D.cfg.winCost, D.cfg.oppWinCost);
            decay *= DECAY;
            safeCost = fmaxf(safeCost, prSafetyCost(o, margin));
        }
        cost += finalCost<NOPP>(st, E, D.cfg.finalAdvWeight, D.cfg.finalOppAdvWeight);
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
        D.decision[0] = c2 < c1;          // resetNom
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

// perturbation of the next step, reference layout noise[T][K][2] (test hook)
__global__ void pr_noise(const PrDev* __restrict__ insts, const PrIn* __restrict__ in, float* __restrict__ out)
{
    const PrDev& D = insts[0];
    const int K = D.cfg.K, T = D.cfg.T;
    size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (size_t)T * K)
        return;
    int s = (int)(i % K), t = (int)(i / K);
    U4 r = draw(D.cfg.k0, D.cfg.k1, (uint32_t)s, (uint32_t)t, in[0].step, S_PR_EPS, 0);
    out[i * 2] = scaled_normal(D.cfg.sigma0, r.x);
    out[i * 2 + 1] = scaled_normal(D.cfg.sigma1, r.y);
}

bool prSupported(int nopp, int nth)
{
    int key = nopp * 16 + nth;
    return key == 17 || key == 18 || key == 20 || key == 24 || key == 34;
}

int prRolloutSamplesPerBlock()
{
    return PR_ROLL_TILE;
}

size_t prRolloutSmem(int T)
{
    return prLayout(T).total;
}

static size_t prCandSmem(int T)
{
    return pa16(16 + sizeof(EnvParams)) + GRID_FLOATS * 4 + 2 * pa16((size_t)T * 2 * 4);
}

cudaError_t launchPrPrologue(const LaunchArgs& a, int nInst)
{
    pr_prologue<<<nInst, 256, 0, a.stream>>>(a.pr, a.prIn, nInst);
    return cudaGetLastError();
}

template <int NOPP, int NTH, int HPT> static cudaError_t prRollH(const LaunchArgs& a, size_t smem)
{
    auto k = pr_rollout<NOPP, NTH, HPT>;
    ensureSmem(k, smem);
    k<<<a.nTiles, PR_ROLL_TILE / HPT, smem, a.stream>>>(a.pr, a.prIn, a.tiles);
    return cudaGetLastError();
}

// a.prSlots hypothesis slots per thread (1, 2 or 4; the caller keeps it to 1 unless the
// launch's egos draw no noise and P is a multiple of it)
template <int NOPP, int NTH> static cudaError_t prRollT(const LaunchArgs& a, size_t smem)
{
    switch (a.prSlots)
    {
    case 2: return prRollH<NOPP, NTH, 2>(a, smem);
    case 4: return prRollH<NOPP, NTH, 4>(a, smem);
    default: return prRollH<NOPP, NTH, 1>(a, smem);
    }
}

template <int NOPP, int NTH> static cudaError_t prCandT(const LaunchArgs& a, int nInst, int T)
{
    auto k = pr_candidates<NOPP, NTH>;
    size_t smem = prCandSmem(T);
    ensureSmem(k, smem);
    k<<<nInst, PRB, smem, a.stream>>>(a.pr, a.prIn, nInst);
    return cudaGetLastError();
}

#define DR_PR_DISPATCH(NOPP_, NTH_, CALL)                                                                                                            \
    switch (NOPP_ * 16 + NTH_)                                                                                                                       \
    {                                                                                                                                                \
    case 1 * 16 + 1: return CALL(1, 1);                                                                                                             \
    case 1 * 16 + 2: return CALL(1, 2);                                                                                                             \
    case 1 * 16 + 4: return CALL(1, 4);                                                                                                             \
    case 1 * 16 + 8: return CALL(1, 8);                                                                                                             \
    case 2 * 16 + 2: return CALL(2, 2);                                                                                                             \
    default: return cudaErrorInvalidValue;                                                                                                           \
    }

cudaError_t launchPrRollout(const LaunchArgs& a, int nopp, int nth, size_t smem)
{
#define CALL(P_, Q_) prRollT<P_, Q_>(a, smem)
    DR_PR_DISPATCH(nopp, nth, CALL)
#undef CALL
}

cudaError_t launchPrReduce(const LaunchArgs& a)
{
    pr_weighted<<<a.nTiles, PUB, 0, a.stream>>>(a.pr, a.prIn, a.tiles);
    return cudaGetLastError();
}

cudaError_t launchPrCandidates(const LaunchArgs& a, int nopp, int nth, int nInst, int maxT, size_t)
{
#define CALL(P_, Q_) prCandT<P_, Q_>(a, nInst, maxT)
    DR_PR_DISPATCH(nopp, nth, CALL)
#undef CALL
}

cudaError_t launchPrNoise(const LaunchArgs& a, size_t n, float* out)
{
    pr_noise<<<(unsigned)((n + 255) / 256), 256, 0, a.stream>>>(a.pr, a.prIn, out);
    return cudaGetLastError();
}

} // namespace dr
