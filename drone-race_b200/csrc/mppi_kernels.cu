// MPPI control-step kernels (reference: src/kernels.cu; host sequence
// src/mppi_controller.cu:250-466).
//
//   mppi_prologue   warm-start shift decided by the previous step (mppi_controller.cu:
//                   426-456 + shiftSplineKernel, kernels.cu:461-486), zeroes the
//                   verification histograms.
//   mppi_rollout    fused perturbation draw + rollout + running/terminal cost + branch
//                   bookkeeping (fullRolloutKernel, kernels.cu:34-171) + per-branch cost
//                   aggregation (aggregateBranchCostsKernel, kernels.cu:175-217). One
//                   thread per (sample, hypothesis); the state stays in registers; the
//                   track, the control sequence and the spline basis are staged in shared
//                   memory by bulk copies; the perturbation is drawn from Philox instead of
//                   being read from a stored noise tensor.
//   mppi_update     per (branch plan, knot): masked minimum, exponential weights and the
//                   weighted average of the regenerated perturbations in one block
//                   (computeMaskedMinCostsKernel + weightedAverageKernelUnified,
//                   kernels.cu:221-408; the sums are accumulated in the reference's
//                   256-thread order); the last block of an instance to finish also does
//                   the spline interpolation and the clamp (kernels.cu:411-456).
//   mppi_verify     Monte-Carlo failure counts of the new and the previous plan
//                   (verifyNominalFailureKernel, kernels.cu:488-551), both plans in one grid.
#include <cstdio>
#include <type_traits>

#include "common.cuh"
#include "instance.cuh"
#include "launch.h"

namespace dr
{

// Rollout block size: RB / n_theta samples a CTA, one thread per (sample, hypothesis), up
// to 128 registers a thread. 256: a rollout CTA takes the registers of one verification
// CTA, so in the overlapped step the SMs that hold one run one verification CTA beside it
// (128 CTAs for 4 x 4096 x 2 threads; 1.53 against 1.55 ms per step with 128-thread CTAs,
// which spread over every SM; 512-thread CTAs: 1.55 ms, the rollout alone 0.39 against
// 0.32 ms).
#ifndef DR_ROLLOUT_BLOCK
#define DR_ROLLOUT_BLOCK 256
#endif
constexpr int RB = DR_ROLLOUT_BLOCK;
constexpr int RB_MIN_BLOCKS = RB <= 128 ? 4 : 512 / RB; // register budget of 128 a thread
// Verification CTAs per SM that the register allocation is sized for (VERIFY_TILE = 512
// threads a CTA: 2 -> 64 registers a thread). Measured on the 4 x 2^17 x 40 verification
// of both plans (B200, 1965 MHz), exact arithmetic and a CTA barrier every step:
// 128-thread CTAs without the barrier 3.14 ms (72 registers); 128 with the barrier 3.05;
// 256 x 3 CTAs 2.90; 512 x 2 2.73; 1024 x 1 2.74. The barrier kept the warps of a CTA on
// the same step, where they fetched the same instructions of the then 55 KB kernel. The
// fast flavour with the ego tables is smaller and the barrier only held warps back: with
// it every 1 / 2 / 4 / 16 / 32 steps 1.292 / 1.272 / 1.200 / 1.180 / 1.174 ms, without it
// 1.171, so the warps now step on their own and leave the loop when their samples are done.
// The larger models (two opponents, or eight hypotheses) spill heavily at 64 registers
// and get one CTA per SM instead.
#ifndef VERIFY_MIN_BLOCKS
#define VERIFY_MIN_BLOCKS 2
#endif
template <int NOPP, int NTH> constexpr int verifyMinBlocks()
{
    return (NOPP == 1 && NTH <= 4) ? VERIFY_MIN_BLOCKS : 1;
}
constexpr int UB = 256; // update block size (the reference's reduction width)

__device__ __forceinline__ int infoPred(int v)
{
    return v >> 16;
}
__device__ __forceinline__ int infoTime(int v)
{
    return (int)(short)(v & 0xffff);
}

// Copies the host-filled part of EnvParams to shared memory and computes the
// device-filled part; the caller's next __syncthreads publishes both.
__device__ __forceinline__ void copyEnv(EnvParams* dst, const EnvParams* src)
{
    for (int i = threadIdx.x; i < ENV_HOST_WORDS; i += blockDim.x)
        ((float*)dst)[i] = ((const float*)src)[i];
    envDeviceTerms(*dst, *src, threadIdx.x, blockDim.x);
}

__host__ __device__ __forceinline__ size_t align16(size_t x)
{
    return (x + 15) & ~(size_t)15;
}

// ---------------------------------------------------------------------------------------
// prologue: apply the previous step's warm-start shift
// ---------------------------------------------------------------------------------------
__global__ void __launch_bounds__(256) mppi_prologue(const MppiDev* __restrict__ insts, const MppiIn* __restrict__ in, int nInst)
{
    extern __shared__ float sh[];
    const int inst = blockIdx.x;
    if (inst >= nInst)
        return;
    const MppiDev& D = insts[inst];
    const MppiIn& I = in[inst];
    const int T = D.cfg.T, M = D.cfg.M, nbp = D.cfg.nth + 1;
    for (int i = threadIdx.x; i < 2 * T; i += blockDim.x)
        D.fail[i] = 0u;
    if (threadIdx.x < 4)
        D.stats[threadIdx.x] = 0;
    const int b = I.pendBranch;
    if (b < 0 || b >= nbp)
        return;
    // prevDense := shift(chosen dense plan) on branch b (host shift, mppi_controller.cu:430-436)
    const float* src = I.pendUseNew ? D.dense : D.prevDense;
    const int n = nbp * T * 2;
    for (int i = threadIdx.x; i < n; i += blockDim.x)
        sh[i] = src[i];
    __syncthreads();
    for (int i = threadIdx.x; i < n; i += blockDim.x)
    {
        int d = i & 1, t = (i >> 1) % T, bb = (i >> 1) / T;
        float v = sh[i];
        if (bb == b)
            v = (t < T - 1) ? sh[(bb * T + t + 1) * 2 + d] : 0.0f;
        D.prevDense[i] = v;
        D.dense[i] = v;
        if (!D.cfg.useSplines)
            D.knots[i] = v; // dense mode: the optimised sequence restarts from the shifted plan
    }
    if (D.cfg.useSplines)
    {
        // shiftSplineKernel on branch b (kernels.cu:461-486)
        float* old = sh + n;
        for (int i = threadIdx.x; i < M * 2; i += blockDim.x)
            old[i] = D.knots[(b * M) * 2 + i];
        __syncthreads();
        for (int i = threadIdx.x; i < M * 2; i += blockDim.x)
        {
            int dim = i & 1, newm = i >> 1;
            float sum = 0.0f;
            int tEval = D.cfg.knots[newm] + 1;
            if (tEval >= T)
                tEval = T - 1;
            for (int m = 0; m < M; m++)
                sum += D.B[tEval * M + m] * old[m * 2 + dim];
            D.knots[(b * M + newm) * 2 + dim] = sum;
        }
    }
}

// ---------------------------------------------------------------------------------------
// rollout + aggregation
// ---------------------------------------------------------------------------------------
struct RolloutSmem
{
    size_t env, grids, knots, B, vbuf, red, total;
};

__host__ __device__ inline RolloutSmem rolloutLayout(int nbp, int T, int M, bool spl)
{
    auto a16 = [](size_t x) { return (x + 15) & ~(size_t)15; };
    RolloutSmem L;
    size_t off = 16; // mbarrier
    L.env = off;
    off = a16(off + sizeof(EnvParams));
    L.grids = off;
    off = a16(off + GRID_FLOATS * 4);
    L.knots = off;
    off = a16(off + (size_t)nbp * M * 2 * 4);
    L.B = off;
    if (spl)
        off = a16(off + (size_t)T * M * 4);
    L.vbuf = off;
    if (spl)
        off = a16(off + (size_t)M * 2 * RB * 4);
    L.red = off;
    off = a16(off + RB * 4);
    L.total = off;
    return L;
}

// One rollout tile: SPB samples x NTH hypotheses, a thread each, with the tile's
// instance already staged in shared memory; then the tile's aggregation.
template <int NOPP, int NTH, bool SPL, bool LOCK>
__device__ __forceinline__ void rolloutTile(const MppiDev& D, const MppiIn& I, const Tile& tile, int K, int T, int M, const EnvParams& E, const float* sGrid,
                                            const float* sKn, const float* sB, float* vbuf, float* red)
{
    constexpr int NA = NOPP + 1;
    const Track tr = trackIn(sGrid);

    const int th = threadIdx.x % NTH;
    const int sl = threadIdx.x / NTH;
    const int s = tile.s0 + sl;
    const bool valid = sl < tile.count;
    const float minConf = D.cfg.minConf;
    const uint32_t k0 = D.cfg.k0, k1 = D.cfg.k1, step = I.step;
    const float sig0 = D.cfg.sigma0, sig1 = D.cfg.sigma1;

    float belief0[NTH];
#pragma unroll
    for (int i = 0; i < NTH; i++)
        belief0[i] = I.belief[i];
    // initBranchState (state.h:154-163)
    const int pt0 = findConfident<NTH>(belief0, minConf);
    const int bt0 = pt0 == 0 ? -1 : 0;
    const bool compatible = (pt0 == 0 || pt0 == th + 1);

    float cost = INFINITY;
    int pt = pt0, bt = bt0;
    bool active = valid && compatible; // with LOCK, idle and incompatible lanes still take the barriers
    if (LOCK || active)
    {
        DState<NA> st;
#pragma unroll
        for (int a = 0; a < NA; a++)
        {
            st.pos[2 * a] = I.state.pos[2 * a];
            st.pos[2 * a + 1] = I.state.pos[2 * a + 1];
            st.vel[2 * a] = I.state.vel[2 * a];
            st.vel[2 * a + 1] = I.state.vel[2 * a + 1];
            st.S[a] = I.state.S[a];
            st.lat[a] = I.state.lat_dist[a];
            st.laps[a] = I.state.laps[a];
        }
        st.locate(E.trackLength);
        BState<NTH> bs;
#pragma unroll
        for (int i = 0; i < NTH; i++)
            bs.belief[i] = belief0[i];
        bs.predTheta = pt0;
        bs.branchingTime = bt0;
        if (active)
            cost = 0.0f;
        float decay = 1.0f;
        int tOrigin = 0;
        EnvNoise rng(k0, k1, (uint32_t)s, (uint32_t)th << 16, step, S_MPPI_ROLL_ENV);
        int curB = -1;
        for (int t = 0; t < T; t++)
        {
            if constexpr (LOCK)
            {
                // every thread of the CTA takes this barrier once per step (T is uniform),
                // keeping the warps on the same step
                if (!__syncthreads_or(active))
                    break;
                if (!active)
                    continue;
            }
            else if (!active)
                break; // the thread's rollout ended
            rng.begin_step((uint32_t)t);
            const int local = t - tOrigin;
            const int b = bs.predTheta;
            float ego0, ego1;
            if constexpr (SPL)
            {
                if (b != curB)
                {
                    // nominal + perturbation of this sample's knots for branch b
                    for (int m = 0; m < M; m++)
                    {
                        U4 r = draw(k0, k1, (uint32_t)s, (uint32_t)(b * M + m), step, S_MPPI_EPS, 0);
                        float e0 = scaled_normal(sig0, r.x);
                        float e1 = scaled_normal(sig1, r.y);
                        vbuf[(m * 2 + 0) * RB + threadIdx.x] = sKn[(b * M + m) * 2 + 0] + e0;
                        vbuf[(m * 2 + 1) * RB + threadIdx.x] = sKn[(b * M + m) * 2 + 1] + e1;
                    }
                    curB = b;
                }
                const float* Brow = sB + local * M;
                float sum = 0.0f;
                for (int m = 0; m < M; m++)
                    sum += Brow[m] * vbuf[(m * 2 + 0) * RB + threadIdx.x];
                ego0 = sum;
                sum = 0.0f;
                for (int m = 0; m < M; m++)
                    sum += Brow[m] * vbuf[(m * 2 + 1) * RB + threadIdx.x];
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
            StepOut o = envStep<NOPP, NTH, true, true, true, true>(t, th, tr, E, ego0, ego1, st, bs, branched, minConf, rng);
            if (branched)
                tOrigin = t + 1;
            if (o.term != TERM_NONE)
                active = false;
            cost += stateCost(o, E, D.cfg.w) * decay;
            decay *= DECAY;
        }
        if (valid && compatible)
        {
            cost += finalCost<NOPP>(st, E, D.cfg.w.finalAdvWeight, D.cfg.w.finalOppAdvWeight);
            pt = bs.predTheta;
            bt = bs.branchingTime;
        }
    }
    if (valid)
    {
        D.costsTrue[th * K + s] = cost;
        D.binfo[th * K + s] = packInfo(pt, bt);
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

template <int NOPP, int NTH, bool SPL, bool PQ, bool LOCK>
__global__ void __launch_bounds__(RB, RB_MIN_BLOCKS) mppi_rollout(const MppiDev* __restrict__ insts, const MppiIn* __restrict__ in,
                                                                       const Tile* __restrict__ tiles, int nTiles, unsigned* __restrict__ queue)
{
    constexpr int NBP = NTH + 1;
    extern __shared__ __align__(128) unsigned char smraw[];
    __shared__ int sTicket;
    pdl_trigger(); // the update may launch once every rollout CTA has started
    uint64_t* bar = (uint64_t*)smraw;
    if (threadIdx.x == 0)
        mbar_init(bar, 1);
    int staged = -1;     // instance whose track, knots and basis are in shared memory
    uint32_t phase = 0u; // parity of the staging barrier's next phase
    for (int iter = 0;; iter++)
    {
        const int ti = nextTile(PQ ? queue : nullptr, iter, &sTicket);
        if (ti >= nTiles)
            break;
        const Tile tile = tiles[ti];
        const MppiDev& D = insts[tile.inst];
        const MppiIn& I = in[tile.inst];
        const int K = D.cfg.K, T = D.cfg.T, M = D.cfg.M;
        const RolloutSmem L = rolloutLayout(NBP, T, M, SPL);
        EnvParams* sE = (EnvParams*)(smraw + L.env);
        float* sGrid = (float*)(smraw + L.grids);
        float* sKn = (float*)(smraw + L.knots);
        float* sB = (float*)(smraw + L.B);
        float* vbuf = (float*)(smraw + L.vbuf);
        float* red = (float*)(smraw + L.red);
        if (tile.inst != staged)
        {
            const uint32_t knBytes = (uint32_t)align16((size_t)NBP * M * 2 * 4);
            const uint32_t bBytes = SPL ? (uint32_t)align16((size_t)T * M * 4) : 0u;
            if (threadIdx.x == 0)
            {
                mbar_expect_tx(bar, GRID_FLOATS * 4 + knBytes + bBytes);
                if (!D.cfg.dbgNoStage)
                {
                    bulk_g2s(sGrid, D.grids, GRID_FLOATS * 4, bar);
                    bulk_g2s(sKn, D.knots, knBytes, bar);
                    if (SPL)
                        bulk_g2s(sB, D.B, bBytes, bar);
                }
            }
            copyEnv(sE, &D.env);
            __syncthreads();
            if (!__syncthreads_and(mbar_wait(bar, phase, D.cfg.waitPolls)))
            {
                // The staging did not complete within the poll limit: write the tile's
                // defined timeout outputs, count the timeout for the host, return.
                rolloutTileTimedOut<NTH>(D, I, tile, K);
                if (threadIdx.x == 0)
                    atomicAdd(&D.stats[1], 1);
                return;
            }
            phase ^= 1u;
            staged = tile.inst;
        }
        rolloutTile<NOPP, NTH, SPL, LOCK>(D, I, tile, K, T, M, *sE, sGrid, sKn, sB, vbuf, red);
        __syncthreads(); // the next tile's staging and reduction buffer reuse shared memory
    }
}

// aggregation alone (used by the update test hook, which takes costsTrue as input)
template <int NTH> __global__ void mppi_aggregate(const MppiDev* __restrict__ insts, const MppiIn* __restrict__ in)
{
    const MppiDev& D = insts[0];
    const MppiIn& I = in[0];
    const int K = D.cfg.K;
    int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= K)
        return;
    float num = 0.0f, den = 0.0f;
    for (int m = 0; m < NTH; m++)
    {
        float cv = D.costsTrue[m * K + s];
        if (!isfinite(cv))
            continue;
        float w = I.belief[m];
        num += w * cv;
        den += w;
    }
    D.costs[s] = (den > 1e-30f) ? (num / den) : INFINITY;
    for (int th = 0; th < NTH; th++)
    {
        float n2 = 0.0f, d2 = 0.0f;
        float cv = D.costsTrue[th * K + s];
        if (isfinite(cv))
        {
            float w = I.belief[th];
            n2 += w * cv;
            d2 += w;
        }
        D.costs[(size_t)(th + 1) * K + s] = (d2 > 1e-30f) ? (n2 / d2) : INFINITY;
    }
}

// ---------------------------------------------------------------------------------------
// update
// ---------------------------------------------------------------------------------------
// sampleContributed (state.h:203-219) for one factor.
__device__ __forceinline__ bool contributed(int b, int tLocal, int bt, int pt, int T)
{
    int origin = (b != 0 && bt > 0) ? bt : 0;
    int tGlobal = tLocal + origin;
    if (tGlobal >= T)
        return false;
    if ((b != 0 && b != pt) || (b == 0 && pt != 0 && tGlobal >= bt))
        return false;
    return true;
}

template <int NTH>
__device__ __forceinline__ float sampleCoeff(const MppiDev& D, const float (&belief)[NTH], int b, int k, int s, bool spl, int T, int M, int K)
{
    float coeff = 0.0f;
#pragma unroll
    for (int th = 0; th < NTH; th++)
    {
        if (belief[th] <= 0.0f)
            continue;
        if (!(b == 0 || b == th + 1))
            continue;
        int v = D.binfo[th * K + s];
        int pt = infoPred(v), bt = infoTime(v);
        bool c;
        if (spl) // splineSampleContributed (state.h:222-228)
            c = (k > 0 && contributed(b, D.cfg.knots[k - 1], bt, pt, T)) || contributed(b, D.cfg.knots[k], bt, pt, T) ||
                (k < M - 1 && contributed(b, D.cfg.knots[k + 1], bt, pt, T));
        else
            c = contributed(b, k, bt, pt, T);
        if (c)
            coeff += belief[th];
    }
    return coeff;
}

template <int NTH> __global__ void __launch_bounds__(UB) mppi_update(const MppiDev* __restrict__ insts, const MppiIn* __restrict__ in, const Tile* __restrict__ tiles)
{
    constexpr int NBP = NTH + 1;
    __shared__ float sNum0[UB], sNum1[UB], sDen[UB];
    __shared__ float sMin[UB / 32];
    __shared__ int sLast;
    pdl_wait(); // the rollout's costs and branch records are complete and visible
    pdl_trigger();
    const Tile tile = tiles[blockIdx.x];
    const MppiDev& D = insts[tile.inst];
    const MppiIn& I = in[tile.inst];
    const int K = D.cfg.K, T = D.cfg.T, M = D.cfg.M;
    const bool spl = D.cfg.useSplines != 0;
    const int b = tile.s0 / M, k = tile.s0 % M;
    const int tid = threadIdx.x;
    float belief[NTH];
#pragma unroll
    for (int i = 0; i < NTH; i++)
        belief[i] = I.belief[i];
    const int initPred = findConfident<NTH>(belief, D.cfg.minConf);
    const float* costs = D.costs + (size_t)b * K;

    // masked minimum (computeMaskedMinCostsKernel, kernels.cu:221-301)
    float mn = INFINITY;
    if (initPred == 0 || initPred == b)
        for (int s = tid; s < K; s += UB)
        {
            float coeff = sampleCoeff<NTH>(D, belief, b, k, s, spl, T, M, K);
            if (coeff > MIN_COEFF)
            {
                float c = costs[s];
                if (c < mn)
                    mn = c;
            }
        }
    mn = warp_min(mn);
    if ((tid & 31) == 0)
        sMin[tid >> 5] = mn;
    __syncthreads();
    float minC = sMin[0];
#pragma unroll
    for (int w = 1; w < UB / 32; w++)
        minC = fminf(minC, sMin[w]);

    // weighted average of the regenerated perturbation (weightedAverageKernelUnified,
    // kernels.cu:307-408); w = exp(-(c - min) / inv_temperature)
    const float lambda = I.lambda;
    const uint32_t k0 = D.cfg.k0, k1 = D.cfg.k1, step = I.step;
    float num0 = 0.0f, num1 = 0.0f, den = 0.0f;
    if (!isinf(minC))
        for (int s = tid; s < K; s += UB)
        {
            float coeff = sampleCoeff<NTH>(D, belief, b, k, s, spl, T, M, K);
            if (coeff > MIN_COEFF)
            {
                float cost = costs[s];
                float w = expf(-(cost - minC) / lambda);
                U4 r = draw(k0, k1, (uint32_t)s, (uint32_t)(b * M + k), step, S_MPPI_EPS, 0);
                float eps0 = scaled_normal(D.cfg.sigma0, r.x);
                float eps1 = scaled_normal(D.cfg.sigma1, r.y);
                num0 += w * coeff * eps0;
                num1 += w * coeff * eps1;
                den += w * coeff;
            }
        }
    // the reference's shared-memory tree: strides 128, 64, 32 across warps, then 16..1
    sNum0[tid] = num0;
    sNum1[tid] = num1;
    sDen[tid] = den;
    __syncthreads();
#pragma unroll
    for (int stride = UB / 2; stride >= 32; stride >>= 1)
    {
        if (tid < stride)
        {
            sNum0[tid] += sNum0[tid + stride];
            sNum1[tid] += sNum1[tid + stride];
            sDen[tid] += sDen[tid + stride];
        }
        __syncthreads();
    }
    if (tid < 32)
    {
        float a0 = sNum0[tid], a1 = sNum1[tid], dd = sDen[tid];
#pragma unroll
        for (int stride = 16; stride > 0; stride >>= 1)
        {
            a0 += __shfl_down_sync(0xffffffffu, a0, stride);
            a1 += __shfl_down_sync(0xffffffffu, a1, stride);
            dd += __shfl_down_sync(0xffffffffu, dd, stride);
        }
        if (tid == 0)
        {
            float* kn = D.knots + (size_t)(b * M + k) * 2;
            if (dd > 1e-30f)
            {
                __stcg(kn + 0, __ldcg(kn + 0) + a0 / dd);
                __stcg(kn + 1, __ldcg(kn + 1) + a1 / dd);
            }
            if (k == 0)
                D.nu[b] = dd;
            D.minCosts[b * M + k] = minC;
            __threadfence();
            unsigned prev = atomicAdd(D.counter, 1u);
            sLast = (prev == (unsigned)(NBP * M - 1));
        }
    }
    __syncthreads();
    if (!sLast)
        return;
    __threadfence();
    // last block of this instance: interpolateSplineKernel + clampNominalKernel
    if (spl)
    {
        for (int idx = tid; idx < NBP * T * 2; idx += UB)
        {
            int dim = idx & 1, t = (idx >> 1) % T, br = (idx >> 1) / T;
            float sum = 0.0f;
            for (int m = 0; m < M; m++)
                sum += D.B[t * M + m] * __ldcg(D.knots + (br * M + m) * 2 + dim);
            D.dense[idx] = sum;
        }
        __syncthreads();
    }
    const float maxAccel = D.env.maxAccel[0];
    for (int v = tid; v < NBP * M; v += UB)
    {
        float x0 = __ldcg(D.knots + v * 2), x1 = __ldcg(D.knots + v * 2 + 1);
        float sq = 0.0f;
        sq += x0 * x0;
        sq += x1 * x1;
        float maxSq = maxAccel * maxAccel;
        if (sq > maxSq)
        {
            float scale = maxAccel / sqrtf(sq);
            x0 *= scale;
            x1 *= scale;
        }
        __stcg(D.knots + v * 2, x0);
        __stcg(D.knots + v * 2 + 1, x1);
        if (!spl)
        {
            D.dense[v * 2] = x0;
            D.dense[v * 2 + 1] = x1;
        }
    }
    if (tid == 0)
        *D.counter = 0u;
}

// ---------------------------------------------------------------------------------------
// sample-sharded update: one controller's samples split across processes (one per GPU),
// the processes' partial results exchanged once per step by the caller's all-gather
// ---------------------------------------------------------------------------------------
// One exchange per step for a sample-sharded controller: this process's masked minimum
// per (branch plan, knot) over its own samples and its weighted sums of the regenerated
// perturbations taken with that local minimum, partial[(b, k)] = (m_r, sum w coeff eps0,
// sum w coeff eps1, sum w coeff), w = exp(-(c - m_r) / lambda). The processes all-gather
// the partials; mppi_shard_merge brings them to the global minimum m with the factor
// exp(-(m_r - m) / lambda) (the weight of a sample relative to m is its weight relative to
// m_r times that factor), so no second exchange is needed for the sums.
template <int NTH> __global__ void __launch_bounds__(UB) mppi_shard_local(const MppiDev* __restrict__ insts, const MppiIn* __restrict__ in,
                                                                          const Tile* __restrict__ tiles, float* __restrict__ partial)
{
    __shared__ float sMin[UB / 32];
    __shared__ float sNum0[UB], sNum1[UB], sDen[UB];
    const Tile tile = tiles[blockIdx.x];
    const MppiDev& D = insts[tile.inst];
    const MppiIn& I = in[tile.inst];
    const int K = D.cfg.K, T = D.cfg.T, M = D.cfg.M, sLo = D.cfg.sLo, sHi = D.cfg.sHi;
    const bool spl = D.cfg.useSplines != 0;
    const int b = tile.s0 / M, k = tile.s0 % M;
    const int tid = threadIdx.x;
    float belief[NTH];
#pragma unroll
    for (int i = 0; i < NTH; i++)
        belief[i] = I.belief[i];
    const int initPred = findConfident<NTH>(belief, D.cfg.minConf);
    const float* costs = D.costs + (size_t)b * K;
    float mn = INFINITY;
    if (initPred == 0 || initPred == b)
        for (int s = sLo + tid; s < sHi; s += UB)
        {
            float coeff = sampleCoeff<NTH>(D, belief, b, k, s, spl, T, M, K);
            if (coeff > MIN_COEFF)
            {
                float c = costs[s];
                if (c < mn)
                    mn = c;
            }
        }
    mn = warp_min(mn);
    if ((tid & 31) == 0)
        sMin[tid >> 5] = mn;
    __syncthreads();
    float minC = sMin[0];
#pragma unroll
    for (int w = 1; w < UB / 32; w++)
        minC = fminf(minC, sMin[w]);
    const float lambda = I.lambda;
    const uint32_t k0 = D.cfg.k0, k1 = D.cfg.k1, step = I.step;
    float num0 = 0.0f, num1 = 0.0f, den = 0.0f;
    if (!isinf(minC))
        for (int s = sLo + tid; s < sHi; s += UB)
        {
            float coeff = sampleCoeff<NTH>(D, belief, b, k, s, spl, T, M, K);
            if (coeff > MIN_COEFF)
            {
                float cost = costs[s];
                float w = expf(-(cost - minC) / lambda);
                U4 r = draw(k0, k1, (uint32_t)s, (uint32_t)(b * M + k), step, S_MPPI_EPS, 0);
                float eps0 = scaled_normal(D.cfg.sigma0, r.x);
                float eps1 = scaled_normal(D.cfg.sigma1, r.y);
                num0 += w * coeff * eps0;
                num1 += w * coeff * eps1;
                den += w * coeff;
            }
        }
    sNum0[tid] = num0;
    sNum1[tid] = num1;
    sDen[tid] = den;
    __syncthreads();
#pragma unroll
    for (int stride = UB / 2; stride >= 32; stride >>= 1)
    {
        if (tid < stride)
        {
            sNum0[tid] += sNum0[tid + stride];
            sNum1[tid] += sNum1[tid + stride];
            sDen[tid] += sDen[tid + stride];
        }
        __syncthreads();
    }
    if (tid < 32)
    {
        float a0 = sNum0[tid], a1 = sNum1[tid], dd = sDen[tid];
#pragma unroll
        for (int stride = 16; stride > 0; stride >>= 1)
        {
            a0 += __shfl_down_sync(0xffffffffu, a0, stride);
            a1 += __shfl_down_sync(0xffffffffu, a1, stride);
            dd += __shfl_down_sync(0xffffffffu, dd, stride);
        }
        if (tid == 0)
        {
            float* o = partial + (size_t)(b * M + k) * 4;
            o[0] = minC;
            o[1] = a0;
            o[2] = a1;
            o[3] = dd;
        }
    }
}

// The partials of all processes (gathered[r * words + ...], rank order), merged the same
// way on every process: the global minimum and the rescaled sums per (branch plan, knot)
// into mins / sums (the layout mppi_shard_apply reads), and the previous plan's failure
// histograms summed into the controller's fail[T .. 2T).
__global__ void __launch_bounds__(UB) mppi_shard_merge(const MppiDev* __restrict__ insts, const MppiIn* __restrict__ in, const float* __restrict__ gathered,
                                                       int words, int world, float* __restrict__ mins, float* __restrict__ sums)
{
    const MppiDev& D = insts[0];
    const int T = D.cfg.T, M = D.cfg.M, nbp = D.cfg.nth + 1;
    const float lambda = in[0].lambda;
    for (int v = threadIdx.x; v < nbp * M; v += blockDim.x)
    {
        float m = INFINITY;
        for (int r = 0; r < world; r++)
            m = fminf(m, gathered[(size_t)r * words + v * 4]);
        float a0 = 0.0f, a1 = 0.0f, dd = 0.0f;
        if (!isinf(m))
            for (int r = 0; r < world; r++)
            {
                const float* p = gathered + (size_t)r * words + v * 4;
                if (isinf(p[0]))
                    continue; // no sample of process r contributes
                const float f = expf(-(p[0] - m) / lambda);
                a0 += p[1] * f;
                a1 += p[2] * f;
                dd += p[3] * f;
            }
        mins[v] = m;
        sums[v * 3] = a0;
        sums[v * 3 + 1] = a1;
        sums[v * 3 + 2] = dd;
    }
    const int hOff = nbp * M * 4;
    for (int t = threadIdx.x; t < T; t += blockDim.x)
    {
        unsigned h = 0u;
        for (int r = 0; r < world; r++)
            h += __float_as_uint(gathered[(size_t)r * words + hOff + t]);
        D.fail[T + t] = h;
    }
}

// the update from the merged sums of all processes, then interpolateSplineKernel and
// clampNominalKernel (kernels.cu:411-456); one block per instance
__global__ void __launch_bounds__(UB) mppi_shard_apply(const MppiDev* __restrict__ insts, int nbp, const float* __restrict__ mins,
                                                       const float* __restrict__ sums)
{
    const MppiDev& D = insts[blockIdx.x];
    const int T = D.cfg.T, M = D.cfg.M;
    const bool spl = D.cfg.useSplines != 0;
    const int tid = threadIdx.x;
    for (int v = tid; v < nbp * M; v += UB)
    {
        const int b = v / M, k = v % M;
        const float a0 = sums[v * 3], a1 = sums[v * 3 + 1], dd = sums[v * 3 + 2];
        if (dd > 1e-30f)
        {
            D.knots[v * 2 + 0] += a0 / dd;
            D.knots[v * 2 + 1] += a1 / dd;
        }
        if (k == 0)
            D.nu[b] = dd;
        D.minCosts[v] = mins[v];
    }
    __syncthreads();
    if (spl)
    {
        for (int idx = tid; idx < nbp * T * 2; idx += UB)
        {
            int dim = idx & 1, t = (idx >> 1) % T, br = (idx >> 1) / T;
            float sum = 0.0f;
            for (int m = 0; m < M; m++)
                sum += D.B[t * M + m] * D.knots[(br * M + m) * 2 + dim];
            D.dense[idx] = sum;
        }
        __syncthreads();
    }
    const float maxAccel = D.env.maxAccel[0];
    for (int v = tid; v < nbp * M; v += UB)
    {
        float x0 = D.knots[v * 2], x1 = D.knots[v * 2 + 1];
        float sq = 0.0f;
        sq += x0 * x0;
        sq += x1 * x1;
        float maxSq = maxAccel * maxAccel;
        if (sq > maxSq)
        {
            float scale = maxAccel / sqrtf(sq);
            x0 *= scale;
            x1 *= scale;
        }
        D.knots[v * 2] = x0;
        D.knots[v * 2 + 1] = x1;
        if (!spl)
        {
            D.dense[v * 2] = x0;
            D.dense[v * 2 + 1] = x1;
        }
    }
}

// ---------------------------------------------------------------------------------------
// verification
// ---------------------------------------------------------------------------------------
// The ego tables of a plan (EgoRow; plan 0 the new one, 1 the previous one, 2 both): one
// warp per row (the trajectory with no branch, and one per branch and branching step)
// moves the ego alone through the verification horizon with the fast arithmetic of the
// verification, its lanes sharing the projection's window scan; each CTA of
// EGO_WARPS warps stages the track, the environment and the plan in shared memory. The
// rows are independent, so the kernel's time is one trajectory's: H steps of one warp.
constexpr int EGO_WARPS = 4;

template <int NTH>
__global__ void __launch_bounds__(EGO_WARPS * 32) mppi_ego_table(const MppiDev* __restrict__ insts, const MppiIn* __restrict__ in, int nInst, int plans)
{
    __shared__ float sg[GRID_FLOATS];
    __shared__ __align__(16) float sPlan[(DR_MAX_THETA + 1) * DR_MAX_T * 2];
    __shared__ EnvParams sE;
    const int inst = blockIdx.x;
    if (inst >= nInst)
        return;
    const MppiDev& D = insts[inst];
    const MppiIn& I = in[inst];
    if (!D.egoTab)
        return;
    const int H = D.cfg.H, T = D.cfg.T, rows = egoRows(NTH, H), nbp = NTH + 1;
    const int warp = threadIdx.x >> 5;
    for (int i = threadIdx.x; i < GRID_FLOATS; i += blockDim.x)
        sg[i] = D.grids[i];
    copyEnv(&sE, &D.env);
    const EnvParams& E = sE;
    const Track tr = trackIn(sg);
    float belief[NTH];
#pragma unroll
    for (int i = 0; i < NTH; i++)
        belief[i] = I.belief[i];
    const int pt0 = findConfident<NTH>(belief, D.cfg.minConf);
    const int p0 = plans == 1 ? 1 : 0, p1 = plans == 0 ? 0 : 1;
    for (int plan = p0; plan <= p1; plan++)
    {
        const float* P = plan == 0 ? D.dense : D.prevDense;
        __syncthreads(); // the previous plan's rows are done with sPlan
        for (int i = threadIdx.x; i < nbp * T * 2; i += blockDim.x)
            sPlan[i] = P[i];
        __syncthreads();
        if (!egoNoiseFree(E))
            continue; // uniform: the verification moves the ego itself
        EgoRow* tab = D.egoTab + (size_t)plan * rows * H;
        for (int r = blockIdx.y * EGO_WARPS + warp; r < rows; r += gridDim.y * EGO_WARPS)
        {
            if (r > 0 && pt0 != 0)
                break; // a confident initial belief never branches
            const int bb = r > 0 ? 1 + (r - 1) / H : 0, tb = r > 0 ? (r - 1) % H : H;
            DState<1> s;
            s.pos[0] = I.state.pos[0];
            s.pos[1] = I.state.pos[1];
            s.vel[0] = I.state.vel[0];
            s.vel[1] = I.state.vel[1];
            s.S[0] = I.state.S[0];
            s.lat[0] = I.state.lat_dist[0];
            s.laps[0] = I.state.laps[0];
            s.locate(E.trackLength);
            for (int t = 0; t < H; t++)
            {
                // the verification's plan index: branch pt0 before any branching, then the
                // branch taken, its clock restarting after the branching step
                const int b = t <= tb ? pt0 : bb, local = t <= tb ? t : t - tb - 1;
                EgoRow row;
                egoStep<true, true>(tr, E, sPlan[(b * T + local) * 2], sPlan[(b * T + local) * 2 + 1], s, row);
                if ((threadIdx.x & 31) == 0)
                    tab[(size_t)r * H + t] = row;
            }
        }
    }
}

// FAST: the fast arithmetic flavour and noise source (the default; the exact flavour
// reproduces the oracle's per-sample results and serves parity tests). EGO (with FAST):
// the ego's moves come from the instance's ego table of the plan (mppi_ego_table).
template <int NOPP, int NTH, bool PQ, bool FAST, bool EGO = false>
__global__ void __launch_bounds__(VERIFY_TILE, (verifyMinBlocks<NOPP, NTH>())) mppi_verify(const MppiDev* __restrict__ insts, const MppiIn* __restrict__ in, const Tile* __restrict__ tiles,
                                                  int nTiles, unsigned* __restrict__ queue, int* __restrict__ dbgFailTime, int* __restrict__ dbgTheta)
{
    constexpr int NA = NOPP + 1;
    constexpr int NBP = NTH + 1;
    extern __shared__ __align__(128) unsigned char smraw[];
    __shared__ int sTicket;
    pdl_wait(); // the plan to verify is complete and visible
    uint64_t* bar = (uint64_t*)smraw;
    EnvParams* sE = (EnvParams*)(smraw + 16);
    const size_t offG = align16(16 + sizeof(EnvParams));
    float* sGrid = (float*)(smraw + offG);
    float* sPlan = (float*)(smraw + offG + GRID_FLOATS * 4);
    if (threadIdx.x == 0)
        mbar_init(bar, 1);
    int staged = -1;     // (instance, plan) whose track and plan are in shared memory
    uint32_t phase = 0u; // parity of the staging barrier's next phase
    for (int iter = 0;; iter++)
    {
        const int ti = nextTile(PQ ? queue : nullptr, iter, &sTicket);
        if (ti >= nTiles)
            break;
        const Tile tile = tiles[ti];
        const MppiDev& D = insts[tile.inst];
        const MppiIn& I = in[tile.inst];
        const int T = D.cfg.T, H = D.cfg.H;
        const int plan = tile.aux;
        const uint32_t planBytes = (uint32_t)align16((size_t)NBP * T * 2 * 4);
        unsigned* hist = (unsigned*)(smraw + offG + GRID_FLOATS * 4 + planBytes);
        const int key = tile.inst * 2 + plan;
        if (key != staged)
        {
            if (threadIdx.x == 0)
            {
                mbar_expect_tx(bar, GRID_FLOATS * 4 + planBytes);
                if (!D.cfg.dbgNoStage)
                {
                    bulk_g2s(sGrid, D.grids, GRID_FLOATS * 4, bar);
                    bulk_g2s(sPlan, plan == 0 ? D.dense : D.prevDense, planBytes, bar);
                }
            }
            copyEnv(sE, &D.env);
        }
        for (int i = threadIdx.x; i < T; i += blockDim.x)
            hist[i] = 0u;
        __syncthreads();
        if (key != staged)
        {
            // on timeout the tile adds nothing to the histograms; the host reports it
            if (!__syncthreads_and(mbar_wait(bar, phase, D.cfg.waitPolls)))
            {
                if (threadIdx.x == 0)
                    atomicAdd(&D.stats[1], 1);
                return;
            }
            phase ^= 1u;
            staged = key;
        }
        const EnvParams& E = *sE;
        const Track tr = trackIn(sGrid);
        const int v = tile.s0 + threadIdx.x;
        bool active = threadIdx.x < tile.count; // idle lanes of a partial tile still take the barriers
        {
            const float minConf = D.cfg.minConf;
            DState<NA> st;
#pragma unroll
            for (int a = 0; a < NA; a++)
            {
                st.pos[2 * a] = I.state.pos[2 * a];
                st.pos[2 * a + 1] = I.state.pos[2 * a + 1];
                st.vel[2 * a] = I.state.vel[2 * a];
                st.vel[2 * a + 1] = I.state.vel[2 * a + 1];
                st.S[a] = I.state.S[a];
                st.lat[a] = I.state.lat_dist[a];
                st.laps[a] = I.state.laps[a];
            }
            st.locate(E.trackLength);
            BState<NTH> bs;
#pragma unroll
            for (int i = 0; i < NTH; i++)
                bs.belief[i] = I.belief[i];
            bs.predTheta = findConfident<NTH>(bs.belief, minConf);
            bs.branchingTime = bs.predTheta == 0 ? -1 : 0;
            const int pt0 = bs.predTheta;
            const EgoRow* egoTab = EGO ? D.egoTab + (size_t)plan * egoRows(NTH, H) * H : nullptr;
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
            int tOrigin = 0, t = 0, tEnd = H;
            bool failed = false;
            for (; t < H; t++)
            {
                // a warp leaves the loop once all its samples are done (no CTA barrier in
                // the loop: see VERIFY_MIN_BLOCKS)
                if (!__any_sync(0xffffffffu, active))
                    break;
                if (!active)
                    continue;
                rng.begin_step((uint32_t)t);
                int local = t - tOrigin;
                int b = bs.predTheta;
                float e0 = sPlan[(b * T + local) * 2], e1 = sPlan[(b * T + local) * 2 + 1];
                bool branched = false;
                StepOut o;
                if constexpr (EGO)
                {
                    const int row = (bs.predTheta == 0 || pt0 != 0) ? 0 : 1 + (bs.predTheta - 1) * H + (tOrigin - 1);
                    const EgoRow er = egoTab[(size_t)row * H + t];
                    o = envStep<NOPP, NTH, true, true, false, true, FAST, Noise, true>(t, theta, tr, E, e0, e1, st, bs, branched, minConf, rng, &er);
                }
                else
                    o = envStep<NOPP, NTH, true, true, false, true, FAST>(t, theta, tr, E, e0, e1, st, bs, branched, minConf, rng);
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
        __syncthreads(); // the next tile's staging and histogram reuse shared memory
    }
}

// perturbation of the next step in the reference layout noise[nbp][M][K][2] (test hook)
__global__ void mppi_noise(const MppiDev* __restrict__ insts, const MppiIn* __restrict__ in, float* __restrict__ out)
{
    const MppiDev& D = insts[0];
    const int K = D.cfg.K, M = D.cfg.M, nbp = D.cfg.nth + 1;
    size_t n = (size_t)nbp * M * K;
    size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    int s = (int)(i % K);
    int bk = (int)(i / K);
    U4 r = draw(D.cfg.k0, D.cfg.k1, (uint32_t)s, (uint32_t)bk, in[0].step, S_MPPI_EPS, 0);
    out[i * 2] = scaled_normal(D.cfg.sigma0, r.x);
    out[i * 2 + 1] = scaled_normal(D.cfg.sigma1, r.y);
}

// ---------------------------------------------------------------------------------------
// dispatch
// ---------------------------------------------------------------------------------------
size_t mppiRolloutSmem(int nth, int T, int M, bool spl)
{
    return rolloutLayout(nth + 1, T, M, spl).total;
}

size_t mppiVerifySmem(int nth, int T)
{
    return align16(16 + sizeof(EnvParams)) + GRID_FLOATS * 4 + ((((size_t)(nth + 1) * T * 2 * 4) + 15) & ~(size_t)15) + (size_t)T * 4;
}

template <int NOPP, int NTH, bool SPL> static cudaError_t launchRolloutS(const LaunchArgs& a, size_t smem)
{
    auto k = a.queue ? (a.lockstep ? mppi_rollout<NOPP, NTH, SPL, true, true> : mppi_rollout<NOPP, NTH, SPL, true, false>)
                     : (a.lockstep ? mppi_rollout<NOPP, NTH, SPL, false, true> : mppi_rollout<NOPP, NTH, SPL, false, false>);
    ensureSmem(k, smem);
    k<<<launchGrid(a), RB, smem, a.stream>>>(a.mppi, a.mppiIn, a.tiles, a.nTiles, a.queue);
    return cudaGetLastError();
}

template <int NOPP, int NTH> static cudaError_t launchRolloutT(const LaunchArgs& a, bool spl, size_t smem)
{
    return spl ? launchRolloutS<NOPP, NTH, true>(a, smem) : launchRolloutS<NOPP, NTH, false>(a, smem);
}

template <int NOPP, int NTH> static cudaError_t launchVerifyT(const LaunchArgs& a, size_t smem, int* ft, int* th)
{
    auto k = a.exactVerify ? (a.queue ? mppi_verify<NOPP, NTH, true, false> : mppi_verify<NOPP, NTH, false, false>)
             : a.egoTable  ? (a.queue ? mppi_verify<NOPP, NTH, true, true, true> : mppi_verify<NOPP, NTH, false, true, true>)
                           : (a.queue ? mppi_verify<NOPP, NTH, true, true> : mppi_verify<NOPP, NTH, false, true>);
    ensureSmem(k, smem);
    return launchMaybePdl(a.pdl != 0, k, dim3(launchGrid(a)), dim3(VERIFY_TILE), smem, a.stream, a.mppi, a.mppiIn, a.tiles, a.nTiles, a.queue, ft, th);
}

// CTAs of the persistent rollout / verification kernel that fit on one SM at once, for
// the given dynamic shared memory: the persistent grid is at most this times the SMs.
template <int NOPP, int NTH> static int residentT(bool verify, bool spl, size_t smem)
{
    int n = 0;
    if (verify)
    {
        ensureSmem(mppi_verify<NOPP, NTH, true, true>, smem);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, mppi_verify<NOPP, NTH, true, true>, VERIFY_TILE, smem);
    }
    else if (spl)
    {
        ensureSmem(mppi_rollout<NOPP, NTH, true, true, false>, smem);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, mppi_rollout<NOPP, NTH, true, true, false>, RB, smem);
    }
    else
    {
        ensureSmem(mppi_rollout<NOPP, NTH, false, true, false>, smem);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, mppi_rollout<NOPP, NTH, false, true, false>, RB, smem);
    }
    return n;
}

#define DR_DISPATCH(NOPP_, NTH_, CALL)                                                                                                               \
    switch (NOPP_ * 16 + NTH_)                                                                                                                       \
    {                                                                                                                                                \
    case 1 * 16 + 1: return CALL(1, 1);                                                                                                             \
    case 1 * 16 + 2: return CALL(1, 2);                                                                                                             \
    case 1 * 16 + 4: return CALL(1, 4);                                                                                                             \
    case 1 * 16 + 8: return CALL(1, 8);                                                                                                             \
    case 2 * 16 + 2: return CALL(2, 2);                                                                                                             \
    default: return cudaErrorInvalidValue;                                                                                                           \
    }

#define DR_DISPATCH_INT(NOPP_, NTH_, CALL)                                                                                                           \
    switch (NOPP_ * 16 + NTH_)                                                                                                                       \
    {                                                                                                                                                \
    case 1 * 16 + 1: return CALL(1, 1);                                                                                                             \
    case 1 * 16 + 2: return CALL(1, 2);                                                                                                             \
    case 1 * 16 + 4: return CALL(1, 4);                                                                                                             \
    case 1 * 16 + 8: return CALL(1, 8);                                                                                                             \
    case 2 * 16 + 2: return CALL(2, 2);                                                                                                             \
    default: return 0;                                                                                                                               \
    }

bool mppiSupported(int nopp, int nth)
{
    int key = nopp * 16 + nth;
    return key == 17 || key == 18 || key == 20 || key == 24 || key == 34;
}

cudaError_t launchMppiPrologue(const LaunchArgs& a, int nInst, size_t smem)
{
    ensureSmem(mppi_prologue, smem);
    mppi_prologue<<<nInst, 256, smem, a.stream>>>(a.mppi, a.mppiIn, nInst);
    return cudaGetLastError();
}

cudaError_t launchMppiRollout(const LaunchArgs& a, int nopp, int nth, bool spl, size_t smem)
{
#define CALL(P, Q) launchRolloutT<P, Q>(a, spl, smem)
    DR_DISPATCH(nopp, nth, CALL)
#undef CALL
}

cudaError_t launchMppiUpdate(const LaunchArgs& a, int nth)
{
    const bool pdl = a.pdl != 0;
    switch (nth)
    {
    case 1: return launchMaybePdl(pdl, mppi_update<1>, dim3(a.nTiles), dim3(UB), 0, a.stream, a.mppi, a.mppiIn, a.tiles);
    case 2: return launchMaybePdl(pdl, mppi_update<2>, dim3(a.nTiles), dim3(UB), 0, a.stream, a.mppi, a.mppiIn, a.tiles);
    case 4: return launchMaybePdl(pdl, mppi_update<4>, dim3(a.nTiles), dim3(UB), 0, a.stream, a.mppi, a.mppiIn, a.tiles);
    case 8: return launchMaybePdl(pdl, mppi_update<8>, dim3(a.nTiles), dim3(UB), 0, a.stream, a.mppi, a.mppiIn, a.tiles);
    default: return cudaErrorInvalidValue;
    }
}

cudaError_t launchShardLocal(const LaunchArgs& a, int nth, float* partial)
{
    switch (nth)
    {
    case 1: mppi_shard_local<1><<<a.nTiles, UB, 0, a.stream>>>(a.mppi, a.mppiIn, a.tiles, partial); break;
    case 2: mppi_shard_local<2><<<a.nTiles, UB, 0, a.stream>>>(a.mppi, a.mppiIn, a.tiles, partial); break;
    case 4: mppi_shard_local<4><<<a.nTiles, UB, 0, a.stream>>>(a.mppi, a.mppiIn, a.tiles, partial); break;
    case 8: mppi_shard_local<8><<<a.nTiles, UB, 0, a.stream>>>(a.mppi, a.mppiIn, a.tiles, partial); break;
    default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

cudaError_t launchShardMerge(cudaStream_t stream, const MppiDev* insts, const MppiIn* in, const float* gathered, int words, int world, float* mins,
                             float* sums)
{
    mppi_shard_merge<<<1, UB, 0, stream>>>(insts, in, gathered, words, world, mins, sums);
    return cudaGetLastError();
}

cudaError_t launchShardApply(cudaStream_t stream, const MppiDev* insts, int nInst, int nth, const float* mins, const float* sums)
{
    mppi_shard_apply<<<nInst, UB, 0, stream>>>(insts, nth + 1, mins, sums);
    return cudaGetLastError();
}

cudaError_t launchMppiAggregate(const LaunchArgs& a, int nth, int K)
{
    int grd = (K + 255) / 256;
    switch (nth)
    {
    case 1: mppi_aggregate<1><<<grd, 256, 0, a.stream>>>(a.mppi, a.mppiIn); break;
    case 2: mppi_aggregate<2><<<grd, 256, 0, a.stream>>>(a.mppi, a.mppiIn); break;
    case 4: mppi_aggregate<4><<<grd, 256, 0, a.stream>>>(a.mppi, a.mppiIn); break;
    case 8: mppi_aggregate<8><<<grd, 256, 0, a.stream>>>(a.mppi, a.mppiIn); break;
    default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

int mppiResident(int nopp, int nth, bool verify, bool spl, size_t smem)
{
#define CALL(P, Q) residentT<P, Q>(verify, spl, smem)
    DR_DISPATCH_INT(nopp, nth, CALL)
#undef CALL
}

cudaError_t launchMppiVerify(const LaunchArgs& a, int nopp, int nth, size_t smem, int* dbgFailTime, int* dbgTheta)
{
#define CALL(P, Q) launchVerifyT<P, Q>(a, smem, dbgFailTime, dbgTheta)
    DR_DISPATCH(nopp, nth, CALL)
#undef CALL
}

cudaError_t launchEgoTable(cudaStream_t stream, int nopp, int nth, const MppiDev* insts, const MppiIn* in, int nInst, int plan, int maxH)
{
    (void)nopp; // the ego's moves do not depend on the opponents
    // blocks per instance: enough warps for the rows of the longest horizon of the batch
    const dim3 grid(nInst, (unsigned)((egoRows(nth, maxH) + EGO_WARPS - 1) / EGO_WARPS));
    switch (nth)
    {
    case 1: mppi_ego_table<1><<<grid, EGO_WARPS * 32, 0, stream>>>(insts, in, nInst, plan); break;
    case 2: mppi_ego_table<2><<<grid, EGO_WARPS * 32, 0, stream>>>(insts, in, nInst, plan); break;
    case 4: mppi_ego_table<4><<<grid, EGO_WARPS * 32, 0, stream>>>(insts, in, nInst, plan); break;
    case 8: mppi_ego_table<8><<<grid, EGO_WARPS * 32, 0, stream>>>(insts, in, nInst, plan); break;
    default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

cudaError_t launchMppiNoise(const LaunchArgs& a, size_t n, float* out)
{
    mppi_noise<<<(unsigned)((n + 255) / 256), 256, 0, a.stream>>>(a.mppi, a.mppiIn, out);
    return cudaGetLastError();
}

int rolloutSamplesPerBlock(int nth)
{
    return RB / nth;
}

} // namespace dr
