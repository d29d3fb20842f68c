// Gradient path of the MPPI controller (strategic race): the objective
//
//   J(U, w) = sum_th b_th J_th(U, w) / sum_th b_th,
//   J_th    = sum_t DECAY^t stateCost(x_{t+1}; w) + finalCost(x_tau; w),
//
// the noise-free rollout of the optimised control sequence U (spline knots or dense
// controls, with the branch plans switched as fullRolloutKernel switches them,
// kernels.cu:87-155) under each hypothesis th compatible with the current commitment,
// averaged with the belief weights b of aggregateBranchCostsKernel (kernels.cu:175-217);
// its gradient with respect to U and to the six cost weights; and a refinement of the
// MPPI update by projected gradient steps judged by J.
//
//   grad_nominal   one CTA per (instance, start point), one warp per hypothesis.
//     forward  the warp rolls the hypothesis out once (values only), keeping the state
//              every `ckpt` steps (checkpoints) in shared memory;
//     reverse  adjoint sweep from the last step back: each segment between two
//              checkpoints is recomputed from its checkpoint, then walked backwards. At
//              step t lane j evaluates the step (and its running cost) with its input j
//              seeded — state component j, or ego control component j - NX — which
//              gives column j of the step's Jacobian; the lane's dot product with the
//              adjoint of the step's output is component j of the adjoint of its
//              input; a warp shuffle broadcasts the new adjoint. The control part is
//              scattered onto U through the spline basis row of the step.
//     refine   with `iters` > 0 the CTA repeats: U <- clamp(U - alpha maxAccel g / |g|_inf)
//              (the per-knot acceleration clamp of clampNominalKernel as the
//              projection), evaluating J at every iterate; the iterate with the lowest J
//              — the plain MPPI update unless a gradient step improved on it — is
//              written back as the new knots and dense plan.
#include <cstdio>

#include "common.cuh"
#include "grad_model.cuh"
#include "instance.cuh"
#include "launch.h"

namespace dr
{
using namespace grad;

namespace
{

constexpr unsigned FULL = 0xffffffffu;

struct GradSmem
{
    size_t env, grids, B, U, Ub, G, gU, ck, seg, fin, sJ, sF, red, total;
};

__host__ __device__ inline size_t a16g(size_t x)
{
    return (x + 15) & ~(size_t)15;
}

__host__ __device__ inline GradSmem gradLayout(int nth, int rw, int T, int M, int ckpt, bool spl)
{
    const int nbp = nth + 1, nU = nbp * M * 2, nck = (T + ckpt - 1) / ckpt;
    GradSmem L;
    size_t off = 0;
    L.env = off;
    off = a16g(off + sizeof(EnvParams));
    L.grids = off;
    off = a16g(off + GRID_FLOATS * 4);
    L.B = off;
    if (spl)
        off = a16g(off + (size_t)T * M * 4);
    L.U = off;
    off = a16g(off + (size_t)nU * 4);
    L.Ub = off;
    off = a16g(off + (size_t)nU * 4);
    L.G = off;
    off = a16g(off + (size_t)nU * 4);
    L.gU = off;
    off = a16g(off + (size_t)nth * nU * 4);
    L.ck = off;
    off = a16g(off + (size_t)nth * nck * rw * 4);
    L.seg = off;
    off = a16g(off + (size_t)nth * ckpt * rw * 4);
    L.fin = off;
    off = a16g(off + (size_t)nth * rw * 4);
    L.sJ = off;
    off = a16g(off + (size_t)nth * 4);
    L.sF = off;
    off = a16g(off + (size_t)nth * N_WEIGHTS * 4);
    L.red = off;
    off = a16g(off + 32 * 4);
    L.total = off;
    return L;
}

// Ego control of plan b at plan time `local`: the spline basis row times the knots
// (interpolateSpline) or the dense control.
template <bool SPL>
__device__ __forceinline__ void egoControl(const float* __restrict__ U, const float* __restrict__ B, int b, int local, int M, int T, float& u0,
                                           float& u1)
{
    if constexpr (SPL)
    {
        const float* Brow = B + local * M;
        float a0 = 0.0f, a1 = 0.0f;
        for (int m = 0; m < M; m++)
        {
            a0 = __fmaf_rn(Brow[m], U[(b * M + m) * 2 + 0], a0);
            a1 = __fmaf_rn(Brow[m], U[(b * M + m) * 2 + 1], a1);
        }
        u0 = a0;
        u1 = a1;
    }
    else
    {
        u0 = U[(b * T + local) * 2 + 0];
        u1 = U[(b * T + local) * 2 + 1];
    }
}

template <int NA, int NTH> __device__ __forceinline__ void initState(XState<NA, NTH>& s, const dr_sim_state& st, const float* belief0, int pt0)
{
#pragma unroll
    for (int a = 0; a < NA; a++)
    {
        s.pos[2 * a] = cst(st.pos[2 * a]);
        s.pos[2 * a + 1] = cst(st.pos[2 * a + 1]);
        s.vel[2 * a] = cst(st.vel[2 * a]);
        s.vel[2 * a + 1] = cst(st.vel[2 * a + 1]);
        s.S[a] = cst(st.S[a]);
        s.lat[a] = cst(st.lat_dist[a]);
        s.laps[a] = st.laps[a];
    }
#pragma unroll
    for (int i = 0; i < NTH; i++)
        s.belief[i] = cst(belief0[i]);
    s.predTheta = pt0;
    s.branchingTime = pt0 == 0 ? -1 : 0; // initBranchState (state.h:154-163)
}

__device__ __forceinline__ float blockMaxAbs(const float* v, int n, float* red)
{
    float m = 0.0f;
    for (int i = threadIdx.x; i < n; i += blockDim.x)
        m = fmaxf(m, fabsf(v[i]));
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
        m = fmaxf(m, __shfl_xor_sync(FULL, m, o));
    if ((threadIdx.x & 31) == 0)
        red[threadIdx.x >> 5] = m;
    __syncthreads();
    float r = 0.0f;
    for (int w = 0; w < (int)(blockDim.x >> 5); w++)
        r = fmaxf(r, red[w]);
    __syncthreads();
    return r;
}

} // namespace

template <int NOPP, int NTH, bool SPL> __global__ void __launch_bounds__(32 * NTH) grad_nominal(const GradJob* __restrict__ jobs)
{
    constexpr int NA = NOPP + 1, NBP = NTH + 1;
    constexpr int NX = XState<NA, NTH>::NX, RW = recWords<NA, NTH>();
    static_assert(NX + 2 <= 32, "one lane per step input");
    extern __shared__ __align__(16) unsigned char smraw[];
    const GradJob job = jobs[blockIdx.x];
    const MppiDev& D = *job.D;
    const MppiIn& I = *job.in;
    const int T = D.cfg.T, M = D.cfg.M, C = job.ckpt;
    const int nU = NBP * M * 2;
    const GradSmem L = gradLayout(NTH, RW, T, M, C, SPL);
    EnvParams* sE = (EnvParams*)(smraw + L.env);
    float* sGrid = (float*)(smraw + L.grids);
    float* sB = (float*)(smraw + L.B);
    float* sU = (float*)(smraw + L.U);
    float* sUb = (float*)(smraw + L.Ub);
    float* sG = (float*)(smraw + L.G);
    float* sGU = (float*)(smraw + L.gU);
    float* sCk = (float*)(smraw + L.ck);
    float* sSeg = (float*)(smraw + L.seg);
    float* sFin = (float*)(smraw + L.fin);
    float* sJ = (float*)(smraw + L.sJ);
    float* sF = (float*)(smraw + L.sF);
    float* red = (float*)(smraw + L.red);

    for (int i = threadIdx.x; i < ENV_HOST_WORDS; i += blockDim.x)
        ((float*)sE)[i] = ((const float*)&D.env)[i];
    envDeviceTerms(*sE, D.env, threadIdx.x, blockDim.x);
    for (int i = threadIdx.x; i < GRID_FLOATS; i += blockDim.x)
        sGrid[i] = D.grids[i];
    if constexpr (SPL)
        for (int i = threadIdx.x; i < T * M; i += blockDim.x)
            sB[i] = D.B[i];
    const float* U0 = job.U ? job.U : D.knots;
    for (int i = threadIdx.x; i < nU; i += blockDim.x)
    {
        sU[i] = U0[i];
        sUb[i] = U0[i];
    }
    MppiCostW w = D.cfg.w;
    if (job.w6)
    {
        w.boundaryCost = job.w6[W_BOUNDARY];
        w.outsideCost = job.w6[W_OUTSIDE];
        w.winCost = job.w6[W_WIN];
        w.oppWinCost = job.w6[W_OPP_WIN];
        w.finalAdvWeight = job.w6[W_FINAL_ADV];
        w.finalOppAdvWeight = job.w6[W_FINAL_OPP_ADV];
    }
    __syncthreads();
    const EnvParams& E = *sE;
    const Track tr = trackIn(sGrid);
    const int th = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const float minConf = D.cfg.minConf;
    float belief0[NTH];
#pragma unroll
    for (int i = 0; i < NTH; i++)
        belief0[i] = I.belief[i];
    const int pt0 = findConfident<NTH>(belief0, minConf);
    const bool compatible = (pt0 == 0 || pt0 == th + 1);
    float* ck = sCk + (size_t)th * ((T + C - 1) / C) * RW;
    float* seg = sSeg + (size_t)th * C * RW;
    float* fin = sFin + (size_t)th * RW;
    float* gUth = sGU + (size_t)th * nU;
    const float maxAccel = E.maxAccel[0];

    float Jbest = INFINITY;
    int best = 0;
    int done = 0;
    for (int it = 0; it <= job.iters; it++)
    {
        const bool wantGrad = it < job.iters || (job.gU != nullptr || job.gW != nullptr);
        // ---- forward: values only, checkpoints every C steps ----
        float Jth = INFINITY;
        float feat[N_WEIGHTS];
#pragma unroll
        for (int i = 0; i < N_WEIGHTS; i++)
            feat[i] = 0.0f;
        int tau = 0;
        if (compatible)
        {
            XState<NA, NTH> s;
            initState<NA, NTH>(s, I.state, belief0, pt0);
            float cost = 0.0f, decay = 1.0f;
            int tOrigin = 0;
            bool stop = false;
            int t = 0;
            for (; t < T && !stop; t++)
            {
                if (t % C == 0 && lane == 0)
                    storeRec<NA, NTH>(ck + (t / C) * RW, s, tOrigin, decay);
                float u0, u1;
                egoControl<SPL>(sU, sB, s.predTheta, t - tOrigin, M, T, u0, u1);
                bool br;
                const GOut o = gstep<NOPP, NTH>(t, th, tr, E, cst(u0), cst(u1), s, minConf, br);
                if (br)
                    tOrigin = t + 1;
                stop = o.term != TERM_NONE;
                float fe[N_WEIGHTS] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
                const Dv c = gcost(o, E, w, fe);
                cost = __fadd_rn(cost, __fmul_rn(c.v, decay));
#pragma unroll
                for (int i = 0; i < 4; i++)
                    feat[i] += fe[i] * decay;
                decay = __fmul_rn(decay, DECAY);
            }
            tau = t;
            if (lane == 0)
                storeRec<NA, NTH>(fin, s, tOrigin, decay);
            float fe[N_WEIGHTS] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
            const Dv f = gfinal<NA, NTH>(s, E, w, fe);
            cost = __fadd_rn(cost, f.v);
            feat[W_FINAL_ADV] = fe[W_FINAL_ADV];
            feat[W_FINAL_OPP_ADV] = fe[W_FINAL_OPP_ADV];
            Jth = cost;
        }
        for (int i = lane; i < nU; i += 32)
            gUth[i] = 0.0f;
        __syncwarp();
        // ---- reverse: adjoint sweep over the segments, last first ----
        if (wantGrad && compatible && isfinite(Jth))
        {
            float mu[NX];
            {
                XState<NA, NTH> s;
                int tO;
                float dec;
                loadRec<NA, NTH>(fin, s, tO, dec);
                Dv e0 = cst(0.0f), e1 = cst(0.0f);
                seed<NA, NTH>(s, e0, e1, lane);
                float fe[N_WEIGHTS];
                const float r = gfinal<NA, NTH>(s, E, w, fe).d;
#pragma unroll
                for (int i = 0; i < NX; i++)
                    mu[i] = __shfl_sync(FULL, r, i);
            }
            for (int k = (tau - 1) / C; k >= 0; k--)
            {
                const int t0 = k * C, t1 = min(t0 + C, tau);
                {
                    XState<NA, NTH> s;
                    int tO;
                    float dec;
                    loadRec<NA, NTH>(ck + k * RW, s, tO, dec);
                    for (int t = t0; t < t1; t++)
                    {
                        if (lane == 0)
                            storeRec<NA, NTH>(seg + (t - t0) * RW, s, tO, dec);
                        if (t + 1 == t1)
                            break;
                        float u0, u1;
                        egoControl<SPL>(sU, sB, s.predTheta, t - tO, M, T, u0, u1);
                        bool br;
                        gstep<NOPP, NTH>(t, th, tr, E, cst(u0), cst(u1), s, minConf, br);
                        if (br)
                            tO = t + 1;
                        dec = __fmul_rn(dec, DECAY);
                    }
                }
                __syncwarp();
                for (int t = t1 - 1; t >= t0; t--)
                {
                    XState<NA, NTH> s;
                    int tO;
                    float dec;
                    loadRec<NA, NTH>(seg + (t - t0) * RW, s, tO, dec);
                    const int b = s.predTheta, local = t - tO;
                    float u0, u1;
                    egoControl<SPL>(sU, sB, b, local, M, T, u0, u1);
                    Dv e0 = cst(u0), e1 = cst(u1);
                    seed<NA, NTH>(s, e0, e1, lane);
                    bool br;
                    const GOut o = gstep<NOPP, NTH>(t, th, tr, E, e0, e1, s, minConf, br);
                    float fe[N_WEIGHTS];
                    const Dv c = gcost(o, E, w, fe);
                    const float r = dec * c.d + dotTangent<NA, NTH>(s, mu);
#pragma unroll
                    for (int i = 0; i < NX; i++)
                        mu[i] = __shfl_sync(FULL, r, i);
                    const float g0 = __shfl_sync(FULL, r, NX), g1 = __shfl_sync(FULL, r, NX + 1);
                    if constexpr (SPL)
                    {
                        for (int m = lane; m < M; m += 32)
                        {
                            const float bm = sB[local * M + m];
                            gUth[(b * M + m) * 2 + 0] += bm * g0;
                            gUth[(b * M + m) * 2 + 1] += bm * g1;
                        }
                    }
                    else if (lane == 0)
                    {
                        gUth[(b * T + local) * 2 + 0] += g0;
                        gUth[(b * T + local) * 2 + 1] += g1;
                    }
                }
                __syncwarp();
            }
        }
        if (lane == 0)
        {
            sJ[th] = (compatible && isfinite(Jth)) ? Jth : INFINITY;
#pragma unroll
            for (int i = 0; i < N_WEIGHTS; i++)
                sF[th * N_WEIGHTS + i] = feat[i];
        }
        __syncthreads();
        // ---- belief-weighted objective over the finite hypotheses ----
        float num = 0.0f, den = 0.0f;
#pragma unroll
        for (int m = 0; m < NTH; m++)
        {
            const float cv = sJ[m];
            if (!isfinite(cv))
                continue;
            num += belief0[m] * cv;
            den += belief0[m];
        }
        const float J = den > 1e-30f ? num / den : INFINITY;
        if (threadIdx.x == 0 && job.J)
            job.J[it] = J;
        if (it == 0 && job.gW && threadIdx.x < N_WEIGHTS)
        {
            float g = 0.0f;
            for (int m = 0; m < NTH; m++)
                if (isfinite(sJ[m]))
                    g += belief0[m] * sF[m * N_WEIGHTS + threadIdx.x];
            job.gW[threadIdx.x] = den > 1e-30f ? g / den : 0.0f;
        }
        done = it;
        if (J < Jbest)
        {
            Jbest = J;
            best = it;
            if (it > 0)
                for (int i = threadIdx.x; i < nU; i += blockDim.x)
                    sUb[i] = sU[i];
        }
        if (!wantGrad)
            break;
        for (int i = threadIdx.x; i < nU; i += blockDim.x)
        {
            float g = 0.0f;
            for (int m = 0; m < NTH; m++)
                if (isfinite(sJ[m]))
                    g += belief0[m] * sGU[(size_t)m * nU + i];
            g = den > 1e-30f ? g / den : 0.0f;
            sG[i] = g;
            if (it == 0 && job.gU)
                job.gU[i] = g;
        }
        if (it == job.iters)
            break;
        __syncthreads();
        const float gmax = blockMaxAbs(sG, nU, red);
        if (!(gmax > 0.0f) || !isfinite(gmax) || !isfinite(J))
            break;
        // projected step: every control moves by at most alpha * maxAccel, then the
        // per-knot acceleration clamp (clampNominalKernel, kernels.cu:434-456)
        const float stepScale = job.alpha * maxAccel / gmax;
        for (int v = threadIdx.x; v < NBP * M; v += blockDim.x)
        {
            float x0 = sU[v * 2] - stepScale * sG[v * 2];
            float x1 = sU[v * 2 + 1] - stepScale * sG[v * 2 + 1];
            const float sq = x0 * x0 + x1 * x1;
            if (sq > maxAccel * maxAccel)
            {
                const float sc = maxAccel / sqrtf(sq);
                x0 *= sc;
                x1 *= sc;
            }
            sU[v * 2] = x0;
            sU[v * 2 + 1] = x1;
        }
        __syncthreads();
    }
    if (job.stats && threadIdx.x == 0)
    {
        job.stats[0] = (float)best;
        job.stats[1] = (float)done;
    }
    if (!job.write || best == 0)
        return;
    __syncthreads();
    for (int i = threadIdx.x; i < nU; i += blockDim.x)
        D.knots[i] = sUb[i];
    if constexpr (SPL)
    {
        for (int idx = threadIdx.x; idx < NBP * T * 2; idx += blockDim.x)
        {
            const int dim = idx & 1, t = (idx >> 1) % T, br = (idx >> 1) / T;
            float sum = 0.0f;
            for (int m = 0; m < M; m++)
                sum += sB[t * M + m] * sUb[(br * M + m) * 2 + dim];
            D.dense[idx] = sum;
        }
    }
    else
    {
        for (int i = threadIdx.x; i < nU; i += blockDim.x)
            D.dense[i] = sUb[i];
    }
}

// ---------------------------------------------------------------------------------------
// dispatch
// ---------------------------------------------------------------------------------------
static int recWordsRt(int nopp, int nth)
{
    return 6 * (nopp + 1) + nth + (nopp + 1) + 4;
}

size_t gradSmem(int nopp, int nth, int T, int M, int ckpt, bool spl)
{
    return gradLayout(nth, recWordsRt(nopp, nth), T, M, ckpt, spl).total;
}

int gradDefaultStride(int T)
{
    int c = 1;
    while (c * c < T)
        c++;
    return c;
}

template <int NOPP, int NTH> static cudaError_t launchGradT(cudaStream_t stream, const GradJob* jobs, int nJobs, bool spl, size_t smem)
{
    static_assert(recWords<NOPP + 1, NTH>() == 6 * (NOPP + 1) + NTH + (NOPP + 1) + 4, "record size");
    if (spl)
    {
        auto k = grad_nominal<NOPP, NTH, true>;
        ensureSmem(k, smem);
        k<<<nJobs, 32 * NTH, smem, stream>>>(jobs);
    }
    else
    {
        auto k = grad_nominal<NOPP, NTH, false>;
        ensureSmem(k, smem);
        k<<<nJobs, 32 * NTH, smem, stream>>>(jobs);
    }
    return cudaGetLastError();
}

cudaError_t launchGradNominal(cudaStream_t stream, const GradJob* jobs, int nJobs, int nopp, int nth, bool spl, size_t smem)
{
    if (nJobs <= 0)
        return cudaSuccess;
    switch (nopp * 16 + nth)
    {
    case 1 * 16 + 1: return launchGradT<1, 1>(stream, jobs, nJobs, spl, smem);
    case 1 * 16 + 2: return launchGradT<1, 2>(stream, jobs, nJobs, spl, smem);
    case 1 * 16 + 4: return launchGradT<1, 4>(stream, jobs, nJobs, spl, smem);
    case 1 * 16 + 8: return launchGradT<1, 8>(stream, jobs, nJobs, spl, smem);
    case 2 * 16 + 2: return launchGradT<2, 2>(stream, jobs, nJobs, spl, smem);
    default: return cudaErrorInvalidValue;
    }
}

} // namespace dr
