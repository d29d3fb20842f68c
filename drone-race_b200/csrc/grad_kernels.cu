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
//   grad_nominal   one thread-block cluster per (instance, start point), one CTA of the
//                  cluster per hypothesis, GW warps per CTA.
//     forward  warp 0 rolls the hypothesis out (values only) and keeps the state every
//              `ckpt` steps (every step when ckpt == 1) in shared memory;
//     reverse  adjoint sweep, last segment first. A segment between two checkpoints is
//              recomputed from its checkpoint; its steps are then taken GW at a time: warp
//              p evaluates step t0 + p with lane j's input seeded — state component j, or
//              ego control component j - NX — which gives column j of the step's Jacobian
//              and of its running cost's gradient, all GW steps at once; warp 0 then runs
//              the adjoint recurrence over them (lane j: component j of the adjoint of the
//              step's input, broadcast by warp shuffles) and scatters the control part onto
//              U through the spline basis row of each step.
//     combine  the CTAs of the cluster read each other's objective, features and gradient
//              through distributed shared memory, so every CTA holds the belief-weighted
//              totals;
//     refine   with `iters` > 0 every CTA then takes the same projected step
//              U <- clamp(U - alpha maxAccel g / |g|_inf) (the per-knot acceleration clamp
//              of clampNominalKernel as the projection) and the cluster evaluates J at each
//              iterate; the iterate with the lowest J — the plain MPPI update unless a
//              gradient step improved on it — is written back as the new knots and dense
//              plan by the cluster's first CTA.
#include <cooperative_groups.h>
#include <cstdio>

#include "common.cuh"
#include "grad_model.cuh"
#include "instance.cuh"
#include "launch.h"

namespace cg = cooperative_groups;

namespace dr
{
using namespace grad;

namespace
{

constexpr unsigned FULL = 0xffffffffu;
constexpr int GW = 8; // warps per hypothesis CTA (steps whose Jacobians are evaluated at once)

struct GradSmem
{
    size_t env, grids, B, U, Ub, G, gU, ck, seg, fin, jc, scal, red, total;
};

__host__ __device__ inline size_t a16g(size_t x)
{
    return (x + 15) & ~(size_t)15;
}

// Words of a Jacobian column: NX state tangents and the running cost's tangent.
__host__ __device__ inline int jcWords(int nx)
{
    return nx + 1;
}

__host__ __device__ inline GradSmem gradLayout(int nth, int nx, int rw, int T, int M, int ckpt, bool spl)
{
    const int nbp = nth + 1, nU = nbp * M * 2;
    const int nck = ckpt == 1 ? T : (T + ckpt - 1) / ckpt;
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
    off = a16g(off + (size_t)nU * 4);
    L.ck = off;
    off = a16g(off + (size_t)nck * rw * 4);
    L.seg = off;
    if (ckpt > 1)
        off = a16g(off + (size_t)ckpt * rw * 4);
    L.fin = off;
    off = a16g(off + (size_t)rw * 4);
    L.jc = off;
    off = a16g(off + (size_t)GW * (nx + 2) * jcWords(nx) * 4);
    L.scal = off; // J, then the N_WEIGHTS features, then the step count
    off = a16g(off + 16 * 4);
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

// Stores the tangent of the step's output state (NX) and of its running cost into a
// Jacobian column.
template <int NA, int NTH> __device__ __forceinline__ void storeColumn(float* col, const XState<NA, NTH>& s, float costTangent)
{
    int i = 0;
#pragma unroll
    for (int k = 0; k < 2 * NA; k++)
        col[i++] = s.pos[k].d;
#pragma unroll
    for (int k = 0; k < 2 * NA; k++)
        col[i++] = s.vel[k].d;
#pragma unroll
    for (int k = 0; k < NA; k++)
        col[i++] = s.S[k].d;
#pragma unroll
    for (int k = 0; k < NA; k++)
        col[i++] = s.lat[k].d;
#pragma unroll
    for (int k = 0; k < NTH; k++)
        col[i++] = s.belief[k].d;
    col[i] = costTangent;
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

template <int NOPP, int NTH, bool SPL> __global__ void __launch_bounds__(GW * 32, 1) grad_nominal(const GradJob* __restrict__ jobs)
{
    constexpr int NA = NOPP + 1, NBP = NTH + 1;
    constexpr int NX = XState<NA, NTH>::NX, RW = recWords<NA, NTH>(), JW = NX + 1;
    static_assert(NX + 2 <= 32, "one lane per step input");
    extern __shared__ __align__(16) unsigned char smraw[];
    cg::cluster_group cluster = cg::this_cluster();
    const int th = (int)cluster.block_rank(); // this CTA's hypothesis
    const GradJob job = jobs[blockIdx.x / NTH];
    const MppiDev& D = *job.D;
    const MppiIn& I = *job.in;
    const int T = D.cfg.T, M = D.cfg.M, C = job.ckpt;
    const int nU = NBP * M * 2;
    const GradSmem L = gradLayout(NTH, NX, RW, T, M, C, SPL);
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
    float* sJc = (float*)(smraw + L.jc);
    float* sScal = (float*)(smraw + L.scal);
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
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const float minConf = D.cfg.minConf;
    float belief0[NTH];
#pragma unroll
    for (int i = 0; i < NTH; i++)
        belief0[i] = I.belief[i];
    const int pt0 = findConfident<NTH>(belief0, minConf);
    const bool compatible = (pt0 == 0 || pt0 == th + 1);
    const float maxAccel = E.maxAccel[0];

    float Jbest = INFINITY;
    int best = 0, done = 0;
    for (int it = 0; it <= job.iters; it++)
    {
        const bool wantGrad = it < job.iters || (job.gU != nullptr || job.gW != nullptr);
        // ---- forward: values only, warp 0 ----
        if (warp == 0)
        {
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
                    if (lane == 0 && (C == 1 || t % C == 0))
                        storeRec<NA, NTH>(sCk + (size_t)(C == 1 ? t : t / C) * RW, s, tOrigin, decay);
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
                    storeRec<NA, NTH>(sFin, s, tOrigin, decay);
                float fe[N_WEIGHTS] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
                const Dv f = gfinal<NA, NTH>(s, E, w, fe);
                cost = __fadd_rn(cost, f.v);
                feat[W_FINAL_ADV] = fe[W_FINAL_ADV];
                feat[W_FINAL_OPP_ADV] = fe[W_FINAL_OPP_ADV];
                Jth = cost;
            }
            if (lane == 0)
            {
                sScal[0] = (compatible && isfinite(Jth)) ? Jth : INFINITY;
#pragma unroll
                for (int i = 0; i < N_WEIGHTS; i++)
                    sScal[1 + i] = feat[i];
                sScal[1 + N_WEIGHTS] = __int_as_float(tau);
            }
        }
        for (int i = threadIdx.x; i < nU; i += blockDim.x)
            sGU[i] = 0.0f;
        __syncthreads();
        // ---- reverse: adjoint sweep, Jacobians of GW steps at a time ----
        if (wantGrad && isfinite(sScal[0]))
        {
            const int tau = __float_as_int(sScal[1 + N_WEIGHTS]);
            float mu[NX]; // adjoint of the current step's output (warp 0; equal in all its lanes)
            if (warp == 0)
            {
                XState<NA, NTH> s;
                int tO;
                float dec;
                loadRec<NA, NTH>(sFin, s, tO, dec);
                Dv e0 = cst(0.0f), e1 = cst(0.0f);
                seed<NA, NTH>(s, e0, e1, lane);
                float fe[N_WEIGHTS];
                const float r = gfinal<NA, NTH>(s, E, w, fe).d;
#pragma unroll
                for (int i = 0; i < NX; i++)
                    mu[i] = __shfl_sync(FULL, r, i);
            }
            // segments between checkpoints (one segment holding every step when C == 1)
            const int segLen = C == 1 ? tau : C;
            for (int k = (tau - 1) / segLen; k >= 0; k--)
            {
                const int t0 = k * segLen, t1 = min(t0 + segLen, tau);
                const float* recs = C == 1 ? sCk : sSeg; // record of step t at recs + (t - base) * RW
                const int base = C == 1 ? 0 : t0;
                if (C > 1)
                {
                    if (warp == 0)
                    {
                        XState<NA, NTH> s;
                        int tO;
                        float dec;
                        loadRec<NA, NTH>(sCk + (size_t)k * RW, s, tO, dec);
                        for (int t = t0; t < t1; t++)
                        {
                            if (lane == 0)
                                storeRec<NA, NTH>(sSeg + (size_t)(t - t0) * RW, s, tO, dec);
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
                    __syncthreads();
                }
                // chunks of GW steps, last chunk first
                for (int cEnd = t1; cEnd > t0; cEnd -= GW)
                {
                    const int cBeg = max(t0, cEnd - GW);
                    const int t = cBeg + warp;
                    if (t < cEnd)
                    {
                        XState<NA, NTH> s;
                        int tO;
                        float dec;
                        loadRec<NA, NTH>(recs + (size_t)(t - base) * RW, s, tO, dec);
                        float u0, u1;
                        egoControl<SPL>(sU, sB, s.predTheta, t - tO, M, T, u0, u1);
                        Dv e0 = cst(u0), e1 = cst(u1);
                        seed<NA, NTH>(s, e0, e1, lane);
                        bool br;
                        const GOut o = gstep<NOPP, NTH>(t, th, tr, E, e0, e1, s, minConf, br);
                        float fe[N_WEIGHTS];
                        const Dv c = gcost(o, E, w, fe);
                        if (lane < NX + 2)
                            storeColumn<NA, NTH>(sJc + ((size_t)warp * (NX + 2) + lane) * JW, s, c.d);
                    }
                    __syncthreads();
                    if (warp == 0)
                    {
                        for (int tt = cEnd - 1; tt >= cBeg; tt--)
                        {
                            const float* r = recs + (size_t)(tt - base) * RW;
                            // record layout (storeRec): NX values, laps[NA], predTheta, branchingTime, tOrigin, decay
                            const int b = __float_as_int(r[NX + NA]), tO = __float_as_int(r[NX + NA + 2]);
                            const float dec = r[NX + NA + 3];
                            const int local = tt - tO;
                            float acc = 0.0f;
                            if (lane < NX + 2)
                            {
                                const float* col = sJc + ((size_t)(tt - cBeg) * (NX + 2) + lane) * JW;
                                acc = dec * col[NX];
#pragma unroll
                                for (int i = 0; i < NX; i++)
                                    acc += mu[i] * col[i];
                            }
#pragma unroll
                            for (int i = 0; i < NX; i++)
                                mu[i] = __shfl_sync(FULL, acc, i);
                            const float g0 = __shfl_sync(FULL, acc, NX), g1 = __shfl_sync(FULL, acc, NX + 1);
                            if constexpr (SPL)
                            {
                                for (int m = lane; m < M; m += 32)
                                {
                                    const float bm = sB[local * M + m];
                                    sGU[(b * M + m) * 2 + 0] += bm * g0;
                                    sGU[(b * M + m) * 2 + 1] += bm * g1;
                                }
                            }
                            else if (lane == 0)
                            {
                                sGU[(b * T + local) * 2 + 0] += g0;
                                sGU[(b * T + local) * 2 + 1] += g1;
                            }
                        }
                    }
                    __syncthreads();
                }
            }
        }
        // ---- combine the hypotheses of the cluster (distributed shared memory) ----
        cluster.sync();
        float num = 0.0f, den = 0.0f;
        float Jr[NTH];
#pragma unroll
        for (int m = 0; m < NTH; m++)
        {
            Jr[m] = cluster.map_shared_rank(sScal, m)[0];
            if (!isfinite(Jr[m]))
                continue;
            num += belief0[m] * Jr[m];
            den += belief0[m];
        }
        const float J = den > 1e-30f ? num / den : INFINITY;
        if (th == 0 && threadIdx.x == 0 && job.J)
            job.J[it] = J;
        if (th == 0 && it == 0 && job.gW && threadIdx.x < N_WEIGHTS)
        {
            float g = 0.0f;
            for (int m = 0; m < NTH; m++)
                if (isfinite(Jr[m]))
                    g += belief0[m] * cluster.map_shared_rank(sScal, m)[1 + threadIdx.x];
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
        if (wantGrad)
            for (int i = threadIdx.x; i < nU; i += blockDim.x)
            {
                float g = 0.0f;
                for (int m = 0; m < NTH; m++)
                    if (isfinite(Jr[m]))
                        g += belief0[m] * cluster.map_shared_rank(sGU, m)[i];
                g = den > 1e-30f ? g / den : 0.0f;
                sG[i] = g;
                if (th == 0 && it == 0 && job.gU)
                    job.gU[i] = g;
            }
        // no CTA may overwrite its scalars or gradient before every CTA has read them
        cluster.sync();
        if (!wantGrad || it == job.iters)
            break;
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
    if (th != 0)
        return;
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
static int nxRt(int nopp, int nth)
{
    return 6 * (nopp + 1) + nth;
}

static int recWordsRt(int nopp, int nth)
{
    return nxRt(nopp, nth) + (nopp + 1) + 4;
}

size_t gradSmem(int nopp, int nth, int T, int M, int ckpt, bool spl)
{
    return gradLayout(nth, nxRt(nopp, nth), recWordsRt(nopp, nth), T, M, ckpt, spl).total;
}

int gradDefaultStride(int nopp, int nth, int T, int M, bool spl)
{
    // every step when the states fit beside the rest (no recomputation), else ceil(sqrt(T))
    if (gradSmem(nopp, nth, T, M, 1, spl) <= 160 * 1024)
        return 1;
    int c = 1;
    while (c * c < T)
        c++;
    return c;
}

template <int NOPP, int NTH, bool SPL> static cudaError_t launchGradT(cudaStream_t stream, const GradJob* jobs, int nJobs, size_t smem)
{
    static_assert(recWords<NOPP + 1, NTH>() == 6 * (NOPP + 1) + NTH + (NOPP + 1) + 4, "record size");
    auto k = grad_nominal<NOPP, NTH, SPL>;
    ensureSmem(k, smem);
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)(nJobs * NTH));
    cfg.blockDim = dim3(GW * 32);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = NTH;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, k, jobs);
}

cudaError_t launchGradNominal(cudaStream_t stream, const GradJob* jobs, int nJobs, int nopp, int nth, bool spl, size_t smem)
{
    if (nJobs <= 0)
        return cudaSuccess;
#define DR_GRAD_CASE(P, Q) \
    return spl ? launchGradT<P, Q, true>(stream, jobs, nJobs, smem) : launchGradT<P, Q, false>(stream, jobs, nJobs, smem)
    switch (nopp * 16 + nth)
    {
    case 1 * 16 + 1: DR_GRAD_CASE(1, 1);
    case 1 * 16 + 2: DR_GRAD_CASE(1, 2);
    case 1 * 16 + 4: DR_GRAD_CASE(1, 4);
    case 1 * 16 + 8: DR_GRAD_CASE(1, 8);
    case 2 * 16 + 2: DR_GRAD_CASE(2, 2);
    default: return cudaErrorInvalidValue;
    }
#undef DR_GRAD_CASE
}

} // namespace dr
