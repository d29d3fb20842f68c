// Device tail of the MPPI control step and the true-dynamics step of a batch, so that a
// batch of controllers can run closed loop without the host.
//
//   mppi_finish       the host part of MPPIController::getControl (mppi_controller.cu:
//                     363-456) for every controller of a batch: Clopper-Pearson
//                     certification of the new plan against the previous one from the two
//                     failure histograms (computeCertifiedLoss, mppi_controller.cu:468-501;
//                     the beta quantiles of state.h:134-151, one thread per horizon step,
//                     read from a table the host fills once per controller for counts below
//                     CP_TAB and evaluated in double precision above), the plan choice, the
//                     partial and total
//                     epsilon (computeEpsilon, :503-514), the branch whose first action is
//                     sent, the temperature adaptation, and the warm-start shift of the next
//                     step (written into the batch's device input records, which carry the
//                     controller state from step to step).
//   batch_env_step    engine dynStep (engine.cpp:286-312) for every controller's race: the
//                     environment step of each controller's state under its true hypothesis
//                     with the action the controller sent, belief update included.
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <tuple>

#include "common.cuh"
#include "cp.hpp"
#include "instance.cuh"
#include "launch.h"

namespace dr
{

namespace
{
constexpr int FB = 320; // threads 0..T-1: one horizon step each; 288, 289: the epsilon candidates
static_assert(FB >= DR_MAX_T + 34, "finish block");
} // namespace

__global__ void __launch_bounds__(FB) mppi_finish(const MppiDev* __restrict__ insts, MppiIn* __restrict__ in, float* __restrict__ actions,
                                                  dr_mppi_info* __restrict__ infos, int nInst)
{
    const int inst = blockIdx.x;
    if (inst >= nInst)
        return;
    const MppiDev& D = insts[inst];
    MppiIn& I = in[inst];
    const int T = D.cfg.T, M = D.cfg.M, nth = D.cfg.nth, tid = threadIdx.x;
    const uint32_t V = (uint32_t)D.cfg.V;
    const bool verify = D.cfg.verify != 0;
    const double beta = (double)D.cfg.beta;
    __shared__ uint32_t cN[DR_MAX_T], cO[DR_MAX_T];
    __shared__ double sMax[FB / 32];
    __shared__ double sEps[2];
    // cumulative failure counts of the new and the previous plan (inclusive scan over t)
    if (tid < DR_MAX_T)
    {
        cN[tid] = tid < T ? D.fail[tid] : 0u;
        cO[tid] = tid < T ? D.fail[T + tid] : 0u;
    }
    __syncthreads();
    for (int off = 1; off < DR_MAX_T; off <<= 1)
    {
        uint32_t a = 0, b = 0;
        if (tid < DR_MAX_T && tid >= off)
        {
            a = cN[tid - off];
            b = cO[tid - off];
        }
        __syncthreads();
        if (tid < DR_MAX_T && tid >= off)
        {
            cN[tid] += a;
            cO[tid] += b;
        }
        __syncthreads();
    }
    // certified loss: max_t upper(new_t) - lower(old_t), starting from -1; counts below
    // CP_TAB read the host's table (the same function, evaluated once per controller),
    // larger ones the device table shared by the controllers of the same (V, beta)
    const double* tab = D.cpTab;
    const uint32_t V1 = V > 0 ? V : 1u;
    auto bound = [&](int which, uint32_t k, uint32_t n, double alpha, bool upper) -> double {
        if (k < (uint32_t)CP_TAB)
            return tab[which * CP_TAB + k];
        if (D.cpFull && k <= V1)
            return D.cpFull[(size_t)which * (V1 + 1) + k];
        return upper ? cpdetail::cpUpper(k, n, alpha) : cpdetail::cpLower(k, n, alpha);
    };
    double d = -1.0;
    if (verify && tid < T)
    {
        const uint32_t kn = cN[tid], ko = cO[tid];
        const double up = bound(0, kn, V, beta / 2.0, true);
        const double lo = bound(1, ko, V, beta / 2.0, false);
        d = fmax(d, up - lo);
    }
    // the two epsilon candidates (new plan kept or previous plan kept)
    if (tid == DR_MAX_T + 32 || tid == DR_MAX_T + 33)
    {
        const uint32_t tot = tid == DR_MAX_T + 32 ? cN[T - 1] : cO[T - 1];
        sEps[tid - DR_MAX_T - 32] = bound(2, tot, V1, beta, true);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
        d = fmax(d, __shfl_xor_sync(0xffffffffu, d, o));
    if ((tid & 31) == 0)
        sMax[tid >> 5] = d;
    __syncthreads();
    if (tid != 0)
        return;
    double cert = -1.0;
    for (int w = 0; w < FB / 32; w++)
        cert = fmax(cert, sMax[w]);
    bool useNew = true;
    if (verify)
        useNew = cert < (double)D.cfg.maxVerifEps;
    else
        cert = -1.0;
    const uint32_t totFail = useNew ? cN[T - 1] : cO[T - 1];
    const double epsPartial = sEps[useNew ? 0 : 1];
    const double eps = epsPartial + (double)(float)((float)D.cfg.H * D.cfg.maxVerifEps);
    float belief[DR_MAX_THETA];
    for (int i = 0; i < DR_MAX_THETA; i++)
        belief[i] = I.belief[i];
    int branchIdx = 0; // findConfident (state.h:93-115)
    for (int th = 0; th < nth; th++)
        if (belief[th] > D.cfg.minConf)
        {
            branchIdx = th + 1;
            break;
        }
    const float* chosen = useNew ? D.dense : D.prevDense;
    actions[inst * 2 + 0] = __ldcg(chosen + (size_t)branchIdx * T * 2 + 0);
    actions[inst * 2 + 1] = __ldcg(chosen + (size_t)branchIdx * T * 2 + 1);
    const float usedNu = D.nu[branchIdx];
    float lambda = I.lambda;
    if (usedNu > D.cfg.maxNu * (float)D.cfg.K)
        lambda *= 0.9f;
    else if (usedNu < D.cfg.minNu * (float)D.cfg.K)
        lambda *= 1.2f;
    dr_mppi_info info;
    info.fail_count_total = totFail;
    info.use_new_plan = useNew ? 1 : 0;
    info.epsilon = eps;
    info.epsilon_partial = epsPartial;
    info.certified_loss = cert;
    info.branch_idx = branchIdx;
    info.min_cost = D.minCosts[branchIdx * M];
    info.nu = usedNu;
    info.inv_temperature = lambda;
    info.nonfinite_costs = D.stats[0];
    info.verif_timeouts = D.stats[1];
    if (D.cfg.gradSteps > 0)
    {
        const int b = min(max((int)D.gstat[DR_GRAD_MAX_STEPS + 1], 0), DR_GRAD_MAX_STEPS);
        info.grad_cost_plain = D.gstat[0];
        info.grad_cost_refined = D.gstat[b];
        info.grad_best_step = b;
    }
    else
    {
        info.grad_cost_plain = 0.0f;
        info.grad_cost_refined = 0.0f;
        info.grad_best_step = -1;
    }
    infos[inst] = info;
    // state of the controller for its next step
    I.lambda = lambda;
    I.step = I.step + 1u;
    I.pendBranch = branchIdx;
    I.pendUseNew = useNew ? 1 : 0;
}

// Clopper-Pearson bounds on the device, for the test hook dr_debug_cp.
__global__ void cp_kernel(const uint32_t* __restrict__ k, int n, uint32_t N, double alpha, int upper, double* __restrict__ out)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n)
        out[i] = upper ? cpdetail::cpUpper(k[i], N, alpha) : cpdetail::cpLower(k[i], N, alpha);
}

template <int NOPP, int NTH>
__global__ void __launch_bounds__(128) batch_env_step(const MppiDev* __restrict__ insts, const MppiIn* __restrict__ in, const int* __restrict__ trueTheta,
                                                      const float* __restrict__ actions, dr_sim_state* __restrict__ states, float* __restrict__ beliefs,
                                                      int updateBelief, uint32_t k0, uint32_t k1, int* __restrict__ terms)
{
    __shared__ float sg[GRID_FLOATS];
    __shared__ EnvParams sE;
    const int inst = blockIdx.x;
    const MppiDev& D = insts[inst];
    for (int i = threadIdx.x; i < GRID_FLOATS; i += blockDim.x)
        sg[i] = D.grids[i];
    for (int i = threadIdx.x; i < ENV_HOST_WORDS; i += blockDim.x)
        ((float*)&sE)[i] = ((const float*)&D.env)[i];
    envDeviceTerms(sE, D.env, threadIdx.x, blockDim.x);
    __syncthreads();
    if (threadIdx.x != 0)
        return;
    const EnvParams& E = sE;
    constexpr int NA = NOPP + 1;
    dr_sim_state& st = states[inst];
    float* belief = beliefs + (size_t)inst * DR_MAX_THETA;
    DState<NA> s;
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
    s.locate(E.trackLength);
    BState<NTH> bs;
    for (int i = 0; i < NTH; i++)
        bs.belief[i] = belief[i];
    bs.predTheta = 0;
    bs.branchingTime = -1;
    const Track tr = trackIn(sg);
    // noise of the step: the stream of dr_env_step at the controller's step counter
    EnvNoise rng(k0, k1, 0u, 0u, in[inst].step, S_ENV_STEP);
    rng.begin_step(0);
    bool branched = false;
    const int th = trueTheta[inst];
    const float a0 = actions[inst * 2], a1 = actions[inst * 2 + 1];
    StepOut o;
    if (updateBelief)
        o = envStep<NOPP, NTH, true, false, false, true>(0, th, tr, E, a0, a1, s, bs, branched, 2.0f, rng);
    else
        o = envStep<NOPP, NTH, false, false, false, false>(0, th, tr, E, a0, a1, s, bs, branched, 2.0f, rng);
    for (int a = 0; a < NA; a++)
    {
        st.pos[2 * a] = s.pos[2 * a];
        st.pos[2 * a + 1] = s.pos[2 * a + 1];
        st.vel[2 * a] = s.vel[2 * a];
        st.vel[2 * a + 1] = s.vel[2 * a + 1];
        st.S[a] = s.S[a];
        st.lat_dist[a] = s.lat[a];
        st.laps[a] = s.laps[a];
    }
    for (int i = 0; i < NTH; i++)
        belief[i] = bs.belief[i];
    terms[inst] = o.term;
}

cudaError_t launchMppiFinish(cudaStream_t stream, const MppiDev* insts, MppiIn* in, float* actions, dr_mppi_info* infos, int nInst)
{
    mppi_finish<<<nInst, FB, 0, stream>>>(insts, in, actions, infos, nInst);
    return cudaGetLastError();
}

// The table of a (V, beta): [0] upper(k, V, beta/2), [1] lower(k, V, beta/2),
// [2] upper(k, max(V, 1), beta) for k = 0 .. max(V, 1), one thread per entry; counts
// below CP_TAB are left out (the controllers' own tables hold them).
__global__ void cp_table_fill(double* __restrict__ out, uint32_t V, double beta)
{
    const uint32_t V1 = V > 0 ? V : 1u;
    const size_t n = (size_t)3 * (V1 + 1);
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    {
        const int which = (int)(i / (V1 + 1));
        const uint32_t k = (uint32_t)(i % (V1 + 1));
        double v;
        if (k < (uint32_t)CP_TAB)
            v = 0.0;
        else if (which == 0)
            v = k <= V && V > 0 ? cpdetail::cpUpper(k, V, beta / 2.0) : 1.0;
        else if (which == 1)
            v = k <= V && V > 0 ? cpdetail::cpLower(k, V, beta / 2.0) : 0.0;
        else
            v = cpdetail::cpUpper(k, V1, beta);
        out[i] = v;
    }
}

namespace
{
struct CpTable
{
    double* ptr = nullptr;
    int refs = 0;
};
std::mutex cpMu;
std::map<std::tuple<int, uint32_t, uint64_t>, CpTable> cpTables;

std::tuple<int, uint32_t, uint64_t> cpKey(int device, uint32_t V, double beta)
{
    uint64_t b;
    std::memcpy(&b, &beta, 8);
    return {device, V, b};
}
} // namespace

bool acquireCpTable(int device, uint32_t V, double beta, const double** out)
{
    *out = nullptr;
    const uint32_t V1 = V > 0 ? V : 1u;
    if (V1 < (uint32_t)CP_TAB)
        return true; // every count is in the controllers' own tables
    std::lock_guard<std::mutex> lock(cpMu);
    CpTable& t = cpTables[cpKey(device, V, beta)];
    if (!t.ptr)
    {
        const size_t n = (size_t)3 * (V1 + 1);
        if (cudaMalloc(&t.ptr, n * sizeof(double)) != cudaSuccess)
        {
            t.ptr = nullptr;
            cpTables.erase(cpKey(device, V, beta));
            return false;
        }
        // filled on a stream of its own (non-blocking: no implicit ordering with the
        // controllers' streams, which may be capturing a graph in another thread)
        cudaStream_t fs = nullptr;
        bool ok = cudaStreamCreateWithFlags(&fs, cudaStreamNonBlocking) == cudaSuccess;
        if (ok)
        {
            cp_table_fill<<<(unsigned)std::min<size_t>((n + 255) / 256, 4096), 256, 0, fs>>>(t.ptr, V, beta);
            ok = cudaGetLastError() == cudaSuccess && cudaStreamSynchronize(fs) == cudaSuccess;
            cudaStreamDestroy(fs);
        }
        if (!ok)
        {
            cudaFree(t.ptr);
            cpTables.erase(cpKey(device, V, beta));
            return false;
        }
    }
    t.refs++;
    *out = t.ptr;
    return true;
}

void releaseCpTable(int device, uint32_t V, double beta)
{
    std::lock_guard<std::mutex> lock(cpMu);
    auto it = cpTables.find(cpKey(device, V, beta));
    if (it == cpTables.end())
        return;
    if (--it->second.refs <= 0)
    {
        if (it->second.ptr)
            cudaFree(it->second.ptr);
        cpTables.erase(it);
    }
}

cudaError_t launchCp(cudaStream_t stream, const uint32_t* k, int n, uint32_t N, double alpha, int upper, double* out)
{
    cp_kernel<<<(n + 127) / 128, 128, 0, stream>>>(k, n, N, alpha, upper, out);
    return cudaGetLastError();
}

cudaError_t launchBatchEnvStep(cudaStream_t stream, int nopp, int nth, const MppiDev* insts, const MppiIn* in, int nInst, const int* trueTheta,
                               const float* actions, dr_sim_state* states, float* beliefs, int updateBelief, uint32_t k0, uint32_t k1, int* terms)
{
#define DR_ENV_CASE(P, Q)                                                                                                                          \
    batch_env_step<P, Q><<<nInst, 128, 0, stream>>>(insts, in, trueTheta, actions, states, beliefs, updateBelief, k0, k1, terms);                  \
    break
    switch (nopp * 16 + nth)
    {
    case 1 * 16 + 1: DR_ENV_CASE(1, 1);
    case 1 * 16 + 2: DR_ENV_CASE(1, 2);
    case 1 * 16 + 4: DR_ENV_CASE(1, 4);
    case 1 * 16 + 8: DR_ENV_CASE(1, 8);
    case 2 * 16 + 2: DR_ENV_CASE(2, 2);
    default: return cudaErrorInvalidValue;
    }
#undef DR_ENV_CASE
    return cudaGetLastError();
}

} // namespace dr
