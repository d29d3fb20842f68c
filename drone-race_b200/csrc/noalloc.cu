// Allocation-free entry point: the fused MPPI rollout + per-branch cost aggregation
// with all of its working memory in one statically allocated device array, for callers
// that cannot call cudaMalloc -- code running where the device allocator is off limits,
// such as inside a region that a memory-pool owner or a real-time loop forbids to
// allocate from, or a host framework that hands the library only the buffers it owns.
//
// The array below is this library's whole scratch for that entry point: every GPU that
// loads the library holds DR_NOALLOC_SCRATCH_BYTES of it until the process exits. All
// calls share it, so calls whose GPU work overlaps (on different streams or threads)
// race on it and must be serialised by the caller. The first call on a device looks up
// the array's device address (cudaGetSymbolAddress) with that device current; make that
// first call before any CUDA stream capture. The address is kept per device and per CUDA
// context, so a device reset (which reloads the module in a new context) is followed by a
// fresh look-up instead of a stale address.
#include <cstring>
#include <mutex>
#include <vector>

#include <cuda.h>
#include <cuda_runtime.h>

#include "../../include/drmppi.h"
#include "hostutil.hpp"
#include "instance.cuh"
#include "launch.h"

using namespace dr;

namespace
{

static __device__ __align__(256) unsigned char g_noallocScratch[DR_NOALLOC_SCRATCH_BYTES];

constexpr int MAX_DEVICES = 64;

// The current CUDA context (driver cuCtxGetCurrent, reached through the runtime's entry
// point query, so the library does not link the driver library), or null.
CUcontext currentContext()
{
    using Fn = CUresult (*)(CUcontext*);
    static Fn fn = [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q{};
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) != cudaSuccess || q != cudaDriverEntryPointSuccess)
            return (Fn) nullptr;
        return (Fn)p;
    }();
    CUcontext c = nullptr;
    if (!fn || fn(&c) != CUDA_SUCCESS)
        return nullptr;
    return c;
}

// device address of g_noallocScratch per device, looked up with the device current the
// first time the device is used in its current context
unsigned char* scratchAddress(int& status)
{
    static std::mutex mu;
    static unsigned char* addr[MAX_DEVICES] = {};
    static CUcontext ctxOf[MAX_DEVICES] = {};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= MAX_DEVICES)
    {
        status = fail(DR_ERR_NO_DEVICE, "no current CUDA device");
        return nullptr;
    }
    // makes the device's primary context current (cudaSetDevice initialises it) before the
    // context is read
    cudaError_t fe = cudaSetDevice(dev);
    if (fe != cudaSuccess)
    {
        status = fail(DR_ERR_CUDA, std::string("CUDA context setup failed: ") + cudaGetErrorString(fe));
        return nullptr;
    }
    const CUcontext ctx = currentContext();
    std::lock_guard<std::mutex> lock(mu);
    if (!addr[dev] || ctxOf[dev] != ctx)
    {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noallocScratch);
        if (e != cudaSuccess || !p)
        {
            status = fail(DR_ERR_CUDA, std::string("cudaGetSymbolAddress of the static scratch failed: ") + cudaGetErrorString(e));
            return nullptr;
        }
        addr[dev] = (unsigned char*)p;
        ctxOf[dev] = ctx;
    }
    status = DR_OK;
    return addr[dev];
}

} // namespace

extern "C" int dr_mppi_rollout_costs_noalloc(const dr_env_config* env, const dr_mppi_config* cfg, uint64_t seed, uint64_t step, const dr_sim_state* state,
                                             const float* belief, const float* knots_dev, float* costs_dev, void* stream)
{
    int rc = checkEnv(env);
    if (rc)
        return rc;
    if (!cfg || !state || !belief || !knots_dev || !costs_dev)
        return fail(DR_ERR_INVALID_ARG, "NULL argument");
    if (cfg->n_samples < 1 || cfg->n_timesteps < 2 || cfg->n_timesteps > DR_MAX_T)
        return fail(DR_ERR_INVALID_ARG, "n_samples must be positive and n_timesteps in [2, 256]");
    const bool spl = cfg->use_splines != 0;
    if (spl)
    {
        if (cfg->n_knots < 2 || cfg->n_knots > DR_MAX_KNOTS)
            return fail(DR_ERR_INVALID_ARG, "n_knots must be in [2, 64]");
        for (int i = 0; i < cfg->n_knots; i++)
            if (cfg->knots[i] < 0 || cfg->knots[i] > cfg->n_timesteps - 2 || (i > 0 && cfg->knots[i] <= cfg->knots[i - 1]))
                return fail(DR_ERR_INVALID_ARG, "knots must be strictly increasing inside [0, T-2]");
    }
    if (!mppiSupported(env->n_opp, env->n_theta))
        return fail(DR_ERR_UNSUPPORTED, "(n_opp, n_theta) combination not compiled in");
    const int K = cfg->n_samples, T = cfg->n_timesteps, M = spl ? cfg->n_knots : T, nth = env->n_theta, nbp = nth + 1;
    const int spb = rolloutSamplesPerBlock(nth);
    const int nTiles = (K + spb - 1) / spb;

    // layout of the scratch for this call (every block 256-byte aligned)
    size_t off = 0;
    auto take = [&](size_t bytes) {
        size_t o = a256(off);
        off = o + a256(bytes > 0 ? bytes : 16);
        return o;
    };
    const size_t oDesc = take(sizeof(MppiDev)), oIn = take(sizeof(MppiIn)), oGrid = take(GRID_FLOATS * 4), oKnots = take(a16((size_t)nbp * M * 2 * 4)),
                 oB = take(spl ? a16((size_t)T * M * 4) : 16), oTiles = take(sizeof(Tile) * (size_t)nTiles), oCT = take((size_t)nth * K * 4),
                 oInfo = take((size_t)nth * K * 4), oStats = take(16);
    if (off > DR_NOALLOC_SCRATCH_BYTES)
        return fail(DR_ERR_INVALID_ARG, "problem too large for the static scratch: needs " + std::to_string(off) + " bytes, the limit is " +
                                            std::to_string((size_t)DR_NOALLOC_SCRATCH_BYTES) +
                                            " (about 2 x n_theta x n_samples x 4 bytes plus the track and the controls)");
    unsigned char* base = scratchAddress(rc);
    if (!base)
        return rc;
    cudaStream_t s = (cudaStream_t)stream;

    // instance description in the scratch, pointing at the caller's output
    MppiDev D{};
    D.env = toEnvParams(*env);
    D.cfg.K = K;
    D.cfg.T = T;
    D.cfg.M = M;
    D.cfg.useSplines = spl ? 1 : 0;
    D.cfg.nth = nth;
    D.cfg.nopp = env->n_opp;
    for (int i = 0; i < DR_MAX_KNOTS; i++)
        D.cfg.knots[i] = spl ? cfg->knots[i] : i;
    float s0 = cfg->sampling_noise_dim[0], s1 = cfg->sampling_noise_dim[1];
    if (s0 == 0.0f && s1 == 0.0f)
        s0 = s1 = cfg->sampling_noise;
    D.cfg.sigma0 = s0;
    D.cfg.sigma1 = s1;
    D.cfg.minConf = cfg->min_confidence;
    D.cfg.w = MppiCostW{cfg->coll_dist_factor, cfg->boundary_cost, cfg->boundary_threshold_factor, cfg->outside_cost,
                        cfg->win_cost,         cfg->opp_win_cost,  cfg->final_adv_weight,          cfg->final_opp_adv_weight};
    D.cfg.k0 = (uint32_t)seed;
    D.cfg.k1 = (uint32_t)(seed >> 32);
    D.grids = (const float*)(base + oGrid);
    D.B = (const float*)(base + oB);
    D.knots = (float*)(base + oKnots);
    D.costsTrue = (float*)(base + oCT);
    D.binfo = (int*)(base + oInfo);
    D.costs = costs_dev;
    D.stats = (int*)(base + oStats);
    MppiIn in{};
    in.state = *state;
    for (int i = 0; i < nth; i++)
        in.belief[i] = belief[i];
    in.lambda = cfg->inv_temperature;
    in.step = (uint32_t)step;
    in.pendBranch = -1;
    std::vector<Tile> tiles(nTiles);
    for (int i = 0; i < nTiles; i++)
        tiles[i] = Tile{0, i * spb, std::min(spb, K - i * spb), 0};
    std::vector<float> grids = packGrids(*env);
    std::vector<float> B;
    if (spl)
        B = splineMatrix(T, M, cfg->knots);

    // only the statistics words need to start at zero; the kernel writes every other
    // word it reads (costs and branch records of all samples)
    CK(cudaMemsetAsync(base + oStats, 0, 16, s));
    CK(cudaMemcpyAsync(base + oDesc, &D, sizeof(MppiDev), cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(base + oIn, &in, sizeof(MppiIn), cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(base + oGrid, grids.data(), GRID_FLOATS * 4, cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(base + oKnots, knots_dev, (size_t)nbp * M * 2 * 4, cudaMemcpyDeviceToDevice, s));
    if (spl)
        CK(cudaMemcpyAsync(base + oB, B.data(), B.size() * 4, cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(base + oTiles, tiles.data(), sizeof(Tile) * tiles.size(), cudaMemcpyHostToDevice, s));
    LaunchArgs a;
    a.stream = s;
    a.mppi = (const MppiDev*)(base + oDesc);
    a.mppiIn = (const MppiIn*)(base + oIn);
    a.tiles = (const Tile*)(base + oTiles);
    a.nTiles = nTiles;
    CK(launchMppiRollout(a, env->n_opp, nth, spl, mppiRolloutSmem(nth, T, M, spl)));
    // copies from pageable host memory have taken their data when they return, so the
    // host records may go out of scope; wait for the kernel so that the caller may read
    // costs_dev on any stream afterwards
    CK(cudaStreamSynchronize(s));
    // the statistics words: [0] samples whose cost is not finite (left in costs_dev as
    // they are), [1] rollout CTAs whose staging wait gave up (their samples cost infinity)
    int stats[4] = {0, 0, 0, 0};
    CK(cudaMemcpy(stats, base + oStats, sizeof(stats), cudaMemcpyDeviceToHost));
    if (stats[1] > 0)
        return fail(DR_ERR_TIMEOUT, "a bounded device wait gave up in " + std::to_string(stats[1]) + " rollout CTA(s); costs_dev is not valid");
    return DR_OK;
}
