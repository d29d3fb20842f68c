// Host-side launch wrappers of the kernels (implemented in mppi_kernels.cu and
// prmppi_kernels.cu).
#pragma once

#include <cstddef>
#include <cuda_runtime.h>

#include "instance.cuh"

namespace dr
{

struct LaunchArgs
{
    cudaStream_t stream = nullptr;
    const MppiDev* mppi = nullptr;
    const MppiIn* mppiIn = nullptr;
    const PrDev* pr = nullptr;
    const PrIn* prIn = nullptr;
    const Tile* tiles = nullptr;
    int nTiles = 0;
    // Persistent launch: `grid` CTAs take tiles from the device work queue `queue` (a
    // ticket counter, zero when the launch starts) until the table is exhausted. With no
    // queue, one CTA per tile.
    unsigned* queue = nullptr;
    int grid = 0;
    // rollout: 1 = the CTA's threads step through the horizon together (a barrier per step)
    int lockstep = 0;
    // update / verification: launch as a programmatic dependent of the previous kernel of
    // the stream (its CTAs take SM slots as they free up and wait in the kernel)
    int pdl = 0;
    // verification: 1 = the exact arithmetic flavour and noise source (per-sample parity
    // with the oracle), 0 = the fast flavour (the default)
    int exactVerify = 0;
    // fast verification: 1 = the ego's moves come from the instances' ego tables
    // (mppi_ego_table must have filled them for the plans verified)
    int egoTable = 0;
    // PR-MPPI rollout: hypothesis slots per thread (1, 2, 4), sharing the ego's moves
    int prSlots = 1;
};

inline int launchGrid(const LaunchArgs& a)
{
    return a.queue ? (a.grid < a.nTiles ? a.grid : a.nTiles) : a.nTiles;
}

// Samples per verification CTA (one thread each). The CTA's warps step through the
// horizon together (a barrier per step), so the warps sharing an SM sub-partition fetch
// the same instructions; 512 threads, two CTAs per SM.
// Largest ego tables (both plans) a controller holds; larger ones (many hypotheses and a
// long verification horizon) are not built and the verification moves the ego itself.
#ifndef DR_EGO_TABLE_MAX_BYTES
#define DR_EGO_TABLE_MAX_BYTES (16u << 20)
#endif
constexpr size_t EGO_TABLE_MAX_BYTES = DR_EGO_TABLE_MAX_BYTES;

#ifndef DR_VERIFY_TILE
#define DR_VERIFY_TILE 512
#endif
constexpr int VERIFY_TILE = DR_VERIFY_TILE;

bool mppiSupported(int nopp, int nth);
int rolloutSamplesPerBlock(int nth);
size_t mppiRolloutSmem(int nth, int T, int M, bool spl);
size_t mppiVerifySmem(int nth, int T);
cudaError_t launchMppiPrologue(const LaunchArgs& a, int nInst, size_t smem);
cudaError_t launchMppiRollout(const LaunchArgs& a, int nopp, int nth, bool spl, size_t smem);
cudaError_t launchMppiUpdate(const LaunchArgs& a, int nth);
cudaError_t launchMppiAggregate(const LaunchArgs& a, int nth, int K);
// sample-sharded update phases (one controller's samples split across processes)
cudaError_t launchShardLocal(const LaunchArgs& a, int nth, float* partial);
cudaError_t launchShardMerge(cudaStream_t stream, const MppiDev* insts, const MppiIn* in, const float* gathered, int words, int world, float* mins,
                             float* sums);
cudaError_t launchShardApply(cudaStream_t stream, const MppiDev* insts, int nInst, int nth, const float* mins, const float* sums);
cudaError_t launchMppiVerify(const LaunchArgs& a, int nopp, int nth, size_t smem, int* dbgFailTime, int* dbgTheta);
// fills the ego tables (MppiDev::egoTab) of plan `plan` (0 new, 1 previous, 2 both) of
// every instance; maxH: the longest verification horizon of the instances
cudaError_t launchEgoTable(cudaStream_t stream, int nopp, int nth, const MppiDev* insts, const MppiIn* in, int nInst, int plan, int maxH);
// CTAs per SM of the persistent rollout (verify = false) or verification kernel
int mppiResident(int nopp, int nth, bool verify, bool spl, size_t smem);
cudaError_t launchMppiNoise(const LaunchArgs& a, size_t n, float* out);

bool gateSupported(int nth);
int gateRolloutSamplesPerBlock(int nth);
size_t gateRolloutSmem(int nth, int T, int M, bool spl);
size_t gateVerifySmem(int nth, int T);
// `me`: the ego's agent index (the environment's i_mppi)
cudaError_t launchGateRollout(const LaunchArgs& a, int nth, int me, bool spl, size_t smem);
cudaError_t launchGateVerify(const LaunchArgs& a, int nth, int me, size_t smem, int* dbgFailTime, int* dbgTheta);
cudaError_t launchGateBatchEnvStep(cudaStream_t stream, int nth, int me, const MppiDev* insts, const MppiIn* in, int nInst, const int* trueTheta,
                                   const float* actions, dr_gate_state* states, float* beliefs, int updateBelief, uint32_t k0, uint32_t k1, int* terms);
cudaError_t launchGateEnvStep(cudaStream_t stream, int nth, int me, const GateParams* gp, const float* track, int trueTheta, float a0, float a1,
                              dr_gate_state* st, float* belief, int updateBelief, uint32_t k0, uint32_t k1, uint32_t step, int* term);

// One gradient-path job (grad_kernels.cu): the objective of an instance's noise-free
// rollout at a start point U, its gradients, and optionally projected gradient steps.
struct GradJob
{
    const MppiDev* D;
    const MppiIn* in;
    const float* U;  // start point [nbp][M][2] (null: the instance's knots)
    const float* w6; // cost weights, grad::WeightIndex order (null: the instance's)
    float* J;        // objective of each iterate, [iters + 1] (or null)
    float* gU;       // gradient at the start point with respect to U (or null)
    float* gW;       // gradient at the start point with respect to the weights (or null)
    float* stats;    // [0] iterate with the lowest objective, [1] last iterate evaluated (or null)
    int iters;       // projected gradient steps (0: evaluate once)
    int ckpt;        // checkpoint stride of the adjoint sweep, 1..T
    float alpha;     // step, as a fraction of the ego's acceleration limit
    int write;       // write the best iterate to the instance's knots and dense plan
};

size_t gradSmem(int nopp, int nth, int T, int M, int ckpt, bool spl);
// checkpoint stride for ckpt == 0: 1 (every state kept) when it fits, else ceil(sqrt(T))
int gradDefaultStride(int nopp, int nth, int T, int M, bool spl);
cudaError_t launchGradNominal(cudaStream_t stream, const GradJob* jobs, int nJobs, int nopp, int nth, bool spl, size_t smem);

// PR-MPPI on the gate race (gate_pr_kernels.cu); prologue and weighted averages are shared
size_t gatePrRolloutSmem(int T);
int gatePrRolloutSamplesPerBlock();
cudaError_t launchGatePrRollout(const LaunchArgs& a, int nth, int me, size_t smem);
cudaError_t launchGatePrCandidates(const LaunchArgs& a, int nth, int me, int nInst, int maxT);

// sample-sharded PR-MPPI update phases (one controller's samples split across processes)
cudaError_t launchPrShardMin(cudaStream_t stream, const PrDev* insts, float* mins);
cudaError_t launchPrShardSums(cudaStream_t stream, const PrDev* insts, const PrIn* in, int T, const float* mins, float* sums);
cudaError_t launchPrShardApply(cudaStream_t stream, const PrDev* insts, const float* mins, const float* sums);
cudaError_t launchPrShardMerge(cudaStream_t stream, const PrDev* insts, const PrIn* in, const float* gathered, int words, int world, float* mins,
                               float* sums);

// Device tail of the control step and the batch's true-dynamics step (finish_kernels.cu).
cudaError_t launchMppiFinish(cudaStream_t stream, const MppiDev* insts, MppiIn* in, float* actions, dr_mppi_info* infos, int nInst);

// Prediction streaming (predict_kernels.cu). Row r of controller i is at (i * rows + r):
// positions [tStride][2 (n_opp + 1)], actions [tStride][2], PREDICT_RECORD ints
// (initial branch, branching time, branch, stop reason, stop time) and one cost.
constexpr int PREDICT_RECORD = 5;
struct PredictOut
{
    float* pos;
    float* act;
    int* rec;
    float* cost;
    int tStride;
};
cudaError_t launchMppiPredict(cudaStream_t stream, int nopp, int nth, const MppiDev* insts, const MppiIn* in, const dr_sim_state* states,
                              const float* beliefs, int beliefStride, const PredictOut& out, int nInst);
cudaError_t launchPrPredict(cudaStream_t stream, int nopp, int nth, const PrDev* insts, const dr_sim_state* prevStates, const PredictOut& out, int nInst);
cudaError_t launchBatchEnvStep(cudaStream_t stream, int nopp, int nth, const MppiDev* insts, const MppiIn* in, int nInst, const int* trueTheta,
                               const float* actions, dr_sim_state* states, float* beliefs, int updateBelief, uint32_t k0, uint32_t k1, int* terms);
// Clopper-Pearson bounds of every failure count for verification size V and level beta,
// on `device` (current), shared by the controllers that acquire the same (V, beta) and
// freed when the last one releases it. *out is null when V < CP_TAB (the controllers' own
// tables hold every count); false when the allocation or the fill failed.
bool acquireCpTable(int device, uint32_t V, double beta, const double** out);
void releaseCpTable(int device, uint32_t V, double beta);
cudaError_t launchCp(cudaStream_t stream, const uint32_t* k, int n, uint32_t N, double alpha, int upper, double* out);

// Track grids of nTracks tracks from their 512 samples q [nTracks][512][2] (track_kernels.cu);
// out [nTracks][7 x 512]: p[512][2] | dp[512][2] | t[512][2] | kappa[512].
cudaError_t launchTrackGrids(cudaStream_t stream, const double* q, int nTracks, float* out, float* lengths);

bool prSupported(int nopp, int nth);
int prRolloutSamplesPerBlock();
size_t prRolloutSmem(int T);
cudaError_t launchPrPrologue(const LaunchArgs& a, int nInst);
cudaError_t launchPrRollout(const LaunchArgs& a, int nopp, int nth, size_t smem);
cudaError_t launchPrReduce(const LaunchArgs& a);
cudaError_t launchPrCandidates(const LaunchArgs& a, int nopp, int nth, int nInst, int maxP, size_t smem);
cudaError_t launchPrNoise(const LaunchArgs& a, size_t n, float* out);

} // namespace dr
