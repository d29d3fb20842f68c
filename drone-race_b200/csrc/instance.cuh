// Device-side description of one controller instance (one agent's MPPI or PR-MPPI
// controller) and of the per-step records exchanged with the host. A batch launch
// covers several instances; each CTA works on one instance, found through a tile table.
#pragma once

#include <cstdint>

#include "../../include/drmppi.h"
#include "gate_model.cuh"
#include "model.cuh"

namespace dr
{

struct MppiCfgDev
{
    int K, T, M, useSplines, V, H, nth, nopp;
    int knots[DR_MAX_KNOTS];
    float sigma0, sigma1, minConf;
    float gateMargin; // gateTraversalMargin (gate race)
    MppiCostW w;
    uint32_t k0, k1; // Philox key (seed)
    // host-tail parameters, for the device tail (finish_kernels.cu)
    float beta, maxVerifEps, minNu, maxNu;
    int verify;
    int gradSteps; // gradient refinement steps (0: off)
    int sLo, sHi;  // this process's samples when the controller is sample-sharded (else 0, K)
    // Bounded-wait test switch (dr_mppi_debug_stage_timeout): when set, the rollout and
    // verification CTAs announce their staging bytes on the mbarrier but issue no copy, so
    // the barrier's phase never completes and the wait gives up after waitPolls polls (0:
    // the default limit). Nothing is in flight when such a CTA returns.
    int dbgNoStage;
    int waitPolls;
};

// Per-step input of an MPPI instance (one H2D copy per step for the whole batch).
struct MppiIn
{
    union
    {
        dr_sim_state state;   // strategic race
        dr_gate_state gstate; // gate race
    };
    float belief[DR_MAX_THETA];
    float lambda;      // inv_temperature of this step
    uint32_t step;     // Philox counter word
    int pendBranch;    // branch to shift (previous step's chosen branch) or -1
    int pendUseNew;    // previous step used the new plan
};

// Device buffers of an MPPI instance. `res` is the start of the contiguous result
// block copied to the host after each step:
//   fail[2][T] u32 | dense[nbp][T][2] | prevDense[nbp][T][2] | nu[nbp] | minCosts[nbp][M] | stats[4] i32 |
//   gstat[DR_GRAD_MAX_STEPS + 3] f32
struct MppiDev
{
    EnvParams env;       // strategic race (for the gate race only maxAccel[0], the ego's, is set)
    MppiCfgDev cfg;
    const float* grids;  // GRID_FLOATS, 16-byte aligned (strategic race)
    const GateParams* gate; // gate race: parameters and racelines (GATE_TRACK_FLOATS), else null
    const float* gtrack;
    const float* B;      // [T][M] (spline mode)
    float* knots;        // [nbp][M][2] optimised sequence (dense mode: M == T)
    float* costsTrue;    // [nth][K]
    int* binfo;          // [nth][K] predTheta << 16 | (branchTime & 0xffff)
    float* costs;        // [nbp][K]
    unsigned* counter;   // completion counter of the update kernel
    // result block
    unsigned* fail;      // [2][T]: 0 = new plan, 1 = previous plan
    float* dense;        // [nbp][T][2]
    float* prevDense;    // [nbp][T][2]
    float* nu;           // [nbp]
    float* minCosts;     // [nbp][M]
    int* stats;          // [0] non-finite costs, [1] timeouts
    float* gstat;        // gradient refinement: objective of iterates 0..DR_GRAD_MAX_STEPS, best iterate, last iterate
    // Clopper-Pearson bounds for counts k < CP_TAB, filled on the host at creation:
    // [0] upper(k, V, beta/2), [1] lower(k, V, beta/2), [2] upper(k, max(V, 1), beta)
    const double* cpTab;
    // the same three bounds for every count, [which][k] for k <= max(V, 1), computed on the
    // device once per (device, V, beta) and shared by the controllers that have them (or null)
    const double* cpFull;
    // The ego's moves under each plan (new = 0, previous = 1), shared by the verification
    // samples (EgoRow): [plan][row][H], row 0 = no branch (or the branch of a confident
    // initial belief), row 1 + (b - 1) H + tb = branch b taken at step tb; or null
    EgoRow* egoTab;
    size_t resBytes;
};

constexpr int CP_TAB = 1024;

// rows of a plan's ego table
__host__ __device__ __forceinline__ int egoRows(int nth, int H)
{
    return 1 + nth * H;
}

struct PrCfgDev
{
    int K, T, P, nth, nopp;
    float sigma0, sigma1;
    float collDistFactor, boundaryCost, boundaryThresholdFactor, winCost, oppWinCost, finalAdvWeight, finalOppAdvWeight, safetyWeight;
    uint32_t k0, k1;
    int sLo, sHi; // this process's samples [sLo, sHi) (all of them unless sharded)
    float gateMargin; // gateTraversalMargin (gate race)
};

struct PrIn
{
    union
    {
        dr_sim_state state;   // strategic race
        dr_gate_state gstate; // gate race
    };
    float belief[DR_MAX_THETA];
    float lambda[3];
    uint32_t step;
    int pad;
};

// result block: nom[T][2] | rob[T][2] | cand1[T][2] | cand2[T][2] | minCosts[3] | nu[3] |
//               candFull[2][P] | candSafe[2][P] | thetas[P] | decision[4] | stats[4]
struct PrDev
{
    EnvParams env;
    PrCfgDev cfg;
    const float* grids;
    const GateParams* gate; // gate race: parameters and racelines (GATE_TRACK_FLOATS), else null
    const float* gtrack;
    float* costNom;   // [P][K][2]
    float* costRob;   // [P][K][2]
    float* avg;       // [2][K][2] per-sample averaged (full, safe) for nom / rob
    float* nomWork;   // [T][2] shifted nominal used this step
    float* robWork;   // [T][2]
    unsigned* counter;
    // result block
    float* nom;       // [T][2] chosen nominal after the step
    float* rob;       // [T][2] new robust nominal
    float* cand1;     // [T][2]
    float* cand2;     // [T][2]
    float* minCosts;  // [3]
    float* nu;        // [3]
    float* candFull;  // [2][P]
    float* candSafe;  // [2][P] safety of each candidate on the re-check stream
    int* thetas;      // [P]
    int* decision;    // [0] resetNom, [1] useNomPlan
    int* stats;
    size_t resBytes;
};

struct Tile
{
    int inst;
    int s0;
    int count;
    int aux;
};

// Branch record of a rollout sample: predTheta << 16 | (branchTime & 0xffff).
__device__ __forceinline__ int packInfo(int pt, int bt)
{
    return (pt << 16) | (bt & 0xffff);
}

// Outputs of a rollout tile whose staging wait gave up: every sample gets an infinite
// cost under every hypothesis and branch plan and the branch record of the initial
// belief, so that the update reads defined values (the step then reports the timeout).
template <int NTH> __device__ __forceinline__ void rolloutTileTimedOut(const MppiDev& D, const MppiIn& I, const Tile& tile, int K)
{
    const int th = threadIdx.x % NTH;
    const int sl = threadIdx.x / NTH;
    if (sl >= tile.count)
        return;
    const int s = tile.s0 + sl;
    float belief0[NTH];
#pragma unroll
    for (int i = 0; i < NTH; i++)
        belief0[i] = I.belief[i];
    const int pt0 = findConfident<NTH>(belief0, D.cfg.minConf);
    D.costsTrue[th * K + s] = INFINITY;
    D.binfo[th * K + s] = packInfo(pt0, pt0 == 0 ? -1 : 0);
    D.costs[(size_t)(th + 1) * K + s] = INFINITY;
    if (th == 0)
        D.costs[s] = INFINITY;
}

} // namespace dr
