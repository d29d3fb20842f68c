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
};

// Samples per verification CTA (one thread each). The CTA's warps step through the
// horizon together (a barrier per step), so the warps sharing an SM sub-partition fetch
// the same instructions; 512 threads, two CTAs per SM.
constexpr int VERIFY_TILE = 512;

bool mppiSupported(int nopp, int nth);
int rolloutSamplesPerBlock(int nth);
size_t mppiRolloutSmem(int nth, int T, int M, bool spl);
size_t mppiVerifySmem(int nth, int T);
cudaError_t launchMppiPrologue(const LaunchArgs& a, int nInst, size_t smem);
cudaError_t launchMppiRollout(const LaunchArgs& a, int nopp, int nth, bool spl, size_t smem);
cudaError_t launchMppiUpdate(const LaunchArgs& a, int nth);
cudaError_t launchMppiAggregate(const LaunchArgs& a, int nth, int K);
cudaError_t launchMppiVerify(const LaunchArgs& a, int nopp, int nth, size_t smem, int* dbgFailTime, int* dbgTheta);
cudaError_t launchMppiNoise(const LaunchArgs& a, size_t n, float* out);

bool gateSupported(int nth);
int gateRolloutSamplesPerBlock(int nth);
size_t gateRolloutSmem(int nth, int T, int M, bool spl);
size_t gateVerifySmem(int nth, int T);
// `me`: the ego's agent index (the environment's i_mppi)
cudaError_t launchGateRollout(const LaunchArgs& a, int nth, int me, bool spl, size_t smem);
cudaError_t launchGateVerify(const LaunchArgs& a, int nth, int me, size_t smem, int* dbgFailTime, int* dbgTheta);
cudaError_t launchGateEnvStep(cudaStream_t stream, int nth, int me, const GateParams* gp, const float* track, int trueTheta, float a0, float a1,
                              dr_gate_state* st, float* belief, int updateBelief, uint32_t k0, uint32_t k1, uint32_t step, int* term);

bool prSupported(int nopp, int nth);
int prRolloutSamplesPerBlock();
size_t prRolloutSmem(int T);
cudaError_t launchPrPrologue(const LaunchArgs& a, int nInst);
cudaError_t launchPrRollout(const LaunchArgs& a, int nopp, int nth, size_t smem);
cudaError_t launchPrReduce(const LaunchArgs& a);
cudaError_t launchPrCandidates(const LaunchArgs& a, int nopp, int nth, int nInst, int maxP, size_t smem);
cudaError_t launchPrNoise(const LaunchArgs& a, size_t n, float* out);

} // namespace dr
