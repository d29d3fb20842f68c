// Small device utilities shared by the kernels: bulk (TMA) global->shared copies
// completed on an mbarrier with a bounded wait, and block reductions.
#pragma once

#include <cstdint>
#include <map>
#include <mutex>
#include <utility>

#include <cuda_runtime.h>

namespace dr
{

// Raises a kernel's dynamic shared-memory limit when a launch needs more than it was
// given before (per device). Calls nothing when the limit already suffices, so a launch
// inside a stream capture makes no attribute call.
template <typename Kern> inline void ensureSmem(Kern kernel, size_t smem)
{
    static std::mutex mu;
    static std::map<std::pair<int, const void*>, size_t> done;
    if (smem <= 48 * 1024)
        return;
    int dev = 0;
    cudaGetDevice(&dev);
    std::lock_guard<std::mutex> lock(mu);
    size_t& have = done[{dev, (const void*)kernel}];
    if (have >= smem)
        return;
    if (cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) == cudaSuccess)
        have = smem;
}

__device__ __forceinline__ uint32_t smem_u32(const void* p)
{
    return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}

// One-dimensional bulk copy global -> shared of `bytes` (multiple of 16, both
// addresses 16-byte aligned), completing on `bar`. No multicast.
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(smem_u32(dst)), "l"(src), "r"(bytes),
                 "r"(smem_u32(bar))
                 : "memory");
}

// Default poll limit of a bounded wait (each poll is one try_wait, which may suspend the
// thread for a short, hardware-defined time).
constexpr int WAIT_POLLS = 1 << 22;

// Waits for phase `parity` of `bar`, giving up after `polls` polls (a non-positive value
// means the default). Returns false on timeout.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, int polls = WAIT_POLLS)
{
    uint32_t done = 0;
    if (polls <= 0)
        polls = WAIT_POLLS;
    for (int it = 0; it < polls; it++)
    {
        asm volatile("{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
                     : "=r"(done)
                     : "r"(smem_u32(bar)), "r"(parity)
                     : "memory");
        if (done)
            return true;
    }
    return false;
}

// Programmatic dependent launch (sm_90 and later). A kernel launched with the
// programmatic-stream-serialization attribute may start while the previous kernel of its
// stream is still running: pdl_wait() blocks until that kernel has completed and its
// writes are visible (it returns at once in a kernel launched without the attribute).
// pdl_trigger() allows the next such kernel to launch once every CTA of this one has
// executed it (or exited).
__device__ __forceinline__ void pdl_wait()
{
    asm volatile("griddepcontrol.wait;" ::: "memory");
}

__device__ __forceinline__ void pdl_trigger()
{
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

// Launches `k` with the programmatic-stream-serialization attribute when `pdl` is set,
// else as a plain launch.
template <typename... KArgs, typename... Args>
inline cudaError_t launchMaybePdl(bool pdl, void (*k)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t stream, Args... args)
{
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = stream;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = pdl ? at : nullptr;
    cfg.numAttrs = pdl ? 1 : 0;
    return cudaLaunchKernelEx(&cfg, k, args...);
}

// The tile a CTA works on in iteration `iter` of its tile loop. A static launch (no queue)
// has one CTA per tile: its own, once. A persistent launch takes the next ticket of the
// device work queue (tiles in table order, so the table lists the longest tiles first);
// a ticket past the table's end ends the loop. `sTicket` is a shared word; the caller
// takes a barrier between two calls.
__device__ __forceinline__ int nextTile(unsigned* queue, int iter, int* sTicket)
{
    if (!queue)
        return iter == 0 ? (int)blockIdx.x : 0x7fffffff;
    if (threadIdx.x == 0)
        *sTicket = (int)atomicAdd(queue, 1u);
    __syncthreads();
    return *sTicket;
}

__device__ __forceinline__ float warp_min(float v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
        v = fminf(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

} // namespace dr
