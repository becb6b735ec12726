// Device-side building blocks: warp/block reductions and the last-block ticket.
#pragma once

#include "dev_types.h"

#include <utility>

namespace cfg
{

/// Entry of a kernel that may be launched as a programmatic dependent of
/// the kernel before it in the stream (launchK with pdl): first let the
/// kernel after this one launch, then wait until the kernel before this one
/// has completed and its writes are visible.  Nothing of this kernel reads
/// or writes global memory before the wait, so the order of memory effects
/// is that of plain stream order; what overlaps is the launch and block
/// scheduling of one kernel with the tail of the one before.  Both
/// instructions are no-ops for a kernel launched without the attribute.
__device__ __forceinline__ void pdl_entry()
{
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
    asm volatile("griddepcontrol.wait;" ::: "memory");
}

/// Launches kernel k on stream s; with pdl, as a programmatic dependent of
/// the kernel before it, which requires k to begin with pdl_entry().
template <class... KArgs, class... Args>
inline void launchK(bool pdl, void (*k)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t s,
                    Args&&... args)
{
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = pdl ? 1 : 0;
    CFG_CUDA(cudaLaunchKernelEx(&cfg, k, std::forward<Args>(args)...));
}

__device__ __forceinline__ double warp_sum(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}
__device__ __forceinline__ double warp_max(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
    {
        const double w = __shfl_down_sync(0xffffffffu, v, o);
        v = (v < w) ? w : v;
    }
    return v;
}

/// Block-wide sums of NV values in a fixed tree order; result in thread 0.
template <int NV>
__device__ __forceinline__ void block_sum(double (&v)[NV])
{
    __shared__ double sh[NV][TPB / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int q = 0; q < NV; ++q) v[q] = warp_sum(v[q]);
    __syncthreads();
    if (lane == 0)
#pragma unroll
        for (int q = 0; q < NV; ++q) sh[q][warp] = v[q];
    __syncthreads();
    if (warp == 0)
#pragma unroll
        for (int q = 0; q < NV; ++q) v[q] = warp_sum(lane < TPB / 32 ? sh[q][lane] : 0.0);
}

template <int NV>
__device__ __forceinline__ void block_max(double (&v)[NV])
{
    __shared__ double sh[NV][TPB / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int q = 0; q < NV; ++q) v[q] = warp_max(v[q]);
    __syncthreads();
    if (lane == 0)
#pragma unroll
        for (int q = 0; q < NV; ++q) sh[q][warp] = v[q];
    __syncthreads();
    if (warp == 0)
#pragma unroll
        for (int q = 0; q < NV; ++q) v[q] = warp_max(lane < TPB / 32 ? sh[q][lane] : 0.0);
}

/// Threadfence-reduction ticket: true in every thread of the block that
/// finishes last.  No block waits for another.
__device__ __forceinline__ bool last_block(unsigned int* ticket)
{
    __shared__ bool amLast;
    __syncthreads();
    if (threadIdx.x == 0)
    {
        __threadfence();
        const unsigned int t = atomicAdd(ticket, 1u);
        amLast = (t == gridDim.x - 1);
    }
    __syncthreads();
    if (amLast) __threadfence();
    return amLast;
}

/// The last block's pass over the per-block partials: for each of the NV
/// arrays in turn, every thread loads FU of its values before the first
/// add, so an array costs ceil(G / (FU * TPB)) memory latencies rather than
/// G / TPB, without holding NV * FU values in registers.  Sums combine in a
/// fixed order (pairwise within a thread, then the block tree), so a given
/// grid size always gives the same bits.
constexpr int FU = 8;

__device__ __forceinline__ double partial_sum(const double* a, int G)
{
    double v = 0.0;
    for (int b0 = threadIdx.x; b0 < G; b0 += FU * TPB)
    {
        double w[FU];
#pragma unroll
        for (int u = 0; u < FU; ++u) w[u] = b0 + u * TPB < G ? __ldcg(a + b0 + u * TPB) : 0.0;
        v += ((w[0] + w[1]) + (w[2] + w[3])) + ((w[4] + w[5]) + (w[6] + w[7]));
    }
    return v;
}
static_assert(FU == 8, "partial_sum's pairwise tree is written for FU = 8");

__device__ __forceinline__ double partial_max(const double* a, int G)
{
    double v = 0.0;
    for (int b0 = threadIdx.x; b0 < G; b0 += FU * TPB)
    {
        double w[FU];
#pragma unroll
        for (int u = 0; u < FU; ++u) w[u] = b0 + u * TPB < G ? __ldcg(a + b0 + u * TPB) : 0.0;
#pragma unroll
        for (int u = 0; u < FU; ++u) v = (v < w[u]) ? w[u] : v;
    }
    return v;
}

/// Sum of NV partial arrays (layout q*G + block) in fixed order; thread 0.
template <int NV>
__device__ __forceinline__ void final_sum(const double* partials, int G, double (&v)[NV])
{
#pragma unroll 1
    for (int q = 0; q < NV; ++q) v[q] = partial_sum(partials + q * G, G);
    block_sum<NV>(v);
}

template <int NV>
__device__ __forceinline__ void final_max(const double* partials, int G, double (&v)[NV])
{
#pragma unroll 1
    for (int q = 0; q < NV; ++q) v[q] = partial_max(partials + q * G, G);
    block_max<NV>(v);
}

/// std::max / std::min semantics (NaN in the second argument is dropped).
__device__ __forceinline__ double smax(double a, double b) { return (a < b) ? b : a; }
__device__ __forceinline__ double smin(double a, double b) { return (b < a) ? b : a; }

/// Non-negative double max through its bit pattern (order-independent).
__device__ __forceinline__ void atomic_max_nonneg(double* addr, double v)
{
    if (!(v > 0.0)) return;  // also drops NaN, as std::max(acc, NaN) does
    atomicMax(reinterpret_cast<unsigned long long*>(addr), static_cast<unsigned long long>(__double_as_longlong(v)));
}

}  // namespace cfg
