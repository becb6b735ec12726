// Device-side building blocks: warp/block reductions and the last-block ticket.
#pragma once

#include "dev_types.h"

namespace cfg
{

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

/// Sum of NV partial arrays (layout q*G + block) in fixed order; thread 0.
template <int NV>
__device__ __forceinline__ void final_sum(const double* partials, int G, double (&v)[NV])
{
#pragma unroll
    for (int q = 0; q < NV; ++q)
    {
        double a = 0.0;
        for (int b = threadIdx.x; b < G; b += TPB) a += __ldcg(partials + q * G + b);
        v[q] = a;
    }
    block_sum<NV>(v);
}

template <int NV>
__device__ __forceinline__ void final_max(const double* partials, int G, double (&v)[NV])
{
#pragma unroll
    for (int q = 0; q < NV; ++q)
    {
        double a = 0.0;
        for (int b = threadIdx.x; b < G; b += TPB)
        {
            const double w = __ldcg(partials + q * G + b);
            a = (a < w) ? w : a;
        }
        v[q] = a;
    }
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
