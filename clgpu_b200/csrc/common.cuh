// Device helpers shared by the B200 iclBLAS kernels.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>

#include "internal.h"

namespace iclb {

constexpr int kWarp = 32;

// Complex product with the reference's fma placement
// (core/src/ocl/complex.h.cl:32-34): re = fma(a.re, b.re, -(a.im*b.im)),
// im = fma(a.re, b.im, a.im*b.re), the inner products rounded on their own.
__device__ __forceinline__ cfloat cmul_fma(cfloat a, cfloat b)
{
    return cfloat{fmaf(a.re, b.re, -__fmul_rn(a.im, b.im)), fmaf(a.re, b.im, __fmul_rn(a.im, b.re))};
}

__device__ __forceinline__ float4 ld_stream4(const float4* p) { return __ldcs(p); }
__device__ __forceinline__ float ld_stream(const float* p) { return __ldcs(p); }

template <class T>
__device__ __forceinline__ T warp_sum(T v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Block-wide sum in a fixed order (xor-tree within warps, then warp 0 over
// the per-warp sums).  Result valid in thread 0.  `sh` holds >= 32 values.
template <class T>
__device__ __forceinline__ T block_sum(T v, T* sh)
{
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
    v = warp_sum(v);
    __syncthreads();
    if (lane == 0) sh[wid] = v;
    __syncthreads();
    T r = T(0);
    if (wid == 0) {
        r = lane < nw ? sh[lane] : T(0);
        r = warp_sum(r);
    }
    return r;
}

// Last-block-done ticket: every block publishes its partial, fences, and
// takes a ticket; the block that draws gridDim.x-1 is last and may read all
// partials.  The last block resets the counter to zero for the next launch.
__device__ __forceinline__ bool last_block(unsigned* counter)
{
    __shared__ bool is_last;
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        unsigned t = atomicAdd(counter, 1u);
        is_last = (t == gridDim.x - 1);
    }
    __syncthreads();
    if (is_last) __threadfence();
    return is_last;
}

// As last_block, for a group of `total` blocks sharing one counter (e.g. the
// column slices of one row tile).  The caller resets the counter.
__device__ __forceinline__ bool last_block_of(unsigned* counter, unsigned total)
{
    __shared__ bool is_last;
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        unsigned t = atomicAdd(counter, 1u);
        is_last = (t == total - 1);
    }
    __syncthreads();
    if (is_last) __threadfence();
    return is_last;
}

inline int ceil_div(long a, long b) { return (int)((a + b - 1) / b); }

}  // namespace iclb
