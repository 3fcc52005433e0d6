// Deterministic block and grid reductions (warp shuffles, then shared memory,
// then one "last block" that sums the per-block partials in block order).  The
// summation order depends only on the launch shape, so results are bitwise
// reproducible run to run; no floating-point atomics are used.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace ufc {

template <int NV>
__device__ __forceinline__ void warp_sum(double (&v)[NV]) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1)
#pragma unroll
    for (int k = 0; k < NV; ++k) v[k] += __shfl_down_sync(0xffffffffu, v[k], o);
}

// Sum over the block; the result is valid in thread 0.  sh holds 32*NV doubles.
template <int NV>
__device__ __forceinline__ void block_sum(double (&v)[NV], double* sh) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
  warp_sum<NV>(v);
  __syncthreads();  // sh may still be read by a previous call
  if (lane == 0)
#pragma unroll
    for (int k = 0; k < NV; ++k) sh[w * NV + k] = v[k];
  __syncthreads();
  if (w == 0) {
#pragma unroll
    for (int k = 0; k < NV; ++k) v[k] = lane < nw ? sh[lane * NV + k] : 0.0;
    warp_sum<NV>(v);
  }
}

// Grid-wide sum: every block calls it once with its per-thread values.  Returns
// true in thread 0 of the last block to finish, whose `out` then holds the
// total; the ticket is reset for the next launch.
//
// WIDE: the last block, which runs alone, keeps eight independent loads of
// partials in flight per thread instead of one (summed in a fixed order).  It
// shortens the tail of launches with thousands of blocks, but the extra code
// also changes how the compiler schedules the caller's main loop: the fused
// SpMV of the CG is faster with it for FP32 symmetric storage and slower for
// the FP64 and full-storage kernels, as measured on B200, so the caller picks.
template <int NV, bool WIDE = false>
__device__ __forceinline__ bool grid_sum(double (&v)[NV], double* __restrict__ partials, uint32_t* ticket,
                                         double (&out)[NV]) {
  __shared__ double sh[32 * NV];
  __shared__ bool last;
  block_sum<NV>(v, sh);
  if (threadIdx.x == 0) {
#pragma unroll
    for (int k = 0; k < NV; ++k) partials[(int64_t)blockIdx.x * NV + k] = v[k];
    __threadfence();
    const uint32_t t = atomicAdd(ticket, 1u);
    last = (t == gridDim.x - 1);
  }
  __syncthreads();
  if (!last) return false;
  __threadfence();
  double acc[NV];
  if constexpr (WIDE) {
    constexpr int kU = 8;
    double part[kU][NV];
#pragma unroll
    for (int u = 0; u < kU; ++u)
#pragma unroll
      for (int k = 0; k < NV; ++k) part[u][k] = 0.0;
    const int64_t nb = gridDim.x, step = blockDim.x;
    int64_t b = threadIdx.x;
    for (; b + (kU - 1) * step < nb; b += kU * step)
#pragma unroll
      for (int u = 0; u < kU; ++u)
#pragma unroll
        for (int k = 0; k < NV; ++k) part[u][k] += __ldcg(partials + (b + u * step) * NV + k);
    for (; b < nb; b += step)
#pragma unroll
      for (int k = 0; k < NV; ++k) part[0][k] += __ldcg(partials + b * NV + k);
#pragma unroll
    for (int k = 0; k < NV; ++k) {
      acc[k] = part[0][k];
#pragma unroll
      for (int u = 1; u < kU; ++u) acc[k] += part[u][k];
    }
  } else {
#pragma unroll
    for (int k = 0; k < NV; ++k) acc[k] = 0.0;
    for (int64_t b = threadIdx.x; b < gridDim.x; b += blockDim.x)
#pragma unroll
      for (int k = 0; k < NV; ++k) acc[k] += __ldcg(partials + b * NV + k);
  }
  block_sum<NV>(acc, sh);
  if (threadIdx.x == 0) {
#pragma unroll
    for (int k = 0; k < NV; ++k) out[k] = acc[k];
    *ticket = 0u;
  }
  return threadIdx.x == 0;
}

}  // namespace ufc
