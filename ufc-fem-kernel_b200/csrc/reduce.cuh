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
template <int NV>
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
#pragma unroll
  for (int k = 0; k < NV; ++k) acc[k] = 0.0;
  for (int64_t b = threadIdx.x; b < gridDim.x; b += blockDim.x)
#pragma unroll
    for (int k = 0; k < NV; ++k) acc[k] += __ldcg(partials + b * NV + k);
  block_sum<NV>(acc, sh);
  if (threadIdx.x == 0) {
#pragma unroll
    for (int k = 0; k < NV; ++k) out[k] = acc[k];
    *ticket = 0u;
  }
  return threadIdx.x == 0;
}

}  // namespace ufc
