// SELL-32 SpMV and the Jacobi-preconditioned CG of NM_Solver_PCG /
// iter_pcg (ufc_core/L2_NM/Solver/NM_Solv_Core.f90:363-423,
// ufc_core/L2_NM/Solver/LinSolv/NM_Solv_IterSolver.f90:713-846).
//
// One CG iteration is three kernels:
//   k_spmv<.., kCg>   q = K p, fused p.q, alpha = r.z / p.q
//   k_cg_update       x += alpha p (x in FP64), r -= alpha q, z = D^-1 r fused,
//                     r.z and r.r, beta, the stop test and the refinement trigger
//   k_cg_pupdate      p = D^-1 r + beta p
// The scalars live in device memory (CgScalars) and every kernel returns at
// once when the run has stopped, so batches of iterations are launched as one
// CUDA graph and the host only looks at the scalars between batches.
//
// UFC_PRECISION_FP32_REFINE keeps the matrix and the CG vectors in FP32 and the
// solution in FP64.  Whenever the FP32 recursive residual has fallen by
// refine_delta since the last replacement, and whenever it meets the tolerance,
// the residual is recomputed in FP64 as r = b - K x with the FP64 element
// operator (matrix-free, K assembled from FP64 element stiffnesses) and
// replaces the recursive one (residual replacement).  The run ends when the
// FP64 residual meets the tolerance.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <utility>

#include "c3d8_device.cuh"
#include "reduce.cuh"
#include "ufc_internal.cuh"

namespace ufc {

int apply_fp64_eliminated(Ctx* c, const double* x, double* y);

namespace {

constexpr int kSpmvBlock = 256;
constexpr int kVecBlock = 256;

// Programmatic dependent launch between the kernels of a CG iteration: each
// kernel lets its successor launch as soon as all of its own blocks are
// running (launch_dependents), and waits for its predecessor's completion and
// memory (wait) before it reads anything; both are no-ops for a kernel
// launched without the attribute.
__device__ __forceinline__ void pdl_enter() {
  asm volatile("griddepcontrol.wait;" ::: "memory");
  asm volatile("griddepcontrol.launch_dependents;" :::);
}

template <typename... K, typename... A>
void launch_pdl(void (*kernel)(K...), int grid, int block, cudaStream_t st, A&&... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(grid);
  cfg.blockDim = dim3(block);
  cfg.dynamicSmemBytes = 0;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  cudaLaunchKernelEx(&cfg, kernel, std::forward<A>(args)...);
}

// The CG variants of the products (MODE kCg) run inside the iteration chain.
template <int MODE, typename... K, typename... A>
void launch_mode(void (*kernel)(K...), int grid, int block, cudaStream_t st, A&&... args) {
  if constexpr (MODE == 1)
    launch_pdl(kernel, grid, block, st, std::forward<A>(args)...);
  else
    kernel<<<grid, block, 0, st>>>(std::forward<A>(args)...);
}

// Grid of the CG vector kernels: they take 4 entries per thread (16-byte
// loads), so n / 4 threads, at most 8 blocks per SM (grid-stride beyond).
// On small meshes the kernels are bound by the launch and the grid reduction,
// which fewer blocks shorten (212k DOF: update 9.7 -> 8.8 us).
int vec_grid(int64_t n) {
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int64_t need = ((n + 3) / 4 + kVecBlock - 1) / kVecBlock;
  return (int)std::max<int64_t>(1, std::min<int64_t>(need, (int64_t)sms * 8));
}

enum SpmvMode { kPlain = 0, kCg = 1 };

// The kernels of a CG iteration do nothing once the run has stopped or asked
// for an FP64 residual replacement: a batch of iterations launched as one graph
// then idles from the triggering iteration on, so the replacement happens at
// that iteration (before its direction update) and not at the end of the batch.
__device__ __forceinline__ bool halted(const CgScalars* s) { return (s->stop | s->want_update) != 0; }

// y = K x, one thread per block row of a SELL-32 slice (a warp = a slice).
// TV: stored value type, TX: vector type, TA: accumulator type of the row sums.
// DIFF: values in difference form (diagonal slot = block row sum S_i), so the
// row is evaluated as sum_{j != i} K_ij (x_j - x_i) + S_i x_i.
template <typename TV, typename TX, typename TA, int MODE, bool DIFF>
__global__ void __launch_bounds__(kSpmvBlock)
    k_spmv(int32_t N, int64_t nrows_pad, const int64_t* __restrict__ sptr, const int32_t* __restrict__ col,
           const TV* __restrict__ val, const TX* __restrict__ x, TX* __restrict__ y, CgScalars* __restrict__ scal,
           double* __restrict__ partials) {
  pdl_enter();
  if (MODE == kCg && halted(scal)) return;
  const int64_t row = (int64_t)blockIdx.x * kSpmvBlock + threadIdx.x;
  double dot[1] = {0.0};
  if (row < nrows_pad) {
    const int64_t s = row >> 5;
    const int t = (int)(row & 31);
    const int64_t base = sptr[s];
    const int len = (int)((sptr[s + 1] - base) >> 5);
    const int32_t* cp = col + base + t;
    const TV* vp = val + 9 * base + t;
    TA a0 = TA(0), a1 = TA(0), a2 = TA(0);
    TA xi0 = TA(0), xi1 = TA(0), xi2 = TA(0);
    if (DIFF && row < N) {
      xi0 = (TA)x[3 * row];
      xi1 = (TA)x[3 * row + 1];
      xi2 = (TA)x[3 * row + 2];
    }
#pragma unroll 2
    for (int j = 0; j < len; ++j) {
      const int64_t cj = __ldcs(cp + 32 * j);
      TA x0 = (TA)__ldg(x + 3 * cj), x1 = (TA)__ldg(x + 3 * cj + 1), x2 = (TA)__ldg(x + 3 * cj + 2);
      if (DIFF && cj != row) {
        x0 -= xi0;
        x1 -= xi1;
        x2 -= xi2;
      }
      const TV* v = vp + 288 * (int64_t)j;
      a0 += (TA)__ldcs(v) * x0 + (TA)__ldcs(v + 32) * x1 + (TA)__ldcs(v + 64) * x2;
      a1 += (TA)__ldcs(v + 96) * x0 + (TA)__ldcs(v + 128) * x1 + (TA)__ldcs(v + 160) * x2;
      a2 += (TA)__ldcs(v + 192) * x0 + (TA)__ldcs(v + 224) * x1 + (TA)__ldcs(v + 256) * x2;
    }
    if (row < N) {
      y[3 * row] = (TX)a0;
      y[3 * row + 1] = (TX)a1;
      y[3 * row + 2] = (TX)a2;
      if (MODE == kCg)
        dot[0] = (double)((TA)x[3 * row] * a0 + (TA)x[3 * row + 1] * a1 + (TA)x[3 * row + 2] * a2);
    }
  }
  if (MODE == kCg) {
    double tot[1];
    if (grid_sum<1>(dot, partials, &scal->ticket[0], tot)) {
      scal->pq = tot[0];
      if (!(fabs(tot[0]) > 1e-300) || !isfinite(tot[0])) {
        scal->stop = 3;
      } else {
        scal->alpha = scal->rz / tot[0];
      }
    }
  }
}

// The same product with SPLIT (2, 4 or 8) warps per slice, for meshes with few
// slices per SM: the warps of a slice take the stored blocks j = part,
// part + SPLIT, ... of their 32 rows (every load stays a coalesced 32-row
// line) and their partial row sums are added in shared memory in warp order,
// so the result depends only on SPLIT, which the launcher derives from the
// problem size.
template <typename TV, typename TX, typename TA, int MODE, bool DIFF, int SPLIT>
__global__ void __launch_bounds__(kSpmvBlock)
    k_spmv_split(int32_t N, int64_t nslices, const int64_t* __restrict__ sptr, const int32_t* __restrict__ col,
           const TV* __restrict__ val, const TX* __restrict__ x, TX* __restrict__ y, CgScalars* __restrict__ scal,
           double* __restrict__ partials) {
  pdl_enter();
  if (MODE == kCg && halted(scal)) return;
  constexpr int kWarps = kSpmvBlock / 32;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int part = warp % SPLIT;
  const int64_t s = (int64_t)blockIdx.x * (kWarps / SPLIT) + warp / SPLIT;
  const int64_t row = s * kSlice + lane;
  TA a0 = TA(0), a1 = TA(0), a2 = TA(0);
  if (s < nslices) {
    const int64_t base = sptr[s];
    const int len = (int)((sptr[s + 1] - base) >> 5);
    const int32_t* cp = col + base + lane;
    const TV* vp = val + 9 * base + lane;
    TA xi0 = TA(0), xi1 = TA(0), xi2 = TA(0);
    if (DIFF && row < N) {
      xi0 = (TA)x[3 * row];
      xi1 = (TA)x[3 * row + 1];
      xi2 = (TA)x[3 * row + 2];
    }
    auto block = [&](int j) {
      const int64_t cj = __ldcs(cp + 32 * j);
      TA x0 = (TA)__ldg(x + 3 * cj), x1 = (TA)__ldg(x + 3 * cj + 1), x2 = (TA)__ldg(x + 3 * cj + 2);
      if (DIFF && cj != row) {
        x0 -= xi0;
        x1 -= xi1;
        x2 -= xi2;
      }
      const TV* v = vp + 288 * (int64_t)j;
      a0 += (TA)__ldcs(v) * x0 + (TA)__ldcs(v + 32) * x1 + (TA)__ldcs(v + 64) * x2;
      a1 += (TA)__ldcs(v + 96) * x0 + (TA)__ldcs(v + 128) * x1 + (TA)__ldcs(v + 160) * x2;
      a2 += (TA)__ldcs(v + 192) * x0 + (TA)__ldcs(v + 224) * x1 + (TA)__ldcs(v + 256) * x2;
    };
#pragma unroll 2
    for (int j = part; j < len; j += SPLIT) block(j);
  }
  {
    __shared__ TA sh[kWarps][3][32];
    sh[warp][0][lane] = a0;
    sh[warp][1][lane] = a1;
    sh[warp][2][lane] = a2;
    __syncthreads();
    if (part == 0) {
#pragma unroll
      for (int q = 1; q < SPLIT; ++q) {
        a0 += sh[warp + q][0][lane];
        a1 += sh[warp + q][1][lane];
        a2 += sh[warp + q][2][lane];
      }
    }
  }
  double dot[1] = {0.0};
  if (part == 0 && s < nslices && row < N) {
    y[3 * row] = (TX)a0;
    y[3 * row + 1] = (TX)a1;
    y[3 * row + 2] = (TX)a2;
    if (MODE == kCg) dot[0] = (double)((TA)x[3 * row] * a0 + (TA)x[3 * row + 1] * a1 + (TA)x[3 * row + 2] * a2);
  }
  if (MODE == kCg) {
    double tot[1];
    if (grid_sum<1>(dot, partials, &scal->ticket[0], tot)) {
      scal->pq = tot[0];
      if (!(fabs(tot[0]) > 1e-300) || !isfinite(tot[0])) {
        scal->stop = 3;
      } else {
        scal->alpha = scal->rz / tot[0];
      }
    }
  }
}

// y = K x on the full SELL storage with coded indices (see build_full_codes):
// each row loads its 32 code bytes with two 16-byte loads when the warp
// starts, and block j's column is row + off[code j], so no column index is
// loaded inside the loop.  The launcher takes it with one warp per slice
// (SPLIT = 1, as k_spmv); the SPLIT form follows k_spmv_split.  Same summation
// order as those kernels, so the same results bit for bit.
template <typename TV, typename TX, typename TA, int MODE, int SPLIT>
__global__ void __launch_bounds__(kSpmvBlock)
    k_spmvc(int32_t N, int64_t nslices, const int64_t* __restrict__ sptr, const uint4* __restrict__ code,
            FullOffsets tab, const TV* __restrict__ val, const TX* __restrict__ x, TX* __restrict__ y,
            CgScalars* __restrict__ scal, double* __restrict__ partials) {
  pdl_enter();
  if (MODE == kCg && halted(scal)) return;
  __shared__ int32_t soff[32];
  if (threadIdx.x < 32) soff[threadIdx.x] = tab.off[threadIdx.x];
  __syncthreads();
  constexpr int kWarps = kSpmvBlock / 32;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int part = warp % SPLIT;
  const int64_t s = (int64_t)blockIdx.x * (kWarps / SPLIT) + warp / SPLIT;
  const int64_t row = s * kSlice + lane;
  TA a0 = TA(0), a1 = TA(0), a2 = TA(0);
  if (s < nslices) {
    const int64_t base = sptr[s];
    const int len = (int)((sptr[s + 1] - base) >> 5);
    const uint4 c0 = __ldcs(code + 2 * row), c1 = __ldcs(code + 2 * row + 1);
    Code256 cw{c0.x | ((uint64_t)c0.y << 32), c0.z | ((uint64_t)c0.w << 32), c1.x | ((uint64_t)c1.y << 32),
               c1.z | ((uint64_t)c1.w << 32)};
    for (int q = 0; q < part; ++q) cw.template drop<1>();
    const TV* vp = val + 9 * base + lane;
#pragma unroll 2
    for (int j = part; j < len; j += SPLIT) {
      const unsigned cd = cw.front();
      cw.template drop<SPLIT>();
      TA x0 = TA(0), x1 = TA(0), x2 = TA(0);
      if (cd != 255u) {
        const int64_t cj = row + soff[cd];
        x0 = (TA)__ldg(x + 3 * cj);
        x1 = (TA)__ldg(x + 3 * cj + 1);
        x2 = (TA)__ldg(x + 3 * cj + 2);
      }
      const TV* v = vp + 288 * (int64_t)j;
      a0 += (TA)__ldcs(v) * x0 + (TA)__ldcs(v + 32) * x1 + (TA)__ldcs(v + 64) * x2;
      a1 += (TA)__ldcs(v + 96) * x0 + (TA)__ldcs(v + 128) * x1 + (TA)__ldcs(v + 160) * x2;
      a2 += (TA)__ldcs(v + 192) * x0 + (TA)__ldcs(v + 224) * x1 + (TA)__ldcs(v + 256) * x2;
    }
  }
  if constexpr (SPLIT > 1) {
    __shared__ TA sh[kWarps][3][32];
    sh[warp][0][lane] = a0;
    sh[warp][1][lane] = a1;
    sh[warp][2][lane] = a2;
    __syncthreads();
    if (part == 0) {
#pragma unroll
      for (int q = 1; q < SPLIT; ++q) {
        a0 += sh[warp + q][0][lane];
        a1 += sh[warp + q][1][lane];
        a2 += sh[warp + q][2][lane];
      }
    }
  }
  double dot[1] = {0.0};
  if (part == 0 && s < nslices && row < N) {
    y[3 * row] = (TX)a0;
    y[3 * row + 1] = (TX)a1;
    y[3 * row + 2] = (TX)a2;
    if (MODE == kCg) dot[0] = (double)((TA)x[3 * row] * a0 + (TA)x[3 * row + 1] * a1 + (TA)x[3 * row + 2] * a2);
  }
  if (MODE == kCg) {
    double tot[1];
    if (grid_sum<1>(dot, partials, &scal->ticket[0], tot)) {
      scal->pq = tot[0];
      if (!(fabs(tot[0]) > 1e-300) || !isfinite(tot[0])) {
        scal->stop = 3;
      } else {
        scal->alpha = scal->rz / tot[0];
      }
    }
  }
}

int sm_count_solver() {
  static int sms = 0;
  if (!sms) {
    int dev = 0;
    cudaGetDevice(&dev);
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || sms <= 0) sms = 148;
  }
  return sms;
}

// Warps per SELL slice: the smallest power of two (<= 8) that puts at least
// 32 warps per SM in flight.
int spmv_split(const Ctx* c) {
  const int sms = sm_count_solver();
  int split = 1;
  while (split < 8 && c->nslices * split < (int64_t)sms * 32) split <<= 1;
  return split;
}

template <typename TV, typename TX, typename TA, int MODE, bool DIFF, int SPLIT>
void launch_spmv_split(const Ctx* c, cudaStream_t st, const TV* val, const TX* x, TX* y) {
  // coded indices with FP32 values and one warp per slice only (measured on
  // B200: 192x96x96 FP32 product 297 against 325 us, FP64 582 against 568 us;
  // with SPLIT warps per slice each warp loads the row's 32 code bytes, more
  // than its share of 4-byte columns: J2 bar 53.7 against 51.8 us per CG
  // iteration)
  if (!DIFF && SPLIT == 1 && sizeof(TV) == 4 && c->full_coded) {
    constexpr int per_block = kSpmvBlock / 32 / SPLIT;
    const int grid = (int)((c->nslices + per_block - 1) / per_block);
    launch_mode<MODE>(k_spmvc<TV, TX, TA, MODE, SPLIT>, grid, kSpmvBlock, st, c->N, c->nslices, c->slice_ptr,
                      reinterpret_cast<const uint4*>(c->full_code), c->full_tab, val, x, y, c->scal, c->partials);
    return;
  }
  if constexpr (SPLIT == 1) {
    const int grid = (int)((c->nslices * kSlice + kSpmvBlock - 1) / kSpmvBlock);
    launch_mode<MODE>(k_spmv<TV, TX, TA, MODE, DIFF>, grid, kSpmvBlock, st, c->N, c->nslices * kSlice,
                      c->slice_ptr, c->sell_col, val, x, y, c->scal, c->partials);
  } else {
    constexpr int per_block = kSpmvBlock / 32 / SPLIT;
    const int grid = (int)((c->nslices + per_block - 1) / per_block);
    launch_mode<MODE>(k_spmv_split<TV, TX, TA, MODE, DIFF, SPLIT>, grid, kSpmvBlock, st, c->N, c->nslices,
                      c->slice_ptr, c->sell_col, val, x, y, c->scal, c->partials);
  }
}

template <typename TV, typename TX, typename TA, int MODE, bool DIFF>
void launch_spmv_diff(const Ctx* c, cudaStream_t st, const TV* val, const TX* x, TX* y) {
  switch (spmv_split(c)) {
    case 1: launch_spmv_split<TV, TX, TA, MODE, DIFF, 1>(c, st, val, x, y); break;
    case 2: launch_spmv_split<TV, TX, TA, MODE, DIFF, 2>(c, st, val, x, y); break;
    case 4: launch_spmv_split<TV, TX, TA, MODE, DIFF, 4>(c, st, val, x, y); break;
    default: launch_spmv_split<TV, TX, TA, MODE, DIFF, 8>(c, st, val, x, y); break;
  }
}

// SELL SpMV over the full (non-symmetric) storage; the FP32 difference form
// when the FP32 values were built that way.
template <typename TV, typename TX, typename TA, int MODE>
void launch_spmv(const Ctx* c, cudaStream_t st, const TV* val, const TX* x, TX* y) {
  if constexpr (sizeof(TV) == 4) {
    if (c->val32_diff) {
      launch_spmv_diff<TV, TX, TA, MODE, true>(c, st, val, x, y);
      return;
    }
  }
  launch_spmv_diff<TV, TX, TA, MODE, false>(c, st, val, x, y);
}

// Bulk L2 prefetch (cp.async.bulk.prefetch, the TMA unit) of the first k1
// steps of one slice's stream, issued by lane 0 when the warp starts: the upper
// values and columns of the steps below ulen and the lower positions and
// columns of those below llen, four contiguous ranges that stay inside the
// slice's own part of the arrays (their starts are multiples of 128 bytes and
// their sizes of 16).  The rest of the slice is loaded on demand: prefetching
// all of it (14 steps) overfills L2 with the resident window's streams, and a
// prefetch per loop trip costs the registers of a fifth resident block.
template <typename TV>
__device__ __forceinline__ void sym_prefetch(int lane, int k1, int ulen, int llen, const TV* uv0,
                                             const int32_t* uc0, const int32_t* lp0, const int32_t* lc0) {
  if (lane != 0) return;
  const int ku = k1 < ulen ? k1 : ulen, kl = k1 < llen ? k1 : llen;
  if (ku > 0) {
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(uv0), "r"((unsigned)(ku * 288 * (int)sizeof(TV)))
                 : "memory");
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(uc0), "r"((unsigned)(ku * 128)) : "memory");
  }
  if (kl > 0) {
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(lp0), "r"((unsigned)(kl * 128)) : "memory");
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(lc0), "r"((unsigned)(kl * 128)) : "memory");
  }
}

// y = K x from the symmetric storage: row i sums its upper blocks K_ij x_j
// (j >= i, SELL-32, coalesced) and its lower blocks as transposes K_ji^T x_j of
// the blocks stored by the earlier rows j.  Those transposed reads are from
// blocks streamed by rows at most about one node plane earlier, so they come
// from L2; the upper values are loaded with the default cache policy so that
// they stay there.
template <typename TV, typename TX, typename TA, int MODE>
__global__ void __launch_bounds__(kSpmvBlock)
    k_spmv_sym(int32_t N, int64_t nrows_pad, const int64_t* __restrict__ uptr, const int32_t* __restrict__ ucol,
               const int64_t* __restrict__ lptr, const int32_t* __restrict__ lpos, const int32_t* __restrict__ lcol,
               const TV* __restrict__ val, const TX* __restrict__ x, TX* __restrict__ y,
               CgScalars* __restrict__ scal, double* __restrict__ partials) {
  pdl_enter();
  if (MODE == kCg && halted(scal)) return;
  const int64_t row = (int64_t)blockIdx.x * kSpmvBlock + threadIdx.x;
  double dot[1] = {0.0};
  if (row < nrows_pad) {
    const int64_t s = row >> 5;
    const int t = (int)(row & 31);
    TA a0 = TA(0), a1 = TA(0), a2 = TA(0);
    const int64_t ub = uptr[s], lb = lptr[s];
    const int ulen = (int)((uptr[s + 1] - ub) >> 5);
    const int llen = (int)((lptr[s + 1] - lb) >> 5);
    const int32_t* ucp = ucol + ub + t;
    const TV* uvp = val + 9 * ub + t;
    const int32_t* lpp = lpos + lb + t;
    const int32_t* lcp = lcol + lb + t;
    // step j handles upper entry j and lower entry j, whose partners are read
    // by the owning rows at about the same step; the common part has no
    // branches so that the loads of both halves are in flight together
    auto upper = [&](int j) {
      const int64_t cj = __ldcs(ucp + 32 * j);
      const TA x0 = (TA)__ldg(x + 3 * cj), x1 = (TA)__ldg(x + 3 * cj + 1), x2 = (TA)__ldg(x + 3 * cj + 2);
      const TV* v = uvp + 288 * (int64_t)j;
      a0 += (TA)v[0] * x0 + (TA)v[32] * x1 + (TA)v[64] * x2;
      a1 += (TA)v[96] * x0 + (TA)v[128] * x1 + (TA)v[160] * x2;
      a2 += (TA)v[192] * x0 + (TA)v[224] * x1 + (TA)v[256] * x2;
    };
    auto lower = [&](int j) {
      const int64_t P = __ldcs(lpp + 32 * j);
      const int64_t cj = __ldcs(lcp + 32 * j);
      const TA x0 = (TA)__ldg(x + 3 * cj), x1 = (TA)__ldg(x + 3 * cj + 1), x2 = (TA)__ldg(x + 3 * cj + 2);
      const TV* v = val + 9 * (P & ~int64_t(31)) + (P & 31);
      // transposed block: (K_ji^T x)_r = sum_c K_ji[c][r] x_c
      a0 += (TA)__ldg(v) * x0 + (TA)__ldg(v + 96) * x1 + (TA)__ldg(v + 192) * x2;
      a1 += (TA)__ldg(v + 32) * x0 + (TA)__ldg(v + 128) * x1 + (TA)__ldg(v + 224) * x2;
      a2 += (TA)__ldg(v + 64) * x0 + (TA)__ldg(v + 160) * x1 + (TA)__ldg(v + 256) * x2;
    };
    const int mlen = ulen < llen ? ulen : llen;
    int j = 0;
    // prefetch depth in steps, measured in the CG on B200 (192x96x96): FP32
    // 8 steps (SpMV 297 -> 291 us), FP64 4 steps (516 -> 502 us)
    sym_prefetch<TV>(t, sizeof(TV) == 8 ? 4 : 8, ulen, llen, val + 9 * ub, ucol + ub, lpos + lb, lcol + lb);
    // four steps per trip for FP64 values, two for FP32 (each the faster of the
    // two on B200, measured in the CG)
    if constexpr (sizeof(TV) == 8) {
#pragma unroll 1
      for (; j + 3 < mlen; j += 4) {
        upper(j);
        lower(j);
        upper(j + 1);
        lower(j + 1);
        upper(j + 2);
        lower(j + 2);
        upper(j + 3);
        lower(j + 3);
      }
    }
#pragma unroll 1
    for (; j + 1 < mlen; j += 2) {
      upper(j);
      lower(j);
      upper(j + 1);
      lower(j + 1);
    }
    for (; j < mlen; ++j) {
      upper(j);
      lower(j);
    }
    for (int k = mlen; k < ulen; ++k) upper(k);
    for (int k = mlen; k < llen; ++k) lower(k);
    if (row < N) {
      y[3 * row] = (TX)a0;
      y[3 * row + 1] = (TX)a1;
      y[3 * row + 2] = (TX)a2;
      if (MODE == kCg)
        dot[0] = (double)((TA)x[3 * row] * a0 + (TA)x[3 * row + 1] * a1 + (TA)x[3 * row + 2] * a2);
    }
  }
  if (MODE == kCg) {
    double tot[1];
    if (grid_sum<1, sizeof(TV) == 4>(dot, partials, &scal->ticket[0], tot)) {
      scal->pq = tot[0];
      if (!(fabs(tot[0]) > 1e-300) || !isfinite(tot[0])) {
        scal->stop = 3;
      } else {
        scal->alpha = scal->rz / tot[0];
      }
    }
  }
}

// The symmetric product with coded indices (stencil-like patterns, see
// build_sym_codes): each row loads its 16 upper and 16 lower code bytes with
// two 16-byte loads when the warp starts, so the loop loads no indices at all.
// Upper step j: column row + off[code], its x gathered at once.  Lower step j:
// column row - off[code], and the block (col, row) at position
// uptr[col / 32] + 32 rank + col % 32 of the upper storage (uptr from L1):
// one dependent load (the slice start) instead of a streamed position and
// column.  Same summation order as k_spmv_sym, so the same results bit for bit.
template <typename TV, typename TX, typename TA, int MODE>
__global__ void __launch_bounds__(kSpmvBlock)
    k_spmv_symc(int32_t N, int64_t nrows_pad, const int64_t* __restrict__ uptr, const int64_t* __restrict__ lptr,
                const uint4* __restrict__ ucode, const uint4* __restrict__ lcode, SymOffsets tab,
                const TV* __restrict__ val, const TX* __restrict__ x, TX* __restrict__ y,
                CgScalars* __restrict__ scal, double* __restrict__ partials) {
  pdl_enter();
  if (MODE == kCg && halted(scal)) return;
  __shared__ int32_t soff[16];
  if (threadIdx.x < 16) soff[threadIdx.x] = tab.off[threadIdx.x];
  __syncthreads();
  double dot[1] = {0.0};
  // FP64 values: a capped grid whose warps step through the slices (measured on
  // B200, 192x96x96: 400-402 us against 453 us with one slice per warp; FP32
  // values are faster with one slice per warp, 235 against 252-275 us)
  constexpr bool kStride = sizeof(TV) == 8;
  const int64_t rstep = kStride ? (int64_t)gridDim.x * kSpmvBlock : nrows_pad;
#pragma unroll 1
  for (int64_t row = (int64_t)blockIdx.x * kSpmvBlock + threadIdx.x; row < nrows_pad; row += rstep) {
    const int64_t s = row >> 5;
    const int t = (int)(row & 31);
    TA a0 = TA(0), a1 = TA(0), a2 = TA(0);
    const int64_t ub = uptr[s];
    const int ulen = (int)((uptr[s + 1] - ub) >> 5);
    const int llen = (int)((lptr[s + 1] - lptr[s]) >> 5);
    const uint4 uc = __ldcs(ucode + row), lc = __ldcs(lcode + row);
    uint64_t ulo = uc.x | ((uint64_t)uc.y << 32), uhi = uc.z | ((uint64_t)uc.w << 32);
    uint64_t llo = lc.x | ((uint64_t)lc.y << 32), lhi = lc.z | ((uint64_t)lc.w << 32);
    const TV* uvp = val + 9 * ub + t;
    if (t == 0) {
      const int k1 = (sizeof(TV) == 8 ? 4 : 8) < ulen ? (sizeof(TV) == 8 ? 4 : 8) : ulen;
      if (k1 > 0)
        asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(val + 9 * ub),
                     "r"((unsigned)(k1 * 288 * (int)sizeof(TV)))
                     : "memory");
    }
    auto upper = [&](int j) {
      const unsigned code = (unsigned)(ulo & 0xFF);
      ulo = (ulo >> 8) | (uhi << 56);
      uhi >>= 8;
      TA x0 = TA(0), x1 = TA(0), x2 = TA(0);
      if (code != kSymCodes) {
        const int64_t cj = row + soff[code];
        x0 = (TA)__ldg(x + 3 * cj);
        x1 = (TA)__ldg(x + 3 * cj + 1);
        x2 = (TA)__ldg(x + 3 * cj + 2);
      }
      const TV* v = uvp + 288 * (int64_t)j;
      a0 += (TA)v[0] * x0 + (TA)v[32] * x1 + (TA)v[64] * x2;
      a1 += (TA)v[96] * x0 + (TA)v[128] * x1 + (TA)v[160] * x2;
      a2 += (TA)v[192] * x0 + (TA)v[224] * x1 + (TA)v[256] * x2;
    };
    auto lower = [&](int) {
      const unsigned b = (unsigned)(llo & 0xFF);
      llo = (llo >> 8) | (lhi << 56);
      lhi >>= 8;
      if (b != 0xFFu) {
        const int64_t cj = row - soff[b >> 4];
        const int64_t P = __ldg(uptr + (cj >> 5)) + 32 * (int64_t)(b & 15u) + (cj & 31);
        const TA x0 = (TA)__ldg(x + 3 * cj), x1 = (TA)__ldg(x + 3 * cj + 1), x2 = (TA)__ldg(x + 3 * cj + 2);
        const TV* v = val + 9 * (P & ~int64_t(31)) + (P & 31);
        a0 += (TA)__ldg(v) * x0 + (TA)__ldg(v + 96) * x1 + (TA)__ldg(v + 192) * x2;
        a1 += (TA)__ldg(v + 32) * x0 + (TA)__ldg(v + 128) * x1 + (TA)__ldg(v + 224) * x2;
        a2 += (TA)__ldg(v + 64) * x0 + (TA)__ldg(v + 160) * x1 + (TA)__ldg(v + 256) * x2;
      }
    };
    const int mlen = ulen < llen ? ulen : llen;
    int j = 0;
#pragma unroll 1
    for (; j + 1 < mlen; j += 2) {
      upper(j);
      lower(j);
      upper(j + 1);
      lower(j + 1);
    }
    for (; j < mlen; ++j) {
      upper(j);
      lower(j);
    }
    for (int k = mlen; k < ulen; ++k) upper(k);
    for (int k = mlen; k < llen; ++k) lower(k);
    if (row < N) {
      y[3 * row] = (TX)a0;
      y[3 * row + 1] = (TX)a1;
      y[3 * row + 2] = (TX)a2;
      if (MODE == kCg)
        dot[0] += (double)((TA)x[3 * row] * a0 + (TA)x[3 * row + 1] * a1 + (TA)x[3 * row + 2] * a2);
    }
  }
  if (MODE == kCg) {
    double tot[1];
    if (grid_sum<1, sizeof(TV) == 4>(dot, partials, &scal->ticket[0], tot)) {
      scal->pq = tot[0];
      if (!(fabs(tot[0]) > 1e-300) || !isfinite(tot[0])) {
        scal->stop = 3;
      } else {
        scal->alpha = scal->rz / tot[0];
      }
    }
  }
}

// The symmetric product with SPLIT warps per slice for meshes with too few
// slices to fill the GPU one warp each: warp `part` of a slice takes the
// upper and lower steps j = part, part + SPLIT, ..., and the row sums of the
// slice's warps are added in shared memory in warp order.
template <typename TV, typename TX, typename TA, int MODE, int SPLIT>
__global__ void __launch_bounds__(kSpmvBlock)
    k_spmv_sym_split(int32_t N, int64_t nslices, const int64_t* __restrict__ uptr, const int32_t* __restrict__ ucol,
                     const int64_t* __restrict__ lptr, const int32_t* __restrict__ lpos,
                     const int32_t* __restrict__ lcol, const TV* __restrict__ val, const TX* __restrict__ x,
                     TX* __restrict__ y, CgScalars* __restrict__ scal, double* __restrict__ partials) {
  pdl_enter();
  if (MODE == kCg && halted(scal)) return;
  constexpr int kWarps = kSpmvBlock / 32;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int part = warp % SPLIT;
  const int64_t s = (int64_t)blockIdx.x * (kWarps / SPLIT) + warp / SPLIT;
  const int64_t row = s * kSlice + lane;
  TA a0 = TA(0), a1 = TA(0), a2 = TA(0);
  if (s < nslices) {
    const int64_t ub = uptr[s], lb = lptr[s];
    const int ulen = (int)((uptr[s + 1] - ub) >> 5);
    const int llen = (int)((lptr[s + 1] - lb) >> 5);
    const int32_t* ucp = ucol + ub + lane;
    const TV* uvp = val + 9 * ub + lane;
    const int32_t* lpp = lpos + lb + lane;
    const int32_t* lcp = lcol + lb + lane;
    auto upper = [&](int j) {
      const int64_t cj = __ldcs(ucp + 32 * j);
      const TA x0 = (TA)__ldg(x + 3 * cj), x1 = (TA)__ldg(x + 3 * cj + 1), x2 = (TA)__ldg(x + 3 * cj + 2);
      const TV* v = uvp + 288 * (int64_t)j;
      a0 += (TA)v[0] * x0 + (TA)v[32] * x1 + (TA)v[64] * x2;
      a1 += (TA)v[96] * x0 + (TA)v[128] * x1 + (TA)v[160] * x2;
      a2 += (TA)v[192] * x0 + (TA)v[224] * x1 + (TA)v[256] * x2;
    };
    auto lower = [&](int j) {
      const int64_t P = __ldcs(lpp + 32 * j);
      const int64_t cj = __ldcs(lcp + 32 * j);
      const TA x0 = (TA)__ldg(x + 3 * cj), x1 = (TA)__ldg(x + 3 * cj + 1), x2 = (TA)__ldg(x + 3 * cj + 2);
      const TV* v = val + 9 * (P & ~int64_t(31)) + (P & 31);
      a0 += (TA)__ldg(v) * x0 + (TA)__ldg(v + 96) * x1 + (TA)__ldg(v + 192) * x2;
      a1 += (TA)__ldg(v + 32) * x0 + (TA)__ldg(v + 128) * x1 + (TA)__ldg(v + 224) * x2;
      a2 += (TA)__ldg(v + 64) * x0 + (TA)__ldg(v + 160) * x1 + (TA)__ldg(v + 256) * x2;
    };
    const int mlen = ulen < llen ? ulen : llen;
    int j = part;
#pragma unroll 1
    for (; j < mlen; j += SPLIT) {
      upper(j);
      lower(j);
    }
    for (int k = j; k < ulen; k += SPLIT) upper(k);
    for (int k = j; k < llen; k += SPLIT) lower(k);
  }
  {
    __shared__ TA sh[kWarps][3][32];
    sh[warp][0][lane] = a0;
    sh[warp][1][lane] = a1;
    sh[warp][2][lane] = a2;
    __syncthreads();
    if (part == 0) {
#pragma unroll
      for (int q = 1; q < SPLIT; ++q) {
        a0 += sh[warp + q][0][lane];
        a1 += sh[warp + q][1][lane];
        a2 += sh[warp + q][2][lane];
      }
    }
  }
  double dot[1] = {0.0};
  if (part == 0 && s < nslices && row < N) {
    y[3 * row] = (TX)a0;
    y[3 * row + 1] = (TX)a1;
    y[3 * row + 2] = (TX)a2;
    if (MODE == kCg) dot[0] = (double)((TA)x[3 * row] * a0 + (TA)x[3 * row + 1] * a1 + (TA)x[3 * row + 2] * a2);
  }
  if (MODE == kCg) {
    double tot[1];
    if (grid_sum<1>(dot, partials, &scal->ticket[0], tot)) {
      scal->pq = tot[0];
      if (!(fabs(tot[0]) > 1e-300) || !isfinite(tot[0])) {
        scal->stop = 3;
      } else {
        scal->alpha = scal->rz / tot[0];
      }
    }
  }
}

// 4 consecutive entries through 16-byte loads and stores (cudaMalloc bases are
// 256-byte aligned; callers pass offsets that are multiples of 4 entries).
template <typename T>
__device__ __forceinline__ void ld4(const T* __restrict__ p, T (&o)[4]) {
  if constexpr (sizeof(T) == 4) {
    const float4 v = *reinterpret_cast<const float4*>(p);
    o[0] = v.x; o[1] = v.y; o[2] = v.z; o[3] = v.w;
  } else {
    const double2 a = *reinterpret_cast<const double2*>(p), b = *reinterpret_cast<const double2*>(p + 2);
    o[0] = a.x; o[1] = a.y; o[2] = b.x; o[3] = b.y;
  }
}

template <typename T>
__device__ __forceinline__ void st4(T* __restrict__ p, const T (&o)[4]) {
  if constexpr (sizeof(T) == 4) {
    *reinterpret_cast<float4*>(p) = make_float4(o[0], o[1], o[2], o[3]);
  } else {
    *reinterpret_cast<double2*>(p) = make_double2(o[0], o[1]);
    *reinterpret_cast<double2*>(p + 2) = make_double2(o[2], o[3]);
  }
}

template <typename T>
__global__ void __launch_bounds__(kVecBlock)
    k_cg_update(int64_t n, const T* __restrict__ p, const T* __restrict__ q, T* __restrict__ r,
                double* __restrict__ x, const T* __restrict__ dinv, CgScalars* __restrict__ scal,
                double* __restrict__ partials) {
  pdl_enter();
  if (halted(scal)) return;
  const double alpha = scal->alpha;
  const T a = (T)alpha;
  T rz = T(0), rr = T(0);
  const int64_t gid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x, stride = (int64_t)gridDim.x * blockDim.x;
  const int64_t n4 = n >> 2;
  for (int64_t k = gid; k < n4; k += stride) {
    const int64_t i = k << 2;
    T pv[4], qv[4], rv[4], dv[4];
    double xv[4];
    ld4(p + i, pv);
    ld4(q + i, qv);
    ld4(r + i, rv);
    ld4(x + i, xv);
    if (dinv) ld4(dinv + i, dv);
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      xv[c] += alpha * (double)pv[c];
      rv[c] -= a * qv[c];
      const T zc = dinv ? dv[c] * rv[c] : rv[c];
      rz += rv[c] * zc;
      rr += rv[c] * rv[c];
    }
    st4(r + i, rv);
    st4(x + i, xv);
  }
  for (int64_t i = (n4 << 2) + gid; i < n; i += stride) {
    const T pi = p[i], qi = q[i];
    x[i] += alpha * (double)pi;
    const T ri = r[i] - a * qi;
    r[i] = ri;
    const T zi = dinv ? dinv[i] * ri : ri;
    rz += ri * zi;
    rr += ri * ri;
  }
  double v[2] = {(double)rz, (double)rr}, tot[2];
  if (grid_sum<2>(v, partials, &scal->ticket[1], tot)) {
    const double rz_old = scal->rz;
    scal->rz_old = rz_old;
    scal->rz = tot[0];
    scal->rr = tot[1];
    scal->beta = tot[0] / rz_old;
    const int it = scal->iter + 1;
    scal->iter = it;
    if (scal->hist && it <= scal->hist_cap) scal->hist[it - 1] = tot[1];
    if (tot[1] <= scal->tol2) scal->stop = 1;
    else if (!(fabs(rz_old) > 1e-300) || !isfinite(tot[0])) scal->stop = 3;
    else if (it >= scal->max_iter) scal->stop = 2;
    if (scal->delta2 > 0.0 && tot[1] < scal->delta2 * scal->rr_ref) scal->want_update = 1;
  }
}

template <typename T>
__global__ void __launch_bounds__(kVecBlock)
    k_cg_pupdate(int64_t n, const T* __restrict__ r, const T* __restrict__ dinv, T* __restrict__ p,
                 const CgScalars* __restrict__ scal) {
  pdl_enter();
  if (halted(scal)) return;
  const T beta = (T)scal->beta;
  // beta = 0 (start, restart after a breakdown): p = z without reading p, whose
  // contents are then undefined (fresh memory, or the NaN of the breakdown)
  const bool fresh = scal->beta == 0.0;
  const int64_t gid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x, stride = (int64_t)gridDim.x * blockDim.x;
  const int64_t n4 = n >> 2;
  for (int64_t k = gid; k < n4; k += stride) {
    const int64_t i = k << 2;
    T rv[4], pv[4] = {T(0), T(0), T(0), T(0)}, dv[4];
    ld4(r + i, rv);
    if (!fresh) ld4(p + i, pv);
    if (dinv) ld4(dinv + i, dv);
#pragma unroll
    for (int c = 0; c < 4; ++c) pv[c] = (dinv ? dv[c] * rv[c] : rv[c]) + beta * pv[c];
    st4(p + i, pv);
  }
  for (int64_t i = (n4 << 2) + gid; i < n; i += stride) {
    const T ri = r[i];
    p[i] = (dinv ? dinv[i] * ri : ri) + (fresh ? T(0) : beta * p[i]);
  }
}

// res = b - y and ||res||^2 -> scal->true_rr (and ||b||^2 -> scal->bb when asked).
__global__ void __launch_bounds__(kVecBlock)
    k_resid(int64_t n, const double* __restrict__ b, const double* y, double* res,
            CgScalars* __restrict__ scal, double* __restrict__ partials, int want_bb) {
  double rr = 0.0, bb = 0.0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const double bi = b[i];
    const double ri = bi - (y ? y[i] : 0.0);
    res[i] = ri;
    rr += ri * ri;
    bb += bi * bi;
  }
  double v[2] = {rr, bb}, tot[2];
  if (grid_sum<2>(v, partials, &scal->ticket[2], tot)) {
    scal->true_rr = tot[0];
    if (want_bb) scal->bb = tot[1];
  }
}

// Residual replacement: r := res (rounded to T), z = D^-1 r, r.z and r.r.
// mode 0: mid-run (p already updated); 1: the run stopped before its p update,
// which is then done with beta = r.z / rz_old; 2: start (beta = 0, p = z).
template <typename T>
__global__ void __launch_bounds__(kVecBlock)
    k_replace(int64_t n, const double* __restrict__ res, T* __restrict__ r, const T* __restrict__ dinv,
              CgScalars* __restrict__ scal, double* __restrict__ partials, int mode) {
  T rz = T(0), rr = T(0);
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const T ri = (T)res[i];
    r[i] = ri;
    const T zi = dinv ? dinv[i] * ri : ri;
    rz += ri * zi;
    rr += ri * ri;
  }
  double v[2] = {(double)rz, (double)rr}, tot[2];
  if (grid_sum<2>(v, partials, &scal->ticket[3], tot)) {
    if (mode == 1) scal->beta = tot[0] / scal->rz_old;
    if (mode == 2) scal->beta = 0.0;
    scal->rz = tot[0];
    scal->rr = tot[1];
    scal->rr_ref = tot[1];
    scal->stop = 0;
    scal->want_update = 0;
  }
}

struct Run {
  Ctx* c;
  int prec;  // UFC_PRECISION_*
  int64_t n;
  int vg;    // vector-kernel grid
  int sg;    // SpMV grid
};

// CG vectors of type TX over stored values of type TV; sym selects the
// symmetric SpMV storage.
template <typename TV, typename TX>
struct Vecs {
  TX *r, *p, *q;
  const TV* val;
  const TX* dinv;
  bool sym;
};

template <typename TV, typename TX>
Vecs<TV, TX> vecs(Ctx* c, bool precond) {
  Vecs<TV, TX> v;
  if constexpr (sizeof(TX) == 8) {
    v.r = c->r64; v.p = c->p64; v.q = c->q64;
    v.dinv = precond ? c->dinv64 : nullptr;
  } else {
    v.r = c->r32; v.p = c->p32; v.q = c->q32;
    v.dinv = precond ? c->dinv32 : nullptr;
  }
  if constexpr (sizeof(TV) == 8) {
    v.sym = c->has_sval64;
    v.val = v.sym ? c->sval64 : c->val64;
  } else {
    v.sym = c->has_sval32;
    v.val = v.sym ? c->sval32 : c->val32;
  }
  return v;
}

template <typename TV, typename TX, typename TA, int MODE, int SPLIT>
void launch_spmv_sym_split(const Ctx* c, cudaStream_t st, const TV* val, const TX* x, TX* y) {
  constexpr int per_block = kSpmvBlock / 32 / SPLIT;
  const int grid = (int)((c->nslices + per_block - 1) / per_block);
  launch_mode<MODE>(k_spmv_sym_split<TV, TX, TA, MODE, SPLIT>, grid, kSpmvBlock, st, c->N, c->nslices, c->uptr,
                    c->ucol, c->lptr, c->lpos, c->lcol, val, x, y, c->scal, c->partials);
}

// The symmetric product: one warp per slice (grid = slices / 8 blocks), or
// SPLIT warps per slice on small meshes (the rule of spmv_split).
template <typename TV, typename TX, typename TA, int MODE>
void launch_spmv_sym(const Ctx* c, int grid, cudaStream_t st, const TV* val, const TX* x, TX* y) {
  switch (spmv_split(c)) {
    case 1:
      if (c->sym_coded)
        launch_mode<MODE>(k_spmv_symc<TV, TX, TA, MODE>,
                          sizeof(TV) == 8 ? std::min(grid, 15 * sm_count_solver()) : grid, kSpmvBlock, st, c->N, c->nslices * kSlice, c->uptr,
                          c->lptr, reinterpret_cast<const uint4*>(c->sym_ucode),
                          reinterpret_cast<const uint4*>(c->sym_lcode), c->sym_tab, val, x, y, c->scal, c->partials);
      else
        launch_mode<MODE>(k_spmv_sym<TV, TX, TA, MODE>, grid, kSpmvBlock, st, c->N, c->nslices * kSlice, c->uptr,
                          c->ucol, c->lptr, c->lpos, c->lcol, val, x, y, c->scal, c->partials);
      break;
    case 2: launch_spmv_sym_split<TV, TX, TA, MODE, 2>(c, st, val, x, y); break;
    case 4: launch_spmv_sym_split<TV, TX, TA, MODE, 4>(c, st, val, x, y); break;
    default: launch_spmv_sym_split<TV, TX, TA, MODE, 8>(c, st, val, x, y); break;
  }
}

template <typename TV, typename TX, typename TA>
void launch_iteration(const Run& R, const Vecs<TV, TX>& V, cudaStream_t st, cudaEvent_t ev0, cudaEvent_t ev1) {
  Ctx* c = R.c;
  if (ev0) cudaEventRecord(ev0, st);
  if (V.sym)
    launch_spmv_sym<TV, TX, TA, kCg>(c, R.sg, st, V.val, V.p, V.q);
  else
    launch_spmv<TV, TX, TA, kCg>(c, st, V.val, V.p, V.q);
  if (ev1) cudaEventRecord(ev1, st);
  launch_pdl(k_cg_update<TX>, R.vg, kVecBlock, st, R.n, V.p, V.q, V.r, c->x64, V.dinv, c->scal, c->partials);
  launch_pdl(k_cg_pupdate<TX>, R.vg, kVecBlock, st, R.n, V.r, V.dinv, V.p, c->scal);
  c->launches += 3;
}

// FP64 residual of the current x64 into y64 / r-source, true_rr on the device.
// FP64 runs use their own matrix; refined FP32 runs use the matrix-free FP64
// element operator for the linear-elastic material and the assembled FP64
// values otherwise (the J2 tangent).
int true_residual(const Run& R, bool want_bb) {
  Ctx* c = R.c;
  if (R.prec == UFC_PRECISION_FP64 || c->mat_model != UFC_MAT_ELASTIC_ISO) {
    if (c->has_sval64)
      launch_spmv_sym<double, double, double, kPlain>(c, R.sg, c->stream, c->sval64, c->x64, c->y64);
    else
      launch_spmv<double, double, double, kPlain>(c, c->stream, c->val64, c->x64, c->y64);
    UFC_CUDA(c, cudaGetLastError());
    c->launches += 1;
  } else {
    UFC_TRY(apply_fp64_eliminated(c, c->x64, c->y64));
  }
  k_resid<<<R.vg, kVecBlock, 0, c->stream>>>(R.n, c->b64, c->y64, c->y64, c->scal, c->partials, want_bb ? 1 : 0);
  UFC_CUDA(c, cudaGetLastError());
  c->launches += 1;
  return UFC_STATUS_OK;
}

template <typename TV, typename TX>
int replace(const Run& R, const Vecs<TV, TX>& V, int mode) {
  Ctx* c = R.c;
  k_replace<TX><<<R.vg, kVecBlock, 0, c->stream>>>(R.n, c->y64, V.r, V.dinv, c->scal, c->partials, mode);
  UFC_CUDA(c, cudaGetLastError());
  c->launches += 1;
  if (mode != 0) {
    k_cg_pupdate<TX><<<R.vg, kVecBlock, 0, c->stream>>>(R.n, V.r, V.dinv, V.p, c->scal);
    UFC_CUDA(c, cudaGetLastError());
    c->launches += 1;
  }
  return UFC_STATUS_OK;
}

int read_scalars(Ctx* c) {
  UFC_CUDA(c, cudaMemcpyAsync(c->h_scal, c->scal, sizeof(CgScalars), cudaMemcpyDeviceToHost, c->stream));
  UFC_CUDA(c, cudaStreamSynchronize(c->stream));
  return UFC_STATUS_OK;
}

template <typename TV, typename TX, typename TA>
int get_graph(const Run& R, const Vecs<TV, TX>& V, int batch, cudaGraphExec_t* out) {
  Ctx* c = R.c;
  // one cached graph per (value, vector, accumulator) type combination
  const int slot = sizeof(TV) == 8 ? 0 : sizeof(TX) == 8 ? 3 : sizeof(TA) == 8 ? 2 : 1;
  // graphs are rebuilt when a buffer they read, the preconditioner, the storage
  // (symmetric or full), the SpMV form (FP32 difference form, coded indices)
  // or the sizes baked into their launches (DOFs, slices) change; a reassembly
  // into the same arrays keeps them.  The vector and pattern buffers are not in
  // the key: ensure_vectors, build_sym_pattern and pack_symmetric, which
  // reallocate them, release the graphs themselves.
  const void* key = (const void*)V.dinv;
  const void* val = (const void*)V.val;
  const int form = (V.sym ? 1 : 0) | (c->val32_diff ? 2 : 0) | (c->sym_coded ? 4 : 0) | (c->full_coded ? 8 : 0);
  if (c->cg_graph[slot] && c->cg_graph_batch[slot] == batch && c->cg_graph_key[slot] == key &&
      c->cg_graph_val[slot] == val && c->cg_graph_form[slot] == form && c->cg_graph_n[slot] == R.n &&
      c->cg_graph_slices[slot] == c->nslices) {
    *out = c->cg_graph[slot];
    return UFC_STATUS_OK;
  }
  if (c->cg_graph[slot]) cudaGraphExecDestroy(c->cg_graph[slot]);
  c->cg_graph[slot] = nullptr;
  cudaGraph_t g;
  const int64_t counted = c->launches;  // captured launches run only when the graph is launched
  UFC_CUDA(c, cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
  for (int k = 0; k < batch; ++k) launch_iteration<TV, TX, TA>(R, V, c->stream, nullptr, nullptr);
  cudaError_t e = cudaStreamEndCapture(c->stream, &g);
  c->launches = counted;
  if (e != cudaSuccess) return cuda_fail(c, e, "cudaStreamEndCapture");
  e = cudaGraphInstantiate(&c->cg_graph[slot], g, 0);
  cudaGraphDestroy(g);
  if (e != cudaSuccess) return cuda_fail(c, e, "cudaGraphInstantiate");
  c->cg_graph_batch[slot] = batch;
  c->cg_graph_key[slot] = key;
  c->cg_graph_val[slot] = val;
  c->cg_graph_form[slot] = form;
  c->cg_graph_n[slot] = R.n;
  c->cg_graph_slices[slot] = c->nslices;
  *out = c->cg_graph[slot];
  return UFC_STATUS_OK;
}

int ensure_vectors(Ctx* c, int prec) {
  const int64_t n = c->n;
  bool realloc = false;
  auto need = [&](auto** p) -> int {
    if (*p) return UFC_STATUS_OK;
    realloc = true;
    return dalloc(c, p, n);
  };
  UFC_TRY(need(&c->x64));
  UFC_TRY(need(&c->b64));
  UFC_TRY(need(&c->y64));
  if (prec == UFC_PRECISION_FP64 || prec == UFC_PRECISION_FP32_MATRIX) {
    UFC_TRY(need(&c->r64));
    UFC_TRY(need(&c->p64));
    UFC_TRY(need(&c->q64));
  } else {
    UFC_TRY(need(&c->r32));
    UFC_TRY(need(&c->p32));
    UFC_TRY(need(&c->q32));
  }
  if (prec != UFC_PRECISION_FP64) UFC_TRY(need(&c->xb64));
  if (realloc) release_graphs(c);
  return UFC_STATUS_OK;
}

template <typename TV, typename TX, typename TA>
int pcg_run(Ctx* c, const ufc_solver_algo* algo, ufc_solver_state* st) {
  const int prec = algo->precision_mode;
  Run R{c, prec, c->n, vec_grid(c->n), (int)((c->nslices * kSlice + kSpmvBlock - 1) / kSpmvBlock)};
  const bool precond = algo->precond_type == UFC_SOLV_PREC_JACOBI;
  Vecs<TV, TX> V = vecs<TV, TX>(c, precond);
  const int batch = algo->check_every > 0 ? algo->check_every : 32;

  cudaEvent_t t0, t1;
  UFC_CUDA(c, cudaEventCreate(&t0));
  UFC_CUDA(c, cudaEventCreate(&t1));
  UFC_CUDA(c, cudaEventRecord(t0, c->stream));
  c->timing = ufc_timing_info{};
  c->timing.precision = prec;
  c->timing.spmv_bytes = spmv_bytes(c, prec);
  c->launches = 0;

  // scalars: reset and configure
  CgScalars h{};
  h.max_iter = algo->max_iter > 0 ? algo->max_iter : 1;
  h.delta2 = 0.0;
  if (prec != UFC_PRECISION_FP64) {
    const double d = algo->refine_delta > 0.0 ? algo->refine_delta : 0.1;
    h.delta2 = d * d;
  }
  // residual history (NM_Solver_State%residual_history): one double per iteration
  const int32_t cap = std::min<int32_t>(h.max_iter, 1 << 20);
  if (c->hist_cap < cap) {
    UFC_TRY(dalloc(c, &c->hist, cap));
    c->hist_cap = cap;
  }
  h.hist = c->hist;
  h.hist_cap = c->hist_cap;
  UFC_CUDA(c, cudaMemcpyAsync(c->scal, &h, sizeof(CgScalars), cudaMemcpyHostToDevice, c->stream));
  UFC_TRY(true_residual(R, true));
  UFC_TRY(read_scalars(c));
  if (!std::isfinite(c->h_scal->bb)) return fail(c, UFC_STATUS_INVALID, "ufc_pcg_solve: non-finite right-hand side");
  if (!std::isfinite(c->h_scal->true_rr))
    return fail(c, UFC_STATUS_INVALID, "ufc_pcg_solve: non-finite initial residual (initial guess or matrix)");
  const double bnorm_raw = std::sqrt(c->h_scal->bb);
  const double bnorm = bnorm_raw < 1e-30 ? 1.0 : bnorm_raw;
  const double tol_nominal = std::max(algo->tolerance * bnorm, algo->abs_tolerance);
  const double tol = kStopMargin * tol_nominal;
  st->initial_residual = std::sqrt(c->h_scal->true_rr);
  double true_rr = c->h_scal->true_rr;
  int flag = 0;
  bool converged = std::sqrt(true_rr) <= tol;
  int n_refine = 0;

  if (!converged) {
    double tol2 = tol * tol;
    UFC_CUDA(c, cudaMemcpyAsync(&c->scal->tol2, &tol2, sizeof(double), cudaMemcpyHostToDevice, c->stream));
    UFC_TRY(replace(R, V, 2));
    cudaGraphExec_t graph = nullptr;
    if (!c->instrument) UFC_TRY((get_graph<TV, TX, TA>(R, V, batch, &graph)));
    std::vector<cudaEvent_t> evs;
    if (c->instrument) {
      evs.resize(2 * batch);
      for (auto& e : evs) UFC_CUDA(c, cudaEventCreate(&e));
    }
    CgScalars* hs[2] = {c->h_scal + 1, c->h_scal + 2};
    cudaEvent_t done[2];
    UFC_CUDA(c, cudaEventCreateWithFlags(&done[0], cudaEventDisableTiming));
    UFC_CUDA(c, cudaEventCreateWithFlags(&done[1], cudaEventDisableTiming));
    int slot = 0, in_flight = 0, iter_seen = 0;
    int stall = 0, restarts = 0;
    double best_rr = true_rr;
    constexpr int kMaxStall = 3;       // replacements without a 4x drop of ||b - K x||^2
    constexpr int kMaxRestarts = 4;    // restarts after a breakdown of the recurrence
    constexpr double kDiverge = 1e4;   // ||b - K x|| grew 100x above the best seen
    const bool keep_best = c->xb64 != nullptr;
    if (keep_best) cudaMemcpyAsync(c->xb64, c->x64, sizeof(double) * c->n, cudaMemcpyDeviceToDevice, c->stream);
    bool finished = false;
    int status = UFC_STATUS_OK;
    while (!finished) {
      if (graph) {
        cudaError_t e = cudaGraphLaunch(graph, c->stream);
        if (e != cudaSuccess) {
          status = cuda_fail(c, e, "cudaGraphLaunch");
          break;
        }
        c->launches += 3 * (int64_t)batch;
      } else {
        for (int k = 0; k < batch; ++k)
          launch_iteration<TV, TX, TA>(R, V, c->stream, evs[2 * k], evs[2 * k + 1]);
      }
      cudaMemcpyAsync(hs[slot], c->scal, sizeof(CgScalars), cudaMemcpyDeviceToHost, c->stream);
      cudaEventRecord(done[slot], c->stream);
      if (c->instrument) {
        // one batch in flight at a time: the events are reused; only the
        // launches that did an iteration (not the no-op tail) are counted
        cudaEventSynchronize(done[slot]);
        const int did = std::min(batch, hs[slot]->iter - iter_seen);
        iter_seen = hs[slot]->iter;
        for (int k = 0; k < did; ++k) {
          float ms = 0.f;
          if (cudaEventElapsedTime(&ms, evs[2 * k], evs[2 * k + 1]) == cudaSuccess) {
            c->timing.spmv_ms += ms;
            c->timing.spmv_launches += 1;
          }
        }
        in_flight = 1;
        slot ^= 1;
      }
      if (in_flight == 0) {
        in_flight = 1;
        slot ^= 1;
        continue;
      }
      const int prev = slot ^ 1;
      cudaEventSynchronize(done[prev]);
      const CgScalars* s = hs[prev];
      if (!(s->stop || s->want_update)) {
        slot ^= 1;
        continue;
      }
      // act on the latest state
      cudaEventSynchronize(done[slot]);
      in_flight = 0;
      const CgScalars cur = *hs[c->instrument ? prev : slot];
      slot = 0;
      if (cur.stop == 0 && !cur.want_update) continue;
      status = true_residual(R, false);
      if (status != UFC_STATUS_OK) break;
      status = read_scalars(c);
      if (status != UFC_STATUS_OK) break;
      true_rr = c->h_scal->true_rr;
      ++n_refine;
      if (std::sqrt(true_rr) <= tol) {
        converged = true;
        finished = true;
        break;
      }
      if (cur.stop == 2 || !std::isfinite(true_rr)) {
        flag = std::isfinite(true_rr) ? 2 : 3;
        finished = true;
        break;
      }
      // progress of the FP64 residual across replacements; the best iterate is
      // kept so that a stalled or diverging run can hand it on
      if (true_rr < best_rr) {
        if (keep_best) cudaMemcpyAsync(c->xb64, c->x64, sizeof(double) * c->n, cudaMemcpyDeviceToDevice, c->stream);
        if (true_rr < 0.25 * best_rr) stall = 0;
        else ++stall;
        best_rr = true_rr;
      } else {
        ++stall;
      }
      if (stall > kMaxStall || true_rr > kDiverge * best_rr) {
        flag = 3;
        finished = true;
        if (keep_best) {  // hand on the best iterate and its residual
          cudaMemcpyAsync(c->x64, c->xb64, sizeof(double) * c->n, cudaMemcpyDeviceToDevice, c->stream);
          true_rr = best_rr;
        }
        break;
      }
      // the iteration kernels halt right after the update that stopped the run or
      // asked for the replacement, before its direction update (mode 1)
      int mode = 1;
      if (cur.stop == 3) {
        // breakdown of the recurrence: restart CG from the FP64 residual
        if (++restarts > kMaxRestarts) {
          flag = 3;
          finished = true;
          if (keep_best) {
            cudaMemcpyAsync(c->x64, c->xb64, sizeof(double) * c->n, cudaMemcpyDeviceToDevice, c->stream);
            true_rr = best_rr;
          }
          break;
        }
        mode = 2;
      }
      if (prec != UFC_PRECISION_FP64 && algo->refine_policy == UFC_REFINE_RESTART) mode = 2;
      status = replace(R, V, mode);
      if (status != UFC_STATUS_OK) break;
    }
    for (auto& e : evs) cudaEventDestroy(e);
    cudaEventDestroy(done[0]);
    cudaEventDestroy(done[1]);
    if (status != UFC_STATUS_OK) return status;
    // stalled or out of iterations short of the margin, but within the tolerance
    if (!converged && std::isfinite(true_rr) && std::sqrt(true_rr) <= tol_nominal) {
      converged = true;
      flag = 0;
    }
  }
  UFC_TRY(read_scalars(c));
  UFC_CUDA(c, cudaEventRecord(t1, c->stream));
  UFC_CUDA(c, cudaEventSynchronize(t1));
  float ms = 0.f;
  cudaEventElapsedTime(&ms, t0, t1);
  cudaEventDestroy(t0);
  cudaEventDestroy(t1);
  c->timing.kernel_launches = c->launches;
  c->hist_len = std::min(c->h_scal->iter, c->hist_cap);
  st->niter = c->h_scal->iter;
  st->n_refine = n_refine;
  st->converged = converged ? 1 : 0;
  st->convergence_flag = converged ? 0 : (flag ? flag : 2);
  st->rnorm = std::sqrt(true_rr) / bnorm;
  st->solve_time = ms;
  UFC_TRY(check_dev_err(c, "ufc_pcg_solve"));
  return converged ? UFC_STATUS_OK : UFC_STATUS_NOT_CONVERGED;
}

}  // namespace

void release_graphs(Ctx* c) {
  for (int k = 0; k < kGraphSlots; ++k) {
    if (c->cg_graph[k]) cudaGraphExecDestroy(c->cg_graph[k]);
    c->cg_graph[k] = nullptr;
    c->cg_graph_batch[k] = 0;
    c->cg_graph_key[k] = nullptr;
    c->cg_graph_val[k] = nullptr;
    c->cg_graph_form[k] = 0;
    c->cg_graph_n[k] = c->cg_graph_slices[k] = 0;
  }
}

int64_t spmv_bytes(const Ctx* c, int precision) {
  // algorithmic bytes of one block-CSR SpMV: values + block column indices +
  // block row pointers + x read once + y written once (slice padding excluded)
  const int64_t sv = precision == UFC_PRECISION_FP64 ? 8 : 4;  // stored value
  const int64_t sx = precision == UFC_PRECISION_FP32_REFINE ? 4 : 8;  // vector entry
  const bool sym = precision == UFC_PRECISION_FP64 ? c->has_sval64 : c->has_sval32;
  if (sym) {
    const int64_t upper = (c->nnzb + c->N) / 2, lower = (c->nnzb - c->N) / 2;
    // coded indices (one-warp-per-slice form): upper values, 32 code bytes per
    // row, x and y; the lower values are re-read from L2
    if (c->sym_coded && spmv_split(c) == 1) return upper * 9 * sv + 32 * c->nslices * kSlice + 2 * c->n * sx;
    // symmetric storage: upper blocks (values + column), lower references
    // (position + column; their values are re-read from L2), x and y
    return upper * (9 * sv + 4) + lower * 8 + 2 * c->n * sx;
  }
  // coded indices: values, 32 code bytes per row, x and y
  if (c->full_coded && sv == 4 && !c->val32_diff && spmv_split(c) == 1)
    return c->nnzb * 9 * sv + 32 * c->nslices * kSlice + 2 * c->n * sx;
  return c->nnzb * (9 * sv + 4) + 4 * ((int64_t)c->N + 1) + 2 * c->n * sx;
}

int sym_grid(const Ctx* c) { return (int)((c->nslices * kSlice + kSpmvBlock - 1) / kSpmvBlock); }

// The products of the multigrid cycle and of its outer PCG take the symmetric
// storage of a level when it holds current values (the finest level of a model
// assembled with UFC_BUILD_SYMMETRIC: FP64 values and the same values rounded
// to FP32, as the cycle's own FP32 copy), else the full SELL storage.
void spmv64_on(const Ctx* lvl, cudaStream_t st, const double* x, double* y) {
  if (lvl->has_sval64)
    launch_spmv_sym<double, double, double, kPlain>(lvl, sym_grid(lvl), st, lvl->sval64, x, y);
  else
    launch_spmv<double, double, double, kPlain>(lvl, st, lvl->val64, x, y);
}

void spmv32_on(const Ctx* lvl, cudaStream_t st, const float* val, const float* x, float* y) {
  if (lvl->has_sval32)
    launch_spmv_sym<float, float, float, kPlain>(lvl, sym_grid(lvl), st, lvl->sval32, x, y);
  else
    launch_spmv_diff<float, float, float, kPlain, false>(lvl, st, val, x, y);
}

void cg_spmv64(Ctx* c, const double* p, double* q) {
  if (c->has_sval64)
    launch_spmv_sym<double, double, double, kCg>(c, sym_grid(c), c->stream, c->sval64, p, q);
  else
    launch_spmv<double, double, double, kCg>(c, c->stream, c->val64, p, q);
}

int true_residual_fp64(Ctx* c, bool want_bb) {
  spmv64_on(c, c->stream, c->x64, c->y64);
  UFC_CUDA(c, cudaGetLastError());
  k_resid<<<vec_grid(c->n), kVecBlock, 0, c->stream>>>(c->n, c->b64, c->y64, c->y64, c->scal, c->partials,
                                                       want_bb ? 1 : 0);
  UFC_CUDA(c, cudaGetLastError());
  c->launches += 2;
  return UFC_STATUS_OK;
}

int spmv(Ctx* c, int precision, const void* x, void* y) {
  if (!c->has_pattern) return fail(c, UFC_STATUS_INVALID, "ufc_spmv: pattern not built");
  const int sg = (int)((c->nslices * kSlice + kSpmvBlock - 1) / kSpmvBlock);
  if (precision == UFC_PRECISION_FP64) {
    if (!c->has_val64) return fail(c, UFC_STATUS_INVALID, "ufc_spmv: FP64 values not assembled");
    if (c->has_sval64)
      launch_spmv_sym<double, double, double, kPlain>(c, sg, c->stream, c->sval64, (const double*)x, (double*)y);
    else
      launch_spmv<double, double, double, kPlain>(c, c->stream, c->val64, (const double*)x, (double*)y);
  } else if (precision == UFC_PRECISION_FP32_REFINE) {
    if (!c->has_val32) return fail(c, UFC_STATUS_INVALID, "ufc_spmv: FP32 values not assembled");
    if (c->has_sval32)
      launch_spmv_sym<float, float, float, kPlain>(c, sg, c->stream, c->sval32, (const float*)x, (float*)y);
    else
      launch_spmv<float, float, float, kPlain>(c, c->stream, c->val32, (const float*)x, (float*)y);
  } else if (precision == UFC_PRECISION_FP32_MATRIX) {
    if (!c->has_val32) return fail(c, UFC_STATUS_INVALID, "ufc_spmv: FP32 values not assembled");
    if (c->has_sval32)
      launch_spmv_sym<float, double, double, kPlain>(c, sg, c->stream, c->sval32, (const double*)x, (double*)y);
    else
      launch_spmv<float, double, double, kPlain>(c, c->stream, c->val32, (const double*)x, (double*)y);
  } else {
    return fail(c, UFC_STATUS_INVALID, "ufc_spmv: precision");
  }
  UFC_CUDA(c, cudaGetLastError());
  return UFC_STATUS_OK;
}

// True when one FP64 product of the stored matrix reads less than half the L2.
bool fp64_fits_l2(const Ctx* c) {
  int dev = 0, l2 = 0;
  cudaGetDevice(&dev);
  if (cudaDeviceGetAttribute(&l2, cudaDevAttrL2CacheSize, dev) != cudaSuccess || l2 <= 0) return false;
  return spmv_bytes(c, UFC_PRECISION_FP64) < (int64_t)l2 / 2;
}

int pcg_solve(Ctx* c, const double* b, double* x, const ufc_solver_algo* algo, ufc_solver_state* st) {
  if (!c->has_pattern) return fail(c, UFC_STATUS_INVALID, "ufc_pcg_solve: pattern not built");
  if (algo->method != UFC_SOLV_METHOD_CG) return fail(c, UFC_STATUS_UNSUPPORTED, "ufc_pcg_solve: method must be CG");
  if (algo->precond_type != UFC_SOLV_PREC_JACOBI && algo->precond_type != UFC_SOLV_PREC_NONE &&
      algo->precond_type != UFC_SOLV_PREC_MG)
    return fail(c, UFC_STATUS_UNSUPPORTED, "ufc_pcg_solve: preconditioner must be Jacobi, multigrid or none");
  const int prec = algo->precision_mode;
  if (prec == UFC_PRECISION_FP64 && !c->has_val64)
    return fail(c, UFC_STATUS_INVALID, "ufc_pcg_solve: FP64 values not assembled (UFC_BUILD_FP64)");
  if (prec != UFC_PRECISION_FP64 && prec != UFC_PRECISION_FP32_REFINE && prec != UFC_PRECISION_FP32_MATRIX)
    return fail(c, UFC_STATUS_INVALID, "ufc_pcg_solve: precision_mode");
  if (prec != UFC_PRECISION_FP64 && !c->has_val32)
    return fail(c, UFC_STATUS_INVALID, "ufc_pcg_solve: FP32 values not assembled (UFC_BUILD_FP32*)");
  if (prec != UFC_PRECISION_FP64 && c->mat_model != UFC_MAT_ELASTIC_ISO && !c->has_val64)
    return fail(c, UFC_STATUS_INVALID,
                "ufc_pcg_solve: refined FP32 solves of a non-elastic tangent need its FP64 values for the residual "
                "(UFC_BUILD_FP64 | UFC_BUILD_FP32_ROUNDED)");
  if (prec == UFC_PRECISION_FP32_MATRIX && algo->precond_type == UFC_SOLV_PREC_JACOBI && !c->has_val64)
    return fail(c, UFC_STATUS_INVALID, "ufc_pcg_solve: FP32_MATRIX takes its Jacobi diagonal from the FP64 values");
  UFC_TRY(ensure_vectors(c, prec));
  UFC_CUDA(c, cudaMemcpyAsync(c->b64, b, sizeof(double) * c->n, cudaMemcpyDeviceToDevice, c->stream));
  if (algo->use_x0)
    UFC_CUDA(c, cudaMemcpyAsync(c->x64, x, sizeof(double) * c->n, cudaMemcpyDeviceToDevice, c->stream));
  else
    UFC_CUDA(c, cudaMemsetAsync(c->x64, 0, sizeof(double) * c->n, c->stream));
  int s;
  if (algo->precond_type == UFC_SOLV_PREC_MG) {
    if (prec != UFC_PRECISION_FP64)
      return fail(c, UFC_STATUS_UNSUPPORTED, "ufc_pcg_solve: the multigrid preconditioner runs in FP64");
    s = pcg_mg(c, algo, st);
    if (s != UFC_STATUS_OK && s != UFC_STATUS_NOT_CONVERGED) return s;
    st->fp64_iters = 0;
    UFC_CUDA(c, cudaMemcpyAsync(x, c->x64, sizeof(double) * c->n, cudaMemcpyDeviceToDevice, c->stream));
    if (s == UFC_STATUS_NOT_CONVERGED) fail(c, UFC_STATUS_NOT_CONVERGED, "[NM_Solver_PCG]: did not converge");
    return s;
  }
  if (prec == UFC_PRECISION_FP32_REFINE && algo->refine_policy != UFC_REFINE_FORCE_FP32 && c->has_val64 &&
      fp64_fits_l2(c)) {
    // a matrix this small is read from L2 in either precision: FP64 iterations
    ufc_solver_algo a64 = *algo;
    a64.precision_mode = UFC_PRECISION_FP64;
    UFC_TRY(ensure_vectors(c, UFC_PRECISION_FP64));
    s = pcg_run<double, double, double>(c, &a64, st);
    if (s != UFC_STATUS_OK && s != UFC_STATUS_NOT_CONVERGED) return s;
    st->fp64_iters = st->niter;
    UFC_CUDA(c, cudaMemcpyAsync(x, c->x64, sizeof(double) * c->n, cudaMemcpyDeviceToDevice, c->stream));
    if (s == UFC_STATUS_NOT_CONVERGED) fail(c, UFC_STATUS_NOT_CONVERGED, "[NM_Solver_PCG]: did not converge");
    return s;
  }
  if (prec == UFC_PRECISION_FP64)
    s = pcg_run<double, double, double>(c, algo, st);
  else if (prec == UFC_PRECISION_FP32_MATRIX)
    s = pcg_run<float, double, double>(c, algo, st);
  else if (algo->accumulate == UFC_ACCUMULATE_FP64)
    s = pcg_run<float, float, double>(c, algo, st);
  else
    s = pcg_run<float, float, float>(c, algo, st);
  st->fp64_iters = 0;
  if (s == UFC_STATUS_NOT_CONVERGED && prec != UFC_PRECISION_FP64 && st->convergence_flag == 3 && c->has_val64 &&
      st->niter < algo->max_iter) {
    // Stall or divergence of the refined FP32 run (the FP32 matrix is too far
    // from K for this problem): finish in FP64 from the best FP32 iterate.
    ufc_solver_algo a64 = *algo;
    a64.precision_mode = UFC_PRECISION_FP64;
    a64.max_iter = algo->max_iter - st->niter;
    ufc_solver_state s64{};
    UFC_TRY(ensure_vectors(c, UFC_PRECISION_FP64));
    s = pcg_run<double, double, double>(c, &a64, &s64);
    if (s != UFC_STATUS_OK && s != UFC_STATUS_NOT_CONVERGED) return s;
    st->fp64_iters = s64.niter;
    st->niter += s64.niter;
    st->n_refine += s64.n_refine;
    st->converged = s64.converged;
    st->convergence_flag = s64.convergence_flag;
    st->rnorm = s64.rnorm;
    st->solve_time += s64.solve_time;
  }
  if (s != UFC_STATUS_OK && s != UFC_STATUS_NOT_CONVERGED) return s;
  UFC_CUDA(c, cudaMemcpyAsync(x, c->x64, sizeof(double) * c->n, cudaMemcpyDeviceToDevice, c->stream));
  if (s == UFC_STATUS_NOT_CONVERGED)
    fail(c, UFC_STATUS_NOT_CONVERGED, "[NM_Solver_PCG]: did not converge");
  return s;
}

}  // namespace ufc
