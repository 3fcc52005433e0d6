// Multi-right-hand-side Jacobi-PCG: nrhs independent FP64 CG runs of
// NM_Solver_PCG (ufc_core/L2_NM/Solver/NM_Solv_Core.f90:363-423) that share
// every SpMV, so the matrix is read once per iteration for all of them.
//
// Vectors are interleaved, entry (dof i, rhs k) at i*nr + k with nr the number
// of right-hand sides rounded up to a power of two (<= 32; padded columns are
// zero and inactive).  A thread owns G = min(nr, 2) consecutive right-hand
// sides of one block row, so the tpr = nr/G threads of a row read the nr
// entries of one x component (nr*8 contiguous bytes, a full 128-byte line for
// 16 right-hand sides) with one 16-byte load each: every x load of a warp
// touches 32/tpr lines, each in full, which keeps the L1 wavefronts per byte
// low; the 9 values of a stored block are loaded once per thread (the lanes of
// a row share them) and the row sums stay in registers.  With 4 to 32
// right-hand sides the product (k_bspmv_pipe) streams each warp task's values,
// columns and x lines through a shared-memory ring with cp.async, so that the
// waits for memory hold no registers.  With 16 right-hand sides on a
// stencil-like pattern (coded full storage) k_bspmv_tile takes each half
// slice's x nodes into shared memory once, by bulk copies, instead.  The vector kernels
// give every thread the same G right-hand sides of successive dofs.
// Each right-hand side has its own alpha, beta and stop test; a converged
// right-hand side is frozen (alpha = beta = 0) while the others continue.
// Reductions are per right-hand side and deterministic: lanes that hold the
// same right-hand sides are combined by shuffles, then warps and blocks in a
// fixed order.  Batches of iterations run as one CUDA graph.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <vector>

#include "c3d8_device.cuh"
#include "ufc_internal.cuh"

namespace ufc {

namespace {

constexpr int kMaxRhs = 32;
constexpr int kBlk = 256;
constexpr int kWarps = kBlk / 32;
constexpr int kNvMax = 3;

struct BScalars {
  double rz[kMaxRhs], rz_old[kMaxRhs], alpha[kMaxRhs], beta[kMaxRhs], rr[kMaxRhs], tol2[kMaxRhs];
  double true_rr[kMaxRhs], bb[kMaxRhs];
  int32_t active[kMaxRhs];  // 1 while the rhs iterates
  int32_t conv[kMaxRhs];    // recursive residual met the tolerance
  int32_t iters[kMaxRhs];
  int32_t iter, max_iter, stop, nr;
  uint32_t ticket[4];
};

// G consecutive doubles (16-byte aligned when G >= 2).
template <int G>
__device__ __forceinline__ void ldg_g(const double* __restrict__ p, double (&o)[G]) {
  if constexpr (G == 1) {
    o[0] = __ldg(p);
  } else {
#pragma unroll
    for (int i = 0; i < G; i += 2) {
      const double2 v = __ldg(reinterpret_cast<const double2*>(p + i));
      o[i] = v.x;
      o[i + 1] = v.y;
    }
  }
}

template <int G>
__device__ __forceinline__ void ld_g(const double* p, double (&o)[G]) {
  if constexpr (G == 1) {
    o[0] = *p;
  } else {
#pragma unroll
    for (int i = 0; i < G; i += 2) {
      const double2 v = *reinterpret_cast<const double2*>(p + i);
      o[i] = v.x;
      o[i + 1] = v.y;
    }
  }
}

template <int G>
__device__ __forceinline__ void st_g(double* p, const double (&o)[G]) {
  if constexpr (G == 1) {
    *p = o[0];
  } else {
#pragma unroll
    for (int i = 0; i < G; i += 2) *reinterpret_cast<double2*>(p + i) = make_double2(o[i], o[i + 1]);
  }
}

// Per-rhs grid sum.  Thread t holds v[q][i] for rhs (t % tpr)*G + i; lanes with
// the same t % tpr are combined by shuffles, then the warps of the block in
// order, then the blocks in order by the last block to finish.  Returns true
// in the threads k < nr of that block, out[q] being the total of value q for
// rhs k; the ticket is reset for the next launch.  BLK = threads per block.
template <int G, int NV, int BLK = kBlk>
__device__ bool rhs_grid_sum(double (&v)[NV][G], int tpr, int nr, double* __restrict__ partials, uint32_t* ticket,
                             double (&out)[NV]) {
  constexpr int W = BLK / 32;
  __shared__ double sh[W][NV][kMaxRhs];
  __shared__ double fin[BLK * NV];
  __shared__ bool last;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  for (int o = 16; o >= tpr; o >>= 1)
#pragma unroll
    for (int q = 0; q < NV; ++q)
#pragma unroll
      for (int i = 0; i < G; ++i) v[q][i] += __shfl_down_sync(0xffffffffu, v[q][i], o);
  if (lane < tpr)
#pragma unroll
    for (int q = 0; q < NV; ++q)
#pragma unroll
      for (int i = 0; i < G; ++i) sh[w][q][lane * G + i] = v[q][i];
  __syncthreads();
  if (threadIdx.x < nr) {
#pragma unroll
    for (int q = 0; q < NV; ++q) {
      double s = 0.0;
      for (int ww = 0; ww < W; ++ww) s += sh[ww][q][threadIdx.x];
      partials[((int64_t)blockIdx.x * NV + q) * kMaxRhs + threadIdx.x] = s;
    }
  }
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) last = (atomicAdd(ticket, 1u) == gridDim.x - 1);
  __syncthreads();
  if (!last) return false;
  __threadfence();
  // last block: thread t sums the blocks b = t/nr (mod blockDim/nr) for rhs t % nr
  const int k = threadIdx.x % nr, gi = threadIdx.x / nr, groups = BLK / nr;
  double acc[NV];
#pragma unroll
  for (int q = 0; q < NV; ++q) acc[q] = 0.0;
  for (int64_t b = gi; b < gridDim.x; b += groups)
#pragma unroll
    for (int q = 0; q < NV; ++q) acc[q] += __ldcg(partials + (b * NV + q) * kMaxRhs + k);
#pragma unroll
  for (int q = 0; q < NV; ++q) fin[(gi * NV + q) * nr + k] = acc[q];
  __syncthreads();
  if (threadIdx.x < nr) {
#pragma unroll
    for (int q = 0; q < NV; ++q) {
      double s = 0.0;
      for (int g = 0; g < groups; ++g) s += fin[(g * NV + q) * nr + threadIdx.x];
      out[q] = s;
    }
    if (threadIdx.x == 0) *ticket = 0u;
    return true;
  }
  return false;
}

// y = K x for nr interleaved vectors (FP64 SELL values); MODE 1 also forms
// p.q per rhs and alpha.  One warp task = 32/tpr rows of a slice.
template <int G, int MODE>
__global__ void __launch_bounds__(kBlk, 4)
    k_bspmv(int32_t N, int64_t nslices, const int64_t* __restrict__ sptr, const int32_t* __restrict__ col,
            const double* __restrict__ val, const double* __restrict__ x, double* __restrict__ y, int nr, int tpr,
            BScalars* __restrict__ s, double* __restrict__ partials) {
  if (MODE == 1 && s->stop) return;
  const int lane = threadIdx.x & 31;
  const int rpw = 32 / tpr;
  const int rl = lane / tpr;
  const int k0 = (lane % tpr) * G;
  double dot[1][G];
#pragma unroll
  for (int i = 0; i < G; ++i) dot[0][i] = 0.0;
  const int64_t tasks = nslices * tpr;
  const int64_t wstride = ((int64_t)gridDim.x * kBlk) >> 5;
  for (int64_t task = ((int64_t)blockIdx.x * kBlk + threadIdx.x) >> 5; task < tasks; task += wstride) {
    const int64_t sl = task / tpr;
    const int t = (int)(task % tpr) * rpw + rl;
    const int64_t row = sl * kSlice + t;
    const int64_t base = sptr[sl];
    const int len = (int)((sptr[sl + 1] - base) >> 5);
    const int32_t* cp = col + base + t;
    const double* vp = val + 9 * base + t;
    double acc[3][G];
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
      for (int i = 0; i < G; ++i) acc[r][i] = 0.0;
#pragma unroll 2
    for (int j = 0; j < len; ++j) {
      const int64_t cj = __ldcs(cp + 32 * j);
      const double* v = vp + 288 * (int64_t)j;
      double m[9];
#pragma unroll
      for (int c = 0; c < 9; ++c) m[c] = __ldcs(v + 32 * c);
#pragma unroll
      for (int comp = 0; comp < 3; ++comp) {
        double xv[G];
        ldg_g<G>(x + (3 * cj + comp) * nr + k0, xv);
#pragma unroll
        for (int i = 0; i < G; ++i) {
          acc[0][i] += m[comp] * xv[i];
          acc[1][i] += m[3 + comp] * xv[i];
          acc[2][i] += m[6 + comp] * xv[i];
        }
      }
    }
    if (row < N) {
#pragma unroll
      for (int r = 0; r < 3; ++r) {
        st_g<G>(y + (3 * row + r) * nr + k0, acc[r]);
        if (MODE == 1) {
          double xr[G];
          ldg_g<G>(x + (3 * row + r) * nr + k0, xr);
#pragma unroll
          for (int i = 0; i < G; ++i) dot[0][i] += xr[i] * acc[r][i];
        }
      }
    }
  }
  if (MODE == 1) {
    double tot[1];
    if (rhs_grid_sum<G, 1>(dot, tpr, nr, partials, &s->ticket[0], tot)) {
      const int kk = threadIdx.x;
      const bool ok = s->active[kk] && fabs(tot[0]) > 1e-300 && isfinite(tot[0]);
      s->alpha[kk] = ok ? s->rz[kk] / tot[0] : 0.0;
      if (s->active[kk] && !ok) s->active[kk] = 0;  // breakdown of this rhs
    }
  }
}

// Asynchronous copies global -> shared (cp.async): the data lands in shared
// memory without occupying registers while in flight; a thread waits for its
// own groups (wait_group) and a warp barrier publishes them to the warp.
__device__ __forceinline__ void cp_async16(void* sdst, const void* gsrc) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(sdst);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(d), "l"(gsrc) : "memory");
}
__device__ __forceinline__ void cp_async16ca(void* sdst, const void* gsrc) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(sdst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 16;" ::"r"(d), "l"(gsrc) : "memory");
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// One step of a warp task in shared memory: the 9 values of the RPW rows'
// stored blocks (component-major, as in the SELL layout), shared by the warp,
// and each lane's own x entries (3 components x its 2 right-hand sides) of the
// step's column.
template <int RPW>
struct __align__(16) BStage {
  double v[9][RPW];
  double xs[32][3][2];
};

constexpr int kPipeD = 4;     // steps in flight per warp
constexpr int kPipeLMax = 32;  // columns staged per chunk of a task

template <int RPW>
constexpr size_t bpipe_smem() {
  return (size_t)kWarps * (kPipeD * sizeof(BStage<RPW>) + (size_t)kPipeLMax * RPW * sizeof(int32_t));
}

// Copies of local step jj of a chunk into a ring stage (none past the chunk);
// every call commits one group, so the group count stays the step count.
// The values of rows t0..t0+RPW-1 of step j sit at vp + 288 j + 32 c (16-byte
// aligned: slice bases are multiples of 32 entries and t0 of RPW >= 2); the
// lane's x entries at x + (3 col + comp) nr + k0 (k0 and nr even).
template <int RPW>
__device__ __forceinline__ void bstage_issue(BStage<RPW>& st, int lane, int rl, int k0, int jj, int cl,
                                             const double* vp, const int32_t (*cols)[RPW],
                                             const double* __restrict__ x, int nr) {
  if (jj < cl) {
    constexpr int kH = RPW / 2;
    const double* vs = vp + 288 * (int64_t)jj;
    for (int q = lane; q < 9 * kH; q += 32) {
      const int cc = q / kH, h = q - cc * kH;
      cp_async16(&st.v[cc][2 * h], vs + 32 * cc + 2 * h);
    }
    const int64_t cj = cols[jj][rl];
#pragma unroll
    for (int comp = 0; comp < 3; ++comp) cp_async16ca(&st.xs[lane][comp][0], x + (3 * cj + comp) * nr + k0);
  }
  cp_commit();
}

// The block SpMV of k_bspmv for G = 2 and 4..32 right-hand sides (RPW = 32 /
// tpr rows per warp task), software-pipelined through shared memory: a task's
// columns are staged first (chunks of 32 steps), then each warp keeps the
// values and its x lines of the next kPipeD steps in flight as asynchronous
// copies into a ring, so that neither the matrix stream nor the dependent x
// gathers hold registers while they wait.  The register-resident version keeps
// a step's 9 values in 18 registers per lane and its x one step ahead, which
// caps its loads in flight (latency-bound at about a fifth of the DRAM
// bandwidth).  Same products in the same order as k_bspmv, same reduction.
template <int RPW, int MODE>
__global__ void __launch_bounds__(kBlk, 3)
    k_bspmv_pipe(int32_t N, int64_t nslices, const int64_t* __restrict__ sptr, const int32_t* __restrict__ col,
                 const double* __restrict__ val, const double* __restrict__ x, double* __restrict__ y, int nr,
                 BScalars* __restrict__ s, double* __restrict__ partials) {
  constexpr int TPR = 32 / RPW;
  constexpr int D = kPipeD;
  extern __shared__ __align__(16) unsigned char bsm[];
  if (MODE == 1 && s->stop) return;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int rl = lane / TPR;
  const int k0 = (lane % TPR) * 2;
  BStage<RPW>* ring = reinterpret_cast<BStage<RPW>*>(bsm) + w * D;
  int32_t(*cols)[RPW] = reinterpret_cast<int32_t(*)[RPW]>(bsm + kWarps * D * sizeof(BStage<RPW>) +
                                                          (size_t)w * kPipeLMax * RPW * sizeof(int32_t));
  double dot[1][2] = {{0.0, 0.0}};
  const int64_t tasks = nslices * TPR;
  const int64_t wstride = ((int64_t)gridDim.x * kBlk) >> 5;
  for (int64_t task = ((int64_t)blockIdx.x * kBlk + threadIdx.x) >> 5; task < tasks; task += wstride) {
    const int64_t sl = task / TPR;
    const int t0 = (int)(task % TPR) * RPW;
    const int64_t row = sl * kSlice + t0 + rl;
    const int64_t base = sptr[sl];
    const int len = (int)((sptr[sl + 1] - base) >> 5);
    double acc[3][2] = {{0.0, 0.0}, {0.0, 0.0}, {0.0, 0.0}};
    for (int c0 = 0; c0 < len; c0 += kPipeLMax) {
      const int cl = len - c0 < kPipeLMax ? len - c0 : kPipeLMax;
      // the chunk's columns: lane l stages the RPW columns of step c0 + l
      if (lane < cl) {
        const int32_t* cs = col + base + t0 + 32 * (int64_t)(c0 + lane);
        if constexpr (RPW >= 4) {
#pragma unroll
          for (int q = 0; q < RPW / 4; ++q)
            *reinterpret_cast<int4*>(&cols[lane][4 * q]) = __ldcs(reinterpret_cast<const int4*>(cs) + q);
        } else {
          *reinterpret_cast<int2*>(&cols[lane][0]) = __ldcs(reinterpret_cast<const int2*>(cs));
        }
      }
      __syncwarp();
      const double* vp = val + 9 * (base + 32 * (int64_t)c0) + t0;
#pragma unroll
      for (int d = 0; d < D; ++d) bstage_issue<RPW>(ring[d], lane, rl, k0, d, cl, vp, cols, x, nr);
      int sidx = 0;
#pragma unroll 1
      for (int j = 0; j < cl; ++j) {
        cp_wait<D - 1>();  // this step's group has landed
        __syncwarp();
        const BStage<RPW>& S = ring[sidx];
#pragma unroll
        for (int comp = 0; comp < 3; ++comp) {
          const double2 xv = *reinterpret_cast<const double2*>(&S.xs[lane][comp][0]);
          const double m0 = S.v[comp][rl], m1 = S.v[3 + comp][rl], m2 = S.v[6 + comp][rl];
          acc[0][0] += m0 * xv.x;
          acc[0][1] += m0 * xv.y;
          acc[1][0] += m1 * xv.x;
          acc[1][1] += m1 * xv.y;
          acc[2][0] += m2 * xv.x;
          acc[2][1] += m2 * xv.y;
        }
        __syncwarp();  // every lane is done with the stage before it is refilled
        bstage_issue<RPW>(ring[sidx], lane, rl, k0, j + D, cl, vp, cols, x, nr);
        sidx = sidx + 1 == D ? 0 : sidx + 1;
      }
      cp_wait<0>();
      __syncwarp();  // the ring and the columns are free for the next chunk or task
    }
    if (row < N) {
#pragma unroll
      for (int r = 0; r < 3; ++r) {
        st_g<2>(y + (3 * row + r) * nr + k0, acc[r]);
        if (MODE == 1) {
          double xr[2];
          ldg_g<2>(x + (3 * row + r) * nr + k0, xr);
          dot[0][0] += xr[0] * acc[r][0];
          dot[0][1] += xr[1] * acc[r][1];
        }
      }
    }
  }
  if (MODE == 1) {
    double tot[1];
    if (rhs_grid_sum<2, 1>(dot, TPR, nr, partials, &s->ticket[0], tot)) {
      const int kk = threadIdx.x;
      const bool ok = s->active[kk] && fabs(tot[0]) > 1e-300 && isfinite(tot[0]);
      s->alpha[kk] = ok ? s->rz[kk] / tot[0] : 0.0;
      if (s->active[kk] && !ok) s->active[kk] = 0;  // breakdown of this rhs
    }
  }
}

// The x tile of a half slice (16 block rows) for the coded full storage: the
// union of the column ranges [row0 + off_k, row0 + off_k + 16) over the
// pattern's offsets, merged into nrange runs of nodes (run m starts at node
// row0 + a[m], has len[m] nodes and sits at node sb[m] of the shared-memory
// tile); node0[k] is the tile node of column row0 + off_k.  On a structured
// mesh the 27 offsets give 9 runs of 18 nodes, so each x line of a tile is
// read once instead of about 2.7 times.
constexpr int kTileRows = 16;
constexpr int kTileNr = 16;                        // right-hand sides (interleaved)
constexpr int kTileCons = kTileRows * kTileNr / 2;  // consumer threads: 2 rhs of one row each
constexpr int kTileBlk = kTileCons + 32;           // and one producer warp
constexpr int kTileNodeBytes = 3 * kTileNr * 8;
constexpr int kTileMaxNodes = 176;
constexpr int kValPad = 10;                        // doubles per block in the tile value layout
constexpr int kStageCodes = kTileRows * 32;        // code bytes of a tile
constexpr int kStageVals = 32 * kTileRows * kValPad * 8;  // values of up to 32 steps
struct BTile {
  int32_t nrange, nodes;
  int32_t a[kFullCodes + 1], len[kFullCodes + 1], sb[kFullCodes + 1], node0[kFullCodes + 1];
};

constexpr size_t tile_stage_bytes(int nodes) {
  return (size_t)kStageCodes + kStageVals + (size_t)nodes * kTileNodeBytes;
}

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// Bounded wait for the completion of phase `parity` of an mbarrier; false when
// it gave up (the caller records kDevTimeout).
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
  const uint32_t a = smem_u32(bar);
  for (int it = 0; it < (1 << 20); ++it) {
    uint32_t done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(a), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   smem_u32(dst)),
               "l"(src), "r"(bytes), "r"(smem_u32(bar))
               : "memory");
}

// The values of the full storage in tile order: half slice h of slice s holds
// its len steps x 16 rows x kValPad doubles (the 9 of the block, row-major by
// output component, then a zero) at 10 * sptr[s] + h * 160 * len, so that a
// tile's values are one contiguous bulk copy and a row's block is five
// 16-byte loads.
__global__ void k_tile_vals(int64_t rows, const int64_t* __restrict__ sptr, const double* __restrict__ val,
                            double* __restrict__ tv) {
  const int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= rows) return;
  const int64_t sl = r >> 5;
  const int t = (int)(r & 31);
  const int64_t base = sptr[sl];
  const int len = (int)((sptr[sl + 1] - base) >> 5);
  double* o = tv + kValPad * base + (int64_t)(t >> 4) * (16 * kValPad) * len + (t & 15) * kValPad;
  for (int j = 0; j < len; ++j) {
#pragma unroll
    for (int c = 0; c < 9; ++c) o[(int64_t)j * 16 * kValPad + c] = val[9 * (base + 32 * (int64_t)j) + 32 * c + t];
    o[(int64_t)j * 16 * kValPad + 9] = 0.0;
  }
}

// The codes in tile form: byte j of row r names the tile node of its column,
// node0[code] + r % 16 (< kTileMaxNodes), or 255 past the row's slice length
// and for rows past the mesh.
__global__ void k_tile_codes(int64_t rows, const uint8_t* __restrict__ code, const BTile T,
                             uint8_t* __restrict__ tc) {
  const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= rows * 32) return;
  const unsigned cd = code[e];
  tc[e] = cd == 255u ? (uint8_t)255 : (uint8_t)(T.node0[cd] + (int)((e >> 5) & 15));
}

// y = K x for 16 interleaved vectors from the coded full storage, one half
// slice (16 rows) per tile, the blocks resident and looping over the tiles.
// A producer warp moves each tile into one of two shared-memory stages with
// bulk copies (cp.async.bulk on an mbarrier counting bytes): the 16 rows'
// code bytes (tile form, k_tile_codes), their values (tile order,
// k_tile_vals) and the runs of x nodes the codes name (384 contiguous bytes
// per node), so that every x line of a tile crosses L2 once.  The 128
// consumer threads (8 per row, 2 rhs each) multiply from shared memory while
// the next tile lands, then release the stage; a step costs them one byte
// extract, one address and eight 16-byte shared loads besides the 18 FMAs.
// The same products in the same order as k_bspmv_pipe, so the same y.  Every
// wait is bounded; a wait that gives up sets kDevTimeout.
template <int MODE>
__global__ void __launch_bounds__(kTileBlk, 1)
    k_bspmv_tile(int32_t N, int64_t nslices, const int64_t* __restrict__ sptr, const uint8_t* __restrict__ tcode,
                 const double* __restrict__ tv, const BTile T, const double* __restrict__ x,
                 double* __restrict__ y, BScalars* __restrict__ s, double* __restrict__ partials,
                 int32_t* __restrict__ err) {
  extern __shared__ __align__(128) unsigned char tsm[];
  __shared__ __align__(8) uint64_t full[2], empty[2];
  if (MODE == 1 && s->stop) return;
  const size_t stage_bytes = tile_stage_bytes(T.nodes);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (threadIdx.x == 0) {
#pragma unroll
    for (int q = 0; q < 2; ++q) {
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&full[q])) : "memory");
      asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(&empty[q])), "r"(kTileCons / 32)
                   : "memory");
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  const int64_t tiles = nslices * 2;
  bool late = false;
  double dot[1][2] = {{0.0, 0.0}};
  if (warp == kTileCons / 32) {
    // producer: one lane issues the copies of the block's tiles in order
    if (lane == 0) {
      int k = 0;
      for (int64_t tile = blockIdx.x; tile < tiles; tile += gridDim.x, ++k) {
        const int st = k & 1;
        if (k >= 2 && !mbar_wait(&empty[st], (uint32_t)((k >> 1) - 1) & 1u)) late = true;
        unsigned char* sb = tsm + st * stage_bytes;
        const int64_t sl = tile >> 1;
        const int h = (int)(tile & 1);
        const int64_t r0 = sl * kSlice + h * kTileRows;
        const int64_t base = sptr[sl];
        const int len = (int)((sptr[sl + 1] - base) >> 5);
        const uint32_t vbytes = (uint32_t)len * (16 * kValPad * 8);
        uint32_t bytes = kStageCodes + vbytes;
        for (int m = 0; m < T.nrange; ++m) {
          const int64_t lo = max(r0 + T.a[m], (int64_t)0), hi = min(r0 + T.a[m] + T.len[m], (int64_t)N);
          if (hi > lo) bytes += (uint32_t)(hi - lo) * kTileNodeBytes;
        }
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(&full[st])),
                     "r"(bytes)
                     : "memory");
        bulk_g2s(sb, tcode + r0 * 32, kStageCodes, &full[st]);
        if (vbytes) bulk_g2s(sb + kStageCodes, tv + kValPad * base + (int64_t)h * (16 * kValPad) * len, vbytes,
                             &full[st]);
        double* xs = reinterpret_cast<double*>(sb + kStageCodes + kStageVals);
        for (int m = 0; m < T.nrange; ++m) {
          // the runs clipped to the mesh; nodes outside it are never named by a code
          const int64_t lo = max(r0 + T.a[m], (int64_t)0), hi = min(r0 + T.a[m] + T.len[m], (int64_t)N);
          if (hi > lo)
            bulk_g2s(xs + (int64_t)(T.sb[m] + (lo - (r0 + T.a[m]))) * (3 * kTileNr), x + lo * (3 * kTileNr),
                     (uint32_t)(hi - lo) * kTileNodeBytes, &full[st]);
        }
      }
    }
  } else {
    const int rl = threadIdx.x >> 3;
    const int k0 = (threadIdx.x & 7) * 2;
    int k = 0;
    for (int64_t tile = blockIdx.x; tile < tiles; tile += gridDim.x, ++k) {
      const int st = k & 1;
      const unsigned char* sb = tsm + st * stage_bytes;
      const int64_t sl = tile >> 1;
      const int64_t row = sl * kSlice + (tile & 1) * kTileRows + rl;
      const int len = (int)((sptr[sl + 1] - sptr[sl]) >> 5);
      double acc[3][2] = {{0.0, 0.0}, {0.0, 0.0}, {0.0, 0.0}};
      if (!mbar_wait(&full[st], (uint32_t)(k >> 1) & 1u)) late = true;
      const uint32_t* cw = reinterpret_cast<const uint32_t*>(sb) + rl * 8;
      const double* vs = reinterpret_cast<const double*>(sb + kStageCodes) + rl * kValPad;
      const double* xs = reinterpret_cast<const double*>(sb + kStageCodes + kStageVals) + k0;
      // rows past the mesh (last tile only) have no blocks; in a real row every
      // step below len names a block (padding blocks: the row itself, zero values)
      const int rlen = row < N ? len : 0;
      auto step = [&](unsigned nd, int j) {
        const double2* v2 = reinterpret_cast<const double2*>(vs + j * (16 * kValPad));
        double mv[10];
#pragma unroll
        for (int q = 0; q < 5; ++q) {
          const double2 w = v2[q];
          mv[2 * q] = w.x;
          mv[2 * q + 1] = w.y;
        }
        const double* xp = xs + nd * (3 * kTileNr);
#pragma unroll
        for (int comp = 0; comp < 3; ++comp) {
          const double2 xv = *reinterpret_cast<const double2*>(xp + comp * kTileNr);
          acc[0][0] += mv[comp] * xv.x;
          acc[0][1] += mv[comp] * xv.y;
          acc[1][0] += mv[3 + comp] * xv.x;
          acc[1][1] += mv[3 + comp] * xv.y;
          acc[2][0] += mv[6 + comp] * xv.x;
          acc[2][1] += mv[6 + comp] * xv.y;
        }
      };
      int j = 0;
#pragma unroll 1
      for (; j + 4 <= rlen; j += 4) {
        const uint32_t w = cw[j >> 2];
        step(w & 0xFFu, j);
        step((w >> 8) & 0xFFu, j + 1);
        step((w >> 16) & 0xFFu, j + 2);
        step(w >> 24, j + 3);
      }
      if (j < rlen) {
        const uint32_t w = cw[j >> 2];
        step(w & 0xFFu, j);
        if (j + 1 < rlen) step((w >> 8) & 0xFFu, j + 1);
        if (j + 2 < rlen) step((w >> 16) & 0xFFu, j + 2);
      }
      // the stage is free once every consumer warp has read it
      __syncwarp();
      if (lane == 0) asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(&empty[st])) : "memory");
      if (row < N) {
#pragma unroll
        for (int r = 0; r < 3; ++r) {
          st_g<2>(y + (3 * row + r) * kTileNr + k0, acc[r]);
          if (MODE == 1) {
            double xr[2];
            ldg_g<2>(x + (3 * row + r) * kTileNr + k0, xr);
            dot[0][0] += xr[0] * acc[r][0];
            dot[0][1] += xr[1] * acc[r][1];
          }
        }
      }
    }
  }
  if (late) atomicOr(err, kDevTimeout);
  if (MODE == 1) {
    double tot[1];
    if (rhs_grid_sum<2, 1, kTileBlk>(dot, kTileNr / 2, kTileNr, partials, &s->ticket[0], tot)) {
      const int kk = threadIdx.x;
      const bool ok = s->active[kk] && fabs(tot[0]) > 1e-300 && isfinite(tot[0]);
      s->alpha[kk] = ok ? s->rz[kk] / tot[0] : 0.0;
      if (s->active[kk] && !ok) s->active[kk] = 0;  // breakdown of this rhs
    }
  } else {
    __syncthreads();  // no block leaves while copies into its stages may be in flight
  }
}

// x += alpha p, r -= alpha q, then r.z and r.r per rhs, beta and the stop tests.
template <int G>
__global__ void __launch_bounds__(kBlk)
    k_bupdate(int64_t n, int nr, int tpr, const double* __restrict__ p, const double* __restrict__ q,
              double* __restrict__ r, double* __restrict__ x, const double* __restrict__ dinv,
              BScalars* __restrict__ s, double* __restrict__ partials) {
  if (s->stop) return;
  const int64_t tid = (int64_t)blockIdx.x * kBlk + threadIdx.x, stride = (int64_t)gridDim.x * kBlk;
  const int k0 = (int)(tid % tpr) * G;
  double a[G];
#pragma unroll
  for (int i = 0; i < G; ++i) a[i] = s->alpha[k0 + i];
  double v[2][G];
#pragma unroll
  for (int i = 0; i < G; ++i) v[0][i] = v[1][i] = 0.0;
  const int64_t groups = n * tpr;
  for (int64_t idx = tid; idx < groups; idx += stride) {
    const int64_t e = idx * G;
    const double d = dinv ? __ldg(dinv + idx / tpr) : 1.0;
    double pv[G], qv[G], rv[G], xv[G];
    ldg_g<G>(p + e, pv);
    ldg_g<G>(q + e, qv);
    ld_g<G>(r + e, rv);
    ld_g<G>(x + e, xv);
#pragma unroll
    for (int i = 0; i < G; ++i) {
      xv[i] += a[i] * pv[i];
      rv[i] -= a[i] * qv[i];
      v[0][i] += rv[i] * (d * rv[i]);
      v[1][i] += rv[i] * rv[i];
    }
    st_g<G>(r + e, rv);
    st_g<G>(x + e, xv);
  }
  double tot[2];
  if (rhs_grid_sum<G, 2>(v, tpr, nr, partials, &s->ticket[1], tot)) {
    const int kk = threadIdx.x;
    if (s->active[kk]) {
      s->rz_old[kk] = s->rz[kk];
      s->beta[kk] = tot[0] / s->rz[kk];
      s->rz[kk] = tot[0];
      s->rr[kk] = tot[1];
      s->iters[kk] += 1;
      if (tot[1] <= s->tol2[kk]) {
        s->conv[kk] = 1;
        s->active[kk] = 0;
      }
    } else {
      s->beta[kk] = 0.0;
    }
    __syncwarp(s->nr >= 32 ? 0xffffffffu : ((1u << s->nr) - 1u));
    if (kk == 0) {
      int any = 0;
      for (int i = 0; i < s->nr; ++i) any |= s->active[i];
      const int it = s->iter + 1;
      s->iter = it;
      if (!any) s->stop = 1;
      else if (it >= s->max_iter) s->stop = 2;
    }
  }
}

// p = D^-1 r + beta p for the rhs still active.
template <int G>
__global__ void __launch_bounds__(kBlk)
    k_bpupdate(int64_t n, int nr, int tpr, const double* __restrict__ r, const double* __restrict__ dinv,
               double* __restrict__ p, const BScalars* __restrict__ s) {
  if (s->stop) return;
  const int64_t tid = (int64_t)blockIdx.x * kBlk + threadIdx.x, stride = (int64_t)gridDim.x * kBlk;
  const int k0 = (int)(tid % tpr) * G;
  double b[G];
  bool act[G], any = false;
#pragma unroll
  for (int i = 0; i < G; ++i) {
    b[i] = s->beta[k0 + i];
    act[i] = s->active[k0 + i] != 0;
    any |= act[i];
  }
  if (!any) return;
  const int64_t groups = n * tpr;
  for (int64_t idx = tid; idx < groups; idx += stride) {
    const int64_t e = idx * G;
    const double d = dinv ? __ldg(dinv + idx / tpr) : 1.0;
    double rv[G], pv[G];
    ldg_g<G>(r + e, rv);
    ld_g<G>(p + e, pv);
#pragma unroll
    for (int i = 0; i < G; ++i)
      if (act[i]) pv[i] = d * rv[i] + b[i] * pv[i];
    st_g<G>(p + e, pv);
  }
}

// r = b - y with ||r||^2, ||b||^2 and r.z per rhs (the state a restart needs).
template <int G>
__global__ void __launch_bounds__(kBlk)
    k_bresid(int64_t n, int nr, int tpr, const double* __restrict__ bv, const double* __restrict__ y,
             double* __restrict__ r, const double* __restrict__ dinv, BScalars* __restrict__ s,
             double* __restrict__ partials) {
  const int64_t tid = (int64_t)blockIdx.x * kBlk + threadIdx.x, stride = (int64_t)gridDim.x * kBlk;
  double v[3][G];
#pragma unroll
  for (int i = 0; i < G; ++i) v[0][i] = v[1][i] = v[2][i] = 0.0;
  const int64_t groups = n * tpr;
  for (int64_t idx = tid; idx < groups; idx += stride) {
    const int64_t e = idx * G;
    const double d = dinv ? __ldg(dinv + idx / tpr) : 1.0;
    double be[G], ye[G], re[G];
    ldg_g<G>(bv + e, be);
    ldg_g<G>(y + e, ye);
#pragma unroll
    for (int i = 0; i < G; ++i) {
      re[i] = be[i] - ye[i];
      v[0][i] += re[i] * re[i];
      v[1][i] += be[i] * be[i];
      v[2][i] += re[i] * (d * re[i]);
    }
    st_g<G>(r + e, re);
  }
  double tot[3];
  if (rhs_grid_sum<G, 3>(v, tpr, nr, partials, &s->ticket[2], tot)) {
    const int kk = threadIdx.x;
    s->true_rr[kk] = tot[0];
    s->bb[kk] = tot[1];
    s->rz[kk] = tot[2];
  }
}

// p = D^-1 r for the rhs that (re)start.
__global__ void k_bpinit(int64_t nn, int nr, const double* __restrict__ r, const double* __restrict__ dinv,
                         double* __restrict__ p, const int32_t* __restrict__ restart) {
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < nn; e += (int64_t)gridDim.x * blockDim.x) {
    const int k = (int)(e % nr);
    if (restart[k]) p[e] = dinv ? dinv[e / nr] * r[e] : r[e];
  }
}

// [nrhs][n] <-> [n][nr] (padding columns zero)
__global__ void k_interleave(int64_t n, int nrhs, int nr, const double* __restrict__ a, double* __restrict__ b) {
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < n * nr; e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = e / nr;
    const int k = (int)(e % nr);
    b[e] = k < nrhs ? a[(int64_t)k * n + i] : 0.0;
  }
}

__global__ void k_deinterleave(int64_t n, int nrhs, int nr, const double* __restrict__ a, double* __restrict__ b) {
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < n * nrhs; e += (int64_t)gridDim.x * blockDim.x) {
    const int k = (int)(e / n);
    const int64_t i = e % n;
    b[e] = a[i * nr + k];
  }
}

int sm_count() {
  static int sms = 0;
  if (!sms) {
    int dev = 0;
    cudaGetDevice(&dev);
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || sms <= 0) sms = 148;
  }
  return sms;
}

// blocks for `threads` grid-stride threads, at most 8 per SM
int grid_blocks(int64_t threads) {
  return (int)std::max<int64_t>(1, std::min<int64_t>((threads + kBlk - 1) / kBlk, (int64_t)sm_count() * 8));
}

struct BlockRun {
  Ctx* c;
  int nr, tpr;
  int64_t n, nn;
  const double* dinv;
  double *bx, *xx, *rx, *px, *qx;
  BScalars* s;
  double* partials;
  int g_spmv, g_vec;
  bool tile;  // k_bspmv_tile (16 rhs, coded full storage)
  BTile T;
  int g_tile;
  double* tv;   // values in tile order (k_tile_vals)
  uint8_t* tc;  // codes in tile form (k_tile_codes)
};

// The tile of k_bspmv_tile from the offsets of the coded storage (ascending);
// false when the pattern's tile would not fit three blocks per SM.
bool make_tile(const Ctx* c, BTile* T) {
  *T = BTile{};
  if (!c->full_coded || c->full_ntab <= 0) return false;
  int m = -1;
  std::vector<int> run(c->full_ntab);
  for (int k = 0; k < c->full_ntab; ++k) {
    const int a = c->full_tab.off[k];
    if (m >= 0 && a <= T->a[m] + T->len[m]) {
      T->len[m] = std::max(T->len[m], a + kTileRows - T->a[m]);
    } else {
      ++m;
      T->a[m] = a;
      T->len[m] = kTileRows;
    }
    run[k] = m;
  }
  T->nrange = m + 1;
  int nodes = 0;
  for (int q = 0; q < T->nrange; ++q) {
    T->sb[q] = nodes;
    nodes += T->len[q];
  }
  T->nodes = nodes;
  for (int k = 0; k < c->full_ntab; ++k) T->node0[k] = T->sb[run[k]] + (c->full_tab.off[k] - T->a[run[k]]);
  return nodes <= kTileMaxNodes;
}

void launch_bspmv_tile(const BlockRun& B, cudaStream_t st, int mode, const double* x, double* y) {
  Ctx* c = B.c;
  const size_t sm = 2 * tile_stage_bytes(B.T.nodes);
  if (mode == 1)
    k_bspmv_tile<1><<<B.g_tile, kTileBlk, sm, st>>>(c->N, c->nslices, c->slice_ptr, B.tc, B.tv, B.T, x, y, B.s,
                                                    B.partials, c->dev_err);
  else
    k_bspmv_tile<0><<<B.g_tile, kTileBlk, sm, st>>>(c->N, c->nslices, c->slice_ptr, B.tc, B.tv, B.T, x, y, B.s,
                                                    B.partials, c->dev_err);
}

cudaError_t prepare_tile(const BTile& T) {
  const int sm = (int)(2 * tile_stage_bytes(T.nodes));
  cudaError_t e = cudaFuncSetAttribute(k_bspmv_tile<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm);
  if (e == cudaSuccess) e = cudaFuncSetAttribute(k_bspmv_tile<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm);
  return e;
}

template <int RPW>
void launch_bspmv_pipe(const BlockRun& B, cudaStream_t st, int mode, const double* x, double* y) {
  Ctx* c = B.c;
  constexpr size_t sm = bpipe_smem<RPW>();
  if (mode == 1)
    k_bspmv_pipe<RPW, 1><<<B.g_spmv, kBlk, sm, st>>>(c->N, c->nslices, c->slice_ptr, c->sell_col, c->val64, x, y,
                                                      B.nr, B.s, B.partials);
  else
    k_bspmv_pipe<RPW, 0><<<B.g_spmv, kBlk, sm, st>>>(c->N, c->nslices, c->slice_ptr, c->sell_col, c->val64, x, y,
                                                      B.nr, B.s, B.partials);
}

// The pipelined kernels use more than the default 48 KB of dynamic shared
// memory; the limit is raised for the current device before any launch (and
// before any graph capture).
template <int RPW>
cudaError_t bpipe_attr() {
  constexpr int sm = (int)bpipe_smem<RPW>();
  cudaError_t e = cudaFuncSetAttribute(k_bspmv_pipe<RPW, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k_bspmv_pipe<RPW, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm);
  return e;
}

cudaError_t prepare_bspmv(int tpr) {
  switch (tpr) {
    case 2: return bpipe_attr<16>();
    case 4: return bpipe_attr<8>();
    case 8: return bpipe_attr<4>();
    case 16: return bpipe_attr<2>();
    default: return cudaSuccess;
  }
}

template <int G>
void launch_bspmv(const BlockRun& B, cudaStream_t st, int mode, const double* x, double* y) {
  Ctx* c = B.c;
  if constexpr (G == 2) {
    if (B.tile) {
      launch_bspmv_tile(B, st, mode, x, y);
      return;
    }
    // 4..32 right-hand sides: the pipelined kernel (rows per warp task = 32 / tpr)
    switch (B.tpr) {
      case 2: launch_bspmv_pipe<16>(B, st, mode, x, y); return;
      case 4: launch_bspmv_pipe<8>(B, st, mode, x, y); return;
      case 8: launch_bspmv_pipe<4>(B, st, mode, x, y); return;
      case 16: launch_bspmv_pipe<2>(B, st, mode, x, y); return;
      default: break;
    }
  }
  if (mode == 1)
    k_bspmv<G, 1><<<B.g_spmv, kBlk, 0, st>>>(c->N, c->nslices, c->slice_ptr, c->sell_col, c->val64, x, y, B.nr,
                                              B.tpr, B.s, B.partials);
  else
    k_bspmv<G, 0><<<B.g_spmv, kBlk, 0, st>>>(c->N, c->nslices, c->slice_ptr, c->sell_col, c->val64, x, y, B.nr,
                                              B.tpr, B.s, B.partials);
}

template <int G>
void launch_biteration(const BlockRun& B, cudaStream_t st) {
  launch_bspmv<G>(B, st, 1, B.px, B.qx);
  k_bupdate<G><<<B.g_vec, kBlk, 0, st>>>(B.n, B.nr, B.tpr, B.px, B.qx, B.rx, B.xx, B.dinv, B.s, B.partials);
  k_bpupdate<G><<<B.g_vec, kBlk, 0, st>>>(B.n, B.nr, B.tpr, B.rx, B.dinv, B.px, B.s);
}

template <int G>
void launch_bresidual(const BlockRun& B, cudaStream_t st) {
  launch_bspmv<G>(B, st, 0, B.xx, B.qx);
  k_bresid<G><<<B.g_vec, kBlk, 0, st>>>(B.n, B.nr, B.tpr, B.bx, B.qx, B.rx, B.dinv, B.s, B.partials);
}

}  // namespace

template <int G>
static int pcg_block_run(BlockRun& B, int nrhs, const ufc_solver_algo* algo, BScalars* hs, int32_t* restart_dev,
                         std::vector<double>& bnorm, std::vector<double>& tol, std::vector<int>& n_refine,
                         ufc_solver_state* st) {
  Ctx* c = B.c;
  const int nr = B.nr;
  auto residual = [&]() -> int {
    launch_bresidual<G>(B, c->stream);
    UFC_CUDA(c, cudaGetLastError());
    c->launches += 2;
    UFC_CUDA(c, cudaMemcpyAsync(hs, B.s, sizeof(BScalars), cudaMemcpyDeviceToHost, c->stream));
    UFC_CUDA(c, cudaStreamSynchronize(c->stream));
    return UFC_STATUS_OK;
  };
  UFC_TRY(residual());
  for (int k = 0; k < nrhs; ++k) {
    if (!std::isfinite(hs->bb[k]))
      return fail(c, UFC_STATUS_INVALID, "ufc_pcg_solve_block: non-finite right-hand side " + std::to_string(k));
    if (!std::isfinite(hs->true_rr[k]))
      return fail(c, UFC_STATUS_INVALID,
                  "ufc_pcg_solve_block: non-finite initial residual of right-hand side " + std::to_string(k));
  }
  for (int k = 0; k < nr; ++k) {
    const double bn = std::sqrt(hs->bb[k]);
    bnorm[k] = bn < 1e-30 ? 1.0 : bn;
    tol[k] = std::max(algo->tolerance * bnorm[k], algo->abs_tolerance);
    if (k < nrhs) st[k].initial_residual = std::sqrt(hs->true_rr[k]);
  }
  const int batch = algo->check_every > 0 ? algo->check_every : 32;
  // one graph of `batch` iterations, launched until every rhs stops
  cudaGraph_t g = nullptr;
  cudaGraphExec_t ge = nullptr;
  UFC_CUDA(c, cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
  for (int b = 0; b < batch; ++b) launch_biteration<G>(B, c->stream);
  cudaError_t e = cudaStreamEndCapture(c->stream, &g);
  if (e != cudaSuccess) return cuda_fail(c, e, "cudaStreamEndCapture");
  e = cudaGraphInstantiate(&ge, g, 0);
  cudaGraphDestroy(g);
  if (e != cudaSuccess) return cuda_fail(c, e, "cudaGraphInstantiate");
  BScalars h{};
  std::vector<int32_t> restart(kMaxRhs, 0);
  int total_iter = 0, status = UFC_STATUS_OK;
  for (int round = 0; round < 64 && status == UFC_STATUS_OK; ++round) {
    // (re)start every rhs whose FP64 residual is above its tolerance
    bool any = false;
    for (int k = 0; k < nr; ++k) {
      const bool ok = k >= nrhs || std::sqrt(hs->true_rr[k]) <= tol[k];
      restart[k] = ok ? 0 : 1;
      any |= !ok;
      h.tol2[k] = tol[k] * tol[k];
      h.active[k] = restart[k];
      h.conv[k] = 0;
      h.rz[k] = hs->rz[k];
      h.iters[k] = hs->iters[k];
    }
    if (!any || total_iter >= algo->max_iter) break;
    h.iter = 0;
    h.stop = 0;
    h.max_iter = algo->max_iter - total_iter;
    h.nr = nr;
    for (int q = 0; q < 4; ++q) h.ticket[q] = 0;
    cudaMemcpyAsync(B.s, &h, sizeof(BScalars), cudaMemcpyHostToDevice, c->stream);
    cudaMemcpyAsync(restart_dev, restart.data(), sizeof(int32_t) * kMaxRhs, cudaMemcpyHostToDevice, c->stream);
    k_bpinit<<<grid_blocks(B.nn), kBlk, 0, c->stream>>>(B.nn, nr, B.rx, B.dinv, B.px, restart_dev);
    c->launches += 1;
    for (;;) {
      e = cudaGraphLaunch(ge, c->stream);
      if (e != cudaSuccess) {
        status = cuda_fail(c, e, "cudaGraphLaunch");
        break;
      }
      c->launches += 3 * (int64_t)batch;
      cudaMemcpyAsync(hs, B.s, sizeof(BScalars), cudaMemcpyDeviceToHost, c->stream);
      e = cudaStreamSynchronize(c->stream);
      if (e != cudaSuccess) {
        status = cuda_fail(c, e, "ufc_pcg_solve_block");
        break;
      }
      if (hs->stop) break;
    }
    if (status != UFC_STATUS_OK) break;
    total_iter += hs->iter;
    const int stop = hs->stop;
    // FP64 true residual of every rhs (residual replacement)
    const std::vector<int32_t> iters_keep(hs->iters, hs->iters + kMaxRhs);
    status = residual();
    if (status != UFC_STATUS_OK) break;
    for (int k = 0; k < nr; ++k) {
      hs->iters[k] = iters_keep[k];
      ++n_refine[k];
    }
    if (stop == 2) break;
  }
  cudaGraphExecDestroy(ge);
  return status;
}

int pcg_solve_block(Ctx* c, int nrhs, const double* Bm, double* X, const ufc_solver_algo* algo,
                    ufc_solver_state* st) {
  if (!c->has_pattern) return fail(c, UFC_STATUS_INVALID, "ufc_pcg_solve_block: pattern not built");
  if (nrhs < 1 || nrhs > kMaxRhs) return fail(c, UFC_STATUS_INVALID, "ufc_pcg_solve_block: nrhs must be 1..32");
  if (algo->precision_mode != UFC_PRECISION_FP64)
    return fail(c, UFC_STATUS_UNSUPPORTED, "ufc_pcg_solve_block: FP64 only");
  if (!c->has_val64) return fail(c, UFC_STATUS_INVALID, "ufc_pcg_solve_block: FP64 values not assembled");
  if (algo->method != UFC_SOLV_METHOD_CG || algo->max_iter <= 0)
    return fail(c, UFC_STATUS_INVALID, "ufc_pcg_solve_block: method must be CG and max_iter > 0");
  int nr = 1;
  while (nr < nrhs) nr <<= 1;
  const int G = std::min(nr, 2);
  BlockRun B{};
  B.c = c;
  B.nr = nr;
  B.tpr = nr / G;
  B.n = c->n;
  B.nn = c->n * nr;
  B.dinv = algo->precond_type == UFC_SOLV_PREC_JACOBI ? c->dinv64 : nullptr;
  B.g_spmv = grid_blocks(c->nslices * B.tpr * 32);
  if (G == 2) UFC_CUDA(c, prepare_bspmv(B.tpr));
  B.tile = nr == kTileNr && make_tile(c, &B.T);
  B.g_tile = (int)std::min<int64_t>(2 * c->nslices, (int64_t)sm_count());
  if (B.tile) UFC_CUDA(c, prepare_tile(B.T));
  B.g_vec = grid_blocks(c->n * B.tpr);
  BScalars* hs = nullptr;
  int32_t* restart_dev = nullptr;
  auto cleanup = [&]() {
    dfree(&B.bx); dfree(&B.xx); dfree(&B.rx); dfree(&B.px); dfree(&B.qx); dfree(&B.s); dfree(&B.partials);
    dfree(&B.tv); dfree(&B.tc);
    dfree(&restart_dev);
    if (hs) cudaFreeHost(hs);
    hs = nullptr;
  };
  int status = UFC_STATUS_OK;
#define BTRY(expr)            \
  do {                        \
    status = (expr);          \
    if (status != UFC_STATUS_OK) { cleanup(); return status; } \
  } while (0)
#define BCUDA(expr)                                                   \
  do {                                                                \
    cudaError_t _e = (expr);                                          \
    if (_e != cudaSuccess) { cleanup(); return cuda_fail(c, _e, #expr); } \
  } while (0)
  BTRY(dalloc(c, &B.bx, B.nn));
  BTRY(dalloc(c, &B.xx, B.nn));
  BTRY(dalloc(c, &B.rx, B.nn));
  BTRY(dalloc(c, &B.px, B.nn));
  // columns that never restart (padding, or converged at the start) are
  // multiplied by alpha = 0: they must hold numbers, not whatever was there
  BCUDA(cudaMemsetAsync(B.px, 0, sizeof(double) * B.nn, c->stream));
  BTRY(dalloc(c, &B.qx, B.nn));
  BTRY(dalloc(c, &B.s, 1));
  BTRY(dalloc(c, &B.partials, (int64_t)std::max({B.g_spmv, B.g_vec, B.g_tile}) * kNvMax * kMaxRhs));
  BTRY(dalloc(c, &restart_dev, kMaxRhs));
  if (B.tile) {
    BTRY(dalloc(c, &B.tv, kValPad * c->sell_blocks));
    const int64_t rows = c->nslices * kSlice;
    k_tile_vals<<<(int)((rows + 255) / 256), 256, 0, c->stream>>>(rows, c->slice_ptr, c->val64, B.tv);
    BCUDA(cudaGetLastError());
    BTRY(dalloc(c, &B.tc, rows * 32));
    k_tile_codes<<<(int)((rows * 32 + 255) / 256), 256, 0, c->stream>>>(rows, c->full_code, B.T, B.tc);
    BCUDA(cudaGetLastError());
  }
  BCUDA(cudaMallocHost((void**)&hs, sizeof(BScalars)));
  cudaEvent_t t0, t1;
  BCUDA(cudaEventCreate(&t0));
  BCUDA(cudaEventCreate(&t1));
  BCUDA(cudaEventRecord(t0, c->stream));
  c->launches = 0;

  const int gi = grid_blocks(B.nn);
  k_interleave<<<gi, kBlk, 0, c->stream>>>(c->n, nrhs, nr, Bm, B.bx);
  if (algo->use_x0)
    k_interleave<<<gi, kBlk, 0, c->stream>>>(c->n, nrhs, nr, X, B.xx);
  else
    BCUDA(cudaMemsetAsync(B.xx, 0, sizeof(double) * B.nn, c->stream));
  BScalars h{};
  h.nr = nr;
  h.max_iter = algo->max_iter;
  BCUDA(cudaMemcpyAsync(B.s, &h, sizeof(BScalars), cudaMemcpyHostToDevice, c->stream));

  std::vector<double> tol(nr, 0.0), bnorm(nr, 1.0);
  std::vector<int> n_refine(nr, 0);
  if (G == 1)
    status = pcg_block_run<1>(B, nrhs, algo, hs, restart_dev, bnorm, tol, n_refine, st);
  else
    status = pcg_block_run<2>(B, nrhs, algo, hs, restart_dev, bnorm, tol, n_refine, st);
  if (status != UFC_STATUS_OK) {
    cleanup();
    return status;
  }
  // final FP64 residual already in hs->true_rr
  k_deinterleave<<<gi, kBlk, 0, c->stream>>>(c->n, nrhs, nr, B.xx, X);
  BCUDA(cudaGetLastError());
  BCUDA(cudaEventRecord(t1, c->stream));
  BCUDA(cudaEventSynchronize(t1));
  float ms = 0.f;
  cudaEventElapsedTime(&ms, t0, t1);
  cudaEventDestroy(t0);
  cudaEventDestroy(t1);
  c->timing = ufc_timing_info{};
  c->timing.kernel_launches = c->launches + 2;
  bool all = true;
  for (int k = 0; k < nrhs; ++k) {
    ufc_solver_state& sk = st[k];
    const double init = sk.initial_residual;
    sk = ufc_solver_state{};
    sk.initial_residual = init;
    sk.niter = hs->iters[k];
    sk.n_refine = n_refine[k];
    sk.rnorm = std::sqrt(hs->true_rr[k]) / bnorm[k];
    sk.converged = std::sqrt(hs->true_rr[k]) <= tol[k];
    sk.convergence_flag = sk.converged ? 0 : 2;
    sk.solve_time = ms;
    all &= sk.converged != 0;
  }
  cleanup();
#undef BTRY
#undef BCUDA
  UFC_TRY(check_dev_err(c, "ufc_pcg_solve_block"));
  if (!all) return fail(c, UFC_STATUS_NOT_CONVERGED, "ufc_pcg_solve_block: not every right-hand side converged");
  return UFC_STATUS_OK;
}

}  // namespace ufc
