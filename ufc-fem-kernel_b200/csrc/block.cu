// Multi-right-hand-side Jacobi-PCG: nrhs independent FP64 CG runs of
// NM_Solver_PCG (ufc_core/L2_NM/Solver/NM_Solv_Core.f90:363-423) that share
// every SpMV, so the matrix is read once per iteration for all of them.
//
// Vectors are interleaved, entry (dof i, rhs k) at i*nr + k with nr the number
// of right-hand sides rounded up to a power of two (<= 32; padded columns are
// zero and inactive).  One thread handles one (block row, rhs) pair of the
// SpMV: the nr threads of a row read the same matrix values (one request per
// warp) and consecutive x entries.  Each right-hand side has its own
// alpha, beta and stop test; a converged right-hand side is frozen (alpha =
// beta = 0) while the others continue.  Reductions are per right-hand side and
// deterministic: lanes that hold the same rhs are combined by shuffles, then
// across warps and blocks in a fixed order.
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

struct BScalars {
  double rz[kMaxRhs], rz_old[kMaxRhs], alpha[kMaxRhs], beta[kMaxRhs], rr[kMaxRhs], tol2[kMaxRhs];
  double true_rr[kMaxRhs], bb[kMaxRhs];
  int32_t active[kMaxRhs];  // 1 while the rhs iterates
  int32_t conv[kMaxRhs];    // recursive residual met the tolerance
  int32_t iters[kMaxRhs];
  int32_t iter, max_iter, stop, nr;
  uint32_t ticket[4];
};

// Sum NV values per rhs over the grid; the rhs of a thread is threadIdx.x % nr
// for every element it touches (block size and grid stride are multiples of
// nr).  Returns true in the threads k < nr of the last block, with out[v] the
// total of value v for rhs k.
template <int NV>
__device__ bool group_grid_sum(double (&v)[NV], int nr, double* __restrict__ partials, uint32_t* ticket,
                               double (&out)[NV]) {
  __shared__ double sh[kBlk / 32][NV][kMaxRhs];
  __shared__ double fin[kBlk][NV];
  __shared__ bool last;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  for (int o = 16; o >= nr; o >>= 1)
#pragma unroll
    for (int q = 0; q < NV; ++q) v[q] += __shfl_down_sync(0xffffffffu, v[q], o);
  if (lane < nr)
#pragma unroll
    for (int q = 0; q < NV; ++q) sh[w][q][lane] = v[q];
  __syncthreads();
  if (threadIdx.x < nr) {
    for (int q = 0; q < NV; ++q) {
      double s = 0.0;
      for (int ww = 0; ww < (int)(blockDim.x >> 5); ++ww) s += sh[ww][q][threadIdx.x];
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
  const int k = threadIdx.x % nr, per = blockDim.x / nr;
  double acc[NV];
#pragma unroll
  for (int q = 0; q < NV; ++q) acc[q] = 0.0;
  for (int64_t b = threadIdx.x / nr; b < gridDim.x; b += per)
#pragma unroll
    for (int q = 0; q < NV; ++q) acc[q] += __ldcg(partials + (b * NV + q) * kMaxRhs + k);
#pragma unroll
  for (int q = 0; q < NV; ++q) fin[threadIdx.x][q] = acc[q];
  __syncthreads();
  if (threadIdx.x < nr) {
#pragma unroll
    for (int q = 0; q < NV; ++q) {
      double s = 0.0;
      for (int g = 0; g < per; ++g) s += fin[g * nr + threadIdx.x][q];
      out[q] = s;
    }
    if (threadIdx.x == 0) *ticket = 0u;
    return true;
  }
  return false;
}

// y = K x for nr interleaved vectors (FP64 SELL values); mode 1 also forms
// p.q per rhs and alpha.
template <int MODE>
__global__ void __launch_bounds__(kBlk)
    k_bspmv(int32_t N, const int64_t* __restrict__ sptr, const int32_t* __restrict__ col,
            const double* __restrict__ val, const double* __restrict__ x, double* __restrict__ y, int nr,
            BScalars* __restrict__ s, double* __restrict__ partials) {
  if (MODE == 1 && s->stop) return;
  const int k = threadIdx.x % nr;
  const int64_t units = (int64_t)N * nr;
  double dot[1] = {0.0};
  for (int64_t u = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; u < units; u += (int64_t)gridDim.x * blockDim.x) {
    const int64_t row = u / nr;
    const int64_t sl = row >> 5;
    const int t = (int)(row & 31);
    const int64_t base = sptr[sl];
    const int len = (int)((sptr[sl + 1] - base) >> 5);
    const int32_t* cp = col + base + t;
    const double* vp = val + 9 * base + t;
    double a0 = 0.0, a1 = 0.0, a2 = 0.0;
    for (int j = 0; j < len; ++j) {
      const int64_t cj = cp[32 * j];
      const double x0 = __ldg(x + (3 * cj) * nr + k), x1 = __ldg(x + (3 * cj + 1) * nr + k),
                   x2 = __ldg(x + (3 * cj + 2) * nr + k);
      const double* v = vp + 288 * (int64_t)j;
      a0 += v[0] * x0 + v[32] * x1 + v[64] * x2;
      a1 += v[96] * x0 + v[128] * x1 + v[160] * x2;
      a2 += v[192] * x0 + v[224] * x1 + v[256] * x2;
    }
    y[(3 * row) * nr + k] = a0;
    y[(3 * row + 1) * nr + k] = a1;
    y[(3 * row + 2) * nr + k] = a2;
    if (MODE == 1)
      dot[0] += x[(3 * row) * nr + k] * a0 + x[(3 * row + 1) * nr + k] * a1 + x[(3 * row + 2) * nr + k] * a2;
  }
  if (MODE == 1) {
    double tot[1];
    if (group_grid_sum<1>(dot, nr, partials, &s->ticket[0], tot)) {
      const int kk = threadIdx.x;
      const bool ok = s->active[kk] && fabs(tot[0]) > 1e-300 && isfinite(tot[0]);
      s->alpha[kk] = ok ? s->rz[kk] / tot[0] : 0.0;
      if (s->active[kk] && !ok) s->active[kk] = 0;  // breakdown of this rhs
    }
  }
}

__global__ void __launch_bounds__(kBlk)
    k_bupdate(int64_t nn, int nr, const double* __restrict__ p, const double* __restrict__ q, double* __restrict__ r,
              double* __restrict__ x, const double* __restrict__ dinv, BScalars* __restrict__ s,
              double* __restrict__ partials) {
  if (s->stop) return;
  const int k = threadIdx.x % nr;
  const double a = s->alpha[k];
  double v[2] = {0.0, 0.0};
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < nn; e += (int64_t)gridDim.x * blockDim.x) {
    x[e] += a * p[e];
    const double re = r[e] - a * q[e];
    r[e] = re;
    const double ze = dinv ? dinv[e / nr] * re : re;
    v[0] += re * ze;
    v[1] += re * re;
  }
  double tot[2];
  if (group_grid_sum<2>(v, nr, partials, &s->ticket[1], tot)) {
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

__global__ void __launch_bounds__(kBlk)
    k_bpupdate(int64_t nn, int nr, const double* __restrict__ r, const double* __restrict__ dinv,
               double* __restrict__ p, const BScalars* __restrict__ s) {
  if (s->stop) return;
  const int k = threadIdx.x % nr;
  const double b = s->beta[k];
  const bool act = s->active[k];
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < nn; e += (int64_t)gridDim.x * blockDim.x) {
    if (!act) continue;
    const double re = r[e];
    p[e] = (dinv ? dinv[e / nr] * re : re) + b * p[e];
  }
}

// r = b - y with ||r||^2, ||b||^2 and r.z per rhs (the state a restart needs).
__global__ void __launch_bounds__(kBlk)
    k_bresid(int64_t nn, int nr, const double* __restrict__ b, const double* __restrict__ y, double* __restrict__ r,
             const double* __restrict__ dinv, BScalars* __restrict__ s, double* __restrict__ partials) {
  double v[3] = {0.0, 0.0, 0.0};
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < nn; e += (int64_t)gridDim.x * blockDim.x) {
    const double be = b[e];
    const double re = be - y[e];
    r[e] = re;
    v[0] += re * re;
    v[1] += be * be;
    v[2] += re * (dinv ? dinv[e / nr] * re : re);
  }
  double tot[3];
  if (group_grid_sum<3>(v, nr, partials, &s->ticket[2], tot)) {
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

int grid_vec(int64_t units) {
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  return (int)std::max<int64_t>(1, std::min<int64_t>((units + kBlk - 1) / kBlk, (int64_t)sms * 8));
}

}  // namespace

int pcg_solve_block(Ctx* c, int nrhs, const double* B, double* X, const ufc_solver_algo* algo,
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
  const int64_t nn = c->n * nr;
  const double* dinv = algo->precond_type == UFC_SOLV_PREC_JACOBI ? c->dinv64 : nullptr;
  double *bx = nullptr, *xx = nullptr, *rx = nullptr, *px = nullptr, *qx = nullptr;
  BScalars* s = nullptr;
  BScalars* hs = nullptr;
  double* partials = nullptr;
  int32_t* restart_dev = nullptr;
  const int gv = grid_vec(nn);
  auto cleanup = [&]() {
    dfree(&bx); dfree(&xx); dfree(&rx); dfree(&px); dfree(&qx); dfree(&s); dfree(&partials); dfree(&restart_dev);
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
  BTRY(dalloc(c, &bx, nn));
  BTRY(dalloc(c, &xx, nn));
  BTRY(dalloc(c, &rx, nn));
  BTRY(dalloc(c, &px, nn));
  BTRY(dalloc(c, &qx, nn));
  BTRY(dalloc(c, &s, 1));
  BTRY(dalloc(c, &partials, (int64_t)gv * 3 * kMaxRhs));
  BTRY(dalloc(c, &restart_dev, kMaxRhs));
  BCUDA(cudaMallocHost((void**)&hs, sizeof(BScalars)));
  cudaEvent_t t0, t1;
  BCUDA(cudaEventCreate(&t0));
  BCUDA(cudaEventCreate(&t1));
  BCUDA(cudaEventRecord(t0, c->stream));

  k_interleave<<<gv, kBlk, 0, c->stream>>>(c->n, nrhs, nr, B, bx);
  if (algo->use_x0)
    k_interleave<<<gv, kBlk, 0, c->stream>>>(c->n, nrhs, nr, X, xx);
  else
    BCUDA(cudaMemsetAsync(xx, 0, sizeof(double) * nn, c->stream));
  BScalars h{};
  h.nr = nr;
  h.max_iter = algo->max_iter;
  BCUDA(cudaMemcpyAsync(s, &h, sizeof(BScalars), cudaMemcpyHostToDevice, c->stream));

  auto residual = [&]() -> int {
    k_bspmv<0><<<gv, kBlk, 0, c->stream>>>(c->N, c->slice_ptr, c->sell_col, c->val64, xx, qx, nr, s, partials);
    k_bresid<<<gv, kBlk, 0, c->stream>>>(nn, nr, bx, qx, rx, dinv, s, partials);
    UFC_CUDA(c, cudaGetLastError());
    UFC_CUDA(c, cudaMemcpyAsync(hs, s, sizeof(BScalars), cudaMemcpyDeviceToHost, c->stream));
    UFC_CUDA(c, cudaStreamSynchronize(c->stream));
    return UFC_STATUS_OK;
  };
  BTRY(residual());
  std::vector<double> tol(nr, 0.0), bnorm(nr, 1.0);
  for (int k = 0; k < nr; ++k) {
    const double bn = std::sqrt(hs->bb[k]);
    bnorm[k] = bn < 1e-30 ? 1.0 : bn;
    tol[k] = std::max(algo->tolerance * bnorm[k], algo->abs_tolerance);
    if (k < nrhs) st[k].initial_residual = std::sqrt(hs->true_rr[k]);
  }
  const int batch = algo->check_every > 0 ? algo->check_every : 32;
  std::vector<int32_t> restart(kMaxRhs, 0);
  std::vector<int> conv(nr, 0), n_refine(nr, 0);
  int total_iter = 0;
  for (int round = 0; round < 64; ++round) {
    // (re)start every rhs whose FP64 residual is above its tolerance
    bool any = false;
    for (int k = 0; k < nr; ++k) {
      const bool ok = k >= nrhs || std::sqrt(hs->true_rr[k]) <= tol[k];
      conv[k] = ok;
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
    cudaMemcpyAsync(s, &h, sizeof(BScalars), cudaMemcpyHostToDevice, c->stream);
    cudaMemcpyAsync(restart_dev, restart.data(), sizeof(int32_t) * kMaxRhs, cudaMemcpyHostToDevice, c->stream);
    k_bpinit<<<gv, kBlk, 0, c->stream>>>(nn, nr, rx, dinv, px, restart_dev);
    // iterate in batches until every active rhs stops
    for (;;) {
      for (int b = 0; b < batch; ++b) {
        k_bspmv<1><<<gv, kBlk, 0, c->stream>>>(c->N, c->slice_ptr, c->sell_col, c->val64, px, qx, nr, s, partials);
        k_bupdate<<<gv, kBlk, 0, c->stream>>>(nn, nr, px, qx, rx, xx, dinv, s, partials);
        k_bpupdate<<<gv, kBlk, 0, c->stream>>>(nn, nr, rx, dinv, px, s);
      }
      cudaError_t e = cudaGetLastError();
      if (e != cudaSuccess) { cleanup(); return cuda_fail(c, e, "ufc_pcg_solve_block"); }
      cudaMemcpyAsync(hs, s, sizeof(BScalars), cudaMemcpyDeviceToHost, c->stream);
      cudaStreamSynchronize(c->stream);
      if (hs->stop) break;
    }
    total_iter += hs->iter;
    for (int k = 0; k < nr; ++k) h.iters[k] = hs->iters[k];
    // FP64 true residual of every rhs (residual replacement)
    const std::vector<int32_t> iters_keep(hs->iters, hs->iters + kMaxRhs);
    BTRY(residual());
    for (int k = 0; k < nr; ++k) {
      hs->iters[k] = iters_keep[k];
      ++n_refine[k];
    }
    if (hs->stop == 2) break;
  }
  // final FP64 residual already in hs->true_rr
  k_deinterleave<<<gv, kBlk, 0, c->stream>>>(c->n, nrhs, nr, xx, X);
  BCUDA(cudaGetLastError());
  BCUDA(cudaEventRecord(t1, c->stream));
  BCUDA(cudaEventSynchronize(t1));
  float ms = 0.f;
  cudaEventElapsedTime(&ms, t0, t1);
  cudaEventDestroy(t0);
  cudaEventDestroy(t1);
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
