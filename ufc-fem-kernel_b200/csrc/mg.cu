// Geometric multigrid preconditioner for structured C3D8 boxes, in the place of
// the reference's AMG (NM_AMG_Setup, NM_AMG_V_Cycle, NM_AMG_Smooth,
// NM_AMG_Galerkin: ufc_core/L2_NM/Solver/LinSolv/NM_Solv_LinPrecAMG.f90:120-675),
// and the PCG that uses it.
//
// Hierarchy.  Level 0 is the context's own assembled FP64 matrix.  Level l+1
// is the box with half the elements in each direction; its nodes are the
// even-indexed nodes of level l.  Prolongation P is trilinear: a fine node
// takes weight 1 from the coarse node it coincides with, 1/2 from each of the
// two coarse nodes it lies between, and so on per direction.  The coarse
// operator is the Galerkin product P^T A P, formed element by element: the
// matrix of coarse element e is sum over its 8 child elements f of
// W_f^T K_f W_f, W_f the 24x24 restriction of P to the nodes of f, which for
// nested boxes adds up to exactly P^T A P.  Dirichlet DOFs stay eliminated on
// every level: P has zero rows at fixed fine DOFs and zero columns at fixed
// coarse DOFs (a coarse DOF is fixed when the fine DOF it coincides with is),
// and fixed coarse rows get a unit diagonal.
//
// Cycle.  V-cycle with a Chebyshev polynomial smoother of D^-1 A (same degree
// before and after the coarse correction, so the preconditioner is symmetric),
// on [lambda_max/ratio, 1.1 lambda_max] with lambda_max from a power iteration
// at set-up; the coarsest level is solved with its dense inverse (<= kDenseMax DOF)
// or a high-degree Chebyshev polynomial.  Restriction and prolongation are
// structured gathers, one thread per coarse or fine node, so they need no
// atomics and are deterministic; the coarse matrices are assembled colour by
// colour like the fine one.
//
// Precision: the cycle runs in FP64, or (precision = UFC_PRECISION_FP32_REFINE)
// in FP32 on values rounded from the FP64 operators, half the bytes; the PCG
// around it stays FP64 (matrix, vectors, residual), so the preconditioner's
// rounding changes only the iteration count, never the answer.
//
// The PCG is NM_Solver_PCG's recurrence with z = M r from the V-cycle; all of
// an iteration's kernels (SpMV, updates, the cycle on every level) are
// captured once into a CUDA graph and replayed.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <vector>

#include "c3d8_device.cuh"
#include "reduce.cuh"
#include "ufc_internal.cuh"

namespace ufc {

struct MgLevel {
  Ctx* c = nullptr;          // the level's context (level 0: the owner)
  ufc_ctx* own = nullptr;    // levels >= 1: a context holding the coarse box
  int32_t nx = 0, ny = 0, nz = 0;
  double* ke = nullptr;      // levels >= 1: Galerkin element matrices [E][24][24]
  // FP64 cycle: level vectors (level 0: x and b are the PCG's z and r)
  double *x = nullptr, *b = nullptr, *r = nullptr, *d = nullptr, *w = nullptr;
  // FP32 cycle: level vectors, and the level's values and diagonal rounded to FP32
  float *x32 = nullptr, *b32 = nullptr, *r32 = nullptr, *d32 = nullptr, *w32 = nullptr;
  float *val32 = nullptr, *dinv32 = nullptr;
  bool own_xb = false;       // x and b allocated here
  double lmax = 0.0;
  double* inv = nullptr;     // coarsest level: dense inverse [n][n]
  float* inv32 = nullptr;
  double *pv = nullptr, *pw = nullptr;  // power-iteration vectors (lambda_max), kept across refreshes
};

struct Mg {
  std::vector<MgLevel> lv;
  int degree = 2;
  double ratio = 15.0;
  bool stale = false;
  bool fp32 = false;         // the cycle runs in FP32 (values, vectors); the PCG around it in FP64
  int cheb_coarse = 0;       // degree of the coarsest Chebyshev solve (0: dense inverse)
  double* dnorm = nullptr;   // ||v||^2 of the power iteration, on the device
};

namespace {

constexpr int kBlk = 256;
// largest coarsest level inverted densely (on the host, O(n^3), at every set-up
// and refresh); larger ones get a degree-24 Chebyshev solve
constexpr int64_t kDenseMax = 1200;

int grid_n(int64_t n) { return (int)std::max<int64_t>(1, std::min<int64_t>((n + kBlk - 1) / kBlk, 148 * 16)); }

__host__ __device__ inline int64_t box_node(int64_t i, int64_t j, int64_t k, int32_t nx, int32_t ny) {
  return i + (int64_t)(nx + 1) * (j + (int64_t)(ny + 1) * k);
}

// Weight of coarse node A (its signs) at a fine node with coarse parametric
// coordinates xi in {-1, 0, 1}: the trilinear hat, prod_d (1 + s_d xi_d) / 2.
__device__ __forceinline__ double hat(int A, int x0, int x1, int x2) {
  const int xi[3] = {x0, x1, x2};
  double w = 1.0;
#pragma unroll
  for (int d = 0; d < 3; ++d) w *= 0.5 * (1.0 + (double)(node_sign(A, d) * xi[d]));
  return w;
}

// Galerkin element matrices of one coarse level, one CTA of 64 threads per
// coarse element.  FROM_KE: the child matrices are read from the finer level's
// element matrices; otherwise they are computed from the fine elements (the
// linear-elastic D, or the J2 tangent per Gauss point when Dt is given).
template <bool FROM_KE, bool TANGENT>
__global__ void __launch_bounds__(64)
    k_mg_galerkin(int32_t nxc, int32_t nyc, int32_t nzc, const double* __restrict__ coords,
                  const int32_t* __restrict__ conn_f, const double* __restrict__ props, int nprops,
                  const double* __restrict__ Dt, const double* __restrict__ ke_f, const uint8_t* __restrict__ fixed_f,
                  const int32_t* __restrict__ conn_c, const uint8_t* __restrict__ fixed_c, double* __restrict__ ke_c,
                  int32_t* __restrict__ err) {
  __shared__ double Kc[576], Kf[576];
  __shared__ double X[24], g[8][8][3], wdet[8];
  __shared__ double D[TANGENT ? 8 : 1][36];
  __shared__ uint8_t ff[24], fc[24];
  const int t = threadIdx.x;
  const int64_t ec = blockIdx.x;
  const int nxf = 2 * nxc, nyf = 2 * nyc;
  const int64_t I = ec % nxc, J = (ec / nxc) % nyc, K = ec / ((int64_t)nxc * nyc);
  for (int q = t; q < 576; q += 64) Kc[q] = 0.0;
  if (t < 24) fc[t] = fixed_c[3 * (int64_t)conn_c[ec * 8 + t / 3] + t % 3];
  for (int ch = 0; ch < 8; ++ch) {
    const int ca = ch & 1, cb = (ch >> 1) & 1, cc = ch >> 2;
    const int64_t ef = (2 * I + ca) + (int64_t)nxf * ((2 * J + cb) + (int64_t)nyf * (2 * K + cc));
    __syncthreads();  // Kf and the gradients of the previous child are consumed
    if (t < 24) ff[t] = fixed_f[3 * (int64_t)conn_f[ef * 8 + t / 3] + t % 3];
    if (FROM_KE) {
      for (int q = t; q < 576; q += 64) Kf[q] = ke_f[ef * 576 + q];
    } else {
      if (t < 24) X[t] = coords[(int64_t)conn_f[ef * 8 + t / 3] * 3 + t % 3];
      if (TANGENT)
        for (int q = t; q < 288; q += 64) (&D[0][0])[q] = Dt[ef * 288 + q];
      __syncthreads();
      if (t < 8) {
        double inv[9];
        const double det = jacobian_inv<double>(X, t, inv);
        if (!(det > 0.0)) atomicOr(err, (int)kDevBadJacobian);
        wdet[t] = det;
#pragma unroll
        for (int a = 0; a < 8; ++a) grad_x<double>(inv, t, a, g[t][a]);
      }
      __syncthreads();
      // thread t: block (p, q) of the 8x8 block grid of the child's Ke
      const int p = t >> 3, q = t & 7;
      double lam = 0.0, mu = 0.0;
      if (!TANGENT) lame<double>(props[ef * nprops], props[ef * nprops + 1], lam, mu);
      double Kb[9];
#pragma unroll
      for (int k = 0; k < 9; ++k) Kb[k] = 0.0;
#pragma unroll 1
      for (int gp = 0; gp < 8; ++gp) {
        const double* ga = g[gp][p];
        const double* gb = g[gp][q];
        if (TANGENT) {
          constexpr int kIdx[3][3] = {{0, 3, 5}, {1, 3, 4}, {2, 4, 5}};
          constexpr int kCmp[3][3] = {{0, 1, 2}, {1, 0, 2}, {2, 1, 0}};
          const double* Dg = D[TANGENT ? gp : 0];
          double DB[6][3];
#pragma unroll
          for (int k = 0; k < 6; ++k)
#pragma unroll
            for (int j = 0; j < 3; ++j)
              DB[k][j] = Dg[k * 6 + kIdx[j][0]] * gb[kCmp[j][0]] + Dg[k * 6 + kIdx[j][1]] * gb[kCmp[j][1]] +
                         Dg[k * 6 + kIdx[j][2]] * gb[kCmp[j][2]];
#pragma unroll
          for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int j = 0; j < 3; ++j)
              Kb[i * 3 + j] += wdet[gp] * (ga[kCmp[i][0]] * DB[kIdx[i][0]][j] + ga[kCmp[i][1]] * DB[kIdx[i][1]][j] +
                                           ga[kCmp[i][2]] * DB[kIdx[i][2]][j]);
        } else {
          const double dot = ga[0] * gb[0] + ga[1] * gb[1] + ga[2] * gb[2];
#pragma unroll
          for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int j = 0; j < 3; ++j) {
              double v = lam * ga[i] * gb[j] + mu * ga[j] * gb[i];
              if (i == j) v += mu * dot;
              Kb[i * 3 + j] += wdet[gp] * v;
            }
        }
      }
#pragma unroll
      for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) Kf[(3 * p + i) * 24 + 3 * q + j] = Kb[i * 3 + j];
    }
    __syncthreads();
    // thread t: coarse block (A, B) += sum_pq W(p, A) Kf[p][q] W(q, B), masked
    const int A = t >> 3, B = t & 7;
    double wA[8], wB[8];
#pragma unroll
    for (int p = 0; p < 8; ++p) {
      const int o0 = ca + ((node_sign(p, 0) + 1) >> 1) - 1, o1 = cb + ((node_sign(p, 1) + 1) >> 1) - 1,
                o2 = cc + ((node_sign(p, 2) + 1) >> 1) - 1;
      wA[p] = hat(A, o0, o1, o2);
      wB[p] = hat(B, o0, o1, o2);
    }
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
      for (int j = 0; j < 3; ++j) {
        if (fc[3 * A + i] || fc[3 * B + j]) continue;
        double acc = 0.0;
#pragma unroll
        for (int p = 0; p < 8; ++p) {
          if (wA[p] == 0.0 || ff[3 * p + i]) continue;
          double row = 0.0;
#pragma unroll
          for (int q = 0; q < 8; ++q)
            if (wB[q] != 0.0 && !ff[3 * q + j]) row += Kf[(3 * p + i) * 24 + 3 * q + j] * wB[q];
          acc += wA[p] * row;
        }
        Kc[(3 * A + i) * 24 + 3 * B + j] += acc;
      }
  }
  __syncthreads();
  for (int q = t; q < 576; q += 64) ke_c[ec * 576 + q] = Kc[q];
}

// Scatter of given element matrices into the SELL values, one thread per
// (element, node pair) of one colour; rows and columns of fixed DOFs skipped.
__global__ void k_mg_scatter(const int32_t* __restrict__ elems, int32_t ne, const int32_t* __restrict__ conn,
                             const double* __restrict__ ke, const int32_t* __restrict__ slot,
                             const uint8_t* __restrict__ fixed, double* __restrict__ val) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (int64_t)ne * 64) return;
  const int64_t e = elems[t >> 6];
  const int a = (int)(t & 63) >> 3, b = (int)(t & 7);
  const int64_t na = conn[e * 8 + a], nb = conn[e * 8 + b];
  const int64_t P = slot[e * 64 + a * 8 + b];
#pragma unroll
  for (int r = 0; r < 3; ++r)
#pragma unroll
    for (int c = 0; c < 3; ++c)
      if (!fixed[3 * na + r] && !fixed[3 * nb + c]) val[vpos(P, r * 3 + c)] += ke[e * 576 + (3 * a + r) * 24 + 3 * b + c];
}

__global__ void k_mg_fix_diag(int32_t nfix, const int32_t* __restrict__ dofs, const int32_t* __restrict__ dpos,
                              double* __restrict__ val) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < nfix) val[vpos(dpos[dofs[i] / 3], (dofs[i] % 3) * 4)] = 1.0;
}

__global__ void k_mg_dinv(int32_t N, const int32_t* __restrict__ dpos, const double* __restrict__ val,
                          double* __restrict__ dinv) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= 3 * (int64_t)N) return;
  const double d = val[vpos(dpos[i / 3], (int)(i % 3) * 4)];
  dinv[i] = fabs(d) > 1e-30 ? 1.0 / d : 1.0;
}

// r_c = P^T r_f: one thread per coarse node gathers the fine nodes within one
// fine spacing of it, weight prod_d (1 or 1/2).
template <typename T>
__global__ void k_mg_restrict(int32_t nxc, int32_t nyc, int32_t nzc, const T* __restrict__ rf,
                              const uint8_t* __restrict__ fixed_f, const uint8_t* __restrict__ fixed_c,
                              T* __restrict__ rc, const CgScalars* __restrict__ scal) {
  if (scal && scal->stop) return;
  const int64_t nc = (int64_t)(nxc + 1) * (nyc + 1) * (nzc + 1);
  const int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= nc) return;
  const int nxf = 2 * nxc, nyf = 2 * nyc, nzf = 2 * nzc;
  const int64_t I = v % (nxc + 1), J = (v / (nxc + 1)) % (nyc + 1), K = v / ((int64_t)(nxc + 1) * (nyc + 1));
  T s[3] = {T(0), T(0), T(0)};
  for (int dk = -1; dk <= 1; ++dk) {
    const int64_t k = 2 * K + dk;
    if (k < 0 || k > nzf) continue;
    for (int dj = -1; dj <= 1; ++dj) {
      const int64_t j = 2 * J + dj;
      if (j < 0 || j > nyf) continue;
      for (int di = -1; di <= 1; ++di) {
        const int64_t i = 2 * I + di;
        if (i < 0 || i > nxf) continue;
        const T w = T((di ? 0.5 : 1.0) * (dj ? 0.5 : 1.0) * (dk ? 0.5 : 1.0));
        const int64_t f = box_node(i, j, k, nxf, nyf);
#pragma unroll
        for (int d = 0; d < 3; ++d)
          if (!fixed_f[3 * f + d]) s[d] += w * rf[3 * f + d];
      }
    }
  }
#pragma unroll
  for (int d = 0; d < 3; ++d) rc[3 * v + d] = fixed_c[3 * v + d] ? T(0) : s[d];
}

// x_f += P x_c: one thread per fine node gathers its 1, 2, 4 or 8 coarse parents.
template <typename T>
__global__ void k_mg_prolong_add(int32_t nxc, int32_t nyc, int32_t nzc, const T* __restrict__ xc,
                                 const uint8_t* __restrict__ fixed_f, const uint8_t* __restrict__ fixed_c,
                                 T* __restrict__ xf, const CgScalars* __restrict__ scal) {
  if (scal && scal->stop) return;
  const int nxf = 2 * nxc, nyf = 2 * nyc, nzf = 2 * nzc;
  const int64_t nf = (int64_t)(nxf + 1) * (nyf + 1) * (nzf + 1);
  const int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= nf) return;
  const int64_t i = v % (nxf + 1), j = (v / (nxf + 1)) % (nyf + 1), k = v / ((int64_t)(nxf + 1) * (nyf + 1));
  const int64_t i0 = i >> 1, j0 = j >> 1, k0 = k >> 1;
  const int ni = (i & 1) ? 2 : 1, nj = (j & 1) ? 2 : 1, nk = (k & 1) ? 2 : 1;
  const T w = T((ni == 2 ? 0.5 : 1.0) * (nj == 2 ? 0.5 : 1.0) * (nk == 2 ? 0.5 : 1.0));
  T s[3] = {T(0), T(0), T(0)};
  for (int c = 0; c < nk; ++c)
    for (int b = 0; b < nj; ++b)
      for (int a = 0; a < ni; ++a) {
        const int64_t cn = box_node(i0 + a, j0 + b, k0 + c, nxc, nyc);
#pragma unroll
        for (int d = 0; d < 3; ++d)
          if (!fixed_c[3 * cn + d]) s[d] += w * xc[3 * cn + d];
      }
#pragma unroll
  for (int d = 0; d < 3; ++d)
    if (!fixed_f[3 * v + d]) xf[3 * v + d] += s[d];
}

// Chebyshev smoother (three-term recurrence of Saad, Iterative Methods for
// Sparse Linear Systems, Alg. 12.1, with the Jacobi preconditioner).
// Start: r = b - w (w = A x, or zero when x starts at zero), d = D^-1 r / theta,
// x (+)= d.
template <typename T>
__global__ void k_cheb_start(int64_t n, const T* __restrict__ b, const T* __restrict__ w,
                             const T* __restrict__ dinv, T inv_theta, int x_zero, T* __restrict__ x,
                             T* __restrict__ r, T* __restrict__ d, const CgScalars* __restrict__ scal) {
  if (scal && scal->stop) return;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const T ri = b[i] - (x_zero ? T(0) : w[i]);
    const T di = dinv[i] * ri * inv_theta;
    r[i] = ri;
    d[i] = di;
    x[i] = x_zero ? di : x[i] + di;
  }
}

// Step: r -= w (w = A d), d = c1 d + c2 D^-1 r, x += d.
template <typename T>
__global__ void k_cheb_step(int64_t n, const T* __restrict__ w, const T* __restrict__ dinv, T c1, T c2,
                            T* __restrict__ x, T* __restrict__ r, T* __restrict__ d,
                            const CgScalars* __restrict__ scal) {
  if (scal && scal->stop) return;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const T ri = r[i] - w[i];
    const T di = c1 * d[i] + c2 * dinv[i] * ri;
    r[i] = ri;
    d[i] = di;
    x[i] += di;
  }
}

// out = b - w
template <typename T>
__global__ void k_mg_sub(int64_t n, const T* __restrict__ b, const T* __restrict__ w, T* __restrict__ out,
                         const CgScalars* __restrict__ scal) {
  if (scal && scal->stop) return;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    out[i] = b[i] - w[i];
}

// x = Inv b (dense, coarsest level), one warp per row.
template <typename T>
__global__ void k_mg_dense(int64_t n, const T* __restrict__ inv, const T* __restrict__ b, T* __restrict__ x,
                           const CgScalars* __restrict__ scal) {
  if (scal && scal->stop) return;
  const int64_t row = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (row >= n) return;
  T s = T(0);
  for (int64_t j = lane; j < n; j += 32) s += inv[row * n + j] * b[j];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  if (lane == 0) x[row] = s;
}

template <typename A, typename B>
__global__ void k_mg_convert(int64_t n, const A* __restrict__ a, B* __restrict__ b, const CgScalars* __restrict__ scal) {
  if (scal && scal->stop) return;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    b[i] = (B)a[i];
}

// ||v||^2 into *out (power iteration at set-up).
__global__ void k_mg_norm2(int64_t n, const double* __restrict__ v, double* __restrict__ partials,
                           uint32_t* ticket, double* __restrict__ out) {
  double a[1] = {0.0};
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    a[0] += v[i] * v[i];
  double tot[1];
  if (grid_sum<1>(a, partials, ticket, tot)) *out = tot[0];
}

// v = D^-1 w / ||v_prev|| with ||v_prev||^2 read from the device (0: v = 0)
__global__ void k_mg_scale_dinv(int64_t n, const double* __restrict__ w, const double* __restrict__ dinv,
                                const double* __restrict__ nrm2, double* __restrict__ v) {
  const double q = *nrm2;
  const double s = q > 0.0 ? 1.0 / sqrt(q) : 0.0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    v[i] = dinv[i] * w[i] * s;
}

__global__ void k_mg_start_vector(int64_t n, const uint8_t* __restrict__ fixed, double* __restrict__ v) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    v[i] = fixed[i] ? 0.0 : 1.0 + 0.5 * (double)((i * 7919) % 13) / 13.0;
}

// ---- the PCG around the V-cycle: the Jacobi kernels' recurrence with z = M r

// x += alpha p, r -= alpha q, ||r||^2, the stop tests.
__global__ void __launch_bounds__(kBlk)
    k_mgcg_update(int64_t n, const double* __restrict__ p, const double* __restrict__ q, double* __restrict__ r,
                  double* __restrict__ x, CgScalars* __restrict__ scal, double* __restrict__ partials) {
  if (scal->stop) return;
  const double a = scal->alpha;
  double v[1] = {0.0};
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    x[i] += a * p[i];
    const double ri = r[i] - a * q[i];
    r[i] = ri;
    v[0] += ri * ri;
  }
  double tot[1];
  if (grid_sum<1>(v, partials, &scal->ticket[1], tot)) {
    scal->rr = tot[0];
    const int it = scal->iter + 1;
    scal->iter = it;
    if (scal->hist && it <= scal->hist_cap) scal->hist[it - 1] = tot[0];
    if (tot[0] <= scal->tol2) scal->stop = 1;
    else if (!isfinite(tot[0])) scal->stop = 3;
    else if (it >= scal->max_iter) scal->stop = 2;
  }
}

// r.z, beta = r.z / r.z_old (first call: beta = 0).
__global__ void __launch_bounds__(kBlk)
    k_mgcg_rz(int64_t n, const double* __restrict__ r, const double* __restrict__ z, CgScalars* __restrict__ scal,
              double* __restrict__ partials, int first) {
  if (scal->stop) return;
  double v[1] = {0.0};
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    v[0] += r[i] * z[i];
  double tot[1];
  if (grid_sum<1>(v, partials, &scal->ticket[2], tot)) {
    const double old = scal->rz;
    scal->beta = first ? 0.0 : tot[0] / old;
    scal->rz_old = old;
    scal->rz = tot[0];
    if (!isfinite(tot[0]) || !(tot[0] > 0.0)) scal->stop = 3;  // M must stay positive definite
  }
}

// p = z + beta p
__global__ void k_mgcg_pupdate(int64_t n, const double* __restrict__ z, double* __restrict__ p,
                               const CgScalars* __restrict__ scal) {
  if (scal->stop) return;
  const double b = scal->beta;
  // beta = 0 (start, restart): p = z without reading p, which may hold anything
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    p[i] = b == 0.0 ? z[i] : z[i] + b * p[i];
}

// ---------------------------------------------------------------- host side

int dinv_of(Ctx* lc) {
  if (!lc->dinv64) UFC_TRY(dalloc(lc, &lc->dinv64, lc->n));
  return UFC_STATUS_OK;
}

__global__ void k_mg_round(int64_t n, const double* __restrict__ a, float* __restrict__ b) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    b[i] = (float)a[i];
}

// lambda_max of D^-1 A on level L by power iteration (deterministic start), in
// FP64: v <- D^-1 A v / ||v||, lambda = ||v|| after the last step.  The norms
// stay on the device, so the iterations run without a host round trip; the
// vectors are kept for the next refresh.
int estimate_lmax(Ctx* owner, Mg& mg, MgLevel& L, int iters) {
  Ctx* lc = L.c;
  const int64_t n = lc->n;
  const int g = grid_n(n);
  if (!L.pv) UFC_TRY(dalloc(owner, &L.pv, n));
  if (!L.pw) UFC_TRY(dalloc(owner, &L.pw, n));
  if (!mg.dnorm) UFC_TRY(dalloc(owner, &mg.dnorm, 1));
  k_mg_start_vector<<<g, kBlk, 0, owner->stream>>>(n, lc->fixed, L.pv);
  k_mg_norm2<<<g, kBlk, 0, owner->stream>>>(n, L.pv, owner->partials, &owner->scal->ticket[6], mg.dnorm);
  for (int it = 0; it < iters; ++it) {
    spmv64_on(lc, owner->stream, L.pv, L.pw);
    k_mg_scale_dinv<<<g, kBlk, 0, owner->stream>>>(n, L.pw, lc->dinv64, mg.dnorm, L.pv);
    k_mg_norm2<<<g, kBlk, 0, owner->stream>>>(n, L.pv, owner->partials, &owner->scal->ticket[6], mg.dnorm);
  }
  UFC_CUDA(owner, cudaGetLastError());
  double q = 0.0;
  UFC_CUDA(owner, cudaMemcpyAsync(&q, mg.dnorm, sizeof(double), cudaMemcpyDeviceToHost, owner->stream));
  UFC_CUDA(owner, cudaStreamSynchronize(owner->stream));
  L.lmax = iters > 0 ? std::sqrt(q) : 0.0;
  return UFC_STATUS_OK;
}

// Dense inverse of the coarsest matrix (Gauss-Jordan with partial pivoting).
int dense_inverse(Ctx* owner, MgLevel& L, bool fp32) {
  Ctx* lc = L.c;
  const int64_t n = lc->n, nnz = 9 * lc->nnzb;
  std::vector<int64_t> rp(n + 1);
  std::vector<int32_t> col(nnz);
  std::vector<double> val(nnz);
  ufc_csr_export_arg a{};
  a.index_base = 0;
  a.mem = UFC_MEM_HOST;
  a.row_ptr = rp.data();
  a.col_ind = col.data();
  a.values = val.data();
  UFC_TRY(export_csr(lc, &a));
  std::vector<double> M((size_t)n * n, 0.0), Inv((size_t)n * n, 0.0);
  for (int64_t i = 0; i < n; ++i) {
    for (int64_t k = rp[i]; k < rp[i + 1]; ++k) M[i * n + col[k]] = val[k];
    Inv[i * n + i] = 1.0;
  }
  for (int64_t c = 0; c < n; ++c) {
    int64_t piv = c;
    for (int64_t i = c + 1; i < n; ++i)
      if (std::fabs(M[i * n + c]) > std::fabs(M[piv * n + c])) piv = i;
    if (!(std::fabs(M[piv * n + c]) > 0.0))
      return fail(owner, UFC_STATUS_ERROR, "ufc_mg_setup: singular coarsest matrix (unconstrained rigid modes?)");
    if (piv != c)
      for (int64_t j = 0; j < n; ++j) {
        std::swap(M[c * n + j], M[piv * n + j]);
        std::swap(Inv[c * n + j], Inv[piv * n + j]);
      }
    const double s = 1.0 / M[c * n + c];
    for (int64_t j = 0; j < n; ++j) {
      M[c * n + j] *= s;
      Inv[c * n + j] *= s;
    }
    for (int64_t i = 0; i < n; ++i) {
      if (i == c) continue;
      const double f = M[i * n + c];
      if (f == 0.0) continue;
      for (int64_t j = 0; j < n; ++j) {
        M[i * n + j] -= f * M[c * n + j];
        Inv[i * n + j] -= f * Inv[c * n + j];
      }
    }
  }
  if (fp32) {
    std::vector<float> f(Inv.begin(), Inv.end());
    if (!L.inv32) UFC_TRY(dalloc(owner, &L.inv32, n * n));  // same size at every refresh
    UFC_CUDA(owner, cudaMemcpyAsync(L.inv32, f.data(), sizeof(float) * n * n, cudaMemcpyHostToDevice, owner->stream));
    UFC_CUDA(owner, cudaStreamSynchronize(owner->stream));
  } else {
    if (!L.inv) UFC_TRY(dalloc(owner, &L.inv, n * n));
    UFC_CUDA(owner, cudaMemcpyAsync(L.inv, Inv.data(), sizeof(double) * n * n, cudaMemcpyHostToDevice, owner->stream));
    UFC_CUDA(owner, cudaStreamSynchronize(owner->stream));
  }
  return UFC_STATUS_OK;
}

void free_level(MgLevel& L) {
  dfree(&L.ke);
  dfree(&L.r);
  dfree(&L.d);
  dfree(&L.w);
  dfree(&L.r32);
  dfree(&L.d32);
  dfree(&L.w32);
  dfree(&L.x32);
  dfree(&L.b32);
  dfree(&L.val32);
  dfree(&L.dinv32);
  dfree(&L.inv);
  dfree(&L.inv32);
  dfree(&L.pv);
  dfree(&L.pw);
  if (L.own_xb) {
    dfree(&L.x);
    dfree(&L.b);
  }
  if (L.own) ufc_ctx_destroy(L.own);
  L.own = nullptr;
}

// The vectors, values and diagonal of a level in the cycle's precision.
template <typename T>
struct View {
  T *x, *b, *r, *d, *w;
  const T *val, *dinv, *inv;
};

View<double> view(MgLevel& L, double*) { return {L.x, L.b, L.r, L.d, L.w, L.c->val64, L.c->dinv64, L.inv}; }
View<float> view(MgLevel& L, float*) { return {L.x32, L.b32, L.r32, L.d32, L.w32, L.val32, L.dinv32, L.inv32}; }

void spmv_lv(const Ctx* lc, cudaStream_t st, const double* val, const double* x, double* y) {
  (void)val;
  spmv64_on(lc, st, x, y);
}
void spmv_lv(const Ctx* lc, cudaStream_t st, const float* val, const float* x, float* y) {
  spmv32_on(lc, st, val, x, y);
}

// Chebyshev smoothing of A x = b on level L (m steps).
template <typename T>
void cheb(Ctx* owner, MgLevel& L, int m, double ratio, bool x_zero, const CgScalars* scal) {
  Ctx* lc = L.c;
  const View<T> V = view(L, (T*)nullptr);
  const int64_t n = lc->n;
  const int g = grid_n(n);
  const double lmax = 1.1 * L.lmax, lmin = lmax / ratio;
  const double theta = 0.5 * (lmax + lmin), delta = 0.5 * (lmax - lmin);
  const double sigma = theta / delta;
  if (!x_zero) spmv_lv(lc, owner->stream, V.val, V.x, V.w);
  k_cheb_start<T><<<g, kBlk, 0, owner->stream>>>(n, V.b, V.w, V.dinv, (T)(1.0 / theta), x_zero ? 1 : 0, V.x, V.r,
                                                 V.d, scal);
  double rho = 1.0 / sigma;
  for (int k = 1; k < m; ++k) {
    spmv_lv(lc, owner->stream, V.val, V.d, V.w);
    const double rho_new = 1.0 / (2.0 * sigma - rho);
    k_cheb_step<T><<<g, kBlk, 0, owner->stream>>>(n, V.w, V.dinv, (T)(rho_new * rho), (T)(2.0 * rho_new / delta),
                                                  V.x, V.r, V.d, scal);
    rho = rho_new;
  }
  owner->launches += 2 * m - (x_zero ? 1 : 0);
}

// One V-cycle from level l: x ~ A_l^-1 b.
template <typename T>
void vcycle(Ctx* owner, Mg& mg, size_t l, const CgScalars* scal) {
  MgLevel& L = mg.lv[l];
  Ctx* lc = L.c;
  const View<T> V = view(L, (T*)nullptr);
  if (l + 1 == mg.lv.size()) {
    if (V.inv) {
      k_mg_dense<T><<<(int)((lc->n * 32 + kBlk - 1) / kBlk), kBlk, 0, owner->stream>>>(lc->n, V.inv, V.b, V.x, scal);
      owner->launches += 1;
    } else {
      cheb<T>(owner, L, mg.cheb_coarse, 1000.0, true, scal);
    }
    return;
  }
  MgLevel& C = mg.lv[l + 1];
  const View<T> W = view(C, (T*)nullptr);
  cheb<T>(owner, L, mg.degree, mg.ratio, true, scal);
  spmv_lv(lc, owner->stream, V.val, V.x, V.w);
  k_mg_sub<T><<<grid_n(lc->n), kBlk, 0, owner->stream>>>(lc->n, V.b, V.w, V.r, scal);
  k_mg_restrict<T><<<grid_for(C.c->N, kBlk), kBlk, 0, owner->stream>>>(C.nx, C.ny, C.nz, V.r, lc->fixed, C.c->fixed,
                                                                      W.b, scal);
  vcycle<T>(owner, mg, l + 1, scal);
  k_mg_prolong_add<T><<<grid_for(lc->N, kBlk), kBlk, 0, owner->stream>>>(C.nx, C.ny, C.nz, W.x, lc->fixed,
                                                                        C.c->fixed, V.x, scal);
  cheb<T>(owner, L, mg.degree, mg.ratio, false, scal);
  owner->launches += 5;
}

// z = M r on the owner's stream (r, z: FP64 vectors of level 0).
void run_cycle(Ctx* c, Mg& mg, const double* r, double* z, const CgScalars* scal) {
  MgLevel& L0 = mg.lv[0];
  const int64_t n = c->n;
  if (mg.fp32) {
    k_mg_convert<double, float><<<grid_n(n), kBlk, 0, c->stream>>>(n, r, L0.b32, scal);
    vcycle<float>(c, mg, 0, scal);
    k_mg_convert<float, double><<<grid_n(n), kBlk, 0, c->stream>>>(n, L0.x32, z, scal);
    c->launches += 2;
  } else {
    L0.b = const_cast<double*>(r);
    L0.x = z;
    vcycle<double>(c, mg, 0, scal);
  }
}

}  // namespace

void mg_mark_stale(Ctx* c) {
  if (c->mg) c->mg->stale = true;
}

void mg_free(Ctx* c) {
  if (!c->mg) return;
  for (auto& L : c->mg->lv) free_level(L);
  dfree(&c->mg->dnorm);
  delete c->mg;
  c->mg = nullptr;
}

// The numerical part of the hierarchy, from the owner's current FP64 values
// (and J2 tangent): Galerkin element matrices, coarse matrices, diagonals,
// FP32 copies, smoother bounds and the coarsest inverse.  Run at set-up and
// again, on the same boxes and patterns, whenever the owner reassembles.
static int mg_alloc(Ctx* c, double** p, int64_t n) { return *p ? UFC_STATUS_OK : dalloc(c, p, n); }
static int mg_alloc(Ctx* c, float** p, int64_t n) { return *p ? UFC_STATUS_OK : dalloc(c, p, n); }

int mg_refresh(Ctx* c);

int mg_numeric(Ctx* c) {
  Mg& mg = *c->mg;
  const bool tangent = c->mat_model == UFC_MAT_J2_ISO;
  if (tangent && !c->Dt) return fail(c, UFC_STATUS_INVALID, "ufc_mg_setup: no J2 tangent");
  if (!c->dinv64) return fail(c, UFC_STATUS_INVALID, "ufc_mg_setup: no FP64 diagonal");
  for (size_t l = 1; l < mg.lv.size(); ++l) {
    MgLevel& F = mg.lv[l - 1];
    MgLevel& L = mg.lv[l];
    Ctx* lc = L.c;
    UFC_TRY(mg_alloc(c, &L.ke, (int64_t)lc->E * 576));
    const int grid = lc->E;
    if (l == 1) {
      if (tangent)
        k_mg_galerkin<false, true><<<grid, 64, 0, c->stream>>>(L.nx, L.ny, L.nz, c->coords, c->conn, c->props,
                                                               c->nprops, c->Dt, nullptr, c->fixed, lc->conn,
                                                               lc->fixed, L.ke, c->dev_err);
      else
        k_mg_galerkin<false, false><<<grid, 64, 0, c->stream>>>(L.nx, L.ny, L.nz, c->coords, c->conn, c->props,
                                                                c->nprops, nullptr, nullptr, c->fixed, lc->conn,
                                                                lc->fixed, L.ke, c->dev_err);
    } else {
      k_mg_galerkin<true, false><<<grid, 64, 0, c->stream>>>(L.nx, L.ny, L.nz, nullptr, F.c->conn, nullptr, 0,
                                                             nullptr, F.ke, F.c->fixed, lc->conn, lc->fixed, L.ke,
                                                             c->dev_err);
    }
    UFC_CUDA(c, cudaGetLastError());
    const int64_t nv = lc->sell_blocks * 9;
    UFC_TRY(mg_alloc(c, &lc->val64, nv));
    UFC_TRY(dinv_of(lc));
    UFC_CUDA(c, cudaMemsetAsync(lc->val64, 0, sizeof(double) * nv, c->stream));
    for (int col = 0; col < lc->ncol; ++col) {
      const int32_t ne = lc->col_off[col + 1] - lc->col_off[col];
      if (ne == 0) continue;
      k_mg_scatter<<<(int)(((int64_t)ne * 64 + kBlk - 1) / kBlk), kBlk, 0, c->stream>>>(
          lc->col_elems + lc->col_off[col], ne, lc->conn, L.ke, lc->slot, lc->fixed, lc->val64);
    }
    if (lc->nfix > 0)
      k_mg_fix_diag<<<grid_for(lc->nfix, kBlk), kBlk, 0, c->stream>>>(lc->nfix, lc->fix_dofs, lc->dpos, lc->val64);
    k_mg_dinv<<<grid_for(lc->n, kBlk), kBlk, 0, c->stream>>>(lc->N, lc->dpos, lc->val64, lc->dinv64);
    UFC_CUDA(c, cudaGetLastError());
    lc->has_val64 = true;
  }
  UFC_TRY(check_dev_err(c, "ufc_mg_setup"));
  // level vectors (and FP32 values) in the cycle's precision, smoother bounds, coarsest solve
  for (size_t l = 0; l < mg.lv.size(); ++l) {
    MgLevel& L = mg.lv[l];
    const int64_t n = L.c->n;
    if (mg.fp32) {
      const int64_t nv = L.c->sell_blocks * 9;
      UFC_TRY(mg_alloc(c, &L.r32, n));
      UFC_TRY(mg_alloc(c, &L.d32, n));
      UFC_TRY(mg_alloc(c, &L.w32, n));
      UFC_TRY(mg_alloc(c, &L.x32, n));
      UFC_TRY(mg_alloc(c, &L.b32, n));
      UFC_TRY(mg_alloc(c, &L.val32, nv));
      UFC_TRY(mg_alloc(c, &L.dinv32, n));
      k_mg_round<<<grid_n(nv), kBlk, 0, c->stream>>>(nv, L.c->val64, L.val32);
      k_mg_round<<<grid_n(n), kBlk, 0, c->stream>>>(n, L.c->dinv64, L.dinv32);
    } else {
      UFC_TRY(mg_alloc(c, &L.r, n));
      UFC_TRY(mg_alloc(c, &L.d, n));
      UFC_TRY(mg_alloc(c, &L.w, n));
      if (l > 0) {
        L.own_xb = true;
        UFC_TRY(mg_alloc(c, &L.x, n));
        UFC_TRY(mg_alloc(c, &L.b, n));
      }
    }
    if (l + 1 < mg.lv.size() || n > kDenseMax) UFC_TRY(estimate_lmax(c, mg, L, 15));
  }
  MgLevel& Cst = mg.lv.back();
  if (Cst.c->n <= kDenseMax) {
    UFC_TRY(dense_inverse(c, Cst, mg.fp32));
    mg.cheb_coarse = 0;
  } else {
    mg.cheb_coarse = 24;
  }
  mg.stale = false;
  return UFC_STATUS_OK;
}

int mg_setup(Ctx* c, ufc_mg_arg* a) {
  const auto t0 = std::chrono::steady_clock::now();
  if (!c->has_pattern || !c->has_val64)
    return fail(c, UFC_STATUS_INVALID, "ufc_mg_setup: assemble the FP64 values first (UFC_BUILD_FP64)");
  const int32_t nx = a->nx, ny = a->ny, nz = a->nz;
  if (nx <= 0 || ny <= 0 || nz <= 0) return fail(c, UFC_STATUS_INVALID, "ufc_mg_setup: nx, ny, nz must be > 0");
  if ((int64_t)(nx + 1) * (ny + 1) * (nz + 1) != c->N || (int64_t)nx * ny * nz != c->E)
    return fail(c, UFC_STATUS_INVALID, "ufc_mg_setup: node or element count is not that of the nx x ny x nz box");
  const bool tangent = c->mat_model == UFC_MAT_J2_ISO;
  if (tangent && !c->has_trial)
    return fail(c, UFC_STATUS_INVALID, "ufc_mg_setup: J2 tangent needs ufc_elem_compute_fint(update_state=1) first");
  // the connectivity must be the box numbering
  for (int64_t e = 0; e < c->E; ++e) {
    const int64_t i = e % nx, j = (e / nx) % ny, k = e / ((int64_t)nx * ny);
    for (int p = 0; p < 8; ++p) {
      const int64_t want = box_node(i + ((node_sign(p, 0) + 1) >> 1), j + ((node_sign(p, 1) + 1) >> 1),
                                    k + ((node_sign(p, 2) + 1) >> 1), nx, ny);
      if (c->h_conn[e * 8 + p] != want)
        return fail(c, UFC_STATUS_INVALID,
                    "ufc_mg_setup: element " + std::to_string(e) + " does not follow the box numbering");
    }
  }
  mg_free(c);
  release_graphs(c);
  c->mg = new Mg();
  Mg& mg = *c->mg;
  mg.degree = a->degree > 0 ? a->degree : 2;
  mg.ratio = a->ratio > 1.0 ? a->ratio : 15.0;
  const int64_t coarse_max = a->coarse_max > 0 ? a->coarse_max : 300;
  const int max_levels = a->max_levels > 0 ? a->max_levels : 32;
  auto bail = [&](int s) {
    mg_free(c);
    return s;
  };

  // level 0: the owner's matrix; its x and b are the PCG's z and r (bound at solve time)
  mg.lv.emplace_back();
  mg.lv[0].c = c;
  mg.lv[0].nx = nx;
  mg.lv[0].ny = ny;
  mg.lv[0].nz = nz;
  // the owner's FP64 Jacobi diagonal is current after every FP64 assembly
  if (!c->dinv64) return bail(fail(c, UFC_STATUS_INVALID, "ufc_mg_setup: no FP64 diagonal"));

  // host copies of the fine coordinates and fixed mask, to derive the coarse boxes
  std::vector<double> h_coords(c->n);
  std::vector<uint8_t> h_fixed(c->n);
  if (cudaMemcpyAsync(h_coords.data(), c->coords, sizeof(double) * c->n, cudaMemcpyDeviceToHost, c->stream) !=
          cudaSuccess ||
      cudaMemcpyAsync(h_fixed.data(), c->fixed, c->n, cudaMemcpyDeviceToHost, c->stream) != cudaSuccess ||
      cudaStreamSynchronize(c->stream) != cudaSuccess)
    return bail(fail(c, UFC_STATUS_ERROR, "ufc_mg_setup: copy of the mesh failed"));

  int32_t fx = nx, fy = ny, fz = nz;
  while ((int)mg.lv.size() < max_levels && fx % 2 == 0 && fy % 2 == 0 && fz % 2 == 0 &&
         3 * (int64_t)(fx + 1) * (fy + 1) * (fz + 1) > coarse_max) {
    const int32_t cx = fx / 2, cy = fy / 2, cz = fz / 2;
    const int64_t Nc = (int64_t)(cx + 1) * (cy + 1) * (cz + 1), Ec = (int64_t)cx * cy * cz;
    std::vector<double> cc(3 * Nc);
    std::vector<uint8_t> cf(3 * Nc);
    for (int64_t k = 0; k <= cz; ++k)
      for (int64_t j = 0; j <= cy; ++j)
        for (int64_t i = 0; i <= cx; ++i) {
          const int64_t vc = box_node(i, j, k, cx, cy), vf = box_node(2 * i, 2 * j, 2 * k, fx, fy);
          for (int d = 0; d < 3; ++d) {
            cc[3 * vc + d] = h_coords[3 * vf + d];
            cf[3 * vc + d] = h_fixed[3 * vf + d];
          }
        }
    std::vector<int32_t> conn(8 * Ec);
    for (int64_t e = 0; e < Ec; ++e) {
      const int64_t i = e % cx, j = (e / cx) % cy, k = e / ((int64_t)cx * cy);
      for (int p = 0; p < 8; ++p)
        conn[8 * e + p] = (int32_t)box_node(i + ((node_sign(p, 0) + 1) >> 1), j + ((node_sign(p, 1) + 1) >> 1),
                                            k + ((node_sign(p, 2) + 1) >> 1), cx, cy);
    }
    std::vector<int32_t> fixed_dofs;
    for (int64_t q = 0; q < 3 * Nc; ++q)
      if (cf[q]) fixed_dofs.push_back((int32_t)q);
    MgLevel L;
    L.nx = cx;
    L.ny = cy;
    L.nz = cz;
    int st = ufc_ctx_create(c->device, &L.own);
    if (st != UFC_STATUS_OK) return bail(fail(c, st, "ufc_mg_setup: coarse context"));
    L.c = L.own;
    mg.lv.push_back(L);
    MgLevel& M = mg.lv.back();
    ufc_mesh_desc md{(int32_t)Nc, (int32_t)Ec, cc.data(), conn.data(), 0, UFC_MEM_HOST};
    ufc_bc_desc bd{(int32_t)fixed_dofs.size(), fixed_dofs.data(), nullptr, UFC_MEM_HOST};
    ufc_pattern_info pi{};
    if ((st = ufc_mesh_set(M.own, &md)) != UFC_STATUS_OK || (st = ufc_bc_set(M.own, &bd)) != UFC_STATUS_OK ||
        (st = ufc_pattern_build(M.own, &pi)) != UFC_STATUS_OK)
      return bail(fail(c, st, "ufc_mg_setup: coarse level " + std::to_string(mg.lv.size() - 1) + ": " + M.c->err));
    h_coords.swap(cc);
    h_fixed.swap(cf);
    fx = cx;
    fy = cy;
    fz = cz;
  }
  if (mg.lv.size() < 2) return bail(fail(c, UFC_STATUS_INVALID, "ufc_mg_setup: the box cannot be coarsened"));

  mg.fp32 = a->precision == UFC_PRECISION_FP32_REFINE;
  {
    const int st = mg_numeric(c);
    if (st != UFC_STATUS_OK) return bail(st);
  }
  a->levels = (int32_t)mg.lv.size();
  a->coarse_dof = mg.lv.back().c->n;
  UFC_CUDA(c, cudaStreamSynchronize(c->stream));
  a->setup_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  return UFC_STATUS_OK;
}

int mg_apply(Ctx* c, const double* r, double* z) {
  if (!c->mg) return fail(c, UFC_STATUS_INVALID, "ufc_mg_apply: multigrid not set up (ufc_mg_setup)");
  if (c->mg->stale) UFC_TRY(mg_refresh(c));
  run_cycle(c, *c->mg, r, z, nullptr);
  UFC_CUDA(c, cudaGetLastError());
  return UFC_STATUS_OK;
}

int mg_level_ctx(Ctx* c, int32_t level, Ctx** out) {
  if (!c->mg) return fail(c, UFC_STATUS_INVALID, "multigrid not set up");
  if (level < 0 || level >= (int32_t)c->mg->lv.size()) return fail(c, UFC_STATUS_INVALID, "multigrid level out of range");
  *out = c->mg->lv[level].c;
  return UFC_STATUS_OK;
}

int mg_refresh(Ctx* c) {
  if (!c->has_val64) return fail(c, UFC_STATUS_INVALID, "multigrid: the FP64 values are not assembled");
  if (c->mat_model == UFC_MAT_J2_ISO && !c->has_trial)
    return fail(c, UFC_STATUS_INVALID, "multigrid: J2 tangent needs ufc_elem_compute_fint(update_state=1) first");
  release_graphs(c);
  return mg_numeric(c);
}

int pcg_mg(Ctx* c, const ufc_solver_algo* algo, ufc_solver_state* st) {
  if (!c->mg) return fail(c, UFC_STATUS_INVALID, "ufc_pcg_solve: multigrid not set up (ufc_mg_setup)");
  if (c->mg->stale) UFC_TRY(mg_refresh(c));
  Mg& mg = *c->mg;
  if (!c->r64 || !c->p64 || !c->q64) return fail(c, UFC_STATUS_INVALID, "ufc_pcg_solve: vectors");
  if (!c->z64) UFC_TRY(dalloc(c, &c->z64, c->n));
  const int64_t n = c->n;
  const int vg = grid_n(n);
  cudaEvent_t t0, t1;
  UFC_CUDA(c, cudaEventCreate(&t0));
  UFC_CUDA(c, cudaEventCreate(&t1));
  UFC_CUDA(c, cudaEventRecord(t0, c->stream));
  c->timing = ufc_timing_info{};
  c->timing.precision = UFC_PRECISION_FP64;
  c->launches = 0;

  CgScalars h{};
  h.max_iter = algo->max_iter > 0 ? algo->max_iter : 1;
  const int32_t cap = std::min<int32_t>(h.max_iter, 1 << 20);
  if (c->hist_cap < cap) {
    UFC_TRY(dalloc(c, &c->hist, cap));
    c->hist_cap = cap;
  }
  h.hist = c->hist;
  h.hist_cap = c->hist_cap;
  UFC_CUDA(c, cudaMemcpyAsync(c->scal, &h, sizeof(CgScalars), cudaMemcpyHostToDevice, c->stream));
  // r = b - K x0 (FP64), ||b||
  UFC_TRY(true_residual_fp64(c, true));
  UFC_CUDA(c, cudaMemcpyAsync(c->h_scal, c->scal, sizeof(CgScalars), cudaMemcpyDeviceToHost, c->stream));
  UFC_CUDA(c, cudaStreamSynchronize(c->stream));
  if (!std::isfinite(c->h_scal->bb)) return fail(c, UFC_STATUS_INVALID, "ufc_pcg_solve: non-finite right-hand side");
  if (!std::isfinite(c->h_scal->true_rr))
    return fail(c, UFC_STATUS_INVALID, "ufc_pcg_solve: non-finite initial residual (initial guess or matrix)");
  const double bnorm_raw = std::sqrt(c->h_scal->bb);
  const double bnorm = bnorm_raw < 1e-30 ? 1.0 : bnorm_raw;
  const double tol = std::max(algo->tolerance * bnorm, algo->abs_tolerance);
  st->initial_residual = std::sqrt(c->h_scal->true_rr);
  double true_rr = c->h_scal->true_rr;
  bool converged = std::sqrt(true_rr) <= tol;
  int flag = 0, restarts = 0;
  const int batch = algo->check_every > 0 ? algo->check_every : 4;
  cudaGraphExec_t ge = nullptr;
  int64_t graph_launches = 0;
  int status = UFC_STATUS_OK;
  while (!converged && status == UFC_STATUS_OK) {
    // (re)start: r = the FP64 residual, z = M r, p = z
    double tol2 = tol * tol;
    UFC_CUDA(c, cudaMemcpyAsync(&c->scal->tol2, &tol2, sizeof(double), cudaMemcpyHostToDevice, c->stream));
    UFC_CUDA(c, cudaMemsetAsync(&c->scal->stop, 0, sizeof(int32_t), c->stream));
    UFC_CUDA(c, cudaMemcpyAsync(c->r64, c->y64, sizeof(double) * n, cudaMemcpyDeviceToDevice, c->stream));
    run_cycle(c, mg, c->r64, c->z64, c->scal);
    k_mgcg_rz<<<vg, kBlk, 0, c->stream>>>(n, c->r64, c->z64, c->scal, c->partials, 1);
    c->launches += 1;
    UFC_CUDA(c, cudaMemcpyAsync(c->p64, c->z64, sizeof(double) * n, cudaMemcpyDeviceToDevice, c->stream));
    if (!ge) {
      cudaGraph_t g;
      const int64_t counted = c->launches;
      UFC_CUDA(c, cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
      for (int b = 0; b < batch; ++b) {
        cg_spmv64(c, c->p64, c->q64);
        k_mgcg_update<<<vg, kBlk, 0, c->stream>>>(n, c->p64, c->q64, c->r64, c->x64, c->scal, c->partials);
        run_cycle(c, mg, c->r64, c->z64, c->scal);
        k_mgcg_rz<<<vg, kBlk, 0, c->stream>>>(n, c->r64, c->z64, c->scal, c->partials, 0);
        k_mgcg_pupdate<<<vg, kBlk, 0, c->stream>>>(n, c->z64, c->p64, c->scal);
        c->launches += 4;
      }
      cudaError_t e = cudaStreamEndCapture(c->stream, &g);
      if (e != cudaSuccess) return cuda_fail(c, e, "cudaStreamEndCapture");
      e = cudaGraphInstantiate(&ge, g, 0);
      cudaGraphDestroy(g);
      if (e != cudaSuccess) return cuda_fail(c, e, "cudaGraphInstantiate");
      graph_launches = c->launches - counted;  // captured launches run when the graph does
      c->launches = counted;
    }
    for (;;) {
      cudaError_t e = cudaGraphLaunch(ge, c->stream);
      if (e != cudaSuccess) {
        status = cuda_fail(c, e, "cudaGraphLaunch");
        break;
      }
      c->launches += graph_launches;
      UFC_CUDA(c, cudaMemcpyAsync(c->h_scal, c->scal, sizeof(CgScalars), cudaMemcpyDeviceToHost, c->stream));
      UFC_CUDA(c, cudaStreamSynchronize(c->stream));
      if (c->h_scal->stop) break;
    }
    if (status != UFC_STATUS_OK) break;
    const int stop = c->h_scal->stop;
    UFC_TRY(true_residual_fp64(c, false));
    UFC_CUDA(c, cudaMemcpyAsync(c->h_scal, c->scal, sizeof(CgScalars), cudaMemcpyDeviceToHost, c->stream));
    UFC_CUDA(c, cudaStreamSynchronize(c->stream));
    true_rr = c->h_scal->true_rr;
    if (std::sqrt(true_rr) <= tol) {
      converged = true;
      break;
    }
    if (stop == 2 || !std::isfinite(true_rr)) {
      flag = std::isfinite(true_rr) ? 2 : 3;
      break;
    }
    if (++restarts > 4) {
      flag = 3;
      break;
    }
  }
  if (ge) cudaGraphExecDestroy(ge);
  if (status != UFC_STATUS_OK) return status;
  UFC_CUDA(c, cudaEventRecord(t1, c->stream));
  UFC_CUDA(c, cudaEventSynchronize(t1));
  float ms = 0.f;
  cudaEventElapsedTime(&ms, t0, t1);
  cudaEventDestroy(t0);
  cudaEventDestroy(t1);
  c->hist_len = std::min(c->h_scal->iter, c->hist_cap);
  st->niter = c->h_scal->iter;
  st->n_refine = restarts;
  st->converged = converged ? 1 : 0;
  st->convergence_flag = converged ? 0 : (flag ? flag : 2);
  st->rnorm = std::sqrt(true_rr) / bnorm;
  st->solve_time = ms;
  c->timing.kernel_launches = c->launches;
  UFC_TRY(check_dev_err(c, "ufc_pcg_solve"));
  return converged ? UFC_STATUS_OK : UFC_STATUS_NOT_CONVERGED;
}

}  // namespace ufc
