// C3D8 element kernels: stiffness assembly, matrix-free FP64 operator,
// internal force with the J2 return map, Gauss-point stress, material-point
// batch update and the adjoint sensitivity.
//
// Assembly is deterministic without floating-point atomics: elements are
// processed colour by colour (no two elements of one colour share a node), and
// inside a colour every matrix or vector entry has exactly one writer, so each
// entry receives its contributions in the fixed colour order.
#include <cuda_runtime.h>

#include <algorithm>

#include "c3d8_device.cuh"
#include "reduce.cuh"
#include "ufc_internal.cuh"

namespace ufc {

namespace {

constexpr int kWarpsPerCta = 4;

// Node pairs (a <= b) of the upper triangle of the 8x8 block grid of Ke.
__constant__ int8_t c_pair_a[36];
__constant__ int8_t c_pair_b[36];

struct PairTable {
  int8_t a[36], b[36];
  PairTable() {
    int k = 0;
    for (int i = 0; i < 8; ++i)
      for (int j = i; j < 8; ++j) {
        a[k] = (int8_t)i;
        b[k] = (int8_t)j;
        ++k;
      }
  }
};

template <typename T>
struct WarpSmem {
  T X[24];
  T g[8][8][3];  // [gp][node][dir] physical gradients
  T wdet[8];
  T D[8][36];    // per-Gauss-point tangent (J2 only)
};

// Stiffness block K_ab (3x3, row-major) contribution of one Gauss point.
template <typename T, bool kTangent>
__device__ __forceinline__ void block_gp(const T* ga, const T* gb, T wd, T lam, T mu, const T* D, T K[9]) {
  if (!kTangent) {
    const T dot = ga[0] * gb[0] + ga[1] * gb[1] + ga[2] * gb[2];
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
      for (int j = 0; j < 3; ++j) {
        T v = lam * ga[i] * gb[j] + mu * ga[j] * gb[i];
        if (i == j) v += mu * dot;
        K[i * 3 + j] += wd * v;
      }
  } else {
    // B column j of a node has non-zeros at Voigt rows kIdx[j][m] with gradient
    // component kCmp[j][m] (B matrix of PH_Elem_ShapeFunc.f90:225-244).
    constexpr int kIdx[3][3] = {{0, 3, 5}, {1, 3, 4}, {2, 4, 5}};
    constexpr int kCmp[3][3] = {{0, 1, 2}, {1, 0, 2}, {2, 1, 0}};
    T DB[6][3];
#pragma unroll
    for (int k = 0; k < 6; ++k)
#pragma unroll
      for (int j = 0; j < 3; ++j)
        DB[k][j] = D[k * 6 + kIdx[j][0]] * gb[kCmp[j][0]] + D[k * 6 + kIdx[j][1]] * gb[kCmp[j][1]] +
                   D[k * 6 + kIdx[j][2]] * gb[kCmp[j][2]];
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
      for (int j = 0; j < 3; ++j)
        K[i * 3 + j] += wd * (ga[kCmp[i][0]] * DB[kIdx[i][0]][j] + ga[kCmp[i][1]] * DB[kIdx[i][1]][j] +
                              ga[kCmp[i][2]] * DB[kIdx[i][2]][j]);
  }
}

// One warp per element of the given colour: Ke = sum_gp w detJ B^T D B, block by
// block, added into the SELL values of the stiffness.  Entries in a row or a
// column of a Dirichlet DOF are skipped (symmetric elimination).
template <typename T, bool kTangent>
__global__ void __launch_bounds__(kWarpsPerCta * 32)
    k_assemble(const int32_t* __restrict__ elems, int32_t ne, const double* __restrict__ coords,
               const int32_t* __restrict__ conn, const double* __restrict__ props, int nprops,
               const double* __restrict__ Dt, const int32_t* __restrict__ slot, const uint8_t* __restrict__ fixed,
               T* __restrict__ val, int32_t* __restrict__ err) {
  __shared__ WarpSmem<T> sm[kWarpsPerCta];
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int64_t idx = (int64_t)blockIdx.x * kWarpsPerCta + w;
  if (idx >= ne) return;
  const int64_t e = elems[idx];
  WarpSmem<T>& s = sm[w];
  if (lane < 24) s.X[lane] = (T)coords[(int64_t)conn[e * 8 + lane / 3] * 3 + lane % 3];
  if (kTangent) {
    for (int k = lane; k < 288; k += 32) (&s.D[0][0])[k] = (T)Dt[e * 288 + k];
  }
  __syncwarp();
  if (lane < 8) {
    T inv[9];
    const T det = jacobian_inv<T>(s.X, lane, inv);
    if (!(det > T(0))) atomicOr(err, (int)kDevBadJacobian);
    s.wdet[lane] = det;
#pragma unroll
    for (int a = 0; a < 8; ++a) grad_x<T>(inv, lane, a, s.g[lane][a]);
  }
  __syncwarp();
  T lam = T(0), mu = T(0);
  if (!kTangent) lame<T>((T)props[e * nprops], (T)props[e * nprops + 1], lam, mu);
  for (int p = lane; p < 36; p += 32) {
    const int a = c_pair_a[p], b = c_pair_b[p];
    T K[9];
#pragma unroll
    for (int k = 0; k < 9; ++k) K[k] = T(0);
    if (kTangent) {
#pragma unroll 1
      for (int gp = 0; gp < 8; ++gp) block_gp<T, true>(s.g[gp][a], s.g[gp][b], s.wdet[gp], lam, mu, s.D[gp], K);
    } else {
#pragma unroll
      for (int gp = 0; gp < 8; ++gp) block_gp<T, false>(s.g[gp][a], s.g[gp][b], s.wdet[gp], lam, mu, s.D[gp], K);
    }
    const int64_t na = conn[e * 8 + a], nb = conn[e * 8 + b];
    const int64_t P = slot[e * 64 + a * 8 + b];
    bool fa[3], fb[3];
#pragma unroll
    for (int r = 0; r < 3; ++r) {
      fa[r] = fixed[3 * na + r] != 0;
      fb[r] = fixed[3 * nb + r] != 0;
    }
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
      for (int c = 0; c < 3; ++c)
        if (!fa[r] && !fb[c]) val[vpos(P, r * 3 + c)] += K[r * 3 + c];
    if (a != b) {
      const int64_t Q = slot[e * 64 + b * 8 + a];
#pragma unroll
      for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int c = 0; c < 3; ++c)
          if (!fb[r] && !fa[c]) val[vpos(Q, r * 3 + c)] += K[c * 3 + r];
    }
  }
}

__global__ void k_round_values(int64_t n, const double* __restrict__ v64, float* __restrict__ v32) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    v32[i] = (float)v64[i];
}

// Difference form: the diagonal slot of each block row holds the FP64 block
// row sum S_i = sum_j K_ij, rounded once (one thread per block row).
__global__ void k_diag_rowsum(int32_t N, const int64_t* __restrict__ sptr, const int32_t* __restrict__ dpos,
                              const double* __restrict__ v64, float* __restrict__ v32) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  const int64_t s = i >> 5, t = i & 31;
  const int64_t base = sptr[s], len = (sptr[s + 1] - base) >> 5;
  double S[9];
#pragma unroll
  for (int c = 0; c < 9; ++c) S[c] = 0.0;
  for (int64_t j = 0; j < len; ++j) {
    const int64_t P = base + j * 32 + t;
#pragma unroll
    for (int c = 0; c < 9; ++c) S[c] += v64[vpos(P, c)];
  }
  const int64_t d = dpos[i];
#pragma unroll
  for (int c = 0; c < 9; ++c) v32[vpos(d, c)] = (float)S[c];
}

// Jacobi diagonal in FP32 from the FP64 diagonal.
__global__ void k_dinv_from64(int32_t N, const int32_t* __restrict__ dpos, const double* __restrict__ val,
                              float* __restrict__ dinv) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= 3 * (int64_t)N) return;
  const double d = val[vpos(dpos[i / 3], (int)(i % 3) * 4)];
  dinv[i] = fabs(d) > 1e-30 ? (float)(1.0 / d) : 1.0f;
}

template <typename T>
__global__ void k_fix_diag(int32_t nfix, const int32_t* __restrict__ dofs, const int32_t* __restrict__ dpos,
                           T* __restrict__ val) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nfix) return;
  const int32_t d = dofs[i];
  val[vpos(dpos[d / 3], (d % 3) * 4)] = T(1);
}

// Jacobi diag_inv = 1/K_ii, or 1 when |K_ii| <= 1e-30 (NM_LinSolv_Prec_Jacobi_Build,
// ufc_core/L2_NM/Solver/LinSolv/NM_Solv_LinPrec.f90:328-353; NM_Solver_PCG uses 1e-30).
template <typename T>
__global__ void k_dinv(int32_t N, const int32_t* __restrict__ dpos, const T* __restrict__ val, T* __restrict__ dinv) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= 3 * (int64_t)N) return;
  const T d = val[vpos(dpos[i / 3], (int)(i % 3) * 4)];
  dinv[i] = fabs((double)d) > 1e-30 ? T(1) / d : T(1);
}

// Matrix-free FP64 operator, one thread per element of one colour:
// y += sum_e Ke x_e with Ke = sum_gp w detJ B^T D B.  masked = true applies the
// eliminated operator (x and y restricted to free DOFs); masked = false gives
// the internal force of the linear-elastic material (PH_Elem_C3D8_IntForce,
// PH_Elem_C3D8.f90:734-757).
__global__ void __launch_bounds__(128)
    k_apply_iso(const int32_t* __restrict__ elems, int32_t ne, const double* __restrict__ coords,
                const int32_t* __restrict__ conn, const double* __restrict__ props, int nprops,
                const double* __restrict__ x, const uint8_t* __restrict__ fixed, double* __restrict__ y,
                int32_t* __restrict__ err) {
  const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= ne) return;
  const int64_t e = elems[idx];
  int64_t nd[8];
  double X[24], ue[24], fe[24];
#pragma unroll
  for (int a = 0; a < 8; ++a) nd[a] = conn[e * 8 + a];
#pragma unroll
  for (int a = 0; a < 8; ++a)
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      X[a * 3 + i] = coords[nd[a] * 3 + i];
      const int64_t d = 3 * nd[a] + i;
      ue[a * 3 + i] = (fixed && fixed[d]) ? 0.0 : x[d];
      fe[a * 3 + i] = 0.0;
    }
  double lam, mu;
  lame<double>(props[e * nprops], props[e * nprops + 1], lam, mu);
  bool bad = false;
#pragma unroll 1
  for (int ip = 0; ip < 8; ++ip) {
    double inv[9], eps[6], sg[6];
    const double det = jacobian_inv<double>(X, ip, inv);
    bad |= !(det > 0.0);
    strain_at<double>(inv, ip, ue, eps);
    iso_stress<double>(lam, mu, eps, sg);
    add_bt_sigma<double>(inv, ip, det, sg, fe);
  }
  if (bad) atomicOr(err, (int)kDevBadJacobian);
#pragma unroll
  for (int a = 0; a < 8; ++a)
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      const int64_t d = 3 * nd[a] + i;
      if (!(fixed && fixed[d])) y[d] += fe[a * 3 + i];
    }
}

// Matrix-free consistent-tangent operator, FP64, one thread per element of one
// colour: y += sum_e B^T D_gp B x_e with the per-Gauss-point tangents of the
// last return map (unmasked: all rows and columns).  Newton uses it to lift a
// prescribed displacement increment into the right-hand side.
__global__ void __launch_bounds__(128)
    k_apply_tangent(const int32_t* __restrict__ elems, int32_t ne, const double* __restrict__ coords,
                    const int32_t* __restrict__ conn, const double* __restrict__ Dt, const double* __restrict__ x,
                    double* __restrict__ y) {
  const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= ne) return;
  const int64_t e = elems[idx];
  int64_t nd[8];
  double X[24], xe[24], fe[24];
#pragma unroll
  for (int a = 0; a < 8; ++a) {
    nd[a] = conn[e * 8 + a];
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      X[a * 3 + i] = coords[nd[a] * 3 + i];
      xe[a * 3 + i] = x[3 * nd[a] + i];
      fe[a * 3 + i] = 0.0;
    }
  }
#pragma unroll 1
  for (int ip = 0; ip < 8; ++ip) {
    double inv[9], eps[6], s[6];
    const double det = jacobian_inv<double>(X, ip, inv);
    strain_at<double>(inv, ip, xe, eps);
    const double* D = Dt + (e * 8 + ip) * 36;
#pragma unroll
    for (int i = 0; i < 6; ++i) {
      double t = 0.0;
#pragma unroll
      for (int j = 0; j < 6; ++j) t += D[i * 6 + j] * eps[j];
      s[i] = t;
    }
    add_bt_sigma<double>(inv, ip, det, s, fe);
  }
#pragma unroll
  for (int a = 0; a < 8; ++a)
#pragma unroll
    for (int i = 0; i < 3; ++i) y[3 * nd[a] + i] += fe[a * 3 + i];
}

// J2 return map at every Gauss point: strain increment from du = u - u_n,
// committed state (sig_n, epeq_n, epl_n) -> trial state and consistent tangent.
__global__ void __launch_bounds__(128)
    k_j2_gp(int64_t G, const double* __restrict__ coords, const int32_t* __restrict__ conn,
            const double* __restrict__ props, int nprops, const double* __restrict__ u,
            const double* __restrict__ u_n, const double* __restrict__ sig_n, const double* __restrict__ epeq_n,
            const double* __restrict__ epl_n, double* __restrict__ sig_t, double* __restrict__ epeq_t,
            double* __restrict__ epl_t, double* __restrict__ Dt, int32_t* __restrict__ err) {
  const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= G) return;
  const int64_t e = g >> 3;
  const int ip = (int)(g & 7);
  double X[24], du[24];
#pragma unroll
  for (int a = 0; a < 8; ++a) {
    const int64_t nd = conn[e * 8 + a];
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      X[a * 3 + i] = coords[nd * 3 + i];
      du[a * 3 + i] = u[3 * nd + i] - u_n[3 * nd + i];
    }
  }
  double inv[9], de[6], s[6], epl[6], D[36], epeq;
  const double det = jacobian_inv<double>(X, ip, inv);
  if (!(det > 0.0)) atomicOr(err, (int)kDevBadJacobian);
  strain_at<double>(inv, ip, du, de);
  j2_update(props + e * nprops, de, sig_n + g * 6, epeq_n[g], epl_n + g * 6, s, &epeq, epl, D);
  bool finite = isfinite(epeq);
#pragma unroll
  for (int i = 0; i < 6; ++i) {
    sig_t[g * 6 + i] = s[i];
    epl_t[g * 6 + i] = epl[i];
    finite &= isfinite(s[i]);
  }
  epeq_t[g] = epeq;
#pragma unroll
  for (int k = 0; k < 36; ++k) Dt[g * 36 + k] = D[k];
  if (!finite) atomicOr(err, (int)kDevNonFinite);
}

// F_int from the Gauss-point stresses, one thread per element of one colour.
__global__ void __launch_bounds__(128)
    k_fint_from_stress(const int32_t* __restrict__ elems, int32_t ne, const double* __restrict__ coords,
                       const int32_t* __restrict__ conn, const double* __restrict__ sig, double* __restrict__ y) {
  const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= ne) return;
  const int64_t e = elems[idx];
  int64_t nd[8];
  double X[24], fe[24];
#pragma unroll
  for (int a = 0; a < 8; ++a) {
    nd[a] = conn[e * 8 + a];
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      X[a * 3 + i] = coords[nd[a] * 3 + i];
      fe[a * 3 + i] = 0.0;
    }
  }
#pragma unroll 1
  for (int ip = 0; ip < 8; ++ip) {
    double inv[9], s[6];
    const double det = jacobian_inv<double>(X, ip, inv);
#pragma unroll
    for (int i = 0; i < 6; ++i) s[i] = sig[(e * 8 + ip) * 6 + i];
    add_bt_sigma<double>(inv, ip, det, s, fe);
  }
#pragma unroll
  for (int a = 0; a < 8; ++a)
#pragma unroll
    for (int i = 0; i < 3; ++i) y[3 * nd[a] + i] += fe[a * 3 + i];
}

// Elastic Gauss-point stress and von Mises (PH_Elem_C3D8_EvalVonMises,
// PH_Elem_C3D8.f90:2768-2780), one thread per Gauss point.
__global__ void __launch_bounds__(128)
    k_stress_iso(int64_t G, const double* __restrict__ coords, const int32_t* __restrict__ conn,
                 const double* __restrict__ props, int nprops, const double* __restrict__ u, double* __restrict__ sig,
                 double* __restrict__ vm) {
  const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= G) return;
  const int64_t e = g >> 3;
  const int ip = (int)(g & 7);
  double X[24], ue[24];
#pragma unroll
  for (int a = 0; a < 8; ++a) {
    const int64_t nd = conn[e * 8 + a];
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      X[a * 3 + i] = coords[nd * 3 + i];
      ue[a * 3 + i] = u[3 * nd + i];
    }
  }
  double inv[9], eps[6], s[6], lam, mu;
  jacobian_inv<double>(X, ip, inv);
  strain_at<double>(inv, ip, ue, eps);
  lame<double>(props[e * nprops], props[e * nprops + 1], lam, mu);
  iso_stress<double>(lam, mu, eps, s);
  if (sig)
#pragma unroll
    for (int i = 0; i < 6; ++i) sig[g * 6 + i] = s[i];
  if (vm) {
    const double p = (s[0] + s[1] + s[2]) / 3.0;
    const double j2 = 0.5 * ((s[0] - p) * (s[0] - p) + (s[1] - p) * (s[1] - p) + (s[2] - p) * (s[2] - p)) +
                      s[3] * s[3] + s[4] * s[4] + s[5] * s[5];
    vm[g] = sqrt(3.0 * fmax(j2, 0.0));
  }
}

__global__ void k_vm_from_stress(int64_t G, const double* __restrict__ s6, double* __restrict__ sig,
                                 double* __restrict__ vm) {
  const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= G) return;
  const double* s = s6 + g * 6;
  if (sig)
    for (int i = 0; i < 6; ++i) sig[g * 6 + i] = s[i];
  if (vm) {
    const double p = (s[0] + s[1] + s[2]) / 3.0;
    const double j2 = 0.5 * ((s[0] - p) * (s[0] - p) + (s[1] - p) * (s[1] - p) + (s[2] - p) * (s[2] - p)) +
                      s[3] * s[3] + s[4] * s[4] + s[5] * s[5];
    vm[g] = sqrt(3.0 * fmax(j2, 0.0));
  }
}

// Material-point batch (PH_Mat_Update_Arg rows): one thread per point.
__global__ void k_mat_batch(int32_t n, int32_t model, const double* __restrict__ props, int nprops, int per_point,
                            const double* __restrict__ stress_n, const double* __restrict__ dstrain,
                            const double* __restrict__ sdv_n, double* __restrict__ stress, double* __restrict__ sdv,
                            double* __restrict__ ddsdde, int32_t* __restrict__ yielded) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double* pr = props + (per_point ? i * nprops : 0);
  double s[6], D[36], epl[6], epeq = 0.0;
  int y = 0;
  if (model == UFC_MAT_J2_ISO) {
    const double epeq_n = sdv_n ? sdv_n[i * 7] : 0.0;
    y = j2_update(pr, dstrain + i * 6, stress_n + i * 6, epeq_n, sdv_n ? sdv_n + i * 7 + 1 : nullptr, s, &epeq, epl,
                  D);
  } else {
    // PH_Mat_Elas_IP_Incr_Eval (PH_Mat_Elas_Eval.f90:41-84): sigma = sigma_n + D dstrain.
    const double big[4] = {pr[0], pr[1], 1e300, 0.0};
    j2_update(big, dstrain + i * 6, stress_n + i * 6, 0.0, nullptr, s, &epeq, epl, D);
    epeq = sdv_n ? sdv_n[i * 7] : 0.0;
    for (int k = 0; k < 6; ++k) epl[k] = sdv_n ? sdv_n[i * 7 + 1 + k] : 0.0;
  }
  for (int k = 0; k < 6; ++k) stress[i * 6 + k] = s[k];
  if (sdv) {
    sdv[i * 7] = epeq;
    for (int k = 0; k < 6; ++k) sdv[i * 7 + 1 + k] = epl[k];
  }
  if (ddsdde)
    for (int k = 0; k < 36; ++k) ddsdde[i * 36 + k] = D[k];
  if (yielded) yielded[i] = y;
}

// Adjoint sensitivity g_e = -sum_k lambda_k,e^T (Ke/E_e) u_k,e, evaluated as
// -sum_k sum_gp w detJ eps(lambda)^T (D/E_e) eps(u); one thread per element,
// no scatter (the output is per element).
__global__ void __launch_bounds__(128)
    k_adjoint_sens(int32_t E, int64_t n, int nrhs, const double* __restrict__ coords,
                   const int32_t* __restrict__ conn, const double* __restrict__ props, int nprops,
                   const double* __restrict__ U, const double* __restrict__ L, double* __restrict__ g) {
  const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= E) return;
  int64_t nd[8];
  double X[24];
#pragma unroll
  for (int a = 0; a < 8; ++a) {
    nd[a] = conn[e * 8 + a];
#pragma unroll
    for (int i = 0; i < 3; ++i) X[a * 3 + i] = coords[nd[a] * 3 + i];
  }
  double lam, mu;
  lame<double>(1.0, props[e * nprops + 1], lam, mu);
  double acc = 0.0;
  for (int k = 0; k < nrhs; ++k) {
    double ue[24], le[24];
#pragma unroll
    for (int a = 0; a < 8; ++a)
#pragma unroll
      for (int i = 0; i < 3; ++i) {
        ue[a * 3 + i] = U[k * n + 3 * nd[a] + i];
        le[a * 3 + i] = L[k * n + 3 * nd[a] + i];
      }
#pragma unroll 1
    for (int ip = 0; ip < 8; ++ip) {
      double inv[9], eu[6], el[6], s[6];
      const double det = jacobian_inv<double>(X, ip, inv);
      strain_at<double>(inv, ip, ue, eu);
      strain_at<double>(inv, ip, le, el);
      iso_stress<double>(lam, mu, eu, s);
      acc += det * (el[0] * s[0] + el[1] * s[1] + el[2] * s[2] + el[3] * s[3] + el[4] * s[4] + el[5] * s[5]);
    }
  }
  g[e] = -acc;
}

__global__ void k_set_fixed(int32_t nfix, const int32_t* __restrict__ dofs, const double* __restrict__ vals,
                            double* __restrict__ y) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < nfix) y[dofs[i]] = vals ? vals[i] : 0.0;
}

bool g_pairs_ready = false;

int ensure_pairs(Ctx* c) {
  if (g_pairs_ready) return UFC_STATUS_OK;
  PairTable t;
  UFC_CUDA(c, cudaMemcpyToSymbol(c_pair_a, t.a, sizeof(t.a)));
  UFC_CUDA(c, cudaMemcpyToSymbol(c_pair_b, t.b, sizeof(t.b)));
  g_pairs_ready = true;
  return UFC_STATUS_OK;
}

}  // namespace

int assemble(Ctx* c, int build, double* elapsed_ms) {
  if (!c->has_pattern) return fail(c, UFC_STATUS_INVALID, "ufc_elem_compute_ke: pattern not built");
  if (!c->has_material) return fail(c, UFC_STATUS_INVALID, "ufc_elem_compute_ke: material not set");
  const bool tangent = c->mat_model == UFC_MAT_J2_ISO;
  if (tangent && !c->has_trial)
    return fail(c, UFC_STATUS_INVALID,
                "ufc_elem_compute_ke: J2 tangent needs ufc_elem_compute_fint(update_state=1) first");
  UFC_TRY(ensure_pairs(c));
  mg_mark_stale(c);  // (cached CG graphs stay: they are keyed by the arrays and the SpMV form they read)
  cudaEvent_t e0, e1;
  UFC_CUDA(c, cudaEventCreate(&e0));
  UFC_CUDA(c, cudaEventCreate(&e1));
  UFC_CUDA(c, cudaEventRecord(e0, c->stream));
  UFC_CUDA(c, cudaMemsetAsync(c->dev_err, 0, sizeof(int32_t), c->stream));
  const int64_t nv = c->sell_blocks * 9;
  const bool diff = (build & UFC_BUILD_FP32_DIFF) != 0;
  const bool rounded = diff || (build & UFC_BUILD_FP32_ROUNDED) != 0;
  const bool sym = (build & UFC_BUILD_SYMMETRIC) != 0;
  const bool sym32 = sym && (build & (UFC_BUILD_FP32 | UFC_BUILD_FP32_ROUNDED | UFC_BUILD_FP32_DIFF)) != 0;
  if (rounded) build = (build | UFC_BUILD_FP64) & ~UFC_BUILD_FP32;
  if (sym) build |= UFC_BUILD_FP64;
  c->has_sval64 = c->has_sval32 = false;  // values change: symmetric copies are stale
  if (build & UFC_BUILD_FP32) c->val32_diff = false;
  for (int prec = 0; prec < 2; ++prec) {
    const bool want = prec == 0 ? (build & UFC_BUILD_FP64) : (build & UFC_BUILD_FP32);
    if (!want) continue;
    if (prec == 0) {
      if (!c->val64) UFC_TRY(dalloc(c, &c->val64, nv));
      if (!c->dinv64) UFC_TRY(dalloc(c, &c->dinv64, c->n));
      UFC_CUDA(c, cudaMemsetAsync(c->val64, 0, sizeof(double) * nv, c->stream));
    } else {
      if (!c->val32) UFC_TRY(dalloc(c, &c->val32, nv));
      if (!c->dinv32) UFC_TRY(dalloc(c, &c->dinv32, c->n));
      UFC_CUDA(c, cudaMemsetAsync(c->val32, 0, sizeof(float) * nv, c->stream));
    }
    for (int col = 0; col < c->ncol; ++col) {
      const int32_t ne = c->col_off[col + 1] - c->col_off[col];
      if (ne == 0) continue;
      const int32_t* el = c->col_elems + c->col_off[col];
      const int grid = (int)((ne + kWarpsPerCta - 1) / kWarpsPerCta);
      if (prec == 0) {
        if (tangent)
          k_assemble<double, true><<<grid, kWarpsPerCta * 32, 0, c->stream>>>(
              el, ne, c->coords, c->conn, c->props, c->nprops, c->Dt, c->slot, c->fixed, c->val64, c->dev_err);
        else
          k_assemble<double, false><<<grid, kWarpsPerCta * 32, 0, c->stream>>>(
              el, ne, c->coords, c->conn, c->props, c->nprops, nullptr, c->slot, c->fixed, c->val64, c->dev_err);
      } else {
        if (tangent)
          k_assemble<float, true><<<grid, kWarpsPerCta * 32, 0, c->stream>>>(
              el, ne, c->coords, c->conn, c->props, c->nprops, c->Dt, c->slot, c->fixed, c->val32, c->dev_err);
        else
          k_assemble<float, false><<<grid, kWarpsPerCta * 32, 0, c->stream>>>(
              el, ne, c->coords, c->conn, c->props, c->nprops, nullptr, c->slot, c->fixed, c->val32, c->dev_err);
      }
      UFC_CUDA(c, cudaGetLastError());
    }
    if (c->nfix > 0) {
      if (prec == 0)
        k_fix_diag<double><<<grid_for(c->nfix, 256), 256, 0, c->stream>>>(c->nfix, c->fix_dofs, c->dpos, c->val64);
      else
        k_fix_diag<float><<<grid_for(c->nfix, 256), 256, 0, c->stream>>>(c->nfix, c->fix_dofs, c->dpos, c->val32);
      UFC_CUDA(c, cudaGetLastError());
    }
    if (prec == 0) {
      k_dinv<double><<<grid_for(c->n, 256), 256, 0, c->stream>>>(c->N, c->dpos, c->val64, c->dinv64);
      c->has_val64 = true;
    } else {
      k_dinv<float><<<grid_for(c->n, 256), 256, 0, c->stream>>>(c->N, c->dpos, c->val32, c->dinv32);
      c->has_val32 = true;
    }
    UFC_CUDA(c, cudaGetLastError());
  }
  if (rounded) {
    // FP32 values = FP64 values rounded to nearest (Dirichlet rows included)
    if (!c->val32) UFC_TRY(dalloc(c, &c->val32, nv));
    if (!c->dinv32) UFC_TRY(dalloc(c, &c->dinv32, c->n));
    k_round_values<<<(int)std::min<int64_t>(grid_for(nv, 256), 148 * 16), 256, 0, c->stream>>>(nv, c->val64,
                                                                                               c->val32);
    if (diff)
      k_diag_rowsum<<<grid_for(c->N, 128), 128, 0, c->stream>>>(c->N, c->slice_ptr, c->dpos, c->val64, c->val32);
    k_dinv_from64<<<grid_for(c->n, 256), 256, 0, c->stream>>>(c->N, c->dpos, c->val64, c->dinv32);
    UFC_CUDA(c, cudaGetLastError());
    c->has_val32 = true;
    c->val32_diff = diff;
  }
  if (sym) UFC_TRY(pack_symmetric(c, true, sym32));
  UFC_CUDA(c, cudaEventRecord(e1, c->stream));
  UFC_CUDA(c, cudaEventSynchronize(e1));
  float ms = 0.f;
  cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (elapsed_ms) *elapsed_ms = ms;
  return check_dev_err(c, "ufc_elem_compute_ke");
}

int apply_fp64(Ctx* c, const double* x, double* y, bool masked) {
  UFC_CUDA(c, cudaMemsetAsync(y, 0, sizeof(double) * c->n, c->stream));
  for (int col = 0; col < c->ncol; ++col) {
    const int32_t ne = c->col_off[col + 1] - c->col_off[col];
    if (ne == 0) continue;
    k_apply_iso<<<grid_for(ne, 128), 128, 0, c->stream>>>(c->col_elems + c->col_off[col], ne, c->coords, c->conn,
                                                          c->props, c->nprops, x, masked ? c->fixed : nullptr, y,
                                                          c->dev_err);
    UFC_CUDA(c, cudaGetLastError());
    c->launches += 1;
  }
  if (masked && c->nfix > 0) {
    // Eliminated rows are identity rows: y_c = x_c.
    k_set_fixed<<<grid_for(c->nfix, 256), 256, 0, c->stream>>>(c->nfix, c->fix_dofs, nullptr, y);
    UFC_CUDA(c, cudaGetLastError());
    c->launches += 1;
  }
  return UFC_STATUS_OK;
}

// y_c = x_c on fixed DOFs of a masked product (used by the solver's residual).
__global__ void k_copy_fixed(int32_t nfix, const int32_t* __restrict__ dofs, const double* __restrict__ x,
                             double* __restrict__ y) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < nfix) y[dofs[i]] = x[dofs[i]];
}

int apply_fp64_eliminated(Ctx* c, const double* x, double* y) {
  UFC_TRY(apply_fp64(c, x, y, true));
  if (c->nfix > 0) {
    k_copy_fixed<<<grid_for(c->nfix, 256), 256, 0, c->stream>>>(c->nfix, c->fix_dofs, x, y);
    UFC_CUDA(c, cudaGetLastError());
    c->launches += 1;
  }
  return UFC_STATUS_OK;
}

// Newton residual R = f_ext - F_int on free DOFs (0 on fixed) and the norms
// ||R||^2, ||F_int||^2, ||F_ext||^2 into the scalars (RT_Asm_ComputeResidual,
// RT_Asm_Solv.f90:1311-1426; RT_NR_CheckConvergence, RT_Step_NR_Core.f90:231-317).
__global__ void __launch_bounds__(256)
    k_nr_resid(int64_t n, const double* __restrict__ fext, const double* __restrict__ fint,
               const uint8_t* __restrict__ fixed, double* __restrict__ R, CgScalars* __restrict__ scal,
               double* __restrict__ partials) {
  double v[3] = {0.0, 0.0, 0.0}, tot[3];
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const double fe = fext ? fext[i] : 0.0, fi = fint[i];
    const double r = fixed[i] ? 0.0 : fe - fi;
    R[i] = r;
    v[0] += r * r;
    v[1] += fi * fi;
    v[2] += fe * fe;
  }
  if (grid_sum<3>(v, partials, &scal->ticket[4], tot)) {
    scal->nr_rr = tot[0];
    scal->nr_ff = tot[1];
    scal->nr_ee = tot[2];
  }
}

int nr_norms(Ctx* c, const double* fext, const double* fint, double* R) {
  const int g = (int)std::min<int64_t>(grid_for(c->n, 256), 148 * 8);
  k_nr_resid<<<g, 256, 0, c->stream>>>(c->n, fext, fint, c->fixed, R, c->scal, c->partials);
  UFC_CUDA(c, cudaGetLastError());
  return UFC_STATUS_OK;
}

int compute_fint(Ctx* c, const double* u, double* fint, bool update_state) {
  (void)update_state;
  if (!c->has_material) return fail(c, UFC_STATUS_INVALID, "ufc_elem_compute_fint: material not set");
  if (c->ncol == 0) return fail(c, UFC_STATUS_INVALID, "ufc_elem_compute_fint: pattern not built");
  if (c->mat_model != UFC_MAT_J2_ISO) return apply_fp64(c, u, fint, false);
  const int64_t G = (int64_t)c->E * 8;
  k_j2_gp<<<grid_for(G, 128), 128, 0, c->stream>>>(G, c->coords, c->conn, c->props, c->nprops, u, c->u_n, c->sig_n,
                                                   c->epeq_n, c->epl_n, c->sig_t, c->epeq_t, c->epl_t, c->Dt,
                                                   c->dev_err);
  UFC_CUDA(c, cudaGetLastError());
  c->has_trial = true;
  UFC_CUDA(c, cudaMemsetAsync(fint, 0, sizeof(double) * c->n, c->stream));
  for (int col = 0; col < c->ncol; ++col) {
    const int32_t ne = c->col_off[col + 1] - c->col_off[col];
    if (ne == 0) continue;
    k_fint_from_stress<<<grid_for(ne, 128), 128, 0, c->stream>>>(c->col_elems + c->col_off[col], ne, c->coords,
                                                                 c->conn, c->sig_t, fint);
    UFC_CUDA(c, cudaGetLastError());
  }
  return UFC_STATUS_OK;
}

int apply_tangent(Ctx* c, const double* x, double* y) {
  if (!c->has_trial) return fail(c, UFC_STATUS_INVALID, "tangent operator needs a return map first");
  UFC_CUDA(c, cudaMemsetAsync(y, 0, sizeof(double) * c->n, c->stream));
  for (int col = 0; col < c->ncol; ++col) {
    const int32_t ne = c->col_off[col + 1] - c->col_off[col];
    if (ne == 0) continue;
    k_apply_tangent<<<grid_for(ne, 128), 128, 0, c->stream>>>(c->col_elems + c->col_off[col], ne, c->coords, c->conn,
                                                              c->Dt, x, y);
    UFC_CUDA(c, cudaGetLastError());
  }
  return UFC_STATUS_OK;
}

int mat_update_batch(Ctx* c, const ufc_mat_update_arg* a, const double* props, const double* stress_n,
                     const double* dstrain, const double* sdv_n, double* stress, double* sdv, double* ddsdde,
                     int32_t* yielded) {
  if (a->n_points <= 0) return UFC_STATUS_OK;
  k_mat_batch<<<grid_for(a->n_points, 128), 128, 0, c->stream>>>(a->n_points, a->mat_model_id, props, a->nprops,
                                                                 a->props_per_point, stress_n, dstrain, sdv_n, stress,
                                                                 sdv, ddsdde, yielded);
  UFC_CUDA(c, cudaGetLastError());
  return UFC_STATUS_OK;
}

int stress_eval(Ctx* c, const double* u, double* sig, double* vm) {
  const int64_t G = (int64_t)c->E * 8;
  if (c->mat_model == UFC_MAT_J2_ISO)
    k_vm_from_stress<<<grid_for(G, 256), 256, 0, c->stream>>>(G, c->sig_n, sig, vm);
  else
    k_stress_iso<<<grid_for(G, 128), 128, 0, c->stream>>>(G, c->coords, c->conn, c->props, c->nprops, u, sig, vm);
  UFC_CUDA(c, cudaGetLastError());
  return UFC_STATUS_OK;
}

int adjoint_sens(Ctx* c, int nrhs, const double* U, const double* L, double* g) {
  k_adjoint_sens<<<grid_for(c->E, 128), 128, 0, c->stream>>>(c->E, c->n, nrhs, c->coords, c->conn, c->props,
                                                             c->nprops, U, L, g);
  UFC_CUDA(c, cudaGetLastError());
  return UFC_STATUS_OK;
}

}  // namespace ufc
