// Device-side C3D8 and J2 building blocks shared by the element kernels.
//
//   shape functions   ComputeShape_Hex8      ufc_core/L4_PH/Element/PH_Elem_ShapeFunc.f90:329-350 (factor 1/8)
//   Gauss rule        InitGauss3D_Hex        ufc_core/L4_PH/Element/PH_Elem_GaussInt.f90:125-143 (xi fastest)
//   Jacobian, dN/dx   ComputeJacobian        ufc_core/L4_PH/Element/PH_Elem_ShapeFunc.f90:125-183
//   B matrix          ComputeStrainDisplacementMatrix  PH_Elem_ShapeFunc.f90:189-249
//   J2 return map     PH_J2_ComputeTrialStress .. ComputeConsistentTangent
//                     ufc_core/L4_PH/Material/Plast/PH_Mat_Plast_J2_Iso_Core.f90:254-539
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace ufc {

// Abaqus hex node signs: bit0 xi, bit1 eta, bit2 zeta of node a.
__host__ __device__ constexpr int node_sign(int a, int dir) {
  return dir == 0 ? ((a == 1 || a == 2 || a == 5 || a == 6) ? 1 : -1)
         : dir == 1 ? ((a == 2 || a == 3 || a == 6 || a == 7) ? 1 : -1)
                    : (a >= 4 ? 1 : -1);
}

// dN_a/dxi at Gauss point ip of the 2x2x2 rule (points +-1/sqrt(3), weight 1).
template <typename T>
__device__ __forceinline__ void dN_dxi(int ip, int a, T& d0, T& d1, T& d2) {
  const T g = T(0.57735026918962576451);
  const T xi = (ip & 1) ? g : -g, eta = (ip & 2) ? g : -g, zeta = (ip & 4) ? g : -g;
  const T s0 = T(node_sign(a, 0)), s1 = T(node_sign(a, 1)), s2 = T(node_sign(a, 2));
  const T f0 = T(1) + s0 * xi, f1 = T(1) + s1 * eta, f2 = T(1) + s2 * zeta;
  d0 = T(0.125) * s0 * f1 * f2;
  d1 = T(0.125) * s1 * f0 * f2;
  d2 = T(0.125) * s2 * f0 * f1;
}

// Jacobian J_ij = sum_a dN_a/dxi_i x_aj at Gauss point ip; returns detJ and J^-1.
template <typename T>
__device__ __forceinline__ T jacobian_inv(const T* X, int ip, T inv[9]) {
  T J[9];
#pragma unroll
  for (int k = 0; k < 9; ++k) J[k] = T(0);
#pragma unroll
  for (int a = 0; a < 8; ++a) {
    T d0, d1, d2;
    dN_dxi<T>(ip, a, d0, d1, d2);
    const T x = X[a * 3], y = X[a * 3 + 1], z = X[a * 3 + 2];
    J[0] += d0 * x; J[1] += d0 * y; J[2] += d0 * z;
    J[3] += d1 * x; J[4] += d1 * y; J[5] += d1 * z;
    J[6] += d2 * x; J[7] += d2 * y; J[8] += d2 * z;
  }
  const T c0 = J[4] * J[8] - J[5] * J[7];
  const T c1 = J[5] * J[6] - J[3] * J[8];
  const T c2 = J[3] * J[7] - J[4] * J[6];
  const T det = J[0] * c0 + J[1] * c1 + J[2] * c2;
  const T id = T(1) / det;
  inv[0] = c0 * id;
  inv[1] = (J[2] * J[7] - J[1] * J[8]) * id;
  inv[2] = (J[1] * J[5] - J[2] * J[4]) * id;
  inv[3] = c1 * id;
  inv[4] = (J[0] * J[8] - J[2] * J[6]) * id;
  inv[5] = (J[2] * J[3] - J[0] * J[5]) * id;
  inv[6] = c2 * id;
  inv[7] = (J[1] * J[6] - J[0] * J[7]) * id;
  inv[8] = (J[0] * J[4] - J[1] * J[3]) * id;
  return det;
}

// dN_a/dx = J^-1 dN_a/dxi.
template <typename T>
__device__ __forceinline__ void grad_x(const T inv[9], int ip, int a, T g[3]) {
  T d0, d1, d2;
  dN_dxi<T>(ip, a, d0, d1, d2);
  g[0] = inv[0] * d0 + inv[1] * d1 + inv[2] * d2;
  g[1] = inv[3] * d0 + inv[4] * d1 + inv[5] * d2;
  g[2] = inv[6] * d0 + inv[7] * d1 + inv[8] * d2;
}

// Voigt strain (engineering shear) of element displacements ue at Gauss point ip.
template <typename T>
__device__ __forceinline__ void strain_at(const T inv[9], int ip, const T* ue, T eps[6]) {
  T H[9];
#pragma unroll
  for (int k = 0; k < 9; ++k) H[k] = T(0);
#pragma unroll
  for (int a = 0; a < 8; ++a) {
    T g[3];
    grad_x<T>(inv, ip, a, g);
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
      for (int j = 0; j < 3; ++j) H[i * 3 + j] += ue[a * 3 + i] * g[j];
  }
  eps[0] = H[0];
  eps[1] = H[4];
  eps[2] = H[8];
  eps[3] = H[1] + H[3];
  eps[4] = H[5] + H[7];
  eps[5] = H[6] + H[2];
}

// fe += wdet * B^T sigma.
template <typename T>
__device__ __forceinline__ void add_bt_sigma(const T inv[9], int ip, T wdet, const T s[6], T* fe) {
#pragma unroll
  for (int a = 0; a < 8; ++a) {
    T g[3];
    grad_x<T>(inv, ip, a, g);
    fe[a * 3 + 0] += wdet * (g[0] * s[0] + g[1] * s[3] + g[2] * s[5]);
    fe[a * 3 + 1] += wdet * (g[1] * s[1] + g[0] * s[3] + g[2] * s[4]);
    fe[a * 3 + 2] += wdet * (g[2] * s[2] + g[1] * s[4] + g[0] * s[5]);
  }
}

// Isotropic sigma = D eps (PH_Elem_C3D8_ConstMatrix, PH_Elem_C3D8.f90:603-625).
template <typename T>
__device__ __forceinline__ void iso_stress(T lam, T mu, const T e[6], T s[6]) {
  const T tr = lam * (e[0] + e[1] + e[2]);
  s[0] = tr + T(2) * mu * e[0];
  s[1] = tr + T(2) * mu * e[1];
  s[2] = tr + T(2) * mu * e[2];
  s[3] = mu * e[3];
  s[4] = mu * e[4];
  s[5] = mu * e[5];
}

template <typename T>
__device__ __forceinline__ void lame(T E, T nu, T& lam, T& mu) {
  lam = E * nu / ((T(1) + nu) * (T(1) - T(2) * nu));
  mu = E / (T(2) * (T(1) + nu));
}

// J2 radial return with linear isotropic hardening, FP64, textbook
// Simo-Hughes form of the reference's PH_J2_* steps (corrections: G*theta1 on
// the engineering-shear diagonal, n(x)n coefficient 2G*(theta2 - 1 + theta1),
// plastic strain increment dgamma*(3/2)*s/q with engineering shear).
// props = (E, nu, sigma_y0, H).  Returns 1 when the point yielded.
__device__ __forceinline__ int j2_update(const double* props, const double de[6], const double sn[6], double epeq_n,
                                         const double* epl_n, double sig[6], double* epeq, double* epl,
                                         double* Dep /* 36 or nullptr */) {
  const double E = props[0], nu = props[1], sy0 = props[2], H = props[3];
  const double G = E / (2.0 * (1.0 + nu));
  const double K = E / (3.0 * (1.0 - 2.0 * nu));
  const double lam = E * nu / ((1.0 + nu) * (1.0 - 2.0 * nu));
  double st[6];
  const double tr = lam * (de[0] + de[1] + de[2]);
  st[0] = sn[0] + tr + 2.0 * G * de[0];
  st[1] = sn[1] + tr + 2.0 * G * de[1];
  st[2] = sn[2] + tr + 2.0 * G * de[2];
  st[3] = sn[3] + G * de[3];
  st[4] = sn[4] + G * de[4];
  st[5] = sn[5] + G * de[5];
  const double p = (st[0] + st[1] + st[2]) / 3.0;
  const double s[6] = {st[0] - p, st[1] - p, st[2] - p, st[3], st[4], st[5]};
  const double snorm = sqrt(s[0] * s[0] + s[1] * s[1] + s[2] * s[2] + 2.0 * (s[3] * s[3] + s[4] * s[4] + s[5] * s[5]));
  const double q = sqrt(1.5) * snorm;
  const double f = q - (sy0 + H * epeq_n);
  if (!(f > 0.0)) {
#pragma unroll
    for (int i = 0; i < 6; ++i) sig[i] = st[i];
    *epeq = epeq_n;
    if (epl)
#pragma unroll
      for (int i = 0; i < 6; ++i) epl[i] = epl_n ? epl_n[i] : 0.0;
    if (Dep) {
#pragma unroll
      for (int k = 0; k < 36; ++k) Dep[k] = 0.0;
#pragma unroll
      for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) Dep[i * 6 + j] = lam;
#pragma unroll
      for (int i = 0; i < 3; ++i) Dep[i * 7] = lam + 2.0 * G;
#pragma unroll
      for (int i = 3; i < 6; ++i) Dep[i * 7] = G;
    }
    return 0;
  }
  const double dg = f / (3.0 * G + H);
  const double th1 = 1.0 - 3.0 * G * dg / q;
  const double th2 = 3.0 * G / (3.0 * G + H);
  const double thb = th2 - (1.0 - th1);
#pragma unroll
  for (int i = 0; i < 3; ++i) sig[i] = th1 * s[i] + p;
#pragma unroll
  for (int i = 3; i < 6; ++i) sig[i] = th1 * s[i];
  *epeq = epeq_n + dg;
  if (epl)
#pragma unroll
    for (int i = 0; i < 6; ++i) epl[i] = (epl_n ? epl_n[i] : 0.0) + dg * 1.5 * s[i] / q * (i < 3 ? 1.0 : 2.0);
  if (Dep) {
    double n[6];
#pragma unroll
    for (int i = 0; i < 6; ++i) n[i] = s[i] / snorm;
#pragma unroll
    for (int i = 0; i < 6; ++i)
#pragma unroll
      for (int j = 0; j < 6; ++j) {
        double v = -2.0 * G * thb * n[i] * n[j];
        if (i < 3 && j < 3) v += K - 2.0 * G * th1 / 3.0;
        if (i == j) v += (i < 3 ? 2.0 : 1.0) * G * th1;
        Dep[i * 6 + j] = v;
      }
  }
  return 1;
}

// SELL-32 value index of component c (0..8, row-major 3x3) of stored block P.
__host__ __device__ __forceinline__ int64_t vpos(int64_t P, int c) {
  return 9 * (P & ~int64_t(31)) + 32 * c + (P & 31);
}

}  // namespace ufc
