/*
 * ufc_oracle.c -- CPU FP64 restatement of UFC's implicit-static C3D8 hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker for the CUDA library
 * (parity tests, smoke check, and the timed CPU baseline of bench.py).  It is
 * never linked into, called by, or used as a fallback for the product path.
 *
 * Parity pinning: the reference (Fortran, ufc_core) cannot be compiled here
 * (no Fortran compiler; its hot-path modules are excluded from its own build).
 * This restatement is pinned against the reference's own known-answer tests,
 * restated as golden fixtures under tests/golden/:
 *   - ufc_core/Testing/test_defn_invoke_umat.f90 (sigma11 = 282.69230769230769)
 *   - tests/ufc_core/test_c3d8_uniaxial.f90 (unit cube, u = sigma/E = 5e-4)
 *   - tests/HARNESS_Elem_C3D8_PatchTest.f90 (symmetry, rigid-body null space, patch)
 *   - tests/integration/E2E_C2_02_Uniaxial_J2Plastic.f90 (J2 uniaxial history)
 *   - tests/HARNESS_Mat_Plastic_VonMises.f90 (perfect plasticity return)
 *   - tests/integration/test_elem_mat_ip_loop.f90 (finite-difference tangent)
 *   - tests/integration/test_assembly_chain.f90 (symmetry, force balance)
 *
 * Conventions (all follow the reference):
 *   - Hex8 node order is Abaqus order: bottom face 1-4, top face 5-8
 *     (PH_Elem_ShapeFunc.f90:329-350), N_a = 1/8 (1+xi_a xi)(1+eta_a eta)(1+zeta_a zeta).
 *   - 2x2x2 Gauss rule, points +-1/sqrt(3), weight 1, xi fastest
 *     (PH_Elem_GaussInt.f90:125-143).
 *   - Voigt order (xx, yy, zz, gxy, gyz, gzx) with engineering shear strain
 *     (PH_Elem_ShapeFunc.f90:189-249).
 *   - DOF numbering eq = 3*node + comp, node-major, 0-based here
 *     (RT_Asm_DofMap.f90:172-249, :641-654).
 *   - CSR pattern: per row the sorted unique set of coupled columns
 *     (RT_Solv_Sparse.f90:336-445, RT_CSR_FromTripletMerged).
 *   - Jacobi-PCG: iter_pcg (NM_Solv_IterSolver.f90:713-846) with the Jacobi
 *     preconditioner of NM_Solv_LinPrec.f90:312-353.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define ORC_OK 0
#define ORC_INVALID 1
#define ORC_ERROR 2
#define ORC_NOT_CONVERGED 4

static const int kSign[8][3] = {{-1, -1, -1}, {1, -1, -1}, {1, 1, -1}, {-1, 1, -1},
                                {-1, -1, 1},  {1, -1, 1},  {1, 1, 1},  {-1, 1, 1}};

int orc_num_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

void orc_set_threads(int n) {
#ifdef _OPENMP
  if (n > 0) omp_set_num_threads(n);
#else
  (void)n;
#endif
}

/* Gauss point ip (0..7) of the 2x2x2 rule, xi fastest (PH_Elem_GaussInt.f90:135-139). */
void orc_gauss_point(int ip, double xi[3]) {
  const double g = 1.0 / sqrt(3.0);
  xi[0] = (ip & 1) ? g : -g;
  xi[1] = (ip & 2) ? g : -g;
  xi[2] = (ip & 4) ? g : -g;
}

/* Trilinear shape functions and parametric derivatives dN[a*3+i] = dN_a/dxi_i
 * (ComputeShape_Hex8, PH_Elem_ShapeFunc.f90:329-350, factor 0.125). */
void orc_hex8_shape(const double xi[3], double N[8], double dN[24]) {
  for (int a = 0; a < 8; ++a) {
    double f0 = 1.0 + kSign[a][0] * xi[0];
    double f1 = 1.0 + kSign[a][1] * xi[1];
    double f2 = 1.0 + kSign[a][2] * xi[2];
    if (N) N[a] = 0.125 * f0 * f1 * f2;
    dN[a * 3 + 0] = 0.125 * kSign[a][0] * f1 * f2;
    dN[a * 3 + 1] = 0.125 * kSign[a][1] * f0 * f2;
    dN[a * 3 + 2] = 0.125 * kSign[a][2] * f0 * f1;
  }
}

/* Jacobian J_ij = sum_k dN_k/dxi_i x_kj, detJ and dN/dx = J^-1 dN/dxi
 * (ComputeJacobian, PH_Elem_ShapeFunc.f90:125-183).  X is [8][3].
 * Returns detJ; dNx[a*3+i] = dN_a/dx_i. */
double orc_hex8_grad(const double X[24], const double xi[3], double dNx[24]) {
  double dN[24], J[9] = {0};
  orc_hex8_shape(xi, NULL, dN);
  for (int k = 0; k < 8; ++k)
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) J[i * 3 + j] += dN[k * 3 + i] * X[k * 3 + j];
  double det = J[0] * (J[4] * J[8] - J[5] * J[7]) - J[1] * (J[3] * J[8] - J[5] * J[6]) +
               J[2] * (J[3] * J[7] - J[4] * J[6]);
  double inv[9];
  inv[0] = (J[4] * J[8] - J[5] * J[7]) / det;
  inv[1] = (J[2] * J[7] - J[1] * J[8]) / det;
  inv[2] = (J[1] * J[5] - J[2] * J[4]) / det;
  inv[3] = (J[5] * J[6] - J[3] * J[8]) / det;
  inv[4] = (J[0] * J[8] - J[2] * J[6]) / det;
  inv[5] = (J[2] * J[3] - J[0] * J[5]) / det;
  inv[6] = (J[3] * J[7] - J[4] * J[6]) / det;
  inv[7] = (J[1] * J[6] - J[0] * J[7]) / det;
  inv[8] = (J[0] * J[4] - J[1] * J[3]) / det;
  for (int a = 0; a < 8; ++a)
    for (int i = 0; i < 3; ++i) {
      double s = 0.0;
      for (int j = 0; j < 3; ++j) s += inv[i * 3 + j] * dN[a * 3 + j];
      dNx[a * 3 + i] = s;
    }
  return det;
}

/* B matrix [6][24] (ComputeStrainDisplacementMatrix, PH_Elem_ShapeFunc.f90:189-249). */
static void orc_bmat(const double dNx[24], double B[6][24]) {
  memset(B, 0, sizeof(double) * 6 * 24);
  for (int a = 0; a < 8; ++a) {
    double x = dNx[a * 3], y = dNx[a * 3 + 1], z = dNx[a * 3 + 2];
    int c = a * 3;
    B[0][c] = x; B[3][c] = y; B[5][c] = z;
    B[1][c + 1] = y; B[3][c + 1] = x; B[4][c + 1] = z;
    B[2][c + 2] = z; B[4][c + 2] = y; B[5][c + 2] = x;
  }
}

/* Isotropic elastic D (PH_Elem_C3D8_ConstMatrix, PH_Elem_C3D8.f90:603-625). */
void orc_iso_D(double E, double nu, double D[36]) {
  double lam = E * nu / ((1.0 + nu) * (1.0 - 2.0 * nu));
  double mu = E / (2.0 * (1.0 + nu));
  memset(D, 0, sizeof(double) * 36);
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) D[i * 6 + j] = lam;
  for (int i = 0; i < 3; ++i) D[i * 6 + i] = lam + 2.0 * mu;
  for (int i = 3; i < 6; ++i) D[i * 6 + i] = mu;
}

/* Element stiffness Ke = sum_gp w detJ B^T D B (PH_Elem_Core_Compute_Ke,
 * PH_Elem_Core.f90:95-166).  D is one [6][6] matrix per element (Dgp == NULL
 * path) or one per Gauss point when Dgp is given ([8][36]).
 * Returns ORC_ERROR on detJ <= 0 (ComputeJacobian rejects it). */
int orc_c3d8_ke(const double X[24], const double D[36], const double* Dgp, double Ke[576]) {
  memset(Ke, 0, sizeof(double) * 576);
  for (int ip = 0; ip < 8; ++ip) {
    double xi[3], dNx[24], B[6][24], DB[6][24];
    orc_gauss_point(ip, xi);
    double det = orc_hex8_grad(X, xi, dNx);
    if (!(det > 0.0)) return ORC_ERROR;
    const double* Dm = Dgp ? Dgp + ip * 36 : D;
    orc_bmat(dNx, B);
    for (int i = 0; i < 6; ++i)
      for (int j = 0; j < 24; ++j) {
        double s = 0.0;
        for (int k = 0; k < 6; ++k) s += Dm[i * 6 + k] * B[k][j];
        DB[i][j] = s;
      }
    for (int i = 0; i < 24; ++i)
      for (int j = 0; j < 24; ++j) {
        double s = 0.0;
        for (int k = 0; k < 6; ++k) s += B[k][i] * DB[k][j];
        Ke[i * 24 + j] += det * s; /* weight 1 */
      }
  }
  return ORC_OK;
}

/* Strain at Gauss point ip for element displacements ue[24]; returns detJ. */
double orc_c3d8_strain(const double X[24], const double ue[24], int ip, double eps[6], double dNx[24]) {
  double xi[3];
  orc_gauss_point(ip, xi);
  double det = orc_hex8_grad(X, xi, dNx);
  double g[3][3] = {{0}}; /* g[i][j] = du_i/dx_j */
  for (int a = 0; a < 8; ++a)
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) g[i][j] += ue[a * 3 + i] * dNx[a * 3 + j];
  eps[0] = g[0][0];
  eps[1] = g[1][1];
  eps[2] = g[2][2];
  eps[3] = g[0][1] + g[1][0];
  eps[4] = g[1][2] + g[2][1];
  eps[5] = g[2][0] + g[0][2];
  return det;
}

/* f_e += w detJ B^T sigma (FormIntForceFromStress, PH_Elem_C3D8.f90:782-798). */
static void orc_add_btsig(const double dNx[24], double wdet, const double s[6], double fe[24]) {
  for (int a = 0; a < 8; ++a) {
    double x = dNx[a * 3], y = dNx[a * 3 + 1], z = dNx[a * 3 + 2];
    fe[a * 3 + 0] += wdet * (x * s[0] + y * s[3] + z * s[5]);
    fe[a * 3 + 1] += wdet * (y * s[1] + x * s[3] + z * s[4]);
    fe[a * 3 + 2] += wdet * (z * s[2] + y * s[4] + x * s[5]);
  }
}

/* von Mises equivalent stress (PH_Elem_C3D8_EvalVonMises, PH_Elem_C3D8.f90:2768-2780). */
double orc_von_mises(const double s[6]) {
  double p = (s[0] + s[1] + s[2]) / 3.0;
  double j2 = 0.5 * ((s[0] - p) * (s[0] - p) + (s[1] - p) * (s[1] - p) + (s[2] - p) * (s[2] - p)) +
              s[3] * s[3] + s[4] * s[4] + s[5] * s[5];
  return sqrt(3.0 * (j2 > 0.0 ? j2 : 0.0));
}

/* J2 radial return with linear isotropic hardening and the consistent tangent.
 * Follows PH_J2_ComputeTrialStress / ComputeYieldCheck / ApplyRadialReturn /
 * ComputeConsistentTangent (PH_Mat_Plast_J2_Iso_Core.f90:254-539) with the
 * textbook (Simo-Hughes) corrections:
 *   - the deviatoric identity carries G*theta1 (not 2G*theta1) on the
 *     engineering-shear diagonal (reference :520-523);
 *   - the n(x)n coefficient is -2G*(theta2 - (1 - theta1)) (Simo-Hughes box 3.2;
 *     the reference writes -2G*(theta1 - theta2), :527-531);
 *   - the plastic strain increment is dgamma*(3/2)*s/q, stored with engineering
 *     shear (reference :445 omits sqrt(3/2)).
 * props = [E, nu, sigma_y0, H].  For linear hardening the local Newton of the
 * reference converges in one step to dgamma = f/(3G+H), used here directly.
 * Returns 1 when the point yielded, 0 when elastic. */
int orc_j2_update(const double props[4], const double deps[6], const double sig_n[6], double epeq_n,
                  const double epl_n[6], double sig[6], double* epeq, double epl[6], double Dep[36]) {
  double E = props[0], nu = props[1], sy0 = props[2], H = props[3];
  double G = E / (2.0 * (1.0 + nu));
  double K = E / (3.0 * (1.0 - 2.0 * nu));
  double D[36];
  orc_iso_D(E, nu, D);
  double st[6];
  for (int i = 0; i < 6; ++i) {
    double s = sig_n[i];
    for (int j = 0; j < 6; ++j) s += D[i * 6 + j] * deps[j];
    st[i] = s;
  }
  double p = (st[0] + st[1] + st[2]) / 3.0;
  double s[6] = {st[0] - p, st[1] - p, st[2] - p, st[3], st[4], st[5]};
  double snorm = sqrt(s[0] * s[0] + s[1] * s[1] + s[2] * s[2] + 2.0 * (s[3] * s[3] + s[4] * s[4] + s[5] * s[5]));
  double q = sqrt(1.5) * snorm;
  double f = q - (sy0 + H * epeq_n);
  if (!(f > 0.0)) {
    memcpy(sig, st, sizeof(double) * 6);
    *epeq = epeq_n;
    memcpy(epl, epl_n, sizeof(double) * 6);
    memcpy(Dep, D, sizeof(double) * 36);
    return 0;
  }
  double dg = f / (3.0 * G + H);
  double th1 = 1.0 - 3.0 * G * dg / q;
  double th2 = 3.0 * G / (3.0 * G + H);
  double thb = th2 - (1.0 - th1);
  for (int i = 0; i < 3; ++i) sig[i] = th1 * s[i] + p;
  for (int i = 3; i < 6; ++i) sig[i] = th1 * s[i];
  *epeq = epeq_n + dg;
  for (int i = 0; i < 6; ++i) epl[i] = epl_n[i] + dg * 1.5 * s[i] / q * (i < 3 ? 1.0 : 2.0);
  double n[6];
  for (int i = 0; i < 6; ++i) n[i] = s[i] / snorm;
  memset(Dep, 0, sizeof(double) * 36);
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) Dep[i * 6 + j] = K - 2.0 * G * th1 / 3.0;
  for (int i = 0; i < 3; ++i) Dep[i * 6 + i] += 2.0 * G * th1;
  for (int i = 3; i < 6; ++i) Dep[i * 6 + i] += G * th1;
  for (int i = 0; i < 6; ++i)
    for (int j = 0; j < 6; ++j) Dep[i * 6 + j] -= 2.0 * G * thb * n[i] * n[j];
  return 1;
}

/* ---------------------------------------------------------------- mesh graph */

/* node -> element adjacency (CSR, elements ascending per node). */
static void orc_node_elems(int32_t N, int32_t E, const int32_t* conn, int32_t** ptr_out, int32_t** lst_out) {
  int32_t* ptr = (int32_t*)calloc((size_t)N + 1, sizeof(int32_t));
  for (int64_t e = 0; e < E; ++e)
    for (int a = 0; a < 8; ++a) ptr[conn[e * 8 + a] + 1]++;
  for (int32_t i = 0; i < N; ++i) ptr[i + 1] += ptr[i];
  int32_t* fill = (int32_t*)malloc(sizeof(int32_t) * (size_t)N);
  memcpy(fill, ptr, sizeof(int32_t) * (size_t)N);
  int32_t* lst = (int32_t*)malloc(sizeof(int32_t) * (size_t)ptr[N] + 4);
  for (int64_t e = 0; e < E; ++e)
    for (int a = 0; a < 8; ++a) {
      int32_t nd = conn[e * 8 + a];
      /* an element listing the same node twice is rejected by callers */
      lst[fill[nd]++] = (int32_t)e;
    }
  free(fill);
  *ptr_out = ptr;
  *lst_out = lst;
}

static int cmp_i32(const void* a, const void* b) {
  int32_t x = *(const int32_t*)a, y = *(const int32_t*)b;
  return (x > y) - (x < y);
}

/* Sorted unique neighbour nodes of node i; returns count. */
static int orc_node_neighbors(int32_t i, const int32_t* conn, const int32_t* nptr, const int32_t* nlst,
                              int32_t* buf) {
  int cnt = 0;
  for (int32_t k = nptr[i]; k < nptr[i + 1]; ++k) {
    int32_t e = nlst[k];
    for (int a = 0; a < 8; ++a) buf[cnt++] = conn[(int64_t)e * 8 + a];
  }
  qsort(buf, (size_t)cnt, sizeof(int32_t), cmp_i32);
  int u = 0;
  for (int k = 0; k < cnt; ++k)
    if (u == 0 || buf[k] != buf[u - 1]) buf[u++] = buf[k];
  return u;
}

/* Canonical scalar CSR pattern (0-based).  row_ptr has 3N+1 entries; col may be
 * NULL to only count.  Returns nnz or -1 when a node's valence exceeds 64
 * elements.  Equivalent to RT_CSR_FromTripletMerged (RT_Solv_Sparse.f90:336-445)
 * applied to every element's 24x24 triplets, without the |Ke|<=1e-15 drop
 * (RT_Asm_Solv.f90:1956), which would make the pattern value-dependent. */
int64_t orc_csr_pattern(int32_t N, int32_t E, const int32_t* conn, int64_t* row_ptr, int32_t* col) {
  int32_t *nptr, *nlst;
  orc_node_elems(N, E, conn, &nptr, &nlst);
  int32_t maxval = 0;
  for (int32_t i = 0; i < N; ++i)
    if (nptr[i + 1] - nptr[i] > maxval) maxval = nptr[i + 1] - nptr[i];
  if (maxval > 64) {
    free(nptr); free(nlst);
    return -1;
  }
  int32_t* cnt = (int32_t*)malloc(sizeof(int32_t) * (size_t)N);
#pragma omp parallel
  {
    int32_t buf[64 * 8];
#pragma omp for schedule(static)
    for (int32_t i = 0; i < N; ++i) cnt[i] = orc_node_neighbors(i, conn, nptr, nlst, buf);
  }
  row_ptr[0] = 0;
  for (int32_t i = 0; i < N; ++i)
    for (int r = 0; r < 3; ++r) row_ptr[3 * (int64_t)i + r + 1] = row_ptr[3 * (int64_t)i + r] + 3 * (int64_t)cnt[i];
  if (col) {
#pragma omp parallel
    {
      int32_t buf[64 * 8];
#pragma omp for schedule(static)
      for (int32_t i = 0; i < N; ++i) {
        int u = orc_node_neighbors(i, conn, nptr, nlst, buf);
        for (int r = 0; r < 3; ++r) {
          int64_t o = row_ptr[3 * (int64_t)i + r];
          for (int k = 0; k < u; ++k)
            for (int c = 0; c < 3; ++c) col[o + 3 * k + c] = 3 * buf[k] + c;
        }
      }
    }
  }
  int64_t nnz = row_ptr[3 * (int64_t)N];
  free(cnt); free(nptr); free(nlst);
  return nnz;
}

/* Greedy element colouring: no two elements of one colour share a node
 * (RT_AsmColor_Build, RT_Asm_Color.f90:36-182).  Returns the colour count. */
int orc_color_elements(int32_t N, int32_t E, const int32_t* conn, int32_t* color) {
  int32_t *nptr, *nlst;
  orc_node_elems(N, E, conn, &nptr, &nlst);
  int ncol = 0;
  for (int64_t e = 0; e < E; ++e) {
    uint64_t used[4] = {0, 0, 0, 0};
    for (int a = 0; a < 8; ++a) {
      int32_t nd = conn[e * 8 + a];
      for (int32_t k = nptr[nd]; k < nptr[nd + 1]; ++k) {
        int32_t f = nlst[k];
        if (f < e) used[color[f] >> 6] |= 1ull << (color[f] & 63);
      }
    }
    int c = 0;
    while (c < 256 && (used[c >> 6] >> (c & 63)) & 1ull) ++c;
    color[e] = c;
    if (c + 1 > ncol) ncol = c + 1;
  }
  free(nptr); free(nlst);
  return ncol;
}

static int64_t orc_find(const int64_t* row_ptr, const int32_t* col, int64_t row, int32_t c) {
  int64_t lo = row_ptr[row], hi = row_ptr[row + 1] - 1;
  while (lo <= hi) {
    int64_t mid = (lo + hi) >> 1;
    if (col[mid] < c) lo = mid + 1;
    else if (col[mid] > c) hi = mid - 1;
    else return mid;
  }
  return -1;
}

static void orc_gather_X(const double* coords, const int32_t* conn, int64_t e, double X[24]) {
  for (int a = 0; a < 8; ++a)
    for (int i = 0; i < 3; ++i) X[a * 3 + i] = coords[(int64_t)conn[e * 8 + a] * 3 + i];
}

/* Global stiffness assembly into the canonical CSR (RT_Asm_GlobalStiffness,
 * RT_Asm_Solv.f90:1762-1985).  Material per element: props[e*stride + 0..1] =
 * (E, nu) when Dgp == NULL, else Dgp holds one 6x6 tangent per Gauss point
 * ([E][8][36]).  Dirichlet DOFs (fixed[dof] != 0) are eliminated symmetrically:
 * their rows and columns are zero and the diagonal is 1 (replacing the penalty
 * of RT_Asm_ApplyBC_Displacement_Penalty, RT_Asm_Solv.f90:427-483).
 * Elements are added colour by colour, in ascending element order inside a
 * colour.  Returns ORC_ERROR on a non-positive Jacobian. */
int orc_assemble(int32_t N, int32_t E, const double* coords, const int32_t* conn, const double* props,
                 int32_t prop_stride, const double* Dgp, const uint8_t* fixed, const int32_t* color, int ncol,
                 const int64_t* row_ptr, const int32_t* col, double* val) {
  int64_t nnz = row_ptr[3 * (int64_t)N];
  memset(val, 0, sizeof(double) * (size_t)nnz);
  int err = 0;
  for (int c = 0; c < ncol; ++c) {
#pragma omp parallel for schedule(dynamic, 64) reduction(| : err)
    for (int64_t e = 0; e < E; ++e) {
      if (color[e] != c) continue;
      double X[24], D[36], Ke[576];
      orc_gather_X(coords, conn, e, X);
      if (!Dgp) orc_iso_D(props[e * prop_stride], props[e * prop_stride + 1], D);
      if (orc_c3d8_ke(X, D, Dgp ? Dgp + e * 288 : NULL, Ke) != ORC_OK) {
        err |= 1;
        continue;
      }
      for (int a = 0; a < 8; ++a)
        for (int r = 0; r < 3; ++r) {
          int64_t row = 3 * (int64_t)conn[e * 8 + a] + r;
          if (fixed[row]) continue;
          for (int b = 0; b < 8; ++b)
            for (int s = 0; s < 3; ++s) {
              int32_t cc = 3 * conn[e * 8 + b] + s;
              if (fixed[cc]) continue;
              int64_t k = orc_find(row_ptr, col, row, cc);
              val[k] += Ke[(a * 3 + r) * 24 + b * 3 + s];
            }
        }
    }
  }
  for (int64_t row = 0; row < 3 * (int64_t)N; ++row)
    if (fixed[row]) val[orc_find(row_ptr, col, row, (int32_t)row)] = 1.0;
  return err ? ORC_ERROR : ORC_OK;
}

/* y = K x over the CSR (RT_CSRMatrix_matvec, NM_Assem_Sparse.f90:199-212). */
void orc_spmv(int64_t n, const int64_t* row_ptr, const int32_t* col, const double* val, const double* x, double* y) {
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < n; ++i) {
    double s = 0.0;
    for (int64_t k = row_ptr[i]; k < row_ptr[i + 1]; ++k) s += val[k] * x[col[k]];
    y[i] = s;
  }
}

static double orc_dot(int64_t n, const double* a, const double* b) {
  double s = 0.0;
#pragma omp parallel for schedule(static) reduction(+ : s)
  for (int64_t i = 0; i < n; ++i) s += a[i] * b[i];
  return s;
}

/* Jacobi-PCG, iter_pcg semantics (NM_Solv_IterSolver.f90:713-846):
 * tol = max(rtol*||b||, atol) on the recursively updated residual; Jacobi
 * diag_inv = 1/K_ii, or 1 when |K_ii| <= 1e-30 (NM_Solv_LinPrec.f90:312-353).
 * x is the initial guess on entry.  max_iter <= 0 means "time exactly
 * |max_iter| iterations" (no convergence exit), used by the CPU baseline.
 * When mark_rtol > 0, the first iterate whose recursive residual is at most
 * mark_rtol*||b|| is copied to x_mark, with its iteration count and the wall
 * time from entry (setup included, the copy excluded): the run an iter_pcg
 * call with rtol = mark_rtol would have made, taken on the way to rtol.
 * Returns ORC_OK, ORC_NOT_CONVERGED or ORC_ERROR (breakdown). */
static int pcg_impl(int64_t n, const int64_t* row_ptr, const int32_t* col, const double* val, const double* b,
                    double* x, double rtol, double atol, int max_iter, int* iters, double* res_final,
                    double* res_init, double mark_rtol, double* x_mark, int* it_mark, double* t_mark) {
  const double t_start = omp_get_wtime();
  double mark_tol = -1.0;
  if (it_mark) *it_mark = -1;
  if (t_mark) *t_mark = -1.0;
  double* r = (double*)malloc(sizeof(double) * (size_t)n);
  double* z = (double*)malloc(sizeof(double) * (size_t)n);
  double* p = (double*)malloc(sizeof(double) * (size_t)n);
  double* q = (double*)malloc(sizeof(double) * (size_t)n);
  double* dinv = (double*)malloc(sizeof(double) * (size_t)n);
  int fixed_count = max_iter <= 0;
  int maxit = fixed_count ? -max_iter : max_iter;
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < n; ++i) {
    double d = 0.0;
    for (int64_t k = row_ptr[i]; k < row_ptr[i + 1]; ++k)
      if (col[k] == i) d = val[k];
    dinv[i] = fabs(d) > 1e-30 ? 1.0 / d : 1.0;
  }
  orc_spmv(n, row_ptr, col, val, x, r);
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < n; ++i) r[i] = b[i] - r[i];
  double bnorm = sqrt(orc_dot(n, b, b));
  double rnorm = sqrt(orc_dot(n, r, r));
  if (res_init) *res_init = rnorm;
  if (bnorm < 1e-30) bnorm = 1.0;
  double tol = rtol * bnorm > atol ? rtol * bnorm : atol;
  if (mark_rtol > 0.0 && x_mark) mark_tol = mark_rtol * bnorm;
  int status = ORC_NOT_CONVERGED, k = 0;
  if (rnorm <= tol && !fixed_count) {
    status = ORC_OK;
    goto done;
  }
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < n; ++i) {
    z[i] = dinv[i] * r[i];
    p[i] = z[i];
  }
  double rho = orc_dot(n, r, z);
  for (k = 1; k <= maxit; ++k) {
    orc_spmv(n, row_ptr, col, val, p, q);
    double pq = orc_dot(n, p, q);
    if (fabs(pq) < 1e-300) {
      status = ORC_ERROR;
      break;
    }
    double alpha = rho / pq;
    double rr = 0.0;
#pragma omp parallel for schedule(static) reduction(+ : rr)
    for (int64_t i = 0; i < n; ++i) {
      x[i] += alpha * p[i];
      r[i] -= alpha * q[i];
      rr += r[i] * r[i];
    }
    rnorm = sqrt(rr);
    if (mark_tol > 0.0 && rnorm <= mark_tol) {
      if (t_mark) *t_mark = omp_get_wtime() - t_start;
      if (it_mark) *it_mark = k;
      memcpy(x_mark, x, sizeof(double) * (size_t)n);
      mark_tol = -1.0;
    }
    if (rnorm <= tol && !fixed_count) {
      status = ORC_OK;
      break;
    }
    double rho_new = 0.0;
#pragma omp parallel for schedule(static) reduction(+ : rho_new)
    for (int64_t i = 0; i < n; ++i) {
      z[i] = dinv[i] * r[i];
      rho_new += r[i] * z[i];
    }
    if (fabs(rho) < 1e-300) {
      status = ORC_ERROR;
      break;
    }
    double beta = rho_new / rho;
    rho = rho_new;
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) p[i] = z[i] + beta * p[i];
  }
  if (k > maxit) k = maxit;
done:
  if (iters) *iters = k;
  if (res_final) *res_final = rnorm;
  free(r); free(z); free(p); free(q); free(dinv);
  return status;
}

int orc_pcg(int64_t n, const int64_t* row_ptr, const int32_t* col, const double* val, const double* b, double* x,
            double rtol, double atol, int max_iter, int* iters, double* res_final, double* res_init) {
  return pcg_impl(n, row_ptr, col, val, b, x, rtol, atol, max_iter, iters, res_final, res_init, 0.0, NULL, NULL,
                  NULL);
}

int orc_pcg_marked(int64_t n, const int64_t* row_ptr, const int32_t* col, const double* val, const double* b,
                   double* x, double rtol, int max_iter, double mark_rtol, double* x_mark, int* it_mark,
                   double* t_mark, int* iters, double* res_final) {
  return pcg_impl(n, row_ptr, col, val, b, x, rtol, 0.0, max_iter, iters, res_final, NULL, mark_rtol, x_mark,
                  it_mark, t_mark);
}

/* Internal force F_int = sum_e sum_gp w detJ B^T sigma (PH_Elem_C3D8_IntForce,
 * PH_Elem_C3D8.f90:734-757), scattered colour by colour.
 *   mode 0: linear elastic, sigma = D(E_e, nu_e) eps(u)
 *   mode 1: J2, sigma from orc_j2_update(props_e, eps(u - u_n) per Gauss point)
 *           with committed state (sig_n, epeq_n, epl_n) and trial outputs
 *           (sig_t, epeq_t, epl_t, Dgp_t); all Gauss-point arrays are [E][8][...].
 * fint has 3N entries and is overwritten. */
int orc_fint(int32_t N, int32_t E, const double* coords, const int32_t* conn, const double* props, int32_t prop_stride,
             int mode, const double* u, const double* u_n, const double* sig_n, const double* epeq_n,
             const double* epl_n, double* sig_t, double* epeq_t, double* epl_t, double* Dgp_t, const int32_t* color,
             int ncol, double* fint) {
  memset(fint, 0, sizeof(double) * 3 * (size_t)N);
  int err = 0;
  for (int c = 0; c < ncol; ++c) {
#pragma omp parallel for schedule(dynamic, 64) reduction(| : err)
    for (int64_t e = 0; e < E; ++e) {
      if (color[e] != c) continue;
      double X[24], ue[24], fe[24] = {0};
      orc_gather_X(coords, conn, e, X);
      const double* pe = props + e * prop_stride;
      for (int a = 0; a < 8; ++a)
        for (int i = 0; i < 3; ++i) {
          int64_t d = 3 * (int64_t)conn[e * 8 + a] + i;
          ue[a * 3 + i] = mode == 1 ? u[d] - u_n[d] : u[d];
        }
      for (int ip = 0; ip < 8; ++ip) {
        double eps[6], dNx[24], s[6];
        double det = orc_c3d8_strain(X, ue, ip, eps, dNx);
        if (!(det > 0.0)) err |= 1;
        int64_t g = e * 8 + ip;
        if (mode == 0) {
          double D[36];
          orc_iso_D(pe[0], pe[1], D);
          for (int i = 0; i < 6; ++i) {
            double t = 0.0;
            for (int j = 0; j < 6; ++j) t += D[i * 6 + j] * eps[j];
            s[i] = t;
          }
        } else {
          orc_j2_update(pe, eps, sig_n + g * 6, epeq_n[g], epl_n + g * 6, s, epeq_t + g, epl_t + g * 6, Dgp_t + g * 36);
          memcpy(sig_t + g * 6, s, sizeof(double) * 6);
        }
        orc_add_btsig(dNx, det, s, fe);
      }
      for (int a = 0; a < 8; ++a)
        for (int i = 0; i < 3; ++i) fint[3 * (int64_t)conn[e * 8 + a] + i] += fe[a * 3 + i];
    }
  }
  return err ? ORC_ERROR : ORC_OK;
}

/* Gauss-point stress and von Mises for a linear-elastic solution: out_sig
 * [E][8][6] (may be NULL), out_vm [E][8]. */
void orc_elastic_stress(int32_t E, const double* coords, const int32_t* conn, const double* props, int32_t prop_stride,
                        const double* u, double* out_sig, double* out_vm) {
#pragma omp parallel for schedule(static)
  for (int64_t e = 0; e < E; ++e) {
    double X[24], ue[24], D[36];
    orc_gather_X(coords, conn, e, X);
    for (int a = 0; a < 8; ++a)
      for (int i = 0; i < 3; ++i) ue[a * 3 + i] = u[3 * (int64_t)conn[e * 8 + a] + i];
    orc_iso_D(props[e * prop_stride], props[e * prop_stride + 1], D);
    for (int ip = 0; ip < 8; ++ip) {
      double eps[6], dNx[24], s[6];
      orc_c3d8_strain(X, ue, ip, eps, dNx);
      for (int i = 0; i < 6; ++i) {
        double t = 0.0;
        for (int j = 0; j < 6; ++j) t += D[i * 6 + j] * eps[j];
        s[i] = t;
      }
      if (out_sig) memcpy(out_sig + (e * 8 + ip) * 6, s, sizeof(double) * 6);
      out_vm[e * 8 + ip] = orc_von_mises(s);
    }
  }
}

/* Adjoint sensitivity with respect to the element modulus:
 * g_e = -sum_k lambda_k,e^T (dKe/dE_e) u_k,e = -sum_k lambda_k,e^T (Ke/E_e) u_k,e,
 * for nrhs pairs stored column-major ([nrhs][3N]).  The reference adjoint is a
 * stub (NM_AI_Adjoint_Solve, NM_AI_AdjointAlgo.f90:116-136, sets lambda = 0);
 * this follows the formulas of its contract: K u = F, K^T lambda = dJ/du,
 * dJ/dtheta = -lambda^T dR/dtheta. */
void orc_adjoint_dJdE(int32_t N, int32_t E, const double* coords, const int32_t* conn, const double* props,
                      int32_t prop_stride, int nrhs, const double* u, const double* lam, double* g) {
#pragma omp parallel for schedule(static)
  for (int64_t e = 0; e < E; ++e) {
    double X[24], D[36], Ke[576];
    orc_gather_X(coords, conn, e, X);
    orc_iso_D(1.0, props[e * prop_stride + 1], D);
    orc_c3d8_ke(X, D, NULL, Ke);
    double acc = 0.0;
    for (int k = 0; k < nrhs; ++k) {
      double ue[24], le[24];
      for (int a = 0; a < 8; ++a)
        for (int i = 0; i < 3; ++i) {
          int64_t d = 3 * (int64_t)conn[e * 8 + a] + i + (int64_t)k * 3 * N;
          ue[a * 3 + i] = u[d];
          le[a * 3 + i] = lam[d];
        }
      for (int i = 0; i < 24; ++i) {
        double t = 0.0;
        for (int j = 0; j < 24; ++j) t += Ke[i * 24 + j] * ue[j];
        acc += le[i] * t;
      }
    }
    g[e] = -acc;
  }
}
