/* A C caller of the drop-in boundary: the call sequence the reference's Fortran
 * (through include/ufc_gpu_brg.f90) would make, written against include/ufc_gpu.h
 * alone, with host arrays only.
 *
 *   1. linear static: mesh, material, Dirichlet set, device pattern, assembly,
 *      face loads, Jacobi-PCG in FP64 and FP32+FP64 refinement, multigrid PCG,
 *      reactions, the 1-based CSR export of the reference's RT_CSRMatrix;
 *   2. J2: one step of automatic increments (ufc_nr_step) to 0.6 % strain and the
 *      committed stress against the uniaxial closed form;
 *   3. an error status with its message.
 *
 * Exit 0 on success, 77 when no sm_100 device is present (context creation
 * reports IF_STATUS_UNSUPPORTED), 1 on a failed check. */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "ufc_gpu.h"

#define CHECK(call)                                                                  \
  do {                                                                               \
    int st_ = (call);                                                                \
    if (st_ != UFC_STATUS_OK) {                                                      \
      char msg_[512] = {0};                                                          \
      ufc_last_error(ctx, msg_, (int32_t)sizeof msg_);                               \
      fprintf(stderr, "%s:%d: %s -> status %d: %s\n", __FILE__, __LINE__, #call, st_, msg_); \
      return 1;                                                                      \
    }                                                                                \
  } while (0)

#define EXPECT(cond)                                                                 \
  do {                                                                               \
    if (!(cond)) {                                                                   \
      fprintf(stderr, "%s:%d: check failed: %s\n", __FILE__, __LINE__, #cond);       \
      return 1;                                                                      \
    }                                                                                \
  } while (0)

static int64_t node(int i, int j, int k, int nx, int ny) { return i + (int64_t)(nx + 1) * (j + (int64_t)(ny + 1) * k); }

/* Structured box nx x ny x nz of size lx x ly x lz, Abaqus node order. */
static void box(int nx, int ny, int nz, double lx, double ly, double lz, double* coords, int32_t* conn) {
  for (int k = 0; k <= nz; ++k)
    for (int j = 0; j <= ny; ++j)
      for (int i = 0; i <= nx; ++i) {
        const int64_t n = node(i, j, k, nx, ny);
        coords[3 * n] = lx * i / nx;
        coords[3 * n + 1] = ly * j / ny;
        coords[3 * n + 2] = lz * k / nz;
      }
  static const int off[8][3] = {{0, 0, 0}, {1, 0, 0}, {1, 1, 0}, {0, 1, 0}, {0, 0, 1}, {1, 0, 1}, {1, 1, 1}, {0, 1, 1}};
  for (int k = 0; k < nz; ++k)
    for (int j = 0; j < ny; ++j)
      for (int i = 0; i < nx; ++i) {
        const int64_t e = i + (int64_t)nx * (j + (int64_t)ny * k);
        for (int a = 0; a < 8; ++a) conn[8 * e + a] = (int32_t)node(i + off[a][0], j + off[a][1], k + off[a][2], nx, ny);
      }
}

static double norm(const double* v, int64_t n) {
  double s = 0.0;
  for (int64_t i = 0; i < n; ++i) s += v[i] * v[i];
  return sqrt(s);
}

static int linear_static(void) {
  const int nx = 16, ny = 4, nz = 4;
  const int32_t N = (nx + 1) * (ny + 1) * (nz + 1), E = nx * ny * nz;
  const int64_t n = 3 * (int64_t)N;
  ufc_ctx* ctx = NULL;
  const int st = ufc_ctx_create(0, &ctx);
  if (st == UFC_STATUS_UNSUPPORTED) {
    printf("no sm_100 device: ufc_ctx_create returned IF_STATUS_UNSUPPORTED\n");
    return 77;
  }
  CHECK(st);
  double* coords = malloc(sizeof(double) * n);
  int32_t* conn = malloc(sizeof(int32_t) * 8 * E);
  box(nx, ny, nz, 4.0, 1.0, 1.0, coords, conn);
  ufc_mesh_desc mesh = {N, E, coords, conn, 0, UFC_MEM_HOST};
  CHECK(ufc_mesh_set(ctx, &mesh));
  const double props[2] = {210e3, 0.3};
  ufc_material_desc mat = {UFC_MAT_ELASTIC_ISO, 2, 0, props, UFC_MEM_HOST};
  CHECK(ufc_material_set(ctx, &mat));
  /* clamp the x = 0 face */
  int32_t nfix = 0;
  int32_t* fix = malloc(sizeof(int32_t) * 3 * (ny + 1) * (nz + 1));
  for (int k = 0; k <= nz; ++k)
    for (int j = 0; j <= ny; ++j)
      for (int d = 0; d < 3; ++d) fix[nfix++] = (int32_t)(3 * node(0, j, k, nx, ny) + d);
  ufc_bc_desc bc = {nfix, fix, NULL, UFC_MEM_HOST};
  CHECK(ufc_bc_set(ctx, &bc));
  ufc_pattern_info info;
  CHECK(ufc_pattern_build(ctx, &info));
  EXPECT(info.n_dof == n && info.n_colors == 8);
  ufc_elem_ke_arg ke = {UFC_BUILD_FP64 | UFC_BUILD_FP32_ROUNDED, 0, 0.0};
  CHECK(ufc_elem_compute_ke(ctx, &ke));

  /* traction (0, 0, -1) on the x = 4 face: reference face 6 of the last element column */
  const int32_t nf = ny * nz;
  int32_t* fe = malloc(sizeof(int32_t) * nf);
  int32_t* ff = malloc(sizeof(int32_t) * nf);
  double* tr = malloc(sizeof(double) * 3 * nf);
  for (int k = 0, q = 0; k < nz; ++k)
    for (int j = 0; j < ny; ++j, ++q) {
      fe[q] = (nx - 1) + nx * (j + ny * k);
      ff[q] = 6;
      tr[3 * q] = 0.0;
      tr[3 * q + 1] = 0.0;
      tr[3 * q + 2] = -1.0;
    }
  double* f = malloc(sizeof(double) * n);
  ufc_face_load_arg load = {nf, fe, ff, tr, NULL, 0, UFC_MEM_HOST, f};
  CHECK(ufc_load_faces(ctx, &load));
  double fz = 0.0;
  for (int64_t i = 2; i < n; i += 3) fz += f[i];
  EXPECT(fabs(fz + 1.0) < 1e-12); /* traction 1 on a 1 x 1 face */

  /* Jacobi-PCG in FP64 and with FP32 iterations refined in FP64 */
  double* u64 = calloc(n, sizeof(double));
  double* u32 = calloc(n, sizeof(double));
  double* umg = calloc(n, sizeof(double));
  ufc_solver_algo algo = {UFC_SOLV_METHOD_CG, UFC_SOLV_PREC_JACOBI, 100000, UFC_PRECISION_FP64, 1e-10, 0.0, 0.0, 0, 0,
                          UFC_REFINE_KEEP_DIRECTION, UFC_ACCUMULATE_STORAGE};
  ufc_solver_state s64, s32, smg;
  CHECK(ufc_pcg_solve(ctx, f, u64, UFC_MEM_HOST, &algo, &s64));
  algo.precision_mode = UFC_PRECISION_FP32_REFINE;
  CHECK(ufc_pcg_solve(ctx, f, u32, UFC_MEM_HOST, &algo, &s32));
  EXPECT(s64.converged && s64.rnorm <= 1e-10 && s32.converged && s32.rnorm <= 1e-10);

  /* the same solve with the multigrid preconditioner */
  ufc_mg_arg mg;
  memset(&mg, 0, sizeof mg);
  mg.nx = nx;
  mg.ny = ny;
  mg.nz = nz;
  mg.coarse_max = 50;
  mg.precision = UFC_PRECISION_FP32_REFINE;
  CHECK(ufc_mg_setup(ctx, &mg));
  EXPECT(mg.levels >= 3);
  algo.precision_mode = UFC_PRECISION_FP64;
  algo.precond_type = UFC_SOLV_PREC_MG;
  CHECK(ufc_pcg_solve(ctx, f, umg, UFC_MEM_HOST, &algo, &smg));
  EXPECT(smg.converged && smg.rnorm <= 1e-10 && smg.niter * 4 < s64.niter);

  double d32 = 0.0, dmg = 0.0;
  for (int64_t i = 0; i < n; ++i) {
    d32 += (u32[i] - u64[i]) * (u32[i] - u64[i]);
    dmg += (umg[i] - u64[i]) * (umg[i] - u64[i]);
  }
  EXPECT(sqrt(d32) <= 1e-7 * norm(u64, n) && sqrt(dmg) <= 1e-7 * norm(u64, n));

  /* reactions carry the applied load */
  double* rf = malloc(sizeof(double) * nfix);
  CHECK(ufc_reactions(ctx, u64, f, rf, UFC_MEM_HOST));
  double rz = 0.0;
  for (int32_t k = 0; k < nfix; ++k)
    if (fix[k] % 3 == 2) rz += rf[k];
  EXPECT(fabs(rz - 1.0) < 1e-7);

  /* the reference's 1-based CSR */
  int64_t* rp = malloc(sizeof(int64_t) * (n + 1));
  ufc_csr_export_arg ex = {1, UFC_MEM_HOST, rp, NULL, NULL, NULL};
  CHECK(ufc_csr_export(ctx, &ex));
  EXPECT(rp[0] == 1 && rp[n] == info.nnz + 1);

  /* an invalid call: a status and a message, the context stays usable */
  algo.method = 99;
  EXPECT(ufc_pcg_solve(ctx, f, u64, UFC_MEM_HOST, &algo, &s64) == UFC_STATUS_UNSUPPORTED);
  char msg[512] = {0};
  ufc_last_error(ctx, msg, (int32_t)sizeof msg);
  EXPECT(strstr(msg, "CG") != NULL);

  printf("linear static: FP64 %d it, FP32+refine %d it, multigrid %d it (%d levels), rnorm %.2e\n", s64.niter,
         s32.niter, smg.niter, mg.levels, smg.rnorm);
  CHECK(ufc_ctx_destroy(ctx));
  free(coords); free(conn); free(fix); free(fe); free(ff); free(tr); free(f); free(u64); free(u32); free(umg);
  free(rf); free(rp);
  return 0;
}

static int j2_step(void) {
  const int nx = 4, ny = 2, nz = 2;
  const int32_t N = (nx + 1) * (ny + 1) * (nz + 1), E = nx * ny * nz;
  const double Ey = 200e3, nu = 0.3, sy = 250.0, H = 1000.0, strain = 0.006;
  ufc_ctx* ctx = NULL;
  CHECK(ufc_ctx_create(0, &ctx));
  double* coords = malloc(sizeof(double) * 3 * N);
  int32_t* conn = malloc(sizeof(int32_t) * 8 * E);
  box(nx, ny, nz, (double)nx, (double)ny, (double)nz, coords, conn);
  ufc_mesh_desc mesh = {N, E, coords, conn, 0, UFC_MEM_HOST};
  CHECK(ufc_mesh_set(ctx, &mesh));
  const double props[4] = {Ey, nu, sy, H};
  ufc_material_desc mat = {UFC_MAT_J2_ISO, 4, 0, props, UFC_MEM_HOST};
  CHECK(ufc_material_set(ctx, &mat));
  /* u_x = 0 on x = 0, u_x prescribed on x = nx, rigid modes pinned at (0,0,0) and (0,ny,0) */
  int32_t* fix = malloc(sizeof(int32_t) * 3 * N);
  double* uend = malloc(sizeof(double) * 3 * N);
  int32_t nfix = 0;
  for (int k = 0; k <= nz; ++k)
    for (int j = 0; j <= ny; ++j) {
      fix[nfix] = (int32_t)(3 * node(0, j, k, nx, ny));
      uend[nfix++] = 0.0;
    }
  fix[nfix] = (int32_t)(3 * node(0, 0, 0, nx, ny) + 1);
  uend[nfix++] = 0.0;
  fix[nfix] = (int32_t)(3 * node(0, 0, 0, nx, ny) + 2);
  uend[nfix++] = 0.0;
  fix[nfix] = (int32_t)(3 * node(0, ny, 0, nx, ny) + 2);
  uend[nfix++] = 0.0;
  for (int k = 0; k <= nz; ++k)
    for (int j = 0; j <= ny; ++j) {
      fix[nfix] = (int32_t)(3 * node(nx, j, k, nx, ny));
      uend[nfix++] = strain * nx;
    }
  ufc_bc_desc bc = {nfix, fix, NULL, UFC_MEM_HOST};
  CHECK(ufc_bc_set(ctx, &bc));
  ufc_pattern_info info;
  CHECK(ufc_pattern_build(ctx, &info));
  ufc_step_arg step;
  memset(&step, 0, sizeof step);
  step.u_prescribed_end = uend;
  step.mem = UFC_MEM_HOST;
  step.time_period = 1.0;
  step.dt_initial = 0.25;
  step.dt_min = 1e-4;
  step.dt_max = 0.5;
  step.max_increments = 50;
  step.max_cutbacks = 5;
  step.auto_dt = 1;
  step.target_iters = 6;
  step.growth_threshold = 0.8;
  step.growth_factor = 1.25;
  step.cutback_factor = 0.5;
  step.max_iterations = 8;
  step.tolerance_force = 1e-8;
  ufc_solver_algo lin = {UFC_SOLV_METHOD_CG, UFC_SOLV_PREC_JACOBI, 100000, UFC_PRECISION_FP64, 1e-12, 0.0, 0.0, 0, 0,
                         UFC_REFINE_KEEP_DIRECTION, UFC_ACCUMULATE_STORAGE};
  step.lin = lin;
  CHECK(ufc_nr_step(ctx, &step));
  EXPECT(step.completed && step.final_time == 1.0);
  double* sig = malloc(sizeof(double) * 6 * 8 * E);
  CHECK(ufc_get_state(ctx, NULL, sig, NULL, UFC_MEM_HOST));
  const double want = sy + Ey * H / (Ey + H) * (strain - sy / Ey);
  for (int64_t g = 0; g < 8 * (int64_t)E; ++g) EXPECT(fabs(sig[6 * g] - want) <= 1e-6 * want);
  printf("J2 step: %d increments, %d cutbacks, %d Newton iterations, sigma_xx %.6f (closed form %.6f)\n",
         step.increments, step.cutbacks, step.nr_iterations, sig[0], want);
  CHECK(ufc_ctx_destroy(ctx));
  free(coords); free(conn); free(fix); free(uend); free(sig);
  return 0;
}

int main(void) {
  int r = linear_static();
  if (r != 0) return r;
  r = j2_step();
  if (r != 0) return r;
  printf("C drop-in OK\n");
  return 0;
}
