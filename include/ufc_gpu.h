/*
 * ufc_gpu.h -- C-ABI of the B200 implementation of UFC's implicit-static C3D8
 * hot path: C3D8 element loop (linear elastic and J2), deterministic assembly
 * into a device-built CSR stiffness, Jacobi-PCG (FP64, or FP32 inner
 * iterations with FP64 residual refinement), Newton-Raphson increments, and the
 * adjoint sensitivity.
 *
 * Every entry point returns an int32 status with the values of the reference's
 * IF_STATUS_* codes (ufc_core/L1_IF/Error/IF_Err_Brg.f90:95-110); the message of
 * the last failure is read with ufc_last_error (the reference's
 * ErrorStatusType%message, ufc_core/L1_IF/Error/IF_Err_Def.f90:118-135).  No
 * entry point exits, aborts or traps.
 *
 * The *_desc / *_arg structs are the batched, device-side counterparts of the
 * reference's Desc/State/Algo/Ctx "*_Arg" bundles: fields marked [IN] are read,
 * [OUT] are written.  Pointers are host or device memory as the struct's `mem`
 * field (UFC_MEM_HOST / UFC_MEM_DEVICE) says; host buffers are borrowed for the
 * duration of the call, device buffers are used in order on the context's
 * stream.  A context owns all device memory it allocates (mesh, pattern, matrix
 * values, solver work vectors, material state) and is not shared between
 * threads; calls on one context are ordered on its stream.
 *
 * DOF numbering: eq = 3*node + component (ufc_core/L5_RT/Assembly/
 * RT_Asm_DofMap.f90:172-249), nodes and elements 0-based unless index_base = 1.
 * Element nodes in Abaqus order (ufc_core/L4_PH/Element/PH_Elem_ShapeFunc.f90:329-350).
 * Voigt order (xx, yy, zz, gxy, gyz, gzx), engineering shear strains.
 */
#ifndef UFC_GPU_H
#define UFC_GPU_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* IF_STATUS_* (IF_Err_Brg.f90:95-110) */
#define UFC_STATUS_OK 0
#define UFC_STATUS_INVALID 1
#define UFC_STATUS_ERROR 2
#define UFC_STATUS_CONVERGED 3
#define UFC_STATUS_NOT_CONVERGED 4
#define UFC_STATUS_NOT_FOUND 5
#define UFC_STATUS_WARN 6
#define UFC_STATUS_MEM_ERROR 7
#define UFC_STATUS_IO_ERROR 8
#define UFC_STATUS_EXISTS 9
#define UFC_STATUS_FATAL 10
#define UFC_STATUS_UNSUPPORTED 11

#define UFC_MEM_HOST 0
#define UFC_MEM_DEVICE 1

/* Material sub-model ids: PH_MAT_ELAS_SUB_ISO (ufc_core/L4_PH/Material/Elas/
 * PH_Mat_Elas_Def.f90:24), PH_MAT_PLAST_SUB_J2_ISO (ufc_core/L4_PH/Material/
 * Plast/PH_Mat_Plast_Def.f90:18). */
#define UFC_MAT_ELASTIC_ISO 101
#define UFC_MAT_J2_ISO 201

/* NM_SOLV_METHOD_CG / NM_SOLV_PREC_* (ufc_core/L2_NM/Solver/NM_Solv_Def.f90:32-46) */
#define UFC_SOLV_METHOD_CG 3
#define UFC_SOLV_PREC_NONE 0
#define UFC_SOLV_PREC_JACOBI 1
#define UFC_SOLV_PREC_MG 5  /* geometric multigrid V-cycle, set up by ufc_mg_setup (NM_PREC_AMG = 5,
                               ufc_core/L2_NM/Solver/LinSolv/NM_Solv_Mgr.f90:35) */

/* Precision of the linear solve. */
#define UFC_PRECISION_FP64 0        /* FP64 matrix, vectors and dot products      */
#define UFC_PRECISION_FP32_REFINE 1 /* FP32 matrix and inner CG, FP64 solution and
                                       FP64 residual replacement (refinement)      */
#define UFC_PRECISION_FP32_MATRIX 2 /* FP32 matrix values only; FP64 CG vectors and
                                       arithmetic, FP64 residual replacement       */

/* Row-sum accumulator of the FP32_REFINE SpMV. */
#define UFC_ACCUMULATE_STORAGE 0 /* FP32, like the stored values */
#define UFC_ACCUMULATE_FP64 1    /* FP32 products summed in FP64 (same bytes moved) */

/* Which matrix values ufc_elem_compute_ke builds (bit mask).  UFC_BUILD_FP32
 * runs the element kernel in FP32; UFC_BUILD_FP32_ROUNDED instead rounds the
 * FP64-assembled values to FP32 (implies UFC_BUILD_FP64); UFC_BUILD_FP32_DIFF
 * stores the FP32 matrix in difference form: off-diagonal blocks rounded from
 * FP64 and, in the diagonal slot, the FP64 block row sum S_i = sum_j K_ij, so
 * that the SpMV evaluates y_i = sum_{j != i} K_ij (x_j - x_i) + S_i x_i, whose
 * rounding error vanishes on rigid translations (implies UFC_BUILD_FP64). */
#define UFC_BUILD_FP64 1
#define UFC_BUILD_FP32 2
#define UFC_BUILD_FP32_ROUNDED 4
#define UFC_BUILD_FP32_DIFF 8
/* Also pack symmetric SpMV copies (upper-triangle blocks only; each row reads
 * its lower blocks transposed from the rows that store them): FP64, and FP32
 * rounded from FP64 when an FP32 build is requested.  The solver and ufc_spmv
 * use them when present.  Implies UFC_BUILD_FP64. */
#define UFC_BUILD_SYMMETRIC 16

/* FP32_REFINE policy at each FP64 residual replacement.  With the first two,
 * a matrix whose FP64 product reads less than half the L2 cache is solved in
 * FP64 (the FP32 storage saves no time there: both products run from L2 and
 * are bound by latency, and the FP32 recursion needs more iterations); the
 * state then reports every iteration in fp64_iters.  UFC_REFINE_FORCE_FP32
 * keeps the FP32 iterations whatever the size (direction kept). */
#define UFC_REFINE_KEEP_DIRECTION 0 /* keep the search direction (reliable update) */
#define UFC_REFINE_RESTART 1        /* restart CG from the new residual (defect correction) */
#define UFC_REFINE_FORCE_FP32 2     /* keep the direction, FP32 iterations on any size */

typedef struct ufc_ctx ufc_ctx;

/* Mesh description: the L3 mesh plus PH_Elem_Desc of a C3D8 domain
 * (ufc_core/L4_PH/Element/PH_Elem_Def.f90:329-355). */
typedef struct {
  int32_t n_nodes;       /* [IN] */
  int32_t n_elems;       /* [IN] */
  const double* coords;  /* [IN] [n_nodes][3] */
  const int32_t* conn;   /* [IN] [n_elems][8], Abaqus node order */
  int32_t index_base;    /* [IN] 0, or 1 for Fortran connectivity */
  int32_t mem;           /* [IN] UFC_MEM_HOST / UFC_MEM_DEVICE */
} ufc_mesh_desc;

/* Material description: PH_Mat_Elas_Desc / PH_J2_Props with the props layout
 * [E, nu] (101) or [E, nu, sigma_y0, H_iso] (201) of config/UMAT_Props_Layout.json. */
typedef struct {
  int32_t mat_model_id;  /* [IN] UFC_MAT_ELASTIC_ISO or UFC_MAT_J2_ISO */
  int32_t nprops;        /* [IN] >= 2 (elastic) or >= 4 (J2) */
  int32_t per_element;   /* [IN] 1: props[n_elems][nprops]; 0: props[nprops] for all */
  const double* props;   /* [IN] */
  int32_t mem;           /* [IN] */
} ufc_material_desc;

/* Dirichlet set: eliminated symmetrically (zero row and column, unit diagonal,
 * lifted right-hand side) in place of the penalty of
 * RT_Asm_ApplyBC_Displacement_Penalty (ufc_core/L5_RT/Assembly/RT_Asm_Solv.f90:427-483). */
typedef struct {
  int32_t n_fixed;       /* [IN] */
  const int32_t* dofs;   /* [IN] [n_fixed] DOF ids (index_base of the mesh) */
  const double* values;  /* [IN] [n_fixed] prescribed values, or NULL for zero */
  int32_t mem;           /* [IN] */
} ufc_bc_desc;

/* Pattern summary returned by ufc_pattern_build. */
typedef struct {
  int64_t n_dof;          /* [OUT] 3 * n_nodes */
  int64_t nnz;            /* [OUT] scalar CSR non-zeros = 9 * nnzb */
  int64_t nnzb;           /* [OUT] 3x3 blocks */
  int64_t sell_blocks;    /* [OUT] stored blocks incl. slice padding */
  int32_t n_colors;       /* [OUT] element colours */
  int32_t max_row_blocks; /* [OUT] */
} ufc_pattern_info;

/* Canonical CSR export: RT_CSRMatrix{rowPtr, colInd, values} of
 * ufc_core/L2_NM/Matrix/NM_Assem_Sparse.f90:45-54. */
typedef struct {
  int32_t index_base;   /* [IN] 1 gives rowPtr(1) = 1 as the reference stores it */
  int32_t mem;          /* [IN] */
  int64_t* row_ptr;     /* [OUT] [n_dof+1] or NULL */
  int32_t* col_ind;     /* [OUT] [nnz] or NULL */
  double* values;       /* [OUT] [nnz] FP64 values or NULL */
  float* values32;      /* [OUT] [nnz] FP32 values or NULL */
} ufc_csr_export_arg;

/* Batched PH_Element_Compute_Ke_Arg (PH_Elem_Def.f90:331-341) over every
 * element, followed by the scatter of RT_Asm_GlobalStiffness
 * (RT_Asm_Solv.f90:1762-1985).  For UFC_MAT_J2_ISO the per-Gauss-point
 * consistent tangents of the last ufc_elem_compute_fint(update_state=1) are used. */
typedef struct {
  int32_t build;        /* [IN] UFC_BUILD_FP64 | UFC_BUILD_FP32 */
  int32_t status;       /* [OUT] */
  double elapsed_ms;    /* [OUT] device time of the assembly kernels */
} ufc_elem_ke_arg;

/* Batched PH_Element_Compute_Fe_Arg (PH_Elem_Def.f90:343-355) and
 * RT_Asm_ComputeResidual (RT_Asm_Solv.f90:1311-1426) with the internal force
 * F_int = sum_e int B^T sigma dV (PH_Elem_C3D8_IntForce, PH_Elem_C3D8.f90:734-757). */
typedef struct {
  const double* u;      /* [IN] [n_dof] displacement, prescribed values included */
  const double* f_ext;  /* [IN] [n_dof] or NULL (zero) */
  double* fint;         /* [OUT] [n_dof] F_int over every DOF, or NULL */
  double* r;            /* [OUT] [n_dof] f_ext - F_int on free DOFs, 0 on fixed, or NULL */
  int32_t mem;          /* [IN] */
  int32_t update_state; /* [IN] J2: return-map every Gauss point from the committed
                           state at u and keep the trial state and tangents */
  double rnorm;         /* [OUT] ||r||_2 over the free DOFs (FP64) */
  double fint_norm;     /* [OUT] ||F_int||_2 over every DOF */
  int32_t status;       /* [OUT] */
} ufc_elem_fe_arg;

/* Batched PH_Mat_Update_Arg (ufc_core/L4_PH/Material/PH_Mat_KernelDefn.f90:18-59)
 * / PH_J2_ComputeStress_Arg (PH_Mat_Plast_J2_Iso_Core.f90:119-126), one
 * material point per entry, array-of-structs rows. */
typedef struct {
  int32_t mat_model_id;   /* [IN] */
  int32_t n_points;       /* [IN] */
  int32_t nprops;         /* [IN] */
  int32_t props_per_point;/* [IN] 1: props[n_points][nprops]; 0: props[nprops] */
  const double* props;    /* [IN] */
  const double* stress_n; /* [IN] [n][6] committed stress */
  const double* dstrain;  /* [IN] [n][6] strain increment */
  const double* sdv_n;    /* [IN] [n][7] (eps_p_eq, eps_p[6]) or NULL (zero) */
  double* stress;         /* [OUT] [n][6] */
  double* sdv;            /* [OUT] [n][7] or NULL */
  double* ddsdde;         /* [OUT] [n][36] row-major consistent tangent, or NULL */
  int32_t* yielded;       /* [OUT] [n] or NULL */
  int32_t mem;            /* [IN] */
  int32_t status;         /* [OUT] */
} ufc_mat_update_arg;

/* NM_Solver_Algo (ufc_core/L2_NM/Solver/NM_Solv_Def.f90:86-100). */
typedef struct {
  int32_t method;         /* [IN] UFC_SOLV_METHOD_CG */
  int32_t precond_type;   /* [IN] UFC_SOLV_PREC_JACOBI, UFC_SOLV_PREC_MG (after ufc_mg_setup) or UFC_SOLV_PREC_NONE */
  int32_t max_iter;       /* [IN] */
  int32_t precision_mode; /* [IN] UFC_PRECISION_FP64 or UFC_PRECISION_FP32_REFINE */
  double tolerance;       /* [IN] stop when ||b - K x||_2 <= max(tolerance*||b||_2, abs_tolerance) */
  double abs_tolerance;   /* [IN] */
  double refine_delta;    /* [IN] FP32_REFINE: replace the FP32 residual by the FP64
                             one whenever it fell by this factor (0: default 0.1) */
  int32_t check_every;    /* [IN] iterations per launch batch between host checks (0: default) */
  int32_t use_x0;         /* [IN] 1: x holds the initial guess; 0: x0 = 0 */
  int32_t refine_policy;  /* [IN] UFC_REFINE_KEEP_DIRECTION, UFC_REFINE_RESTART or UFC_REFINE_FORCE_FP32 */
  int32_t accumulate;     /* [IN] FP32_REFINE: UFC_ACCUMULATE_STORAGE or UFC_ACCUMULATE_FP64 */
} ufc_solver_algo;

/* NM_Solver_State (ufc_core/L2_NM/Solver/NM_Solv_Def.f90:105-117). */
typedef struct {
  int32_t niter;           /* [OUT] CG iterations */
  int32_t n_refine;        /* [OUT] FP64 residual replacements */
  int32_t converged;       /* [OUT] */
  int32_t convergence_flag;/* [OUT] 0 converged, 2 max-iter, 3 breakdown */
  double rnorm;            /* [OUT] final ||b - K x||_2 / ||b||_2 in FP64 */
  double initial_residual; /* [OUT] ||b - K x0||_2 */
  double solve_time;       /* [OUT] ms, CUDA events around the device work */
  int32_t fp64_iters;      /* [OUT] FP32 modes: FP64 iterations run after the FP32 run
                              stalled or diverged (continued from its best iterate when
                              FP64 values are assembled); included in niter */
  int32_t reserved;
} ufc_solver_state;

/* One Newton-Raphson increment: RT_NLSolver_NewtonRaph
 * (ufc_core/L5_RT/Solver/RT_Solv_Nonlin.f90:807-1002). */
typedef struct {
  const double* u_prescribed; /* [IN] [n_fixed] values of the Dirichlet DOFs at the end of the increment */
  const double* f_ext;        /* [IN] [n_dof] or NULL */
  int32_t mem;                /* [IN] */
  int32_t max_iterations;     /* [IN] */
  double tolerance_force;     /* [IN] ||R_free|| <= tol * max(||F_ext||, ||F_int||) */
  ufc_solver_algo lin;        /* [IN] linear solver for K du = R */
  int32_t iterations;         /* [OUT] */
  int32_t converged;          /* [OUT] */
  int32_t lin_iters_total;    /* [OUT] */
  double residual_norm;       /* [OUT] final relative residual */
  double res_hist[32];        /* [OUT] relative residual before each iteration's solve */
  int32_t status;             /* [OUT] */
} ufc_nr_arg;

/* One analysis step with automatic increments: RT_StepDriver_Execute
 * (ufc_core/L5_RT/StepDriver/RT_Step_Exec.f90:415-600) with the increment
 * control of RT_StepDriver_End_Increment / RT_StepDriver_Cutback
 * (RT_Step_Core.f90:215-300, defaults RT_Step_Def.f90:147-153).  The prescribed
 * values and the external force are ramped linearly in step time from their
 * values at the start of the step (the committed displacement, f_ext_start) to
 * u_prescribed_end / f_ext_end at time_period.  Each increment runs
 * ufc_nr_increment; a converged increment is committed, and the next one grows
 * by growth_factor when it took <= (int)(target_iters * growth_threshold)
 * Newton iterations (capped by dt_max and the end of the step); a failed one is
 * rolled back and retried with dt * cutback_factor, the step failing when dt
 * drops below dt_min or more than max_cutbacks cutbacks follow one another. */
typedef struct {
  const double* u_prescribed_end; /* [IN] [n_fixed] Dirichlet values at the end of the step, or NULL (kept) */
  const double* f_ext_start;      /* [IN] [n_dof] external force at the start of the step, or NULL (zero) */
  const double* f_ext_end;        /* [IN] [n_dof] external force at the end of the step, or NULL (zero) */
  int32_t mem;                    /* [IN] memory of the three arrays */
  double time_period;             /* [IN] step time, > 0 */
  double dt_initial, dt_min, dt_max; /* [IN] increment sizes in step time */
  int32_t max_increments;         /* [IN] attempted increments, converged or not */
  int32_t max_cutbacks;           /* [IN] consecutive cutbacks before the step fails */
  int32_t auto_dt;                /* [IN] 1: grow dt after easy increments (RT_Step_Stp_Ctl_Algo%auto_dt) */
  int32_t target_iters;           /* [IN] 6 in the reference */
  double growth_threshold;        /* [IN] 0.8 */
  double growth_factor;           /* [IN] 1.25 */
  double cutback_factor;          /* [IN] 0.5 */
  int32_t max_iterations;         /* [IN] Newton iterations per increment */
  double tolerance_force;         /* [IN] as ufc_nr_arg */
  ufc_solver_algo lin;            /* [IN] linear solver of every Newton iteration */
  double* hist_time;              /* [OUT] host [hist_cap]: step time at the end of each attempt, or NULL */
  double* hist_dt;                /* [OUT] host [hist_cap]: increment size of each attempt, or NULL */
  int32_t* hist_iters;            /* [OUT] host [hist_cap]: Newton iterations of each attempt, or NULL */
  int32_t* hist_converged;        /* [OUT] host [hist_cap]: 1 converged, 0 cut back, or NULL */
  int32_t hist_cap;               /* [IN] */
  int32_t attempts;               /* [OUT] increments attempted (entries written: min(attempts, hist_cap)) */
  int32_t increments;             /* [OUT] converged increments */
  int32_t cutbacks;               /* [OUT] total cutbacks */
  int32_t nr_iterations;          /* [OUT] Newton iterations of the converged increments */
  int64_t lin_iters_total;        /* [OUT] CG iterations of all attempts */
  double final_time;              /* [OUT] step time reached */
  int32_t completed;              /* [OUT] 1 when final_time reached time_period */
  int32_t status;                 /* [OUT] */
} ufc_step_arg;

/* Multigrid preconditioner for a structured box mesh, in the place of the
 * reference's AMG (NM_AMG_Setup / NM_AMG_V_Cycle / NM_AMG_Smooth / NM_AMG_Galerkin,
 * ufc_core/L2_NM/Solver/LinSolv/NM_Solv_LinPrecAMG.f90:120-675).  The mesh must be
 * the nx x ny x nz box numbering: node (i,j,k) = i + (nx+1)(j + (ny+1)k),
 * element (i,j,k) = i + nx(j + ny k) with nodes in Abaqus order.  Levels halve
 * the box while nx, ny and nz are even and the level has more than coarse_max
 * DOF; prolongation is trilinear, coarse operators are Galerkin products
 * P^T A P formed element by element, Dirichlet DOFs stay eliminated on every
 * level (a coarse DOF is fixed when its coincident fine DOF is).  Smoother:
 * Chebyshev polynomial of D^-1 A of the given degree before and after the
 * coarse correction, on [lambda_max/ratio, 1.1 lambda_max] with lambda_max
 * from a power iteration; coarsest level: dense inverse (<= 1200 DOF) or a
 * degree-24 Chebyshev solve.  Uses the assembled FP64 values (and, for J2, the
 * tangent of the trial state): call it after ufc_elem_compute_ke; after a
 * reassembly the numerical part (coarse operators, smoother bounds, coarsest
 * inverse) is rebuilt on the boxes already set up, at the next multigrid solve.
 * Solve with ufc_solver_algo.precond_type = UFC_SOLV_PREC_MG and precision FP64
 * (the outer PCG; the cycle's own precision is chosen here). */
typedef struct {
  int32_t nx, ny, nz;        /* [IN] */
  int32_t max_levels;        /* [IN] 0: as many as the grid allows */
  int32_t degree;            /* [IN] Chebyshev degree of each smoothing, 0: 2 */
  double ratio;              /* [IN] lambda_max / lambda_min of the smoother interval, 0: 15 */
  int64_t coarse_max;        /* [IN] stop coarsening at or below this many DOF, 0: 300 */
  int32_t levels;            /* [OUT] */
  int32_t precision;         /* [IN] UFC_PRECISION_FP64: FP64 cycle; UFC_PRECISION_FP32_REFINE: the
                                cycle in FP32 on values rounded from the FP64 operators (the PCG
                                around it stays FP64) */
  int64_t coarse_dof;        /* [OUT] DOF of the coarsest level */
  double setup_ms;           /* [OUT] */
} ufc_mg_arg;

/* Equivalent nodal forces of face loads on C3D8 faces: the 2x2 face Gauss rule
 * of PH_Elem_C3D8_FormFacePressure (ufc_core/L4_PH/Element/Solid3D/PH_Elem_C3D8.f90:2360-2541)
 * and its face numbering (1: nodes 1-2-3-4, zeta = -1; 2: 5-8-7-6, zeta = +1;
 * 3: 1-2-6-5, eta = -1; 4: 4-3-7-8, eta = +1; 5: 1-4-8-5, xi = -1; 6: 2-6-7-3,
 * xi = +1), with N_a = (1/8)(1 +- xi)(1 +- eta)(1 +- zeta).  Per face, a
 * traction vector t (force per unit area) and/or a pressure p acting against
 * the outward normal: f_a += sum_gp N_a (t - p n_out) dA.  Faces are assembled
 * in element-colour order, so the result is deterministic; f is overwritten. */
typedef struct {
  int32_t n_faces;         /* [IN] */
  const int32_t* elem;     /* [IN] [n_faces] element ids (index_base) */
  const int32_t* face;     /* [IN] [n_faces] face ids 1..6 */
  const double* traction;  /* [IN] [n_faces][3] or NULL */
  const double* pressure;  /* [IN] [n_faces] or NULL */
  int32_t index_base;      /* [IN] 0 or 1 */
  int32_t mem;             /* [IN] memory of every array */
  double* f;               /* [OUT] [n_dof] */
} ufc_face_load_arg;

/* Device-time counters of the last ufc_pcg_solve (filled when instrumentation
 * is on, see ufc_ctx_set_instrument). */
typedef struct {
  int32_t spmv_launches;
  double spmv_ms;        /* sum of CUDA-event durations of the SpMV launches */
  int64_t spmv_bytes;    /* algorithmic bytes of one SpMV launch */
  int32_t precision;     /* UFC_PRECISION_* of the timed SpMV */
  int64_t kernel_launches; /* kernels the last solve enqueued (always counted) */
} ufc_timing_info;

/* ---- context (replaces the reference's L0 global container g_ufc_global,
 *      ufc_core/L0_Global/UFC_GlobalContainer_Core.f90) ---- */
int ufc_ctx_create(int32_t device, ufc_ctx** ctx);
int ufc_ctx_destroy(ufc_ctx* ctx);
/* Use a caller-owned cudaStream_t (e.g. torch.cuda.current_stream().cuda_stream); NULL = own stream.
 * No counterpart in the reference, which runs on the CPU. */
int ufc_ctx_set_stream(ufc_ctx* ctx, void* cuda_stream);
/* Time every SpMV of the following solves with CUDA events (read with
 * ufc_last_timing); no counterpart in the reference. */
int ufc_ctx_set_instrument(ufc_ctx* ctx, int32_t on);
/* ErrorStatusType%message (IF_Err_Def.f90:118-135) of the last failure. */
int ufc_last_error(const ufc_ctx* ctx, char* buf, int32_t buflen);

/* ---- model set-up ---- */
int ufc_mesh_set(ufc_ctx* ctx, const ufc_mesh_desc* mesh);
int ufc_material_set(ufc_ctx* ctx, const ufc_material_desc* mat);
int ufc_bc_set(ufc_ctx* ctx, const ufc_bc_desc* bc);

/* Device-built sorted-unique CSR pattern, once per mesh: replaces
 * RT_CSR_FromTripletMerged (ufc_core/L5_RT/Solver/RT_Solv_Sparse.f90:336-445)
 * and NM_COO_to_CSR (ufc_core/L2_NM/Matrix/NM_Mtx_Sparse.f90:164-222), plus the
 * element colouring of RT_AsmColor_Build (ufc_core/L5_RT/Assembly/RT_Asm_Color.f90:36-182). */
int ufc_pattern_build(ufc_ctx* ctx, ufc_pattern_info* info);
int ufc_csr_export(ufc_ctx* ctx, const ufc_csr_export_arg* arg);
/* The element colours of the last ufc_pattern_build: RT_AsmColorResult%color_of
 * of RT_AsmColor_Build (ufc_core/L5_RT/Assembly/RT_Asm_Color.f90:36-182), the
 * greedy colouring (elements in ascending order, each the smallest colour that
 * no lower-numbered element sharing a node has), computed on the device.
 * color_of[e] lies in index_base .. index_base + n_colors - 1 (index_base 1 gives
 * the reference's 1-based colours); mem: memory of color_of ([n_elems]). */
int ufc_pattern_colors(ufc_ctx* ctx, int32_t* color_of, int32_t index_base, int32_t mem);

/* ---- element / material ---- */
int ufc_elem_compute_ke(ufc_ctx* ctx, ufc_elem_ke_arg* arg);
int ufc_elem_compute_fint(ufc_ctx* ctx, ufc_elem_fe_arg* arg);
int ufc_mat_update_batch(ufc_ctx* ctx, ufc_mat_update_arg* arg);
/* Gauss-point stress ([n_elems][8][6]) and von Mises ([n_elems][8]) at u
 * (PH_Elem_C3D8_EvalVonMises, PH_Elem_C3D8.f90:2768-2780); J2 models report the
 * committed state and ignore u.  Either output may be NULL. */
int ufc_stress_eval(ufc_ctx* ctx, const double* u, double* stress_gp, double* vm_gp, int32_t mem);

/* ---- loads and output on either side of the solve ---- */
/* External load vector from face tractions / pressures (RT_Asm_GlobalLoad's
 * surface-load branch, ufc_core/L5_RT/Assembly/RT_Asm_Solv.f90:1443). */
int ufc_load_faces(ufc_ctx* ctx, const ufc_face_load_arg* arg);
/* Nodal stress ([n_nodes][6]) and von Mises of that stress ([n_nodes]): the
 * Gauss-point stress of each element extrapolated to its nodes with the
 * inverse of the Gauss-point interpolation matrix (PH_Elem_C3D8_GetExtrapMat /
 * PH_Elem_C3D8_MapToNode, PH_Elem_C3D8.f90:2782-2824, with N_a = (1/8)...),
 * then averaged over the elements that share the node (colour-ordered,
 * deterministic).  u as ufc_stress_eval; either output may be NULL. */
int ufc_stress_nodal(ufc_ctx* ctx, const double* u, double* stress_node, double* vm_node, int32_t mem);
/* Reaction forces RF = F_int(u) - F_ext at the prescribed DOFs, in the order of
 * ufc_bc_desc (the constrained rows of R = F_ext - F_int of
 * RT_Asm_ComputeResidual, RT_Asm_Solv.f90:1311-1426).  u NULL: the current
 * displacement; f_ext NULL: zero.  J2 models use the trial state of u without
 * changing it. */
int ufc_reactions(ufc_ctx* ctx, const double* u, const double* f_ext, double* rf, int32_t mem);

/* ---- linear algebra ---- */
/* y = K x with the assembled matrix of the given precision (RT_CSRMatrix_matvec,
 * ufc_core/L2_NM/Matrix/NM_Assem_Sparse.f90:199-212).  UFC_PRECISION_FP32_REFINE
 * takes float x/y; FP64 and FP32_MATRIX take double x/y. */
int ufc_spmv(ufc_ctx* ctx, int32_t precision, const void* x, void* y, int32_t mem);
/* Jacobi-PCG on the eliminated system K x = b: NM_Solver_PCG
 * (ufc_core/L2_NM/Solver/NM_Solv_Core.f90:363-423) and iter_pcg
 * (ufc_core/L2_NM/Solver/LinSolv/NM_Solv_IterSolver.f90:713-846).  b holds the
 * lifted right-hand side (prescribed values on fixed DOFs).  Returns
 * UFC_STATUS_NOT_CONVERGED when max_iter is reached. */
int ufc_pcg_solve(ufc_ctx* ctx, const double* b, double* x, int32_t mem, const ufc_solver_algo* algo,
                  ufc_solver_state* state);
/* Builds the geometric multigrid hierarchy described at ufc_mg_arg (in the place
 * of NM_AMG_Setup, NM_Solv_LinPrecAMG.f90:120-675). */
int ufc_mg_setup(ufc_ctx* ctx, ufc_mg_arg* arg);
/* z = M r: one V-cycle of the multigrid preconditioner ([n_dof] vectors). */
int ufc_mg_apply(ufc_ctx* ctx, const double* r, double* z, int32_t mem);
/* Canonical CSR of the operator of multigrid level `level` (0 = the assembled
 * matrix), as ufc_csr_export; ufc_mg_level_info gives its DOF and non-zeros. */
int ufc_mg_level_info(ufc_ctx* ctx, int32_t level, int64_t* n_dof, int64_t* nnz);
int ufc_mg_export(ufc_ctx* ctx, int32_t level, const ufc_csr_export_arg* arg);
/* nrhs independent Jacobi-PCG solves sharing every SpMV (one matrix read per
 * iteration for all right-hand sides).  B and X are [nrhs][n_dof]; states[nrhs]. */
int ufc_pcg_solve_block(ufc_ctx* ctx, int32_t nrhs, const double* B, double* X, int32_t mem,
                        const ufc_solver_algo* algo, ufc_solver_state* states);
/* Device-time counters of the last solve (ufc_timing_info); no counterpart in the reference. */
int ufc_last_timing(const ufc_ctx* ctx, ufc_timing_info* info);
/* NM_Solver_State%residual_history (NM_Solv_Def.f90:114) of the last solve:
 * ||r_k||_2 of the CG recurrence after each iteration k (host array, at most
 * max_len entries, the count in *len; the first 2^20 iterations are kept). */
int ufc_last_residual_history(ufc_ctx* ctx, double* out, int32_t max_len, int32_t* len);

/* ---- nonlinear driver and material state (RT_Step_Exec.f90:415-600) ---- */
int ufc_nr_increment(ufc_ctx* ctx, ufc_nr_arg* arg);
/* Returns UFC_STATUS_OK when the step completed, UFC_STATUS_NOT_CONVERGED when
 * it failed (the state is that of the last converged increment). */
int ufc_nr_step(ufc_ctx* ctx, ufc_step_arg* arg);
int ufc_state_commit(ufc_ctx* ctx);
int ufc_state_rollback(ufc_ctx* ctx);
/* Current displacement held by the context ([n_dof]): the Newton state's u of
 * RT_NLSolver_NewtonRaph (ufc_core/L5_RT/Solver/RT_Solv_Nonlin.f90:807-830). */
int ufc_get_displacement(ufc_ctx* ctx, double* u, int32_t mem);
int ufc_set_displacement(ufc_ctx* ctx, const double* u, int32_t mem);
/* Committed J2 state: eps_p_eq [n_elems*8], stress [n_elems*8][6], eps_p [n_elems*8][6]; any may be NULL
 * (the solution-dependent variables sdv(1) and sdv(2:7) and the stress of
 * PH_Mat_Plast_J2_Iso_Core.f90:91-93 and PH_Mat_Reg.f90:232-235). */
int ufc_get_state(ufc_ctx* ctx, double* eps_p_eq, double* stress, double* eps_p, int32_t mem);

/* ---- adjoint: dJ/dE_e = -sum_k lambda_k,e^T (dK_e/dE_e) u_k,e for nrhs pairs
 * ([nrhs][n_dof]); replaces the stubs NM_AI_Adjoint_Solve
 * (ufc_core/L2_NM/Solver/AI/NM_AI_AdjointAlgo.f90:116-136) and
 * PH_Elem_dRdTheta_FD (ufc_core/L4_PH/Element/PH_Elem_dRdTheta.f90:59-78). ---- */
int ufc_adjoint_sensitivity(ufc_ctx* ctx, int32_t nrhs, const double* U, const double* Lam, double* dJdE,
                            int32_t mem);

/* ---- allocation-free SpMV (no counterpart in the reference) ----
 * y = A x and *xy = x.y for a caller-owned FP64 CSR matrix (0-based row_ptr,
 * col_ind, values, e.g. from ufc_csr_export with mem = UFC_MEM_DEVICE), all
 * pointers in device memory, enqueued on cuda_stream (NULL: legacy stream).
 * It is for callers that cannot allocate device memory -- a host code whose
 * device memory all comes from its own fixed pool, or one that may not enter
 * the CUDA allocator on its hot path: it calls no cudaMalloc/cudaFree and needs
 * no context.  The dot-product scratch is a static device array: at most
 * UFC_NOALLOC_MAX_ROWS rows (larger calls return UFC_STATUS_INVALID); each GPU
 * that loads the library keeps the array (about 512 KiB) until exit; the first
 * call on a device looks up its address and should come before any stream
 * capture, and that address is not looked up again (do not use the entry point
 * on a device after a cudaDeviceReset of it); cuda_stream must belong to the
 * current device (else UFC_STATUS_INVALID); calls that overlap on the GPU share
 * the array and race, so the caller serialises them.  The message of a failure
 * is written to errbuf (may be NULL). */
#define UFC_NOALLOC_MAX_ROWS 16777216
int ufc_csr_spmv_dot_noalloc(int64_t n_rows, const int64_t* row_ptr, const int32_t* col_ind,
                             const double* values, const double* x, double* y, double* xy, void* cuda_stream,
                             char* errbuf, int32_t errlen);

#ifdef __cplusplus
}
#endif
#endif /* UFC_GPU_H */
