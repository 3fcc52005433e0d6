!===============================================================================
! ufc_gpu_brg.f90 -- ISO_C_BINDING interface to libufc_gpu.so (include/ufc_gpu.h)
!
! The Fortran side of the drop-in boundary: derived types with BIND(C) that
! mirror the C structs field by field, and interfaces to the extern "C" entry
! points, in the style of the reference's existing BIND(C) bridges
! (ufc_core/L2_NM/Solver/LinSolv/NM_Solv_Dir.f90:19-47).  Status values are the
! IF_STATUS_* codes of ufc_core/L1_IF/Error/IF_Err_Brg.f90:95-110.
!
! Not compiled in this repository (no Fortran compiler is available where it is
! built); the C layouts it must match are checked by tests/test_abi.py.
!===============================================================================
MODULE ufc_gpu_brg
  USE, INTRINSIC :: ISO_C_BINDING
  IMPLICIT NONE
  PRIVATE

  INTEGER(C_INT32_T), PARAMETER, PUBLIC :: UFC_MEM_HOST = 0, UFC_MEM_DEVICE = 1
  INTEGER(C_INT32_T), PARAMETER, PUBLIC :: UFC_MAT_ELASTIC_ISO = 101, UFC_MAT_J2_ISO = 201
  INTEGER(C_INT32_T), PARAMETER, PUBLIC :: UFC_SOLV_METHOD_CG = 3, UFC_SOLV_PREC_JACOBI = 1, UFC_SOLV_PREC_MG = 5
  INTEGER(C_INT32_T), PARAMETER, PUBLIC :: UFC_PRECISION_FP64 = 0, UFC_PRECISION_FP32_REFINE = 1
  INTEGER(C_INT32_T), PARAMETER, PUBLIC :: UFC_BUILD_FP64 = 1, UFC_BUILD_FP32 = 2
  INTEGER(C_INT32_T), PARAMETER, PUBLIC :: UFC_BUILD_FP32_ROUNDED = 4, UFC_BUILD_FP32_DIFF = 8
  INTEGER(C_INT32_T), PARAMETER, PUBLIC :: UFC_BUILD_SYMMETRIC = 16
  INTEGER(C_INT32_T), PARAMETER, PUBLIC :: UFC_SOLV_PREC_NONE = 0, UFC_PRECISION_FP32_MATRIX = 2
  INTEGER(C_INT32_T), PARAMETER, PUBLIC :: UFC_ACCUMULATE_STORAGE = 0, UFC_ACCUMULATE_FP64 = 1
  INTEGER(C_INT32_T), PARAMETER, PUBLIC :: UFC_REFINE_KEEP_DIRECTION = 0, UFC_REFINE_RESTART = 1
  INTEGER(C_INT32_T), PARAMETER, PUBLIC :: UFC_REFINE_FORCE_FP32 = 2
  ! IF_Err_Brg status codes (ufc_core/L1_IF/Error/IF_Err_Brg.f90:95-110)
  INTEGER(C_INT), PARAMETER, PUBLIC :: UFC_STATUS_OK = 0, UFC_STATUS_INVALID = 1, UFC_STATUS_ERROR = 2
  INTEGER(C_INT), PARAMETER, PUBLIC :: UFC_STATUS_CONVERGED = 3, UFC_STATUS_NOT_CONVERGED = 4
  INTEGER(C_INT), PARAMETER, PUBLIC :: UFC_STATUS_NOT_FOUND = 5, UFC_STATUS_WARN = 6, UFC_STATUS_MEM_ERROR = 7
  INTEGER(C_INT), PARAMETER, PUBLIC :: UFC_STATUS_IO_ERROR = 8, UFC_STATUS_EXISTS = 9, UFC_STATUS_FATAL = 10
  INTEGER(C_INT), PARAMETER, PUBLIC :: UFC_STATUS_UNSUPPORTED = 11
  INTEGER(C_INT64_T), PARAMETER, PUBLIC :: UFC_NOALLOC_MAX_ROWS = 16777216_C_INT64_T

  TYPE, BIND(C), PUBLIC :: ufc_mesh_desc
    INTEGER(C_INT32_T) :: n_nodes, n_elems
    TYPE(C_PTR)        :: coords, conn          ! REAL(C_DOUBLE)(3,n_nodes), INTEGER(C_INT32_T)(8,n_elems)
    INTEGER(C_INT32_T) :: index_base, mem       ! index_base = 1 for Fortran connectivity
  END TYPE

  TYPE, BIND(C), PUBLIC :: ufc_material_desc
    INTEGER(C_INT32_T) :: mat_model_id, nprops, per_element
    TYPE(C_PTR)        :: props                 ! REAL(C_DOUBLE)(nprops[,n_elems])
    INTEGER(C_INT32_T) :: mem
  END TYPE

  TYPE, BIND(C), PUBLIC :: ufc_bc_desc
    INTEGER(C_INT32_T) :: n_fixed
    TYPE(C_PTR)        :: dofs, values
    INTEGER(C_INT32_T) :: mem
  END TYPE

  TYPE, BIND(C), PUBLIC :: ufc_pattern_info
    INTEGER(C_INT64_T) :: n_dof, nnz, nnzb, sell_blocks
    INTEGER(C_INT32_T) :: n_colors, max_row_blocks
  END TYPE

  TYPE, BIND(C), PUBLIC :: ufc_csr_export_arg
    INTEGER(C_INT32_T) :: index_base, mem
    TYPE(C_PTR)        :: row_ptr, col_ind, values, values32
  END TYPE

  TYPE, BIND(C), PUBLIC :: ufc_elem_ke_arg
    INTEGER(C_INT32_T) :: build, status
    REAL(C_DOUBLE)     :: elapsed_ms
  END TYPE

  TYPE, BIND(C), PUBLIC :: ufc_elem_fe_arg
    TYPE(C_PTR)        :: u, f_ext, fint, r
    INTEGER(C_INT32_T) :: mem, update_state
    REAL(C_DOUBLE)     :: rnorm, fint_norm
    INTEGER(C_INT32_T) :: status
  END TYPE

  TYPE, BIND(C), PUBLIC :: ufc_mat_update_arg
    INTEGER(C_INT32_T) :: mat_model_id, n_points, nprops, props_per_point
    TYPE(C_PTR)        :: props, stress_n, dstrain, sdv_n, stress, sdv, ddsdde, yielded
    INTEGER(C_INT32_T) :: mem, status
  END TYPE

  TYPE, BIND(C), PUBLIC :: ufc_solver_algo          ! NM_Solver_Algo
    INTEGER(C_INT32_T) :: method = UFC_SOLV_METHOD_CG, precond_type = UFC_SOLV_PREC_JACOBI
    INTEGER(C_INT32_T) :: max_iter = 100000, precision_mode = UFC_PRECISION_FP64
    REAL(C_DOUBLE)     :: tolerance = 1.0D-10, abs_tolerance = 0.0D0, refine_delta = 0.0D0
    INTEGER(C_INT32_T) :: check_every = 0, use_x0 = 0, refine_policy = 0, accumulate = 0
  END TYPE

  TYPE, BIND(C), PUBLIC :: ufc_solver_state         ! NM_Solver_State
    INTEGER(C_INT32_T) :: niter, n_refine, converged, convergence_flag
    REAL(C_DOUBLE)     :: rnorm, initial_residual, solve_time
    INTEGER(C_INT32_T) :: fp64_iters, reserved
  END TYPE

  TYPE, BIND(C), PUBLIC :: ufc_nr_arg               ! RT_NLSolver_NewtonRaph, one increment
    TYPE(C_PTR)           :: u_prescribed, f_ext
    INTEGER(C_INT32_T)    :: mem, max_iterations
    REAL(C_DOUBLE)        :: tolerance_force
    TYPE(ufc_solver_algo) :: lin
    INTEGER(C_INT32_T)    :: iterations, converged, lin_iters_total
    REAL(C_DOUBLE)        :: residual_norm, res_hist(32)
    INTEGER(C_INT32_T)    :: status
  END TYPE

  TYPE, BIND(C), PUBLIC :: ufc_step_arg             ! RT_StepDriver_Execute, one step with cutbacks
    TYPE(C_PTR)           :: u_prescribed_end, f_ext_start, f_ext_end
    INTEGER(C_INT32_T)    :: mem
    REAL(C_DOUBLE)        :: time_period = 1.0D0, dt_initial = 1.0D0, dt_min = 1.0D-5, dt_max = 1.0D0
    INTEGER(C_INT32_T)    :: max_increments = 100, max_cutbacks = 5, auto_dt = 1, target_iters = 6
    REAL(C_DOUBLE)        :: growth_threshold = 0.8D0, growth_factor = 1.25D0, cutback_factor = 0.5D0
    INTEGER(C_INT32_T)    :: max_iterations = 25
    REAL(C_DOUBLE)        :: tolerance_force = 1.0D-8
    TYPE(ufc_solver_algo) :: lin
    TYPE(C_PTR)           :: hist_time, hist_dt, hist_iters, hist_converged
    INTEGER(C_INT32_T)    :: hist_cap = 0, attempts, increments, cutbacks, nr_iterations
    INTEGER(C_INT64_T)    :: lin_iters_total
    REAL(C_DOUBLE)        :: final_time
    INTEGER(C_INT32_T)    :: completed, status
  END TYPE

  TYPE, BIND(C), PUBLIC :: ufc_mg_arg               ! multigrid in the place of NM_AMG_Setup
    INTEGER(C_INT32_T)    :: nx, ny, nz, max_levels = 0, degree = 0
    REAL(C_DOUBLE)        :: ratio = 0.0D0
    INTEGER(C_INT64_T)    :: coarse_max = 0
    INTEGER(C_INT32_T)    :: levels, precision = 0
    INTEGER(C_INT64_T)    :: coarse_dof
    REAL(C_DOUBLE)        :: setup_ms
  END TYPE

  TYPE, BIND(C), PUBLIC :: ufc_face_load_arg        ! PH_Elem_C3D8_FormFacePressure over a face set
    INTEGER(C_INT32_T)    :: n_faces
    TYPE(C_PTR)           :: elem, face, traction, pressure
    INTEGER(C_INT32_T)    :: index_base, mem
    TYPE(C_PTR)           :: f
  END TYPE

  TYPE, BIND(C), PUBLIC :: ufc_timing_info          ! device-time counters of the last solve
    INTEGER(C_INT32_T) :: spmv_launches
    REAL(C_DOUBLE)     :: spmv_ms
    INTEGER(C_INT64_T) :: spmv_bytes
    INTEGER(C_INT32_T) :: precision
    INTEGER(C_INT64_T) :: kernel_launches
  END TYPE

  PUBLIC :: ufc_ctx_create, ufc_ctx_destroy, ufc_last_error, ufc_mesh_set, ufc_material_set, ufc_bc_set
  PUBLIC :: ufc_ctx_set_stream, ufc_ctx_set_instrument, ufc_stress_eval, ufc_spmv, ufc_mg_level_info
  PUBLIC :: ufc_mg_export, ufc_last_timing, ufc_last_residual_history, ufc_set_displacement, ufc_get_state
  PUBLIC :: ufc_csr_spmv_dot_noalloc
  PUBLIC :: ufc_pattern_build, ufc_csr_export, ufc_pattern_colors, ufc_elem_compute_ke, ufc_elem_compute_fint
  PUBLIC :: ufc_mat_update_batch, ufc_pcg_solve, ufc_pcg_solve_block, ufc_nr_increment
  PUBLIC :: ufc_state_commit, ufc_state_rollback, ufc_get_displacement, ufc_adjoint_sensitivity
  PUBLIC :: ufc_nr_step, ufc_load_faces, ufc_stress_nodal, ufc_reactions, ufc_mg_setup, ufc_mg_apply

  INTERFACE
    INTEGER(C_INT) FUNCTION ufc_ctx_create(device, ctx) BIND(C, NAME='ufc_ctx_create')
      IMPORT :: C_INT, C_INT32_T, C_PTR
      INTEGER(C_INT32_T), VALUE :: device
      TYPE(C_PTR), INTENT(OUT)  :: ctx
    END FUNCTION
    INTEGER(C_INT) FUNCTION ufc_ctx_destroy(ctx) BIND(C, NAME='ufc_ctx_destroy')
      IMPORT :: C_INT, C_PTR
      TYPE(C_PTR), VALUE :: ctx
    END FUNCTION
    INTEGER(C_INT) FUNCTION ufc_last_error(ctx, buf, buflen) BIND(C, NAME='ufc_last_error')
      IMPORT :: C_INT, C_PTR, C_CHAR, C_INT32_T
      TYPE(C_PTR), VALUE            :: ctx
      CHARACTER(KIND=C_CHAR)        :: buf(*)
      INTEGER(C_INT32_T), VALUE     :: buflen
    END FUNCTION
    INTEGER(C_INT) FUNCTION ufc_mesh_set(ctx, mesh) BIND(C, NAME='ufc_mesh_set')
      IMPORT :: C_INT, C_PTR, ufc_mesh_desc
      TYPE(C_PTR), VALUE               :: ctx
      TYPE(ufc_mesh_desc), INTENT(IN)  :: mesh
    END FUNCTION
    INTEGER(C_INT) FUNCTION ufc_material_set(ctx, mat) BIND(C, NAME='ufc_material_set')
      IMPORT :: C_INT, C_PTR, ufc_material_desc
      TYPE(C_PTR), VALUE                  :: ctx
      TYPE(ufc_material_desc), INTENT(IN) :: mat
    END FUNCTION
    INTEGER(C_INT) FUNCTION ufc_bc_set(ctx, bc) BIND(C, NAME='ufc_bc_set')
      IMPORT :: C_INT, C_PTR, ufc_bc_desc
      TYPE(C_PTR), VALUE            :: ctx
      TYPE(ufc_bc_desc), INTENT(IN) :: bc
    END FUNCTION
    INTEGER(C_INT) FUNCTION ufc_pattern_build(ctx, info) BIND(C, NAME='ufc_pattern_build')
      IMPORT :: C_INT, C_PTR, ufc_pattern_info
      TYPE(C_PTR), VALUE                   :: ctx
      TYPE(ufc_pattern_info), INTENT(OUT)  :: info
    END FUNCTION
    INTEGER(C_INT) FUNCTION ufc_csr_export(ctx, arg) BIND(C, NAME='ufc_csr_export')
      IMPORT :: C_INT, C_PTR, ufc_csr_export_arg
      TYPE(C_PTR), VALUE                   :: ctx
      TYPE(ufc_csr_export_arg), INTENT(IN) :: arg
    END FUNCTION
    INTEGER(C_INT) FUNCTION ufc_pattern_colors(ctx, color_of, index_base, mem) &
        BIND(C, NAME='ufc_pattern_colors')
      IMPORT :: C_INT, C_PTR, C_INT32_T
      TYPE(C_PTR), VALUE               :: ctx
      INTEGER(C_INT32_T), INTENT(OUT)  :: color_of(*)
      INTEGER(C_INT32_T), VALUE        :: index_base
      INTEGER(C_INT32_T), VALUE        :: mem
    END FUNCTION
    INTEGER(C_INT) FUNCTION ufc_elem_compute_ke(ctx, arg) BIND(C, NAME='ufc_elem_compute_ke')
      IMPORT :: C_INT, C_PTR, ufc_elem_ke_arg
      TYPE(C_PTR), VALUE                  :: ctx
      TYPE(ufc_elem_ke_arg), INTENT(INOUT) :: arg
    END FUNCTION
    INTEGER(C_INT) FUNCTION ufc_elem_compute_fint(ctx, arg) BIND(C, NAME='ufc_elem_compute_fint')
      IMPORT :: C_INT, C_PTR, ufc_elem_fe_arg
      TYPE(C_PTR), VALUE                  :: ctx
      TYPE(ufc_elem_fe_arg), INTENT(INOUT) :: arg
    END FUNCTION
    INTEGER(C_INT) FUNCTION ufc_mat_update_batch(ctx, arg) BIND(C, NAME='ufc_mat_update_batch')
      IMPORT :: C_INT, C_PTR, ufc_mat_update_arg
      TYPE(C_PTR), VALUE                      :: ctx
      TYPE(ufc_mat_update_arg), INTENT(INOUT) :: arg
    END FUNCTION
    INTEGER(C_INT) FUNCTION ufc_pcg_solve(ctx, b, x, mem, algo, state) BIND(C, NAME='ufc_pcg_solve')
      IMPORT :: C_INT, C_PTR, C_DOUBLE, C_INT32_T, ufc_solver_algo, ufc_solver_state
      TYPE(C_PTR), VALUE                    :: ctx
      REAL(C_DOUBLE), INTENT(IN)            :: b(*)
      REAL(C_DOUBLE), INTENT(INOUT)         :: x(*)
      INTEGER(C_INT32_T), VALUE             :: mem
      TYPE(ufc_solver_algo), INTENT(IN)     :: algo
      TYPE(ufc_solver_state), INTENT(OUT)   :: state
    END FUNCTION
    INTEGER(C_INT) FUNCTION ufc_pcg_solve_block(ctx, nrhs, b, x, mem, algo, states) &
        BIND(C, NAME='ufc_pcg_solve_block')
      IMPORT :: C_INT, C_PTR, C_DOUBLE, C_INT32_T, ufc_solver_algo, ufc_solver_state
      TYPE(C_PTR), VALUE                    :: ctx
      INTEGER(C_INT32_T), VALUE             :: nrhs
      REAL(C_DOUBLE), INTENT(IN)            :: b(*)
      REAL(C_DOUBLE), INTENT(INOUT)         :: x(*)
      INTEGER(C_INT32_T), VALUE             :: mem
      TYPE(ufc_solver_algo), INTENT(IN)     :: algo
      TYPE(ufc_solver_state), INTENT(OUT)   :: states(*)
    END FUNCTION
    INTEGER(C_INT) FUNCTION ufc_nr_increment(ctx, arg) BIND(C, NAME='ufc_nr_increment')
      IMPORT :: C_INT, C_PTR, ufc_nr_arg
      TYPE(C_PTR), VALUE               :: ctx
      TYPE(ufc_nr_arg), INTENT(INOUT)  :: arg
    END FUNCTION
    INTEGER(C_INT) FUNCTION ufc_nr_step(ctx, arg) BIND(C, NAME='ufc_nr_step')
      IMPORT :: C_INT, C_PTR, ufc_step_arg
      TYPE(C_PTR), VALUE                 :: ctx
      TYPE(ufc_step_arg), INTENT(INOUT)  :: arg
    END FUNCTION
    INTEGER(C_INT) FUNCTION ufc_mg_setup(ctx, arg) BIND(C, NAME='ufc_mg_setup')
      IMPORT :: C_INT, C_PTR, ufc_mg_arg
      TYPE(C_PTR), VALUE               :: ctx
      TYPE(ufc_mg_arg), INTENT(INOUT)  :: arg
    END FUNCTION
    INTEGER(C_INT) FUNCTION ufc_mg_apply(ctx, r, z, mem) BIND(C, NAME='ufc_mg_apply')
      IMPORT :: C_INT, C_PTR, C_DOUBLE, C_INT32_T
      TYPE(C_PTR), VALUE            :: ctx
      REAL(C_DOUBLE), INTENT(IN)    :: r(*)
      REAL(C_DOUBLE), INTENT(OUT)   :: z(*)
      INTEGER(C_INT32_T), VALUE     :: mem
    END FUNCTION
    INTEGER(C_INT) FUNCTION ufc_load_faces(ctx, arg) BIND(C, NAME='ufc_load_faces')
      IMPORT :: C_INT, C_PTR, ufc_face_load_arg
      TYPE(C_PTR), VALUE                  :: ctx
      TYPE(ufc_face_load_arg), INTENT(IN) :: arg
    END FUNCTION
    INTEGER(C_INT) FUNCTION ufc_stress_nodal(ctx, u, stress_node, vm_node, mem) BIND(C, NAME='ufc_stress_nodal')
      IMPORT :: C_INT, C_PTR, C_INT32_T
      TYPE(C_PTR), VALUE            :: ctx, u, stress_node, vm_node   ! C_NULL_PTR where not wanted
      INTEGER(C_INT32_T), VALUE     :: mem
    END FUNCTION
    INTEGER(C_INT) FUNCTION ufc_reactions(ctx, u, f_ext, rf, mem) BIND(C, NAME='ufc_reactions')
      IMPORT :: C_INT, C_PTR, C_INT32_T
      TYPE(C_PTR), VALUE            :: ctx, u, f_ext, rf              ! u, f_ext may be C_NULL_PTR
      INTEGER(C_INT32_T), VALUE     :: mem
    END FUNCTION
    INTEGER(C_INT) FUNCTION ufc_state_commit(ctx) BIND(C, NAME='ufc_state_commit')
      IMPORT :: C_INT, C_PTR
      TYPE(C_PTR), VALUE :: ctx
    END FUNCTION
    INTEGER(C_INT) FUNCTION ufc_state_rollback(ctx) BIND(C, NAME='ufc_state_rollback')
      IMPORT :: C_INT, C_PTR
      TYPE(C_PTR), VALUE :: ctx
    END FUNCTION
    INTEGER(C_INT) FUNCTION ufc_get_displacement(ctx, u, mem) BIND(C, NAME='ufc_get_displacement')
      IMPORT :: C_INT, C_PTR, C_DOUBLE, C_INT32_T
      TYPE(C_PTR), VALUE            :: ctx
      REAL(C_DOUBLE), INTENT(OUT)   :: u(*)
      INTEGER(C_INT32_T), VALUE     :: mem
    END FUNCTION
    INTEGER(C_INT) FUNCTION ufc_adjoint_sensitivity(ctx, nrhs, u, lam, dJdE, mem) &
        BIND(C, NAME='ufc_adjoint_sensitivity')
      IMPORT :: C_INT, C_PTR, C_DOUBLE, C_INT32_T
      TYPE(C_PTR), VALUE            :: ctx
      INTEGER(C_INT32_T), VALUE     :: nrhs
      REAL(C_DOUBLE), INTENT(IN)    :: u(*), lam(*)
      REAL(C_DOUBLE), INTENT(OUT)   :: dJdE(*)
      INTEGER(C_INT32_T), VALUE     :: mem
    END FUNCTION
    INTEGER(C_INT) FUNCTION ufc_ctx_set_stream(ctx, cuda_stream) BIND(C, NAME='ufc_ctx_set_stream')
      IMPORT :: C_INT, C_PTR
      TYPE(C_PTR), VALUE            :: ctx, cuda_stream   ! a cudaStream_t, or C_NULL_PTR for the context's own
    END FUNCTION
    INTEGER(C_INT) FUNCTION ufc_ctx_set_instrument(ctx, on) BIND(C, NAME='ufc_ctx_set_instrument')
      IMPORT :: C_INT, C_PTR, C_INT32_T
      TYPE(C_PTR), VALUE            :: ctx
      INTEGER(C_INT32_T), VALUE     :: on
    END FUNCTION
    INTEGER(C_INT) FUNCTION ufc_stress_eval(ctx, u, stress_gp, vm_gp, mem) BIND(C, NAME='ufc_stress_eval')
      IMPORT :: C_INT, C_PTR, C_INT32_T
      TYPE(C_PTR), VALUE            :: ctx, u, stress_gp, vm_gp   ! C_NULL_PTR where not wanted
      INTEGER(C_INT32_T), VALUE     :: mem
    END FUNCTION
    INTEGER(C_INT) FUNCTION ufc_spmv(ctx, precision, x, y, mem) BIND(C, NAME='ufc_spmv')
      IMPORT :: C_INT, C_PTR, C_INT32_T
      TYPE(C_PTR), VALUE            :: ctx, x, y          ! REAL(C_DOUBLE) or REAL(C_FLOAT) by precision
      INTEGER(C_INT32_T), VALUE     :: precision, mem
    END FUNCTION
    INTEGER(C_INT) FUNCTION ufc_mg_level_info(ctx, level, n_dof, nnz) BIND(C, NAME='ufc_mg_level_info')
      IMPORT :: C_INT, C_PTR, C_INT32_T, C_INT64_T
      TYPE(C_PTR), VALUE            :: ctx
      INTEGER(C_INT32_T), VALUE     :: level
      INTEGER(C_INT64_T), INTENT(OUT) :: n_dof, nnz
    END FUNCTION
    INTEGER(C_INT) FUNCTION ufc_mg_export(ctx, level, arg) BIND(C, NAME='ufc_mg_export')
      IMPORT :: C_INT, C_PTR, C_INT32_T, ufc_csr_export_arg
      TYPE(C_PTR), VALUE                   :: ctx
      INTEGER(C_INT32_T), VALUE            :: level
      TYPE(ufc_csr_export_arg), INTENT(IN) :: arg
    END FUNCTION
    INTEGER(C_INT) FUNCTION ufc_last_timing(ctx, info) BIND(C, NAME='ufc_last_timing')
      IMPORT :: C_INT, C_PTR, ufc_timing_info
      TYPE(C_PTR), VALUE                   :: ctx
      TYPE(ufc_timing_info), INTENT(OUT)   :: info
    END FUNCTION
    INTEGER(C_INT) FUNCTION ufc_last_residual_history(ctx, out, max_len, out_len) &
        BIND(C, NAME='ufc_last_residual_history')
      IMPORT :: C_INT, C_PTR, C_DOUBLE, C_INT32_T
      TYPE(C_PTR), VALUE            :: ctx
      REAL(C_DOUBLE), INTENT(OUT)   :: out(*)
      INTEGER(C_INT32_T), VALUE     :: max_len
      INTEGER(C_INT32_T), INTENT(OUT) :: out_len
    END FUNCTION
    INTEGER(C_INT) FUNCTION ufc_set_displacement(ctx, u, mem) BIND(C, NAME='ufc_set_displacement')
      IMPORT :: C_INT, C_PTR, C_DOUBLE, C_INT32_T
      TYPE(C_PTR), VALUE            :: ctx
      REAL(C_DOUBLE), INTENT(IN)    :: u(*)
      INTEGER(C_INT32_T), VALUE     :: mem
    END FUNCTION
    INTEGER(C_INT) FUNCTION ufc_get_state(ctx, eps_p_eq, stress, eps_p, mem) BIND(C, NAME='ufc_get_state')
      IMPORT :: C_INT, C_PTR, C_INT32_T
      TYPE(C_PTR), VALUE            :: ctx, eps_p_eq, stress, eps_p   ! C_NULL_PTR where not wanted
      INTEGER(C_INT32_T), VALUE     :: mem
    END FUNCTION
    ! device pointers (C_PTR from a CUDA Fortran or C allocation); no allocation inside
    INTEGER(C_INT) FUNCTION ufc_csr_spmv_dot_noalloc(n_rows, row_ptr, col_ind, values, x, y, xy, cuda_stream, &
        errbuf, errlen) BIND(C, NAME='ufc_csr_spmv_dot_noalloc')
      IMPORT :: C_INT, C_PTR, C_INT64_T, C_INT32_T, C_CHAR
      INTEGER(C_INT64_T), VALUE     :: n_rows
      TYPE(C_PTR), VALUE            :: row_ptr, col_ind, values, x, y, xy, cuda_stream
      CHARACTER(KIND=C_CHAR), INTENT(OUT) :: errbuf(*)
      INTEGER(C_INT32_T), VALUE     :: errlen
    END FUNCTION
  END INTERFACE
END MODULE ufc_gpu_brg
