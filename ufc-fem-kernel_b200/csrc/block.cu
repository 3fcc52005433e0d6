// Multi-right-hand-side Jacobi-PCG (placeholder until the shared-SpMV kernel lands).
#include "ufc_internal.cuh"

namespace ufc {

int pcg_solve_block(Ctx* c, int nrhs, const double* B, double* X, const ufc_solver_algo* algo,
                    ufc_solver_state* st) {
  (void)nrhs; (void)B; (void)X; (void)algo; (void)st;
  return fail(c, UFC_STATUS_UNSUPPORTED, "ufc_pcg_solve_block: not available in this build");
}

}  // namespace ufc
