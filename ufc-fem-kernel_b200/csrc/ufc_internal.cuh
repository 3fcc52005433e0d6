// Internal declarations of the B200 C3D8 hot path (not part of the C-ABI).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <vector>

#include "../../include/ufc_gpu.h"

namespace ufc {

constexpr int kSlice = 32;       // rows per SELL slice = one warp
constexpr int kMaxValence = 32;  // elements sharing one node (general hex meshes)
constexpr int kMaxRowBlocks = 128;
// The Jacobi-PCG aims for an FP64 residual ||b - K x|| of at most kStopMargin
// times the requested max(rtol ||b||, atol): an evaluation of the same residual
// with another summation order (the CPU oracle's CSR) differs by rounding of
// order u ||K|| ||x||, 0.5 % of the tolerance on the 5.4M-DOF cantilever, and
// the margin keeps that evaluation within the tolerance too.  When the residual
// stops decreasing before the margin is met (rtol 1e-10 is at the FP64
// rounding floor of that problem: the oracle evaluates its own rtol-1e-13
// solution at 1.4e-10), the run is accepted once it is within the requested
// tolerance itself.
constexpr double kStopMargin = 0.97;
constexpr int kGraphSlots = 4;   // cached CG-batch graphs: one per solver type combination

// Scalars of one CG run, kept on the device so iterations need no host sync.
struct CgScalars {
  double rz;        // r.z of the current iterate
  double rz_old;    // r.z used by the last alpha
  double pq;        // p.Ap
  double alpha, beta;
  double rr;        // ||r||^2 of the recursive residual
  double rr_ref;    // ||r||^2 at the last FP64 residual replacement
  double tol2;      // stop threshold on ||r||^2
  double delta2;    // replacement trigger (FP32_REFINE)
  double true_rr;   // ||b - K x||^2 from the last FP64 residual
  double bb;        // ||b||^2
  int32_t iter;
  int32_t max_iter;
  int32_t stop;     // 1 converged (recursive), 2 max-iter, 3 breakdown
  int32_t want_update;
  double nr_rr, nr_ff, nr_ee;  // Newton: ||R_free||^2, ||F_int||^2, ||F_ext||^2
  double* hist;        // ||r||^2 of the recursive residual per iteration (or null)
  int32_t hist_cap;
  uint32_t ticket[8];  // last-block election counters, one per reduction site
};

// Error word written by device kernels (never trap).
enum DevErr : int32_t {
  kDevOk = 0,
  kDevBadJacobian = 1,
  kDevNonFinite = 2,
  kDevValence = 4,
  kDevRowBlocks = 8,
  kDevPattern = 16,
  kDevTimeout = 32,  // a bounded wait (mbarrier) gave up
};

// 32 code bytes of one row, consumed from the front one block step at a time.
struct Code256 {
  uint64_t w0, w1, w2, w3;
  __device__ __forceinline__ unsigned front() const { return (unsigned)(w0 & 0xFFu); }
  template <int B>
  __device__ __forceinline__ void drop() {
    if constexpr (B >= 8) {
      w0 = w1;
      w1 = w2;
      w2 = w3;
      w3 = 0;
    } else {
      constexpr int sh = 8 * B;
      w0 = (w0 >> sh) | (w1 << (64 - sh));
      w1 = (w1 >> sh) | (w2 << (64 - sh));
      w2 = (w2 >> sh) | (w3 << (64 - sh));
      w3 >>= sh;
    }
  }
};

struct Mg;  // multigrid hierarchy (mg.cu)

// Block-column offsets (col - row) of the upper half of a stencil-like block
// pattern: entry k of a row's coded index is the position of its offset here.
constexpr int kSymCodes = 15;      // offsets a code can name; code 15 = no block
struct SymOffsets {
  int32_t off[16];
};
// The same for the full block pattern (col - row of either sign): up to 31
// offsets, code 255 = no block; 32 code bytes per row.
constexpr int kFullCodes = 31;
struct FullOffsets {
  int32_t off[32];
};

struct Ctx {
  int device = 0;
  cudaStream_t stream = nullptr;  // own non-blocking stream: all work runs here
  cudaStream_t ext = nullptr;     // caller's stream, joined on entry and exit
  bool has_ext = false;
  cudaEvent_t ev_join = nullptr;
  std::string err;
  bool instrument = false;
  ufc_timing_info timing{};
  int64_t launches = 0;  // kernels enqueued by the library (counted at each launch site)

  // mesh
  int32_t N = 0, E = 0;
  int64_t n = 0;
  double* coords = nullptr;  // [N*3]
  int32_t* conn = nullptr;   // [E*8], 0-based
  std::vector<int32_t> h_conn;

  // material
  int32_t mat_model = 0, nprops = 0;
  double* props = nullptr;  // [E*nprops]
  bool has_material = false;

  // colouring
  int32_t ncol = 0;
  std::vector<int32_t> col_off;      // ncol+1
  int32_t* col_elems = nullptr;      // [E] elements grouped by colour, ascending inside a colour
  std::vector<int32_t> h_color;      // [E] colour of each element (host)

  // pattern: canonical block CSR + SELL-32 storage
  bool has_pattern = false;
  int64_t nnzb = 0;
  int32_t max_row_blocks = 0;
  int32_t* brow = nullptr;    // [N+1]
  int32_t* bcol = nullptr;    // [nnzb]
  int64_t nslices = 0, sell_blocks = 0;
  int64_t* slice_ptr = nullptr;  // [nslices+1] block offsets
  int32_t* sell_col = nullptr;   // [sell_blocks]
  int32_t* slot = nullptr;       // [E*64] SELL position of block (a, b)
  int32_t* dpos = nullptr;       // [N] SELL position of the diagonal block
  double* val64 = nullptr;       // [sell_blocks*9]
  float* val32 = nullptr;
  bool has_val64 = false, has_val32 = false;
  bool val32_diff = false;       // FP32 values in difference form (diagonal slot = block row sum)
  double* dinv64 = nullptr;
  float* dinv32 = nullptr;

  // symmetric SpMV storage: upper-triangle blocks (j >= i) in SELL-32, plus per
  // row the positions of its lower blocks (stored transposed in earlier rows)
  bool has_sym_pattern = false;
  int64_t s_ublocks = 0, s_lblocks = 0;  // stored upper blocks (+ one zero slice), lower refs
  int64_t* uptr = nullptr;               // [nslices+1]
  int32_t* ucol = nullptr;               // [s_ublocks]
  int64_t* lptr = nullptr;               // [nslices+1]
  int32_t* lpos = nullptr;               // [s_lblocks] upper-storage position of block (j, i)
  int32_t* lcol = nullptr;               // [s_lblocks] j
  int32_t* s_lcnt = nullptr;             // [N] lower blocks per row (= position of the diagonal)
  double* sval64 = nullptr;              // [(s_ublocks + 32) * 9]
  float* sval32 = nullptr;
  bool has_sval64 = false, has_sval32 = false;
  // coded indices of the symmetric storage (when every slice has at most 16
  // upper and 16 lower steps and the pattern has at most 15 distinct upper
  // offsets): per row 16 bytes of upper codes and 16 of lower codes, one
  // 16-byte load each; a lower code holds the offset code (high nibble) and
  // the rank of the block in its row's upper list (low nibble)
  bool sym_coded = false;
  // coded indices of the full SELL storage (rows of at most 32 blocks, at most
  // 31 distinct offsets): 32 code bytes per row, lane-major
  bool full_coded = false;
  FullOffsets full_tab{};
  int32_t full_ntab = 0;  // offsets in full_tab (ascending)
  uint8_t* full_code = nullptr;          // [nslices * 32 * 32]
  SymOffsets sym_tab{};
  uint8_t* sym_ucode = nullptr;          // [nslices * 32 * 16]
  uint8_t* sym_lcode = nullptr;

  // Dirichlet set
  uint8_t* fixed = nullptr;  // [n]
  int32_t nfix = 0;
  int32_t* fix_dofs = nullptr;
  double* fix_vals = nullptr;

  // solver work
  double *x64 = nullptr, *r64 = nullptr, *p64 = nullptr, *q64 = nullptr, *b64 = nullptr, *y64 = nullptr;
  float *r32 = nullptr, *p32 = nullptr, *q32 = nullptr;
  double* xb64 = nullptr;  // best iterate of an FP32 run (handed to the FP64 continuation)
  CgScalars* scal = nullptr;
  double* hist = nullptr;       // residual history of the last solve (device)
  int32_t hist_cap = 0, hist_len = 0;
  double* partials = nullptr;   // [partials_cap] per-block partial sums of grid reductions
  int64_t partials_cap = 0;
  CgScalars* h_scal = nullptr;  // pinned mirror
  int32_t* dev_err = nullptr;
  int32_t* h_err = nullptr;     // pinned

  // Newton work vectors
  double *nr_fint = nullptr, *nr_R = nullptr, *nr_du = nullptr, *nr_dc = nullptr;

  // displacement and J2 state
  double* u = nullptr;      // [n] current
  double* u_n = nullptr;    // [n] committed
  double *sig_n = nullptr, *epeq_n = nullptr, *epl_n = nullptr;  // committed [G*6],[G],[G*6]
  double *sig_t = nullptr, *epeq_t = nullptr, *epl_t = nullptr;  // trial
  double* Dt = nullptr;     // [G*36] consistent tangent of the trial state
  bool has_trial = false;

  // multigrid preconditioner (ufc_mg_setup), and the preconditioned vector z
  Mg* mg = nullptr;
  double* z64 = nullptr;

  // cached CUDA graphs of CG batches
  cudaGraphExec_t cg_graph[kGraphSlots] = {};
  int cg_graph_batch[kGraphSlots] = {};
  // what a cached graph baked in: value and diagonal arrays, storage and SpMV form
  const void* cg_graph_val[kGraphSlots] = {};
  const void* cg_graph_key[kGraphSlots] = {};
  int cg_graph_form[kGraphSlots] = {};
  int64_t cg_graph_n[kGraphSlots] = {}, cg_graph_slices[kGraphSlots] = {};
  std::vector<cudaEvent_t> ev_pool;
};

int grid_for(int64_t work, int block);
int fail(Ctx* c, int status, const std::string& msg);
int cuda_fail(Ctx* c, cudaError_t e, const char* where);
int check_dev_err(Ctx* c, const char* where);

// pattern.cu
int build_pattern(Ctx* c);
int build_sym_pattern(Ctx* c);
int build_sym_codes(Ctx* c);
int build_full_codes(Ctx* c);
int pack_symmetric(Ctx* c, bool fp64, bool fp32);  // full SELL values -> symmetric SpMV copies
int export_csr(Ctx* c, const ufc_csr_export_arg* a);

// c3d8.cu
int assemble(Ctx* c, int build, double* elapsed_ms);
int apply_fp64(Ctx* c, const double* x, double* y, bool masked);  // y = K x matrix-free, FP64
int apply_fp64_eliminated(Ctx* c, const double* x, double* y);    // eliminated operator incl. identity rows
int nr_norms(Ctx* c, const double* fext, const double* fint, double* R);  // R = fext - fint (free), norms
int compute_fint(Ctx* c, const double* u, double* fint, bool update_state);
int apply_tangent(Ctx* c, const double* x, double* y);  // y = K_tangent x, matrix-free, all DOFs
int mat_update_batch(Ctx* c, const ufc_mat_update_arg* a, const double* props, const double* stress_n,
                     const double* dstrain, const double* sdv_n, double* stress, double* sdv, double* ddsdde,
                     int32_t* yielded);
int stress_eval(Ctx* c, const double* u, double* sig, double* vm);
int adjoint_sens(Ctx* c, int nrhs, const double* U, const double* L, double* g);

// mg.cu
int mg_setup(Ctx* c, ufc_mg_arg* a);
void mg_free(Ctx* c);
void mg_mark_stale(Ctx* c);  // the matrix changed: the hierarchy must be set up again
int mg_apply(Ctx* c, const double* r, double* z);
int mg_level_ctx(Ctx* c, int32_t level, Ctx** out);
int pcg_mg(Ctx* c, const ufc_solver_algo* algo, ufc_solver_state* st);
// FP64 SELL SpMV (full storage) of any context's values, on the given stream (solver.cu)
void spmv64_on(const Ctx* lvl, cudaStream_t st, const double* x, double* y);
// FP32 SELL SpMV of the given values (standard form) on any context's pattern
void spmv32_on(const Ctx* lvl, cudaStream_t st, const float* val, const float* x, float* y);
void cg_spmv64(Ctx* c, const double* p, double* q);  // q = K p, p.q and alpha = r.z / p.q into the scalars
int true_residual_fp64(Ctx* c, bool want_bb);  // y64 = b64 - K x64, scal->true_rr (and bb)

// output.cu
int face_loads(Ctx* c, int32_t n_faces, const int32_t* h_elem, const int32_t* h_face, const double* traction,
               const double* pressure, double* f);  // h_elem 0-based, h_face 1..6 (host); others device
int stress_nodal(Ctx* c, const double* u, double* sig_node, double* vm_node);
int reactions(Ctx* c, const double* u, const double* f_ext, double* rf);
int build_dinv(Ctx* c, int precision);

// spmv.cu
int spmv(Ctx* c, int precision, const void* x, void* y);
int64_t spmv_bytes(const Ctx* c, int precision);

// pcg.cu
int pcg_solve(Ctx* c, const double* b, double* x, const ufc_solver_algo* algo, ufc_solver_state* st);
int pcg_solve_block(Ctx* c, int nrhs, const double* B, double* X, const ufc_solver_algo* algo,
                    ufc_solver_state* st);
void release_graphs(Ctx* c);

// device memory helper
template <class T>
int dalloc(Ctx* c, T** p, int64_t count) {
  if (*p) {
    cudaFree(*p);
    *p = nullptr;
  }
  if (count <= 0) count = 1;
  cudaError_t e = cudaMalloc((void**)p, sizeof(T) * (size_t)count);
  if (e != cudaSuccess) {
    *p = nullptr;
    return cuda_fail(c, e, "cudaMalloc");
  }
  return UFC_STATUS_OK;
}

template <class T>
void dfree(T** p) {
  if (*p) cudaFree(*p);
  *p = nullptr;
}

}  // namespace ufc

// the C-ABI's opaque context is the internal one
struct ufc_ctx : public ufc::Ctx {};

#define UFC_TRY(expr)                      \
  do {                                     \
    int _s = (expr);                       \
    if (_s != UFC_STATUS_OK) return _s;    \
  } while (0)

#define UFC_CUDA(c, expr)                                      \
  do {                                                         \
    cudaError_t _e = (expr);                                   \
    if (_e != cudaSuccess) return ufc::cuda_fail((c), _e, #expr); \
  } while (0)
