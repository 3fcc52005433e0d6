// extern "C" entry points of include/ufc_gpu.h: argument checking, host/device
// staging, stream joining, status codes, and the Newton-Raphson driver.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "ufc_internal.cuh"

namespace ufc {

int grid_for(int64_t work, int block) {
  int64_t g = (work + block - 1) / block;
  if (g < 1) g = 1;
  if (g > 0x7fffffff) g = 0x7fffffff;
  return (int)g;
}

int fail(Ctx* c, int status, const std::string& msg) {
  if (c) c->err = msg;
  return status;
}

int cuda_fail(Ctx* c, cudaError_t e, const char* where) {
  return fail(c, e == cudaErrorMemoryAllocation ? UFC_STATUS_MEM_ERROR : UFC_STATUS_ERROR,
              std::string(where) + ": " + cudaGetErrorString(e));
}

int check_dev_err(Ctx* c, const char* where) {
  UFC_CUDA(c, cudaMemcpyAsync(c->h_err, c->dev_err, sizeof(int32_t), cudaMemcpyDeviceToHost, c->stream));
  UFC_CUDA(c, cudaStreamSynchronize(c->stream));
  const int32_t e = *c->h_err;
  if (e == 0) return UFC_STATUS_OK;
  std::string m = std::string(where) + ":";
  if (e & kDevBadJacobian) m += " non-positive Jacobian determinant;";
  if (e & kDevNonFinite) m += " non-finite material state;";
  if (e & kDevValence) m += " a node is shared by more than 32 elements;";
  if (e & kDevRowBlocks) m += " a node couples to more than 128 nodes;";
  if (e & kDevPattern) m += " element block missing from the pattern;";
  if (e & kDevTimeout) m += " a bounded wait for an asynchronous copy gave up;";
  cudaMemsetAsync(c->dev_err, 0, sizeof(int32_t), c->stream);
  return fail(c, UFC_STATUS_ERROR, m);
}

namespace {

// Joins the caller's stream on entry and exit so that calls are ordered with it.
struct Scope {
  Ctx* c;
  int st = UFC_STATUS_OK;
  explicit Scope(Ctx* cc) : c(cc) {
    cudaSetDevice(c->device);
    if (c->has_ext) {
      cudaEventRecord(c->ev_join, c->ext);
      cudaStreamWaitEvent(c->stream, c->ev_join, 0);
    }
  }
  ~Scope() {
    if (c->has_ext) {
      cudaEventRecord(c->ev_join, c->stream);
      cudaStreamWaitEvent(c->ext, c->ev_join, 0);
    }
  }
};

// Device view of a caller buffer: device pointers pass through; host buffers
// are staged through stream-ordered allocations.
template <class T>
struct Staged {
  Ctx* c;
  T* host = nullptr;
  T* dev = nullptr;
  int64_t count = 0;
  bool owned = false;
  bool copy_back = false;
  ~Staged() {
    if (owned && dev) cudaFreeAsync(dev, c->stream);
  }
};

template <class T>
int stage_in(Ctx* c, Staged<T>& s, const T* p, int64_t count, int mem, bool copy_back = false) {
  s.c = c;
  s.count = count;
  s.host = const_cast<T*>(p);
  if (!p) return UFC_STATUS_OK;
  if (mem == UFC_MEM_DEVICE) {
    s.dev = const_cast<T*>(p);
    return UFC_STATUS_OK;
  }
  if (mem != UFC_MEM_HOST) return fail(c, UFC_STATUS_INVALID, "mem must be UFC_MEM_HOST or UFC_MEM_DEVICE");
  UFC_CUDA(c, cudaMallocAsync((void**)&s.dev, sizeof(T) * std::max<int64_t>(count, 1), c->stream));
  s.owned = true;
  s.copy_back = copy_back;
  UFC_CUDA(c, cudaMemcpyAsync(s.dev, p, sizeof(T) * count, cudaMemcpyHostToDevice, c->stream));
  return UFC_STATUS_OK;
}

template <class T>
int stage_out(Ctx* c, Staged<T>& s, T* p, int64_t count, int mem) {
  s.c = c;
  s.count = count;
  s.host = p;
  if (!p) return UFC_STATUS_OK;
  if (mem == UFC_MEM_DEVICE) {
    s.dev = p;
    return UFC_STATUS_OK;
  }
  if (mem != UFC_MEM_HOST) return fail(c, UFC_STATUS_INVALID, "mem must be UFC_MEM_HOST or UFC_MEM_DEVICE");
  UFC_CUDA(c, cudaMallocAsync((void**)&s.dev, sizeof(T) * std::max<int64_t>(count, 1), c->stream));
  s.owned = true;
  s.copy_back = true;
  return UFC_STATUS_OK;
}

template <class T>
int finish(Ctx* c, Staged<T>& s) {
  if (s.owned && s.copy_back && s.host)
    UFC_CUDA(c, cudaMemcpyAsync(s.host, s.dev, sizeof(T) * s.count, cudaMemcpyDeviceToHost, c->stream));
  return UFC_STATUS_OK;
}

int sync(Ctx* c) {
  UFC_CUDA(c, cudaStreamSynchronize(c->stream));
  return UFC_STATUS_OK;
}

void free_all(Ctx* c) {
  release_graphs(c);
  mg_free(c);
  dfree(&c->z64);
  dfree(&c->coords); dfree(&c->conn); dfree(&c->props); dfree(&c->col_elems);
  dfree(&c->brow); dfree(&c->bcol); dfree(&c->slice_ptr); dfree(&c->sell_col); dfree(&c->slot); dfree(&c->dpos);
  dfree(&c->val64); dfree(&c->val32); dfree(&c->dinv64); dfree(&c->dinv32);
  dfree(&c->uptr); dfree(&c->ucol); dfree(&c->lptr); dfree(&c->lpos); dfree(&c->lcol); dfree(&c->s_lcnt);
  dfree(&c->sval64); dfree(&c->sval32); dfree(&c->sym_ucode); dfree(&c->sym_lcode); dfree(&c->full_code);
  c->has_sym_pattern = c->has_sval64 = c->has_sval32 = false;
  dfree(&c->fixed); dfree(&c->fix_dofs); dfree(&c->fix_vals);
  dfree(&c->x64); dfree(&c->r64); dfree(&c->p64); dfree(&c->q64); dfree(&c->b64); dfree(&c->y64);
  dfree(&c->r32); dfree(&c->p32); dfree(&c->q32); dfree(&c->xb64); dfree(&c->hist);
  c->hist_cap = c->hist_len = 0;
  dfree(&c->nr_fint); dfree(&c->nr_R); dfree(&c->nr_du); dfree(&c->nr_dc);
  dfree(&c->u); dfree(&c->u_n);
  dfree(&c->sig_n); dfree(&c->epeq_n); dfree(&c->epl_n); dfree(&c->sig_t); dfree(&c->epeq_t); dfree(&c->epl_t);
  dfree(&c->Dt);
}

int alloc_state(Ctx* c) {
  const int64_t G = (int64_t)c->E * 8;
  UFC_TRY(dalloc(c, &c->u, c->n));
  UFC_TRY(dalloc(c, &c->u_n, c->n));
  UFC_CUDA(c, cudaMemsetAsync(c->u, 0, sizeof(double) * c->n, c->stream));
  UFC_CUDA(c, cudaMemsetAsync(c->u_n, 0, sizeof(double) * c->n, c->stream));
  if (c->mat_model == UFC_MAT_J2_ISO) {
    UFC_TRY(dalloc(c, &c->sig_n, G * 6)); UFC_TRY(dalloc(c, &c->epeq_n, G)); UFC_TRY(dalloc(c, &c->epl_n, G * 6));
    UFC_TRY(dalloc(c, &c->sig_t, G * 6)); UFC_TRY(dalloc(c, &c->epeq_t, G)); UFC_TRY(dalloc(c, &c->epl_t, G * 6));
    UFC_TRY(dalloc(c, &c->Dt, G * 36));
    UFC_CUDA(c, cudaMemsetAsync(c->sig_n, 0, sizeof(double) * G * 6, c->stream));
    UFC_CUDA(c, cudaMemsetAsync(c->epeq_n, 0, sizeof(double) * G, c->stream));
    UFC_CUDA(c, cudaMemsetAsync(c->epl_n, 0, sizeof(double) * G * 6, c->stream));
  }
  c->has_trial = false;
  return UFC_STATUS_OK;
}

__global__ void k_set_vals(int32_t nfix, const int32_t* __restrict__ dofs, const double* __restrict__ vals,
                           double* __restrict__ u) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < nfix) u[dofs[i]] = vals ? vals[i] : 0.0;
}

// dc[dof] = target - u[dof] on the Dirichlet DOFs (dc is zero elsewhere);
// flags *changed when any prescribed value moves.
__global__ void k_prescribed_delta(int32_t nfix, const int32_t* __restrict__ dofs, const double* __restrict__ vals,
                                   const double* __restrict__ u, double* __restrict__ dc, int32_t* __restrict__ changed) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nfix) return;
  const double d = vals[i] - u[dofs[i]];
  dc[dofs[i]] = d;
  if (d != 0.0) atomicOr(changed, 1);
}

// R -= y on the free DOFs (R is zero on the fixed ones).
__global__ void k_sub_free(int64_t n, const uint8_t* __restrict__ fixed, const double* __restrict__ y,
                           double* __restrict__ R) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    if (!fixed[i]) R[i] -= y[i];
}

__global__ void k_axpy(int64_t n, double a, const double* __restrict__ x, double* __restrict__ y) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    y[i] += a * x[i];
}

// out = a + s (b - a), a or b NULL meaning zero.
__global__ void k_lerp(int64_t n, const double* __restrict__ a, const double* __restrict__ b, double s,
                       double* __restrict__ out) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const double ai = a ? a[i] : 0.0, bi = b ? b[i] : 0.0;
    out[i] = ai + s * (bi - ai);
  }
}

__global__ void k_gather_dofs(int32_t nfix, const int32_t* __restrict__ dofs, const double* __restrict__ u,
                              double* __restrict__ out) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < nfix) out[i] = u[dofs[i]];
}

}  // namespace
}  // namespace ufc

using namespace ufc;


#define CTX_CHECK(c)                 \
  do {                               \
    if (!(c)) return UFC_STATUS_INVALID; \
  } while (0)

extern "C" {

int ufc_ctx_create(int32_t device, ufc_ctx** out) {
  if (!out) return UFC_STATUS_INVALID;
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return UFC_STATUS_UNSUPPORTED;
  if (device < 0 || device >= ndev) return UFC_STATUS_INVALID;
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) return UFC_STATUS_ERROR;
  if (prop.major != 10) return UFC_STATUS_UNSUPPORTED;  // built for sm_100a only
  ufc_ctx* c = new ufc_ctx();
  c->device = device;
  cudaSetDevice(device);
  if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreateWithFlags(&c->ev_join, cudaEventDisableTiming) != cudaSuccess ||
      cudaMalloc((void**)&c->scal, sizeof(CgScalars)) != cudaSuccess ||
      cudaMalloc((void**)&c->dev_err, sizeof(int32_t)) != cudaSuccess ||
      cudaMallocHost((void**)&c->h_scal, 3 * sizeof(CgScalars)) != cudaSuccess ||
      cudaMallocHost((void**)&c->h_err, sizeof(int32_t)) != cudaSuccess) {
    delete c;
    return UFC_STATUS_MEM_ERROR;
  }
  cudaMemset(c->scal, 0, sizeof(CgScalars));
  cudaMemset(c->dev_err, 0, sizeof(int32_t));
  // per-block partial sums of the grid reductions: enough for the largest grid
  // any kernel of this context uses (SpMV: one thread per block row)
  c->partials_cap = 4 * 65536;
  if (cudaMalloc((void**)&c->partials, sizeof(double) * c->partials_cap) != cudaSuccess) {
    delete c;
    return UFC_STATUS_MEM_ERROR;
  }
  *out = c;
  return UFC_STATUS_OK;
}

int ufc_ctx_destroy(ufc_ctx* c) {
  CTX_CHECK(c);
  cudaSetDevice(c->device);
  cudaStreamSynchronize(c->stream);
  free_all(c);
  if (c->scal) cudaFree(c->scal);
  if (c->partials) cudaFree(c->partials);
  if (c->dev_err) cudaFree(c->dev_err);
  if (c->h_scal) cudaFreeHost(c->h_scal);
  if (c->h_err) cudaFreeHost(c->h_err);
  if (c->ev_join) cudaEventDestroy(c->ev_join);
  if (c->stream) cudaStreamDestroy(c->stream);
  delete c;
  return UFC_STATUS_OK;
}

int ufc_ctx_set_stream(ufc_ctx* c, void* stream) {
  CTX_CHECK(c);
  c->ext = (cudaStream_t)stream;
  c->has_ext = true;  // NULL selects the legacy default stream
  return UFC_STATUS_OK;
}

int ufc_ctx_set_instrument(ufc_ctx* c, int32_t on) {
  CTX_CHECK(c);
  c->instrument = on != 0;
  return UFC_STATUS_OK;
}

int ufc_last_error(const ufc_ctx* c, char* buf, int32_t buflen) {
  if (!c || !buf || buflen <= 0) return UFC_STATUS_INVALID;
  const std::string& m = c->err;
  const size_t k = std::min<size_t>(m.size(), (size_t)buflen - 1);
  std::memcpy(buf, m.data(), k);
  buf[k] = 0;
  return UFC_STATUS_OK;
}

int ufc_mesh_set(ufc_ctx* c, const ufc_mesh_desc* m) {
  CTX_CHECK(c);
  if (!m || !m->coords || !m->conn || m->n_nodes <= 0 || m->n_elems <= 0)
    return fail(c, UFC_STATUS_INVALID, "ufc_mesh_set: empty mesh or NULL arrays");
  if (m->index_base != 0 && m->index_base != 1) return fail(c, UFC_STATUS_INVALID, "ufc_mesh_set: index_base");
  if ((int64_t)m->n_nodes * 3 >= ((int64_t)1 << 31))
    return fail(c, UFC_STATUS_UNSUPPORTED, "ufc_mesh_set: more than 2^31 DOF");
  Scope sc(c);
  free_all(c);
  c->has_pattern = c->has_material = c->has_val64 = c->has_val32 = false;
  c->N = m->n_nodes;
  c->E = m->n_elems;
  c->n = 3 * (int64_t)c->N;
  c->nfix = 0;
  // connectivity on the host (colouring) and validated there
  c->h_conn.resize((size_t)c->E * 8);
  if (m->mem == UFC_MEM_DEVICE) {
    UFC_CUDA(c, cudaMemcpyAsync(c->h_conn.data(), m->conn, sizeof(int32_t) * c->h_conn.size(),
                                cudaMemcpyDeviceToHost, c->stream));
    UFC_TRY(sync(c));
  } else {
    std::memcpy(c->h_conn.data(), m->conn, sizeof(int32_t) * c->h_conn.size());
  }
  for (auto& v : c->h_conn) {
    v -= m->index_base;
    if (v < 0 || v >= c->N) return fail(c, UFC_STATUS_INVALID, "ufc_mesh_set: connectivity out of range");
  }
  for (int64_t e = 0; e < c->E; ++e)
    for (int a = 0; a < 8; ++a)
      for (int b = a + 1; b < 8; ++b)
        if (c->h_conn[e * 8 + a] == c->h_conn[e * 8 + b])
          return fail(c, UFC_STATUS_INVALID, "ufc_mesh_set: element " + std::to_string(e) + " repeats a node");
  UFC_TRY(dalloc(c, &c->conn, (int64_t)c->E * 8));
  UFC_CUDA(c, cudaMemcpyAsync(c->conn, c->h_conn.data(), sizeof(int32_t) * c->h_conn.size(), cudaMemcpyHostToDevice,
                              c->stream));
  UFC_TRY(dalloc(c, &c->coords, c->n));
  UFC_CUDA(c, cudaMemcpyAsync(c->coords, m->coords, sizeof(double) * c->n,
                              m->mem == UFC_MEM_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, c->stream));
  UFC_TRY(dalloc(c, &c->fixed, c->n));
  UFC_CUDA(c, cudaMemsetAsync(c->fixed, 0, c->n, c->stream));
  return sync(c);
}

int ufc_material_set(ufc_ctx* c, const ufc_material_desc* m) {
  CTX_CHECK(c);
  if (!m || !m->props) return fail(c, UFC_STATUS_INVALID, "ufc_material_set: NULL props");
  if (c->E <= 0) return fail(c, UFC_STATUS_INVALID, "ufc_material_set: mesh not set");
  if (m->mat_model_id != UFC_MAT_ELASTIC_ISO && m->mat_model_id != UFC_MAT_J2_ISO)
    return fail(c, UFC_STATUS_UNSUPPORTED, "ufc_material_set: mat_model_id must be 101 or 201");
  const int need = m->mat_model_id == UFC_MAT_J2_ISO ? 4 : 2;
  if (m->nprops < need) return fail(c, UFC_STATUS_INVALID, "ufc_material_set: too few props");
  Scope sc(c);
  const int64_t cnt = (m->per_element ? (int64_t)c->E : 1) * m->nprops;
  std::vector<double> h(cnt);
  if (m->mem == UFC_MEM_DEVICE) {
    UFC_CUDA(c, cudaMemcpyAsync(h.data(), m->props, sizeof(double) * cnt, cudaMemcpyDeviceToHost, c->stream));
    UFC_TRY(sync(c));
  } else {
    std::memcpy(h.data(), m->props, sizeof(double) * cnt);
  }
  // expand to per-element rows and validate (E > 0, -1 < nu < 0.5)
  std::vector<double> full((size_t)c->E * m->nprops);
  for (int64_t e = 0; e < c->E; ++e) {
    const double* src = h.data() + (m->per_element ? e * m->nprops : 0);
    if (!(src[0] > 0.0) || !(src[1] > -1.0 && src[1] < 0.5))
      return fail(c, UFC_STATUS_INVALID, "ufc_material_set: element " + std::to_string(e) + " has E <= 0 or nu outside (-1, 0.5)");
    if (need == 4 && (!(src[2] > 0.0) || !(src[3] >= 0.0)))
      return fail(c, UFC_STATUS_INVALID, "ufc_material_set: sigma_y0 must be > 0 and H >= 0");
    std::memcpy(full.data() + e * m->nprops, src, sizeof(double) * m->nprops);
  }
  c->mat_model = m->mat_model_id;
  c->nprops = m->nprops;
  UFC_TRY(dalloc(c, &c->props, (int64_t)full.size()));
  UFC_CUDA(c, cudaMemcpyAsync(c->props, full.data(), sizeof(double) * full.size(), cudaMemcpyHostToDevice, c->stream));
  UFC_TRY(alloc_state(c));
  c->has_material = true;
  c->has_val64 = c->has_val32 = c->has_sval64 = c->has_sval32 = false;  // values depend on the material
  return sync(c);
}

int ufc_bc_set(ufc_ctx* c, const ufc_bc_desc* bc) {
  CTX_CHECK(c);
  if (!bc || bc->n_fixed < 0 || (bc->n_fixed > 0 && !bc->dofs)) return fail(c, UFC_STATUS_INVALID, "ufc_bc_set");
  if (c->N <= 0) return fail(c, UFC_STATUS_INVALID, "ufc_bc_set: mesh not set");
  Scope sc(c);
  std::vector<int32_t> d(bc->n_fixed);
  std::vector<double> v(bc->n_fixed, 0.0);
  if (bc->n_fixed > 0) {
    if (bc->mem == UFC_MEM_DEVICE) {
      UFC_CUDA(c, cudaMemcpyAsync(d.data(), bc->dofs, sizeof(int32_t) * d.size(), cudaMemcpyDeviceToHost, c->stream));
      if (bc->values)
        UFC_CUDA(c, cudaMemcpyAsync(v.data(), bc->values, sizeof(double) * v.size(), cudaMemcpyDeviceToHost, c->stream));
      UFC_TRY(sync(c));
    } else {
      std::memcpy(d.data(), bc->dofs, sizeof(int32_t) * d.size());
      if (bc->values) std::memcpy(v.data(), bc->values, sizeof(double) * v.size());
    }
  }
  std::vector<uint8_t> mask(c->n, 0);
  for (int32_t k = 0; k < bc->n_fixed; ++k) {
    if (d[k] < 0 || d[k] >= c->n) return fail(c, UFC_STATUS_INVALID, "ufc_bc_set: DOF out of range");
    if (mask[d[k]]) return fail(c, UFC_STATUS_INVALID, "ufc_bc_set: DOF listed twice");
    mask[d[k]] = 1;
  }
  c->nfix = bc->n_fixed;
  UFC_TRY(dalloc(c, &c->fix_dofs, std::max(1, c->nfix)));
  UFC_TRY(dalloc(c, &c->fix_vals, std::max(1, c->nfix)));
  if (c->nfix > 0) {
    UFC_CUDA(c, cudaMemcpyAsync(c->fix_dofs, d.data(), sizeof(int32_t) * c->nfix, cudaMemcpyHostToDevice, c->stream));
    UFC_CUDA(c, cudaMemcpyAsync(c->fix_vals, v.data(), sizeof(double) * c->nfix, cudaMemcpyHostToDevice, c->stream));
  }
  UFC_CUDA(c, cudaMemcpyAsync(c->fixed, mask.data(), c->n, cudaMemcpyHostToDevice, c->stream));
  c->has_val64 = c->has_val32 = c->has_sval64 = c->has_sval32 = false;  // elimination is part of the values
  return sync(c);
}

int ufc_pattern_build(ufc_ctx* c, ufc_pattern_info* info) {
  CTX_CHECK(c);
  Scope sc(c);
  UFC_TRY(build_pattern(c));
  if (info) {
    info->n_dof = c->n;
    info->nnzb = c->nnzb;
    info->nnz = 9 * c->nnzb;
    info->sell_blocks = c->sell_blocks;
    info->n_colors = c->ncol;
    info->max_row_blocks = c->max_row_blocks;
  }
  return sync(c);
}

int ufc_csr_export(ufc_ctx* c, const ufc_csr_export_arg* a) {
  CTX_CHECK(c);
  if (!a) return fail(c, UFC_STATUS_INVALID, "ufc_csr_export: NULL arg");
  Scope sc(c);
  UFC_TRY(export_csr(c, a));
  return sync(c);
}

int ufc_pattern_colors(ufc_ctx* c, int32_t* color_of, int32_t index_base, int32_t mem) {
  CTX_CHECK(c);
  if (!c->has_pattern) return fail(c, UFC_STATUS_INVALID, "ufc_pattern_colors: pattern not built");
  if (!color_of || (index_base != 0 && index_base != 1))
    return fail(c, UFC_STATUS_INVALID, "ufc_pattern_colors: NULL color_of or index_base not 0 or 1");
  Scope sc(c);
  std::vector<int32_t> h(c->h_color);
  for (int32_t& v : h) v += index_base;
  if (mem == UFC_MEM_DEVICE) {
    UFC_CUDA(c, cudaMemcpyAsync(color_of, h.data(), sizeof(int32_t) * h.size(), cudaMemcpyHostToDevice, c->stream));
    UFC_CUDA(c, cudaStreamSynchronize(c->stream));
  } else {
    std::copy(h.begin(), h.end(), color_of);
  }
  return sync(c);
}

int ufc_elem_compute_ke(ufc_ctx* c, ufc_elem_ke_arg* a) {
  CTX_CHECK(c);
  if (!a || (a->build & (UFC_BUILD_FP64 | UFC_BUILD_FP32 | UFC_BUILD_FP32_ROUNDED | UFC_BUILD_FP32_DIFF |
                         UFC_BUILD_SYMMETRIC)) == 0)
    return fail(c, UFC_STATUS_INVALID, "ufc_elem_compute_ke: build must select FP64 and/or FP32");
  Scope sc(c);
  a->status = assemble(c, a->build, &a->elapsed_ms);
  return a->status;
}

int ufc_elem_compute_fint(ufc_ctx* c, ufc_elem_fe_arg* a) {
  CTX_CHECK(c);
  if (!a || !a->u) return fail(c, UFC_STATUS_INVALID, "ufc_elem_compute_fint: NULL u");
  if (!c->has_pattern) return fail(c, UFC_STATUS_INVALID, "ufc_elem_compute_fint: pattern not built");
  Scope sc(c);
  Staged<double> u, fe, fi, r;
  UFC_TRY(stage_in(c, u, a->u, c->n, a->mem));
  UFC_TRY(stage_in(c, fe, a->f_ext, c->n, a->mem));
  UFC_TRY(stage_out(c, fi, a->fint, c->n, a->mem));
  UFC_TRY(stage_out(c, r, a->r, c->n, a->mem));
  if (!c->nr_fint) UFC_TRY(dalloc(c, &c->nr_fint, c->n));
  if (!c->nr_R) UFC_TRY(dalloc(c, &c->nr_R, c->n));
  UFC_TRY(compute_fint(c, u.dev, c->nr_fint, a->update_state != 0));
  UFC_TRY(nr_norms(c, fe.dev, c->nr_fint, c->nr_R));
  if (fi.dev) UFC_CUDA(c, cudaMemcpyAsync(fi.dev, c->nr_fint, sizeof(double) * c->n, cudaMemcpyDeviceToDevice, c->stream));
  if (r.dev) UFC_CUDA(c, cudaMemcpyAsync(r.dev, c->nr_R, sizeof(double) * c->n, cudaMemcpyDeviceToDevice, c->stream));
  UFC_TRY(finish(c, fi));
  UFC_TRY(finish(c, r));
  UFC_CUDA(c, cudaMemcpyAsync(c->h_scal, c->scal, sizeof(CgScalars), cudaMemcpyDeviceToHost, c->stream));
  UFC_TRY(sync(c));
  a->rnorm = std::sqrt(c->h_scal->nr_rr);
  a->fint_norm = std::sqrt(c->h_scal->nr_ff);
  a->status = check_dev_err(c, "ufc_elem_compute_fint");
  return a->status;
}

int ufc_mat_update_batch(ufc_ctx* c, ufc_mat_update_arg* a) {
  CTX_CHECK(c);
  if (!a || a->n_points < 0 || !a->props || !a->stress_n || !a->dstrain || !a->stress)
    return fail(c, UFC_STATUS_INVALID, "ufc_mat_update_batch: NULL arrays");
  if (a->mat_model_id != UFC_MAT_ELASTIC_ISO && a->mat_model_id != UFC_MAT_J2_ISO)
    return fail(c, UFC_STATUS_UNSUPPORTED, "ufc_mat_update_batch: mat_model_id must be 101 or 201");
  if (a->nprops < (a->mat_model_id == UFC_MAT_J2_ISO ? 4 : 2))
    return fail(c, UFC_STATUS_INVALID, "ufc_mat_update_batch: too few props");
  Scope sc(c);
  const int64_t n = a->n_points;
  Staged<double> pr, sn, de, vn, s, v, dd;
  Staged<int32_t> y;
  UFC_TRY(stage_in(c, pr, a->props, (a->props_per_point ? n : 1) * a->nprops, a->mem));
  UFC_TRY(stage_in(c, sn, a->stress_n, n * 6, a->mem));
  UFC_TRY(stage_in(c, de, a->dstrain, n * 6, a->mem));
  UFC_TRY(stage_in(c, vn, a->sdv_n, n * 7, a->mem));
  UFC_TRY(stage_out(c, s, a->stress, n * 6, a->mem));
  UFC_TRY(stage_out(c, v, a->sdv, n * 7, a->mem));
  UFC_TRY(stage_out(c, dd, a->ddsdde, n * 36, a->mem));
  UFC_TRY(stage_out(c, y, a->yielded, n, a->mem));
  UFC_TRY(mat_update_batch(c, a, pr.dev, sn.dev, de.dev, vn.dev, s.dev, v.dev, dd.dev, y.dev));
  UFC_TRY(finish(c, s));
  UFC_TRY(finish(c, v));
  UFC_TRY(finish(c, dd));
  UFC_TRY(finish(c, y));
  a->status = sync(c);
  return a->status;
}

int ufc_stress_eval(ufc_ctx* c, const double* u, double* sig, double* vm, int32_t mem) {
  CTX_CHECK(c);
  if (!c->has_material) return fail(c, UFC_STATUS_INVALID, "ufc_stress_eval: material not set");
  if (c->mat_model != UFC_MAT_J2_ISO && !u) return fail(c, UFC_STATUS_INVALID, "ufc_stress_eval: NULL u");
  Scope sc(c);
  const int64_t G = (int64_t)c->E * 8;
  Staged<double> su, ss, sv;
  UFC_TRY(stage_in(c, su, u, c->n, mem));
  UFC_TRY(stage_out(c, ss, sig, G * 6, mem));
  UFC_TRY(stage_out(c, sv, vm, G, mem));
  UFC_TRY(stress_eval(c, su.dev, ss.dev, sv.dev));
  UFC_TRY(finish(c, ss));
  UFC_TRY(finish(c, sv));
  return sync(c);
}

int ufc_mg_setup(ufc_ctx* c, ufc_mg_arg* a) {
  CTX_CHECK(c);
  if (!a) return fail(c, UFC_STATUS_INVALID, "ufc_mg_setup: NULL arg");
  Scope sc(c);
  a->levels = 0;
  a->coarse_dof = 0;
  a->setup_ms = 0.0;
  UFC_TRY(mg_setup(c, a));
  return sync(c);
}

int ufc_mg_apply(ufc_ctx* c, const double* r, double* z, int32_t mem) {
  CTX_CHECK(c);
  if (!r || !z) return fail(c, UFC_STATUS_INVALID, "ufc_mg_apply: NULL vector");
  Scope sc(c);
  Staged<double> sr, sz;
  UFC_TRY(stage_in(c, sr, r, c->n, mem));
  UFC_TRY(stage_out(c, sz, z, c->n, mem));
  UFC_TRY(mg_apply(c, sr.dev, sz.dev));
  UFC_TRY(finish(c, sz));
  return sync(c);
}

int ufc_mg_level_info(ufc_ctx* c, int32_t level, int64_t* n_dof, int64_t* nnz) {
  CTX_CHECK(c);
  Ctx* lc = nullptr;
  UFC_TRY(mg_level_ctx(c, level, &lc));
  if (n_dof) *n_dof = lc->n;
  if (nnz) *nnz = 9 * lc->nnzb;
  return UFC_STATUS_OK;
}

int ufc_mg_export(ufc_ctx* c, int32_t level, const ufc_csr_export_arg* a) {
  CTX_CHECK(c);
  if (!a) return fail(c, UFC_STATUS_INVALID, "ufc_mg_export: NULL arg");
  Ctx* lc = nullptr;
  UFC_TRY(mg_level_ctx(c, level, &lc));
  Scope sc(c);
  UFC_CUDA(c, cudaStreamSynchronize(c->stream));
  const int s = export_csr(lc, a);
  if (s != UFC_STATUS_OK && lc != c) return fail(c, s, lc->err);
  return s;
}

int ufc_load_faces(ufc_ctx* c, const ufc_face_load_arg* a) {
  CTX_CHECK(c);
  if (!a || !a->f || a->n_faces < 0 || (a->n_faces > 0 && (!a->elem || !a->face)))
    return fail(c, UFC_STATUS_INVALID, "ufc_load_faces: NULL arrays");
  if (!c->has_pattern) return fail(c, UFC_STATUS_INVALID, "ufc_load_faces: pattern not built");
  if (a->index_base != 0 && a->index_base != 1) return fail(c, UFC_STATUS_INVALID, "ufc_load_faces: index_base");
  Scope sc(c);
  const int32_t nf = a->n_faces;
  std::vector<int32_t> he(nf), hf(nf);
  if (nf > 0) {
    const cudaMemcpyKind k = a->mem == UFC_MEM_DEVICE ? cudaMemcpyDeviceToHost : cudaMemcpyHostToHost;
    UFC_CUDA(c, cudaMemcpyAsync(he.data(), a->elem, sizeof(int32_t) * nf, k, c->stream));
    UFC_CUDA(c, cudaMemcpyAsync(hf.data(), a->face, sizeof(int32_t) * nf, k, c->stream));
    UFC_TRY(sync(c));
  }
  for (int32_t i = 0; i < nf; ++i) {
    he[i] -= a->index_base;
    if (he[i] < 0 || he[i] >= c->E) return fail(c, UFC_STATUS_INVALID, "ufc_load_faces: element id out of range");
    if (hf[i] < 1 || hf[i] > 6) return fail(c, UFC_STATUS_INVALID, "ufc_load_faces: face id must be 1..6");
  }
  Staged<double> st, sp, sf;
  UFC_TRY(stage_in(c, st, a->traction, (int64_t)nf * 3, a->mem));
  UFC_TRY(stage_in(c, sp, a->pressure, nf, a->mem));
  UFC_TRY(stage_out(c, sf, a->f, c->n, a->mem));
  UFC_TRY(face_loads(c, nf, he.data(), hf.data(), st.dev, sp.dev, sf.dev));
  UFC_TRY(finish(c, sf));
  return sync(c);
}

int ufc_stress_nodal(ufc_ctx* c, const double* u, double* sig, double* vm, int32_t mem) {
  CTX_CHECK(c);
  if (!c->has_material || !c->has_pattern) return fail(c, UFC_STATUS_INVALID, "ufc_stress_nodal: model not set up");
  Scope sc(c);
  Staged<double> su, ss, sv;
  UFC_TRY(stage_in(c, su, u, c->n, mem));
  UFC_TRY(stage_out(c, ss, sig, (int64_t)c->N * 6, mem));
  UFC_TRY(stage_out(c, sv, vm, c->N, mem));
  UFC_TRY(stress_nodal(c, su.dev ? su.dev : c->u, ss.dev, sv.dev));
  UFC_TRY(finish(c, ss));
  UFC_TRY(finish(c, sv));
  return sync(c);
}

int ufc_reactions(ufc_ctx* c, const double* u, const double* f_ext, double* rf, int32_t mem) {
  CTX_CHECK(c);
  if (!rf) return fail(c, UFC_STATUS_INVALID, "ufc_reactions: NULL rf");
  if (!c->has_material || !c->has_pattern) return fail(c, UFC_STATUS_INVALID, "ufc_reactions: model not set up");
  Scope sc(c);
  Staged<double> su, se, sr;
  UFC_TRY(stage_in(c, su, u, c->n, mem));
  UFC_TRY(stage_in(c, se, f_ext, c->n, mem));
  UFC_TRY(stage_out(c, sr, rf, c->nfix, mem));
  UFC_TRY(reactions(c, su.dev ? su.dev : c->u, se.dev, sr.dev));
  UFC_TRY(finish(c, sr));
  UFC_TRY(sync(c));
  return check_dev_err(c, "ufc_reactions");
}

int ufc_spmv(ufc_ctx* c, int32_t precision, const void* x, void* y, int32_t mem) {
  CTX_CHECK(c);
  if (!x || !y) return fail(c, UFC_STATUS_INVALID, "ufc_spmv: NULL vector");
  Scope sc(c);
  if (mem == UFC_MEM_DEVICE) return spmv(c, precision, x, y);
  if (precision == UFC_PRECISION_FP64) {
    Staged<double> sx, sy;
    UFC_TRY(stage_in(c, sx, (const double*)x, c->n, mem));
    UFC_TRY(stage_out(c, sy, (double*)y, c->n, mem));
    UFC_TRY(spmv(c, precision, sx.dev, sy.dev));
    UFC_TRY(finish(c, sy));
  } else {
    Staged<float> sx, sy;
    UFC_TRY(stage_in(c, sx, (const float*)x, c->n, mem));
    UFC_TRY(stage_out(c, sy, (float*)y, c->n, mem));
    UFC_TRY(spmv(c, precision, sx.dev, sy.dev));
    UFC_TRY(finish(c, sy));
  }
  return sync(c);
}

int ufc_pcg_solve(ufc_ctx* c, const double* b, double* x, int32_t mem, const ufc_solver_algo* algo,
                  ufc_solver_state* st) {
  CTX_CHECK(c);
  if (!b || !x || !algo || !st) return fail(c, UFC_STATUS_INVALID, "ufc_pcg_solve: NULL argument");
  if (!(algo->tolerance >= 0.0) || algo->max_iter <= 0)
    return fail(c, UFC_STATUS_INVALID, "ufc_pcg_solve: tolerance must be >= 0 and max_iter > 0");
  Scope sc(c);
  std::memset(st, 0, sizeof(*st));
  Staged<double> sb, sx;
  UFC_TRY(stage_in(c, sb, b, c->n, mem));
  if (algo->use_x0)
    UFC_TRY(stage_in(c, sx, (const double*)x, c->n, mem, true));
  else
    UFC_TRY(stage_out(c, sx, x, c->n, mem));
  const int s = pcg_solve(c, sb.dev, sx.dev, algo, st);
  if (s != UFC_STATUS_OK && s != UFC_STATUS_NOT_CONVERGED) return s;
  UFC_TRY(finish(c, sx));
  UFC_TRY(sync(c));
  return s;
}

int ufc_pcg_solve_block(ufc_ctx* c, int32_t nrhs, const double* B, double* X, int32_t mem,
                        const ufc_solver_algo* algo, ufc_solver_state* states) {
  CTX_CHECK(c);
  if (!B || !X || !algo || !states || nrhs <= 0)
    return fail(c, UFC_STATUS_INVALID, "ufc_pcg_solve_block: NULL argument or nrhs <= 0");
  Scope sc(c);
  Staged<double> sb, sx;
  const int64_t cnt = (int64_t)nrhs * c->n;
  UFC_TRY(stage_in(c, sb, B, cnt, mem));
  if (algo->use_x0)
    UFC_TRY(stage_in(c, sx, (const double*)X, cnt, mem, true));
  else
    UFC_TRY(stage_out(c, sx, X, cnt, mem));
  const int s = pcg_solve_block(c, nrhs, sb.dev, sx.dev, algo, states);
  if (s != UFC_STATUS_OK && s != UFC_STATUS_NOT_CONVERGED) return s;
  UFC_TRY(finish(c, sx));
  UFC_TRY(sync(c));
  return s;
}

int ufc_last_timing(const ufc_ctx* c, ufc_timing_info* info) {
  if (!c || !info) return UFC_STATUS_INVALID;
  *info = c->timing;
  return UFC_STATUS_OK;
}

int ufc_last_residual_history(ufc_ctx* c, double* out, int32_t max_len, int32_t* len) {
  CTX_CHECK(c);
  if (!out || !len || max_len < 0) return fail(c, UFC_STATUS_INVALID, "ufc_last_residual_history: NULL argument");
  Scope sc(c);
  const int32_t k = std::min(max_len, c->hist_len);
  *len = k;
  if (k == 0) return UFC_STATUS_OK;
  UFC_CUDA(c, cudaMemcpyAsync(out, c->hist, sizeof(double) * k, cudaMemcpyDeviceToHost, c->stream));
  UFC_TRY(sync(c));
  for (int32_t i = 0; i < k; ++i) out[i] = std::sqrt(out[i]);
  return UFC_STATUS_OK;
}

int ufc_nr_increment(ufc_ctx* c, ufc_nr_arg* a) {
  CTX_CHECK(c);
  if (!a) return fail(c, UFC_STATUS_INVALID, "ufc_nr_increment: NULL arg");
  if (!c->has_pattern || !c->has_material) return fail(c, UFC_STATUS_INVALID, "ufc_nr_increment: model not set up");
  if (a->max_iterations <= 0 || a->max_iterations > 32)
    return fail(c, UFC_STATUS_INVALID, "ufc_nr_increment: max_iterations must be 1..32");
  Scope sc(c);
  a->iterations = 0;
  a->converged = 0;
  a->lin_iters_total = 0;
  a->residual_norm = 0.0;
  Staged<double> up, fe;
  UFC_TRY(stage_in(c, up, a->u_prescribed, c->nfix, a->mem));
  UFC_TRY(stage_in(c, fe, a->f_ext, c->n, a->mem));
  if (!c->nr_fint) UFC_TRY(dalloc(c, &c->nr_fint, c->n));
  if (!c->nr_R) UFC_TRY(dalloc(c, &c->nr_R, c->n));
  if (!c->nr_du) UFC_TRY(dalloc(c, &c->nr_du, c->n));
  if (!c->nr_dc) UFC_TRY(dalloc(c, &c->nr_dc, c->n));
  // prescribed values at the end of the increment, and their change du_c
  bool lift = false;
  if (c->nfix > 0 && up.dev) {
    UFC_CUDA(c, cudaMemcpyAsync(c->fix_vals, up.dev, sizeof(double) * c->nfix, cudaMemcpyDeviceToDevice, c->stream));
    UFC_CUDA(c, cudaMemsetAsync(c->nr_dc, 0, sizeof(double) * c->n, c->stream));
    k_prescribed_delta<<<grid_for(c->nfix, 256), 256, 0, c->stream>>>(c->nfix, c->fix_dofs, c->fix_vals, c->u,
                                                                      c->nr_dc, c->dev_err);
    UFC_CUDA(c, cudaGetLastError());
    UFC_CUDA(c, cudaMemcpyAsync(c->h_err, c->dev_err, sizeof(int32_t), cudaMemcpyDeviceToHost, c->stream));
    UFC_TRY(sync(c));
    lift = *c->h_err != 0;  // some prescribed value changed
    UFC_CUDA(c, cudaMemsetAsync(c->dev_err, 0, sizeof(int32_t), c->stream));
  }
  ufc_solver_algo lin = a->lin;
  lin.use_x0 = 0;
  // FP64 CG on the FP64 tangent, or (UFC_PRECISION_FP32_REFINE) FP32 CG on the
  // tangent rounded from its FP64 assembly, whose FP64 values give the
  // refinement residual
  if (lin.precision_mode != UFC_PRECISION_FP32_REFINE) lin.precision_mode = UFC_PRECISION_FP64;
  const int build =
      lin.precision_mode == UFC_PRECISION_FP64 ? UFC_BUILD_FP64 : (UFC_BUILD_FP64 | UFC_BUILD_FP32_ROUNDED);
  const int vg = std::min(grid_for(c->n, 256), 148 * 8);
  for (int it = 0; it < a->max_iterations; ++it) {
    UFC_TRY(compute_fint(c, c->u, c->nr_fint, true));
    UFC_TRY(nr_norms(c, fe.dev, c->nr_fint, c->nr_R));
    UFC_CUDA(c, cudaMemcpyAsync(c->h_scal, c->scal, sizeof(CgScalars), cudaMemcpyDeviceToHost, c->stream));
    UFC_TRY(sync(c));
    UFC_TRY(check_dev_err(c, "ufc_nr_increment (internal force)"));
    const double rn = std::sqrt(c->h_scal->nr_rr);
    const double ref = std::max({std::sqrt(c->h_scal->nr_ee), std::sqrt(c->h_scal->nr_ff), 1e-30});
    a->res_hist[it] = rn / ref;
    a->residual_norm = rn / ref;
    if (!std::isfinite(rn)) {  // a diverged iterate: a non-convergence the step driver cuts back on
      a->iterations = it;
      a->status = UFC_STATUS_NOT_CONVERGED;
      return fail(c, UFC_STATUS_NOT_CONVERGED, "ufc_nr_increment: non-finite residual");
    }
    if (!lift && rn <= a->tolerance_force * ref) {
      a->converged = 1;
      a->iterations = it;
      break;
    }
    ufc_elem_ke_arg ka{};
    UFC_TRY(assemble(c, build, &ka.elapsed_ms));
    if (lift) {
      // predictor: K_ff du_f = R_f - K_fc du_c with the tangent of the start of the
      // increment, then u_c takes its prescribed values
      UFC_TRY(apply_tangent(c, c->nr_dc, c->nr_du));
      k_sub_free<<<vg, 256, 0, c->stream>>>(c->n, c->fixed, c->nr_du, c->nr_R);
      UFC_CUDA(c, cudaGetLastError());
    }
    ufc_solver_state ls{};
    const int s = pcg_solve(c, c->nr_R, c->nr_du, &lin, &ls);
    a->lin_iters_total += ls.niter;
    if (s != UFC_STATUS_OK) return s;
    k_axpy<<<vg, 256, 0, c->stream>>>(c->n, 1.0, c->nr_du, c->u);
    UFC_CUDA(c, cudaGetLastError());
    if (lift) {
      k_set_vals<<<grid_for(c->nfix, 256), 256, 0, c->stream>>>(c->nfix, c->fix_dofs, c->fix_vals, c->u);
      UFC_CUDA(c, cudaGetLastError());
      lift = false;
    }
    a->iterations = it + 1;
  }
  a->status = a->converged ? UFC_STATUS_OK : UFC_STATUS_NOT_CONVERGED;
  if (!a->converged) fail(c, UFC_STATUS_NOT_CONVERGED, "ufc_nr_increment: Newton-Raphson did not converge");
  return a->status;
}

int ufc_nr_step(ufc_ctx* c, ufc_step_arg* a) {
  CTX_CHECK(c);
  if (!a) return fail(c, UFC_STATUS_INVALID, "ufc_nr_step: NULL arg");
  if (!c->has_pattern || !c->has_material) return fail(c, UFC_STATUS_INVALID, "ufc_nr_step: model not set up");
  if (!(a->time_period > 0.0) || !(a->dt_initial > 0.0) || !(a->dt_min > 0.0) || a->dt_max < a->dt_min ||
      a->max_increments <= 0 || a->max_cutbacks < 0 || !(a->cutback_factor > 0.0 && a->cutback_factor < 1.0) ||
      !(a->growth_factor >= 1.0) || a->max_iterations <= 0 || a->max_iterations > 32 || a->hist_cap < 0)
    return fail(c, UFC_STATUS_INVALID, "ufc_nr_step: invalid increment controls");
  Scope sc(c);
  a->attempts = a->increments = a->cutbacks = a->nr_iterations = 0;
  a->lin_iters_total = 0;
  a->final_time = 0.0;
  a->completed = 0;
  Staged<double> ue, fs, fe;
  UFC_TRY(stage_in(c, ue, a->u_prescribed_end, c->nfix, a->mem));
  UFC_TRY(stage_in(c, fs, a->f_ext_start, c->n, a->mem));
  UFC_TRY(stage_in(c, fe, a->f_ext_end, c->n, a->mem));
  // prescribed values at the start of the step: those of the committed displacement
  double *u0 = nullptr, *ut = nullptr, *ft = nullptr;
  auto cleanup = [&]() {
    if (u0) cudaFreeAsync(u0, c->stream);
    if (ut) cudaFreeAsync(ut, c->stream);
    if (ft) cudaFreeAsync(ft, c->stream);
  };
  const int64_t nf = std::max<int32_t>(c->nfix, 1);
  if (cudaMallocAsync((void**)&u0, sizeof(double) * nf, c->stream) != cudaSuccess ||
      cudaMallocAsync((void**)&ut, sizeof(double) * nf, c->stream) != cudaSuccess ||
      cudaMallocAsync((void**)&ft, sizeof(double) * c->n, c->stream) != cudaSuccess) {
    cleanup();
    return fail(c, UFC_STATUS_MEM_ERROR, "ufc_nr_step: cudaMallocAsync failed");
  }
  if (c->nfix > 0)
    k_gather_dofs<<<grid_for(c->nfix, 256), 256, 0, c->stream>>>(c->nfix, c->fix_dofs, c->u_n, u0);
  const double T = a->time_period;
  const double* uend = ue.dev ? ue.dev : u0;
  const int vg = std::min(grid_for(c->n, 256), 148 * 8);
  double t = 0.0, dt = std::min(a->dt_initial, a->dt_max);
  int cut_run = 0, status = UFC_STATUS_OK;
  while (t < T * (1.0 - 1e-12) && a->attempts < a->max_increments) {
    dt = std::min(dt, T - t);
    const double t1 = t + dt;
    const double sfrac = t1 >= T ? 1.0 : t1 / T;
    if (c->nfix > 0) k_lerp<<<grid_for(c->nfix, 256), 256, 0, c->stream>>>(c->nfix, u0, uend, sfrac, ut);
    k_lerp<<<vg, 256, 0, c->stream>>>(c->n, fs.dev, fe.dev, sfrac, ft);
    if (cudaGetLastError() != cudaSuccess) {
      status = fail(c, UFC_STATUS_ERROR, "ufc_nr_step: launch failed");
      break;
    }
    ufc_nr_arg na{};
    na.u_prescribed = c->nfix > 0 ? ut : nullptr;
    na.f_ext = ft;
    na.mem = UFC_MEM_DEVICE;
    na.max_iterations = a->max_iterations;
    na.tolerance_force = a->tolerance_force;
    na.lin = a->lin;
    const int s = ufc_nr_increment(c, &na);
    const int k = a->attempts++;
    a->lin_iters_total += na.lin_iters_total;
    const bool ok = s == UFC_STATUS_OK && na.converged;
    if (k < a->hist_cap) {
      if (a->hist_time) a->hist_time[k] = t1;
      if (a->hist_dt) a->hist_dt[k] = dt;
      if (a->hist_iters) a->hist_iters[k] = na.iterations;
      if (a->hist_converged) a->hist_converged[k] = ok ? 1 : 0;
    }
    if (ok) {
      status = ufc_state_commit(c);
      if (status != UFC_STATUS_OK) break;
      t = t1 >= T ? T : t1;
      a->increments += 1;
      a->nr_iterations += na.iterations;
      cut_run = 0;
      if (a->auto_dt && na.iterations <= (int)(a->target_iters * a->growth_threshold))
        dt = std::min(dt * a->growth_factor, a->dt_max);
      continue;
    }
    if (s != UFC_STATUS_NOT_CONVERGED) {  // not a convergence failure: report it as is
      ufc_state_rollback(c);
      status = s;
      break;
    }
    status = ufc_state_rollback(c);
    if (status != UFC_STATUS_OK) break;
    a->cutbacks += 1;
    if (++cut_run > a->max_cutbacks) {
      status = fail(c, UFC_STATUS_NOT_CONVERGED, "ufc_nr_step: max cutbacks exceeded");
      break;
    }
    dt *= a->cutback_factor;
    if (dt < a->dt_min) {
      status = fail(c, UFC_STATUS_NOT_CONVERGED, "ufc_nr_step: increment below dt_min");
      break;
    }
  }
  cleanup();
  a->final_time = t;
  a->completed = t >= T * (1.0 - 1e-12) ? 1 : 0;
  if (status == UFC_STATUS_OK && !a->completed)
    status = fail(c, UFC_STATUS_NOT_CONVERGED, "ufc_nr_step: max_increments reached before the end of the step");
  a->status = status;
  UFC_TRY(sync(c));
  return status;
}

int ufc_state_commit(ufc_ctx* c) {
  CTX_CHECK(c);
  if (!c->has_material) return fail(c, UFC_STATUS_INVALID, "ufc_state_commit: material not set");
  Scope sc(c);
  UFC_CUDA(c, cudaMemcpyAsync(c->u_n, c->u, sizeof(double) * c->n, cudaMemcpyDeviceToDevice, c->stream));
  if (c->mat_model == UFC_MAT_J2_ISO && c->has_trial) {
    const int64_t G = (int64_t)c->E * 8;
    UFC_CUDA(c, cudaMemcpyAsync(c->sig_n, c->sig_t, sizeof(double) * G * 6, cudaMemcpyDeviceToDevice, c->stream));
    UFC_CUDA(c, cudaMemcpyAsync(c->epeq_n, c->epeq_t, sizeof(double) * G, cudaMemcpyDeviceToDevice, c->stream));
    UFC_CUDA(c, cudaMemcpyAsync(c->epl_n, c->epl_t, sizeof(double) * G * 6, cudaMemcpyDeviceToDevice, c->stream));
  }
  return sync(c);
}

int ufc_state_rollback(ufc_ctx* c) {
  CTX_CHECK(c);
  if (!c->has_material) return fail(c, UFC_STATUS_INVALID, "ufc_state_rollback: material not set");
  Scope sc(c);
  UFC_CUDA(c, cudaMemcpyAsync(c->u, c->u_n, sizeof(double) * c->n, cudaMemcpyDeviceToDevice, c->stream));
  c->has_trial = false;
  return sync(c);
}

int ufc_get_displacement(ufc_ctx* c, double* u, int32_t mem) {
  CTX_CHECK(c);
  if (!u || !c->u) return fail(c, UFC_STATUS_INVALID, "ufc_get_displacement");
  Scope sc(c);
  UFC_CUDA(c, cudaMemcpyAsync(u, c->u, sizeof(double) * c->n,
                              mem == UFC_MEM_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, c->stream));
  return sync(c);
}

int ufc_set_displacement(ufc_ctx* c, const double* u, int32_t mem) {
  CTX_CHECK(c);
  if (!u || !c->u) return fail(c, UFC_STATUS_INVALID, "ufc_set_displacement");
  Scope sc(c);
  UFC_CUDA(c, cudaMemcpyAsync(c->u, u, sizeof(double) * c->n,
                              mem == UFC_MEM_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, c->stream));
  return sync(c);
}

int ufc_get_state(ufc_ctx* c, double* epeq, double* sig, double* epl, int32_t mem) {
  CTX_CHECK(c);
  if (c->mat_model != UFC_MAT_J2_ISO) return fail(c, UFC_STATUS_INVALID, "ufc_get_state: no J2 state");
  Scope sc(c);
  const int64_t G = (int64_t)c->E * 8;
  const cudaMemcpyKind k = mem == UFC_MEM_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
  if (epeq) UFC_CUDA(c, cudaMemcpyAsync(epeq, c->epeq_n, sizeof(double) * G, k, c->stream));
  if (sig) UFC_CUDA(c, cudaMemcpyAsync(sig, c->sig_n, sizeof(double) * G * 6, k, c->stream));
  if (epl) UFC_CUDA(c, cudaMemcpyAsync(epl, c->epl_n, sizeof(double) * G * 6, k, c->stream));
  return sync(c);
}

int ufc_adjoint_sensitivity(ufc_ctx* c, int32_t nrhs, const double* U, const double* L, double* g, int32_t mem) {
  CTX_CHECK(c);
  if (!U || !L || !g || nrhs <= 0) return fail(c, UFC_STATUS_INVALID, "ufc_adjoint_sensitivity: NULL argument");
  if (!c->has_material || c->mat_model != UFC_MAT_ELASTIC_ISO)
    return fail(c, UFC_STATUS_INVALID, "ufc_adjoint_sensitivity: needs the linear-elastic material");
  Scope sc(c);
  Staged<double> su, sl, sg;
  UFC_TRY(stage_in(c, su, U, (int64_t)nrhs * c->n, mem));
  UFC_TRY(stage_in(c, sl, L, (int64_t)nrhs * c->n, mem));
  UFC_TRY(stage_out(c, sg, g, c->E, mem));
  UFC_TRY(adjoint_sens(c, nrhs, su.dev, sl.dev, sg.dev));
  UFC_TRY(finish(c, sg));
  return sync(c);
}

}  // extern "C"
