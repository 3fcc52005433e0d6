// The steps either side of the solve: the external load vector of face
// tractions and pressures, nodal stress by Gauss-point extrapolation, and
// reaction forces.
//
//   face loads        PH_Elem_C3D8_FormFacePressure (ufc_core/L4_PH/Element/Solid3D/PH_Elem_C3D8.f90:2360-2541),
//                     surface branch of RT_Asm_GlobalLoad (ufc_core/L5_RT/Assembly/RT_Asm_Solv.f90:1443)
//   nodal stress      PH_Elem_C3D8_GetExtrapMat / PH_Elem_C3D8_MapToNode (PH_Elem_C3D8.f90:2782-2824),
//                     PH_Elem_C3D8_EvalVonMises (:2768-2780)
//   reactions         constrained rows of R = F_ext - F_int, RT_Asm_ComputeResidual (RT_Asm_Solv.f90:1311-1426)
//
// Both scatters (face loads into nodal forces, element extrapolations into
// nodal sums) run per element colour, so no two threads of a launch touch the
// same node and the sums are deterministic without atomics.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <numeric>
#include <vector>

#include "c3d8_device.cuh"
#include "ufc_internal.cuh"

namespace ufc {

namespace {

// Face f (0-based, = reference face id - 1): the fixed parametric direction and
// its value, the two in-plane directions (u, v), the four face nodes in the
// reference's order, and the sign that turns n = dr/du x dr/dv into the
// outward normal of a positively oriented element.
struct FaceDef {
  int fixed_dim, fixed_sign, udim, vdim, nodes[4], out_sign;
};
__constant__ FaceDef kFaces[6] = {
    {2, -1, 0, 1, {0, 1, 2, 3}, -1},  // 1: zeta = -1
    {2, +1, 0, 1, {4, 7, 6, 5}, +1},  // 2: zeta = +1
    {1, -1, 0, 2, {0, 1, 5, 4}, +1},  // 3: eta = -1
    {1, +1, 0, 2, {3, 2, 6, 7}, -1},  // 4: eta = +1
    {0, -1, 1, 2, {0, 3, 7, 4}, -1},  // 5: xi = -1
    {0, +1, 1, 2, {1, 5, 6, 2}, +1},  // 6: xi = +1
};

// One thread per face of this pass: 2x2 Gauss rule (+-1/sqrt(3), weight 1) on
// the face, f_a += N_a (t - p n_out) dA for its four nodes.
__global__ void k_face_load(int32_t nf, const int32_t* __restrict__ idx, const int32_t* __restrict__ elem,
                            const int32_t* __restrict__ face, const double* __restrict__ traction,
                            const double* __restrict__ pressure, const double* __restrict__ coords,
                            const int32_t* __restrict__ conn, double* __restrict__ f) {
  const int32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nf) return;
  const int32_t k = idx[t];
  const int64_t e = elem[k];
  const FaceDef fd = kFaces[face[k] - 1];
  double X[4][3];
  int32_t nd[4];
#pragma unroll
  for (int a = 0; a < 4; ++a) {
    nd[a] = conn[e * 8 + fd.nodes[a]];
#pragma unroll
    for (int i = 0; i < 3; ++i) X[a][i] = coords[(int64_t)nd[a] * 3 + i];
  }
  double tr[3] = {0.0, 0.0, 0.0};
  if (traction)
#pragma unroll
    for (int i = 0; i < 3; ++i) tr[i] = traction[(int64_t)k * 3 + i];
  const double p = pressure ? pressure[k] : 0.0;
  double F[4][3] = {};
  const double g = 0.57735026918962576451;
#pragma unroll
  for (int gp = 0; gp < 4; ++gp) {
    double xi[3];
    xi[fd.fixed_dim] = (double)fd.fixed_sign;
    xi[fd.udim] = (gp & 1) ? g : -g;
    xi[fd.vdim] = (gp & 2) ? g : -g;
    double N[4], du[3] = {0, 0, 0}, dv[3] = {0, 0, 0};
#pragma unroll
    for (int a = 0; a < 4; ++a) {
      const int an = fd.nodes[a];
      double fac[3], s[3];
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        s[d] = (double)node_sign(an, d);
        fac[d] = 1.0 + s[d] * xi[d];
      }
      N[a] = 0.125 * fac[0] * fac[1] * fac[2];
      // in-plane derivatives: the factor of the derivative's own direction drops
      const double dNu = 0.125 * s[fd.udim] * fac[fd.vdim] * fac[fd.fixed_dim];
      const double dNv = 0.125 * s[fd.vdim] * fac[fd.udim] * fac[fd.fixed_dim];
#pragma unroll
      for (int i = 0; i < 3; ++i) {
        du[i] += dNu * X[a][i];
        dv[i] += dNv * X[a][i];
      }
    }
    const double n0 = du[1] * dv[2] - du[2] * dv[1];
    const double n1 = du[2] * dv[0] - du[0] * dv[2];
    const double n2 = du[0] * dv[1] - du[1] * dv[0];
    const double dA = sqrt(n0 * n0 + n1 * n1 + n2 * n2);
    if (dA < 1e-15) continue;  // degenerate face point, skipped as the reference does
    const double so = (double)fd.out_sign / dA;
    const double load[3] = {tr[0] - p * so * n0, tr[1] - p * so * n1, tr[2] - p * so * n2};
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
      for (int i = 0; i < 3; ++i) F[a][i] += N[a] * load[i] * dA;
  }
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int i = 0; i < 3; ++i) f[(int64_t)nd[a] * 3 + i] += F[a][i];
}

// Extrapolation from the 2x2x2 Gauss points to node a: the inverse of the
// interpolation matrix A(ip, a) = N_a(gauss point ip), which factors into 1-D
// inverses: E(a, ip) = prod_d (1 + sqrt(3) s_a,d s_ip,d) / 2.
__device__ __forceinline__ double extrap(int a, int ip) {
  const double r3 = 1.7320508075688772935;
  double v = 1.0;
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    const double sip = ((ip >> d) & 1) ? 1.0 : -1.0;
    v *= 0.5 * (1.0 + r3 * (double)node_sign(a, d) * sip);
  }
  return v;
}

// One thread per element of this colour: nodal values of the element's
// Gauss-point stress added to the node sums.
__global__ void k_extrap_scatter(const int32_t* __restrict__ el, int32_t ne, const int32_t* __restrict__ conn,
                                 const double* __restrict__ sig_gp, double* __restrict__ sum,
                                 int32_t* __restrict__ cnt) {
  const int32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= ne) return;
  const int64_t e = el[t];
  double s[8][6];
#pragma unroll
  for (int ip = 0; ip < 8; ++ip)
#pragma unroll
    for (int c = 0; c < 6; ++c) s[ip][c] = sig_gp[(e * 8 + ip) * 6 + c];
#pragma unroll 1
  for (int a = 0; a < 8; ++a) {
    const int64_t nd = conn[e * 8 + a];
    double v[6] = {0, 0, 0, 0, 0, 0};
#pragma unroll
    for (int ip = 0; ip < 8; ++ip) {
      const double w = extrap(a, ip);
#pragma unroll
      for (int c = 0; c < 6; ++c) v[c] += w * s[ip][c];
    }
#pragma unroll
    for (int c = 0; c < 6; ++c) sum[nd * 6 + c] += v[c];
    cnt[nd] += 1;
  }
}

__global__ void k_nodal_finish(int32_t N, const double* __restrict__ sum, const int32_t* __restrict__ cnt,
                               double* __restrict__ sig, double* __restrict__ vm) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  const double w = cnt[i] > 0 ? 1.0 / (double)cnt[i] : 0.0;
  double s[6];
#pragma unroll
  for (int c = 0; c < 6; ++c) s[c] = sum[i * 6 + c] * w;
  if (sig)
#pragma unroll
    for (int c = 0; c < 6; ++c) sig[i * 6 + c] = s[c];
  if (vm) {
    const double p = (s[0] + s[1] + s[2]) / 3.0;
    const double j2 = 0.5 * ((s[0] - p) * (s[0] - p) + (s[1] - p) * (s[1] - p) + (s[2] - p) * (s[2] - p)) +
                      s[3] * s[3] + s[4] * s[4] + s[5] * s[5];
    vm[i] = sqrt(3.0 * fmax(j2, 0.0));
  }
}

__global__ void k_gather_rf(int32_t nfix, const int32_t* __restrict__ dofs, const double* __restrict__ fint,
                            const double* __restrict__ fext, double* __restrict__ rf) {
  const int32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= nfix) return;
  const int32_t d = dofs[k];
  rf[k] = fint[d] - (fext ? fext[d] : 0.0);
}

template <class T>
struct AsyncBuf {
  T* p = nullptr;
  cudaStream_t s = nullptr;
  ~AsyncBuf() {
    if (p) cudaFreeAsync(p, s);
  }
};

template <class T>
int async_alloc(Ctx* c, AsyncBuf<T>& b, int64_t count) {
  b.s = c->stream;
  UFC_CUDA(c, cudaMallocAsync((void**)&b.p, sizeof(T) * (size_t)std::max<int64_t>(count, 1), c->stream));
  return UFC_STATUS_OK;
}

}  // namespace

int face_loads(Ctx* c, int32_t n_faces, const int32_t* h_elem, const int32_t* h_face, const double* traction,
               const double* pressure, double* f) {
  UFC_CUDA(c, cudaMemsetAsync(f, 0, sizeof(double) * c->n, c->stream));
  if (n_faces == 0) return UFC_STATUS_OK;
  // passes: for each colour, the j-th face (in input order) of every element of
  // that colour; faces of one pass belong to distinct elements of one colour,
  // which share no node
  std::vector<int32_t> order(n_faces);
  std::iota(order.begin(), order.end(), 0);
  std::stable_sort(order.begin(), order.end(), [&](int32_t a, int32_t b) {
    const int32_t ca = c->h_color[h_elem[a]], cb = c->h_color[h_elem[b]];
    if (ca != cb) return ca < cb;
    return h_elem[a] < h_elem[b];
  });
  std::vector<int32_t> flat;
  std::vector<int64_t> off{0};
  flat.reserve(n_faces);
  size_t i = 0;
  while (i < order.size()) {
    const int32_t col = c->h_color[h_elem[order[i]]];
    size_t j = i;
    while (j < order.size() && c->h_color[h_elem[order[j]]] == col) ++j;
    // faces [i, j) of this colour, grouped by element; rank of each face in its element
    std::vector<int32_t> rank(j - i, 0);
    int32_t maxr = 0;
    for (size_t q = i + 1; q < j; ++q)
      if (h_elem[order[q]] == h_elem[order[q - 1]]) {
        rank[q - i] = rank[q - 1 - i] + 1;
        maxr = std::max(maxr, rank[q - i]);
      }
    for (int32_t r = 0; r <= maxr; ++r) {
      for (size_t q = i; q < j; ++q)
        if (rank[q - i] == r) flat.push_back(order[q]);
      off.push_back((int64_t)flat.size());
    }
    i = j;
  }
  AsyncBuf<int32_t> didx, delem, dface;
  UFC_TRY(async_alloc(c, didx, n_faces));
  UFC_TRY(async_alloc(c, delem, n_faces));
  UFC_TRY(async_alloc(c, dface, n_faces));
  UFC_CUDA(c, cudaMemcpyAsync(didx.p, flat.data(), sizeof(int32_t) * n_faces, cudaMemcpyHostToDevice, c->stream));
  UFC_CUDA(c, cudaMemcpyAsync(delem.p, h_elem, sizeof(int32_t) * n_faces, cudaMemcpyHostToDevice, c->stream));
  UFC_CUDA(c, cudaMemcpyAsync(dface.p, h_face, sizeof(int32_t) * n_faces, cudaMemcpyHostToDevice, c->stream));
  for (size_t pz = 0; pz + 1 < off.size(); ++pz) {
    const int32_t nf = (int32_t)(off[pz + 1] - off[pz]);
    if (nf == 0) continue;
    k_face_load<<<grid_for(nf, 128), 128, 0, c->stream>>>(nf, didx.p + off[pz], delem.p, dface.p, traction, pressure,
                                                          c->coords, c->conn, f);
    UFC_CUDA(c, cudaGetLastError());
  }
  // the host vectors above are read by the copies: wait before they go
  UFC_CUDA(c, cudaStreamSynchronize(c->stream));
  return UFC_STATUS_OK;
}

int stress_nodal(Ctx* c, const double* u, double* sig_node, double* vm_node) {
  const int64_t G = (int64_t)c->E * 8;
  AsyncBuf<double> sgp, sum;
  AsyncBuf<int32_t> cnt;
  UFC_TRY(async_alloc(c, sgp, G * 6));
  UFC_TRY(async_alloc(c, sum, (int64_t)c->N * 6));
  UFC_TRY(async_alloc(c, cnt, c->N));
  UFC_TRY(stress_eval(c, u, sgp.p, nullptr));
  UFC_CUDA(c, cudaMemsetAsync(sum.p, 0, sizeof(double) * c->N * 6, c->stream));
  UFC_CUDA(c, cudaMemsetAsync(cnt.p, 0, sizeof(int32_t) * c->N, c->stream));
  for (int col = 0; col < c->ncol; ++col) {
    const int32_t ne = c->col_off[col + 1] - c->col_off[col];
    if (ne == 0) continue;
    k_extrap_scatter<<<grid_for(ne, 128), 128, 0, c->stream>>>(c->col_elems + c->col_off[col], ne, c->conn, sgp.p,
                                                               sum.p, cnt.p);
    UFC_CUDA(c, cudaGetLastError());
  }
  k_nodal_finish<<<grid_for(c->N, 256), 256, 0, c->stream>>>(c->N, sum.p, cnt.p, sig_node, vm_node);
  UFC_CUDA(c, cudaGetLastError());
  return UFC_STATUS_OK;
}

int reactions(Ctx* c, const double* u, const double* f_ext, double* rf) {
  if (c->nfix == 0) return UFC_STATUS_OK;
  AsyncBuf<double> fint;
  UFC_TRY(async_alloc(c, fint, c->n));
  UFC_TRY(compute_fint(c, u, fint.p, false));
  k_gather_rf<<<grid_for(c->nfix, 256), 256, 0, c->stream>>>(c->nfix, c->fix_dofs, fint.p, f_ext, rf);
  UFC_CUDA(c, cudaGetLastError());
  return UFC_STATUS_OK;
}

}  // namespace ufc
