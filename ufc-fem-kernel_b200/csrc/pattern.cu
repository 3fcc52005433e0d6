// Device-built stiffness pattern, built once per mesh.
//
// The canonical pattern is the block form of RT_CSR_FromTripletMerged
// (ufc_core/L5_RT/Solver/RT_Solv_Sparse.f90:336-445): per node row, the sorted
// unique set of nodes that share an element with it; every coupled node pair is
// a dense 3x3 block, so the scalar CSR row 3i+r lists 3*col+c for every block
// column col in ascending order and c = 0..2.  That canonical pattern is what
// ufc_csr_export returns.
//
// Values are stored in SELL-32 form: block rows are grouped into slices of 32
// consecutive rows, each slice padded to its longest row, and a slice's entry j
// of all 32 rows is stored contiguously, component by component.  One warp then
// reads 128 contiguous bytes (FP32) per load instruction in the SpMV.
//
// Element colouring for the deterministic scatter is the greedy colouring of
// RT_AsmColor_Build (ufc_core/L5_RT/Assembly/RT_Asm_Color.f90:36-182), elements
// visited in ascending order, smallest free colour first; it is computed on the
// device as the fixed point of that rule (k_color_sweep).
#include <cub/cub.cuh>
#include <cuda_runtime.h>

#include <algorithm>
#include <vector>

#include "c3d8_device.cuh"
#include "ufc_internal.cuh"

namespace ufc {

namespace {

__global__ void k_count_node_elems(int32_t E, const int32_t* __restrict__ conn, int32_t* __restrict__ cnt) {
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= 8 * (int64_t)E) return;
  atomicAdd(&cnt[conn[k]], 1);  // integer counts: order-independent
}

__global__ void k_fill_node_elems(int32_t E, const int32_t* __restrict__ conn, const int32_t* __restrict__ nptr,
                                  int32_t* __restrict__ fill, int32_t* __restrict__ nlst) {
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= 8 * (int64_t)E) return;
  const int32_t nd = conn[k];
  const int32_t pos = atomicAdd(&fill[nd], 1);
  nlst[nptr[nd] + pos] = (int32_t)(k >> 3);
}

// Sort each node's element list (the fill order above is not deterministic) and
// check the valence bound.
__global__ void k_sort_node_elems(int32_t N, const int32_t* __restrict__ nptr, int32_t* __restrict__ nlst,
                                  int32_t* __restrict__ err) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  const int32_t b = nptr[i], m = nptr[i + 1] - b;
  if (m > kMaxValence) {
    atomicOr(err, (int)kDevValence);
    return;
  }
  for (int k = 1; k < m; ++k) {
    const int32_t v = nlst[b + k];
    int j = k - 1;
    while (j >= 0 && nlst[b + j] > v) {
      nlst[b + j + 1] = nlst[b + j];
      --j;
    }
    nlst[b + j + 1] = v;
  }
}

// Element colouring on the device.  The sequential greedy colouring (elements
// in ascending order, each taking the smallest colour that none of its lower
// neighbours -- elements f < e sharing a node with e -- has) is the unique
// fixed point of the map colour[e] = mex{colour[f] : f a lower neighbour of e}:
// element 0 has no lower neighbour, and by induction every element is fixed
// once its lower neighbours are.  Sweeping that map over all elements at once,
// in place, from colour 0 everywhere therefore reaches exactly the sequential
// colouring, and a sweep that changes nothing proves it has been reached (every
// element then read values that did not move).  The number of sweeps follows
// the longest chain of lower neighbours along which the colours still change:
// about nx + ny + nz on a structured box numbered lexicographically, fewer on
// shuffled numberings.

// Lower neighbours of element e, ascending and unique: an 8-way merge of its
// nodes' element lists (sorted by k_sort_node_elems), stopped at e itself.
// kFill = false counts them into cnt[e], true writes them at elst + eptr[e].
template <bool kFill>
__global__ void __launch_bounds__(128)
    k_elem_lower(int32_t E, const int32_t* __restrict__ conn, const int32_t* __restrict__ nptr,
                 const int32_t* __restrict__ nlst, int64_t* __restrict__ cnt, const int64_t* __restrict__ eptr,
                 int32_t* __restrict__ elst) {
  const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= E) return;
  int32_t pos[8], end[8];
#pragma unroll
  for (int a = 0; a < 8; ++a) {
    const int32_t nd = conn[e * 8 + a];
    pos[a] = nptr[nd];
    end[a] = nptr[nd + 1];
  }
  int32_t* out = kFill ? elst + eptr[e] : nullptr;
  int64_t m = 0;
  for (;;) {
    int32_t best = INT32_MAX;
#pragma unroll
    for (int a = 0; a < 8; ++a)
      if (pos[a] < end[a]) best = min(best, nlst[pos[a]]);
    if (best >= e) break;  // every list holds e itself; what follows it is higher
#pragma unroll
    for (int a = 0; a < 8; ++a)
      if (pos[a] < end[a] && nlst[pos[a]] == best) ++pos[a];
    if (kFill) out[m] = best;
    ++m;
  }
  if (!kFill) cnt[e] = m;
}

// One in-place sweep of the colouring map.  flag[0] is set when a colour moved,
// flag[1] when a mex exceeded 255 (impossible while a node has at most
// kMaxValence elements: an element then has at most 8 (kMaxValence - 1) lower
// neighbours; the host colouring takes over if it happens).  Reads of colours
// other threads write in the same sweep see either value, both of which the
// fixed-point argument allows.
__global__ void __launch_bounds__(256)
    k_color_sweep(int32_t E, const int64_t* __restrict__ eptr, const int32_t* __restrict__ elst,
                  uint8_t* color, int32_t* __restrict__ flag) {
  const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= E) return;
  uint64_t used[4] = {0, 0, 0, 0};
  for (int64_t k = eptr[e]; k < eptr[e + 1]; ++k) {
    const unsigned cf = color[elst[k]];
    used[cf >> 6] |= 1ull << (cf & 63);
  }
  unsigned c = 256;
#pragma unroll
  for (int w = 3; w >= 0; --w)
    if (~used[w]) c = 64 * w + __ffsll((long long)~used[w]) - 1;
  if (c > 255) {
    flag[1] = 1;
    return;
  }
  if (color[e] != c) {
    color[e] = (uint8_t)c;
    flag[0] = 1;
  }
}

// Sorted unique neighbours of node i into buf (capacity kMaxRowBlocks); returns
// the count, or -1 when it would exceed the capacity.
__device__ int node_neighbours(int64_t i, const int32_t* __restrict__ conn, const int32_t* __restrict__ nptr,
                               const int32_t* __restrict__ nlst, int32_t* buf) {
  int u = 0;
  for (int32_t k = nptr[i]; k < nptr[i + 1]; ++k) {
    const int64_t e = nlst[k];
    for (int a = 0; a < 8; ++a) {
      const int32_t v = conn[e * 8 + a];
      int lo = 0, hi = u;
      while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (buf[mid] < v) lo = mid + 1;
        else hi = mid;
      }
      if (lo < u && buf[lo] == v) continue;
      if (u == kMaxRowBlocks) return -1;
      for (int j = u; j > lo; --j) buf[j] = buf[j - 1];
      buf[lo] = v;
      ++u;
    }
  }
  return u;
}

__global__ void k_row_count(int32_t N, const int32_t* __restrict__ conn, const int32_t* __restrict__ nptr,
                            const int32_t* __restrict__ nlst, int32_t* __restrict__ cnt, int32_t* __restrict__ err) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  int32_t buf[kMaxRowBlocks];
  const int u = node_neighbours(i, conn, nptr, nlst, buf);
  if (u < 0) atomicOr(err, (int)kDevRowBlocks);
  cnt[i] = u < 0 ? 0 : u;
}

__global__ void k_row_fill(int32_t N, const int32_t* __restrict__ conn, const int32_t* __restrict__ nptr,
                           const int32_t* __restrict__ nlst, const int32_t* __restrict__ brow,
                           int32_t* __restrict__ bcol) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  int32_t buf[kMaxRowBlocks];
  const int u = node_neighbours(i, conn, nptr, nlst, buf);
  for (int k = 0; k < u; ++k) bcol[brow[i] + k] = buf[k];
}

// Longest row of each slice, in blocks.
__global__ void k_slice_len(int32_t N, int64_t nslices, const int32_t* __restrict__ brow, int64_t* __restrict__ len) {
  const int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= nslices) return;
  int32_t m = 0;
  for (int t = 0; t < kSlice; ++t) {
    const int64_t r = s * kSlice + t;
    if (r < N) m = max(m, brow[r + 1] - brow[r]);
  }
  len[s] = (int64_t)m * kSlice;
}

// SELL column array: real entries, then padding that points at the row itself
// (zero values), one thread per padded row.
__global__ void k_sell_fill(int32_t N, int64_t nslices, const int32_t* __restrict__ brow,
                            const int32_t* __restrict__ bcol, const int64_t* __restrict__ sptr,
                            int32_t* __restrict__ scol, int32_t* __restrict__ dpos) {
  const int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= nslices * kSlice) return;
  const int64_t s = r / kSlice, t = r % kSlice;
  const int64_t base = sptr[s], len = (sptr[s + 1] - base) / kSlice;
  const int32_t b = r < N ? brow[r] : 0, m = r < N ? brow[r + 1] - b : 0;
  const int32_t self = r < N ? (int32_t)r : 0;
  for (int64_t j = 0; j < len; ++j) {
    const int32_t cj = j < m ? bcol[b + j] : self;
    scol[base + j * kSlice + t] = cj;
    if (r < N && j < m && cj == r) dpos[r] = (int32_t)(base + j * kSlice + t);
  }
}

// slot[e][a][b] = SELL position of block (conn[a], conn[b]).
__global__ void k_slots(int32_t E, const int32_t* __restrict__ conn, const int32_t* __restrict__ brow,
                        const int32_t* __restrict__ bcol, const int64_t* __restrict__ sptr,
                        int32_t* __restrict__ slot, int32_t* __restrict__ err) {
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= 8 * (int64_t)E) return;
  const int64_t e = k >> 3;
  const int a = (int)(k & 7);
  const int32_t r = conn[e * 8 + a];
  const int64_t s = r / kSlice, t = r % kSlice;
  for (int b = 0; b < 8; ++b) {
    const int32_t cb = conn[e * 8 + b];
    int lo = brow[r], hi = brow[r + 1] - 1, found = -1;
    while (lo <= hi) {
      const int mid = (lo + hi) >> 1;
      const int32_t v = bcol[mid];
      if (v < cb) lo = mid + 1;
      else if (v > cb) hi = mid - 1;
      else {
        found = mid - brow[r];
        break;
      }
    }
    if (found < 0) {
      atomicOr(err, (int)kDevPattern);
      found = 0;
    }
    slot[e * 64 + a * 8 + b] = (int32_t)(sptr[s] + (int64_t)found * kSlice + t);
  }
}

// Position of column v in canonical block row r (binary search), or -1.
__device__ __forceinline__ int find_in_row(const int32_t* __restrict__ brow, const int32_t* __restrict__ bcol,
                                           int64_t r, int32_t v) {
  int lo = brow[r], hi = brow[r + 1] - 1;
  while (lo <= hi) {
    const int mid = (lo + hi) >> 1;
    const int32_t x = bcol[mid];
    if (x < v) lo = mid + 1;
    else if (x > v) hi = mid - 1;
    else return mid - brow[r];
  }
  return -1;
}

// Lower (j < i) and upper (j >= i) block counts of every row.
__global__ void k_sym_counts(int32_t N, const int32_t* __restrict__ brow, const int32_t* __restrict__ bcol,
                             int32_t* __restrict__ lcnt, int32_t* __restrict__ ucnt) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  const int d = find_in_row(brow, bcol, i, (int32_t)i);  // the diagonal is always present
  lcnt[i] = d;
  ucnt[i] = brow[i + 1] - brow[i] - d;
}

__global__ void k_slice_len_counts(int32_t N, int64_t nslices, const int32_t* __restrict__ cnt,
                                   int64_t* __restrict__ len) {
  const int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= nslices) return;
  int32_t m = 0;
  for (int t = 0; t < kSlice; ++t) {
    const int64_t r = s * kSlice + t;
    if (r < N) m = max(m, cnt[r]);
  }
  len[s] = (int64_t)m * kSlice;
}

// Symmetric storage index arrays, one thread per (padded) row: upper columns
// (padding points at the row itself, zero values) and, for every lower block
// (j, i), its position in row j's upper storage (padding points at the zero
// slice appended after the last stored block).
__global__ void k_sym_fill(int32_t N, int64_t nslices, const int32_t* __restrict__ brow,
                           const int32_t* __restrict__ bcol, const int32_t* __restrict__ lcnt,
                           const int64_t* __restrict__ uptr, const int64_t* __restrict__ lptr, int64_t zero_pos,
                           int32_t* __restrict__ ucol, int32_t* __restrict__ lpos, int32_t* __restrict__ lcol,
                           int32_t* __restrict__ err) {
  const int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= nslices * kSlice) return;
  const int64_t s = r / kSlice, t = r % kSlice;
  const int64_t ub = uptr[s], ul = (uptr[s + 1] - ub) / kSlice;
  const int64_t lb = lptr[s], ll = (lptr[s + 1] - lb) / kSlice;
  const bool real = r < N;
  const int32_t b = real ? brow[r] : 0;
  const int32_t nl = real ? lcnt[r] : 0;
  const int32_t nu = real ? brow[r + 1] - b - nl : 0;
  const int32_t self = real ? (int32_t)r : 0;
  for (int64_t j = 0; j < ul; ++j) ucol[ub + j * kSlice + t] = j < nu ? bcol[b + nl + j] : self;
  // lower entries in descending column order: the k-th lower entry of row r is
  // then paired with (about) the k-th upper entry of the row that stores it, so
  // the SpMV touches both within one loop step and the second read hits L2
  for (int64_t j = 0; j < ll; ++j) {
    int32_t pos = (int32_t)zero_pos, cj = 0;
    if (j < nl) {
      cj = bcol[b + nl - 1 - j];  // cj < r: block (cj, r) lives in row cj's upper part
      const int k = find_in_row(brow, bcol, cj, (int32_t)r);
      if (k < 0) {
        atomicOr(err, (int)kDevPattern);
      } else {
        const int64_t sj = cj / kSlice, tj = cj % kSlice;
        pos = (int32_t)(uptr[sj] + (int64_t)(k - lcnt[cj]) * kSlice + tj);
      }
    }
    lpos[lb + j * kSlice + t] = pos;
    lcol[lb + j * kSlice + t] = cj;
  }
}

// Coded indices of the symmetric storage.  First the set of upper offsets
// (col - row >= 0) of the real blocks, as bits of a bitmap over [0, kOffRange);
// a larger offset sets bit 0 of *flags (the pattern is not stencil-like).
constexpr int64_t kOffRange = 1 << 21;

__global__ void k_sym_offsets(int32_t N, int64_t nslices, const int64_t* __restrict__ uptr,
                              const int32_t* __restrict__ ucol, uint32_t* __restrict__ bits,
                              int32_t* __restrict__ flags) {
  const int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= N) return;
  const int64_t s = r / kSlice, t = r % kSlice;
  const int64_t ub = uptr[s], ul = (uptr[s + 1] - ub) / kSlice;
  if (ul > 16) atomicOr(flags, 2);
  for (int64_t k = 0; k < ul; ++k) {
    const int64_t c = ucol[ub + k * kSlice + t];
    if (k > 0 && c == r) continue;  // padding
    const int64_t d = c - r;
    if (d < 0 || d >= kOffRange) {
      atomicOr(flags, 1);
      continue;
    }
    const uint32_t m = 1u << (d & 31);
    if (!(bits[d >> 5] & m)) atomicOr(bits + (d >> 5), m);  // most rows repeat the same few bits
  }
}

// The code bytes, lane-major: row r's 16 upper codes at ucode[16 r], its 16
// lower codes at lcode[16 r].  Upper code: index of col - row in tab (15: no
// block, the padding).  Lower code: (index of row - col) << 4 | rank of the
// block (col, row) in row col's upper list (0xFF: no block).  Sets bit 2 of
// *flags when a slice has more than 16 lower steps or an offset is not in tab.
__global__ void k_sym_codes(int32_t N, int64_t nslices, const int64_t* __restrict__ uptr,
                            const int64_t* __restrict__ lptr, const int32_t* __restrict__ ucol,
                            const int32_t* __restrict__ lpos, const int32_t* __restrict__ lcol, int64_t zero_pos,
                            SymOffsets tab, int ntab, uint8_t* __restrict__ ucode, uint8_t* __restrict__ lcode,
                            int32_t* __restrict__ flags) {
  const int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= nslices * kSlice) return;
  const int64_t s = r / kSlice, t = r % kSlice;
  const int64_t ub = uptr[s], ul = (uptr[s + 1] - ub) / kSlice;
  const int64_t lb = lptr[s], ll = (lptr[s + 1] - lb) / kSlice;
  if (ll > 16 || ul > 16) atomicOr(flags, 4);
  auto find = [&](int64_t d) -> int {
    for (int q = 0; q < ntab; ++q)
      if (tab.off[q] == d) return q;
    atomicOr(flags, 4);
    return kSymCodes;
  };
  for (int k = 0; k < 16; ++k) {
    uint8_t u = kSymCodes, l = 0xFF;
    if (r < N && k < ul) {
      const int64_t c = ucol[ub + k * kSlice + t];
      if (k == 0 || c != r) u = (uint8_t)find(c - r);
    }
    if (r < N && k < ll) {
      const int64_t pos = lpos[lb + k * kSlice + t];
      if (pos != zero_pos) {
        const int64_t c = lcol[lb + k * kSlice + t];
        const int64_t rank = (pos - uptr[c / kSlice] - c % kSlice) / kSlice;
        const int q = find(r - c);
        if (rank < 0 || rank > 15 || q >= kSymCodes) atomicOr(flags, 4);
        else l = (uint8_t)((q << 4) | rank);
      }
    }
    ucode[r * 16 + k] = u;
    lcode[r * 16 + k] = l;
  }
}

// Coded indices of the full SELL storage: the offsets col - row of the real
// blocks as bits over [-kOffRange, kOffRange), then 32 code bytes per row.
__global__ void k_full_offsets(int32_t N, int64_t nslices, const int64_t* __restrict__ sptr,
                               const int32_t* __restrict__ col, uint32_t* __restrict__ bits,
                               int32_t* __restrict__ flags) {
  const int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= N) return;
  const int64_t s = r / kSlice, t = r % kSlice;
  const int64_t b = sptr[s], len = (sptr[s + 1] - b) / kSlice;
  if (len > 32) atomicOr(flags, 2);
  for (int64_t k = 0; k < len; ++k) {
    const int64_t d = (int64_t)col[b + k * kSlice + t] - r + kOffRange;
    if (d < 0 || d >= 2 * kOffRange) {
      atomicOr(flags, 1);
      continue;
    }
    const uint32_t m = 1u << (d & 31);
    if (!(bits[d >> 5] & m)) atomicOr(bits + (d >> 5), m);
  }
}

// Code of block k of row r at code[32 r + k]: index of col - row in tab, 255
// for no block (k beyond the slice, or a row past the mesh).  Padding blocks of
// a real row point at the row itself (offset 0) with zero values.
__global__ void k_full_codes(int32_t N, int64_t nslices, const int64_t* __restrict__ sptr,
                             const int32_t* __restrict__ col, FullOffsets tab, int ntab, uint8_t* __restrict__ code,
                             int32_t* __restrict__ flags) {
  const int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= nslices * kSlice) return;
  const int64_t s = r / kSlice, t = r % kSlice;
  const int64_t b = sptr[s], len = (sptr[s + 1] - b) / kSlice;
  for (int k = 0; k < 32; ++k) {
    uint8_t u = 255;
    if (r < N && k < len) {
      const int64_t d = (int64_t)col[b + k * kSlice + t] - r;
      int q = 0;
      while (q < ntab && tab.off[q] != d) ++q;
      if (q == ntab) atomicOr(flags, 4);
      else u = (uint8_t)q;
    }
    code[r * 32 + k] = u;
  }
}

// Copy the upper blocks of the full SELL values into the symmetric storage.
template <typename TO>
__global__ void k_sym_pack(int32_t N, const int64_t* __restrict__ sptr, const int64_t* __restrict__ uptr,
                           const int32_t* __restrict__ brow, const int32_t* __restrict__ lcnt,
                           const double* __restrict__ v64, TO* __restrict__ out) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  const int64_t s = i / kSlice, t = i % kSlice;
  const int32_t nl = lcnt[i], nu = brow[i + 1] - brow[i] - nl;
  for (int32_t j = 0; j < nu; ++j) {
    const int64_t src = sptr[s] + (int64_t)(nl + j) * kSlice + t;
    const int64_t dst = uptr[s] + (int64_t)j * kSlice + t;
#pragma unroll
    for (int c = 0; c < 9; ++c) out[vpos(dst, c)] = (TO)v64[vpos(src, c)];
  }
}

// Scalar CSR export from the block pattern, one thread per (block row, entry).
template <typename TV>
__global__ void k_export(int32_t N, const int32_t* __restrict__ brow, const int32_t* __restrict__ bcol,
                         const int64_t* __restrict__ sptr, const TV* __restrict__ val, int base,
                         int64_t* __restrict__ row_ptr, int32_t* __restrict__ col, double* __restrict__ v64,
                         float* __restrict__ v32) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  const int64_t b = brow[i], m = brow[i + 1] - b;
  if (row_ptr) {
    for (int r = 0; r < 3; ++r) row_ptr[3 * i + r] = 9 * b + r * 3 * m + base;
    if (i == N - 1) row_ptr[3 * (int64_t)N] = 9 * (int64_t)brow[N] + base;
  }
  const int64_t s = i / kSlice, t = i % kSlice;
  for (int64_t k = 0; k < m; ++k) {
    const int64_t P = sptr[s] + k * kSlice + t;
    const int32_t cb = bcol[b + k];
    for (int r = 0; r < 3; ++r) {
      const int64_t o = 9 * b + r * 3 * m + 3 * k;
      for (int cc = 0; cc < 3; ++cc) {
        if (col) col[o + cc] = 3 * cb + cc + base;
        if (val) {
          const TV x = val[vpos(P, r * 3 + cc)];
          if (v64) v64[o + cc] = (double)x;
          if (v32) v32[o + cc] = (float)x;
        }
      }
    }
  }
}

// Greedy colouring on the host (deterministic, visits elements in order): the
// same colouring as the device sweeps, used only when they have not settled
// within kMaxColorSweeps.
int color_elements(Ctx* c, std::vector<int32_t>& color) {
  const int32_t N = c->N, E = c->E;
  const std::vector<int32_t>& conn = c->h_conn;
  std::vector<int32_t> nptr(N + 1, 0), nlst((size_t)E * 8);
  for (int64_t k = 0; k < 8 * (int64_t)E; ++k) nptr[conn[k] + 1]++;
  for (int32_t i = 0; i < N; ++i) nptr[i + 1] += nptr[i];
  {
    std::vector<int32_t> fill(nptr.begin(), nptr.end() - 1);
    for (int64_t k = 0; k < 8 * (int64_t)E; ++k) nlst[fill[conn[k]]++] = (int32_t)(k >> 3);
  }
  color.assign(E, -1);
  int ncol = 0;
  for (int64_t e = 0; e < E; ++e) {
    uint64_t used[4] = {0, 0, 0, 0};
    for (int a = 0; a < 8; ++a) {
      const int32_t nd = conn[e * 8 + a];
      for (int32_t k = nptr[nd]; k < nptr[nd + 1]; ++k) {
        const int32_t f = nlst[k];
        if (f < e) used[color[f] >> 6] |= 1ull << (color[f] & 63);
      }
    }
    int col = 0;
    while (col < 256 && ((used[col >> 6] >> (col & 63)) & 1ull)) ++col;
    if (col >= 256) return fail(c, UFC_STATUS_UNSUPPORTED, "element colouring needs more than 256 colours");
    color[e] = col;
    ncol = std::max(ncol, col + 1);
  }
  c->ncol = ncol;
  return UFC_STATUS_OK;
}

template <class T>
int scan_exclusive(Ctx* c, const T* in, T* out, int64_t n) {
  size_t bytes = 0;
  UFC_CUDA(c, cub::DeviceScan::ExclusiveSum(nullptr, bytes, in, out, (int)n, c->stream));
  void* tmp = nullptr;
  UFC_CUDA(c, cudaMallocAsync(&tmp, bytes, c->stream));
  cudaError_t e = cub::DeviceScan::ExclusiveSum(tmp, bytes, in, out, (int)n, c->stream);
  cudaFreeAsync(tmp, c->stream);
  if (e != cudaSuccess) return cuda_fail(c, e, "cub::DeviceScan::ExclusiveSum");
  return UFC_STATUS_OK;
}

// Sweeps launched between two looks at their flags, and the number after which
// the host colouring takes over (numberings whose lower-neighbour chains keep
// changing colours for that long, e.g. a strip one element thick numbered
// along its length, which settles one element per sweep).
constexpr int kColorBatch = 32;
constexpr int kMaxColorSweeps = 4096;

struct ColorTmp {
  int64_t* cnt = nullptr;
  int64_t* eptr = nullptr;
  int32_t* elst = nullptr;
  uint8_t* col8 = nullptr;
  int32_t* flags = nullptr;
  ~ColorTmp() {
    dfree(&cnt);
    dfree(&eptr);
    dfree(&elst);
    dfree(&col8);
    dfree(&flags);
  }
};

// The greedy colouring of RT_AsmColor_Build (RT_Asm_Color.f90:36-182) by
// in-place sweeps on the device (see k_color_sweep) over the lower-neighbour
// lists, from the node -> element lists nptr / nlst; color[e] on the host.
int color_elements_device(Ctx* c, const int32_t* nptr, const int32_t* nlst, std::vector<int32_t>& color) {
  const int32_t E = c->E;
  ColorTmp t;
  UFC_TRY(dalloc(c, &t.cnt, (int64_t)E + 1));
  UFC_TRY(dalloc(c, &t.eptr, (int64_t)E + 1));
  UFC_CUDA(c, cudaMemsetAsync(t.cnt + E, 0, sizeof(int64_t), c->stream));
  k_elem_lower<false><<<grid_for(E, 128), 128, 0, c->stream>>>(E, c->conn, nptr, nlst, t.cnt, nullptr, nullptr);
  UFC_CUDA(c, cudaGetLastError());
  UFC_TRY(scan_exclusive(c, t.cnt, t.eptr, (int64_t)E + 1));
  int64_t total = 0;
  UFC_CUDA(c, cudaMemcpyAsync(&total, t.eptr + E, sizeof(int64_t), cudaMemcpyDeviceToHost, c->stream));
  UFC_CUDA(c, cudaStreamSynchronize(c->stream));
  UFC_TRY(dalloc(c, &t.elst, total));
  k_elem_lower<true><<<grid_for(E, 128), 128, 0, c->stream>>>(E, c->conn, nptr, nlst, nullptr, t.eptr, t.elst);
  UFC_CUDA(c, cudaGetLastError());
  UFC_TRY(dalloc(c, &t.col8, E));
  UFC_TRY(dalloc(c, &t.flags, 2 * kColorBatch));
  UFC_CUDA(c, cudaMemsetAsync(t.col8, 0, (size_t)E, c->stream));
  int32_t hf[2 * kColorBatch];
  bool settled = false, overflow = false;
  for (int sweeps = 0; !settled && !overflow && sweeps < kMaxColorSweeps; sweeps += kColorBatch) {
    UFC_CUDA(c, cudaMemsetAsync(t.flags, 0, sizeof(int32_t) * 2 * kColorBatch, c->stream));
    for (int b = 0; b < kColorBatch; ++b)
      k_color_sweep<<<grid_for(E, 256), 256, 0, c->stream>>>(E, t.eptr, t.elst, t.col8, t.flags + 2 * b);
    UFC_CUDA(c, cudaGetLastError());
    UFC_CUDA(c, cudaMemcpyAsync(hf, t.flags, sizeof(hf), cudaMemcpyDeviceToHost, c->stream));
    UFC_CUDA(c, cudaStreamSynchronize(c->stream));
    for (int b = 0; b < kColorBatch && !settled; ++b) {
      overflow |= hf[2 * b + 1] != 0;
      settled = hf[2 * b] == 0 && hf[2 * b + 1] == 0;
    }
  }
  if (!settled) return color_elements(c, color);
  std::vector<uint8_t> h((size_t)E);
  UFC_CUDA(c, cudaMemcpyAsync(h.data(), t.col8, (size_t)E, cudaMemcpyDeviceToHost, c->stream));
  UFC_CUDA(c, cudaStreamSynchronize(c->stream));
  color.resize(E);
  int ncol = 0;
  for (int32_t e = 0; e < E; ++e) {
    color[e] = h[e];
    ncol = std::max(ncol, (int)h[e] + 1);
  }
  c->ncol = ncol;
  return UFC_STATUS_OK;
}

}  // namespace

// The coded indices, when the pattern allows them (else sym_coded stays false
// and the products read the 4-byte columns and lower references).
int build_sym_codes(Ctx* c) {
  c->sym_coded = false;
  dfree(&c->sym_ucode);
  dfree(&c->sym_lcode);
  const int64_t nwords = kOffRange / 32;
  uint32_t* bits = nullptr;
  int32_t* flags = nullptr;
  UFC_TRY(dalloc(c, &bits, nwords));
  UFC_TRY(dalloc(c, &flags, 1));
  auto done = [&](int st) {
    dfree(&bits);
    dfree(&flags);
    return st;
  };
  if (cudaMemsetAsync(bits, 0, sizeof(uint32_t) * nwords, c->stream) != cudaSuccess ||
      cudaMemsetAsync(flags, 0, sizeof(int32_t), c->stream) != cudaSuccess)
    return done(cuda_fail(c, cudaGetLastError(), "symmetric codes"));
  k_sym_offsets<<<grid_for(c->N, 256), 256, 0, c->stream>>>(c->N, c->nslices, c->uptr, c->ucol, bits, flags);
  std::vector<uint32_t> h(nwords);
  int32_t hf = 0;
  if (cudaMemcpyAsync(h.data(), bits, sizeof(uint32_t) * nwords, cudaMemcpyDeviceToHost, c->stream) != cudaSuccess ||
      cudaMemcpyAsync(&hf, flags, sizeof(int32_t), cudaMemcpyDeviceToHost, c->stream) != cudaSuccess ||
      cudaStreamSynchronize(c->stream) != cudaSuccess)
    return done(cuda_fail(c, cudaGetLastError(), "symmetric codes"));
  if (hf) return done(UFC_STATUS_OK);  // not stencil-like, or rows too long
  SymOffsets tab{};
  int ntab = 0;
  for (int64_t w = 0; w < nwords; ++w)
    for (int b = 0; b < 32 && h[w] >> b; ++b)
      if ((h[w] >> b) & 1u) {
        if (ntab == kSymCodes) return done(UFC_STATUS_OK);  // too many distinct offsets
        tab.off[ntab++] = (int32_t)(32 * w + b);
      }
  for (int q = ntab; q < 16; ++q) tab.off[q] = 0;
  const int64_t rows = c->nslices * kSlice;
  UFC_TRY(dalloc(c, &c->sym_ucode, rows * 16));
  UFC_TRY(dalloc(c, &c->sym_lcode, rows * 16));
  k_sym_codes<<<grid_for(rows, 256), 256, 0, c->stream>>>(c->N, c->nslices, c->uptr, c->lptr, c->ucol, c->lpos,
                                                           c->lcol, c->s_ublocks, tab, ntab, c->sym_ucode,
                                                           c->sym_lcode, flags);
  if (cudaMemcpyAsync(&hf, flags, sizeof(int32_t), cudaMemcpyDeviceToHost, c->stream) != cudaSuccess ||
      cudaStreamSynchronize(c->stream) != cudaSuccess)
    return done(cuda_fail(c, cudaGetLastError(), "symmetric codes"));
  if (hf) {
    dfree(&c->sym_ucode);
    dfree(&c->sym_lcode);
    return done(UFC_STATUS_OK);
  }
  c->sym_tab = tab;
  c->sym_coded = true;
  return done(UFC_STATUS_OK);
}

// The coded indices of the full storage, when the pattern allows them (else
// full_coded stays false and the products read the 4-byte columns).
int build_full_codes(Ctx* c) {
  c->full_coded = false;
  dfree(&c->full_code);
  const int64_t nwords = 2 * kOffRange / 32;
  uint32_t* bits = nullptr;
  int32_t* flags = nullptr;
  UFC_TRY(dalloc(c, &bits, nwords));
  UFC_TRY(dalloc(c, &flags, 1));
  auto done = [&](int st) {
    dfree(&bits);
    dfree(&flags);
    return st;
  };
  if (cudaMemsetAsync(bits, 0, sizeof(uint32_t) * nwords, c->stream) != cudaSuccess ||
      cudaMemsetAsync(flags, 0, sizeof(int32_t), c->stream) != cudaSuccess)
    return done(cuda_fail(c, cudaGetLastError(), "full codes"));
  k_full_offsets<<<grid_for(c->N, 256), 256, 0, c->stream>>>(c->N, c->nslices, c->slice_ptr, c->sell_col, bits,
                                                             flags);
  std::vector<uint32_t> h(nwords);
  int32_t hf = 0;
  if (cudaMemcpyAsync(h.data(), bits, sizeof(uint32_t) * nwords, cudaMemcpyDeviceToHost, c->stream) != cudaSuccess ||
      cudaMemcpyAsync(&hf, flags, sizeof(int32_t), cudaMemcpyDeviceToHost, c->stream) != cudaSuccess ||
      cudaStreamSynchronize(c->stream) != cudaSuccess)
    return done(cuda_fail(c, cudaGetLastError(), "full codes"));
  if (hf) return done(UFC_STATUS_OK);
  FullOffsets tab{};
  int ntab = 0;
  for (int64_t w = 0; w < nwords; ++w)
    for (int b = 0; b < 32 && h[w] >> b; ++b)
      if ((h[w] >> b) & 1u) {
        if (ntab == kFullCodes) return done(UFC_STATUS_OK);
        tab.off[ntab++] = (int32_t)(32 * w + b - kOffRange);
      }
  const int64_t rows = c->nslices * kSlice;
  UFC_TRY(dalloc(c, &c->full_code, rows * 32));
  k_full_codes<<<grid_for(rows, 256), 256, 0, c->stream>>>(c->N, c->nslices, c->slice_ptr, c->sell_col, tab, ntab,
                                                           c->full_code, flags);
  if (cudaMemcpyAsync(&hf, flags, sizeof(int32_t), cudaMemcpyDeviceToHost, c->stream) != cudaSuccess ||
      cudaStreamSynchronize(c->stream) != cudaSuccess)
    return done(cuda_fail(c, cudaGetLastError(), "full codes"));
  if (hf) {
    dfree(&c->full_code);
    return done(UFC_STATUS_OK);
  }
  c->full_tab = tab;
  c->full_ntab = ntab;
  c->full_coded = true;
  return done(UFC_STATUS_OK);
}

int build_pattern(Ctx* c) {
  if (c->E <= 0 || c->N <= 0) return fail(c, UFC_STATUS_INVALID, "ufc_pattern_build: mesh not set");
  release_graphs(c);
  dfree(&c->uptr); dfree(&c->ucol); dfree(&c->lptr); dfree(&c->lpos); dfree(&c->lcol); dfree(&c->s_lcnt);
  dfree(&c->sval64); dfree(&c->sval32); dfree(&c->sym_ucode); dfree(&c->sym_lcode); dfree(&c->full_code);
  c->full_coded = false;
  c->has_sym_pattern = c->has_sval64 = c->has_sval32 = c->sym_coded = false;
  const int32_t N = c->N, E = c->E;

  // 1. node -> element adjacency on the device
  int32_t *cnt = nullptr, *nptr = nullptr, *fill = nullptr, *nlst = nullptr;
  UFC_TRY(dalloc(c, &cnt, (int64_t)N + 1));
  UFC_TRY(dalloc(c, &nptr, (int64_t)N + 1));
  UFC_TRY(dalloc(c, &fill, N));
  UFC_TRY(dalloc(c, &nlst, 8 * (int64_t)E));
  UFC_CUDA(c, cudaMemsetAsync(cnt, 0, sizeof(int32_t) * ((size_t)N + 1), c->stream));
  UFC_CUDA(c, cudaMemsetAsync(fill, 0, sizeof(int32_t) * N, c->stream));
  UFC_CUDA(c, cudaMemsetAsync(c->dev_err, 0, sizeof(int32_t), c->stream));
  k_count_node_elems<<<grid_for(8 * (int64_t)E, 256), 256, 0, c->stream>>>(E, c->conn, cnt);
  UFC_TRY(scan_exclusive(c, cnt, nptr, (int64_t)N + 1));
  k_fill_node_elems<<<grid_for(8 * (int64_t)E, 256), 256, 0, c->stream>>>(E, c->conn, nptr, fill, nlst);
  k_sort_node_elems<<<grid_for(N, 128), 128, 0, c->stream>>>(N, nptr, nlst, c->dev_err);
  UFC_CUDA(c, cudaGetLastError());
  int st = check_dev_err(c, "ufc_pattern_build (node adjacency)");
  if (st != UFC_STATUS_OK) {
    dfree(&cnt); dfree(&nptr); dfree(&fill); dfree(&nlst);
    return st;
  }

  // 2. colouring (device sweeps) and colour-grouped element lists
  {
    std::vector<int32_t> color;
    st = color_elements_device(c, nptr, nlst, color);
    if (st != UFC_STATUS_OK) {
      dfree(&cnt); dfree(&nptr); dfree(&fill); dfree(&nlst);
      return st;
    }
    c->col_off.assign(c->ncol + 1, 0);
    for (int32_t e = 0; e < E; ++e) c->col_off[color[e] + 1]++;
    for (int k = 0; k < c->ncol; ++k) c->col_off[k + 1] += c->col_off[k];
    std::vector<int32_t> lst(E), pos(c->col_off.begin(), c->col_off.end() - 1);
    for (int32_t e = 0; e < E; ++e) lst[pos[color[e]]++] = e;
    c->h_color = std::move(color);
    st = dalloc(c, &c->col_elems, E);
    if (st == UFC_STATUS_OK) {
      cudaError_t ce =
          cudaMemcpyAsync(c->col_elems, lst.data(), sizeof(int32_t) * E, cudaMemcpyHostToDevice, c->stream);
      if (ce == cudaSuccess) ce = cudaStreamSynchronize(c->stream);
      if (ce != cudaSuccess) st = cuda_fail(c, ce, "ufc_pattern_build (colour lists)");
    }
    if (st != UFC_STATUS_OK) {
      dfree(&cnt); dfree(&nptr); dfree(&fill); dfree(&nlst);
      return st;
    }
  }

  // 3. block rows: count, scan, fill
  UFC_TRY(dalloc(c, &c->brow, (int64_t)N + 1));
  UFC_CUDA(c, cudaMemsetAsync(cnt, 0, sizeof(int32_t) * ((size_t)N + 1), c->stream));
  k_row_count<<<grid_for(N, 128), 128, 0, c->stream>>>(N, c->conn, nptr, nlst, cnt, c->dev_err);
  UFC_TRY(scan_exclusive(c, cnt, c->brow, (int64_t)N + 1));
  st = check_dev_err(c, "ufc_pattern_build (row count)");
  if (st != UFC_STATUS_OK) {
    dfree(&cnt); dfree(&nptr); dfree(&fill); dfree(&nlst);
    return st;
  }
  int32_t nnzb = 0;
  UFC_CUDA(c, cudaMemcpyAsync(&nnzb, c->brow + N, sizeof(int32_t), cudaMemcpyDeviceToHost, c->stream));
  UFC_CUDA(c, cudaStreamSynchronize(c->stream));
  c->nnzb = nnzb;
  UFC_TRY(dalloc(c, &c->bcol, nnzb));
  k_row_fill<<<grid_for(N, 128), 128, 0, c->stream>>>(N, c->conn, nptr, nlst, c->brow, c->bcol);
  UFC_CUDA(c, cudaGetLastError());
  {
    std::vector<int32_t> h(N + 1);
    UFC_CUDA(c, cudaMemcpyAsync(h.data(), c->brow, sizeof(int32_t) * (N + 1), cudaMemcpyDeviceToHost, c->stream));
    UFC_CUDA(c, cudaStreamSynchronize(c->stream));
    int32_t m = 0;
    for (int32_t i = 0; i < N; ++i) m = std::max(m, h[i + 1] - h[i]);
    c->max_row_blocks = m;
  }

  // 4. SELL-32 layout
  c->nslices = (N + kSlice - 1) / kSlice;
  int64_t* slen = nullptr;
  UFC_TRY(dalloc(c, &slen, c->nslices + 1));
  UFC_CUDA(c, cudaMemsetAsync(slen, 0, sizeof(int64_t) * (c->nslices + 1), c->stream));
  k_slice_len<<<grid_for(c->nslices, 256), 256, 0, c->stream>>>(N, c->nslices, c->brow, slen);
  UFC_TRY(dalloc(c, &c->slice_ptr, c->nslices + 1));
  UFC_TRY(scan_exclusive(c, slen, c->slice_ptr, c->nslices + 1));
  UFC_CUDA(c, cudaMemcpyAsync(&c->sell_blocks, c->slice_ptr + c->nslices, sizeof(int64_t), cudaMemcpyDeviceToHost,
                              c->stream));
  UFC_CUDA(c, cudaStreamSynchronize(c->stream));
  dfree(&slen);
  if (c->sell_blocks >= (int64_t)1 << 31)
    return fail(c, UFC_STATUS_UNSUPPORTED, "ufc_pattern_build: more than 2^31 stored blocks");
  UFC_TRY(dalloc(c, &c->sell_col, c->sell_blocks));
  UFC_TRY(dalloc(c, &c->dpos, N));
  k_sell_fill<<<grid_for(c->nslices * kSlice, 128), 128, 0, c->stream>>>(N, c->nslices, c->brow, c->bcol,
                                                                         c->slice_ptr, c->sell_col, c->dpos);
  UFC_TRY(dalloc(c, &c->slot, 64 * (int64_t)E));
  k_slots<<<grid_for(8 * (int64_t)E, 128), 128, 0, c->stream>>>(E, c->conn, c->brow, c->bcol, c->slice_ptr, c->slot,
                                                                c->dev_err);
  UFC_CUDA(c, cudaGetLastError());
  st = check_dev_err(c, "ufc_pattern_build (slots)");
  dfree(&cnt); dfree(&nptr); dfree(&fill); dfree(&nlst);
  if (st != UFC_STATUS_OK) return st;

  // grid reductions keep 4 partial sums per block; the SpMV grid has one
  // thread per (padded) block row
  const int64_t need = 4 * std::max<int64_t>((c->nslices * kSlice + 255) / 256, 65536);
  if (need > c->partials_cap) {
    UFC_TRY(dalloc(c, &c->partials, need));
    c->partials_cap = need;
  }

  // values are (re)allocated on the next assembly
  dfree(&c->val64);
  dfree(&c->val32);
  c->has_val64 = c->has_val32 = false;
  c->has_pattern = true;
  return build_full_codes(c);
}

int export_csr(Ctx* c, const ufc_csr_export_arg* a) {
  if (!c->has_pattern) return fail(c, UFC_STATUS_INVALID, "ufc_csr_export: pattern not built");
  if (a->index_base != 0 && a->index_base != 1) return fail(c, UFC_STATUS_INVALID, "ufc_csr_export: index_base");
  if ((a->values && !c->has_val64 && !c->has_val32) || (a->values32 && !c->has_val32 && !c->has_val64))
    return fail(c, UFC_STATUS_INVALID, "ufc_csr_export: no assembled values");
  const int64_t nnz = 9 * c->nnzb;
  const bool dev = a->mem == UFC_MEM_DEVICE;
  int64_t* rp = a->row_ptr;
  int32_t* col = a->col_ind;
  double* v64 = a->values;
  float* v32 = a->values32;
  int64_t* d_rp = nullptr;
  int32_t* d_col = nullptr;
  double* d_v64 = nullptr;
  float* d_v32 = nullptr;
  if (!dev) {
    if (rp) UFC_TRY(dalloc(c, &d_rp, c->n + 1));
    if (col) UFC_TRY(dalloc(c, &d_col, nnz));
    if (v64) UFC_TRY(dalloc(c, &d_v64, nnz));
    if (v32) UFC_TRY(dalloc(c, &d_v32, nnz));
  } else {
    d_rp = rp; d_col = col; d_v64 = v64; d_v32 = v32;
  }
  const int g = grid_for(c->N, 128);
  // FP64 export reads the FP64 values; FP32 export reads the FP32 values when present.
  if (d_rp || d_col || d_v64) {
    if (c->has_val64 || !d_v64)
      k_export<double><<<g, 128, 0, c->stream>>>(c->N, c->brow, c->bcol, c->slice_ptr, d_v64 ? c->val64 : nullptr,
                                                 a->index_base, d_rp, d_col, d_v64, nullptr);
    else
      k_export<float><<<g, 128, 0, c->stream>>>(c->N, c->brow, c->bcol, c->slice_ptr, c->val32, a->index_base, d_rp,
                                                d_col, d_v64, nullptr);
  }
  if (d_v32) {
    // difference-form FP32 values hold row sums on the diagonal: export the
    // standard form, rounded from FP64, instead
    if (c->has_val32 && !(c->val32_diff && c->has_val64))
      k_export<float><<<g, 128, 0, c->stream>>>(c->N, c->brow, c->bcol, c->slice_ptr, c->val32, a->index_base,
                                                nullptr, nullptr, nullptr, d_v32);
    else
      k_export<double><<<g, 128, 0, c->stream>>>(c->N, c->brow, c->bcol, c->slice_ptr, c->val64, a->index_base,
                                                 nullptr, nullptr, nullptr, d_v32);
  }
  UFC_CUDA(c, cudaGetLastError());
  if (!dev) {
    if (rp) UFC_CUDA(c, cudaMemcpyAsync(rp, d_rp, sizeof(int64_t) * (c->n + 1), cudaMemcpyDeviceToHost, c->stream));
    if (col) UFC_CUDA(c, cudaMemcpyAsync(col, d_col, sizeof(int32_t) * nnz, cudaMemcpyDeviceToHost, c->stream));
    if (v64) UFC_CUDA(c, cudaMemcpyAsync(v64, d_v64, sizeof(double) * nnz, cudaMemcpyDeviceToHost, c->stream));
    if (v32) UFC_CUDA(c, cudaMemcpyAsync(v32, d_v32, sizeof(float) * nnz, cudaMemcpyDeviceToHost, c->stream));
    UFC_CUDA(c, cudaStreamSynchronize(c->stream));
    dfree(&d_rp); dfree(&d_col); dfree(&d_v64); dfree(&d_v32);
  }
  return UFC_STATUS_OK;
}

int build_sym_pattern(Ctx* c) {
  if (!c->has_pattern) return fail(c, UFC_STATUS_INVALID, "symmetric storage: pattern not built");
  if (c->has_sym_pattern) return UFC_STATUS_OK;
  const int32_t N = c->N;
  int32_t* ucnt = nullptr;
  int64_t* len = nullptr;
  UFC_TRY(dalloc(c, &c->s_lcnt, N));
  UFC_TRY(dalloc(c, &ucnt, N));
  UFC_TRY(dalloc(c, &len, c->nslices + 1));
  k_sym_counts<<<grid_for(N, 128), 128, 0, c->stream>>>(N, c->brow, c->bcol, c->s_lcnt, ucnt);
  UFC_CUDA(c, cudaMemsetAsync(len, 0, sizeof(int64_t) * (c->nslices + 1), c->stream));
  k_slice_len_counts<<<grid_for(c->nslices, 256), 256, 0, c->stream>>>(N, c->nslices, ucnt, len);
  UFC_TRY(dalloc(c, &c->uptr, c->nslices + 1));
  UFC_TRY(scan_exclusive(c, len, c->uptr, c->nslices + 1));
  UFC_CUDA(c, cudaMemsetAsync(len, 0, sizeof(int64_t) * (c->nslices + 1), c->stream));
  k_slice_len_counts<<<grid_for(c->nslices, 256), 256, 0, c->stream>>>(N, c->nslices, c->s_lcnt, len);
  UFC_TRY(dalloc(c, &c->lptr, c->nslices + 1));
  UFC_TRY(scan_exclusive(c, len, c->lptr, c->nslices + 1));
  UFC_CUDA(c, cudaGetLastError());
  UFC_CUDA(c, cudaMemcpyAsync(&c->s_ublocks, c->uptr + c->nslices, sizeof(int64_t), cudaMemcpyDeviceToHost,
                              c->stream));
  UFC_CUDA(c, cudaMemcpyAsync(&c->s_lblocks, c->lptr + c->nslices, sizeof(int64_t), cudaMemcpyDeviceToHost,
                              c->stream));
  UFC_CUDA(c, cudaStreamSynchronize(c->stream));
  dfree(&len);
  dfree(&ucnt);
  if (c->s_ublocks + kSlice >= ((int64_t)1 << 31))
    return fail(c, UFC_STATUS_UNSUPPORTED, "symmetric storage: more than 2^31 stored blocks");
  UFC_TRY(dalloc(c, &c->ucol, c->s_ublocks));
  UFC_TRY(dalloc(c, &c->lpos, std::max<int64_t>(c->s_lblocks, 1)));
  UFC_TRY(dalloc(c, &c->lcol, std::max<int64_t>(c->s_lblocks, 1)));
  UFC_CUDA(c, cudaMemsetAsync(c->dev_err, 0, sizeof(int32_t), c->stream));
  k_sym_fill<<<grid_for(c->nslices * kSlice, 128), 128, 0, c->stream>>>(
      N, c->nslices, c->brow, c->bcol, c->s_lcnt, c->uptr, c->lptr, c->s_ublocks, c->ucol, c->lpos, c->lcol,
      c->dev_err);
  UFC_CUDA(c, cudaGetLastError());
  UFC_TRY(check_dev_err(c, "symmetric storage"));
  c->has_sym_pattern = true;
  return build_sym_codes(c);
}

int pack_symmetric(Ctx* c, bool fp64, bool fp32) {
  if (!c->has_val64) return fail(c, UFC_STATUS_INVALID, "symmetric storage: FP64 values not assembled");
  UFC_TRY(build_sym_pattern(c));
  // stored blocks plus one zero slice that padded lower references point at
  const int64_t nv = (c->s_ublocks + kSlice) * 9;
  if (fp64) {
    if (!c->sval64) UFC_TRY(dalloc(c, &c->sval64, nv));
    UFC_CUDA(c, cudaMemsetAsync(c->sval64, 0, sizeof(double) * nv, c->stream));
    k_sym_pack<double><<<grid_for(c->N, 128), 128, 0, c->stream>>>(c->N, c->slice_ptr, c->uptr, c->brow, c->s_lcnt,
                                                                   c->val64, c->sval64);
    UFC_CUDA(c, cudaGetLastError());
    c->has_sval64 = true;
  }
  if (fp32) {
    if (!c->sval32) UFC_TRY(dalloc(c, &c->sval32, nv));
    UFC_CUDA(c, cudaMemsetAsync(c->sval32, 0, sizeof(float) * nv, c->stream));
    k_sym_pack<float><<<grid_for(c->N, 128), 128, 0, c->stream>>>(c->N, c->slice_ptr, c->uptr, c->brow, c->s_lcnt,
                                                                  c->val64, c->sval32);
    UFC_CUDA(c, cudaGetLastError());
    c->has_sval32 = true;
  }
  release_graphs(c);
  return UFC_STATUS_OK;
}

}  // namespace ufc
