// ufc_csr_spmv_dot_noalloc: y = A x and x.y on a caller-owned CSR matrix,
// for callers that cannot allocate device memory.
//
// Who needs it: host codes that own every device buffer themselves and may not
// allocate on their hot path -- a Fortran or C solver whose device memory all
// comes from its own fixed pool (its allocator must not be bypassed, and its
// budget is fixed when the run starts), or code running where a call to
// cudaMalloc would synchronise the device and stall work the caller keeps in
// flight.  They pass the matrix and vectors; the only scratch the kernel needs,
// the per-block partial sums of the dot product and the counter that elects
// the block finishing the reduction, lives in a file-scope static device array
// instead of an allocation.
//
// Limits and behaviour:
//  * at most UFC_NOALLOC_MAX_ROWS rows (one thread per row, 256 rows per block,
//    one partial sum per block in the static array); larger calls are rejected
//    with UFC_STATUS_INVALID;
//  * every GPU that loads this library holds the array (about 512 KiB) until the
//    process exits;
//  * the first call on a device looks up the array's device address with
//    cudaGetSymbolAddress (the host-side name of the array is not a device
//    address) and keeps it for that device; make that first call before any
//    stream capture.  A cudaDeviceReset of the device invalidates the kept
//    address, so the entry point must not be used on a device after resetting
//    it in the same process;
//  * the stream must belong to the current device (checked: UFC_STATUS_INVALID
//    otherwise);
//  * all calls share the array, and each call clears the counter it needs at
//    zero: calls that overlap on the GPU (on different streams, or from several
//    threads) race on the array and must be serialised by the caller.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <mutex>

#include "reduce.cuh"
#include "ufc_internal.cuh"

namespace {

constexpr int kRowsPerBlock = 256;
constexpr int64_t kMaxBlocks = UFC_NOALLOC_MAX_ROWS / kRowsPerBlock;
constexpr int kMaxDevices = 64;

struct NoAllocScratch {
  double partials[kMaxBlocks];  // one partial dot product per block
  uint32_t ticket;              // blocks finished; must be 0 when a call starts
};

static __device__ __align__(256) NoAllocScratch g_scratch;

std::mutex g_mutex;
NoAllocScratch* g_scratch_ptr[kMaxDevices] = {};

__global__ void __launch_bounds__(kRowsPerBlock)
    k_csr_spmv_dot(int64_t n, const int64_t* __restrict__ rp, const int32_t* __restrict__ col,
                   const double* __restrict__ val, const double* __restrict__ x, double* __restrict__ y,
                   NoAllocScratch* __restrict__ s, double* __restrict__ xy) {
  const int64_t row = (int64_t)blockIdx.x * kRowsPerBlock + threadIdx.x;
  double dot[1] = {0.0};
  if (row < n) {
    double acc = 0.0;
    for (int64_t k = rp[row]; k < rp[row + 1]; ++k) acc += val[k] * x[col[k]];
    y[row] = acc;
    dot[0] = x[row] * acc;
  }
  double tot[1];
  if (ufc::grid_sum<1>(dot, s->partials, &s->ticket, tot)) *xy = tot[0];
}

int set_error(char* buf, int32_t len, const char* msg, int status) {
  if (buf && len > 0) {
    const size_t k = std::min<size_t>(std::strlen(msg), (size_t)len - 1);
    std::memcpy(buf, msg, k);
    buf[k] = 0;
  }
  return status;
}

}  // namespace

extern "C" int ufc_csr_spmv_dot_noalloc(int64_t n_rows, const int64_t* row_ptr, const int32_t* col_ind,
                                        const double* values, const double* x, double* y, double* xy,
                                        void* cuda_stream, char* errbuf, int32_t errlen) {
  if (n_rows <= 0 || !row_ptr || !col_ind || !values || !x || !y || !xy)
    return set_error(errbuf, errlen, "ufc_csr_spmv_dot_noalloc: n_rows <= 0 or NULL pointer", UFC_STATUS_INVALID);
  if (n_rows > UFC_NOALLOC_MAX_ROWS)
    return set_error(errbuf, errlen,
                     "ufc_csr_spmv_dot_noalloc: n_rows exceeds UFC_NOALLOC_MAX_ROWS (16777216), the size of "
                     "the static reduction scratch",
                     UFC_STATUS_INVALID);
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices)
    return set_error(errbuf, errlen, "ufc_csr_spmv_dot_noalloc: no usable current device", UFC_STATUS_ERROR);
  NoAllocScratch* s = nullptr;
  {
    std::lock_guard<std::mutex> lock(g_mutex);
    if (!g_scratch_ptr[dev]) {
      // once per device, with that device current: the host-side name of the
      // array is not a device address; look the address up
      void* p = nullptr;
      const cudaError_t e = cudaGetSymbolAddress(&p, g_scratch);
      if (e != cudaSuccess || !p)
        return set_error(errbuf, errlen, "ufc_csr_spmv_dot_noalloc: cudaGetSymbolAddress failed", UFC_STATUS_ERROR);
      g_scratch_ptr[dev] = static_cast<NoAllocScratch*>(p);
    }
    s = g_scratch_ptr[dev];
  }
  cudaStream_t st = (cudaStream_t)cuda_stream;
  int stream_dev = dev;
  if (cudaStreamGetDevice(st, &stream_dev) != cudaSuccess)
    return set_error(errbuf, errlen, "ufc_csr_spmv_dot_noalloc: invalid stream", UFC_STATUS_INVALID);
  if (stream_dev != dev)
    return set_error(errbuf, errlen,
                     "ufc_csr_spmv_dot_noalloc: the stream belongs to another device than the current one",
                     UFC_STATUS_INVALID);
  // the election counter must start at zero whatever the last call left there
  if (cudaMemsetAsync(&s->ticket, 0, sizeof(uint32_t), st) != cudaSuccess)
    return set_error(errbuf, errlen, "ufc_csr_spmv_dot_noalloc: cudaMemsetAsync failed", UFC_STATUS_ERROR);
  const int64_t grid = (n_rows + kRowsPerBlock - 1) / kRowsPerBlock;
  k_csr_spmv_dot<<<(unsigned)grid, kRowsPerBlock, 0, st>>>(n_rows, row_ptr, col_ind, values, x, y, s, xy);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return set_error(errbuf, errlen, cudaGetErrorString(e), UFC_STATUS_ERROR);
  return set_error(errbuf, errlen, "", UFC_STATUS_OK);
}
