// rvsp_cuda_numeric_noalloc: the numeric pass for callers that cannot
// allocate device memory.
//
// Who needs it.  Some callers may not call cudaMalloc at the moment they want
// values computed: memory pools and allocators that forbid re-entrant
// allocation from inside their own callbacks, and real-time loops that must
// not take the driver's allocation locks.  Every other numeric entry point
// here needs a caller-provided device workspace for its dense accumulators;
// this one needs none.
//
// How.  The dense accumulators live in one file-scope device array of
// kScratchBytes (16 MiB), which every GPU that loads the library keeps until
// the process exits.  Host code cannot use the array's name as a device
// address, so the first call on each device (with that device current) looks
// the address up with cudaGetSymbolAddress and caches it; make that first
// call before any stream capture begins.  Each call then
// clears the part of the array it uses (cudaMemsetAsync, no allocation) and
// launches one kernel.  All calls share the array: calls whose kernels
// overlap on the GPU (other streams, other host threads) race and must be
// serialised by the caller.
//
// What it computes.  C's values for a structure (c_row_ptr, c_col_idx)
// already produced by the symbolic pass for this sparsity pattern, with the
// same arithmetic as every other path: per row, one A nonzero at a time in
// ascending order, each B row's entries spread over the block's threads
// (distinct columns), acc = fl(acc + fl(a * b)) from +0.0f.  The values are
// bit-identical to rvsp_cuda_numeric's.
#include <cuda_runtime.h>

#include <mutex>

#include "device_common.cuh"
#include "kernels.cuh"
#include "rvsp_cuda.h"

namespace {

constexpr size_t kScratchBytes = RVSP_NOALLOC_SCRATCH_BYTES;
constexpr size_t kScratchFloats = kScratchBytes / sizeof(float);
constexpr int kThreads = 256;
constexpr int kStage = 256;
constexpr int kMaxDevices = 64;

}  // namespace

// The scratch: per block, a dense float accumulator over B's columns.
static __device__ __align__(256) float rvsp_noalloc_scratch[kScratchFloats];

namespace {

std::mutex g_mutex;
float *g_scratch[kMaxDevices] = {};
int g_sms[kMaxDevices] = {};

rvsp_status_t scratch_of_current_device(float **ptr, int *sms) {
  int dev = -1;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
    cudaGetLastError();
    return RVSP_ERROR_UNSUPPORTED_BACKEND;
  }
  std::lock_guard<std::mutex> lock(g_mutex);
  if (!g_scratch[dev]) {
    int major = 0, minor = 0, count = 0;
    cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev);
    cudaDeviceGetAttribute(&minor, cudaDevAttrComputeCapabilityMinor, dev);
    cudaDeviceGetAttribute(&count, cudaDevAttrMultiProcessorCount, dev);
    if (major != 10 || minor != 0) return RVSP_ERROR_UNSUPPORTED_BACKEND;
    void *p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, rvsp_noalloc_scratch);
    if (e != cudaSuccess || p == nullptr) {
      cudaGetLastError();
      return e == cudaErrorMemoryAllocation ? RVSP_ERROR_ALLOCATION_FAILED
                                            : RVSP_ERROR_DEVICE;
    }
    g_scratch[dev] = static_cast<float *>(p);
    g_sms[dev] = count > 0 ? count : 148;
  }
  *ptr = g_scratch[dev];
  *sms = g_sms[dev];
  return RVSP_SUCCESS;
}

// One block per row (grid-stride).  Column indices are range-checked (A's
// against b_rows, B's and C's against b_cols) and an out-of-range one is
// skipped; row pointers are not checked, so the operands must be canonical
// CSR (as rvsp_cuda_csr_check accepts).  After each row the block zeroes
// every accumulator its B rows touched, so a C structure that misses a
// column of the product leaves only that entry wrong.
__global__ void __launch_bounds__(kThreads)
noalloc_numeric_kernel(rvsp::Operands op, int32_t b_rows,
                       const int32_t *__restrict__ c_rp,
                       const int32_t *__restrict__ c_col,
                       float *__restrict__ c_val, float *__restrict__ scratch,
                       size_t stride) {
  __shared__ int32_t s_bbeg[kStage];
  __shared__ int32_t s_len[kStage];
  __shared__ float s_a[kStage];
  float *acc = scratch + stride * blockIdx.x;
  for (int32_t row = blockIdx.x; row < op.a_rows; row += gridDim.x) {
    const int32_t p0 = op.a_rp[row], p1 = op.a_rp[row + 1];
    for (int32_t p = p0; p < p1; p += kStage) {
      const int cnt = min(kStage, p1 - p);
      __syncthreads();
      for (int q = threadIdx.x; q < cnt; q += blockDim.x) {
        const int32_t k = __ldg(op.a_col + p + q);
        const bool ok = static_cast<uint32_t>(k) < static_cast<uint32_t>(b_rows);
        const int32_t b0 = ok ? __ldg(op.b_rp + k) : 0;
        s_bbeg[q] = b0;
        s_len[q] = ok ? __ldg(op.b_rp + k + 1) - b0 : 0;
        s_a[q] = __ldg(op.a_val + p + q);
      }
      __syncthreads();
      for (int q = 0; q < cnt; ++q) {
        const int32_t bbeg = s_bbeg[q], len = s_len[q];
        const float a = s_a[q];
        for (int32_t e = threadIdx.x; e < len; e += blockDim.x) {
          const int32_t col = __ldg(op.b_col + bbeg + e);
          if (static_cast<uint32_t>(col) < static_cast<uint32_t>(op.b_cols))
            acc[col] = __fadd_rn(acc[col], __fmul_rn(a, __ldg(op.b_val + bbeg + e)));
        }
        __syncthreads();
      }
    }
    // Drain in C's column order.
    for (int32_t e = c_rp[row] + threadIdx.x; e < c_rp[row + 1]; e += blockDim.x) {
      const int32_t col = __ldg(c_col + e);
      c_val[e] = static_cast<uint32_t>(col) < static_cast<uint32_t>(op.b_cols) ? acc[col]
                                                                            : 0.0f;
    }
    __syncthreads();
    // Leave the accumulator zeroed at every column this row touched.
    for (int32_t p = p0; p < p1; ++p) {
      const int32_t k = __ldg(op.a_col + p);
      if (static_cast<uint32_t>(k) >= static_cast<uint32_t>(b_rows)) continue;
      const int32_t bbeg = __ldg(op.b_rp + k), len = __ldg(op.b_rp + k + 1) - bbeg;
      for (int32_t e = threadIdx.x; e < len; e += blockDim.x) {
        const int32_t col = __ldg(op.b_col + bbeg + e);
        if (static_cast<uint32_t>(col) < static_cast<uint32_t>(op.b_cols)) acc[col] = 0.0f;
      }
    }
    __syncthreads();
  }
}

}  // namespace

extern "C" rvsp_status_t rvsp_cuda_numeric_noalloc(
    void *stream, int32_t a_rows, int32_t b_rows, int32_t b_cols,
    const int32_t *a_row_ptr, const int32_t *a_col_idx, const float *a_values,
    const int32_t *b_row_ptr, const int32_t *b_col_idx, const float *b_values,
    const int32_t *c_row_ptr, const int32_t *c_col_idx, float *c_values) {
  if (!a_row_ptr || !a_col_idx || !a_values || !b_row_ptr || !b_col_idx ||
      !b_values || !c_row_ptr || !c_col_idx || !c_values)
    return RVSP_ERROR_NULL_POINTER;
  if (a_rows < 0 || b_rows < 0 || b_cols < 0) return RVSP_ERROR_INVALID_ARGUMENT;
  // An empty product (no rows of A, or no columns of B) has no values.
  if (a_rows == 0 || b_cols == 0) return RVSP_SUCCESS;
  // One accumulator of b_cols floats must fit the fixed scratch.
  if (static_cast<size_t>(b_cols) > RVSP_NOALLOC_MAX_B_COLS)
    return RVSP_ERROR_INVALID_ARGUMENT;
  float *scratch = nullptr;
  int sms = 0;
  rvsp_status_t st = scratch_of_current_device(&scratch, &sms);
  if (st != RVSP_SUCCESS) return st;

  const size_t stride = (static_cast<size_t>(b_cols) + 63) & ~size_t(63);
  size_t slots = kScratchFloats / stride;
  if (slots > static_cast<size_t>(sms)) slots = static_cast<size_t>(sms);
  if (slots > static_cast<size_t>(a_rows)) slots = static_cast<size_t>(a_rows);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  // The array keeps the previous call's contents: clear what this call uses.
  cudaError_t e = cudaMemsetAsync(scratch, 0, slots * stride * sizeof(float), s);
  if (e != cudaSuccess) return RVSP_ERROR_DEVICE;
  const rvsp::Operands op{a_rows, b_cols, a_row_ptr, a_col_idx, a_values,
                          b_row_ptr, b_col_idx, b_values};
  noalloc_numeric_kernel<<<static_cast<int>(slots), kThreads, 0, s>>>(
      op, b_rows, c_row_ptr, c_col_idx, c_values, scratch, stride);
  e = cudaGetLastError();
  return e == cudaSuccess ? RVSP_SUCCESS : RVSP_ERROR_DEVICE;
}
