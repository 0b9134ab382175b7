// FP64 and INT8 -> INT32 products: the values pass and the dropping of
// entries that cancel to zero, as the reference's legacy scalar kernels do
// (src/kernels/spgemm/legacy/csr_scalar_f64.c:196-262 and
// csr_scalar_i8.c:137-185).
//
// The structure comes from the FP32 path's symbolic pass and column fill (a
// product's columns do not depend on its values).  Then, per row of C, the
// products are added into C's values in the reference's order: A nonzeros
// ascending, each into the entry of its column, the entry starting from zero
// -- FP64: acc = fl(acc + fl(a * b)) (the reference is built with -std=c11,
// so GCC contracts no multiply-add; here __dmul_rn / __dadd_rn); INT8: the
// int32 sum of int32 products, wrapping on overflow.  Last, entries equal to
// zero are removed (the legacy kernels store only acc != 0; -0.0 compares
// equal to zero and goes too), row by row in column order.
#include <cuda_runtime.h>

#include <climits>

#include "device_common.cuh"
#include "kernels.cuh"
#include "rvsp_cuda.h"

namespace rvsp {

namespace {

constexpr int kTypedWarps = 8;       // warps per block, one row each
constexpr int kTypedCache = 1024;    // C row columns kept in shared memory per warp
constexpr int kFlatThreads = 256;

__device__ __forceinline__ double typed_term(double acc, double a, double b) {
  return __dadd_rn(acc, __dmul_rn(a, b));
}

__device__ __forceinline__ int32_t typed_term(int32_t acc, int8_t a, int8_t b) {
  const int32_t p = static_cast<int32_t>(a) * static_cast<int32_t>(b);  // |p| <= 16384
  return static_cast<int32_t>(static_cast<uint32_t>(acc) + static_cast<uint32_t>(p));
}

// Position of col in the sorted columns cols[0..m) (present by construction).
__device__ __forceinline__ int32_t find_col(const int32_t *cols, int32_t m, int32_t col) {
  int32_t lo = 0, hi = m;
  while (lo < hi) {
    const int32_t mid = (lo + hi) >> 1;
    if (cols[mid] < col) lo = mid + 1;
    else hi = mid;
  }
  return lo;
}

// Warp per row of C; c_val zeroed by the caller.  One A nonzero at a time,
// lanes over its B row: the columns of one B row are distinct, so no two
// lanes of a step touch the same entry, and __syncwarp orders the steps.
template <typename V, typename T>
__global__ void __launch_bounds__(kTypedWarps * 32)
typed_numeric_kernel(int32_t rows, const int32_t *__restrict__ a_rp,
                     const int32_t *__restrict__ a_col, const V *__restrict__ a_val,
                     const int32_t *__restrict__ b_rp, const int32_t *__restrict__ b_col,
                     const V *__restrict__ b_val, const int32_t *__restrict__ c_rp,
                     const int32_t *__restrict__ c_col, T *__restrict__ c_val) {
  __shared__ int32_t s_cols[kTypedWarps][kTypedCache];
  const int wb = threadIdx.x >> 5;
  const int lane = lane_id();
  const int64_t stride = (int64_t(gridDim.x) * blockDim.x) >> 5;
  for (int64_t w = (int64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5; w < rows;
       w += stride) {
    const int32_t row = static_cast<int32_t>(w);
    const int32_t cs = c_rp[row], m = c_rp[row + 1] - cs;
    if (m == 0) continue;
    const int32_t *cols = c_col + cs;
    if (m <= kTypedCache) {
      for (int32_t q = lane; q < m; q += 32) s_cols[wb][q] = cols[q];
      __syncwarp();
      cols = s_cols[wb];
    }
    T *acc = c_val + cs;
    for (int32_t p = a_rp[row]; p < a_rp[row + 1]; ++p) {
      const int32_t k = a_col[p];
      const V a = a_val[p];
      const int32_t b1 = b_rp[k + 1];
      for (int32_t e = b_rp[k] + lane; e < b1; e += 32) {
        const int32_t q = find_col(cols, m, b_col[e]);
        acc[q] = typed_term(acc[q], a, b_val[e]);
      }
      __syncwarp();
    }
    __syncwarp();  // s_cols is rewritten by the warp's next row
  }
}

template <typename T>
__global__ void __launch_bounds__(kFlatThreads)
nonzero_flags_kernel(int64_t n, const T *__restrict__ v, int32_t *__restrict__ keep) {
  const int64_t stride = int64_t(gridDim.x) * blockDim.x;
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride)
    keep[i] = v[i] != T(0) ? 1 : 0;
}

template <typename T>
__global__ void __launch_bounds__(kFlatThreads)
compact_nonzero_kernel(int64_t n, const int32_t *__restrict__ keep,
                       const int64_t *__restrict__ off, const int32_t *__restrict__ col,
                       const T *__restrict__ v, int32_t *__restrict__ out_col,
                       T *__restrict__ out_val) {
  const int64_t stride = int64_t(gridDim.x) * blockDim.x;
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride) {
    if (!keep[i]) continue;
    out_col[off[i]] = col[i];
    out_val[off[i]] = v[i];
  }
}

// out_rp[r] = kept entries before row r's first entry.
__global__ void __launch_bounds__(kFlatThreads)
kept_row_ptr_kernel(int32_t rows, const int32_t *__restrict__ c_rp,
                    const int64_t *__restrict__ off, int64_t n, int64_t total,
                    int32_t *__restrict__ out_rp) {
  const int64_t r = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (r > rows) return;
  const int64_t p = c_rp[r];
  out_rp[r] = static_cast<int32_t>(p < n ? off[p] : total);
}

int flat_grid(int64_t n) {
  int64_t g = (n + kFlatThreads - 1) / kFlatThreads;
  if (g < 1) g = 1;
  if (g > 148 * 32) g = 148 * 32;
  return static_cast<int>(g);
}

rvsp_status_t typed_status(cudaError_t e) {
  if (e == cudaSuccess) return RVSP_SUCCESS;
  return e == cudaErrorMemoryAllocation ? RVSP_ERROR_ALLOCATION_FAILED : RVSP_ERROR_DEVICE;
}

size_t align256(size_t b) { return (b + 255) & ~size_t(255); }

// Scratch layout: keep int32[n] | off int64[n] | scan partials | total int64.
size_t drop_scratch_bytes(int64_t n) {
  const size_t nb = size_t(n > 0 ? n : 1);
  return align256(nb * sizeof(int32_t)) + align256(nb * sizeof(int64_t)) +
         align256(scan_partials_bytes(static_cast<int32_t>(n > 0 ? n : 1))) +
         align256(sizeof(int64_t));
}

template <typename T>
rvsp_status_t drop_zeros(cudaStream_t s, int32_t rows, const int32_t *c_rp, int64_t n,
                         const int32_t *c_col, const T *c_val, char *scratch,
                         int32_t *out_rp, int32_t *out_col, T *out_val, int32_t *out_nnz) {
  const size_t nb = size_t(n > 0 ? n : 1);
  int32_t *keep = reinterpret_cast<int32_t *>(scratch);
  char *p = scratch + align256(nb * sizeof(int32_t));
  int64_t *off = reinterpret_cast<int64_t *>(p);
  p += align256(nb * sizeof(int64_t));
  int64_t *partials = reinterpret_cast<int64_t *>(p);
  p += align256(scan_partials_bytes(static_cast<int32_t>(n > 0 ? n : 1)));
  int64_t *total = reinterpret_cast<int64_t *>(p);
  int64_t kept = 0;
  cudaMemsetAsync(total, 0, sizeof(int64_t), s);
  if (n > 0) {
    nonzero_flags_kernel<T><<<flat_grid(n), kFlatThreads, 0, s>>>(n, c_val, keep);
    launch_scan_i64(static_cast<int32_t>(n), keep, off, partials, total, s);
  }
  cudaError_t e = cudaMemcpyAsync(&kept, total, sizeof(int64_t), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e == cudaSuccess) {
    kept_row_ptr_kernel<<<static_cast<unsigned>((int64_t(rows) + kFlatThreads) / kFlatThreads),
                          kFlatThreads, 0, s>>>(rows, c_rp, off, n, kept, out_rp);
    if (n > 0)
      compact_nonzero_kernel<T><<<flat_grid(n), kFlatThreads, 0, s>>>(
          n, keep, off, c_col, c_val, out_col, out_val);
    e = cudaGetLastError();
  }
  if (e != cudaSuccess) return typed_status(e);
  *out_nnz = static_cast<int32_t>(kept);
  return RVSP_SUCCESS;
}

}  // namespace

}  // namespace rvsp

using namespace rvsp;

extern "C" rvsp_status_t rvsp_cuda_typed_numeric(void *stream, int32_t in_dtype,
                                                 int32_t a_rows, const int32_t *a_row_ptr,
                                                 const int32_t *a_col_idx, const void *a_values,
                                                 const int32_t *b_row_ptr,
                                                 const int32_t *b_col_idx, const void *b_values,
                                                 const int32_t *c_row_ptr,
                                                 const int32_t *c_col_idx, void *c_values) {
  if (!a_row_ptr || !a_col_idx || !a_values || !b_row_ptr || !b_col_idx || !b_values ||
      !c_row_ptr || !c_col_idx || !c_values)
    return RVSP_ERROR_NULL_POINTER;
  if (a_rows < 0) return RVSP_ERROR_INVALID_ARGUMENT;
  if (a_rows == 0) return RVSP_SUCCESS;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  int64_t grid = (int64_t(a_rows) + kTypedWarps - 1) / kTypedWarps;
  if (grid > 148 * 64) grid = 148 * 64;
  if (in_dtype == RVSP_DTYPE_FP64) {
    typed_numeric_kernel<double, double><<<static_cast<unsigned>(grid), kTypedWarps * 32, 0, s>>>(
        a_rows, a_row_ptr, a_col_idx, static_cast<const double *>(a_values), b_row_ptr,
        b_col_idx, static_cast<const double *>(b_values), c_row_ptr, c_col_idx,
        static_cast<double *>(c_values));
  } else if (in_dtype == RVSP_DTYPE_INT8) {
    typed_numeric_kernel<int8_t, int32_t>
        <<<static_cast<unsigned>(grid), kTypedWarps * 32, 0, s>>>(
            a_rows, a_row_ptr, a_col_idx, static_cast<const int8_t *>(a_values), b_row_ptr,
            b_col_idx, static_cast<const int8_t *>(b_values), c_row_ptr, c_col_idx,
            static_cast<int32_t *>(c_values));
  } else {
    return RVSP_ERROR_UNSUPPORTED_DTYPE;
  }
  return typed_status(cudaGetLastError());
}

extern "C" size_t rvsp_cuda_drop_zeros_scratch_bytes(int64_t nnz) {
  return drop_scratch_bytes(nnz);
}

extern "C" rvsp_status_t rvsp_cuda_drop_zeros(void *stream, int32_t out_dtype, int32_t rows,
                                              const int32_t *c_row_ptr, int64_t nnz,
                                              const int32_t *c_col_idx, const void *c_values,
                                              void *scratch, size_t scratch_bytes,
                                              int32_t *out_row_ptr, int32_t *out_col_idx,
                                              void *out_values, int32_t *out_nnz) {
  if (!c_row_ptr || !c_col_idx || !c_values || !out_row_ptr || !out_col_idx || !out_values ||
      !out_nnz || !scratch)
    return RVSP_ERROR_NULL_POINTER;
  if (rows < 0 || nnz < 0 || nnz > int64_t(INT32_MAX)) return RVSP_ERROR_INVALID_ARGUMENT;
  if (scratch_bytes < drop_scratch_bytes(nnz)) return RVSP_ERROR_INVALID_ARGUMENT;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  char *sc = static_cast<char *>(scratch);
  if (out_dtype == RVSP_DTYPE_FP64)
    return drop_zeros<double>(s, rows, c_row_ptr, nnz, c_col_idx,
                              static_cast<const double *>(c_values), sc, out_row_ptr,
                              out_col_idx, static_cast<double *>(out_values), out_nnz);
  if (out_dtype == RVSP_DTYPE_INT32)
    return drop_zeros<int32_t>(s, rows, c_row_ptr, nnz, c_col_idx,
                               static_cast<const int32_t *>(c_values), sc, out_row_ptr,
                               out_col_idx, static_cast<int32_t *>(out_values), out_nnz);
  return RVSP_ERROR_UNSUPPORTED_DTYPE;
}
