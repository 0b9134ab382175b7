// Device canonical-CSR check, the GPU form of rvsp_csr_check
// (rvsp_support.c:37-126): row_ptr[0] == 0 and non-decreasing, columns in
// range, strictly ascending within a row.  The reference reports the first
// offending row in row order with the first violation in that row; every
// thread checks one row sequentially and the minimum packed (row, code) wins,
// which reproduces that choice exactly.
//
// One addition keeps the check itself in bounds: a row pointer outside
// [0, nnz] is reported as a malformed row pointer before any column of that
// row is read (the reference would read past the array there).
#include <climits>

#include "device_common.cuh"
#include "kernels.cuh"

namespace rvsp {

namespace {

constexpr int kThreads = 256;
constexpr int kBadRowPtr = 1, kColRange = 2, kUnsorted = 3, kDuplicate = 4;

__device__ __forceinline__ unsigned long long pack(int32_t row, int code) {
  // row -1 (whole-matrix problem) sorts before row 0.
  return (static_cast<unsigned long long>(static_cast<uint32_t>(row + 1)) << 8) |
         static_cast<unsigned>(code);
}

// Rows longer than this are checked by a warp each (long_row_check_kernel);
// one thread walking a power-law hub row of tens of thousands of entries
// would hold up the whole check.
constexpr int32_t kCheckLongRow = 256;

// Violation code of column c at a position whose predecessor in the row is
// last (-1 at the row's start), 0 if none.
__device__ __forceinline__ int col_code(int32_t c, int32_t last, int32_t cols) {
  if (c < 0 || c >= cols) return kColRange;
  if (c == last) return kDuplicate;
  if (c < last) return kUnsorted;
  return 0;
}

__global__ void __launch_bounds__(kThreads)
csr_check_kernel(int32_t rows, int32_t cols, const int32_t *__restrict__ row_ptr,
                 const int32_t *__restrict__ col_idx, int32_t nnz,
                 unsigned long long *__restrict__ result, int32_t *__restrict__ long_rows,
                 int32_t long_cap) {
  const int32_t r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r == 0 && row_ptr[0] != 0) atomicMin(result, pack(-1, kBadRowPtr));
  if (r >= rows) return;
  const int32_t lo = row_ptr[r], hi = row_ptr[r + 1];
  int code = 0;
  if (hi < lo || lo < 0 || hi > nnz) {
    code = kBadRowPtr;
  } else if (hi - lo > kCheckLongRow) {
    // rows of more than kCheckLongRow entries (at most nnz / 257 of them)
    const int32_t at = atomicAdd(long_rows, 1);
    if (at < long_cap) long_rows[1 + at] = r;
  } else {
    int32_t last = -1;
    for (int32_t p = lo; p < hi && !code; ++p) {
      const int32_t c = col_idx[p];
      code = col_code(c, last, cols);
      last = c;
    }
  }
  if (code) atomicMin(result, pack(r, code));
}

// One warp per listed long row: 32 columns at a time, each compared with its
// predecessor; the lowest violating position of the first chunk that has one
// is the row's first violation.
__global__ void __launch_bounds__(kThreads)
long_row_check_kernel(int32_t cols, const int32_t *__restrict__ row_ptr,
                      const int32_t *__restrict__ col_idx,
                      unsigned long long *__restrict__ result,
                      const int32_t *__restrict__ long_rows, int32_t long_cap) {
  const int lane = lane_id();
  const int32_t warps = (gridDim.x * blockDim.x) >> 5;
  const int32_t n = min(long_rows[0], long_cap);
  for (int32_t i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < n; i += warps) {
    const int32_t r = long_rows[1 + i];
    const int32_t lo = row_ptr[r], hi = row_ptr[r + 1];
    int32_t prev_last = -1;
    for (int32_t p0 = lo; p0 < hi; p0 += 32) {
      const int32_t p = p0 + lane;
      const int32_t c = p < hi ? col_idx[p] : INT32_MAX;
      int32_t last = __shfl_up_sync(kFull, c, 1);
      if (lane == 0) last = prev_last;
      const int code = p < hi ? col_code(c, last, cols) : 0;
      const unsigned bad = __ballot_sync(kFull, code != 0);
      if (bad) {
        const int first = __ffs(bad) - 1;
        if (lane == first) atomicMin(result, pack(r, code));
        break;  // uniform
      }
      prev_last = __shfl_sync(kFull, c, 31);
    }
  }
}

}  // namespace

int32_t check_long_rows_cap(int32_t rows, int32_t nnz) {
  const int32_t by_nnz = nnz / (kCheckLongRow + 1) + 1;
  return rows < by_nnz ? rows : by_nnz;
}

void launch_csr_check(int32_t rows, int32_t cols, const int32_t *row_ptr,
                      const int32_t *col_idx, int32_t nnz,
                      unsigned long long *result, int32_t *long_rows,
                      cudaStream_t s) {
  const int32_t cap = check_long_rows_cap(rows, nnz);
  const int grid = rows > 0 ? (rows + kThreads - 1) / kThreads : 1;
  csr_check_kernel<<<grid, kThreads, 0, s>>>(rows, cols, row_ptr, col_idx, nnz, result,
                                             long_rows, cap);
  if (rows > 0 && nnz > kCheckLongRow) {
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    long_row_check_kernel<<<sms * 2, kThreads, 0, s>>>(cols, row_ptr, col_idx, result,
                                                       long_rows, cap);
  }
}

}  // namespace rvsp
