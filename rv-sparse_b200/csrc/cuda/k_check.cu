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

__global__ void __launch_bounds__(kThreads)
csr_check_kernel(int32_t rows, int32_t cols, const int32_t *__restrict__ row_ptr,
                 const int32_t *__restrict__ col_idx, int32_t nnz,
                 unsigned long long *__restrict__ result) {
  const int32_t r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r == 0 && row_ptr[0] != 0) atomicMin(result, pack(-1, kBadRowPtr));
  if (r >= rows) return;
  const int32_t lo = row_ptr[r], hi = row_ptr[r + 1];
  int code = 0;
  if (hi < lo || lo < 0 || hi > nnz) {
    code = kBadRowPtr;
  } else {
    int32_t last = -1;
    for (int32_t p = lo; p < hi; ++p) {
      const int32_t c = col_idx[p];
      if (c < 0 || c >= cols) { code = kColRange; break; }
      if (c == last) { code = kDuplicate; break; }
      if (c < last) { code = kUnsorted; break; }
      last = c;
    }
  }
  if (code) atomicMin(result, pack(r, code));
}

}  // namespace

void launch_csr_check(int32_t rows, int32_t cols, const int32_t *row_ptr,
                      const int32_t *col_idx, int32_t nnz,
                      unsigned long long *result, cudaStream_t s) {
  const int grid = rows > 0 ? (rows + kThreads - 1) / kThreads : 1;
  csr_check_kernel<<<grid, kThreads, 0, s>>>(rows, cols, row_ptr, col_idx, nnz,
                                             result);
}

}  // namespace rvsp
