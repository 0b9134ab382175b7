// Per-row statistics and row binning.
//
// ops_i = sum over A row i of |B row k| is the op count the reference
// records per row (rvsp_symbolic.c:41 with op_counts_out at :61-64, exposed by
// rvsp_spgemm_get_op_counts, spgemm_descr.c:357-380).  It is also the upper
// bound on row i's output nnz that sizes the symbolic pass.
#include "device_common.cuh"
#include "kernels.cuh"

namespace rvsp {

namespace {

constexpr int kThreads = 256;

// Adds one to class_count[c] for every lane with take, one atomic per class
// per warp.
// A row's entry range, cut to [0, a_nnz] when the bound is known.
__device__ __forceinline__ void row_range(const Operands &op, int32_t i, int32_t &p0,
                                          int32_t &p1) {
  p0 = op.a_rp[i];
  p1 = op.a_rp[i + 1];
  if (op.a_nnz >= 0) {
    p0 = min(max(p0, 0), op.a_nnz);
    p1 = min(max(p1, p0), op.a_nnz);
  }
}

// |B row k|, or 0 for a k outside B when B's row count is known.
__device__ __forceinline__ int32_t b_len(const Operands &op, int32_t k) {
  if (op.b_rows >= 0 && (k < 0 || k >= op.b_rows)) return 0;
  return __ldg(op.b_rp + k + 1) - __ldg(op.b_rp + k);
}

__device__ __forceinline__ void count_class(int32_t *s_cnt, bool take, int c) {
  const unsigned peers = __match_any_sync(kFull, take ? c : (-1 - lane_id()));
  if (take && (peers & lanemask_lt()) == 0) atomicAdd(&s_cnt[c], __popc(peers));
}

__global__ void __launch_bounds__(kThreads)
rowstats_kernel(Operands op, int64_t *__restrict__ ops, uint8_t *__restrict__ cls,
                int32_t *__restrict__ counts, int32_t *__restrict__ class_count,
                int32_t *__restrict__ long_rows, int32_t *__restrict__ long_count,
                int32_t max_long) {
  __shared__ int32_t s_cnt[kNumClasses];
  for (int c = threadIdx.x; c < kNumClasses; c += blockDim.x) s_cnt[c] = 0;
  __syncthreads();

  const int32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  bool take = false;
  int c = kEmpty_;
  if (i < op.a_rows) {
    int32_t p0, p1;
    row_range(op, i, p0, p1);
    if (p1 - p0 > kLongRowNnz) {
      const int32_t slot = atomicAdd(long_count, 1);
      if (slot < max_long) long_rows[slot] = i;
    } else {
      int64_t s = 0;
      for (int32_t p = p0; p < p1; ++p) s += b_len(op, __ldg(op.a_col + p));
      c = classify_row(p1 - p0, s, s < op.b_cols ? s : op.b_cols, op.merge_ok);
      ops[i] = s;
      cls[i] = static_cast<uint8_t>(c);
      if (c == kEmpty_) counts[i] = 0;
      take = true;
    }
  }
  count_class(s_cnt, take, c);
  __syncthreads();
  for (int k = threadIdx.x; k < kNumClasses; k += blockDim.x)
    if (s_cnt[k]) atomicAdd(&class_count[k], s_cnt[k]);
}

// One warp per long A row; the number of long rows is read on the device.
__global__ void __launch_bounds__(kThreads)
rowstats_long_kernel(Operands op, const int32_t *__restrict__ long_rows,
                     const int32_t *__restrict__ long_count,
                     int64_t *__restrict__ ops, uint8_t *__restrict__ cls,
                     int32_t *__restrict__ counts,
                     int32_t *__restrict__ class_count) {
  const int32_t n_long = *long_count;
  const int lane = lane_id();
  const int warps = (gridDim.x * blockDim.x) >> 5;
  for (int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; w < n_long;
       w += warps) {
    const int32_t i = long_rows[w];
    int32_t p0, p1;
    row_range(op, i, p0, p1);
    long long s = 0;
    for (int32_t p = p0 + lane; p < p1; p += 32) s += b_len(op, __ldg(op.a_col + p));
    s = warp_sum64(s);
    if (lane == 0) {
      const int c = classify_row(p1 - p0, s, s < op.b_cols ? s : op.b_cols, op.merge_ok);
      ops[i] = s;
      cls[i] = static_cast<uint8_t>(c);
      if (c == kEmpty_) counts[i] = 0;
      atomicAdd(&class_count[c], 1);
    }
  }
}

__global__ void __launch_bounds__(kThreads)
scatter_rows_kernel(int32_t n, const uint8_t *__restrict__ cls,
                    const int32_t *__restrict__ class_off,
                    int32_t *__restrict__ class_fill,
                    int32_t *__restrict__ rows_by_class) {
  __shared__ int32_t s_cnt[kNumClasses];
  __shared__ int32_t s_base[kNumClasses];
  for (int c = threadIdx.x; c < kNumClasses; c += blockDim.x) s_cnt[c] = 0;
  __syncthreads();

  const int32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  const int c = i < n ? cls[i] : kEmpty_;
  const bool take = i < n && c != kEmpty_;
  const unsigned peers = __match_any_sync(kFull, take ? c : (-1 - lane_id()));
  const int leader = __ffs(peers) - 1;
  const int rank = __popc(peers & lanemask_lt());
  int wbase = 0;
  if (take && rank == 0) wbase = atomicAdd(&s_cnt[c], __popc(peers));
  wbase = __shfl_sync(kFull, wbase, leader);
  __syncthreads();
  if (threadIdx.x < kNumClasses) {
    const int k = threadIdx.x;
    s_base[k] = s_cnt[k] ? atomicAdd(&class_fill[k], s_cnt[k]) : 0;
  }
  __syncthreads();
  if (take) rows_by_class[class_off[c] + s_base[c] + wbase + rank] = i;
}

// off[c] = sum of count[c'] over non-empty classes c' < c (one warp).
__global__ void class_offsets_kernel(const int32_t *__restrict__ count,
                                     int32_t *__restrict__ off) {
  const int c = threadIdx.x;
  const int v = (c < kNumClasses && c != kEmpty_) ? count[c] : 0;
  const int incl = warp_incl_scan(v);
  if (c < kNumClasses) off[c] = incl - v;
}

}  // namespace

void launch_class_offsets(const int32_t *count, int32_t *off, cudaStream_t s) {
  class_offsets_kernel<<<1, 32, 0, s>>>(count, off);
}

void launch_rowstats(const Operands &op, int64_t *ops, uint8_t *cls,
                     int32_t *counts, int32_t *class_count, int32_t *long_rows,
                     int32_t *long_count, int32_t max_long, cudaStream_t s) {
  const int grid = (op.a_rows + kThreads - 1) / kThreads;
  rowstats_kernel<<<grid, kThreads, 0, s>>>(op, ops, cls, counts, class_count,
                                             long_rows, long_count, max_long);
}

void launch_rowstats_long(const Operands &op, const int32_t *long_rows,
                          const int32_t *long_count, int64_t *ops, uint8_t *cls,
                          int32_t *counts, int32_t *class_count, int num_sms,
                          cudaStream_t s) {
  // The kernel reads the number of long rows on the device, so no host
  // round trip is needed; the grid strides over however many there are.
  const int grid = num_sms * 2;
  rowstats_long_kernel<<<grid, kThreads, 0, s>>>(op, long_rows, long_count, ops,
                                                 cls, counts, class_count);
}

void launch_scatter_rows(int32_t n, const uint8_t *cls, const int32_t *class_off,
                         int32_t *class_fill, int32_t *rows_by_class,
                         cudaStream_t s) {
  const int grid = (n + kThreads - 1) / kThreads;
  scatter_rows_kernel<<<grid, kThreads, 0, s>>>(n, cls, class_off, class_fill,
                                                rows_by_class);
}

}  // namespace rvsp
