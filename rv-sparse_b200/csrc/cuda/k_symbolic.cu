// Symbolic pass: the exact output nnz of every row (the count half of
// rvsp_symbolic_count, rvsp_symbolic.c:27-73).  The reference marks each
// column in a byte array and counts first touches; here each row class uses
// the structure that fits its upper bound ub = min(ops_i, b_cols):
//
//   M<K>    few A nonzeros: one thread merges the sorted B rows and counts
//           distinct heads (k_merge.cu)
//   W<T>    warp per row, shared-memory hash set of T >= 2 ub slots
//   B8192   256-thread block per row, hash set of 8192 slots
//   DENSE   512-thread block per row, bitmap over all of B's columns (shared
//           memory when it fits in 192 KiB, else a per-block global bitmap
//           that every row leaves cleared)
//
// Counting needs no order, so products are expanded 32 at a time in
// flattened order (all lanes busy whatever the B row lengths).
#include <climits>

#include "device_common.cuh"
#include "kernels.cuh"
#include "product_walk.cuh"

namespace rvsp {

namespace {

template <int LOG2T>
__global__ void __launch_bounds__(kWarpsPerBlock * 32)
sym_warp_hash_kernel(Operands op, const int32_t *__restrict__ rows,
                     int32_t nrows, int32_t *__restrict__ counts,
                     int32_t *__restrict__ status) {
  constexpr int T = 1 << LOG2T;
  extern __shared__ __align__(16) int32_t smem_i32[];
  int32_t *keys = smem_i32 + (threadIdx.x >> 5) * T;
  const int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (w >= nrows) return;
  const int lane = lane_id();
  fill_words(keys, T, 0xffffffffu, lane, 32);
  __syncwarp();
  const int32_t row = row_of(rows, w);
  int cnt = 0;
  bool bad = false;
  for_each_product_col(op, op.a_rp[row], op.a_rp[row + 1], 0, 1,
                       [&](int32_t col) {
                         bool created;
                         if (hash_insert(keys, LOG2T, col, created) < 0) bad = true;
                         cnt += created;
                       });
  cnt = warp_sum(cnt);
  if (__any_sync(kFull, bad) && lane == 0) report(status, kDevHashFull);
  if (lane == 0) counts[row] = cnt;
}

__global__ void __launch_bounds__(kBlockHashThreads)
sym_block_hash_kernel(Operands op, const int32_t *__restrict__ rows,
                      int32_t *__restrict__ counts,
                      int32_t *__restrict__ status) {
  constexpr int T = 1 << kBlockHashLog2;
  extern __shared__ __align__(16) int32_t smem_i32[];
  int32_t *keys = smem_i32;
  __shared__ int32_t s_cnt;
  __shared__ int32_t s_bad;
  fill_words(keys, T, 0xffffffffu, threadIdx.x, blockDim.x);
  if (threadIdx.x == 0) {
    s_cnt = 0;
    s_bad = 0;
  }
  __syncthreads();
  const int32_t row = row_of(rows, blockIdx.x);
  int cnt = 0;
  bool bad = false;
  for_each_product_col(op, op.a_rp[row], op.a_rp[row + 1], threadIdx.x >> 5,
                       blockDim.x >> 5, [&](int32_t col) {
                         bool created;
                         if (hash_insert(keys, kBlockHashLog2, col, created) < 0)
                           bad = true;
                         cnt += created;
                       });
  cnt = warp_sum(cnt);
  const bool any_bad = __any_sync(kFull, bad);
  if (lane_id() == 0) {
    atomicAdd(&s_cnt, cnt);
    if (any_bad) s_bad = 1;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    counts[row] = s_cnt;
    if (s_bad) report(status, kDevHashFull);
  }
}

template <bool kSmemBits>
__global__ void __launch_bounds__(kDenseThreads)
sym_dense_kernel(Operands op, const int32_t *__restrict__ rows, int32_t nrows,
                 int32_t *__restrict__ counts, uint32_t *__restrict__ gbits,
                 size_t gbits_stride) {
  extern __shared__ uint32_t smem_u32[];
  __shared__ int32_t s_cnt, s_lo, s_hi;
  const int32_t words = (op.b_cols + 31) >> 5;
  uint32_t *bits = kSmemBits ? smem_u32 : gbits + gbits_stride * blockIdx.x;
  if (kSmemBits) {
    for (int32_t w = threadIdx.x; w < words; w += blockDim.x) bits[w] = 0u;
  }
  for (int32_t r = blockIdx.x; r < nrows; r += gridDim.x) {
    if (threadIdx.x == 0) {
      s_cnt = 0;
      s_lo = INT_MAX;
      s_hi = -1;
    }
    __syncthreads();
    const int32_t row = row_of(rows, r);
    int cnt = 0, lo = INT_MAX, hi = -1;
    for_each_product_col(op, op.a_rp[row], op.a_rp[row + 1], threadIdx.x >> 5,
                         blockDim.x >> 5, [&](int32_t col) {
                           const uint32_t bit = 1u << (col & 31);
                           const uint32_t old = atomicOr(&bits[col >> 5], bit);
                           cnt += (old & bit) ? 0 : 1;
                           lo = min(lo, col);
                           hi = max(hi, col);
                         });
    cnt = warp_sum(cnt);
    lo = warp_min(lo);
    hi = warp_max(hi);
    if (lane_id() == 0) {
      atomicAdd(&s_cnt, cnt);
      atomicMin(&s_lo, lo);
      atomicMax(&s_hi, hi);
    }
    __syncthreads();
    if (threadIdx.x == 0) counts[row] = s_cnt;
    if (s_hi >= 0) {
      for (int32_t w = (s_lo >> 5) + threadIdx.x; w <= (s_hi >> 5); w += blockDim.x)
        bits[w] = 0u;
    }
    __syncthreads();
  }
}

// Optimistic sizing of the W1024 / W2048 rows.  Their class comes from the
// product count, an upper bound that can be far above the row's distinct
// columns (a 27-point stencil row: 729 products, 125 columns), and a table of
// 2048 slots per warp leaves few warps resident.  Such a row first counts in
// a table of 1 << kOptLog2 slots with at most kOptProbes probes per insert;
// the count is exact whenever every insert succeeds.  A row whose insert
// fails (more columns than the table holds, or a probe run that long) is
// appended to a retry list and counted again at its class size.
constexpr int kOptLog2 = 9;
constexpr uint32_t kOptProbes = 32;

__device__ __forceinline__ int hash_insert_bounded(int32_t *keys, int log2t, int32_t col,
                                                   bool &created) {
  const uint32_t mask = (1u << log2t) - 1u;
  uint32_t h = hash_slot(col, log2t);
  created = false;
  for (uint32_t probe = 0; probe < kOptProbes; ++probe) {
    int32_t cur = *reinterpret_cast<volatile int32_t *>(&keys[h]);
    if (cur == col) return static_cast<int>(h);
    if (cur == kEmpty) {
      int32_t prev = atomicCAS(&keys[h], kEmpty, col);
      if (prev == kEmpty) {
        created = true;
        return static_cast<int>(h);
      }
      if (prev == col) return static_cast<int>(h);
    }
    h = (h + 1u) & mask;
  }
  return -1;
}

__global__ void __launch_bounds__(kWarpsPerBlock * 32)
sym_warp_hash_try_kernel(Operands op, const int32_t *__restrict__ rows, int32_t nrows,
                         int32_t *__restrict__ counts, int32_t *__restrict__ retry,
                         int32_t *__restrict__ retry_n) {
  constexpr int T = 1 << kOptLog2;
  __shared__ int32_t s_keys[kWarpsPerBlock][T];
  int32_t *keys = s_keys[threadIdx.x >> 5];
  const int64_t w = (int64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
  if (w >= nrows) return;
  const int lane = lane_id();
  fill_words(keys, T, 0xffffffffu, lane, 32);
  __syncwarp();
  const int32_t row = row_of(rows, static_cast<int32_t>(w));
  int cnt = 0;
  bool bad = false;
  for_each_product_col(op, op.a_rp[row], op.a_rp[row + 1], 0, 1, [&](int32_t col) {
    if (bad) return;
    bool created;
    if (hash_insert_bounded(keys, kOptLog2, col, created) < 0) bad = true;
    cnt += created;
  });
  cnt = warp_sum(cnt);
  const bool any_bad = __any_sync(kFull, bad);
  if (lane == 0) {
    if (any_bad) retry[atomicAdd(retry_n, 1)] = row;
    else counts[row] = cnt;
  }
}

// The retried rows at their class size: persistent warps over the list,
// whose length is read on the device.
template <int LOG2T>
__global__ void __launch_bounds__(kWarpsPerBlock * 32)
sym_warp_hash_list_kernel(Operands op, const int32_t *__restrict__ list,
                          const int32_t *__restrict__ list_n, int32_t *__restrict__ counts,
                          int32_t *__restrict__ status) {
  constexpr int T = 1 << LOG2T;
  extern __shared__ __align__(16) int32_t smem_i32[];
  int32_t *keys = smem_i32 + (threadIdx.x >> 5) * T;
  const int lane = lane_id();
  const int32_t n = *list_n;
  const int64_t stride = (int64_t(gridDim.x) * blockDim.x) >> 5;
  for (int64_t w = (int64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5; w < n;
       w += stride) {
    fill_words(keys, T, 0xffffffffu, lane, 32);
    __syncwarp();
    const int32_t row = list[w];
    int cnt = 0;
    bool bad = false;
    for_each_product_col(op, op.a_rp[row], op.a_rp[row + 1], 0, 1, [&](int32_t col) {
      bool created;
      if (hash_insert(keys, LOG2T, col, created) < 0) bad = true;
      cnt += created;
    });
    cnt = warp_sum(cnt);
    if (__any_sync(kFull, bad) && lane == 0) report(status, kDevHashFull);
    if (lane == 0) counts[row] = cnt;
    __syncwarp();  // the table is cleared for the warp's next row
  }
}

template <int LOG2T>
void launch_list_hash(const Operands &op, const int32_t *list, const int32_t *list_n,
                      int32_t max_rows, int32_t *counts, int32_t *status, int num_sms,
                      cudaStream_t s) {
  const size_t smem = size_t(kWarpsPerBlock) * (size_t(1) << LOG2T) * sizeof(int32_t);
  const int threads = kWarpsPerBlock * 32;
  int per_sm = 1;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, sym_warp_hash_list_kernel<LOG2T>,
                                                    threads, smem) != cudaSuccess ||
      per_sm < 1)
    per_sm = 1;
  int64_t grid = int64_t(num_sms) * per_sm;
  const int64_t need = (int64_t(max_rows) + kWarpsPerBlock - 1) / kWarpsPerBlock;
  if (grid > need) grid = need;
  if (grid < 1) grid = 1;
  sym_warp_hash_list_kernel<LOG2T><<<static_cast<unsigned>(grid), threads, smem, s>>>(
      op, list, list_n, counts, status);
}

template <int LOG2T>
void launch_warp_hash(const Operands &op, const int32_t *rows, int32_t nrows,
                      int32_t *counts, int32_t *status, cudaStream_t s) {
  const size_t smem = size_t(kWarpsPerBlock) * (size_t(1) << LOG2T) * sizeof(int32_t);
  const int threads = kWarpsPerBlock * 32;
  const int grid = (nrows + kWarpsPerBlock - 1) / kWarpsPerBlock;
  sym_warp_hash_kernel<LOG2T><<<grid, threads, smem, s>>>(op, rows, nrows, counts,
                                                          status);
}

}  // namespace

bool symbolic_optimistic_class(int cls) { return cls == kW1024 || cls == kW2048; }

void launch_symbolic_optimistic(int cls, const Operands &op, const int32_t *rows,
                                int32_t nrows, int32_t *counts, int32_t *retry,
                                int32_t *retry_n, int32_t *status, int num_sms,
                                cudaStream_t s) {
  if (nrows <= 0 || !symbolic_optimistic_class(cls)) return;
  const int64_t grid = (int64_t(nrows) + kWarpsPerBlock - 1) / kWarpsPerBlock;
  sym_warp_hash_try_kernel<<<static_cast<unsigned>(grid), kWarpsPerBlock * 32, 0, s>>>(
      op, rows, nrows, counts, retry, retry_n);
  if (cls == kW1024)
    launch_list_hash<10>(op, retry, retry_n, nrows, counts, status, num_sms, s);
  else
    launch_list_hash<11>(op, retry, retry_n, nrows, counts, status, num_sms, s);
}

void launch_symbolic_class(int cls, const Operands &op, const int32_t *rows,
                           int32_t nrows, int32_t *counts, uint32_t *gbitmap,
                           int32_t gbitmap_slots, int32_t *status, int num_sms,
                           cudaStream_t s) {
  if (nrows <= 0) return;
  if ((cls == kB8192 || cls == kDense) && heavy_fits(op.b_cols)) {
    launch_heavy_symbolic(op, rows, nrows, counts, num_sms, s);
    return;
  }
  switch (cls) {
    case kM4:
    case kM8:
    case kM16: launch_merge_symbolic(cls, op, rows, nrows, counts, s); break;
    case kW64: launch_warp_hash<6>(op, rows, nrows, counts, status, s); break;
    case kW128: launch_warp_hash<7>(op, rows, nrows, counts, status, s); break;
    case kW256: launch_warp_hash<8>(op, rows, nrows, counts, status, s); break;
    case kW512: launch_warp_hash<9>(op, rows, nrows, counts, status, s); break;
    case kW1024: launch_warp_hash<10>(op, rows, nrows, counts, status, s); break;
    case kW2048: launch_warp_hash<11>(op, rows, nrows, counts, status, s); break;
    case kB8192: {
      const size_t smem = (size_t(1) << kBlockHashLog2) * sizeof(int32_t);
      sym_block_hash_kernel<<<nrows, kBlockHashThreads, smem, s>>>(op, rows, counts,
                                                                  status);
      break;
    }
    case kDense: {
      const int64_t words = (int64_t(op.b_cols) + 31) >> 5;
      if (op.b_cols <= kSmemBitmapMaxCols) {
        const size_t smem = size_t(words) * sizeof(uint32_t);
        cudaFuncSetAttribute(sym_dense_kernel<true>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize,
                             static_cast<int>(smem));
        const int grid = nrows < num_sms ? nrows : num_sms;
        sym_dense_kernel<true><<<grid, kDenseThreads, smem, s>>>(op, rows, nrows,
                                                                 counts, nullptr, 0);
      } else {
        const size_t stride = dense_slot_bits_bytes(op.b_cols) / sizeof(uint32_t);
        const int grid = nrows < gbitmap_slots ? nrows : gbitmap_slots;
        sym_dense_kernel<false><<<grid, kDenseThreads, 0, s>>>(op, rows, nrows,
                                                               counts, gbitmap, stride);
      }
      break;
    }
    default: break;
  }
}

}  // namespace rvsp
