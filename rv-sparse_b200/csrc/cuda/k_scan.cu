// Exclusive prefix scan of per-row output counts into C.row_ptr, with the
// int64 total and the numeric-pass row classes computed on the way.
//
// Replaces the serial prefix of rvsp_symbolic_count (rvsp_symbolic.c:75-85)
// and its overflow guard (:69-72): the total is accumulated in int64, so a
// product whose nnz(C) exceeds INT32_MAX is detected exactly and reported by
// the host as RVSP_ERROR_ALLOCATION_FAILED.
//
// Three launches, no inter-block waiting: tile sums, a one-block scan of the
// tile sums, then a tile-local scan plus offset.  Each tile is 4096 rows.
#include "device_common.cuh"
#include "kernels.cuh"

namespace rvsp {

namespace {

constexpr int kThreads = 256;
constexpr int kItems = 16;
constexpr int kTile = kThreads * kItems;

// Skewed shared-memory index: one pad word per 32 keeps both the coalesced
// pass (consecutive idx per warp) and the per-thread pass (stride kItems)
// free of bank conflicts.
__device__ __forceinline__ int skew(int idx) { return idx + (idx >> 5); }

__device__ __forceinline__ long long block_excl_scan64(long long v,
                                                       long long *s_warp,
                                                       long long *total) {
  const int lane = lane_id(), warp = threadIdx.x >> 5;
  long long x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    long long n = __shfl_up_sync(kFull, x, o);
    if (lane >= o) x += n;
  }
  if (lane == 31) s_warp[warp] = x;
  __syncthreads();
  if (warp == 0) {
    long long w = lane < (kThreads / 32) ? s_warp[lane] : 0;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      long long n = __shfl_up_sync(kFull, w, o);
      if (lane >= o) w += n;
    }
    if (lane < (kThreads / 32)) s_warp[lane] = w;
  }
  __syncthreads();
  const long long before = warp > 0 ? s_warp[warp - 1] : 0;
  *total = s_warp[kThreads / 32 - 1];
  return before + x - v;
}

__global__ void __launch_bounds__(kThreads)
tile_sum_kernel(int32_t n, const int32_t *__restrict__ counts,
                int64_t *__restrict__ partials) {
  __shared__ long long s_warp[kThreads / 32];
  const int64_t base = static_cast<int64_t>(blockIdx.x) * kTile;
  long long s = 0;
#pragma unroll
  for (int r = 0; r < kItems; ++r) {
    const int64_t i = base + r * kThreads + threadIdx.x;
    if (i < n) s += counts[i];
  }
  s = warp_sum64(s);
  if (lane_id() == 0) s_warp[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    long long t = 0;
    for (int w = 0; w < kThreads / 32; ++w) t += s_warp[w];
    partials[blockIdx.x] = t;
  }
}

// One block: partials[0..nt) becomes its exclusive scan; total to *total and,
// when it fits, row_ptr[n].
__global__ void __launch_bounds__(kThreads)
partials_scan_kernel(int32_t n, int32_t nt, int64_t *__restrict__ partials,
                     int64_t *__restrict__ total, int32_t *__restrict__ row_ptr,
                     CheckGuard guard) {
  __shared__ long long s_warp[kThreads / 32];
  if (guard.failed()) return;
  long long carry = 0;
  for (int32_t b = 0; b < nt; b += kThreads) {
    const int32_t i = b + threadIdx.x;
    const long long v = i < nt ? partials[i] : 0;
    long long chunk_total;
    const long long ex = block_excl_scan64(v, s_warp, &chunk_total);
    if (i < nt) partials[i] = carry + ex;
    carry += chunk_total;
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    *total = carry;
    row_ptr[n] = carry <= 0x7fffffffLL ? static_cast<int32_t>(carry) : -1;
  }
}

__global__ void __launch_bounds__(kThreads)
tile_apply_kernel(int32_t n, const int32_t *__restrict__ counts,
                  const int64_t *__restrict__ ops,
                  const int32_t *__restrict__ a_rp,
                  const int64_t *__restrict__ partials,
                  int32_t *__restrict__ row_ptr, uint8_t *__restrict__ cls,
                  int32_t *__restrict__ class_count, bool merge_ok, CheckGuard guard,
                  const int32_t *__restrict__ skip) {
  __shared__ int32_t s_items[kTile + kTile / 32];
  __shared__ long long s_warp[kThreads / 32];
  __shared__ int32_t s_cnt[kNumClasses];
  if (guard.failed()) return;
  for (int c = threadIdx.x; c < kNumClasses; c += blockDim.x) s_cnt[c] = 0;
  const int64_t base = static_cast<int64_t>(blockIdx.x) * kTile;
  __syncthreads();

  // Coalesced load of the tile; class each row for the numeric pass.
#pragma unroll 4
  for (int r = 0; r < kItems; ++r) {
    const int idx = r * kThreads + threadIdx.x;
    const int64_t i = base + idx;
    int m = 0;
    int c = kEmpty_;
    if (i < n) {
      m = counts[i];
      c = (skip && skip[i] >= 0) ? kEmpty_
                                 : classify_row(a_rp[i + 1] - a_rp[i], ops[i], m, merge_ok);
      cls[i] = static_cast<uint8_t>(c);
    }
    s_items[skew(idx)] = m;
    const bool take = i < n;
    const unsigned peers =
        __match_any_sync(kFull, take ? c : (-1 - lane_id()));
    if (take && (peers & lanemask_lt()) == 0)
      atomicAdd(&s_cnt[c], __popc(peers));
  }
  __syncthreads();

  // Thread t scans items [t * kItems, (t + 1) * kItems) of the tile.
  long long mine = 0;
#pragma unroll
  for (int q = 0; q < kItems; ++q) mine += s_items[skew(threadIdx.x * kItems + q)];
  long long tile_total;
  long long run = partials[blockIdx.x] + block_excl_scan64(mine, s_warp, &tile_total);
#pragma unroll
  for (int q = 0; q < kItems; ++q) {
    const int idx = threadIdx.x * kItems + q;
    const int v = s_items[skew(idx)];
    s_items[skew(idx)] = run <= 0x7fffffffLL ? static_cast<int32_t>(run) : -1;
    run += v;
  }
  __syncthreads();
#pragma unroll 4
  for (int r = 0; r < kItems; ++r) {
    const int idx = r * kThreads + threadIdx.x;
    const int64_t i = base + idx;
    if (i < n) row_ptr[i] = s_items[skew(idx)];
  }
  for (int k = threadIdx.x; k < kNumClasses; k += blockDim.x)
    if (s_cnt[k]) atomicAdd(&class_count[k], s_cnt[k]);
}

// One block: exclusive scan of partials[0..nt) in place, total to *total.
__global__ void __launch_bounds__(kThreads)
partials_scan64_kernel(int32_t nt, int64_t *__restrict__ partials,
                       int64_t *__restrict__ total) {
  __shared__ long long s_warp[kThreads / 32];
  long long carry = 0;
  for (int32_t b = 0; b < nt; b += kThreads) {
    const int32_t i = b + threadIdx.x;
    const long long v = i < nt ? partials[i] : 0;
    long long chunk_total;
    const long long ex = block_excl_scan64(v, s_warp, &chunk_total);
    if (i < nt) partials[i] = carry + ex;
    carry += chunk_total;
    __syncthreads();
  }
  if (threadIdx.x == 0) *total = carry;
}

// out[i] = partials[tile] + exclusive prefix of in within the tile (int64).
__global__ void __launch_bounds__(kThreads)
tile_apply64_kernel(int32_t n, const int32_t *__restrict__ in,
                    const int64_t *__restrict__ partials, int64_t *__restrict__ out) {
  __shared__ int32_t s_items[kTile + kTile / 32];
  __shared__ long long s_warp[kThreads / 32];
  const int64_t base = static_cast<int64_t>(blockIdx.x) * kTile;
#pragma unroll 4
  for (int r = 0; r < kItems; ++r) {
    const int idx = r * kThreads + threadIdx.x;
    s_items[skew(idx)] = base + idx < n ? in[base + idx] : 0;
  }
  __syncthreads();
  long long mine = 0;
#pragma unroll
  for (int q = 0; q < kItems; ++q) mine += s_items[skew(threadIdx.x * kItems + q)];
  long long tile_total;
  long long run = partials[blockIdx.x] + block_excl_scan64(mine, s_warp, &tile_total);
#pragma unroll
  for (int q = 0; q < kItems; ++q) {
    const int64_t i = base + threadIdx.x * kItems + q;
    if (i < n) out[i] = run;
    run += s_items[skew(threadIdx.x * kItems + q)];
  }
}

}  // namespace

void launch_scan_i64(int32_t n, const int32_t *in, int64_t *out, int64_t *partials,
                     int64_t *total, cudaStream_t s) {
  const int32_t nt = static_cast<int32_t>((static_cast<int64_t>(n) + kTile - 1) / kTile);
  tile_sum_kernel<<<nt, kThreads, 0, s>>>(n, in, partials);
  partials_scan64_kernel<<<1, kThreads, 0, s>>>(nt, partials, total);
  tile_apply64_kernel<<<nt, kThreads, 0, s>>>(n, in, partials, out);
}

size_t scan_partials_bytes(int32_t n) {
  const size_t nt = (static_cast<size_t>(n) + kTile - 1) / kTile;
  return (nt + 1) * sizeof(int64_t);
}

void launch_scan_and_class(int32_t n, const int32_t *counts, const int64_t *ops,
                           const int32_t *a_rp, int32_t *row_ptr,
                           int64_t *partials, int64_t *total, uint8_t *cls,
                           int32_t *class_count, bool merge_ok, cudaStream_t s,
                           CheckGuard guard, const int32_t *skip) {
  const int32_t nt = static_cast<int32_t>((static_cast<int64_t>(n) + kTile - 1) / kTile);
  tile_sum_kernel<<<nt, kThreads, 0, s>>>(n, counts, partials);
  partials_scan_kernel<<<1, kThreads, 0, s>>>(n, nt, partials, total, row_ptr, guard);
  tile_apply_kernel<<<nt, kThreads, 0, s>>>(n, counts, ops, a_rp, partials, row_ptr,
                                            cls, class_count, merge_ok, guard, skip);
}

}  // namespace rvsp
