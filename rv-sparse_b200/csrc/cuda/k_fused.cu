// Support kernels of the learned (fused single-pass) path: compaction of the
// slab into C, classing and scattering of the overflow-row list, and the
// fingerprint of A's and B's values that tells a later compute() whether the
// values the fused pass used are still current.
#include "device_common.cuh"
#include "kernels.cuh"

namespace rvsp {

namespace {

constexpr int kThreads = 256;

// Rows of at least this many entries are copied by whole blocks.
constexpr int32_t kCompactLarge = 4096;

// Rows of kCompactLarge entries or more, listed by compact_small_kernel in
// big[1..big[0]]: one block per row (a power-law matrix has rows of tens of
// thousands of entries).  Coalesced copies.
__global__ void __launch_bounds__(kThreads)
compact_large_kernel(const int32_t *__restrict__ big, const int32_t *__restrict__ counts,
                     const int64_t *__restrict__ off, const int32_t *__restrict__ row_ptr,
                     const int32_t *__restrict__ slab_col,
                     const float *__restrict__ slab_val, int32_t *__restrict__ c_col,
                     float *__restrict__ c_val, bool with_values) {
  const int32_t n = big[0];
  for (int32_t i = blockIdx.x; i < n; i += gridDim.x) {
    const int32_t row = big[1 + i];
    const int32_t m = counts[row];
    const int64_t src = off[row];
    const int32_t dst = row_ptr[row];
    for (int32_t e = threadIdx.x; e < m; e += kThreads) {
      c_col[dst + e] = slab_col[src + e];
      if (with_values) c_val[dst + e] = slab_val[src + e];
    }
  }
}

// Shorter rows: a block takes `rows_per_chunk` (a power of two, at most
// kThreads) consecutive rows and copies all of their entries as one flat
// range, each thread finding the row of its entry by binary search over the
// block's prefix of row lengths, so short rows keep every thread busy and
// reads and writes stay contiguous.  Rows of kCompactLarge entries or more
// are appended to big[1..] for compact_large_kernel.
__global__ void __launch_bounds__(kThreads)
compact_small_kernel(int32_t a_rows, int rows_per_chunk, const int32_t *__restrict__ counts,
                     const int64_t *__restrict__ off, const int32_t *__restrict__ row_ptr,
                     const int32_t *__restrict__ slab_col,
                     const float *__restrict__ slab_val, int32_t *__restrict__ c_col,
                     float *__restrict__ c_val, bool with_values,
                     int32_t *__restrict__ big) {
  __shared__ int32_t s_incl[kThreads];
  __shared__ int64_t s_src[kThreads];
  __shared__ int32_t s_dst[kThreads];
  __shared__ int32_t s_wsum[kThreads / 32];
  const int tid = threadIdx.x, lane = lane_id(), w = tid >> 5;
  const int64_t chunks = (int64_t(a_rows) + rows_per_chunk - 1) / rows_per_chunk;
  for (int64_t ch = blockIdx.x; ch < chunks; ch += gridDim.x) {
    const int64_t row = ch * rows_per_chunk + tid;
    int32_t m = (tid < rows_per_chunk && row < a_rows) ? counts[row] : 0;
    const bool large = m >= kCompactLarge;
    const unsigned large_mask = __ballot_sync(kFull, large);
    if (large_mask) {
      int32_t base = 0;
      if (lane == 0) base = atomicAdd(big, __popc(large_mask));
      base = __shfl_sync(kFull, base, 0);
      if (large) big[1 + base + __popc(large_mask & ((1u << lane) - 1))] = int32_t(row);
    }
    if (m < 0 || large) m = 0;  // redone by the plain path / copied by blocks
    int64_t src = 0;
    int32_t dst = 0;
    if (m > 0) {
      src = off[row];
      dst = row_ptr[row];
    }
    const int incl = warp_incl_scan(m);
    if (lane == 31) s_wsum[w] = incl;
    __syncthreads();
    int wbase = 0, total = 0;
#pragma unroll
    for (int i = 0; i < kThreads / 32; ++i) {
      if (i < w) wbase += s_wsum[i];
      total += s_wsum[i];
    }
    s_incl[tid] = wbase + incl;
    s_src[tid] = src;
    s_dst[tid] = dst;
    __syncthreads();
    for (int32_t e = tid; e < total; e += kThreads) {
      // the first row j with s_incl[j] > e (e < total, so j < rows_per_chunk)
      int j = 0;
      for (int sz = rows_per_chunk >> 1; sz >= 1; sz >>= 1)
        if (s_incl[j + sz - 1] <= e) j += sz;
      const int32_t k = e - (j ? s_incl[j - 1] : 0);
      c_col[s_dst[j] + k] = slab_col[s_src[j] + k];
      if (with_values) c_val[s_dst[j] + k] = slab_val[s_src[j] + k];
    }
    __syncthreads();  // the next chunk overwrites the tables
  }
}

__global__ void __launch_bounds__(kThreads)
list_classify_kernel(const int32_t *__restrict__ list, int32_t n,
                     const int64_t *__restrict__ ops, const int32_t *__restrict__ a_rp,
                     const int32_t *__restrict__ counts, int32_t b_cols, bool numeric,
                     uint8_t *__restrict__ cls_out, int32_t *__restrict__ class_count) {
  const int32_t j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n) return;
  const int32_t row = list[j];
  const long long o = ops[row];
  const long long bound = numeric ? counts[row] : (o < b_cols ? o : b_cols);
  const int c = classify_row(a_rp[row + 1] - a_rp[row], o, bound, false);
  cls_out[j] = static_cast<uint8_t>(c);
  atomicAdd(&class_count[c], 1);
}

__global__ void __launch_bounds__(kThreads)
scatter_list_kernel(const int32_t *__restrict__ list, int32_t n,
                    const uint8_t *__restrict__ cls, const int32_t *__restrict__ class_off,
                    int32_t *__restrict__ class_fill, int32_t *__restrict__ out) {
  const int32_t j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n) return;
  const int c = cls[j];
  out[class_off[c] + atomicAdd(&class_fill[c], 1)] = list[j];
}

__device__ __forceinline__ unsigned long long mix64(unsigned long long z) {
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

// Sum over i of mix(salt, i, bits(v[i])): a change of any value or position
// changes the sum except with probability about 2^-64.
__global__ void __launch_bounds__(kThreads)
values_hash_kernel(const float *__restrict__ v, int64_t n, unsigned long long salt,
                   unsigned long long *__restrict__ h) {
  unsigned long long acc = 0;
  const int64_t stride = int64_t(gridDim.x) * blockDim.x;
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride) {
    const unsigned long long key =
        (static_cast<unsigned long long>(i) << 32) ^ __float_as_uint(v[i]) ^ salt;
    acc += mix64(key + 0x9E3779B97F4A7C15ull);
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(kFull, acc, o);
  if (lane_id() == 0) atomicAdd(h, acc);
}

}  // namespace

void launch_compact(int32_t a_rows, const int32_t *counts, const int64_t *off,
                    const int32_t *row_ptr, const int32_t *slab_col,
                    const float *slab_val, int32_t *c_col, float *c_val,
                    bool with_values, int32_t *big, int num_sms, cudaStream_t s) {
  if (a_rows <= 0) return;
  const int blocks = num_sms * 8;
  // enough chunks to give every block some: 32 .. kThreads rows each
  int rows_per_chunk = kThreads;
  while (rows_per_chunk > 32 && int64_t(a_rows) < int64_t(rows_per_chunk) * blocks)
    rows_per_chunk >>= 1;
  cudaMemsetAsync(big, 0, sizeof(int32_t), s);
  compact_small_kernel<<<blocks, kThreads, 0, s>>>(a_rows, rows_per_chunk, counts, off,
                                                   row_ptr, slab_col, slab_val, c_col,
                                                   c_val, with_values, big);
  compact_large_kernel<<<blocks, kThreads, 0, s>>>(big, counts, off, row_ptr, slab_col,
                                                   slab_val, c_col, c_val, with_values);
}

void launch_list_classify(const int32_t *list, int32_t n, const int64_t *ops,
                          const int32_t *a_rp, const int32_t *counts, int32_t b_cols,
                          bool numeric, uint8_t *cls_out, int32_t *class_count,
                          cudaStream_t s) {
  if (n <= 0) return;
  list_classify_kernel<<<(n + kThreads - 1) / kThreads, kThreads, 0, s>>>(
      list, n, ops, a_rp, counts, b_cols, numeric, cls_out, class_count);
}

void launch_scatter_list(const int32_t *list, int32_t n, const uint8_t *cls,
                         const int32_t *class_off, int32_t *class_fill, int32_t *out,
                         cudaStream_t s) {
  if (n <= 0) return;
  scatter_list_kernel<<<(n + kThreads - 1) / kThreads, kThreads, 0, s>>>(
      list, n, cls, class_off, class_fill, out);
}

void launch_values_hash(const float *v, int64_t n, unsigned long long salt,
                        unsigned long long *h, cudaStream_t s) {
  if (n <= 0) return;
  int64_t blocks = (n + kThreads - 1) / kThreads;
  if (blocks > 148 * 16) blocks = 148 * 16;
  values_hash_kernel<<<static_cast<int>(blocks), kThreads, 0, s>>>(v, n, salt, h);
}

}  // namespace rvsp
