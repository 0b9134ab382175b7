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

// kLarge = false: one warp per row below kCompactLarge entries; true: one
// block per row of kCompactLarge or more (a power-law matrix has rows of
// tens of thousands of entries, which would leave one warp copying long
// after the rest).  Coalesced copies either way.
template <bool kLarge>
__global__ void __launch_bounds__(kThreads)
compact_kernel(int32_t a_rows, const int32_t *__restrict__ counts,
               const int64_t *__restrict__ off, const int32_t *__restrict__ row_ptr,
               const int32_t *__restrict__ slab_col, const float *__restrict__ slab_val,
               int32_t *__restrict__ c_col, float *__restrict__ c_val, bool with_values) {
  const int lanes = kLarge ? kThreads : 32;
  const int me = kLarge ? threadIdx.x : lane_id();
  const int32_t first = kLarge ? blockIdx.x : (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int32_t stride = kLarge ? gridDim.x : (gridDim.x * blockDim.x) >> 5;
  for (int32_t row = first; row < a_rows; row += stride) {
    const int32_t m = counts[row];
    if (m <= 0) continue;  // empty, or redone by the plain path
    if ((m >= kCompactLarge) != kLarge) continue;
    const int64_t src = off[row];
    const int32_t dst = row_ptr[row];
    for (int32_t e = me; e < m; e += lanes) {
      c_col[dst + e] = slab_col[src + e];
      if (with_values) c_val[dst + e] = slab_val[src + e];
    }
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
                    bool with_values, int num_sms, cudaStream_t s) {
  compact_kernel<false><<<num_sms * 8, kThreads, 0, s>>>(
      a_rows, counts, off, row_ptr, slab_col, slab_val, c_col, c_val, with_values);
  compact_kernel<true><<<num_sms * 8, kThreads, 0, s>>>(
      a_rows, counts, off, row_ptr, slab_col, slab_val, c_col, c_val, with_values);
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
