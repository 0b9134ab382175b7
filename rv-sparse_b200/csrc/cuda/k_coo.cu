// Coordinate (COO) entries to canonical CSR on the GPU: the canonicalisation
// of a Matrix Market file's entries (tools/src/mtx_to_csr_formatter.c:67-146
// and :214-311 in the reference).
//
// The reference appends, for a symmetric file, the mirror of every
// off-diagonal entry after all stored entries (in stored order), scatters
// the entries to their rows in that order, sorts each row by column with
// glibc's qsort (a merge sort there: equal columns keep their order) and sums
// each run of equal columns from its first value, left to right.  Here every
// entry carries its index in that order (file entries k, mirrors 2^31 | k,
// which sort after all file entries and among themselves by k), each row is
// sorted by (column, index), and a run is summed in index order with the
// same roundings (acc = v0, acc = fl(acc + v) ...), so the result is the
// reference's bit for bit.
//
// Passes (one stream, the host waits once for the output size):
//   check ranges | count per row | scan | scatter (column, index) keys |
//   sort each row (warp, block or global bitonic by length) | count runs per
//   row | scan to row_ptr | write one (column, sum) per run.
#include <cuda_runtime.h>

#include <climits>
#include <mutex>

#include "device_common.cuh"
#include "kernels.cuh"
#include "rvsp_cuda.h"

namespace rvsp {

namespace {

constexpr int kCooThreads = 256;
constexpr int kBlockSortMax = 4096;  // keys a block sorts in shared memory (32 KB)
constexpr uint32_t kMirrorBit = 0x80000000u;
constexpr unsigned long long kKeyInf = ~0ull;

__global__ void __launch_bounds__(kCooThreads)
coo_count_kernel(int64_t n, int32_t rows, int32_t cols, const int32_t *__restrict__ row,
                 const int32_t *__restrict__ col, int symmetric, int32_t *__restrict__ counts,
                 int32_t *__restrict__ bad) {
  const int64_t stride = int64_t(gridDim.x) * blockDim.x;
  for (int64_t k = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; k < n; k += stride) {
    const int32_t r = row[k], c = col[k];
    if (r < 0 || r >= rows || c < 0 || c >= cols) {
      atomicExch(bad, 1);
      continue;
    }
    atomicAdd(counts + r, 1);
    if (symmetric && r != c) {
      if (c >= rows || r >= cols) {  // the mirror falls outside a non-square matrix
        atomicExch(bad, 1);
        continue;
      }
      atomicAdd(counts + c, 1);
    }
  }
}

// keys[seg[r] + slot] = column << 32 | index; cursor (zeroed) hands out slots.
__global__ void __launch_bounds__(kCooThreads)
coo_scatter_kernel(int64_t n, const int32_t *__restrict__ row, const int32_t *__restrict__ col,
                   int symmetric, const int64_t *__restrict__ seg,
                   int32_t *__restrict__ cursor, unsigned long long *__restrict__ keys) {
  const int64_t stride = int64_t(gridDim.x) * blockDim.x;
  for (int64_t k = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; k < n; k += stride) {
    const int32_t r = row[k], c = col[k];
    const int64_t p = seg[r] + atomicAdd(cursor + r, 1);
    keys[p] = (static_cast<unsigned long long>(c) << 32) | static_cast<uint32_t>(k);
    if (symmetric && r != c) {
      const int64_t q = seg[c] + atomicAdd(cursor + c, 1);
      keys[q] = (static_cast<unsigned long long>(r) << 32) |
                (static_cast<uint32_t>(k) | kMirrorBit);
    }
  }
}

// Bitonic network in the form whose every comparator puts the smaller key at
// the lower index (stage k: first compare i with i ^ (k - 1), then i with
// i ^ j for j = k/4 .. 1), so keys past the end act as +infinity and are
// never touched.

// Rows of at most 32 entries: a warp per row, keys in registers.  Longer rows
// go to the block list (at most kBlockSortMax) or the global list.
__global__ void __launch_bounds__(kCooThreads)
coo_sort_warp_kernel(int32_t rows, const int64_t *__restrict__ seg,
                     const int32_t *__restrict__ counts, unsigned long long *__restrict__ keys,
                     int32_t *__restrict__ mid_list, int32_t *__restrict__ big_list) {
  const int64_t w = (int64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
  if (w >= rows) return;
  const int lane = lane_id();
  const int32_t r = static_cast<int32_t>(w);
  const int32_t len = counts[r];
  if (len <= 1) return;
  if (len > 32) {
    if (lane == 0) {
      if (len <= kBlockSortMax) mid_list[1 + atomicAdd(mid_list, 1)] = r;
      else big_list[1 + atomicAdd(big_list, 1)] = r;
    }
    return;
  }
  unsigned long long *kr = keys + seg[r];
  unsigned long long x = lane < len ? kr[lane] : kKeyInf;
#pragma unroll
  for (int k = 2; k <= 32; k <<= 1) {
#pragma unroll
    for (int j = k >> 1; j > 0; j >>= 1) {
      const int partner = (j == (k >> 1)) ? (lane ^ (k - 1)) : (lane ^ j);
      const unsigned long long y = __shfl_sync(kFull, x, partner);
      const bool lower = lane < partner;
      x = lower ? (x < y ? x : y) : (x > y ? x : y);
    }
  }
  if (lane < len) kr[lane] = x;
}

// Rows of 33 .. kBlockSortMax entries: a block per listed row, in shared memory.
__global__ void __launch_bounds__(kCooThreads)
coo_sort_block_kernel(const int32_t *__restrict__ list, const int64_t *__restrict__ seg,
                      const int32_t *__restrict__ counts,
                      unsigned long long *__restrict__ keys) {
  __shared__ unsigned long long s[kBlockSortMax];
  const int32_t n = list[0];
  for (int32_t i = blockIdx.x; i < n; i += gridDim.x) {
    const int32_t r = list[1 + i];
    const int32_t len = counts[r];
    unsigned long long *kr = keys + seg[r];
    int p2 = 64;
    while (p2 < len) p2 <<= 1;
    for (int t = threadIdx.x; t < p2; t += kCooThreads) s[t] = t < len ? kr[t] : kKeyInf;
    __syncthreads();
    for (int k = 2; k <= p2; k <<= 1) {
      for (int j = k >> 1; j > 0; j >>= 1) {
        for (int t = threadIdx.x; t < p2; t += kCooThreads) {
          const int partner = (j == (k >> 1)) ? (t ^ (k - 1)) : (t ^ j);
          if (partner > t) {
            const unsigned long long a = s[t], b = s[partner];
            if (b < a) {
              s[t] = b;
              s[partner] = a;
            }
          }
        }
        __syncthreads();
      }
    }
    for (int t = threadIdx.x; t < len; t += kCooThreads) kr[t] = s[t];
    __syncthreads();  // s is reused by the next row
  }
}

// Rows longer than kBlockSortMax (rare): one block per listed row runs the
// same network over the row in global memory.
__global__ void __launch_bounds__(1024)
coo_sort_global_kernel(const int32_t *__restrict__ list, const int64_t *__restrict__ seg,
                       const int32_t *__restrict__ counts,
                       unsigned long long *__restrict__ keys) {
  const int32_t n = list[0];
  for (int32_t i = blockIdx.x; i < n; i += gridDim.x) {
    const int32_t r = list[1 + i];
    const int64_t len = counts[r];
    unsigned long long *kr = keys + seg[r];
    int64_t p2 = 1;
    while (p2 < len) p2 <<= 1;
    for (int64_t k = 2; k <= p2; k <<= 1) {
      for (int64_t j = k >> 1; j > 0; j >>= 1) {
        for (int64_t t = threadIdx.x; t < len; t += blockDim.x) {
          const int64_t partner = (j == (k >> 1)) ? (t ^ (k - 1)) : (t ^ j);
          if (partner > t && partner < len) {
            const unsigned long long a = kr[t], b = kr[partner];
            if (b < a) {
              kr[t] = b;
              kr[partner] = a;
            }
          }
        }
        __syncthreads();
      }
    }
  }
}

__device__ __forceinline__ int32_t key_col(unsigned long long x) {
  return static_cast<int32_t>(x >> 32);
}

// Runs (distinct columns) per row: warp per row.
__global__ void __launch_bounds__(kCooThreads)
coo_runs_kernel(int32_t rows, const int64_t *__restrict__ seg,
                const int32_t *__restrict__ counts, const unsigned long long *__restrict__ keys,
                int32_t *__restrict__ runs) {
  const int64_t w = (int64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
  if (w >= rows) return;
  const int lane = lane_id();
  const int32_t r = static_cast<int32_t>(w);
  const int32_t len = counts[r];
  const unsigned long long *kr = keys + seg[r];
  int32_t n = 0;
  for (int32_t p = lane; p < len; p += 32)
    n += (p == 0 || key_col(kr[p]) != key_col(kr[p - 1])) ? 1 : 0;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) n += __shfl_xor_sync(kFull, n, o);
  if (lane == 0) runs[r] = n;
}

// One output per run: its column, and its values summed in index order from
// the first (file entries index val directly; a mirror carries its source's
// index with the top bit set).
__global__ void __launch_bounds__(kCooThreads)
coo_write_kernel(int32_t rows, const int64_t *__restrict__ seg,
                 const int32_t *__restrict__ counts, const unsigned long long *__restrict__ keys,
                 const float *__restrict__ val, const int64_t *__restrict__ out_off,
                 int32_t *__restrict__ c_col, float *__restrict__ c_val) {
  const int64_t w = (int64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
  if (w >= rows) return;
  const int lane = lane_id();
  const int32_t r = static_cast<int32_t>(w);
  const int32_t len = counts[r];
  const unsigned long long *kr = keys + seg[r];
  int64_t out = out_off[r];
  for (int32_t p0 = 0; p0 < len; p0 += 32) {
    const int32_t p = p0 + lane;
    bool head = false;
    unsigned long long x = 0;
    if (p < len) {
      x = kr[p];
      head = p == 0 || key_col(x) != key_col(kr[p - 1]);
    }
    const unsigned mask = __ballot_sync(kFull, head);
    if (head) {
      const int32_t c = key_col(x);
      float acc = __ldg(val + (static_cast<uint32_t>(x) & ~kMirrorBit));
      for (int32_t q = p + 1; q < len; ++q) {
        const unsigned long long y = kr[q];
        if (key_col(y) != c) break;
        acc = __fadd_rn(acc, __ldg(val + (static_cast<uint32_t>(y) & ~kMirrorBit)));
      }
      const int64_t at = out + __popc(mask & ((1u << lane) - 1));
      c_col[at] = c;
      c_val[at] = acc;
    }
    out += __popc(mask);
  }
}

__global__ void __launch_bounds__(kCooThreads)
coo_row_ptr_kernel(int32_t rows, const int64_t *__restrict__ off, int64_t total,
                   int32_t *__restrict__ c_rp) {
  const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i < rows) c_rp[i] = static_cast<int32_t>(off[i]);
  if (i == rows) c_rp[i] = static_cast<int32_t>(total);
}

int grid_for(int64_t n, int per_block) {
  int64_t g = (n + per_block - 1) / per_block;
  if (g < 1) g = 1;
  if (g > 148 * 32) g = 148 * 32;
  return static_cast<int>(g);
}

int warp_grid(int32_t rows) {
  return static_cast<int>((int64_t(rows) * 32 + kCooThreads - 1) / kCooThreads);
}

rvsp_status_t status_of(cudaError_t e) {
  if (e == cudaSuccess) return RVSP_SUCCESS;
  return e == cudaErrorMemoryAllocation ? RVSP_ERROR_ALLOCATION_FAILED : RVSP_ERROR_DEVICE;
}

// A stream-ordered memory pool per device, owned by this file: the
// canonicalisation's scratch (a few buffers per call, tens of MB for large
// files) comes from it, and up to kPoolKeepBytes stay reserved between calls,
// so repeated reads pay no cudaMalloc / cudaFree (which synchronise and map
// or unmap pages).  Created on first use on each device.
constexpr int kMaxDevices = 64;
constexpr unsigned long long kPoolKeepBytes = 1ull << 30;
cudaMemPool_t g_pool[kMaxDevices] = {};
std::once_flag g_pool_once[kMaxDevices];

cudaMemPool_t scratch_pool() {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return nullptr;
  std::call_once(g_pool_once[dev], [dev] {
    cudaMemPoolProps props = {};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = dev;
    cudaMemPool_t pool = nullptr;
    if (cudaMemPoolCreate(&pool, &props) == cudaSuccess) {
      unsigned long long keep = kPoolKeepBytes;
      cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
      g_pool[dev] = pool;
    } else {
      cudaGetLastError();
    }
  });
  return g_pool[dev];
}

// Device scratch of one call, from the pool (cudaMalloc when the pool could
// not be made), released in stream order when the call returns.
struct Scratch {
  static constexpr int kSlots = 16;
  void *p[kSlots] = {};
  int n = 0;
  cudaStream_t s = nullptr;
  cudaMemPool_t pool = nullptr;
  explicit Scratch(cudaStream_t st) : s(st), pool(scratch_pool()) {}
  cudaError_t alloc(void **out, size_t bytes) {
    if (n >= kSlots) return cudaErrorMemoryAllocation;  // more buffers than slots
    const size_t b = bytes ? bytes : 1;
    cudaError_t e = pool ? cudaMallocFromPoolAsync(out, b, pool, s) : cudaMalloc(out, b);
    if (e == cudaSuccess) p[n++] = *out;
    return e;
  }
  ~Scratch() {
    for (int i = 0; i < n; ++i) {
      if (pool) cudaFreeAsync(p[i], s);
      else cudaFree(p[i]);
    }
  }
};

}  // namespace

}  // namespace rvsp

using namespace rvsp;

extern "C" rvsp_status_t rvsp_cuda_coo_to_csr(void *stream, int32_t rows, int32_t cols,
                                              int64_t n, int symmetric, const int32_t *row,
                                              const int32_t *col, const float *val,
                                              int32_t *c_row_ptr, int32_t **c_col_out,
                                              float **c_val_out, int32_t *c_nnz_out) {
  if (!c_row_ptr || !c_col_out || !c_val_out || !c_nnz_out) return RVSP_ERROR_NULL_POINTER;
  if (n > 0 && (!row || !col || !val)) return RVSP_ERROR_NULL_POINTER;
  if (rows < 0 || cols < 0 || n < 0 || n > int64_t(INT32_MAX))
    return RVSP_ERROR_INVALID_ARGUMENT;
  *c_col_out = nullptr;
  *c_val_out = nullptr;
  *c_nnz_out = 0;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  Scratch sc(s);
  int32_t *counts = nullptr, *cursor = nullptr, *flags = nullptr, *mid = nullptr, *big = nullptr;
  int64_t *seg = nullptr, *partials = nullptr, *total = nullptr;
  const size_t nr = size_t(rows) + 1;
  cudaError_t e = sc.alloc(reinterpret_cast<void **>(&counts), nr * sizeof(int32_t));
  if (e == cudaSuccess) e = sc.alloc(reinterpret_cast<void **>(&cursor), nr * sizeof(int32_t));
  if (e == cudaSuccess) e = sc.alloc(reinterpret_cast<void **>(&flags), sizeof(int32_t));
  if (e == cudaSuccess) e = sc.alloc(reinterpret_cast<void **>(&mid), nr * sizeof(int32_t));
  if (e == cudaSuccess) e = sc.alloc(reinterpret_cast<void **>(&big), nr * sizeof(int32_t));
  if (e == cudaSuccess) e = sc.alloc(reinterpret_cast<void **>(&seg), nr * sizeof(int64_t));
  if (e == cudaSuccess)
    e = sc.alloc(reinterpret_cast<void **>(&partials), scan_partials_bytes(rows + 1));
  if (e == cudaSuccess) e = sc.alloc(reinterpret_cast<void **>(&total), sizeof(int64_t));
  if (e != cudaSuccess) return status_of(e);
  cudaMemsetAsync(counts, 0, nr * sizeof(int32_t), s);
  cudaMemsetAsync(cursor, 0, nr * sizeof(int32_t), s);
  cudaMemsetAsync(flags, 0, sizeof(int32_t), s);
  cudaMemsetAsync(mid, 0, sizeof(int32_t), s);
  cudaMemsetAsync(big, 0, sizeof(int32_t), s);
  if (n > 0)
    coo_count_kernel<<<grid_for(n, kCooThreads), kCooThreads, 0, s>>>(
        n, rows, cols, row, col, symmetric, counts, flags);
  launch_scan_i64(rows, counts, seg, partials, total, s);
  int32_t bad = 0;
  int64_t entries = 0;
  e = cudaMemcpyAsync(&bad, flags, sizeof(int32_t), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(&entries, total, sizeof(int64_t), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return status_of(e);
  if (bad) return RVSP_ERROR_INVALID_CSR;
  if (rows == 0 || entries == 0) {  // no entries: row_ptr of zeros, 1-entry arrays
    int32_t *c_col = nullptr;
    float *c_val = nullptr;
    cudaMemsetAsync(c_row_ptr, 0, nr * sizeof(int32_t), s);
    e = cudaMalloc(reinterpret_cast<void **>(&c_col), sizeof(int32_t));
    if (e == cudaSuccess) e = cudaMalloc(reinterpret_cast<void **>(&c_val), sizeof(float));
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) {
      cudaFree(c_col);
      cudaFree(c_val);
      return status_of(e);
    }
    *c_col_out = c_col;
    *c_val_out = c_val;
    return RVSP_SUCCESS;
  }
  unsigned long long *keys = nullptr;
  e = sc.alloc(reinterpret_cast<void **>(&keys), size_t(entries) * sizeof(unsigned long long));
  if (e != cudaSuccess) return status_of(e);
  coo_scatter_kernel<<<grid_for(n, kCooThreads), kCooThreads, 0, s>>>(n, row, col, symmetric,
                                                                       seg, cursor, keys);
  coo_sort_warp_kernel<<<warp_grid(rows), kCooThreads, 0, s>>>(rows, seg, counts, keys, mid,
                                                                big);
  coo_sort_block_kernel<<<148 * 4, kCooThreads, 0, s>>>(mid, seg, counts, keys);
  coo_sort_global_kernel<<<148, 1024, 0, s>>>(big, seg, counts, keys);
  // runs per row (into cursor), their scan, the output arrays
  coo_runs_kernel<<<warp_grid(rows), kCooThreads, 0, s>>>(rows, seg, counts, keys, cursor);
  int64_t *runs_off = nullptr;
  e = sc.alloc(reinterpret_cast<void **>(&runs_off), nr * sizeof(int64_t));
  if (e != cudaSuccess) return status_of(e);
  launch_scan_i64(rows, cursor, runs_off, partials, total, s);
  int64_t nnz = 0;
  e = cudaMemcpyAsync(&nnz, total, sizeof(int64_t), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return status_of(e);
  if (nnz > int64_t(INT32_MAX)) return RVSP_ERROR_ALLOCATION_FAILED;
  int32_t *c_col = nullptr;
  float *c_val = nullptr;
  e = cudaMalloc(reinterpret_cast<void **>(&c_col), size_t(nnz) * sizeof(int32_t));
  if (e == cudaSuccess) e = cudaMalloc(reinterpret_cast<void **>(&c_val), size_t(nnz) * sizeof(float));
  if (e != cudaSuccess) {
    cudaFree(c_col);
    return status_of(e);
  }
  coo_write_kernel<<<warp_grid(rows), kCooThreads, 0, s>>>(rows, seg, counts, keys, val,
                                                            runs_off, c_col, c_val);
  coo_row_ptr_kernel<<<static_cast<unsigned>((int64_t(rows) + kCooThreads) / kCooThreads),
                       kCooThreads, 0, s>>>(rows, runs_off, nnz, c_row_ptr);
  e = cudaStreamSynchronize(s);
  if (e == cudaSuccess) e = cudaGetLastError();
  if (e != cudaSuccess) {
    cudaFree(c_col);
    cudaFree(c_val);
    return status_of(e);
  }
  *c_col_out = c_col;
  *c_val_out = c_val;
  *c_nnz_out = static_cast<int32_t>(nnz);
  return RVSP_SUCCESS;
}
