// Reuse map: numeric-only repeats of the warp-per-row (W<T>) classes.
//
// A numeric-only compute (structure already in C) must find, for every
// product, the position of its column in C's row; the plain reuse kernel
// does that with a hash of C's row, rebuilt on every call.  The reuse map
// does it once per structure: map[moff[row] + t] is the position in C's row
// of the row's t-th product in flattened order (ascending A nonzero, then B
// position), as uint16 (a W<T> row has at most T/2 <= 1024 outputs).  The
// repeats then skip B's column indices and every hash probe:
//
//   acc[map[k]] += a * b_val      in a shared-memory accumulator of m floats
//
// Order is the plain path's: stepping (one A nonzero at a time, lanes over
// its B row, whose positions are distinct) for long B rows, flattened tiles
// with ordered_apply for short ones; each output receives its terms in
// ascending A-nonzero order from +0.0f, rounded separately
// (gustavson_core_f32.inc:31-62, accum_scalar_f32.c:20-71).
#include <climits>

#include "device_common.cuh"
#include "kernels.cuh"
#include "map_walk.cuh"

namespace rvsp {

namespace {


__global__ void __launch_bounds__(256)
map_ops_kernel(const int32_t *__restrict__ rows, int32_t nrows,
               const int64_t *__restrict__ ops, int32_t *__restrict__ mops,
               int32_t *__restrict__ too_long) {
  const int32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nrows) return;
  const int32_t row = row_of(rows, i);
  const int64_t o = ops[row];
  if (o > INT32_MAX / 2) {
    atomicOr(too_long, 1);
    return;
  }
  mops[row] = static_cast<int32_t>(o);
}

__device__ __forceinline__ unsigned long long map_mix(unsigned long long z) {
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

// Shared memory per warp: keys[T] i32 | posv[T] i32 = 8 T bytes.
// key[row]: a fingerprint of the row's whole map (every (t, position) pair,
// the product count and C's row length); 0 for a row with a missing key.
template <int LOG2T>
__global__ void __launch_bounds__(kWarpsPerBlock * 32)
map_build_kernel(Operands op, const int32_t *__restrict__ rows, int32_t nrows,
                 const int32_t *__restrict__ c_rp, const int32_t *__restrict__ c_col,
                 const int64_t *__restrict__ moff, uint16_t *__restrict__ map,
                 unsigned long long *__restrict__ key, int32_t *__restrict__ status) {
  constexpr int T = 1 << LOG2T;
  extern __shared__ __align__(16) int32_t smem_i32[];
  int32_t *keys = smem_i32 + size_t(threadIdx.x >> 5) * 2 * T;
  int32_t *posv = keys + T;
  const int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (w >= nrows) return;
  const int lane = lane_id();
  fill_words(keys, T, 0xffffffffu, lane, 32);
  __syncwarp();
  const int32_t row = row_of(rows, w);
  const int32_t cs = c_rp[row];
  const int m = c_rp[row + 1] - cs;
  bool bad = false;
  for (int e = lane; e < m; e += 32) {
    bool created;
    const int s = hash_insert(keys, LOG2T, __ldg(c_col + cs + e), created);
    if (s >= 0) posv[s] = e;
    else bad = true;
  }
  __syncwarp();
  const int64_t base = moff[row];
  const int32_t p0 = op.a_rp[row], p1 = op.a_rp[row + 1];
  int64_t run = 0;
  unsigned long long h = 0;
  for (int32_t p = p0; p < p1; p += 32) {
    const AChunk c = load_chunk(op.a_col, op.a_val, op.b_rp, p + lane, p1, false);
    for (int t0 = 0; t0 < c.total; t0 += 32) {
      const int t = t0 + lane;
      const bool v = t < c.total;
      const int j = warp_owner_of(c.incl, v ? t : 0);
      const int excl = __shfl_sync(kFull, c.incl - c.len, j);
      const int bbeg = __shfl_sync(kFull, c.bbeg, j);
      if (v) {
        const int s = hash_find(keys, LOG2T, __ldg(op.b_col + bbeg + (t - excl)));
        if (s < 0) bad = true;
        const uint16_t pos = s >= 0 ? static_cast<uint16_t>(posv[s]) : uint16_t(0xffff);
        map[base + run + t] = pos;
        h += map_mix((static_cast<unsigned long long>(run + t) << 16) | pos);
      }
    }
    run += c.total;
  }
  const bool any_bad = __any_sync(kFull, bad);
  if (any_bad && lane == 0) report(status, kDevKeyMissing);
  if (key) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) h += __shfl_xor_sync(kFull, h, o);
    if (lane == 0) {
      h = map_mix(h ^ map_mix((static_cast<unsigned long long>(run) << 20) ^
                              static_cast<unsigned>(m)));
      key[row] = any_bad ? 0ull : (h ? h : 1ull);
    }
  }
}

// Rows whose maps are identical (a structured matrix repeats a handful of
// position patterns over millions of rows) share one copy: the repeats then
// read a few kilobytes of map from L2 instead of 2 bytes per product from
// HBM.  Step 1: every row's fingerprint into an open-addressed table
// (capacity a power of two, at least twice the rows, so probing ends);
// trow[slot] = the smallest row with that fingerprint.
__global__ void __launch_bounds__(256)
map_dedup_insert_kernel(const int32_t *__restrict__ rows, int32_t nrows,
                        const unsigned long long *__restrict__ key,
                        unsigned long long *__restrict__ tkey, int32_t *__restrict__ trow,
                        unsigned long long mask) {
  const int32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nrows) return;
  const int32_t row = row_of(rows, i);
  const unsigned long long k = key[row];
  if (k == 0) return;
  unsigned long long s = map_mix(k) & mask;
  for (unsigned long long probe = 0; probe <= mask; ++probe, s = (s + 1) & mask) {
    const unsigned long long old = atomicCAS(tkey + s, 0ull, k);
    if (old == 0ull || old == k) {
      atomicMin(trow + s, row);
      return;
    }
  }
}

// Step 2 (warp per row): a row whose canonical row c (smallest row of the
// same fingerprint) has the same product count, the same C row length and,
// compared entry by entry, the same map, points moff[row] at c's map.
// Canonical rows never change their own moff, so reads of moff[c] race with
// nothing.
__global__ void __launch_bounds__(256)
map_dedup_resolve_kernel(const int32_t *__restrict__ rows, int32_t nrows,
                         const unsigned long long *__restrict__ key,
                         const unsigned long long *__restrict__ tkey,
                         const int32_t *__restrict__ trow, unsigned long long mask,
                         const int32_t *__restrict__ c_rp, const int32_t *__restrict__ mops,
                         int64_t *__restrict__ moff, const uint16_t *__restrict__ map,
                         int32_t *__restrict__ shared_rows, int32_t *__restrict__ canon,
                         int32_t *__restrict__ share_count) {
  const int64_t w = (int64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
  if (w >= nrows) return;
  const int lane = lane_id();
  const int32_t row = row_of(rows, static_cast<int32_t>(w));
  const unsigned long long k = key[row];
  if (lane == 0) canon[row] = k == 0 ? -1 : row;
  if (k == 0) return;
  int32_t c = row;
  if (lane == 0) {
    unsigned long long s = map_mix(k) & mask;
    for (unsigned long long probe = 0; probe <= mask; ++probe, s = (s + 1) & mask) {
      const unsigned long long t = tkey[s];
      if (t == k) {
        c = trow[s];
        break;
      }
      if (t == 0ull) break;
    }
  }
  c = __shfl_sync(kFull, c, 0);
  if (c == row || c < 0) return;
  const int32_t n = mops[row];
  if (mops[c] != n || c_rp[c + 1] - c_rp[c] != c_rp[row + 1] - c_rp[row]) return;
  const uint16_t *mine = map + moff[row];
  const uint16_t *theirs = map + moff[c];
  for (int32_t t0 = 0; t0 < n; t0 += 32) {
    const int32_t t = t0 + lane;
    const bool differ = t < n && __ldg(mine + t) != __ldg(theirs + t);
    if (__any_sync(kFull, differ)) return;
  }
  if (lane == 0) {
    moff[row] = moff[c];
    canon[row] = c;
    atomicAdd(shared_rows, 1);
    atomicAdd(share_count + c, 1);
  }
}

// Shared memory per warp: acc[T/2] f32 = 2 T bytes.
template <int LOG2T>
__global__ void __launch_bounds__(kWarpsPerBlock * 32)
map_numeric_kernel(Operands op, const int64_t *__restrict__ ops,
                   const int32_t *__restrict__ rows, int32_t nrows,
                   const int32_t *__restrict__ c_rp, float *__restrict__ c_val,
                   const int64_t *__restrict__ moff, const uint16_t *__restrict__ map,
                   int32_t *__restrict__ status) {
  constexpr int H = 1 << (LOG2T - 1);
  extern __shared__ __align__(16) float smem_f32[];
  float *acc = smem_f32 + size_t(threadIdx.x >> 5) * H;
  const int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (w >= nrows) return;
  map_numeric_row(op, ops, row_of(rows, w), c_rp, c_val, moff, map, status, acc, lane_id());
}

template <int LOG2T>
void launch_build(const Operands &op, const int32_t *rows, int32_t nrows,
                  const int32_t *c_rp, const int32_t *c_col, const int64_t *moff,
                  uint16_t *map, unsigned long long *key, int32_t *status,
                  cudaStream_t s) {
  const size_t smem = size_t(kWarpsPerBlock) * 8 * (size_t(1) << LOG2T);
  cudaFuncSetAttribute(map_build_kernel<LOG2T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       static_cast<int>(smem));
  const int grid = (nrows + kWarpsPerBlock - 1) / kWarpsPerBlock;
  map_build_kernel<LOG2T><<<grid, kWarpsPerBlock * 32, smem, s>>>(
      op, rows, nrows, c_rp, c_col, moff, map, key, status);
}

template <int LOG2T>
void launch_numeric(const Operands &op, const int64_t *ops, const int32_t *rows,
                    int32_t nrows, const int32_t *c_rp, float *c_val, const int64_t *moff,
                    const uint16_t *map, int32_t *status, cudaStream_t s) {
  const size_t smem = size_t(kWarpsPerBlock) * 2 * (size_t(1) << LOG2T);
  const int grid = (nrows + kWarpsPerBlock - 1) / kWarpsPerBlock;
  map_numeric_kernel<LOG2T><<<grid, kWarpsPerBlock * 32, smem, s>>>(
      op, ops, rows, nrows, c_rp, c_val, moff, map, status);
}

}  // namespace

bool map_class(int cls) { return cls >= kW64 && cls <= kW2048; }

void launch_map_ops(const int32_t *rows, int32_t nrows, const int64_t *ops, int32_t *mops,
                    int32_t *too_long, cudaStream_t s) {
  if (nrows <= 0) return;
  map_ops_kernel<<<(nrows + 255) / 256, 256, 0, s>>>(rows, nrows, ops, mops, too_long);
}

void launch_map_build(int cls, const Operands &op, const int32_t *rows, int32_t nrows,
                      const int32_t *c_rp, const int32_t *c_col, const int64_t *moff,
                      uint16_t *map, unsigned long long *key, int32_t *status,
                      cudaStream_t s) {
  if (nrows <= 0) return;
  switch (cls) {
    case kW64: launch_build<6>(op, rows, nrows, c_rp, c_col, moff, map, key, status, s); break;
    case kW128: launch_build<7>(op, rows, nrows, c_rp, c_col, moff, map, key, status, s); break;
    case kW256: launch_build<8>(op, rows, nrows, c_rp, c_col, moff, map, key, status, s); break;
    case kW512: launch_build<9>(op, rows, nrows, c_rp, c_col, moff, map, key, status, s); break;
    case kW1024: launch_build<10>(op, rows, nrows, c_rp, c_col, moff, map, key, status, s); break;
    case kW2048: launch_build<11>(op, rows, nrows, c_rp, c_col, moff, map, key, status, s); break;
    default: break;
  }
}

void launch_map_dedup_insert(const int32_t *rows, int32_t nrows,
                             const unsigned long long *key, unsigned long long *tkey,
                             int32_t *trow, unsigned long long mask, cudaStream_t s) {
  if (nrows <= 0) return;
  map_dedup_insert_kernel<<<(nrows + 255) / 256, 256, 0, s>>>(rows, nrows, key, tkey, trow,
                                                               mask);
}

void launch_map_dedup_resolve(const int32_t *rows, int32_t nrows,
                              const unsigned long long *key,
                              const unsigned long long *tkey, const int32_t *trow,
                              unsigned long long mask, const int32_t *c_rp,
                              const int32_t *mops, int64_t *moff, const uint16_t *map,
                              int32_t *shared_rows, int32_t *canon, int32_t *share_count,
                              cudaStream_t s) {
  if (nrows <= 0) return;
  const int64_t grid = (int64_t(nrows) * 32 + 255) / 256;
  map_dedup_resolve_kernel<<<static_cast<unsigned>(grid), 256, 0, s>>>(
      rows, nrows, key, tkey, trow, mask, c_rp, mops, moff, map, shared_rows, canon,
      share_count);
}

void launch_map_numeric(int cls, const Operands &op, const int64_t *ops, const int32_t *rows,
                        int32_t nrows, const int32_t *c_rp, float *c_val,
                        const int64_t *moff, const uint16_t *map, int32_t *status,
                        cudaStream_t s) {
  if (nrows <= 0) return;
  switch (cls) {
    case kW64: launch_numeric<6>(op, ops, rows, nrows, c_rp, c_val, moff, map, status, s); break;
    case kW128: launch_numeric<7>(op, ops, rows, nrows, c_rp, c_val, moff, map, status, s); break;
    case kW256: launch_numeric<8>(op, ops, rows, nrows, c_rp, c_val, moff, map, status, s); break;
    case kW512: launch_numeric<9>(op, ops, rows, nrows, c_rp, c_val, moff, map, status, s); break;
    case kW1024: launch_numeric<10>(op, ops, rows, nrows, c_rp, c_val, moff, map, status, s); break;
    case kW2048: launch_numeric<11>(op, ops, rows, nrows, c_rp, c_val, moff, map, status, s); break;
    default: break;
  }
}

}  // namespace rvsp
