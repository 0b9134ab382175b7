// Device helpers shared by the SpGEMM kernels (sm_100a).
//
// Arithmetic contract.  Every output value is accumulated with separately
// rounded multiply and add (__fmul_rn, __fadd_rn: never contracted into an
// FMA), starting from +0.0f, in ascending A-nonzero order.  That is the order
// and rounding of the reference scalar backend of merledu/rv-sparse
// (src/kernels/spgemm/gustavson_core_f32.inc:31-62 with accum_scalar_f32.c:
// 20-71), so values come out bit-identical.  Parallelism is only ever across
// distinct output columns, or across the entries of one B row (which have
// distinct columns), or is resolved by ordered rounds (see ordered_apply).
//
// Every loop that could spin is bounded; a bound that runs out records an
// error code in the plan's device status word and the kernel skips the work
// instead of trapping or hanging.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace rvsp {

constexpr unsigned kFull = 0xffffffffu;
constexpr int32_t kEmpty = -1;  // empty hash slot

// Device status codes (first error wins).
enum DevStatus : int32_t {
  kDevOk = 0,
  kDevHashFull = 1,       // a hash table ran out of probes
  kDevKeyMissing = 2,     // numeric reuse looked up a column not in C's row
  kDevCountMismatch = 3,  // a row produced a different nnz than analysed
  kDevBadClass = 4,
  kDevWaitTimeout = 5,    // a bounded wait on a copy ran out
};

__device__ __forceinline__ int lane_id() { return threadIdx.x & 31; }

// The t-th row of a class.  A null list means the class holds every row of
// the matrix in order (the plan then skips building the list).
__device__ __forceinline__ int32_t row_of(const int32_t *rows, int32_t t) {
  return rows ? rows[t] : t;
}
__device__ __forceinline__ unsigned lanemask_lt() {
  return (1u << lane_id()) - 1u;
}

__device__ __forceinline__ void report(int32_t *status, int32_t code) {
  atomicCAS(status, 0, code);
}

// Fibonacci hashing: the high bits of col * 2^32/phi; log2t in [5, 16].
__device__ __forceinline__ uint32_t hash_slot(int32_t col, int log2t) {
  return (static_cast<uint32_t>(col) * 0x9E3779B1u) >> (32 - log2t);
}

// Insert col into an open-addressed table of 2^log2t keys (linear probing).
// Returns the slot and whether this call created it; -1 after 2^log2t probes.
__device__ __forceinline__ int hash_insert(int32_t *keys, int log2t,
                                           int32_t col, bool &created) {
  const uint32_t mask = (1u << log2t) - 1u;
  uint32_t h = hash_slot(col, log2t);
  created = false;
  for (uint32_t probe = 0; probe <= mask; ++probe) {
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

// Find col in a table built by hash_insert; -1 if absent.
__device__ __forceinline__ int hash_find(const int32_t *keys, int log2t,
                                         int32_t col) {
  const uint32_t mask = (1u << log2t) - 1u;
  uint32_t h = hash_slot(col, log2t);
  for (uint32_t probe = 0; probe <= mask; ++probe) {
    int32_t cur = keys[h];
    if (cur == col) return static_cast<int>(h);
    if (cur == kEmpty) return -1;
    h = (h + 1u) & mask;
  }
  return -1;
}

// Fills n (a multiple of 4) 32-bit words at p (16-byte aligned) with v using
// 128-bit stores; threads [tid, ...) step by nthreads.
__device__ __forceinline__ void fill_words(void *p, int n, uint32_t v, int tid,
                                           int nthreads) {
  uint4 *q = reinterpret_cast<uint4 *>(p);
  const uint4 x = make_uint4(v, v, v, v);
  for (int i = tid; i < (n >> 2); i += nthreads) q[i] = x;
}

__device__ __forceinline__ int warp_incl_scan(int v) {
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    int n = __shfl_up_sync(kFull, v, o);
    if (lane_id() >= o) v += n;
  }
  return v;
}

__device__ __forceinline__ int warp_sum(int v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(kFull, v, o);
  return v;
}

__device__ __forceinline__ float warp_sum_f(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(kFull, v, o);
  return v;
}

__device__ __forceinline__ long long warp_sum64(long long v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(kFull, v, o);
  return v;
}

__device__ __forceinline__ int warp_max(int v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = max(v, __shfl_xor_sync(kFull, v, o));
  return v;
}

__device__ __forceinline__ int warp_min(int v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = min(v, __shfl_xor_sync(kFull, v, o));
  return v;
}

// Lane j holds the inclusive prefix incl_j of 32 non-decreasing counts.
// Returns, for each lane's t < incl_31, the j with incl_{j-1} <= t < incl_j.
__device__ __forceinline__ int warp_owner_of(int incl, int t) {
  int j = 0;
#pragma unroll
  for (int s = 16; s >= 1; s >>= 1) {
    int v = __shfl_sync(kFull, incl, j + s - 1);
    if (v <= t) j += s;
  }
  return j;
}

// A chunk of up to 32 consecutive A nonzeros of one row, one per lane, with
// the B row each one selects.  Used to expand the row's products ("flattened"
// order = ascending A nonzero, then ascending B position) 32 at a time.
struct AChunk {
  int32_t k;      // B row (A column)
  float a;        // A value
  int32_t bbeg;   // B row start
  int32_t len;    // B row length (0 past the chunk end)
  int32_t incl;   // inclusive prefix of len over lanes
  int32_t total;  // products in this chunk (uniform)
};

__device__ __forceinline__ AChunk load_chunk(const int32_t *__restrict__ a_col,
                                             const float *__restrict__ a_val,
                                             const int32_t *__restrict__ b_rp,
                                             int32_t p, int32_t pend,
                                             bool need_values) {
  AChunk c;
  c.k = 0;
  c.a = 0.0f;
  c.bbeg = 0;
  c.len = 0;
  if (p < pend) {
    c.k = __ldg(a_col + p);
    if (need_values) c.a = __ldg(a_val + p);
    c.bbeg = __ldg(b_rp + c.k);
    c.len = __ldg(b_rp + c.k + 1) - c.bbeg;
  }
  c.incl = warp_incl_scan(c.len);
  c.total = __shfl_sync(kFull, c.incl, 31);
  return c;
}

// Ordered accumulation of one 32-product tile into acc[slot] (shared or
// global memory).  Lanes are in flattened product order, so among lanes that
// hit the same slot the lower lane holds the earlier A nonzero.  The lowest
// lane of each group loads the slot once, adds its own term and then its
// peers' terms in ascending lane order (fetched by shuffle), and stores once:
// the same sequence of roundings as applying the lanes one by one, with one
// memory round trip per group however many terms a hot column collects.
// Invalid lanes pass valid = false.
__device__ __forceinline__ void ordered_apply(float *acc, bool valid, int slot,
                                              float term) {
  const int lane = lane_id();
  const int key = valid ? slot : (-1 - lane);
  const unsigned peers = __match_any_sync(kFull, key);
  const bool leader = valid && (peers & lanemask_lt()) == 0u;
  const unsigned longest = __reduce_max_sync(kFull, valid ? __popc(peers) : 0u);
  float a = 0.0f;
  if (leader) a = __fadd_rn(acc[slot], term);
  unsigned rest = peers & ~(1u << lane);  // the group's later lanes, ascending
  for (unsigned r = 1; r < longest; ++r) {
    const int src = rest ? __ffs(rest) - 1 : lane;
    const float t = __shfl_sync(kFull, term, src);
    if (leader && rest) {
      a = __fadd_rn(a, t);
      rest &= rest - 1u;
    }
  }
  if (leader) acc[slot] = a;
  __syncwarp();
}

// Bitonic sort of n (power of two) 64-bit keys in shared memory by one warp.
// Pair p of a stage with distance j (a power of two) compares i and i + j,
// i = (p / j) * 2j + p % j, computed as p + (p & -j) (no division).
__device__ __forceinline__ void warp_bitonic_sort(unsigned long long *s, int n) {
  for (int k = 2; k <= n; k <<= 1) {
    for (int j = k >> 1; j > 0; j >>= 1) {
      for (int p = lane_id(); p < (n >> 1); p += 32) {
        const int i = p + (p & -j);
        const int l = i + j;
        const unsigned long long x = s[i], y = s[l];
        const bool up = (i & k) == 0;
        if ((x > y) == up) {
          s[i] = y;
          s[l] = x;
        }
      }
      __syncwarp();
    }
  }
}

// Bitonic sort of 32 R 64-bit keys held in registers by one warp: element
// e = 32 r + lane is v[r] of that lane.  Stages with distance j < 32 pair
// lanes (shuffle; the lane with bit j clear holds the lower index and keeps
// the minimum in an ascending block, the maximum in a descending one);
// stages with j >= 32 pair registers r and r | j/32 inside a lane.  No
// shared memory.
template <int R>
__device__ __forceinline__ void warp_bitonic_sort_regs(unsigned long long (&v)[R]) {
  constexpr int N = 32 * R;
  const int lane = lane_id();
#pragma unroll
  for (int k = 2; k <= N; k <<= 1) {
#pragma unroll
    for (int j = k >> 1; j > 0; j >>= 1) {
      if (j >= 32) {
        const int jr = j >> 5;
#pragma unroll
        for (int r = 0; r < R; ++r) {
          if (r & jr) continue;  // r holds the pair's lower index
          const bool up = ((r * 32 + lane) & k) == 0;
          const unsigned long long x = v[r], y = v[r | jr];
          if ((x > y) == up) {
            v[r] = y;
            v[r | jr] = x;
          }
        }
      } else {
        const bool lower = (lane & j) == 0;
#pragma unroll
        for (int r = 0; r < R; ++r) {
          const bool up = ((r * 32 + lane) & k) == 0;
          const unsigned long long y = __shfl_xor_sync(kFull, v[r], j);
          const unsigned long long lo = v[r] < y ? v[r] : y;
          const unsigned long long hi = v[r] < y ? y : v[r];
          v[r] = lower == up ? lo : hi;
        }
      }
    }
  }
}

// Same, by a whole block (n power of two).
__device__ __forceinline__ void block_bitonic_sort(unsigned long long *s, int n) {
  for (int k = 2; k <= n; k <<= 1) {
    for (int j = k >> 1; j > 0; j >>= 1) {
      for (int p = threadIdx.x; p < (n >> 1); p += blockDim.x) {
        const int i = p + (p & -j);
        const int l = i + j;
        const unsigned long long x = s[i], y = s[l];
        const bool up = (i & k) == 0;
        if ((x > y) == up) {
          s[i] = y;
          s[l] = x;
        }
      }
      __syncthreads();
    }
  }
}

__device__ __forceinline__ unsigned long long pack_col_val(int32_t col, float v) {
  return (static_cast<unsigned long long>(static_cast<uint32_t>(col)) << 32) |
         static_cast<unsigned long long>(__float_as_uint(v));
}
__device__ __forceinline__ int32_t packed_col(unsigned long long x) {
  return static_cast<int32_t>(x >> 32);
}
__device__ __forceinline__ float packed_val(unsigned long long x) {
  return __uint_as_float(static_cast<uint32_t>(x & 0xffffffffull));
}

__host__ __device__ constexpr int ilog2_ceil(int v) {
  int l = 0;
  while ((1 << l) < v) ++l;
  return l;
}

}  // namespace rvsp
