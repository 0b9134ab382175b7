// Numeric pass: C values, and (fill mode) C's sorted column indices.
//
// Replaces rvsp_symbolic_fill + rvsp_sort_columns (rvsp_symbolic.c:91-137,
// rvsp_sort.h:106-122) and the Gustavson numeric pass
// (gustavson_core_f32.inc:18-64, accum_scalar_f32.c:20-71).
//
// Order.  The reference adds the terms of each output entry in ascending
// A-nonzero order into an accumulator that starts at +0.0f, rounding the
// product and the sum separately.  Every class here keeps that order exactly:
//
//   M<K>    one thread merges the row's sorted B rows (k_merge.cu).
//   W<T>    warp per row.  "Stepping": one A nonzero at a time, lanes over
//           its B row (distinct columns), __syncwarp between A nonzeros.
//           "Tiles" (short B rows): 32 flattened products at a time; lanes
//           that hit the same accumulator are ranked by lane (= A order) and
//           applied in rounds (ordered_apply).
//   B8192   256-thread block, one A nonzero at a time, barrier between.
//   DENSE   512-thread block, same stepping, dense accumulator in global
//           memory that each row leaves zeroed.
//
// Fill mode emits columns sorted: hash classes compact their (col, value)
// pairs and bitonic-sort them (in registers up to 128 pairs a warp, else in
// shared memory); the dense class walks its column bitmap in order.  Reuse mode (columns already in C) maps column -> position through
// a hash of C's row and writes the values coalesced.
#include <climits>

#include "device_common.cuh"
#include "kernels.cuh"

namespace rvsp {

namespace {

constexpr int kSteppingMinAvgLen = 16;  // avg B row length that favours stepping

// ---- product walkers for warp-per-row classes --------------------------------

// A walker's `stop` functor is called with the warp converged after each A
// nonzero (stepping) or each tile (tiles); it returns a warp-uniform bool and
// true ends the walk.  The plain path never stops (NoStop).
struct NoStop {
  __device__ __forceinline__ bool operator()() const { return false; }
};

// Stepping: f(col, term) for each entry of A nonzero p's B row, lanes over
// the B row, __syncwarp after each A nonzero.
template <typename F, typename S = NoStop>
__device__ __forceinline__ void warp_stepping(const Operands &op, int32_t p0,
                                              int32_t p1, F f, S stop = S()) {
  const int lane = lane_id();
  for (int32_t p = p0; p < p1; p += 32) {
    const AChunk c = load_chunk(op.a_col, op.a_val, op.b_rp, p + lane, p1, true);
    const int cnt = min(32, p1 - p);
    for (int jj = 0; jj < cnt; ++jj) {
      const int len = __shfl_sync(kFull, c.len, jj);
      const int bbeg = __shfl_sync(kFull, c.bbeg, jj);
      const float a = __shfl_sync(kFull, c.a, jj);
      for (int e = lane; e < len; e += 32) {
        const int32_t col = __ldg(op.b_col + bbeg + e);
        f(col, __fmul_rn(a, __ldg(op.b_val + bbeg + e)));
      }
      __syncwarp();
      if (stop()) return;
    }
  }
}

// Tiles: g(valid, col, term) for 32 flattened products at a time (all lanes
// call g, invalid ones with valid == false).
template <typename G, typename S = NoStop>
__device__ __forceinline__ void warp_tiles(const Operands &op, int32_t p0,
                                           int32_t p1, G g, S stop = S()) {
  const int lane = lane_id();
  for (int32_t p = p0; p < p1; p += 32) {
    const AChunk c = load_chunk(op.a_col, op.a_val, op.b_rp, p + lane, p1, true);
    for (int t0 = 0; t0 < c.total; t0 += 32) {
      const int t = t0 + lane;
      const bool v = t < c.total;
      const int j = warp_owner_of(c.incl, v ? t : 0);
      const int excl = __shfl_sync(kFull, c.incl - c.len, j);
      const int bbeg = __shfl_sync(kFull, c.bbeg, j);
      const float a = __shfl_sync(kFull, c.a, j);
      int32_t col = 0;
      float term = 0.0f;
      if (v) {
        const int32_t bp = bbeg + (t - excl);
        col = __ldg(op.b_col + bp);
        term = __fmul_rn(a, __ldg(op.b_val + bp));
      }
      g(v, col, term);
      if (stop()) return;
    }
  }
}

__device__ __forceinline__ bool use_stepping(const int64_t *ops, int32_t row,
                                             int32_t nnz_a) {
  return ops[row] >= static_cast<int64_t>(kSteppingMinAvgLen) * nnz_a;
}

// ---- W<T>: warp per row, fill mode --------------------------------------------

// Output of one row in the fill kernels.  Plain: C at c_rp[row] with the
// exact nnz c_rp[row + 1] - c_rp[row].  Fused (kFused): the row's slab slot
// at fo.off[row] with capacity fo.cap[row]; the kernel writes the row's nnz
// to fo.counts[row], or, when the row needs more than its capacity (or its
// table fills), marks it -1, appends it to fo.ovf_rows and writes nothing.
template <bool kFused>
__device__ __forceinline__ int64_t out_begin(const FusedOut &fo, const int32_t *c_rp,
                                             int32_t row) {
  return kFused ? fo.off[row] : static_cast<int64_t>(c_rp[row]);
}
template <bool kFused>
__device__ __forceinline__ int out_limit(const FusedOut &fo, const int32_t *c_rp,
                                         int32_t row) {
  return kFused ? fo.cap[row] : c_rp[row + 1] - c_rp[row];
}
__device__ __forceinline__ void mark_overflow(const FusedOut &fo, int32_t row) {
  fo.counts[row] = -1;
  fo.ovf_rows[atomicAdd(fo.ovf_count, 1)] = row;
}

// Writes a row's kept (column, value) pairs, compacted in sbuf, sorted by
// column: up to 32 R of them are sorted in registers (no shared-memory
// traffic, which bounds this kernel) and the first `out` go to C from out0,
// 32 consecutive entries per store.
template <int R>
__device__ __forceinline__ void write_sorted_regs(const unsigned long long *sbuf, int kept,
                                                  int out, int64_t out0, int32_t *c_col,
                                                  float *c_val) {
  const int lane = lane_id();
  unsigned long long v[R];
#pragma unroll
  for (int r = 0; r < R; ++r) {
    const int e = r * 32 + lane;
    v[r] = e < kept ? sbuf[e] : ~0ull;
  }
  warp_bitonic_sort_regs<R>(v);
#pragma unroll
  for (int r = 0; r < R; ++r) {
    const int e = r * 32 + lane;
    if (e < out) {
      c_col[out0 + e] = packed_col(v[r]);
      c_val[out0 + e] = packed_val(v[r]);
    }
  }
}

// Blocks per SM the fill kernel asks the compiler to fit: 16 (32 registers)
// for W64, W128 and non-fused W256 rows, which fit 16 blocks by shared memory
// too and need no spill at 32 registers; 12 (up to 42) for the others.
constexpr int fill_min_blocks(int log2t, bool fused) {
  return log2t <= 7 || (log2t == 8 && !fused) ? 16 : 12;
}

// Shared memory per warp: sbuf[T/2] u64 | keys[T] i32 | vals[T] f32 = 12 T bytes.
template <int LOG2T, bool kFused>
__global__ void __launch_bounds__(kWarpsPerBlock * 32, fill_min_blocks(LOG2T, kFused))
num_warp_fill_kernel(Operands op, const int64_t *__restrict__ ops,
                     const int32_t *__restrict__ rows, int32_t nrows,
                     const int32_t *__restrict__ c_rp, int32_t *__restrict__ c_col,
                     float *__restrict__ c_val, int32_t *__restrict__ status,
                     FusedOut fo) {
  constexpr int T = 1 << LOG2T, H = T / 2;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  unsigned char *base = smem_raw + size_t(threadIdx.x >> 5) * (12 * T);
  unsigned long long *sbuf = reinterpret_cast<unsigned long long *>(base);
  int32_t *keys = reinterpret_cast<int32_t *>(base + 4 * T);
  float *vals = reinterpret_cast<float *>(base + 8 * T);

  const int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (w >= nrows) return;
  const int lane = lane_id();
  fill_words(keys, T, 0xffffffffu, lane, 32);
  fill_words(vals, T, 0u, lane, 32);  // +0.0f
  __syncwarp();
  const int32_t row = row_of(rows, w);
  const int32_t p0 = op.a_rp[row], p1 = op.a_rp[row + 1];
  const int64_t out0 = out_begin<kFused>(fo, c_rp, row);
  const int m = out_limit<kFused>(fo, c_rp, row);
  bool bad = false;
  int my_new = 0;     // distinct columns this lane created (stepping)
  int total_new = 0;  // distinct columns so far (tiles; warp-uniform)
  bool over = false;  // fused: the row outgrew its capacity (warp-uniform)
  if (use_stepping(ops, row, p1 - p0)) {
    warp_stepping(
        op, p0, p1,
        [&](int32_t col, float term) {
          bool created;
          const int s = hash_insert(keys, LOG2T, col, created);
          if (s >= 0) vals[s] = __fadd_rn(vals[s], term);
          else bad = true;
          my_new += created;
        },
        [&]() {
          if (!kFused) return false;
          over = warp_sum(my_new) > m || __any_sync(kFull, bad);
          return over;
        });
  } else {
    warp_tiles(
        op, p0, p1,
        [&](bool v, int32_t col, float term) {
          int s = -1;
          bool created = false;
          if (v) {
            s = hash_insert(keys, LOG2T, col, created);
            if (s < 0) bad = true;
          }
          total_new += __popc(__ballot_sync(kFull, created));
          ordered_apply(vals, v && s >= 0, s, term);
        },
        [&]() {
          if (!kFused) return false;
          over = total_new > m || __any_sync(kFull, bad);
          return over;
        });
  }
  __syncwarp();
  if (kFused && over) {
    if (lane == 0) mark_overflow(fo, row);
    return;
  }

  // Compact the occupied slots, sort by column, write the row.
  int n = 0;
  for (int s0 = 0; s0 < T; s0 += 32) {
    const int s = s0 + lane;
    const int32_t key = keys[s];
    const bool occ = key != kEmpty;
    const unsigned msk = __ballot_sync(kFull, occ);
    const int pos = n + __popc(msk & lanemask_lt());
    if (occ && pos < H) sbuf[pos] = pack_col_val(key, vals[s]);
    n += __popc(msk);
  }
  const int kept = n < H ? n : H;
  const int out = kept < m ? kept : m;
  __syncwarp();
  if (kept <= 32) {
    write_sorted_regs<1>(sbuf, kept, out, out0, c_col, c_val);
  } else if (H >= 64 && kept <= 64) {
    write_sorted_regs<2>(sbuf, kept, out, out0, c_col, c_val);
  } else if (H >= 128 && kept <= 128) {
    write_sorted_regs<4>(sbuf, kept, out, out0, c_col, c_val);
  } else {
    int npow = 1;
    while (npow < kept) npow <<= 1;
    for (int e = kept + lane; e < npow; e += 32) sbuf[e] = ~0ull;
    __syncwarp();
    warp_bitonic_sort(sbuf, npow);
    for (int e = lane; e < out; e += 32) {
      const unsigned long long x = sbuf[e];
      c_col[out0 + e] = packed_col(x);
      c_val[out0 + e] = packed_val(x);
    }
  }
  const bool any_bad = __any_sync(kFull, bad);
  if (lane == 0) {
    if (kFused) {
      fo.counts[row] = n;
    } else {
      if (any_bad) report(status, kDevHashFull);
      if (n != m) report(status, kDevCountMismatch);
    }
  }
}

// ---- W<T>: warp per row, reuse mode -------------------------------------------

// Shared memory per warp: keys[T] i32 | posv[T] i32 | acc[T/2] f32 = 10 T bytes.
template <int LOG2T>
__global__ void __launch_bounds__(kWarpsPerBlock * 32)
num_warp_reuse_kernel(Operands op, const int64_t *__restrict__ ops,
                      const int32_t *__restrict__ rows, int32_t nrows,
                      const int32_t *__restrict__ c_rp,
                      const int32_t *__restrict__ c_col,
                      float *__restrict__ c_val, int32_t *__restrict__ status) {
  constexpr int T = 1 << LOG2T;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  unsigned char *base = smem_raw + size_t(threadIdx.x >> 5) * (10 * T);
  int32_t *keys = reinterpret_cast<int32_t *>(base);
  int32_t *posv = reinterpret_cast<int32_t *>(base + 4 * T);
  float *acc = reinterpret_cast<float *>(base + 8 * T);

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
    acc[e] = 0.0f;
  }
  __syncwarp();
  const int32_t p0 = op.a_rp[row], p1 = op.a_rp[row + 1];
  bool missing = false;
  if (use_stepping(ops, row, p1 - p0)) {
    warp_stepping(op, p0, p1, [&](int32_t col, float term) {
      const int s = hash_find(keys, LOG2T, col);
      if (s >= 0) {
        const int pos = posv[s];
        acc[pos] = __fadd_rn(acc[pos], term);
      } else {
        missing = true;
      }
    });
  } else {
    warp_tiles(op, p0, p1, [&](bool v, int32_t col, float term) {
      int pos = -1;
      if (v) {
        const int s = hash_find(keys, LOG2T, col);
        if (s >= 0) pos = posv[s];
        else missing = true;
      }
      ordered_apply(acc, v && pos >= 0, pos, term);
    });
  }
  __syncwarp();
  for (int e = lane; e < m; e += 32) c_val[cs + e] = acc[e];
  const bool any_bad = __any_sync(kFull, bad);
  const bool any_missing = __any_sync(kFull, missing);
  if (lane == 0) {
    if (any_bad) report(status, kDevHashFull);
    if (any_missing) report(status, kDevKeyMissing);
  }
}

// ---- block-per-row stepping helpers ------------------------------------------

constexpr int kAStage = 256;  // A nonzeros staged in shared memory at a time

struct AStage {
  int32_t bbeg[kAStage];
  int32_t len[kAStage];
  float a[kAStage];
};

// f(col, term) for every product of the row, one A nonzero at a time across
// the whole block, with a barrier between A nonzeros.  stop() is evaluated
// after each barrier and must return the same value on every thread.
template <typename F, typename S = NoStop>
__device__ __forceinline__ void block_stepping(const Operands &op, int32_t p0,
                                               int32_t p1, AStage &st, F f,
                                               S stop = S()) {
  for (int32_t p = p0; p < p1; p += kAStage) {
    const int cnt = min(kAStage, p1 - p);
    __syncthreads();
    for (int q = threadIdx.x; q < cnt; q += blockDim.x) {
      const int32_t k = __ldg(op.a_col + p + q);
      st.a[q] = __ldg(op.a_val + p + q);
      const int32_t b0 = __ldg(op.b_rp + k);
      st.bbeg[q] = b0;
      st.len[q] = __ldg(op.b_rp + k + 1) - b0;
    }
    __syncthreads();
    for (int q = 0; q < cnt; ++q) {
      const int32_t bbeg = st.bbeg[q];
      const int32_t len = st.len[q];
      const float a = st.a[q];
      for (int32_t e = threadIdx.x; e < len; e += blockDim.x) {
        const int32_t col = __ldg(op.b_col + bbeg + e);
        f(col, __fmul_rn(a, __ldg(op.b_val + bbeg + e)));
      }
      __syncthreads();
      if (stop()) return;
    }
  }
}

// ---- B8192: block per row -------------------------------------------------------

// Shared memory: sbuf[4096] u64 | keys[8192] i32 | vals[8192] f32 (96 KiB) in
// fill mode; keys | posv | acc[4096] (80 KiB) in reuse mode.
template <bool kFill, bool kFused>
__global__ void __launch_bounds__(kBlockHashThreads)
num_block_kernel(Operands op, const int32_t *__restrict__ rows,
                 const int32_t *__restrict__ c_rp, int32_t *__restrict__ c_col,
                 float *__restrict__ c_val, int32_t *__restrict__ status,
                 FusedOut fo) {
  constexpr int LOG2T = kBlockHashLog2, T = 1 << LOG2T, H = T / 2;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ AStage st;
  __shared__ int32_t s_n, s_flags, s_new;
  unsigned long long *sbuf = reinterpret_cast<unsigned long long *>(smem_raw);
  int32_t *keys = reinterpret_cast<int32_t *>(smem_raw + (kFill ? 4 * T : 0));
  float *vals = reinterpret_cast<float *>(smem_raw + 8 * T);           // fill
  int32_t *posv = reinterpret_cast<int32_t *>(smem_raw + 4 * T);       // reuse
  float *acc = reinterpret_cast<float *>(smem_raw + 8 * T);            // reuse

  const int32_t row = row_of(rows, blockIdx.x);
  const int64_t cs = out_begin<kFused>(fo, c_rp, row);
  const int m = out_limit<kFused>(fo, c_rp, row);
  fill_words(keys, T, 0xffffffffu, threadIdx.x, blockDim.x);
  if (kFill) fill_words(vals, T, 0u, threadIdx.x, blockDim.x);  // +0.0f
  if (threadIdx.x == 0) {
    s_n = 0;
    s_flags = 0;
    s_new = 0;
  }
  __syncthreads();
  int flags = 0;
  if (!kFill) {
    for (int e = threadIdx.x; e < m; e += blockDim.x) {
      bool created;
      const int s = hash_insert(keys, LOG2T, __ldg(c_col + cs + e), created);
      if (s >= 0) posv[s] = e;
      else flags |= 1;
      acc[e] = 0.0f;
    }
  }
  const int32_t p0 = op.a_rp[row], p1 = op.a_rp[row + 1];
  block_stepping(
      op, p0, p1, st,
      [&](int32_t col, float term) {
        if (kFill) {
          bool created;
          const int s = hash_insert(keys, LOG2T, col, created);
          if (s >= 0) vals[s] = __fadd_rn(vals[s], term);
          else flags |= 1;
          if (kFused) {
            if (created) atomicAdd(&s_new, 1);
            if (s < 0) atomicOr(&s_flags, 1);
          }
        } else {
          const int s = hash_find(keys, LOG2T, col);
          if (s >= 0) {
            const int pos = posv[s];
            acc[pos] = __fadd_rn(acc[pos], term);
          } else {
            flags |= 2;
          }
        }
      },
      [&]() { return kFused && (s_new > m || (s_flags & 1)); });
  if (kFused) {
    // The row outgrew its predicted capacity (or its table): leave it to the
    // plain path.  s_new and s_flags are read after the last barrier.
    if (s_new > m || (s_flags & 1)) {
      if (threadIdx.x == 0) mark_overflow(fo, row);
      return;
    }
  }
  if (flags) atomicOr(&s_flags, flags);
  if (kFill) {
    // Compact occupied slots (any order), then sort by column.
    for (int s = threadIdx.x; s < T; s += blockDim.x) {
      const int32_t key = keys[s];
      const bool occ = key != kEmpty;
      const unsigned msk = __ballot_sync(kFull, occ);
      int wbase = 0;
      if (lane_id() == 0 && msk) wbase = atomicAdd(&s_n, __popc(msk));
      wbase = __shfl_sync(kFull, wbase, 0);
      const int pos = wbase + __popc(msk & lanemask_lt());
      if (occ && pos < H) sbuf[pos] = pack_col_val(key, vals[s]);
    }
    __syncthreads();
    const int n = s_n;
    const int kept = n < H ? n : H;
    int npow = 1;
    while (npow < kept) npow <<= 1;
    for (int e = kept + threadIdx.x; e < npow; e += blockDim.x) sbuf[e] = ~0ull;
    __syncthreads();
    block_bitonic_sort(sbuf, npow);
    const int out = kept < m ? kept : m;
    for (int e = threadIdx.x; e < out; e += blockDim.x) {
      const unsigned long long x = sbuf[e];
      c_col[cs + e] = packed_col(x);
      c_val[cs + e] = packed_val(x);
    }
    if (threadIdx.x == 0) {
      if (kFused) fo.counts[row] = n;
      else if (n != m) report(status, kDevCountMismatch);
    }
  } else {
    __syncthreads();
    for (int e = threadIdx.x; e < m; e += blockDim.x) c_val[cs + e] = acc[e];
  }
  __syncthreads();
  if (threadIdx.x == 0 && s_flags) {
    if (s_flags & 1) report(status, kDevHashFull);
    if (s_flags & 2) report(status, kDevKeyMissing);
  }
}

// ---- DENSE: block per row, global dense accumulator ------------------------------

// Fused (kFused, fill only): rows write into their slab slot; the capacity is
// the row's exact upper bound min(ops, b_cols), so a dense row never
// overflows, and its nnz goes to fo.counts[row].
template <bool kFill, bool kSmemBits, bool kFused>
__global__ void __launch_bounds__(kDenseThreads)
num_dense_kernel(Operands op, const int32_t *__restrict__ rows, int32_t nrows,
                 const int32_t *__restrict__ c_rp, int32_t *__restrict__ c_col,
                 float *__restrict__ c_val, float *__restrict__ dense_acc,
                 size_t acc_stride, uint32_t *__restrict__ gbits,
                 size_t bits_stride, int32_t *__restrict__ status, FusedOut fo) {
  extern __shared__ uint32_t smem_u32[];
  __shared__ AStage st;
  __shared__ int32_t s_lo, s_hi, s_total;
  __shared__ int32_t s_scan[kDenseThreads];
  float *acc = dense_acc + acc_stride * blockIdx.x;
  uint32_t *bits = kSmemBits ? smem_u32 : gbits + bits_stride * blockIdx.x;
  const int32_t words = (op.b_cols + 31) >> 5;
  if (kFill && kSmemBits) {
    for (int32_t w = threadIdx.x; w < words; w += blockDim.x) bits[w] = 0u;
  }
  for (int32_t r = blockIdx.x; r < nrows; r += gridDim.x) {
    const int32_t row = row_of(rows, r);
    const int64_t cs = out_begin<kFused>(fo, c_rp, row);
    const int m = out_limit<kFused>(fo, c_rp, row);
    if (threadIdx.x == 0) {
      s_lo = INT_MAX;
      s_hi = -1;
    }
    int lo = INT_MAX, hi = -1;
    block_stepping(op, op.a_rp[row], op.a_rp[row + 1], st,
                   [&](int32_t col, float term) {
                     acc[col] = __fadd_rn(acc[col], term);
                     if (kFill) {
                       atomicOr(&bits[col >> 5], 1u << (col & 31));
                       lo = min(lo, col);
                       hi = max(hi, col);
                     }
                   });
    if (kFill) {
      lo = warp_min(lo);
      hi = warp_max(hi);
      if (lane_id() == 0) {
        atomicMin(&s_lo, lo);
        atomicMax(&s_hi, hi);
      }
      __syncthreads();
      // Walk the bitmap in column order: thread t owns a contiguous run of
      // words; an exclusive scan of per-thread bit counts gives positions.
      const int32_t w0 = s_hi >= 0 ? (s_lo >> 5) : 0;
      const int32_t nw = s_hi >= 0 ? (s_hi >> 5) - w0 + 1 : 0;
      const int32_t per = (nw + blockDim.x - 1) / blockDim.x;
      const int32_t mw0 = w0 + threadIdx.x * per;
      const int32_t mw1 = min(mw0 + per, w0 + nw);
      int cnt = 0;
      for (int32_t w = mw0; w < mw1; ++w) cnt += __popc(bits[w]);
      s_scan[threadIdx.x] = cnt;
      __syncthreads();
      if (threadIdx.x == 0) {
        int run = 0;
        for (int t = 0; t < static_cast<int>(blockDim.x); ++t) {
          const int c = s_scan[t];
          s_scan[t] = run;
          run += c;
        }
        s_total = run;
      }
      __syncthreads();
      int pos = s_scan[threadIdx.x];
      for (int32_t w = mw0; w < mw1; ++w) {
        uint32_t word = bits[w];
        while (word) {
          const int b = __ffs(word) - 1;
          word &= word - 1u;
          const int32_t col = (w << 5) + b;
          if (pos < m) {
            c_col[cs + pos] = col;
            c_val[cs + pos] = acc[col];
          }
          acc[col] = 0.0f;
          ++pos;
        }
        bits[w] = 0u;
      }
      if (threadIdx.x == 0) {
        if (kFused) fo.counts[row] = s_total;
        else if (s_total != m) report(status, kDevCountMismatch);
      }
    } else {
      for (int e = threadIdx.x; e < m; e += blockDim.x) {
        const int32_t col = __ldg(c_col + cs + e);
        c_val[cs + e] = acc[col];
        acc[col] = 0.0f;
      }
    }
    __syncthreads();
  }
}

template <int LOG2T>
void launch_warp(const Operands &op, const int64_t *ops, const int32_t *rows,
                 int32_t nrows, const int32_t *c_rp, int32_t *c_col,
                 float *c_val, bool fill, int32_t *status, const FusedOut *fo,
                 cudaStream_t s) {
  constexpr int T = 1 << LOG2T;
  const int threads = kWarpsPerBlock * 32;
  const int grid = (nrows + kWarpsPerBlock - 1) / kWarpsPerBlock;
  if (fo) {
    const size_t smem = size_t(kWarpsPerBlock) * 12 * T;
    cudaFuncSetAttribute(num_warp_fill_kernel<LOG2T, true>,
                         cudaFuncAttributeMaxDynamicSharedMemorySize,
                         static_cast<int>(smem));
    num_warp_fill_kernel<LOG2T, true><<<grid, threads, smem, s>>>(
        op, ops, rows, nrows, c_rp, c_col, c_val, status, *fo);
  } else if (fill) {
    const size_t smem = size_t(kWarpsPerBlock) * 12 * T;
    cudaFuncSetAttribute(num_warp_fill_kernel<LOG2T, false>,
                         cudaFuncAttributeMaxDynamicSharedMemorySize,
                         static_cast<int>(smem));
    num_warp_fill_kernel<LOG2T, false><<<grid, threads, smem, s>>>(
        op, ops, rows, nrows, c_rp, c_col, c_val, status, FusedOut{});
  } else {
    const size_t smem = size_t(kWarpsPerBlock) * 10 * T;
    cudaFuncSetAttribute(num_warp_reuse_kernel<LOG2T>,
                         cudaFuncAttributeMaxDynamicSharedMemorySize,
                         static_cast<int>(smem));
    num_warp_reuse_kernel<LOG2T><<<grid, threads, smem, s>>>(
        op, ops, rows, nrows, c_rp, c_col, c_val, status);
  }
}

}  // namespace

size_t dense_slot_acc_bytes(int32_t b_cols) {
  if (heavy_fits(b_cols)) return 0;  // the heavy kernels need no global scratch
  const size_t b = size_t(b_cols > 0 ? b_cols : 1) * sizeof(float);
  return (b + 255) & ~size_t(255);
}

size_t dense_slot_bits_bytes(int32_t b_cols) {
  if (heavy_fits(b_cols) || b_cols <= kSmemBitmapMaxCols) return 0;
  const size_t b = ((size_t(b_cols) + 31) >> 5) * sizeof(uint32_t);
  return (b + 255) & ~size_t(255);
}

namespace {

template <bool kFill, bool kFused>
void launch_block(const Operands &op, const int32_t *rows, int32_t nrows,
                  const int32_t *c_rp, int32_t *c_col, float *c_val, int32_t *status,
                  const FusedOut &fo, cudaStream_t s) {
  constexpr int T = 1 << kBlockHashLog2;
  const size_t smem = size_t(kFill ? 12 : 10) * T;
  cudaFuncSetAttribute(num_block_kernel<kFill, kFused>,
                       cudaFuncAttributeMaxDynamicSharedMemorySize,
                       static_cast<int>(smem));
  num_block_kernel<kFill, kFused><<<nrows, kBlockHashThreads, smem, s>>>(
      op, rows, c_rp, c_col, c_val, status, fo);
}

template <bool kFill, bool kSmemBits, bool kFused>
void launch_dense(const Operands &op, const int32_t *rows, int32_t nrows,
                  const int32_t *c_rp, int32_t *c_col, float *c_val, float *dense_acc,
                  uint32_t *dense_bits, int32_t dense_slots, int32_t *status,
                  const FusedOut &fo, cudaStream_t s) {
  const size_t acc_stride = dense_slot_acc_bytes(op.b_cols) / sizeof(float);
  const size_t bits_stride = dense_slot_bits_bytes(op.b_cols) / sizeof(uint32_t);
  const int grid = nrows < dense_slots ? nrows : dense_slots;
  size_t smem = 0;
  if (kFill && kSmemBits) {
    smem = ((size_t(op.b_cols) + 31) >> 5) * sizeof(uint32_t);
    cudaFuncSetAttribute(num_dense_kernel<kFill, kSmemBits, kFused>,
                         cudaFuncAttributeMaxDynamicSharedMemorySize,
                         static_cast<int>(smem));
  }
  num_dense_kernel<kFill, kSmemBits, kFused><<<grid, kDenseThreads, smem, s>>>(
      op, rows, nrows, c_rp, c_col, c_val, dense_acc, acc_stride,
      kSmemBits ? nullptr : dense_bits, kSmemBits ? 0 : bits_stride, status, fo);
}

}  // namespace

void launch_numeric_class(int cls, const Operands &op, const int64_t *ops,
                          const int32_t *rows, int32_t nrows,
                          const int32_t *c_rp, int32_t *c_col, float *c_val,
                          bool fill, float *dense_acc, uint32_t *dense_bits,
                          int32_t dense_slots, int32_t *status, int num_sms,
                          cudaStream_t s, const FusedOut *fo) {
  if (nrows <= 0) return;
  if ((cls == kB8192 || cls == kDense) && heavy_fits(op.b_cols)) {
    launch_heavy_numeric(op, rows, nrows, c_rp, c_col, c_val, fill, status, fo, num_sms, s);
    return;
  }
  const FusedOut none{};
  switch (cls) {
    case kM4:
    case kM8:
    case kM16:
      launch_merge_numeric(cls, op, rows, nrows, c_rp, c_col, c_val, fill, status, fo, s);
      break;
    case kW64: launch_warp<6>(op, ops, rows, nrows, c_rp, c_col, c_val, fill, status, fo, s); break;
    case kW128: launch_warp<7>(op, ops, rows, nrows, c_rp, c_col, c_val, fill, status, fo, s); break;
    case kW256: launch_warp<8>(op, ops, rows, nrows, c_rp, c_col, c_val, fill, status, fo, s); break;
    case kW512: launch_warp<9>(op, ops, rows, nrows, c_rp, c_col, c_val, fill, status, fo, s); break;
    case kW1024: launch_warp<10>(op, ops, rows, nrows, c_rp, c_col, c_val, fill, status, fo, s); break;
    case kW2048: launch_warp<11>(op, ops, rows, nrows, c_rp, c_col, c_val, fill, status, fo, s); break;
    case kB8192:
      if (fo) launch_block<true, true>(op, rows, nrows, c_rp, c_col, c_val, status, *fo, s);
      else if (fill) launch_block<true, false>(op, rows, nrows, c_rp, c_col, c_val, status, none, s);
      else launch_block<false, false>(op, rows, nrows, c_rp, c_col, c_val, status, none, s);
      break;
    case kDense: {
      const bool smem_bits = op.b_cols <= kSmemBitmapMaxCols;
      if (fo && smem_bits)
        launch_dense<true, true, true>(op, rows, nrows, c_rp, c_col, c_val, dense_acc,
                                       dense_bits, dense_slots, status, *fo, s);
      else if (fo)
        launch_dense<true, false, true>(op, rows, nrows, c_rp, c_col, c_val, dense_acc,
                                        dense_bits, dense_slots, status, *fo, s);
      else if (fill && smem_bits)
        launch_dense<true, true, false>(op, rows, nrows, c_rp, c_col, c_val, dense_acc,
                                        dense_bits, dense_slots, status, none, s);
      else if (fill)
        launch_dense<true, false, false>(op, rows, nrows, c_rp, c_col, c_val, dense_acc,
                                         dense_bits, dense_slots, status, none, s);
      else
        launch_dense<false, false, false>(op, rows, nrows, c_rp, c_col, c_val, dense_acc,
                                          dense_bits, dense_slots, status, none, s);
      break;
    }
    default: break;
  }
}

}  // namespace rvsp
