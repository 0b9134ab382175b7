// Heavy rows: the B8192 and DENSE classes when B has at most kHeavyMaxCols
// columns (wider B keeps the hash and global-memory kernels of k_symbolic.cu
// and k_numeric.cu).
//
// One 512-thread block per row, rows strided over a grid of one or two blocks
// per SM.  A row's A nonzeros are staged 512 at a time with a block prefix of
// their B row lengths, and the stage's products, in flattened order
// (ascending A nonzero, then B position), are spread evenly over all 512
// threads: a row of few A nonzeros that select long B rows (the hubs of a
// power-law matrix) keeps the whole block busy.  A thread finds the A nonzero
// of flattened product q by binary search over the staged prefix.
//
// The row's output columns are marked in a shared-memory bitmap; a bit is
// read before it is set, so the hot columns of power-law rows cost broadcast
// loads instead of contended atomics.  The symbolic pass (count half of
// rvsp_symbolic_count, rvsp_symbolic.c:27-73) counts the bits.
//
// The numeric pass turns the bitmap into output positions.  With gpre[g] the
// exclusive count of set bits before 128-column group g, column j sits at
// index gpre[j/128] + (bits set in the words of its group before its own) +
// popc(word & bits below j) of the sorted output row.  Fill mode writes the
// columns by walking the bitmap in order (rvsp_symbolic_fill + the sort of
// rvsp_sort_columns, rvsp_symbolic.c:91-137); reuse mode marks the bitmap
// from C's own columns.  Values accumulate at their output position in a
// shared-memory window of acc_cap positions; a row with more outputs makes
// one pass over its products per window.
//
// Order.  Each stage of A nonzeros is applied one of two ways, chosen by its
// mean B row length.  Long rows step: one A nonzero at a time, the block over
// its B row (distinct columns), a barrier between A nonzeros.  Short rows
// tile: products in flattened order, 2048 at a time, stably partitioned to
// the 16 warps by the low 4 bits of the output position, so one warp makes
// every update of a given position; each warp applies its share 32 at a time
// with ordered_apply (equal positions in lane order).  Either way each output
// entry receives its terms in ascending A-nonzero order, starting from +0.0f,
// each product and sum rounded separately: the order and rounding of
// gustavson_core_f32.inc:31-62 with accum_scalar_f32.c:20-71.
#include <climits>

#include "device_common.cuh"
#include "kernels.cuh"

namespace rvsp {

namespace {

constexpr int kHT = kDenseThreads;            // 512 threads
constexpr int kHW = kHT / 32;                 // 16 warps = 16 column buckets
constexpr int kHRounds = 4;                   // products per thread per tile
constexpr int kHTile = kHT * kHRounds;        // 2048 products per tile
constexpr int kHStage = kHT;                  // A nonzeros staged at a time
constexpr int kHCnt = kHRounds * kHW * kHW;   // partition table entries
constexpr int kStepMinAvgLen = 64;            // mean B row length that steps

// A stage of up to kHStage A nonzeros of one row.
struct StageShared {
  long long incl[kHStage];   // inclusive prefix of the B row lengths
  int32_t bbeg[kHStage];     // B row start
  float a[kHStage];          // A value (numeric pass)
  long long wsum64[kHW];
  long long total;
};

struct HeavyShared {
  StageShared st;
  int32_t cnt[kHCnt];        // [round][warp][bucket]: counts, then offsets
  int32_t icol[kHTile];      // the tile's positions, partitioned by bucket
  float iterm[kHTile];
  int32_t wsum[kHW];
  int32_t bstart[kHW + 1];
  int32_t lo, hi, n;
};

// Words of the bitmap rounded up to 16, so that the bitmap and the group
// prefix array (one int per 4 words) both stay 16-byte multiples.
__host__ __device__ inline int32_t heavy_words16(int32_t b_cols) {
  const int32_t words = (b_cols + 31) >> 5;
  return (words + 15) & ~15;
}

// Exclusive block prefix of one int per thread; *total = block sum.  Every
// thread of the block must call it.
__device__ __forceinline__ int heavy_scan(int v, HeavyShared &sh, int *total) {
  const int lane = lane_id(), w = threadIdx.x >> 5;
  const int incl = warp_incl_scan(v);
  if (lane == 31) sh.wsum[w] = incl;
  __syncthreads();
  if (w == 0) {
    const int x = lane < kHW ? sh.wsum[lane] : 0;
    const int xi = warp_incl_scan(x);
    if (lane < kHW) sh.wsum[lane] = xi - x;
    if (lane == 31) sh.n = xi;
  }
  __syncthreads();
  *total = sh.n;
  return sh.wsum[w] + incl - v;
}

// First index i in [0, n) with c[i] >= key (n if none); c sorted.
__device__ __forceinline__ int32_t lower_bound_col(const int32_t *__restrict__ c,
                                                   int32_t n, int32_t key) {
  int32_t lo = 0, hi = n;
  while (lo < hi) {
    const int32_t mid = (lo + hi) >> 1;
    if (__ldg(c + mid) < key) lo = mid + 1;
    else hi = mid;
  }
  return lo;
}

// Stages A nonzeros [pc, min(pc + kHStage, p1)) and returns their product
// count; the stage is visible to the whole block on return.  With a window
// (c_lo <= c_hi), each B row is cut to its entries in columns [c_lo, c_hi],
// which are contiguous since B's rows are sorted.  Every thread must call it,
// and no thread may still read the previous stage.
template <bool kValues>
__device__ __forceinline__ long long heavy_stage(const Operands &op, int32_t pc,
                                                 int32_t p1, StageShared &st,
                                                 int32_t c_lo = 0, int32_t c_hi = -1) {
  const int tid = threadIdx.x, lane = lane_id(), w = tid >> 5;
  const int na = min(kHStage, p1 - pc);
  int len = 0;
  int32_t bb = 0;
  float av = 0.0f;
  if (tid < na) {
    const int32_t k = __ldg(op.a_col + pc + tid);
    if (kValues) av = __ldg(op.a_val + pc + tid);
    bb = __ldg(op.b_rp + k);
    len = __ldg(op.b_rp + k + 1) - bb;
    if (c_lo <= c_hi && len > 0) {
      const int32_t s = lower_bound_col(op.b_col + bb, len, c_lo);
      const int32_t e = s + lower_bound_col(op.b_col + bb + s, len - s, c_hi + 1);
      bb += s;
      len = e - s;
    }
  }
  long long x = len;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const long long n = __shfl_up_sync(kFull, x, o);
    if (lane >= o) x += n;
  }
  if (lane == 31) st.wsum64[w] = x;
  __syncthreads();
  if (w == 0) {
    const long long y = lane < kHW ? st.wsum64[lane] : 0;
    long long yi = y;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const long long n = __shfl_up_sync(kFull, yi, o);
      if (lane >= o) yi += n;
    }
    if (lane < kHW) st.wsum64[lane] = yi - y;
    if (lane == 31) st.total = yi;
  }
  __syncthreads();
  st.incl[tid] = st.wsum64[w] + x;
  st.bbeg[tid] = bb;
  if (kValues) st.a[tid] = av;
  const long long total = st.total;
  __syncthreads();
  return total;
}

// B position of flattened product q < total of the stage, and (j) the staged
// A nonzero it belongs to: the first j with incl[j] > q.  Entries past the
// stage's end hold incl = total, so j stays inside the stage.
__device__ __forceinline__ int32_t heavy_locate(const StageShared &st, long long q,
                                                int &j) {
  j = 0;
#pragma unroll
  for (int s = kHStage / 2; s >= 1; s >>= 1)
    if (st.incl[j + s - 1] <= q) j += s;
  const long long ex = j ? st.incl[j - 1] : 0;
  return st.bbeg[j] + static_cast<int32_t>(q - ex);
}

// Marks the columns of A row [p0, p1)'s products in bits; lo / hi = this
// thread's smallest and largest column (INT_MAX / -1 if none).
__device__ __forceinline__ void heavy_mark(const Operands &op, int32_t p0, int32_t p1,
                                           uint32_t *bits, StageShared &st, int &lo,
                                           int &hi) {
  auto mark = [&](int32_t col) {
    uint32_t *wp = bits + (col >> 5);
    const uint32_t bit = 1u << (col & 31);
    if (!(*reinterpret_cast<volatile uint32_t *>(wp) & bit)) atomicOr(wp, bit);
    lo = min(lo, col);
    hi = max(hi, col);
  };
  for (int32_t pc = p0; pc < p1; pc += kHStage) {
    const long long total = heavy_stage<false>(op, pc, p1, st);
    const int na = min(kHStage, p1 - pc);
    if (total >= static_cast<long long>(kStepMinAvgLen) * na) {
      // long B rows: each one strided over the block (no order needed, so
      // no barrier between them)
      for (int j = 0; j < na; ++j) {
        const long long ex = j ? st.incl[j - 1] : 0;
        const int32_t len = static_cast<int32_t>(st.incl[j] - ex);
        const int32_t bb = st.bbeg[j];
        for (int32_t e = threadIdx.x; e < len; e += kHT) mark(__ldg(op.b_col + bb + e));
      }
    } else {
      for (long long q = threadIdx.x; q < total; q += kHT) {
        int j;
        mark(__ldg(op.b_col + heavy_locate(st, q, j)));
      }
    }
    __syncthreads();  // the next stage overwrites this one
  }
}

// Block-wide min / max of the threads' lo / hi into *s_lo / *s_hi (which
// thread 0 set to INT_MAX / -1 before the last barrier).
__device__ __forceinline__ void heavy_range(int lo, int hi, int32_t *s_lo, int32_t *s_hi) {
  lo = warp_min(lo);
  hi = warp_max(hi);
  if (lane_id() == 0) {
    atomicMin(s_lo, lo);
    atomicMax(s_hi, hi);
  }
}

__device__ __forceinline__ void heavy_overflow(const FusedOut &fo, int32_t row) {
  fo.counts[row] = -1;
  fo.ovf_rows[atomicAdd(fo.ovf_count, 1)] = row;
}

// Bit position of the n-th (from 0) set bit of w; n < popc(w).
__device__ __forceinline__ int nth_set_bit(uint32_t w, int n) {
  int pos = 0;
#pragma unroll
  for (int s = 16; s >= 1; s >>= 1) {
    const int c = __popc(w & ((1u << s) - 1u));
    if (n >= c) {
      n -= c;
      w >>= s;
      pos += s;
    }
  }
  return pos;
}

__device__ __forceinline__ int popc4(const uint4 q) {
  return __popc(q.x) + __popc(q.y) + __popc(q.z) + __popc(q.w);
}

// Position of col in the sorted output row; present = its bit is set.
__device__ __forceinline__ int heavy_rank(const uint32_t *bits, const int32_t *gpre,
                                          int32_t col, bool &present) {
  const int g = col >> 7;
  const uint4 q = reinterpret_cast<const uint4 *>(bits)[g];
  const int wi = (col >> 5) & 3;
  const uint32_t w = wi == 0 ? q.x : wi == 1 ? q.y : wi == 2 ? q.z : q.w;
  present = (w >> (col & 31)) & 1u;
  int r = gpre[g] + __popc(w & ((1u << (col & 31)) - 1u));
  if (wi > 0) r += __popc(q.x);
  if (wi > 1) r += __popc(q.y);
  if (wi > 2) r += __popc(q.z);
  return r;
}

// acc[position - wlo] += term for a product whose position falls in the
// window [wlo, wlo + wn); missing = its column is not in the bitmap.
__device__ __forceinline__ void heavy_add(const uint32_t *bits, const int32_t *gpre,
                                          float *acc, int32_t wlo, int32_t wn,
                                          int32_t col, float term, bool &missing) {
  bool present;
  const int32_t slot = heavy_rank(bits, gpre, col, present) - wlo;
  if (!present) {
    missing = true;
    return;
  }
  if (static_cast<uint32_t>(slot) < static_cast<uint32_t>(wn))
    acc[slot] = __fadd_rn(acc[slot], term);
}

// Stepping, for stages of long B rows: one staged A nonzero at a time, the
// block over its B row (whose columns are distinct, so no two threads touch
// one accumulator), a barrier between A nonzeros.  Each thread's first entry
// of the next B row is loaded while the current one is applied.
__device__ __forceinline__ void heavy_steps(const Operands &op, const StageShared &st,
                                            int na, const uint32_t *bits,
                                            const int32_t *gpre, float *acc, int32_t wlo,
                                            int32_t wn, bool &missing) {
  const int tid = threadIdx.x;
  int32_t nc = 0;
  float nv = 0.0f;
  if (tid < static_cast<int32_t>(st.incl[0])) {
    nc = __ldg(op.b_col + st.bbeg[0] + tid);
    nv = __ldg(op.b_val + st.bbeg[0] + tid);
  }
  for (int j = 0; j < na; ++j) {
    const long long ex = j ? st.incl[j - 1] : 0;
    const int32_t len = static_cast<int32_t>(st.incl[j] - ex);
    const int32_t bb = st.bbeg[j];
    const float a = st.a[j];
    const int32_t c0 = nc;
    const float v0 = nv;
    if (j + 1 < na && tid < static_cast<int32_t>(st.incl[j + 1] - st.incl[j])) {
      nc = __ldg(op.b_col + st.bbeg[j + 1] + tid);
      nv = __ldg(op.b_val + st.bbeg[j + 1] + tid);
    }
    if (tid < len) heavy_add(bits, gpre, acc, wlo, wn, c0, __fmul_rn(a, v0), missing);
    for (int32_t e = tid + kHT; e < len; e += kHT)
      heavy_add(bits, gpre, acc, wlo, wn, __ldg(op.b_col + bb + e),
                __fmul_rn(a, __ldg(op.b_val + bb + e)), missing);
    __syncthreads();
  }
}

// Tiles, for stages of short B rows: 2048 flattened products at a time,
// stably partitioned to the warps by output position (low 4 bits), each warp
// applying its share in order with ordered_apply.  Products outside the
// window are dropped at the partition.
__device__ __forceinline__ void heavy_tiles(const Operands &op, HeavyShared &sh,
                                            long long total, const uint32_t *bits,
                                            const int32_t *gpre, float *acc, int32_t wlo,
                                            int32_t wn, bool &missing) {
  const int tid = threadIdx.x, lane = lane_id(), wid = tid >> 5;
  for (long long t0 = 0; t0 < total; t0 += kHTile) {
    for (int e = tid; e < kHCnt; e += kHT) sh.cnt[e] = 0;
    __syncthreads();
    int32_t slot[kHRounds];
    float term[kHRounds];
    int rk[kHRounds], bk[kHRounds];
#pragma unroll
    for (int i = 0; i < kHRounds; ++i) {
      const long long q = t0 + i * kHT + tid;
      bool v = q < total;
      slot[i] = 0;
      term[i] = 0.0f;
      if (v) {
        int j;
        const int32_t bp = heavy_locate(sh.st, q, j);
        bool present;
        slot[i] = heavy_rank(bits, gpre, __ldg(op.b_col + bp), present) - wlo;
        if (!present) {
          missing = true;
          v = false;
        } else if (static_cast<uint32_t>(slot[i]) >= static_cast<uint32_t>(wn)) {
          v = false;
        } else {
          term[i] = __fmul_rn(sh.st.a[j], __ldg(op.b_val + bp));
        }
      }
      bk[i] = v ? (slot[i] & (kHW - 1)) : kHW;
      const unsigned peers = __match_any_sync(kFull, bk[i]);
      rk[i] = __popc(peers & lanemask_lt());
      if (v && rk[i] == 0) sh.cnt[(i * kHW + wid) * kHW + bk[i]] = __popc(peers);
    }
    __syncthreads();
    // Offsets in (bucket, round, warp) order, which is flattened order within
    // each bucket.  Entry o = (b * kHRounds + i) * kHW + w.
    const int o0 = 2 * tid;
    const int w0 = o0 % kHW, i0 = (o0 / kHW) % kHRounds, b0 = o0 / (kHW * kHRounds);
    const int x0 = (i0 * kHW + w0) * kHW + b0;
    const int x1 = (i0 * kHW + w0 + 1) * kHW + b0;
    const int v0 = sh.cnt[x0], v1 = sh.cnt[x1];
    int nvalid = 0;
    const int ex = heavy_scan(v0 + v1, sh, &nvalid);
    sh.cnt[x0] = ex;
    sh.cnt[x1] = ex + v0;
    if (o0 % (kHW * kHRounds) == 0) sh.bstart[b0] = ex;
    if (tid == 0) sh.bstart[kHW] = nvalid;
    __syncthreads();
#pragma unroll
    for (int i = 0; i < kHRounds; ++i) {
      if (bk[i] < kHW) {
        const int at = sh.cnt[(i * kHW + wid) * kHW + bk[i]] + rk[i];
        sh.icol[at] = slot[i];
        sh.iterm[at] = term[i];
      }
    }
    __syncthreads();
    const int e0 = sh.bstart[wid], e1 = sh.bstart[wid + 1];
    for (int e = e0; e < e1; e += 32) {
      const bool v = e + lane < e1;
      ordered_apply(acc, v, v ? sh.icol[e + lane] : 0, v ? sh.iterm[e + lane] : 0.0f);
    }
    __syncthreads();  // the next tile (or stage) overwrites the tables
  }
}

__global__ void __launch_bounds__(kHT, 2)
heavy_symbolic_kernel(Operands op, const int32_t *__restrict__ rows, int32_t nrows,
                      int32_t *__restrict__ counts, int32_t words16) {
  extern __shared__ __align__(16) uint32_t hbits[];
  __shared__ StageShared st;
  __shared__ int32_t s_lo, s_hi, s_cnt;
  fill_words(hbits, words16, 0u, threadIdx.x, kHT);
  for (int32_t r = blockIdx.x; r < nrows; r += gridDim.x) {
    if (threadIdx.x == 0) {
      s_lo = INT_MAX;
      s_hi = -1;
      s_cnt = 0;
    }
    __syncthreads();
    const int32_t row = row_of(rows, r);
    int lo = INT_MAX, hi = -1;
    heavy_mark(op, op.a_rp[row], op.a_rp[row + 1], hbits, st, lo, hi);
    heavy_range(lo, hi, &s_lo, &s_hi);
    __syncthreads();
    int cnt = 0;
    if (s_hi >= 0) {
      for (int32_t w = (s_lo >> 5) + threadIdx.x; w <= (s_hi >> 5); w += kHT) {
        cnt += __popc(hbits[w]);
        hbits[w] = 0u;
      }
    }
    cnt = warp_sum(cnt);
    if (lane_id() == 0 && cnt) atomicAdd(&s_cnt, cnt);
    __syncthreads();
    if (threadIdx.x == 0) counts[row] = s_cnt;
  }
}

// kFill: write C's columns (plain: at c_rp[row], exactly c_rp[row+1] -
// c_rp[row] of them; fused: at fo.off[row], up to fo.cap[row], else the row
// overflows).  !kFill: C's columns are given; write values only.
template <bool kFill, bool kFused>
__global__ void __launch_bounds__(kHT, 2)
heavy_numeric_kernel(Operands op, const int32_t *__restrict__ rows, int32_t nrows,
                     const int32_t *__restrict__ c_rp, int32_t *__restrict__ c_col,
                     float *__restrict__ c_val, int32_t *__restrict__ status,
                     FusedOut fo, int32_t words16, int32_t acc_cap) {
  extern __shared__ __align__(16) uint32_t hbits[];
  int32_t *gpre = reinterpret_cast<int32_t *>(hbits + words16);
  float *sacc = reinterpret_cast<float *>(gpre + (words16 >> 2));
  __shared__ HeavyShared sh;
  const int tid = threadIdx.x;
  fill_words(hbits, words16, 0u, tid, kHT);
  bool missing = false;
  for (int32_t r = blockIdx.x; r < nrows; r += gridDim.x) {
    const int32_t row = row_of(rows, r);
    const int32_t p0 = op.a_rp[row], p1 = op.a_rp[row + 1];
    const int64_t cs = kFused ? fo.off[row] : static_cast<int64_t>(c_rp[row]);
    const int32_t lim = kFused ? fo.cap[row] : c_rp[row + 1] - c_rp[row];
    if (tid == 0) {
      sh.lo = INT_MAX;
      sh.hi = -1;
    }
    __syncthreads();
    int lo = INT_MAX, hi = -1;
    if (kFill) {
      heavy_mark(op, p0, p1, hbits, sh.st, lo, hi);
    } else {
      for (int32_t e = tid; e < lim; e += kHT) {
        const int32_t col = __ldg(c_col + cs + e);
        if (static_cast<uint32_t>(col) >= static_cast<uint32_t>(op.b_cols)) {
          missing = true;  // not a column of B: C is not this product's
          continue;
        }
        atomicOr(&hbits[col >> 5], 1u << (col & 31));
        lo = min(lo, col);
        hi = max(hi, col);
      }
    }
    heavy_range(lo, hi, &sh.lo, &sh.hi);
    __syncthreads();
    const int32_t rlo = sh.lo, rhi = sh.hi;
    // Thread tid owns groups [ga, gb) of the row's column range.
    const int32_t g0 = rhi >= 0 ? (rlo >> 7) : 0;
    const int32_t ng = rhi >= 0 ? (rhi >> 7) - g0 + 1 : 0;
    const int32_t per = (ng + kHT - 1) / kHT;
    const int32_t ga = g0 + min(tid * per, ng);
    const int32_t gb = g0 + min(tid * per + per, ng);
    const uint4 *bits4 = reinterpret_cast<const uint4 *>(hbits);
    int mine = 0;
    for (int32_t g = ga; g < gb; ++g) mine += popc4(bits4[g]);
    int m = 0;
    int pos = heavy_scan(mine, sh, &m);
    for (int32_t g = ga; g < gb; ++g) {
      gpre[g] = pos;
      pos += popc4(bits4[g]);
    }
    __syncthreads();  // gpre complete
    // m is block-uniform: so are these branches.
    bool skip = false;
    if (kFused && m > lim) {
      if (tid == 0) heavy_overflow(fo, row);
      skip = true;
    } else if (!kFused && m != lim) {
      if (tid == 0) report(status, kDevCountMismatch);
      skip = true;
    } else if (acc_cap <= 0) {  // the launch found no room for a window
      if (tid == 0) report(status, kDevBadClass);
      skip = true;
    }
    if (!skip) {
      if (kFill) {
        // Columns in order: warp-strided chunks of 32 words (8 groups, so a
        // chunk starts at gpre of its first group), each written with
        // coalesced stores.
        const int lane = lane_id();
        const int32_t wend = (g0 + ng) * 4;
        for (int32_t c0 = g0 * 4 + (tid >> 5) * 32; c0 < wend; c0 += kHW * 32) {
          const int32_t w = c0 + lane;
          const uint32_t word = w < wend ? hbits[w] : 0u;
          const int cnt = __popc(word);
          const int incl = warp_incl_scan(cnt);
          const int n = __shfl_sync(kFull, incl, 31);
          const int32_t base = gpre[c0 >> 2];
          for (int t0 = 0; t0 < n; t0 += 32) {
            const int t = t0 + lane;
            const bool v = t < n;
            const int j = warp_owner_of(incl, v ? t : 0);
            const uint32_t wj = __shfl_sync(kFull, word, j);
            const int before = __shfl_sync(kFull, incl - cnt, j);
            if (v) c_col[cs + base + t] = ((c0 + j) << 5) + nth_set_bit(wj, t - before);
          }
        }
      }
      if (kFused && tid == 0) fo.counts[row] = m;
      // Output positions in windows of acc_cap, each accumulated in shared
      // memory.  A row wider than one window stages each B row cut to the
      // window's columns (read back from C's columns).
      const bool windows = m > acc_cap;
      if (windows) __syncthreads();  // the columns written above
      for (int32_t wlo = 0; wlo < m; wlo += acc_cap) {
        const int32_t wn = min(acc_cap, m - wlo);
        int32_t c_lo = 0, c_hi = -1;
        if (windows) {
          c_lo = c_col[cs + wlo];
          c_hi = c_col[cs + wlo + wn - 1];
        }
        for (int32_t e = tid; e < wn; e += kHT) sacc[e] = 0.0f;
        for (int32_t pc = p0; pc < p1; pc += kHStage) {
          // (heavy_stage's barriers also publish gpre and the zeroed window)
          const long long total = heavy_stage<true>(op, pc, p1, sh.st, c_lo, c_hi);
          const int na = min(kHStage, p1 - pc);
          if (total >= static_cast<long long>(kStepMinAvgLen) * na)
            heavy_steps(op, sh.st, na, hbits, gpre, sacc, wlo, wn, missing);
          else
            heavy_tiles(op, sh, total, hbits, gpre, sacc, wlo, wn, missing);
        }
        __syncthreads();
        for (int32_t e = tid; e < wn; e += kHT) c_val[cs + wlo + e] = sacc[e];
        __syncthreads();  // the next window zeroes the accumulator
      }
    }
    if (rhi >= 0) {
      for (int32_t w = (rlo >> 5) + tid; w <= (rhi >> 5); w += kHT) hbits[w] = 0u;
    }
    __syncthreads();
  }
  if (missing) report(status, kDevKeyMissing);
}

}  // namespace

bool heavy_fits(int32_t b_cols) { return b_cols <= kHeavyMaxCols; }

void launch_heavy_symbolic(const Operands &op, const int32_t *rows, int32_t nrows,
                           int32_t *counts, int num_sms, cudaStream_t s) {
  if (nrows <= 0) return;
  const int32_t words16 = heavy_words16(op.b_cols);
  const size_t smem = size_t(words16) * sizeof(uint32_t);
  cudaFuncSetAttribute(heavy_symbolic_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       static_cast<int>(smem));
  int per_sm = 1;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, heavy_symbolic_kernel, kHT, smem);
  if (per_sm < 1) per_sm = 1;
  const int64_t want = int64_t(num_sms) * per_sm;
  const int grid = nrows < want ? nrows : static_cast<int>(want);
  heavy_symbolic_kernel<<<grid, kHT, smem, s>>>(op, rows, nrows, counts, words16);
}

namespace {

template <bool kFill, bool kFused>
void launch_heavy_numeric_t(const Operands &op, const int32_t *rows, int32_t nrows,
                            const int32_t *c_rp, int32_t *c_col, float *c_val,
                            int32_t *status, const FusedOut &fo, int num_sms,
                            cudaStream_t s) {
  auto kern = heavy_numeric_kernel<kFill, kFused>;
  int dev = 0, optin = 0, per_sm_bytes = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  cudaDeviceGetAttribute(&per_sm_bytes, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev);
  const int32_t words16 = heavy_words16(op.b_cols);
  const size_t fixed = size_t(words16) * sizeof(uint32_t) + size_t(words16);  // bits + gpre
  const size_t stat = sizeof(HeavyShared);
  // Two blocks per SM when that still leaves room for 8192 accumulators,
  // else one block with the largest accumulator that fits.
  const size_t half = size_t(per_sm_bytes) / 2;
  const size_t two = half > stat + 1024 ? half - stat - 1024 : 0;
  size_t dyn = 0;
  if (two >= fixed + 8192 * sizeof(float)) {
    dyn = two;
  } else {
    dyn = size_t(optin) > stat ? size_t(optin) - stat : 0;
  }
  dyn &= ~size_t(15);
  const int32_t acc_cap = dyn > fixed ? static_cast<int32_t>((dyn - fixed) / sizeof(float)) : 0;
  cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(dyn));
  int per_sm = 1;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kHT, dyn);
  if (per_sm < 1) per_sm = 1;
  const int64_t want = int64_t(num_sms) * per_sm;
  const int grid = nrows < want ? nrows : static_cast<int>(want);
  kern<<<grid, kHT, dyn, s>>>(op, rows, nrows, c_rp, c_col, c_val, status, fo, words16,
                              acc_cap);
}

}  // namespace

void launch_heavy_numeric(const Operands &op, const int32_t *rows, int32_t nrows,
                          const int32_t *c_rp, int32_t *c_col, float *c_val, bool fill,
                          int32_t *status, const FusedOut *fo, int num_sms,
                          cudaStream_t s) {
  if (nrows <= 0) return;
  if (fo)
    launch_heavy_numeric_t<true, true>(op, rows, nrows, c_rp, c_col, c_val, status, *fo,
                                       num_sms, s);
  else if (fill)
    launch_heavy_numeric_t<true, false>(op, rows, nrows, c_rp, c_col, c_val, status,
                                        FusedOut{}, num_sms, s);
  else
    launch_heavy_numeric_t<false, false>(op, rows, nrows, c_rp, c_col, c_val, status,
                                         FusedOut{}, num_sms, s);
}

}  // namespace rvsp
