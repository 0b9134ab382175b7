// Thread-per-row K-way merge for rows with few A nonzeros and modest work.
//
// Row i of C is the merge of the B rows its A nonzeros select, each scaled by
// its A value.  B rows are sorted (canonical CSR), so one thread can produce
// row i's columns in ascending order by repeatedly taking the smallest head
// among the K lists: no hash table, no sort, no shared memory.  When several
// lists share the smallest head column, their terms are added in list order,
// which is ascending A-nonzero order, into an accumulator that starts at
// +0.0f, with __fmul_rn / __fadd_rn.  That is exactly the order and rounding
// of the reference scalar backend (gustavson_core_f32.inc:31-62 with
// accum_scalar_f32.c:20-71), and the emitted columns are its sorted fill
// (rvsp_symbolic.c:91-137).
//
// The per-list state lives in registers: every loop over lists is unrolled
// over K and guarded by j < k.  Each list also holds its NEXT entry (column,
// and value in the numeric pass), loaded when the list advances and used
// only at its following advance, so the merge loop never waits on a load it
// has just issued.
#include <climits>

#include "device_common.cuh"
#include "kernels.cuh"
#include "merge_lists.cuh"

namespace rvsp {

namespace {

using namespace merge;

// Blocks per SM the merge kernels ask the compiler to fit: the register
// budget of K lists (the numeric pass also keeps two values per list).  The
// numeric M8 kernel asks for 7 (72 registers, no spill): at 8 it spilled, and
// measured 3% slower on 5-nonzero rows.
template <int K, bool kValues>
struct MergeOccupancy {
  static constexpr int value = kValues ? (K <= 4 ? 12 : K <= 8 ? 7 : 4)
                                       : (K <= 4 ? 16 : K <= 8 ? 10 : 6);
};

template <int K>
constexpr int merge_class_of() {
  return K == 4 ? kM4 : K == 8 ? kM8 : kM16;
}

// The narrower list count a class's kernel switches to when all of a warp's
// rows fit it (unused list slots still cost a compare and a select a step).
template <int K>
struct NarrowK {
  static constexpr int value = K == 8 ? 6 : K == 16 ? 12 : K;
};

// The number of distinct columns of one row (the merge without values).
template <int K>
__device__ __forceinline__ int32_t count_row(const Operands &op, int32_t p0, int32_t k) {
  Lists<K> L;
  open_lists<K, false>(op, p0, k, L);
  int32_t n = 0;
  for (;;) {
    const int32_t mn = min_head<K>(L);
    if (mn == INT_MAX) break;
#pragma unroll
    for (int j = 0; j < K; ++j)
      if (L.cur[j] == mn) advance<K, false>(op, L, j);
    ++n;
  }
  return n;
}

// One row's merge with values, its outputs to shared memory (staged) or to
// C; returns the outputs made.
template <int K>
__device__ __forceinline__ int32_t fill_row(const Operands &op, int32_t p0, int32_t k,
                                            int32_t m, bool staged, int32_t *sc, float *sv,
                                            int32_t base, int32_t *c_col, float *c_val,
                                            int64_t out0, bool fill) {
  Lists<K> L;
  open_lists<K, true>(op, p0, k, L);
  int32_t n = 0;
  for (;;) {
    const int32_t mn = min_head<K>(L);
    if (mn == INT_MAX) break;
    float acc = 0.0f;
#pragma unroll
    for (int j = 0; j < K; ++j) {
      if (L.cur[j] == mn) {
        acc = __fadd_rn(acc, __fmul_rn(L.a[j], L.curv[j]));
        advance<K, true>(op, L, j);
      }
    }
    if (n < m) {
      if (staged) {
        sc[base + n] = mn;
        sv[base + n] = acc;
      } else {
        if (fill) c_col[out0 + n] = mn;
        c_val[out0 + n] = acc;
      }
    }
    ++n;
  }
  return n;
}

// Rows: rows[0..nrows) (rows == nullptr: rows 0..nrows).  With sel, rows
// whose sel entry is not this kernel's class are skipped.
template <int K>
__global__ void __launch_bounds__(kMergeThreads, MergeOccupancy<K, false>::value)
merge_symbolic_kernel(Operands op, const int32_t *__restrict__ rows,
                      int32_t nrows, int32_t *__restrict__ counts,
                      const uint8_t *__restrict__ sel, CheckGuard guard) {
  const int32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nrows) return;
  const int32_t row = row_of(rows, t);
  if (sel && sel[row] != merge_class_of<K>()) return;
  if (guard.failed()) return;
  const int32_t p0 = op.a_rp[row];
  const int32_t k = op.a_rp[row + 1] - p0;
  // a warp whose rows all fit fewer lists runs the narrower merge
  constexpr int KN = NarrowK<K>::value;
  if (KN < K && __all_sync(__activemask(), k <= KN))
    counts[row] = count_row<KN>(op, p0, k);
  else
    counts[row] = count_row<K>(op, p0, k);
}

// kFused: the row goes to its slab slot (fo.off[row], capacity fo.cap[row] =
// its op count, an exact upper bound, so it cannot overflow) and its nnz to
// fo.counts[row].
template <int K, bool kFused>
__global__ void __launch_bounds__(kMergeThreads, MergeOccupancy<K, true>::value)
merge_numeric_kernel(Operands op, const int32_t *__restrict__ rows, int32_t nrows,
                     const int32_t *__restrict__ c_rp, int32_t *__restrict__ c_col,
                     float *__restrict__ c_val, bool fill,
                     int32_t *__restrict__ status, FusedOut fo) {
  const int32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nrows) return;
  const int32_t row = row_of(rows, t);
  const int32_t p0 = op.a_rp[row];
  const int32_t k = op.a_rp[row + 1] - p0;
  Lists<K> L;
  open_lists<K, true>(op, p0, k, L);
  const int64_t out0 = kFused ? fo.off[row] : static_cast<int64_t>(c_rp[row]);
  int64_t out = out0;
  const int64_t out_end = kFused ? out0 + fo.cap[row] : static_cast<int64_t>(c_rp[row + 1]);
  for (;;) {
    const int32_t mn = min_head<K>(L);
    if (mn == INT_MAX) break;
    float acc = 0.0f;
#pragma unroll
    for (int j = 0; j < K; ++j) {
      if (L.cur[j] == mn) {
        acc = __fadd_rn(acc, __fmul_rn(L.a[j], L.curv[j]));
        advance<K, true>(op, L, j);
      }
    }
    if (out < out_end) {
      if (fill || kFused) c_col[out] = mn;
      c_val[out] = acc;
    }
    ++out;
  }
  if (kFused) fo.counts[row] = static_cast<int32_t>(out - out0);
  else if (out != out_end) report(status, kDevCountMismatch);
}

// Outputs a warp can stage in shared memory (24 KB a block of 4 warps).
constexpr int kStageOut = 768;

// The non-fused numeric pass: the same merge, order and roundings as
// merge_numeric_kernel, but a warp whose 32 rows have at most kStageOut
// outputs in all writes them to shared memory first and then copies them to
// C together, 32 consecutive outputs per step: the rows of a warp are mostly
// consecutive rows, so the copy writes whole lines instead of 32 scattered
// words per store.  A warp with more outputs writes them directly.
template <int K>
__global__ void __launch_bounds__(kMergeThreads, MergeOccupancy<K, true>::value)
merge_numeric_fill_kernel(Operands op, const int32_t *__restrict__ rows, int32_t nrows,
                          const int32_t *__restrict__ c_rp, int32_t *__restrict__ c_col,
                          float *__restrict__ c_val, bool fill,
                          int32_t *__restrict__ status) {
  __shared__ int32_t s_col[kMergeThreads / 32][kStageOut];
  __shared__ float s_val[kMergeThreads / 32][kStageOut];
  const int32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  const int lane = lane_id(), wb = threadIdx.x >> 5;
  const bool valid = t < nrows;
  int32_t row = 0;
  int64_t out0 = 0, out_end = 0;
  if (valid) {
    row = row_of(rows, t);
    out0 = c_rp[row];
    out_end = c_rp[row + 1];
  }
  const int32_t m = static_cast<int32_t>(out_end - out0);  // <= 2048 in these classes
  const int32_t incl = warp_incl_scan(m);
  const int32_t total = __shfl_sync(kFull, incl, 31);
  const int32_t base = incl - m;
  const bool staged = total <= kStageOut;  // the same in every lane
  int32_t p0 = 0, k = 0;
  if (valid) {
    p0 = op.a_rp[row];
    k = op.a_rp[row + 1] - p0;
  }
  // a warp whose rows all fit fewer lists runs the narrower merge
  constexpr int KN = NarrowK<K>::value;
  const bool narrow = KN < K && __all_sync(kFull, k <= KN);
  if (valid) {
    const int32_t n =
        narrow ? fill_row<KN>(op, p0, k, m, staged, s_col[wb], s_val[wb], base, c_col, c_val,
                              out0, fill)
               : fill_row<K>(op, p0, k, m, staged, s_col[wb], s_val[wb], base, c_col, c_val,
                             out0, fill);
    if (n != m) report(status, kDevCountMismatch);
  }
  if (!staged) return;
  __syncwarp();
  for (int32_t e0 = 0; e0 < total; e0 += 32) {
    const int32_t e = e0 + lane;
    const bool v = e < total;
    const int j = warp_owner_of(incl, v ? e : 0);
    const int64_t dst0 = __shfl_sync(kFull, out0, j);
    const int32_t b = __shfl_sync(kFull, base, j);
    if (v) {
      const int64_t d = dst0 + (e - b);
      if (fill) c_col[d] = s_col[wb][e];
      c_val[d] = s_val[wb][e];
    }
  }
}

template <int K>
void sym(const Operands &op, const int32_t *rows, int32_t nrows, int32_t *counts,
         cudaStream_t s, const uint8_t *sel = nullptr, CheckGuard guard = CheckGuard()) {
  const int grid = (nrows + kMergeThreads - 1) / kMergeThreads;
  merge_symbolic_kernel<K><<<grid, kMergeThreads, 0, s>>>(op, rows, nrows, counts, sel,
                                                           guard);
}

template <int K>
void num(const Operands &op, const int32_t *rows, int32_t nrows, const int32_t *c_rp,
         int32_t *c_col, float *c_val, bool fill, int32_t *status, const FusedOut *fo,
         cudaStream_t s) {
  const int grid = (nrows + kMergeThreads - 1) / kMergeThreads;
  if (fo)
    merge_numeric_kernel<K, true><<<grid, kMergeThreads, 0, s>>>(
        op, rows, nrows, c_rp, c_col, c_val, true, status, *fo);
  else
    merge_numeric_fill_kernel<K><<<grid, kMergeThreads, 0, s>>>(op, rows, nrows, c_rp, c_col,
                                                                c_val, fill, status);
}

}  // namespace

void launch_merge_symbolic(int cls, const Operands &op, const int32_t *rows,
                           int32_t nrows, int32_t *counts, cudaStream_t s) {
  if (nrows <= 0) return;
  switch (cls) {
    case kM4: sym<4>(op, rows, nrows, counts, s); break;
    case kM8: sym<8>(op, rows, nrows, counts, s); break;
    case kM16: sym<16>(op, rows, nrows, counts, s); break;
    default: break;
  }
}

void launch_merge_symbolic_all(const Operands &op, const uint8_t *cls, int32_t a_rows,
                               int32_t *counts, CheckGuard guard, cudaStream_t s) {
  if (a_rows <= 0) return;
  sym<4>(op, nullptr, a_rows, counts, s, cls, guard);
  sym<8>(op, nullptr, a_rows, counts, s, cls, guard);
  sym<16>(op, nullptr, a_rows, counts, s, cls, guard);
}

void launch_merge_numeric(int cls, const Operands &op, const int32_t *rows,
                          int32_t nrows, const int32_t *c_rp, int32_t *c_col,
                          float *c_val, bool fill, int32_t *status, const FusedOut *fo,
                          cudaStream_t s) {
  if (nrows <= 0) return;
  switch (cls) {
    case kM4: num<4>(op, rows, nrows, c_rp, c_col, c_val, fill, status, fo, s); break;
    case kM8: num<8>(op, rows, nrows, c_rp, c_col, c_val, fill, status, fo, s); break;
    case kM16: num<16>(op, rows, nrows, c_rp, c_col, c_val, fill, status, fo, s); break;
    default: break;
  }
}

}  // namespace rvsp
