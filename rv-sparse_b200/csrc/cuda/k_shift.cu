// Shift classes: rows of C that are exact translates of another row.
//
// For a banded or stencil matrix most rows of C = A x B look alike: row i's
// A nonzeros sit at the same offsets from i as row r's at offsets from r, and
// each selects a B row whose columns sit at the same offsets from its own
// index as the matching B row of r.  Then C's row i is C's row r moved by
// i - r: the same count, columns + (i - r), and the same position of every
// product in the row (so the same term table, k_tile.cu / k_pattern.cu).
//
// Classes are found in two levels, each by a 64-bit key, a hash table that
// keeps the smallest row per key, and an entry-by-entry check against that
// row (a row that fails the check stays in a class of its own, so nothing
// rests on the hash):
//
//   B rows: key(len, (column - k) at each position e); bcls[k] = the
//           smallest B row with the same translated columns, else k;
//   rows:   key(nA, (A column - i, bcls of that B row) at each position j);
//           rcls[i] = the smallest row with the same translated A row over
//           the same B classes, else i.
//
// A class of at least min_share rows whose canonical row fits a term table
// (at most 32 A nonzeros, 1024 products and kShiftMaxOut outputs) is a
// pattern: its other rows (members) skip the symbolic pass and the fill,
// take their count from the canonical row, their columns by translation, and
// their values from the term tables built on the canonical row's map.  Every
// value is still summed in ascending A-nonzero order from +0.0f with
// separately rounded products and sums (the reference's order,
// gustavson_core_f32.inc:31-62), so results are bit-identical to the plain
// path.
//
// Whether to look at all is decided on the device: a probe keys rows spread
// over A and one block sorts the keys; the analysis runs when at least half
// of them have a translate among the others and they average enough
// products.  The plan reads that flag (*on) back before it queues the
// passes; every pass also reads it on the device and returns at once when it
// is 0.
//
// The key and check passes give each warp 32 consecutive rows, a lane per
// row, over the rows' column indices staged in the warp's shared memory
// (see SegRows below).
#include <climits>

#include "device_common.cuh"
#include "kernels.cuh"

namespace rvsp {

namespace {

constexpr int kShiftMaxA = 32;
constexpr int kShiftMaxOps = 1024;
constexpr int kShiftMaxOut = 512;    // C entries of a pattern (the term tables' limit)
constexpr int kShiftSamples = 2048;  // rows the probe keys
constexpr int kThreads = 256;

__device__ __forceinline__ unsigned long long mix64(unsigned long long z) {
  z = (z ^ (z >> 31)) * 0x7FB5D329728EA185ull;
  z = (z ^ (z >> 27)) * 0x81DADEF4BC2DD44Dull;
  return z ^ (z >> 33);
}

__device__ __forceinline__ unsigned long long warp_xor64(unsigned long long h) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) h ^= __shfl_xor_sync(kFull, h, o);
  return h;
}

// Key of B row k (warp-wide; every lane returns it).  Never 0.
__device__ __forceinline__ unsigned long long brow_key(const int32_t *__restrict__ b_rp,
                                                       const int32_t *__restrict__ b_col,
                                                       int32_t k, int lane) {
  const int32_t b0 = __ldg(b_rp + k), len = __ldg(b_rp + k + 1) - b0;
  unsigned long long h = 0;
  for (int32_t e = lane; e < len; e += 32) {
    const uint32_t off = static_cast<uint32_t>(__ldg(b_col + b0 + e) - k);
    h ^= mix64((static_cast<unsigned long long>(e) << 32) | off);
  }
  h = warp_xor64(h);
  return mix64(h ^ (static_cast<unsigned long long>(len) * 0x9E3779B97F4A7C15ull)) | 1ull;
}

// A row key's term for A nonzero j at column offset d over a B row whose
// class (or key) is cls_word; the key XORs the terms of all positions.
__device__ __forceinline__ unsigned long long row_term(int32_t j, int32_t d,
                                                       unsigned long long cls_word) {
  return mix64(((static_cast<unsigned long long>(j) << 32) | static_cast<uint32_t>(d)) ^
               (cls_word * 0xD6E8FEB86659FD93ull));
}
__device__ __forceinline__ unsigned long long row_key_of(unsigned long long h, int32_t na) {
  return mix64(h ^ (static_cast<unsigned long long>(na) * 0xA0761D6478BD642Full)) | 1ull;
}

// Row key from per-position terms (lane j < na contributes its A nonzero j).
__device__ __forceinline__ unsigned long long row_key(int32_t na, int lane, int32_t d,
                                                      unsigned long long cls_word) {
  const unsigned long long h = lane < na ? row_term(lane, d, cls_word) : 0ull;
  return row_key_of(warp_xor64(h), na);
}

__device__ __forceinline__ uint32_t key_slot(unsigned long long key, unsigned long long mask) {
  return static_cast<uint32_t>((key * 0x9E3779B97F4A7C15ull) >> 32) & static_cast<uint32_t>(mask);
}

// A row that may join a pattern: 1..32 A nonzeros and at most 1024 products.
__device__ __forceinline__ bool shiftable(int32_t na, int64_t ops) {
  return na > 0 && na <= kShiftMaxA && ops > 0 && ops <= kShiftMaxOps;
}

// Probe: keys of `samples` rows spread over A, computed directly (B keys on
// the fly).  Warp per sampled row.  Reads nothing when the structure check
// queued before it failed.
__global__ void __launch_bounds__(kThreads)
shift_probe_kernel(Operands op, int32_t samples, unsigned long long *__restrict__ keys,
                   CheckGuard guard) {
  const int32_t w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (w >= samples) return;
  const int lane = lane_id();
  if (guard.failed()) {
    if (lane == 0) keys[w] = 0;
    return;
  }
  const int32_t i = static_cast<int32_t>((static_cast<int64_t>(w) * op.a_rows) / samples);
  const int32_t p0 = op.a_rp[i], na = op.a_rp[i + 1] - p0;
  if (na <= 0 || na > kShiftMaxA) {
    // a row of more A nonzeros than a pattern takes counts as a costly row
    if (lane == 0) {
      keys[w] = 0;
      keys[samples + w] = na > 0 ? kShiftMaxOps : 0;
    }
    return;
  }
  int32_t k = 0, len = 0;
  if (lane < na) {
    k = __ldg(op.a_col + p0 + lane);
    len = __ldg(op.b_rp + k + 1) - __ldg(op.b_rp + k);
  }
  unsigned long long mine = 0;
  for (int32_t j = 0; j < na; ++j) {
    const int32_t kj = __shfl_sync(kFull, k, j);
    const unsigned long long bk = brow_key(op.b_rp, op.b_col, kj, lane);
    if (lane == j) mine = bk;
  }
  const unsigned long long key = row_key(na, lane, k - i, mine);
  const int32_t ops = warp_sum(len);
  if (lane == 0) {
    keys[w] = key;
    keys[samples + w] = static_cast<unsigned long long>(ops);
  }
}

// The decision: sorts the probe's keys (one block) and sets *on when at
// least half of the sampled rows share their key with another sampled row
// and the sampled rows average at least min_mean_ops products (the caller's
// bar: rows of few products are cheap on the merge kernels, and the
// analysis and the tile builds would cost more than they save in a single
// product).  *on stays 0 when the structure check failed.
__global__ void __launch_bounds__(1024)
shift_decide_kernel(const unsigned long long *__restrict__ keys, int32_t samples,
                    int32_t min_mean_ops, int32_t *__restrict__ on, CheckGuard guard) {
  __shared__ unsigned long long sk[kShiftSamples];
  __shared__ int32_t dup;
  __shared__ unsigned long long total_ops;
  const int tid = threadIdx.x;
  if (tid == 0) {
    *on = 0;
    dup = 0;
    total_ops = 0;
  }
  if (guard.failed()) return;
  {
    unsigned long long o = 0;
    for (int t = tid; t < samples; t += blockDim.x) o += keys[samples + t];
    for (int d = 16; d; d >>= 1) o += __shfl_xor_sync(kFull, o, d);
    __syncthreads();
    if (lane_id() == 0 && o) atomicAdd(&total_ops, o);
  }
  for (int t = tid; t < kShiftSamples; t += blockDim.x)
    sk[t] = t < samples ? keys[t] : ~0ull;
  __syncthreads();
  block_bitonic_sort(sk, kShiftSamples);
  int mine = 0;
  for (int t = tid; t < samples; t += blockDim.x) {
    const unsigned long long v = sk[t];
    const bool shared = v != 0ull && v != ~0ull &&
                        ((t > 0 && sk[t - 1] == v) || (t + 1 < samples && sk[t + 1] == v));
    mine += shared ? 1 : 0;
  }
  mine = warp_sum(mine);
  if (lane_id() == 0 && mine) atomicAdd(&dup, mine);
  __syncthreads();
  if (tid == 0)
    *on = (2 * dup >= samples &&
           total_ops >= static_cast<unsigned long long>(min_mean_ops) *
                            static_cast<unsigned long long>(samples))
              ? 1
              : 0;
}

// Gated fills.
__global__ void __launch_bounds__(kThreads)
shift_fill64_kernel(const int32_t *__restrict__ on, unsigned long long *__restrict__ p, size_t n,
                    unsigned long long v) {
  if (!*on) return;
  for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
       i += size_t(gridDim.x) * blockDim.x)
    p[i] = v;
}
__global__ void __launch_bounds__(kThreads)
shift_fill32_kernel(const int32_t *__restrict__ on, int32_t *__restrict__ p, size_t n,
                    int32_t v) {
  if (!*on) return;
  for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
       i += size_t(gridDim.x) * blockDim.x)
    p[i] = v;
}

// Rows per warp in the member fill: a warp takes kShiftRows consecutive
// rows and issues each step's loads for all of them before it waits, so one
// warp keeps kShiftRows dependent load chains in flight.
constexpr int kShiftRows = 4;

// The key and resolve passes take 32 consecutive rows per warp, a lane per
// row.  The warp first copies the rows' column indices (one contiguous
// segment of the CSR column array) into its own shared memory with 16-byte
// loads issued together, so the column array leaves HBM once, in coalesced
// lines, and each lane then walks its own row in shared memory.  A segment
// longer than kSegCap entries is read from global memory by the lanes
// instead; B rows longer than kLaneMax entries are keyed and checked
// afterwards by the whole warp, one row at a time (A rows of more than
// kShiftMaxA nonzeros never join a pattern).
constexpr int kSegCap = 1024;                // column indices one warp stages (4 KB)
constexpr int kSegVec = kSegCap / 128;       // 16-byte loads a lane issues for it
constexpr int kBWarps = 8, kAWarps = 4;      // warps per block: B passes, A passes
constexpr int kLaneMax = 64;                 // longest B row one lane walks

// A warp's 32 rows: this lane's row and bounds, and the staged segment.
struct SegRows {
  int64_t r0;    // first row of the warp
  int32_t r;     // this lane's row
  bool live;     // r < rows
  int32_t lo, len;
  int64_t base;  // column position held in seg[0], or -1 (rows read from global)
  int32_t n;     // entries staged, seg[0, n)
};

// The warp's rows and their bounds; the segment's 16-byte loads are issued
// into v (the caller may issue other loads before seg_land stores them).
// base is s0 rounded down to a multiple of four; the whole four-entry groups
// below the segment's end come by 16-byte loads when col is 16-byte aligned,
// the rest by single loads in seg_land; every load stays inside [0, s1).
__device__ __forceinline__ SegRows seg_issue(int32_t rows, int warps,
                                             const int32_t *__restrict__ rp,
                                             const int32_t *__restrict__ col, int lane,
                                             int4 (&v)[kSegVec]) {
  SegRows s;
  s.r0 = (int64_t(blockIdx.x) * warps + (threadIdx.x >> 5)) * 32;
  s.r = static_cast<int32_t>(s.r0) + lane;
  s.live = s.r0 + lane < rows;
  s.lo = s.live ? __ldg(rp + s.r) : 0;
  const int32_t hi = s.live ? __ldg(rp + s.r + 1) : 0;
  s.len = hi - s.lo;
  const int64_t left = rows - s.r0;
  const int last = left < 32 ? static_cast<int>(left) - 1 : 31;
  const int64_t s0 = __shfl_sync(kFull, s.lo, 0), s1 = __shfl_sync(kFull, hi, last);
  s.base = s0 & ~int64_t(3);
  s.n = static_cast<int32_t>(s1 - s.base);
  if (s1 - s.base > kSegCap) {
    s.base = -1;
    s.n = 0;
  } else if ((reinterpret_cast<uintptr_t>(col) & 15u) == 0) {
    const int64_t g0 = s.base >> 2, g1 = s1 >> 2;
    const int4 *vec = reinterpret_cast<const int4 *>(col);
#pragma unroll
    for (int q = 0; q < kSegVec; ++q) {
      const int64_t g = g0 + q * 32 + lane;
      if (g < g1) v[q] = __ldg(vec + g);
    }
  }
  return s;
}

// Stores the loads of seg_issue into seg and fetches the rest of the segment.
__device__ __forceinline__ void seg_land(const SegRows &s, const int32_t *__restrict__ col,
                                         int32_t *seg, int lane, const int4 (&v)[kSegVec]) {
  if (s.base < 0) return;
  const int64_t s1 = s.base + s.n;
  int64_t e = s.base;
  if ((reinterpret_cast<uintptr_t>(col) & 15u) == 0) {
    const int64_t g1 = s1 >> 2;
    int4 *d = reinterpret_cast<int4 *>(seg);
#pragma unroll
    for (int q = 0; q < kSegVec; ++q) {
      const int64_t g = (s.base >> 2) + q * 32 + lane;
      if (g < g1) d[q * 32 + lane] = v[q];
    }
    e = g1 << 2;
  }
  for (int64_t t = e + lane; t < s1; t += 32) seg[t - s.base] = __ldg(col + t);
  __syncwarp();
}

// brow_key's value, computed by one lane over its own row c[0, len).
template <typename P>
__device__ __forceinline__ unsigned long long brow_key_lane(P c, int32_t len, int32_t k) {
  unsigned long long h = 0;
  for (int32_t e = 0; e < len; ++e)
    h ^= mix64((static_cast<unsigned long long>(e) << 32) | static_cast<uint32_t>(c[e] - k));
  return mix64(h ^ (static_cast<unsigned long long>(len) * 0x9E3779B97F4A7C15ull)) | 1ull;
}

// Whether row a (at row index ka) is row b (at kb) moved by ka - kb, entry
// by entry; both rows have len entries.  No early exit, so the loads of
// several entries are in flight together.
template <typename P>
__device__ __forceinline__ bool same_translate(P a, const int32_t *__restrict__ b, int32_t len,
                                               int32_t ka, int32_t kb) {
  bool same = true;
#pragma unroll 4
  for (int32_t e = 0; e < len; ++e) same &= (a[e] - ka == __ldg(b + e) - kb);
  return same;
}

// B row keys, a lane per row.  A B row longer than kShiftMaxOps gets key 0:
// every A row that reaches it has more products than a pattern takes.
__global__ void __launch_bounds__(kBWarps * 32)
shift_bkey_kernel(const int32_t *__restrict__ on, int32_t b_rows,
                  const int32_t *__restrict__ b_rp, const int32_t *__restrict__ b_col,
                  unsigned long long *__restrict__ bkey) {
  __shared__ __align__(16) int32_t segs[kBWarps][kSegCap];
  if (!*on) return;
  if ((int64_t(blockIdx.x) * kBWarps + (threadIdx.x >> 5)) * 32 >= b_rows) return;
  const int lane = lane_id();
  int32_t *seg = segs[threadIdx.x >> 5];
  int4 v[kSegVec];
  const SegRows s = seg_issue(b_rows, kBWarps, b_rp, b_col, lane, v);
  seg_land(s, b_col, seg, lane, v);
  if (s.live && s.len <= kLaneMax)
    bkey[s.r] = s.base >= 0 ? brow_key_lane(seg + (s.lo - s.base), s.len, s.r)
                            : brow_key_lane(b_col + s.lo, s.len, s.r);
  else if (s.live && s.len > kShiftMaxOps)
    bkey[s.r] = 0ull;
  unsigned heavy = __ballot_sync(kFull, s.live && s.len > kLaneMax && s.len <= kShiftMaxOps);
  while (heavy) {
    const int32_t k = static_cast<int32_t>(s.r0) + (__ffs(heavy) - 1);
    heavy &= heavy - 1;
    const unsigned long long key = brow_key(b_rp, b_col, k, lane);
    if (lane == 0) bkey[k] = key;
  }
}

// Inserts every nonzero key into the table (tkey zeroed, trow INT_MAX), the
// slot keeping the smallest row of its key.  Lanes with equal keys make one
// insert (the lowest lane, which holds the smallest row).  The probe loop is
// bounded by the table size (at least twice the keys, so it never fills).
__global__ void __launch_bounds__(kThreads)
shift_insert_kernel(const int32_t *__restrict__ on, int32_t n,
                    const unsigned long long *__restrict__ keys,
                    unsigned long long *__restrict__ tkey, int32_t *__restrict__ trow,
                    unsigned long long mask) {
  if (!*on) return;
  const int32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  const unsigned long long key = i < n ? keys[i] : 0ull;
  const unsigned peers = __match_any_sync(kFull, key);
  if (key == 0ull || (peers & lanemask_lt()) != 0u) return;
  uint32_t s = key_slot(key, mask);
  for (unsigned long long t = 0; t <= mask; ++t) {
    // A slot that already holds the key with a row no larger than i needs
    // no atomics: most rows of a stencil share one key, and most of them
    // arrive after a smaller row of it.
    const unsigned long long seen = *reinterpret_cast<volatile unsigned long long *>(tkey + s);
    if (seen == key) {
      if (*reinterpret_cast<volatile int32_t *>(trow + s) > i) atomicMin(trow + s, i);
      return;
    }
    if (seen == 0ull) {
      const unsigned long long prev = atomicCAS(tkey + s, 0ull, key);
      if (prev == 0ull || prev == key) {
        atomicMin(trow + s, i);
        return;
      }
    }
    s = (s + 1) & static_cast<uint32_t>(mask);
  }
}

// The table's row for key; -1 if not found.
__device__ __forceinline__ int32_t lookup(unsigned long long key,
                                          const unsigned long long *__restrict__ tkey,
                                          const int32_t *__restrict__ trow,
                                          unsigned long long mask) {
  uint32_t s = key_slot(key, mask);
  for (unsigned long long t = 0; t <= mask; ++t) {
    const unsigned long long v = tkey[s];
    if (v == key) return trow[s];
    if (v == 0ull) return -1;
    s = (s + 1) & static_cast<uint32_t>(mask);
  }
  return -1;
}

// bcls[k]: the smallest B row with k's translated columns (checked entry by
// entry), else k.  A lane per row: it looks up the row's key (while the
// segment's loads are in flight) and compares the row with the canonical
// row; B rows longer than kLaneMax are compared by the whole warp.
__global__ void __launch_bounds__(kBWarps * 32)
shift_bresolve_kernel(const int32_t *__restrict__ on, int32_t b_rows,
                      const unsigned long long *__restrict__ bkey,
                      const unsigned long long *__restrict__ tkey,
                      const int32_t *__restrict__ trow, unsigned long long mask,
                      const int32_t *__restrict__ b_rp, const int32_t *__restrict__ b_col,
                      int32_t *__restrict__ bcls) {
  __shared__ __align__(16) int32_t segs[kBWarps][kSegCap];
  if (!*on) return;
  if ((int64_t(blockIdx.x) * kBWarps + (threadIdx.x >> 5)) * 32 >= b_rows) return;
  const int lane = lane_id();
  int32_t *seg = segs[threadIdx.x >> 5];
  int4 v[kSegVec];
  const SegRows s = seg_issue(b_rows, kBWarps, b_rp, b_col, lane, v);
  const unsigned long long key = s.live ? bkey[s.r] : 0ull;
  int32_t c = -1, c0 = 0;
  bool check = false;
  if (key != 0ull) {
    c = lookup(key, tkey, trow, mask);
    if (c >= 0 && c < b_rows && c != s.r) {
      c0 = __ldg(b_rp + c);
      check = __ldg(b_rp + c + 1) - c0 == s.len;
    }
  }
  seg_land(s, b_col, seg, lane, v);
  const bool found = c >= 0 && c < b_rows;
  const bool wide = check && s.len > kLaneMax;
  if (s.live && !wide) {
    bool ok = found && c == s.r;
    if (check)
      ok = s.base >= 0 ? same_translate(seg + (s.lo - s.base), b_col + c0, s.len, s.r, c)
                       : same_translate(b_col + s.lo, b_col + c0, s.len, s.r, c);
    bcls[s.r] = ok ? c : s.r;
  }
  unsigned todo = __ballot_sync(kFull, wide);
  while (todo) {
    const int u = __ffs(todo) - 1;
    todo &= todo - 1;
    const int32_t k = static_cast<int32_t>(s.r0) + u;
    const int32_t cu = __shfl_sync(kFull, c, u), cb = __shfl_sync(kFull, c0, u);
    const int32_t kb = __shfl_sync(kFull, s.lo, u), len = __shfl_sync(kFull, s.len, u);
    bool same = true;
    for (int32_t e = lane; e < len; e += 32)
      same = same && (__ldg(b_col + kb + e) - k) == (__ldg(b_col + cb + e) - cu);
    const bool ok = __all_sync(kFull, same);
    if (lane == 0) bcls[k] = ok ? cu : k;
  }
}

// The B class of every staged column, gathered by the whole warp (eight
// loads a lane in flight at a time) into cls.
__device__ __forceinline__ void gather_classes(const SegRows &s, const int32_t *seg,
                                               const int32_t *__restrict__ bcls, int32_t *cls,
                                               int lane) {
  for (int32_t t0 = 0; t0 < s.n; t0 += 256) {
    int32_t g[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      const int32_t t = t0 + q * 32 + lane;
      g[q] = t < s.n ? __ldg(bcls + seg[t]) : 0;
    }
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      const int32_t t = t0 + q * 32 + lane;
      if (t < s.n) cls[t] = g[q];
    }
  }
  __syncwarp();
}

// Row keys, a lane per row: the XOR of row_term(j, A column - i, class of
// that B row) over the row's positions j, then row_key_of; 0 for a row that
// cannot join a pattern.
__global__ void __launch_bounds__(kAWarps * 32)
shift_rkey_kernel(const int32_t *__restrict__ on, int32_t a_rows,
                  const int32_t *__restrict__ a_rp, const int32_t *__restrict__ a_col,
                  const int64_t *__restrict__ ops, const int32_t *__restrict__ bcls,
                  unsigned long long *__restrict__ rkey) {
  __shared__ __align__(16) int32_t segs[kAWarps][kSegCap];
  __shared__ int32_t clss[kAWarps][kSegCap];
  if (!*on) return;
  if ((int64_t(blockIdx.x) * kAWarps + (threadIdx.x >> 5)) * 32 >= a_rows) return;
  const int lane = lane_id();
  int32_t *seg = segs[threadIdx.x >> 5], *cls = clss[threadIdx.x >> 5];
  int4 v[kSegVec];
  const SegRows s = seg_issue(a_rows, kAWarps, a_rp, a_col, lane, v);
  const int64_t o = s.live ? ops[s.r] : 0;
  seg_land(s, a_col, seg, lane, v);
  gather_classes(s, seg, bcls, cls, lane);
  if (!s.live) return;
  unsigned long long key = 0ull;
  if (shiftable(s.len, o)) {
    unsigned long long h = 0;
    if (s.base >= 0) {
      const int32_t *m = seg + (s.lo - s.base), *mc = cls + (s.lo - s.base);
      for (int32_t j = 0; j < s.len; ++j)
        h ^= row_term(j, m[j] - s.r, static_cast<uint32_t>(mc[j]));
    } else {
      for (int32_t j = 0; j < s.len; ++j) {
        const int32_t k = __ldg(a_col + s.lo + j);
        h ^= row_term(j, k - s.r, static_cast<uint32_t>(__ldg(bcls + k)));
      }
    }
    key = row_key_of(h, s.len);
  }
  rkey[s.r] = key;
}

// rcls[i]: the smallest row with i's translated A row over the same B
// classes (checked entry by entry), else i.  A lane per row; its own row's
// columns and classes staged, the canonical row's read from global memory
// (a few rows, so cache hits).
__global__ void __launch_bounds__(kAWarps * 32)
shift_rresolve_kernel(const int32_t *__restrict__ on, int32_t a_rows,
                      const unsigned long long *__restrict__ rkey,
                      const unsigned long long *__restrict__ tkey,
                      const int32_t *__restrict__ trow, unsigned long long mask,
                      const int32_t *__restrict__ a_rp, const int32_t *__restrict__ a_col,
                      const int32_t *__restrict__ bcls, int32_t *__restrict__ rcls) {
  __shared__ __align__(16) int32_t segs[kAWarps][kSegCap];
  __shared__ int32_t clss[kAWarps][kSegCap];
  if (!*on) return;
  if ((int64_t(blockIdx.x) * kAWarps + (threadIdx.x >> 5)) * 32 >= a_rows) return;
  const int lane = lane_id();
  int32_t *seg = segs[threadIdx.x >> 5], *cls = clss[threadIdx.x >> 5];
  int4 v[kSegVec];
  const SegRows s = seg_issue(a_rows, kAWarps, a_rp, a_col, lane, v);
  const unsigned long long key = s.live ? rkey[s.r] : 0ull;
  int32_t c = key ? lookup(key, tkey, trow, mask) : -1, c0 = 0;
  bool check = false;
  if (c >= 0 && c < a_rows && c != s.r && s.len <= kShiftMaxA) {
    c0 = __ldg(a_rp + c);
    check = __ldg(a_rp + c + 1) - c0 == s.len;
  }
  seg_land(s, a_col, seg, lane, v);
  gather_classes(s, seg, bcls, cls, lane);
  if (!s.live) return;
  bool same = check;
  if (check) {
    if (s.base >= 0) {
      const int32_t *m = seg + (s.lo - s.base), *mc = cls + (s.lo - s.base);
#pragma unroll 4
      for (int32_t j = 0; j < s.len; ++j) {
        const int32_t kc = __ldg(a_col + c0 + j);
        same &= m[j] - s.r == kc - c && mc[j] == __ldg(bcls + kc);
      }
    } else {
#pragma unroll 4
      for (int32_t j = 0; j < s.len; ++j) {
        const int32_t ki = __ldg(a_col + s.lo + j), kc = __ldg(a_col + c0 + j);
        same &= ki - s.r == kc - c && __ldg(bcls + ki) == __ldg(bcls + kc);
      }
    }
  }
  rcls[s.r] = same ? c : s.r;
}

// share[c] += rows whose class is c (other than c); warp-aggregated.
__global__ void __launch_bounds__(kThreads)
shift_share_kernel(const int32_t *__restrict__ on, int32_t n, const int32_t *__restrict__ rcls,
                   int32_t *__restrict__ share) {
  __shared__ int32_t s_c, s_n;
  if (!*on) return;
  const int32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  const int32_t c = i < n ? rcls[i] : -1;
  const bool member = i < n && c != i;
  // the block's first row's class is counted in shared memory (a stencil
  // block is mostly one class), the others warp-aggregated
  if (threadIdx.x == 0) {
    s_c = member ? c : -1;
    s_n = 0;
  }
  __syncthreads();
  const bool local = member && c == s_c;
  const unsigned peers = __match_any_sync(kFull, member && !local ? c : -1 - lane_id());
  if (member && !local && (peers & lanemask_lt()) == 0u) atomicAdd(share + c, __popc(peers));
  const unsigned lb = __ballot_sync(kFull, local);
  if (lb && lane_id() == 0) atomicAdd(&s_n, __popc(lb));
  __syncthreads();
  if (threadIdx.x == 0 && s_n) atomicAdd(share + s_c, s_n);
}

// Candidates: a canonical row shared by at least min_share - 1 others gets
// an id (pat_of[c], pat_canon[id]) and its table capacity (the warp-per-row
// table kernel's record count, k_pattern.cu: (2 ceil(ops/32) + nA) * 32).
__global__ void __launch_bounds__(kThreads)
shift_pat_kernel(const int32_t *__restrict__ on, int32_t n, const int32_t *__restrict__ rcls,
                 const int32_t *__restrict__ share, int32_t min_share,
                 const int32_t *__restrict__ a_rp, const int64_t *__restrict__ ops,
                 int32_t *__restrict__ pat_of, int32_t *__restrict__ pat_canon,
                 int32_t *__restrict__ pat_cap, int32_t *__restrict__ npat, int32_t cap_pat) {
  if (!*on) return;
  const int32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  pat_of[i] = -1;
  if (rcls[i] != i || share[i] + 1 < min_share) return;
  const int32_t id = atomicAdd(npat, 1);
  if (id >= cap_pat) return;  // cannot happen: cap_pat >= n / min_share + 1
  pat_of[i] = id;
  pat_canon[id] = i;
  const int32_t tiles = static_cast<int32_t>((ops[i] + 31) / 32);
  pat_cap[id] = (2 * tiles + (a_rp[i + 1] - a_rp[i])) * 32;
}

// The output count of each candidate's canonical row (distinct columns of
// its at most 1024 products: one block sort), and whether the pattern is
// kept: at most kShiftMaxOut outputs, which the term tables hold.  Blocks
// stride over the candidates; pat_m[id] = count, or -1 when dropped.
__global__ void __launch_bounds__(1024)
shift_canon_count_kernel(const int32_t *__restrict__ on, const int32_t *__restrict__ npat,
                         int32_t cap_pat, const int32_t *__restrict__ pat_canon,
                         const int32_t *__restrict__ a_rp, const int32_t *__restrict__ a_col,
                         const int32_t *__restrict__ b_rp, const int32_t *__restrict__ b_col,
                         int32_t *__restrict__ pat_m) {
  __shared__ unsigned long long cols[kShiftMaxOps];
  __shared__ int32_t bstart[kShiftMaxA + 1];
  __shared__ int32_t s_m;
  if (!*on) return;
  const int32_t np = min(*npat, cap_pat);
  const int tid = threadIdx.x;
  for (int32_t id = blockIdx.x; id < np; id += gridDim.x) {
    const int32_t row = pat_canon[id];
    const int32_t p0 = a_rp[row], na = a_rp[row + 1] - p0;
    if (tid == 0) {
      int32_t run = 0;
      for (int32_t j = 0; j < na; ++j) {
        bstart[j] = run;
        const int32_t k = a_col[p0 + j];
        run += b_rp[k + 1] - b_rp[k];
      }
      bstart[na] = run;
      s_m = 0;
    }
    __syncthreads();
    const int32_t ops = bstart[na];
    for (int32_t t = tid; t < kShiftMaxOps; t += blockDim.x) {
      unsigned long long v = ~0ull;
      if (t < ops) {
        int32_t j = 0;
        while (j + 1 < na && bstart[j + 1] <= t) ++j;
        const int32_t k = a_col[p0 + j];
        v = static_cast<unsigned long long>(
            static_cast<uint32_t>(b_col[b_rp[k] + t - bstart[j]]));
      }
      cols[t] = v;
    }
    __syncthreads();
    block_bitonic_sort(cols, kShiftMaxOps);
    int mine = 0;
    for (int32_t t = tid; t < ops; t += blockDim.x)
      mine += (t == 0 || cols[t] != cols[t - 1]) ? 1 : 0;
    mine = warp_sum(mine);
    if (lane_id() == 0 && mine) atomicAdd(&s_m, mine);
    __syncthreads();
    if (tid == 0) pat_m[id] = s_m <= kShiftMaxOut ? s_m : -1;
    __syncthreads();
  }
}

// Members: pid_of_row[i] = pattern of a member row (else -1; every row -1
// when *on is 0), its symbolic class set to empty (it skips the symbolic
// pass); *members counts them.
__global__ void __launch_bounds__(kThreads)
shift_members_kernel(const int32_t *__restrict__ on, int32_t n, const int32_t *__restrict__ rcls,
                     const int32_t *__restrict__ pat_of, const int32_t *__restrict__ pat_m,
                     int32_t *__restrict__ pid_of_row, uint8_t *__restrict__ cls,
                     int32_t *__restrict__ members) {
  const int32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  const bool live = *on != 0;
  bool m = false;
  if (i < n) {
    int32_t pid = -1;
    if (live) {
      const int32_t c = rcls[i];
      pid = c != i ? pat_of[c] : -1;
      if (pid >= 0 && pat_m[pid] < 0) pid = -1;
    }
    pid_of_row[i] = pid;
    if (pid >= 0) {
      cls[i] = static_cast<uint8_t>(kEmpty_);
      m = true;
    }
  }
  const unsigned b = __ballot_sync(kFull, m);
  if (b && lane_id() == 0) atomicAdd(members, __popc(b));
}

// Class census of cls (class_count zeroed before).
__global__ void __launch_bounds__(kThreads)
shift_census_kernel(const int32_t *__restrict__ on, int32_t n, const uint8_t *__restrict__ cls,
                    int32_t *__restrict__ class_count) {
  __shared__ int32_t s_cnt[kNumClasses];
  if (!*on) return;
  for (int c = threadIdx.x; c < kNumClasses; c += blockDim.x) s_cnt[c] = 0;
  __syncthreads();
  const int32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  const int c = i < n ? cls[i] : -1;
  const unsigned peers = __match_any_sync(kFull, c);
  if (c >= 0 && (peers & lanemask_lt()) == 0u) atomicAdd(&s_cnt[c], __popc(peers));
  __syncthreads();
  for (int k = threadIdx.x; k < kNumClasses; k += blockDim.x)
    if (s_cnt[k]) atomicAdd(class_count + k, s_cnt[k]);
}

// counts[i] = counts[canonical] for member rows.
__global__ void __launch_bounds__(kThreads)
shift_copy_counts_kernel(const int32_t *__restrict__ on, int32_t n,
                         const int32_t *__restrict__ pid_of_row,
                         const int32_t *__restrict__ rcls, int32_t *__restrict__ counts) {
  if (!*on) return;
  const int32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n || pid_of_row[i] < 0) return;
  counts[i] = counts[rcls[i]];
}

// Member rows' columns: the canonical row's, moved by i - c.  kShiftRows
// rows per warp (lane u < kShiftRows finds row i0 + u's canonical row and
// bounds), every lane copying one entry of each row per step.
__global__ void __launch_bounds__(kThreads)
shift_fill_kernel(int32_t n, const int32_t *__restrict__ pid_of_row,
                  const int32_t *__restrict__ rcls, const int32_t *__restrict__ c_rp,
                  int32_t *__restrict__ c_col) {
  const int64_t i0 = ((int64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5) * kShiftRows;
  if (i0 >= n) return;
  const int lane = lane_id();
  int32_t mcs = 0, mcc = 0, mm = 0, md = 0;
  if (lane < kShiftRows && i0 + lane < n) {
    const int32_t i = static_cast<int32_t>(i0) + lane;
    if (pid_of_row[i] >= 0) {
      const int32_t c = rcls[i];
      mcs = c_rp[i];
      mm = c_rp[i + 1] - mcs;
      mcc = c_rp[c];
      md = i - c;
    }
  }
  int32_t cs[kShiftRows], cc[kShiftRows], m[kShiftRows], d[kShiftRows];
  int32_t longest = 0;
#pragma unroll
  for (int u = 0; u < kShiftRows; ++u) {
    cs[u] = __shfl_sync(kFull, mcs, u);
    cc[u] = __shfl_sync(kFull, mcc, u);
    m[u] = __shfl_sync(kFull, mm, u);
    d[u] = __shfl_sync(kFull, md, u);
    longest = max(longest, m[u]);
  }
  for (int32_t e = lane; e < longest; e += 32) {
    int32_t v[kShiftRows];
#pragma unroll
    for (int u = 0; u < kShiftRows; ++u) v[u] = e < m[u] ? __ldg(c_col + cc[u] + e) : 0;
#pragma unroll
    for (int u = 0; u < kShiftRows; ++u)
      if (e < m[u]) c_col[cs[u] + e] = v[u] + d[u];
  }
}

// Map of each pattern's canonical row: for product t in flattened order
// (A nonzero j, then B position e), its position in C's sorted row, by
// binary search; 0xffff when the column is missing (C is not this product's).
// moff[canonical row] = id * kShiftMaxOps.  Warp per pattern.
__global__ void __launch_bounds__(kThreads)
shift_canon_map_kernel(int32_t npat, const int32_t *__restrict__ pat_canon,
                       const int32_t *__restrict__ a_rp, const int32_t *__restrict__ a_col,
                       const int32_t *__restrict__ b_rp, const int32_t *__restrict__ b_col,
                       const int32_t *__restrict__ c_rp, const int32_t *__restrict__ c_col,
                       int64_t *__restrict__ moff, uint16_t *__restrict__ map) {
  const int32_t id = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (id >= npat) return;
  const int lane = lane_id();
  const int32_t row = pat_canon[id];
  const int32_t p0 = a_rp[row], na = a_rp[row + 1] - p0;
  const int32_t cs = c_rp[row], m = c_rp[row + 1] - cs;
  const int64_t base = int64_t(id) * kShiftMaxOps;
  if (lane == 0) moff[row] = base;
  int32_t t0 = 0;
  for (int32_t j = 0; j < na; ++j) {
    const int32_t k = __ldg(a_col + p0 + j);
    const int32_t b0 = __ldg(b_rp + k), len = __ldg(b_rp + k + 1) - b0;
    for (int32_t e = lane; e < len && t0 + e < kShiftMaxOps; e += 32) {
      const int32_t col = __ldg(b_col + b0 + e);
      int32_t lo = 0, hi = m;
      while (lo < hi) {
        const int32_t mid = (lo + hi) >> 1;
        if (__ldg(c_col + cs + mid) < col) lo = mid + 1;
        else hi = mid;
      }
      const bool found = lo < m && __ldg(c_col + cs + lo) == col;
      map[base + t0 + e] = found ? static_cast<uint16_t>(lo) : uint16_t(0xffff);
    }
    t0 += len;
  }
}

// Largest products (rounded up to 32) and outputs over the kept patterns
// (out[0], out[1], zeroed by the caller).
__global__ void __launch_bounds__(kThreads)
shift_maxima_kernel(int32_t npat, const int32_t *__restrict__ pat_canon,
                    const int32_t *__restrict__ pat_m, const int64_t *__restrict__ ops,
                    int32_t *__restrict__ out) {
  const int32_t id = blockIdx.x * blockDim.x + threadIdx.x;
  if (id >= npat || pat_m[id] < 0) return;
  atomicMax(out, static_cast<int32_t>((ops[pat_canon[id]] + 31) / 32) * 32);
  atomicMax(out + 1, pat_m[id]);
}

unsigned grid_warps(int64_t warps) {
  return static_cast<unsigned>((warps * 32 + kThreads - 1) / kThreads);
}
unsigned grid_threads(int64_t n) {
  return static_cast<unsigned>((n + kThreads - 1) / kThreads);
}
// Blocks of the key and resolve passes: 32 rows a warp.
unsigned grid_segs(int32_t rows, int warps) {
  const int64_t per = int64_t(32) * warps;
  const int64_t b = (int64_t(rows) + per - 1) / per;
  return static_cast<unsigned>(b ? b : 1);
}
unsigned grid_fill(size_t n) {
  const size_t b = (n + kThreads - 1) / kThreads;
  return static_cast<unsigned>(b < 4096 ? (b ? b : 1) : 4096);
}

}  // namespace

int32_t shift_max_ops() { return kShiftMaxOps; }
int32_t shift_samples() { return kShiftSamples; }

void launch_shift_decide(const Operands &op, unsigned long long *keys, int32_t min_mean_ops,
                         int32_t *on, CheckGuard guard, cudaStream_t s) {
  const int32_t samples = op.a_rows < kShiftSamples ? op.a_rows : kShiftSamples;
  shift_probe_kernel<<<grid_warps(samples), kThreads, 0, s>>>(op, samples, keys, guard);
  shift_decide_kernel<<<1, 1024, 0, s>>>(keys, samples, min_mean_ops, on, guard);
}

void launch_shift_classes(const int32_t *on, const Operands &op, int32_t b_rows,
                          const int64_t *ops, unsigned long long *bkey,
                          unsigned long long *rkey, unsigned long long *tkey, int32_t *trow,
                          size_t tcap, int32_t *bcls, int32_t *rcls, cudaStream_t s) {
  const unsigned long long mask = tcap - 1;
  // B classes
  shift_fill64_kernel<<<grid_fill(tcap), kThreads, 0, s>>>(on, tkey, tcap, 0ull);
  shift_fill32_kernel<<<grid_fill(tcap), kThreads, 0, s>>>(on, trow, tcap, INT_MAX);
  const unsigned bg = grid_segs(b_rows, kBWarps), ag = grid_segs(op.a_rows, kAWarps);
  shift_bkey_kernel<<<bg, kBWarps * 32, 0, s>>>(on, b_rows, op.b_rp, op.b_col, bkey);
  shift_insert_kernel<<<grid_threads(b_rows), kThreads, 0, s>>>(on, b_rows, bkey, tkey, trow,
                                                                mask);
  shift_bresolve_kernel<<<bg, kBWarps * 32, 0, s>>>(on, b_rows, bkey, tkey, trow, mask, op.b_rp,
                                                   op.b_col, bcls);
  // row classes
  shift_fill64_kernel<<<grid_fill(tcap), kThreads, 0, s>>>(on, tkey, tcap, 0ull);
  shift_fill32_kernel<<<grid_fill(tcap), kThreads, 0, s>>>(on, trow, tcap, INT_MAX);
  shift_rkey_kernel<<<ag, kAWarps * 32, 0, s>>>(on, op.a_rows, op.a_rp, op.a_col, ops, bcls,
                                               rkey);
  shift_insert_kernel<<<grid_threads(op.a_rows), kThreads, 0, s>>>(on, op.a_rows, rkey, tkey,
                                                                   trow, mask);
  shift_rresolve_kernel<<<ag, kAWarps * 32, 0, s>>>(on, op.a_rows, rkey, tkey, trow, mask,
                                                   op.a_rp, op.a_col, bcls, rcls);
}

void launch_shift_patterns(const int32_t *on, const Operands &op, const int32_t *rcls,
                           int32_t *share, int32_t min_share, const int64_t *ops,
                           int32_t *pat_of, int32_t *pat_canon, int32_t *pat_cap,
                           int32_t *pat_m, int32_t *npat, int32_t cap_pat,
                           int32_t *pid_of_row, uint8_t *cls, int32_t *members,
                           int32_t *class_count, int num_sms, cudaStream_t s) {
  const int32_t n = op.a_rows;
  shift_fill32_kernel<<<grid_fill(size_t(n)), kThreads, 0, s>>>(on, share, size_t(n), 0);
  shift_share_kernel<<<grid_threads(n), kThreads, 0, s>>>(on, n, rcls, share);
  shift_pat_kernel<<<grid_threads(n), kThreads, 0, s>>>(on, n, rcls, share, min_share, op.a_rp,
                                                        ops, pat_of, pat_canon, pat_cap, npat,
                                                        cap_pat);
  shift_canon_count_kernel<<<num_sms, 1024, 0, s>>>(on, npat, cap_pat, pat_canon, op.a_rp,
                                                    op.a_col, op.b_rp, op.b_col, pat_m);
  shift_members_kernel<<<grid_threads(n), kThreads, 0, s>>>(on, n, rcls, pat_of, pat_m,
                                                            pid_of_row, cls, members);
  shift_fill32_kernel<<<1, kThreads, 0, s>>>(on, class_count, kNumClasses, 0);
  shift_census_kernel<<<grid_threads(n), kThreads, 0, s>>>(on, n, cls, class_count);
}

void launch_shift_copy_counts(const int32_t *on, int32_t n, const int32_t *pid_of_row,
                              const int32_t *rcls, int32_t *counts, cudaStream_t s) {
  shift_copy_counts_kernel<<<grid_threads(n), kThreads, 0, s>>>(on, n, pid_of_row, rcls,
                                                                counts);
}

void launch_shift_fill(int32_t n, const int32_t *pid_of_row, const int32_t *rcls,
                       const int32_t *c_rp, int32_t *c_col, cudaStream_t s) {
  shift_fill_kernel<<<grid_warps((int64_t(n) + kShiftRows - 1) / kShiftRows), kThreads, 0, s>>>(
      n, pid_of_row, rcls, c_rp, c_col);
}

void launch_shift_canon_map(int32_t npat, const int32_t *pat_canon, const Operands &op,
                            const int32_t *c_rp, const int32_t *c_col, int64_t *moff,
                            uint16_t *map, cudaStream_t s) {
  if (npat <= 0) return;
  shift_canon_map_kernel<<<grid_warps(npat), kThreads, 0, s>>>(
      npat, pat_canon, op.a_rp, op.a_col, op.b_rp, op.b_col, c_rp, c_col, moff, map);
}

void launch_pat_maxima(int32_t npat, const int32_t *pat_canon, const int32_t *pat_m,
                       const int64_t *ops, int32_t *out, cudaStream_t s) {
  if (npat <= 0) return;
  shift_maxima_kernel<<<grid_threads(npat), kThreads, 0, s>>>(npat, pat_canon, pat_m, ops, out);
}

}  // namespace rvsp
