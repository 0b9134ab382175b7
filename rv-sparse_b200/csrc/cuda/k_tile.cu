// Row tiles: numeric-only repeats of runs of rows that share one term table.
//
// A structured matrix (a stencil, a finite-element mesh) has long runs of
// consecutive rows with the same reuse map (k_reuse.cu): their products land
// at the same positions of C's row, in the same order.  The warp-per-row
// table kernel (k_pattern.cu) spends most of its time moving each product
// through shared memory twice.  Here one warp takes a tile of up to 32
// consecutive rows of one pattern, one row per lane, so every table read is
// uniform across the warp and every lane does the same work:
//
//   for each A nonzero j of the row, in ascending order:
//     the warp stages the B values its lanes need for j (the span from the
//     smallest to the largest of the lanes' B rows k_j, contiguous in B) into
//     shared memory with 16-byte cp.async copies, one A nonzero ahead of the
//     arithmetic (double buffer);
//     for each entry e of B row k_j (the pattern's B row length):
//       q = slot[j][e]                      (uniform: position in C's row)
//       acc[q] = (first term of q ? +0.0f : acc[q]) + fl(a_j * b[k_j][e])
//
// acc is a shared-memory column per lane (q * 33 + lane: conflict-free for
// the lanes and for the coalesced write of each row to C at the end).  The
// entries of one B row have distinct positions, so within one j no two
// products meet; across j the order is ascending A nonzero.  Each output is
// therefore fl(...fl(fl(0 + p_1) + p_2)... + p_n) over its products in A
// order, every product and sum rounded separately: the reference scalar
// kernel's order (gustavson_core_f32.inc:31-62, accum_scalar_f32.c:20-71),
// so the values equal the plain path's bit for bit.
//
// Tables (one per pattern, built once per structure from the canonical
// row's map): per A nonzero j a block of round_up(len_j, 8) uint16 slots,
// bit 15 set on a product that is the first term of its output.  The padding
// entries name the pattern's spare accumulator row m (with bit 15), so the
// inner loop runs whole groups of eight with no bounds test: the padding
// products read staged values past the lane's B row (inside the stage
// buffer, which keeps 8 floats of margin) and write the spare row, which is
// never read.
//
// Tiles are formed once per structure: the rows are cut into chunks of 32
// consecutive rows; in each chunk the largest group of table rows with one
// pattern becomes a tile when it has at least kTileMinRows rows, its A
// segment and every B span fit the buffers, and every row's C length is the
// pattern's.  Every other table row goes to a leftover list that the
// warp-per-row table kernel takes.
#include <climits>

#include "device_common.cuh"
#include "kernels.cuh"

namespace rvsp {

namespace {

constexpr int kTileMaxA = 32;           // A nonzeros of a tiled pattern (kPatMaxA)
constexpr int kTileMinRows = 8;         // rows of one pattern that make a tile
constexpr int kTileStageMax = 4096;     // floats in one stage buffer
constexpr int kTileASegMax = 2048;      // A entries of one chunk
constexpr int kTileMaxOut = 256;        // C entries of a tiled row
constexpr int kTileStages = 2;          // B spans in flight per warp (ring)
// uint16 entries of one pattern's table: at most kPatMaxOps (1024) products
// plus 7 padding entries per A nonzero, rounded to a multiple of 8
constexpr int kTileTabStride = 1280;
constexpr uint16_t kFirst = 0x8000u;

// maxima words (zeroed by the caller)
constexpr int kStageNeedWord = 0, kASegWord = 1, kMaxOutWord = 2;

__device__ __forceinline__ void cp_async16(void *smem, const void *gmem) {
  const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async4(void *smem, const void *gmem) {
  const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() {
  asm volatile("cp.async.commit_group;\n" ::: "memory");
}
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// One table per pattern: warp per pattern.  desc[id] = (na, m, ops, 0), or
// na = -1 when the pattern cannot be tiled (no table, too many outputs).
// lens[id * 32 + j] = length of the B row of A nonzero j.
__global__ void __launch_bounds__(128)
tile_tab_kernel(int32_t npat, const int32_t *__restrict__ pat_canon,
                const int32_t *__restrict__ psteps, const int32_t *__restrict__ a_rp,
                const int32_t *__restrict__ a_col, const int32_t *__restrict__ b_rp,
                const int32_t *__restrict__ c_rp, const int64_t *__restrict__ moff,
                const uint16_t *__restrict__ map, int32_t max_out,
                uint16_t *__restrict__ tab, uint16_t *__restrict__ lens,
                int4 *__restrict__ desc) {
  __shared__ uint32_t seen[4][(kTileMaxOut + 31) / 32];
  const int wib = threadIdx.x >> 5;
  const int32_t id = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (id >= npat) return;
  const int lane = lane_id();
  const int32_t row = pat_canon[id];
  const int32_t p0 = a_rp[row], na = a_rp[row + 1] - p0;
  const int32_t m = c_rp[row + 1] - c_rp[row];
  if (psteps[id] < 0 || na <= 0 || na > kTileMaxA || m <= 0 || m > max_out) {
    if (lane == 0) desc[id] = make_int4(-1, 0, 0, 0);
    return;
  }
  int32_t len = 0;
  if (lane < na) {
    const int32_t k = __ldg(a_col + p0 + lane);
    len = __ldg(b_rp + k + 1) - __ldg(b_rp + k);
  }
  lens[size_t(id) * 32 + lane] = static_cast<uint16_t>(lane < na ? len : 0);
  const int32_t r8 = (len + 7) & ~7;
  const int32_t jo = warp_incl_scan(r8) - r8;  // block offset of A nonzero lane
  for (int w = lane; w < (kTileMaxOut + 31) / 32; w += 32) seen[wib][w] = 0u;
  __syncwarp();
  uint16_t *const t = tab + size_t(id) * kTileTabStride;
  const int64_t base = moff[row];
  int32_t t0 = 0;
  for (int32_t j = 0; j < na; ++j) {
    const int32_t lj = __shfl_sync(kFull, len, j);
    const int32_t oj = __shfl_sync(kFull, jo, j);
    const int32_t rj = (lj + 7) & ~7;
    for (int32_t e = lane; e < rj; e += 32) {
      uint16_t u = static_cast<uint16_t>(m) | kFirst;  // padding: the spare row
      if (e < lj) {
        const int32_t q = __ldg(map + base + t0 + e);
        const bool first = ((seen[wib][q >> 5] >> (q & 31)) & 1u) == 0u;
        u = static_cast<uint16_t>(q) | (first ? kFirst : uint16_t(0));
      }
      t[oj + e] = u;
    }
    __syncwarp();
    // positions within one B row are distinct: mark them after the block
    for (int32_t e = lane; e < lj; e += 32) {
      const int32_t q = __ldg(map + base + t0 + e);
      atomicOr(&seen[wib][q >> 5], 1u << (q & 31));
    }
    __syncwarp();
    t0 += lj;
  }
  if (lane == 0) desc[id] = make_int4(na, m, t0, 0);
}

// Warps per block of the tile builder, and the A entries of a chunk whose B
// row starts it stages in shared memory.
constexpr int kBuildWarps = 4;
constexpr int kBuildStage = 1024;

// Warp per chunk of 32 consecutive rows (see the file comment).
__global__ void __launch_bounds__(kBuildWarps * 32, 8)
tile_build_kernel(int32_t n, const int32_t *__restrict__ pid_of_row,
                  const int4 *__restrict__ desc, const uint16_t *__restrict__ lens,
                  const int32_t *__restrict__ a_rp, const int32_t *__restrict__ a_col,
                  const int32_t *__restrict__ b_rp, const int32_t *__restrict__ c_rp,
                  int4 *__restrict__ tiles, int32_t *__restrict__ ntiles,
                  int32_t *__restrict__ lo_rows, int32_t *__restrict__ lo_ids,
                  int32_t *__restrict__ lo_n, int32_t *__restrict__ maxima) {
  const int64_t chunk = (int64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
  const int64_t row0 = chunk * 32;
  if (row0 >= n) return;
  const int lane = lane_id();
  const int32_t row = static_cast<int32_t>(row0) + lane;
  const int32_t pid = row < n ? pid_of_row[row] : -1;
  const unsigned peers = __match_any_sync(kFull, pid);
  const int cnt = pid >= 0 ? __popc(peers) : 0;
  const int leader = __ffs(peers) - 1;
  const int key = cnt > 0 ? (cnt << 5) | (31 - leader) : 0;
  const int best = __reduce_max_sync(kFull, key);
  bool ok = (best >> 5) >= kTileMinRows;
  const int32_t bpid = __shfl_sync(kFull, pid, 31 - (best & 31));
  const bool in = ok && pid == bpid;
  int4 d = make_int4(-1, 0, 0, 0);
  int32_t seg = 0, need = 0;
  if (ok) {
    d = desc[bpid];
    ok = d.x > 0;
  }
  if (ok) {
    const int32_t last = row0 + 32 < n ? static_cast<int32_t>(row0) + 32 : n;
    seg = a_rp[last] - a_rp[row0];
    bool fits = seg <= kTileASegMax;
    if (in) fits = fits && (c_rp[row + 1] - c_rp[row] == d.y) && (a_rp[row + 1] - a_rp[row] == d.x);
    ok = __all_sync(kFull, fits);
  }
  if (ok) {
    // the chunk's B row starts: a segment of up to kBuildStage entries is
    // staged in shared memory with coalesced loads of a_col (16 a lane in
    // flight, then their gathers), a longer one read through a_col (4 KB a
    // warp and at most 64 registers keep 32 warps an SM resident: this
    // kernel is bound by load latency)
    __shared__ int32_t sseg[kBuildWarps][kBuildStage];
    int32_t *const sb = sseg[(threadIdx.x >> 5) % kBuildWarps];
    const int32_t seg0 = a_rp[row0];
    const bool staged = seg <= kBuildStage;
    if (staged) {
      for (int32_t i0 = 0; i0 < seg; i0 += 512) {
        int32_t c[16];
#pragma unroll
        for (int u = 0; u < 16; ++u) {
          const int32_t i = i0 + u * 32 + lane;
          c[u] = i < seg ? __ldg(a_col + seg0 + i) : 0;
        }
#pragma unroll
        for (int u = 0; u < 16; ++u) {
          const int32_t i = i0 + u * 32 + lane;
          c[u] = i < seg ? __ldg(b_rp + c[u]) : 0;
        }
#pragma unroll
        for (int u = 0; u < 16; ++u) {
          const int32_t i = i0 + u * 32 + lane;
          if (i < seg) sb[i] = c[u];
        }
      }
    }
    __syncwarp();
    const int32_t p = in ? a_rp[row] - seg0 : 0;
    for (int32_t j = 0; j < d.x; ++j) {
      const int32_t lj = lens[size_t(bpid) * 32 + j];
      const int32_t rp =
          in ? (staged ? sb[p + j] : __ldg(b_rp + __ldg(a_col + seg0 + p + j))) : 0;
      const int32_t lo = __reduce_min_sync(kFull, in ? rp : INT_MAX);
      const int32_t hi = __reduce_max_sync(kFull, in ? rp + lj : INT_MIN);
      need = max(need, hi - (lo & ~3) + 8);
    }
    ok = need <= kTileStageMax;
  }
  const unsigned tmask = __ballot_sync(kFull, ok && in);
  if (ok && lane == 0) {
    const int32_t t = atomicAdd(ntiles, 1);
    tiles[t] = make_int4(static_cast<int32_t>(row0), static_cast<int32_t>(tmask), bpid, 0);
    atomicMax(maxima + kStageNeedWord, need);
    atomicMax(maxima + kASegWord, seg);
    atomicMax(maxima + kMaxOutWord, d.y);
  }
  // leftovers: table rows that are not in the tile
  const bool left = pid >= 0 && !(ok && in);
  const unsigned lmask = __ballot_sync(kFull, left);
  if (lmask) {
    int32_t base = 0;
    if (lane == 0) base = atomicAdd(lo_n, __popc(lmask));
    base = __shfl_sync(kFull, base, 0);
    if (left) {
      const int32_t at = base + __popc(lmask & lanemask_lt());
      lo_rows[at] = row;
      lo_ids[at] = pid;
    }
  }
}

// Copies B values [lo, hi) into dst (shared, 16-byte aligned); returns c0,
// the B index that dst[0] stands for.  Whole aligned 16-byte chunks while they
// lie inside B's nnz values, single floats for a chunk that would not.
__device__ __forceinline__ int32_t stage_span(float *dst, const float *__restrict__ b_val,
                                              int32_t lo, int32_t hi, int32_t b_nnz,
                                              bool aligned16, int lane) {
  if (aligned16) {
    const int32_t c0 = lo & ~3;
    const int32_t chunks = (hi - c0 + 3) >> 2;
    for (int32_t c = lane; c < chunks; c += 32) {
      const int32_t g = c0 + 4 * c;
      if (g + 4 <= b_nnz) {
        cp_async16(dst + 4 * c, b_val + g);
      } else {
        for (int32_t x = g; x < hi; ++x) cp_async4(dst + (x - c0), b_val + x);
      }
    }
    return c0;
  }
  for (int32_t x = lo + lane; x < hi; x += 32) cp_async4(dst + (x - lo), b_val + x);
  return lo;
}

// Values of the tiled rows: warp per tile.  Shared memory per warp:
// acc[(acc_rows) * 33] floats, then a work area of work_floats floats that
// first holds the chunk's A segment (columns, then values) and then the
// kTileStages stage buffers of stage_cap floats each.
__global__ void __launch_bounds__(kTileKernelWarps * 32)
tile_numeric_kernel(const int32_t *__restrict__ a_rp, const int32_t *__restrict__ a_col,
                    const float *__restrict__ a_val, const int32_t *__restrict__ b_rp,
                    const float *__restrict__ b_val, int32_t b_nnz,
                    const int4 *__restrict__ tiles, int32_t ntiles,
                    const int4 *__restrict__ desc, const uint16_t *__restrict__ lens,
                    const uint16_t *__restrict__ tab, const int32_t *__restrict__ c_rp,
                    float *__restrict__ c_val, int acc_rows, int work_floats,
                    int stage_cap) {
  extern __shared__ __align__(16) float smem_f32[];
  const int wib = threadIdx.x >> 5;
  const int acc_floats = (acc_rows * 33 + 3) & ~3;
  float *const acc = smem_f32 + size_t(wib) * (acc_floats + work_floats);
  float *const work = acc + acc_floats;
  const int64_t w = (int64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
  if (w >= ntiles) return;
  const int lane = lane_id();
  const int4 tile = tiles[w];
  const int32_t row0 = tile.x;
  const unsigned mask = static_cast<unsigned>(tile.y);
  const int32_t pid = tile.z;
  const int4 d = desc[pid];
  if (d.w != 0) return;  // a pattern kernel (k_jit.cu) takes these tiles
  const int32_t na = d.x, m = d.y;
  const bool active = (mask >> lane) & 1u;
  const int32_t row = row0 + lane;
  const bool aligned16 = (reinterpret_cast<uintptr_t>(b_val) & 15u) == 0;

  // A segment of the chunk's rows (every lane of the chunk, active or not,
  // lies inside it: the tile was only formed when it fits the work area)
  const int32_t seg0 = a_rp[row0];
  int32_t my_p = 0, cs = 0;
  if (active) {
    my_p = a_rp[row] - seg0;
    cs = c_rp[row];
  }
  {
    const int32_t last_row = __reduce_max_sync(kFull, active ? row : row0);
    const int32_t seg = a_rp[last_row + 1] - seg0;
    int32_t *scol = reinterpret_cast<int32_t *>(work);
    float *sval = work + seg;
    for (int32_t i = lane; i < seg; i += 32) {
      scol[i] = __ldg(a_col + seg0 + i);
      sval[i] = __ldg(a_val + seg0 + i);
    }
  }
  __syncwarp();
  // per lane: a_j and B row start of each A nonzero (registers: j is unrolled)
  int32_t len = lane < na ? static_cast<int32_t>(lens[size_t(pid) * 32 + lane]) : 0;
  const int32_t r8 = (len + 7) & ~7;
  const int32_t jo = warp_incl_scan(r8) - r8;
  float av[kTileMaxA];
  int32_t rp[kTileMaxA];
  {
    const int32_t seg = a_rp[__reduce_max_sync(kFull, active ? row : row0) + 1] - seg0;
    const int32_t *scol = reinterpret_cast<const int32_t *>(work);
    const float *sval = work + seg;
#pragma unroll
    for (int j = 0; j < kTileMaxA; ++j) {
      av[j] = 0.0f;
      rp[j] = 0;
      if (j < na && active) {
        av[j] = sval[my_p + j];
        rp[j] = __ldg(b_rp + scol[my_p + j]);
      }
    }
  }
  __syncwarp();  // the work area becomes the stage buffers

  const uint4 *const tq = reinterpret_cast<const uint4 *>(tab + size_t(pid) * kTileTabStride);
  // A ring of kTileStages stage buffers: the B span of A nonzero j + S - 1 is
  // requested while j is computed, so S - 1 spans are always in flight.
  // Every iteration commits one cp.async group (empty past the row's end),
  // so waiting for all but the newest S - 1 groups means span j is in.
  int32_t c0s[kTileStages];
#pragma unroll
  for (int j = 0; j < kTileStages - 1; ++j) {
    c0s[j] = 0;
    if (j < kTileMaxA && j < na) {
      const int32_t lj = __shfl_sync(kFull, len, j);
      const int32_t lo = __reduce_min_sync(kFull, active ? rp[j] : INT_MAX);
      const int32_t hi = __reduce_max_sync(kFull, active ? rp[j] + lj : INT_MIN);
      c0s[j] = stage_span(work + j * stage_cap, b_val, lo, hi, b_nnz, aligned16, lane);
    }
    cp_async_commit();
  }
#pragma unroll
  for (int j = 0; j < kTileMaxA; ++j) {
    if (j >= na) break;
    constexpr int kS = kTileStages;
    const int jn = j + kS - 1;
    if (jn < kTileMaxA && jn < na) {
      const int32_t ln = __shfl_sync(kFull, len, jn);
      const int32_t lo = __reduce_min_sync(kFull, active ? rp[jn] : INT_MAX);
      const int32_t hi = __reduce_max_sync(kFull, active ? rp[jn] + ln : INT_MIN);
      c0s[jn % kS] =
          stage_span(work + (jn % kS) * stage_cap, b_val, lo, hi, b_nnz, aligned16, lane);
    }
    cp_async_commit();
    cp_async_wait<kS - 1>();
    __syncwarp();
    const float *st = work + (j % kS) * stage_cap;
    const int32_t bl = active ? rp[j] - c0s[j % kS] : 0;
    const float aj = av[j];
    const int32_t lj = __shfl_sync(kFull, len, j);
    const uint4 *tj = tq + (__shfl_sync(kFull, jo, j) >> 3);
    float *const accl = acc + lane;
    for (int32_t g = 0; g < ((lj + 7) >> 3); ++g) {
      const uint4 s8 = tj[g];
      const uint32_t wv[4] = {s8.x, s8.y, s8.z, s8.w};
      float b[8], v[8];
      uint32_t u[8];
#pragma unroll
      for (int i = 0; i < 8; ++i) {
        u[i] = (wv[i >> 1] >> ((i & 1) * 16)) & 0xffffu;
        b[i] = __fmul_rn(aj, st[bl + g * 8 + i]);
      }
#pragma unroll
      for (int i = 0; i < 8; ++i)
        v[i] = (u[i] & kFirst) ? 0.0f : accl[(u[i] & 0x7fffu) * 33];
#pragma unroll
      for (int i = 0; i < 8; ++i) accl[(u[i] & 0x7fffu) * 33] = __fadd_rn(v[i], b[i]);
    }
    __syncwarp();  // every lane is done with this buffer before it is refilled
  }
  cp_async_wait<0>();  // (only empty groups can be left)
  // C: each row's m values, lanes over positions (coalesced)
  for (int r = 0; r < 32; ++r) {
    const int32_t base = __shfl_sync(kFull, cs, r);
    if (!((mask >> r) & 1u)) continue;
    for (int32_t q = lane; q < m; q += 32) c_val[base + q] = acc[q * 33 + r];
  }
}

// rows / ids: every row with pid_of_row[row] >= 0, in chunk order.
__global__ void __launch_bounds__(256)
tile_list_kernel(int32_t n, const int32_t *__restrict__ pid_of_row, int32_t *__restrict__ rows,
                 int32_t *__restrict__ ids, int32_t *__restrict__ count) {
  const int32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  const int32_t pid = i < n ? pid_of_row[i] : -1;
  const unsigned b = __ballot_sync(kFull, pid >= 0);
  if (!b) return;
  int32_t base = 0;
  if (lane_id() == 0) base = atomicAdd(count, __popc(b));
  base = __shfl_sync(kFull, base, 0);
  if (pid >= 0) {
    const int32_t at = base + __popc(b & lanemask_lt());
    rows[at] = i;
    ids[at] = pid;
  }
}

}  // namespace

int32_t tile_tab_stride() { return kTileTabStride; }

void launch_tile_list(int32_t n, const int32_t *pid_of_row, int32_t *rows, int32_t *ids,
                      int32_t *count, cudaStream_t s) {
  if (n <= 0) return;
  tile_list_kernel<<<(n + 255) / 256, 256, 0, s>>>(n, pid_of_row, rows, ids, count);
}

void launch_tile_tab(int32_t npat, const int32_t *pat_canon, const int32_t *psteps,
                     const int32_t *a_rp, const int32_t *a_col, const int32_t *b_rp,
                     const int32_t *c_rp, const int64_t *moff, const uint16_t *map,
                     uint16_t *tab, uint16_t *lens, int4 *desc, cudaStream_t s) {
  if (npat <= 0) return;
  tile_tab_kernel<<<(npat + 3) / 4, 128, 0, s>>>(npat, pat_canon, psteps, a_rp, a_col, b_rp,
                                                 c_rp, moff, map, kTileMaxOut, tab, lens, desc);
}

void launch_tile_build(int32_t n, const int32_t *pid_of_row, const int4 *desc,
                       const uint16_t *lens, const int32_t *a_rp, const int32_t *a_col,
                       const int32_t *b_rp, const int32_t *c_rp, int4 *tiles, int32_t *ntiles,
                       int32_t *lo_rows, int32_t *lo_ids, int32_t *lo_n, int32_t *maxima,
                       cudaStream_t s) {
  if (n <= 0) return;
  const int64_t chunks = (int64_t(n) + 31) / 32;
  const int64_t grid = (chunks + kBuildWarps - 1) / kBuildWarps;
  tile_build_kernel<<<static_cast<unsigned>(grid), kBuildWarps * 32, 0, s>>>(
      n, pid_of_row, desc, lens, a_rp, a_col, b_rp, c_rp, tiles, ntiles, lo_rows, lo_ids, lo_n,
      maxima);
}

size_t tile_smem_per_warp(int32_t stage_need, int32_t a_seg, int32_t max_out,
                          int32_t *acc_rows, int32_t *work_floats, int32_t *stage_cap) {
  *acc_rows = max_out + 1;
  *stage_cap = (stage_need + 3) & ~3;
  const int32_t work = kTileStages * *stage_cap > 2 * a_seg ? kTileStages * *stage_cap
                                                            : 2 * a_seg;
  *work_floats = (work + 3) & ~3;
  const int32_t acc_floats = (*acc_rows * 33 + 3) & ~3;
  return size_t(acc_floats + *work_floats) * sizeof(float);
}

void launch_tile_numeric(const Operands &op, int32_t b_nnz, const int4 *tiles, int32_t ntiles,
                         const int4 *desc, const uint16_t *lens, const uint16_t *tab,
                         const int32_t *c_rp, float *c_val, int32_t stage_need, int32_t a_seg,
                         int32_t max_out, cudaStream_t s) {
  if (ntiles <= 0) return;
  int32_t acc_rows = 0, work_floats = 0, stage_cap = 0;
  const size_t per_warp =
      tile_smem_per_warp(stage_need, a_seg, max_out, &acc_rows, &work_floats, &stage_cap);
  const size_t smem = per_warp * kTileKernelWarps;
  cudaFuncSetAttribute(tile_numeric_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       static_cast<int>(smem));
  const int64_t grid = (int64_t(ntiles) + kTileKernelWarps - 1) / kTileKernelWarps;
  tile_numeric_kernel<<<static_cast<unsigned>(grid), kTileKernelWarps * 32, smem, s>>>(
      op.a_rp, op.a_col, op.a_val, op.b_rp, op.b_val, b_nnz, tiles, ntiles, desc, lens, tab,
      c_rp, c_val, acc_rows, work_floats, stage_cap);
}

}  // namespace rvsp
