// Term tables: numeric-only repeats of rows that share one reuse map.
//
// A structured matrix (a stencil, a finite-element mesh) repeats a handful of
// row patterns over most of its rows: rows whose products land at the same
// positions of C's row in the same order (the reuse map finds them, k_reuse.cu).
// Such a pattern gets a table with two parts:
//
//   stage records, one per product t in flattened order (A nonzero j, entry e
//   of B row A_col[j]): the warp computes prod[t] = a[j] * B_val[bbeg[j] + e]
//   into shared memory, 32 consecutive products per step, so B is read in
//   row runs;
//   term records, per lane: the outputs dealt to that lane (about the same
//   number of terms each), each output's products t in ascending j:
//     acc = acc + prod[t]; if last: out[q] = acc, acc = +0.0f
//
// then C's row is written from `out` in one coalesced pass.  There is no
// shared accumulator and no step-to-step synchronisation.  Each output's terms
// are summed by one lane, from +0.0f, in ascending A-nonzero order with every
// product and every sum rounded -- the reference scalar kernel's order
// (gustavson_core_f32.inc:31-62, accum_scalar_f32.c:20-71) -- so the values
// are the plain path's bit for bit.
//
// Stage record (uint32): j bits 0-4 | e bits 5-31 (the tail of the last step
// reads j = 0, e = 0 and its products are never summed).  Term record
// (uint32): last bit 1 | 4 t bits 2-15 | 4 q bits 16-31 (byte offsets into
// prod and out); a lane with fewer terms than the table's steps reads zero
// records, which add prod[0] to an accumulator that is never written.  Both
// are stored step-major, rec[s * 32 + lane]: one 128-byte line per warp step.
#include <climits>

#include "device_common.cuh"
#include "kernels.cuh"

namespace rvsp {

namespace {

constexpr int kPatMaxA = 32;      // A nonzeros of a tabled row (a lane each)
constexpr int kPatMaxOps = 1024;  // products of a tabled row (prod[] in shared memory)
constexpr int kPatMaxOut = 512;   // C entries of a tabled row (out[] in shared memory)
constexpr int kPatBuildThreads = 256;
constexpr uint32_t kTermLast = 2u;

// Counters after the row counts in pat_counts: largest products (rounded up
// to 32) and largest C row over the tables, which size the shared memory.
constexpr int kMaxOpsWord = 0, kMaxOutWord = 1;

// A canonical row (its own map, shared by at least min_share - 1 other rows)
// that fits the record fields gets a table: pat_of[row] = id,
// pat_canon[id] = row, pat_cap[id] = records reserved: ceil(ops / 32) stage
// steps plus at most nA + ceil(ops / 32) term steps (outputs sorted by term
// count and dealt in alternating directions, each output with at most nA
// terms, so no lane carries more than that).
__global__ void __launch_bounds__(256)
pat_select_kernel(const int32_t *__restrict__ rows, int32_t nrows,
                  const int32_t *__restrict__ canon, const int32_t *__restrict__ share_count,
                  int32_t min_share, const int32_t *__restrict__ a_rp,
                  const int32_t *__restrict__ c_rp, const int32_t *__restrict__ mops,
                  int32_t *__restrict__ pat_of, int32_t *__restrict__ pat_canon,
                  int32_t *__restrict__ pat_cap, int32_t *__restrict__ npat,
                  int32_t *__restrict__ maxima) {
  const int32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nrows) return;
  const int32_t row = row_of(rows, i);
  if (canon[row] != row) return;
  const int32_t na = a_rp[row + 1] - a_rp[row];
  const int32_t ops = mops[row];
  const int32_t m = c_rp[row + 1] - c_rp[row];
  if (share_count[row] + 1 < min_share || na <= 0 || na > kPatMaxA || ops <= 0 ||
      ops > kPatMaxOps || m <= 0 || m > kPatMaxOut)
    return;
  const int32_t id = atomicAdd(npat, 1);
  const int32_t tiles = (ops + 31) / 32;
  pat_of[row] = id;
  pat_canon[id] = row;
  pat_cap[id] = (2 * tiles + na) * 32;
  atomicMax(maxima + kMaxOpsWord, tiles * 32);
  atomicMax(maxima + kMaxOutWord, m);
}

// One block per table, from the canonical row's map.  psteps[id] = term
// steps of the table, or -1 when the map held a position outside C's row
// (the rows of that pattern keep the map path).
__global__ void __launch_bounds__(kPatBuildThreads)
pat_build_kernel(const int32_t *__restrict__ pat_canon, const int32_t *__restrict__ a_rp,
                 const int32_t *__restrict__ a_col, const int32_t *__restrict__ b_rp,
                 const int32_t *__restrict__ c_rp, const int64_t *__restrict__ moff,
                 const uint16_t *__restrict__ map, const int64_t *__restrict__ pat_off,
                 const int32_t *__restrict__ pat_cap, uint32_t *__restrict__ rec,
                 int32_t *__restrict__ psteps) {
  __shared__ int32_t cnt[kPatMaxOut];
  __shared__ int32_t start[kPatMaxOut + 1];
  __shared__ int32_t sorted[kPatMaxOut];
  __shared__ uint16_t terms[kPatMaxOps];
  __shared__ int32_t bucket[kPatMaxA + 2];
  __shared__ int32_t bad;
  const int id = blockIdx.x;
  const int tid = threadIdx.x, lane = lane_id();
  const int32_t row = pat_canon[id];
  const int32_t p0 = a_rp[row], na = a_rp[row + 1] - p0;
  const int32_t m = c_rp[row + 1] - c_rp[row];
  if (na > kPatMaxA || m > kPatMaxOut) {  // does not fit the tables
    if (tid == 0) psteps[id] = -1;
    return;
  }
  const int64_t base = moff[row];
  uint32_t *const tab = rec + pat_off[id];
  for (int q = tid; q < m; q += kPatBuildThreads) cnt[q] = 0;
  if (tid <= kPatMaxA + 1) bucket[tid] = 0;
  if (tid == 0) bad = 0;
  __syncthreads();
  // 1. stage records, terms per output, and the product count (warp 0 walks
  //    A's row one nonzero at a time)
  int32_t ops = 0;
  if (tid < 32) {
    for (int32_t j = 0; j < na; ++j) {
      const int32_t k = __ldg(a_col + p0 + j);
      const int32_t bb = __ldg(b_rp + k), len = __ldg(b_rp + k + 1) - bb;
      for (int32_t e = lane; e < len; e += 32) {
        const int32_t t = ops + e;
        const int q = t < kPatMaxOps ? __ldg(map + base + t) : INT_MAX;
        if (q < m) {
          cnt[q] += 1;  // distinct positions within one B row
          tab[t] = static_cast<uint32_t>(j) | (static_cast<uint32_t>(e) << 5);
        } else {
          bad = 1;
        }
      }
      __syncwarp();
      ops += len;
    }
    if (ops > kPatMaxOps) bad = 1;
  }
  __syncthreads();
  if (bad) {
    if (tid == 0) psteps[id] = -1;
    return;
  }
  const int32_t tiles = (ops + 31) / 32;  // uniform in warp 0, the only user
  // 2. starts, and the outputs sorted by term count (descending; counting
  //    sort, serial: at most kPatMaxOut outputs, once per table)
  if (tid == 0) {
    int32_t run = 0;
    for (int q = 0; q < m; ++q) {
      start[q] = run;
      run += cnt[q];
      bucket[cnt[q]] += 1;
    }
    start[m] = run;
    int32_t off = 0;
    for (int v = kPatMaxA; v >= 0; --v) {
      const int32_t c = bucket[v];
      bucket[v] = off;
      off += c;
    }
    for (int q = 0; q < m; ++q) sorted[bucket[cnt[q]]++] = q;
  }
  __syncthreads();
  if (tid >= 32) return;
  // 3. each output's products in ascending j (one A nonzero at a time; the
  //    positions of one B row are distinct, so the cursors do not collide)
  for (int t = ops + lane; t < tiles * 32; t += 32) tab[t] = 0u;  // tail of the stage
  for (int q = lane; q < m; q += 32) cnt[q] = start[q];
  __syncwarp();
  {
    int32_t t0 = 0;
    for (int32_t j = 0; j < na; ++j) {
      const int32_t k = __ldg(a_col + p0 + j);
      const int32_t len = __ldg(b_rp + k + 1) - __ldg(b_rp + k);
      for (int32_t e = lane; e < len; e += 32) {
        const int q = __ldg(map + base + t0 + e);
        terms[cnt[q]++] = static_cast<uint16_t>(t0 + e);
      }
      __syncwarp();
      t0 += len;
    }
  }
  // 4. deal: block b of 32 sorted outputs goes to lanes 0..31 when b is even,
  //    31..0 when odd; lane loads, then the term records
  int32_t load = 0;
  for (int b = 0; b * 32 < m; ++b) {
    const int i = b * 32 + ((b & 1) ? 31 - lane : lane);
    if (i < m) {
      const int q = sorted[i];
      load += start[q + 1] - start[q];
    }
  }
  int32_t steps = load;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) steps = max(steps, __shfl_xor_sync(kFull, steps, o));
  if (tiles * 32 + steps * 32 > pat_cap[id]) {  // cannot happen (see pat_select_kernel)
    if (lane == 0) psteps[id] = -1;
    return;
  }
  uint32_t *out = tab + tiles * 32 + lane;
  int32_t s = 0;
  for (int b = 0; b * 32 < m; ++b) {
    const int i = b * 32 + ((b & 1) ? 31 - lane : lane);
    if (i >= m) continue;
    const int q = sorted[i];
    for (int32_t t = start[q]; t < start[q + 1]; ++t, ++s) {
      uint32_t x = (static_cast<uint32_t>(terms[t]) << 2) | (static_cast<uint32_t>(q) << 18);
      if (t == start[q + 1] - 1) x |= kTermLast;
      out[size_t(s) * 32] = x;
    }
  }
  for (; s < steps; ++s) out[size_t(s) * 32] = 0u;
  if (lane == 0) psteps[id] = steps;
}

// Splits one class's rows: a row whose canonical row has a table, and whose
// own A row has the canonical's length and B row lengths (the records name
// A nonzeros and B entries, not just positions), goes to the table list
// (pat_rows, pat_ids; count at *pat_n, and pid_of_row[row] = id when
// pid_of_row is given); the rest to res_rows (count *res_n), which keep the
// map path.
__global__ void __launch_bounds__(256)
pat_split_kernel(const int32_t *__restrict__ rows, int32_t nrows,
                 const int32_t *__restrict__ canon, const int32_t *__restrict__ pat_of,
                 const int32_t *__restrict__ psteps, const int32_t *__restrict__ a_rp,
                 const int32_t *__restrict__ a_col, const int32_t *__restrict__ b_rp,
                 int32_t *__restrict__ pat_rows, int32_t *__restrict__ pat_ids,
                 int32_t *__restrict__ pat_n, int32_t *__restrict__ res_rows,
                 int32_t *__restrict__ res_n, int32_t *__restrict__ pid_of_row) {
  const int32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  const int lane = lane_id();
  const bool valid = i < nrows;
  int32_t row = 0, pid = -1;
  if (valid) {
    row = row_of(rows, i);
    const int32_t c = canon[row];
    pid = c >= 0 ? pat_of[c] : -1;
    if (pid >= 0 && psteps[pid] < 0) pid = -1;
    if (pid >= 0 && c != row) {
      const int32_t pr = a_rp[row], na = a_rp[row + 1] - pr;
      const int32_t pc = a_rp[c];
      if (na != a_rp[c + 1] - pc) {
        pid = -1;
      } else {
        for (int32_t j = 0; j < na; ++j) {
          const int32_t kr = a_col[pr + j], kc = a_col[pc + j];
          if (b_rp[kr + 1] - b_rp[kr] != b_rp[kc + 1] - b_rp[kc]) {
            pid = -1;
            break;
          }
        }
      }
    }
  }
  const unsigned to_pat = __ballot_sync(kFull, valid && pid >= 0);
  const unsigned to_res = __ballot_sync(kFull, valid && pid < 0);
  const unsigned below = (1u << lane) - 1;
  int32_t base = 0;
  if (to_pat) {
    if (lane == 0) base = atomicAdd(pat_n, __popc(to_pat));
    base = __shfl_sync(kFull, base, 0);
    if (valid && pid >= 0) {
      const int32_t at = base + __popc(to_pat & below);
      pat_rows[at] = row;
      pat_ids[at] = pid;
      if (pid_of_row) pid_of_row[row] = pid;
    }
  }
  if (to_res) {
    if (lane == 0) base = atomicAdd(res_n, __popc(to_res));
    base = __shfl_sync(kFull, base, 0);
    if (valid && pid < 0) res_rows[base + __popc(to_res & below)] = row;
  }
}

// Values of the table rows: warp per row (see the file comment).  Shared
// memory per warp: prod[prod_cap] | out[out_cap] floats.
__global__ void __launch_bounds__(kWarpsPerBlock * 32)
pat_numeric_kernel(const int32_t *__restrict__ a_rp, const int32_t *__restrict__ a_col,
                   const float *__restrict__ a_val, const int32_t *__restrict__ b_rp,
                   const float *__restrict__ b_val, const int64_t *__restrict__ ops,
                   const int32_t *__restrict__ pat_rows, const int32_t *__restrict__ pat_ids,
                   int32_t n, const int32_t *__restrict__ c_rp, float *__restrict__ c_val,
                   const int64_t *__restrict__ pat_off, const int32_t *__restrict__ psteps,
                   const uint32_t *__restrict__ rec, int prod_cap, int out_cap) {
  extern __shared__ __align__(16) float smem_f32[];
  float *prod = smem_f32 + size_t(threadIdx.x >> 5) * (prod_cap + out_cap);
  float *outv = prod + prod_cap;
  const int64_t w = (int64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
  if (w >= n) return;
  const int lane = lane_id();
  const int32_t row = pat_rows[w];
  const int32_t pid = pat_ids[w];
  const int32_t p0 = a_rp[row], na = a_rp[row + 1] - p0;
  float a = 0.0f;
  int32_t bb = 0;
  if (lane < na) {
    a = __ldg(a_val + p0 + lane);
    bb = __ldg(b_rp + __ldg(a_col + p0 + lane));
  }
  const uint32_t *tab = rec + pat_off[pid];
  const int32_t tiles = static_cast<int32_t>((ops[row] + 31) >> 5);
  const int32_t steps = psteps[pid];
  // products, 32 consecutive ones per step
  {
    const uint32_t *st = tab + lane;
#pragma unroll 4
    for (int32_t s = 0; s < tiles; ++s) {
      const uint32_t x = __ldg(st + s * 32);
      const float av = __shfl_sync(kFull, a, x & 31);
      const int32_t bv = __shfl_sync(kFull, bb, x & 31);
      prod[s * 32 + lane] = __fmul_rn(av, __ldg(b_val + bv + (x >> 5)));
    }
  }
  __syncwarp();
  // every lane's outputs, each from +0.0f in ascending A-nonzero order
  {
    const uint32_t *tr = tab + tiles * 32 + lane;
    const char *pb = reinterpret_cast<const char *>(prod);
    char *ob = reinterpret_cast<char *>(outv);
    float acc = 0.0f;
#pragma unroll 4
    for (int32_t s = 0; s < steps; ++s) {
      const uint32_t x = __ldg(tr + s * 32);
      acc = __fadd_rn(acc, *reinterpret_cast<const float *>(pb + (x & 0xfffcu)));
      if (x & kTermLast) {
        *reinterpret_cast<float *>(ob + (x >> 16)) = acc;
        acc = 0.0f;
      }
    }
  }
  __syncwarp();
  const int32_t cs = c_rp[row], m = min(c_rp[row + 1] - cs, out_cap);
  for (int32_t q = lane; q < m; q += 32) c_val[cs + q] = outv[q];
}

}  // namespace

void launch_pat_select(const int32_t *rows, int32_t nrows, const int32_t *canon,
                       const int32_t *share_count, int32_t min_share, const int32_t *a_rp,
                       const int32_t *c_rp, const int32_t *mops, int32_t *pat_of,
                       int32_t *pat_canon, int32_t *pat_cap, int32_t *npat, int32_t *maxima,
                       cudaStream_t s) {
  if (nrows <= 0) return;
  pat_select_kernel<<<(nrows + 255) / 256, 256, 0, s>>>(rows, nrows, canon, share_count,
                                                         min_share, a_rp, c_rp, mops, pat_of,
                                                         pat_canon, pat_cap, npat, maxima);
}

void launch_pat_build(int32_t npat, const int32_t *pat_canon, const int32_t *a_rp,
                      const int32_t *a_col, const int32_t *b_rp, const int32_t *c_rp,
                      const int64_t *moff, const uint16_t *map, const int64_t *pat_off,
                      const int32_t *pat_cap, uint32_t *rec, int32_t *psteps,
                      cudaStream_t s) {
  if (npat <= 0) return;
  pat_build_kernel<<<npat, kPatBuildThreads, 0, s>>>(pat_canon, a_rp, a_col, b_rp, c_rp,
                                                     moff, map, pat_off, pat_cap, rec,
                                                     psteps);
}

void launch_pat_split(const int32_t *rows, int32_t nrows, const int32_t *canon,
                      const int32_t *pat_of, const int32_t *psteps, const int32_t *a_rp,
                      const int32_t *a_col, const int32_t *b_rp, int32_t *pat_rows,
                      int32_t *pat_ids, int32_t *pat_n, int32_t *res_rows, int32_t *res_n,
                      int32_t *pid_of_row, cudaStream_t s) {
  if (nrows <= 0) return;
  pat_split_kernel<<<(nrows + 255) / 256, 256, 0, s>>>(rows, nrows, canon, pat_of, psteps,
                                                        a_rp, a_col, b_rp, pat_rows, pat_ids,
                                                        pat_n, res_rows, res_n, pid_of_row);
}

void launch_pat_numeric(const Operands &op, const int64_t *ops, const int32_t *pat_rows,
                        const int32_t *pat_ids, int32_t n, const int32_t *c_rp, float *c_val,
                        const int64_t *pat_off, const int32_t *psteps, const uint32_t *rec,
                        int32_t max_ops, int32_t max_out, cudaStream_t s) {
  if (n <= 0) return;
  const int prod_cap = (max_ops + 31) & ~31;
  const int out_cap = (max_out + 3) & ~3;
  const size_t smem = size_t(kWarpsPerBlock) * (prod_cap + out_cap) * sizeof(float);
  cudaFuncSetAttribute(pat_numeric_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       static_cast<int>(smem));
  const int64_t grid = (int64_t(n) + kWarpsPerBlock - 1) / kWarpsPerBlock;
  pat_numeric_kernel<<<static_cast<unsigned>(grid), kWarpsPerBlock * 32, smem, s>>>(
      op.a_rp, op.a_col, op.a_val, op.b_rp, op.b_val, ops, pat_rows, pat_ids, n, c_rp, c_val,
      pat_off, psteps, rec, prod_cap, out_cap);
}

}  // namespace rvsp
