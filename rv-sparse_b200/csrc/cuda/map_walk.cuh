// The map walk of one row (k_reuse.cu), shared with the persistent numeric
// kernel (k_persist.cu): C's row values from the reuse map, one warp, into a
// shared-memory accumulator of at least the row's C length.  Each output gets
// its terms in ascending A-nonzero order from +0.0f, rounded separately:
// stepping (one A nonzero at a time, lanes over its B row, whose positions
// are distinct) for long B rows, flattened tiles with ordered_apply for short
// ones.
#pragma once

#include "device_common.cuh"
#include "kernels.cuh"

namespace rvsp {

constexpr int kMapSteppingMinAvgLen = 16;  // same rule as the plain walkers

__device__ __forceinline__ void map_numeric_row(const Operands &op,
                                                const int64_t *__restrict__ ops, int32_t row,
                                                const int32_t *__restrict__ c_rp,
                                                float *__restrict__ c_val,
                                                const int64_t *__restrict__ moff,
                                                const uint16_t *__restrict__ map,
                                                int32_t *__restrict__ status, float *acc,
                                                int lane) {
  const int32_t cs = c_rp[row];
  const int m = c_rp[row + 1] - cs;
  for (int e = lane; e < m; e += 32) acc[e] = 0.0f;
  __syncwarp();
  const int64_t base = moff[row];
  const int32_t p0 = op.a_rp[row], p1 = op.a_rp[row + 1];
  const bool stepping =
      ops[row] >= static_cast<int64_t>(kMapSteppingMinAvgLen) * (p1 - p0);
  bool bad = false;
  int64_t run = 0;
  for (int32_t p = p0; p < p1; p += 32) {
    const AChunk c = load_chunk(op.a_col, op.a_val, op.b_rp, p + lane, p1, true);
    if (stepping) {
      const int cnt = min(32, p1 - p);
      for (int jj = 0; jj < cnt; ++jj) {
        const int len = __shfl_sync(kFull, c.len, jj);
        const int bbeg = __shfl_sync(kFull, c.bbeg, jj);
        const float a = __shfl_sync(kFull, c.a, jj);
        const int64_t k0 = base + run + __shfl_sync(kFull, c.incl - c.len, jj);
        for (int e = lane; e < len; e += 32) {
          const int pos = __ldg(map + k0 + e);
          const float term = __fmul_rn(a, __ldg(op.b_val + bbeg + e));
          if (pos < m) acc[pos] = __fadd_rn(acc[pos], term);
          else bad = true;
        }
        __syncwarp();
      }
    } else {
      for (int t0 = 0; t0 < c.total; t0 += 32) {
        const int t = t0 + lane;
        bool v = t < c.total;
        const int j = warp_owner_of(c.incl, v ? t : 0);
        const int excl = __shfl_sync(kFull, c.incl - c.len, j);
        const int bbeg = __shfl_sync(kFull, c.bbeg, j);
        const float a = __shfl_sync(kFull, c.a, j);
        int pos = 0;
        float term = 0.0f;
        if (v) {
          pos = __ldg(map + base + run + t);
          if (pos >= m) {
            bad = true;
            v = false;
          } else {
            term = __fmul_rn(a, __ldg(op.b_val + bbeg + (t - excl)));
          }
        }
        ordered_apply(acc, v, pos, term);
      }
    }
    run += c.total;
  }
  __syncwarp();
  for (int e = lane; e < m; e += 32) c_val[cs + e] = acc[e];
  if (__any_sync(kFull, bad) && lane == 0) report(status, kDevKeyMissing);
}

}  // namespace rvsp
