// Order-free expansion of a row's products, shared by the counting kernels.
#pragma once

#include "device_common.cuh"
#include "kernels.cuh"

namespace rvsp {

// Calls f(col) for every product of A row [p0, p1) that this warp owns.  The
// row's A nonzeros are split into 32-wide chunks; chunk c goes to warp
// (c % nwarps == wid).  Products are expanded 32 at a time in flattened order
// (all lanes busy whatever the B row lengths).  Loop bounds are warp-uniform.
template <typename F>
__device__ __forceinline__ void for_each_product_col(const Operands &op,
                                                     int32_t p0, int32_t p1,
                                                     int wid, int nwarps, F f) {
  const int lane = lane_id();
  for (int32_t p = p0 + wid * 32; p < p1; p += nwarps * 32) {
    const AChunk c = load_chunk(op.a_col, op.a_val, op.b_rp, p + lane, p1, false);
    for (int t0 = 0; t0 < c.total; t0 += 32) {
      const int t = t0 + lane;
      const bool v = t < c.total;
      const int j = warp_owner_of(c.incl, v ? t : 0);
      const int excl = __shfl_sync(kFull, c.incl - c.len, j);
      const int bbeg = __shfl_sync(kFull, c.bbeg, j);
      if (v) f(__ldg(op.b_col + bbeg + (t - excl)));
    }
  }
}

}  // namespace rvsp
