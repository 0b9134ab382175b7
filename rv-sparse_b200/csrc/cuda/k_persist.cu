// Persistent numeric-only pass: one launch for the merge rows and the map
// rows of a plan (every product of a batch group, k_batch.cu), pulling work
// from a global queue of row bins.
//
// The queue is the plan's numeric row lists cut into items: a merge-class
// item is up to `per_item` rows (a thread each, the K-way merge of
// merge_lists.cuh writing values into C's known structure), a map-class
// item is 8 rows (a warp each, the map walk of map_walk.cuh).  Items are
// numbered heaviest class first (W2048 ... W64, then M16 ... M4), and each
// block of kPersistThreads threads takes the next item with one atomicAdd on
// a counter the launch clears first; the grid is blocks_per_sm blocks per SM,
// so the launch needs no host-side knowledge of how the rows are spread.
// There is no spin-wait: a block that draws a number past the last item
// returns.
//
// Order and rounding are those of the per-class kernels (k_merge.cu,
// k_reuse.cu): every output gets its terms in ascending A-nonzero order from
// +0.0f with separately rounded products and sums (the reference's order,
// gustavson_core_f32.inc:31-62), so results are bit-identical to them.
#include <climits>

#include "device_common.cuh"
#include "kernels.cuh"
#include "map_walk.cuh"
#include "merge_lists.cuh"

namespace rvsp {

namespace {

using namespace merge;

// Values of one merge row whose structure is in C (no staging, no fill).
template <int K>
__device__ __forceinline__ void merge_value_row(const Operands &op, int32_t row,
                                                const int32_t *__restrict__ c_rp,
                                                float *__restrict__ c_val,
                                                int32_t *__restrict__ status) {
  const int32_t p0 = op.a_rp[row];
  const int32_t k = op.a_rp[row + 1] - p0;
  Lists<K> L;
  open_lists<K, true>(op, p0, k, L);
  const int64_t out0 = c_rp[row], out_end = c_rp[row + 1];
  int64_t out = out0;
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
    if (out < out_end) c_val[out] = acc;
    ++out;
  }
  if (out != out_end) report(status, kDevCountMismatch);
}

__global__ void __launch_bounds__(kPersistThreads)
persist_numeric_kernel(Operands op, const int64_t *__restrict__ ops, PersistPlan pp,
                       int32_t *__restrict__ head, const int32_t *__restrict__ c_rp,
                       float *__restrict__ c_val, const int64_t *__restrict__ moff,
                       const uint16_t *__restrict__ map, int32_t *__restrict__ status,
                       int32_t acc_floats) {
  extern __shared__ __align__(16) float smem_f32[];
  __shared__ int32_t s_item;
  const int tid = threadIdx.x, lane = lane_id(), wid = tid >> 5;
  float *const acc = smem_f32 + size_t(wid) * acc_floats;
  for (;;) {
    if (tid == 0) s_item = atomicAdd(head, 1);
    __syncthreads();
    const int32_t item = s_item;
    __syncthreads();  // every thread has read s_item before it is drawn again
    if (item >= pp.n_items) return;
    int sg = 0;
    while (sg + 1 < pp.nseg && pp.seg[sg + 1].item0 <= item) ++sg;
    const PersistSeg g = pp.seg[sg];
    const int32_t local = (item - g.item0) * g.per_item;
    const int32_t cnt = min(g.per_item, g.count - local);
    if (g.cls == kM4 || g.cls == kM8 || g.cls == kM16) {
      if (tid < cnt) {
        const int32_t row = row_of(g.rows, local + tid);
        if (g.cls == kM4) merge_value_row<4>(op, row, c_rp, c_val, status);
        else if (g.cls == kM8) merge_value_row<8>(op, row, c_rp, c_val, status);
        else merge_value_row<16>(op, row, c_rp, c_val, status);
      }
    } else {
      for (int32_t r = wid; r < cnt; r += kPersistThreads / 32)
        map_numeric_row(op, ops, row_of(g.rows, local + r), c_rp, c_val, moff, map, status,
                        acc, lane);
    }
  }
}

}  // namespace

bool persist_class(int cls) { return is_merge_class(cls) || map_class(cls); }

void launch_persist_numeric(const Operands &op, const int64_t *ops, const PersistPlan &pp,
                            int32_t *head, const int32_t *c_rp, float *c_val,
                            const int64_t *moff, const uint16_t *map, int32_t *status,
                            int32_t max_map_out, int blocks_per_sm, int num_sms,
                            cudaStream_t s) {
  if (pp.n_items <= 0) return;
  const int32_t acc_floats = (max_map_out + 3) & ~3;
  const size_t smem = size_t(kPersistThreads / 32) * size_t(acc_floats) * sizeof(float);
  cudaFuncSetAttribute(persist_numeric_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       static_cast<int>(smem));
  cudaMemsetAsync(head, 0, sizeof(int32_t), s);
  int grid = num_sms * (blocks_per_sm > 0 ? blocks_per_sm : 1);
  if (grid > pp.n_items) grid = pp.n_items;
  persist_numeric_kernel<<<grid, kPersistThreads, smem, s>>>(op, ops, pp, head, c_rp, c_val,
                                                             moff, map, status, acc_floats);
}

}  // namespace rvsp
