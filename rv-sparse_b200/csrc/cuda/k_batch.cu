// Batches: packing many independent products into one operand pair per
// group, and the per-product views of the packed result (C-ABI, declared in
// include/rvsp_cuda.h).  No reference counterpart: the reference computes
// one product per call (spgemm.c:135-210, spgemm_descr.c:66-380).
//
// Every kernel runs a 2-D grid: blockIdx.y strides over the products,
// blockIdx.x and the threads stride over one product's rows or entries, so
// one launch covers products of any mix of sizes.  Copies are coalesced.
#include "device_common.cuh"
#include "kernels.cuh"
#include "rvsp_cuda.h"

namespace rvsp {

namespace {

constexpr int kBT = 256;

int grid_y(int32_t count) { return count < 65535 ? count : 65535; }

__global__ void __launch_bounds__(kBT)
batch_entries_kernel(rvsp_cuda_batch_item_t *items, int32_t count) {
  const int32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= count) return;
  items[i].a_nnz = items[i].a_row_ptr[items[i].a_rows];
  items[i].b_nnz = items[i].b_row_ptr[items[i].b_rows];
}

__global__ void __launch_bounds__(kBT)
batch_ops_kernel(const rvsp_cuda_batch_item_t *__restrict__ items, int32_t count,
                 int64_t *__restrict__ ops, int32_t *__restrict__ err) {
  for (int32_t p = blockIdx.y; p < count; p += gridDim.y) {
    const rvsp_cuda_batch_item_t it = items[p];
    long long acc = 0;
    bool bad = false;
    for (int32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < it.a_nnz;
         j += gridDim.x * blockDim.x) {
      const int32_t k = __ldg(it.a_col_idx + j);
      if (static_cast<uint32_t>(k) >= static_cast<uint32_t>(it.b_rows)) {
        bad = true;
        continue;
      }
      acc += __ldg(it.b_row_ptr + k + 1) - __ldg(it.b_row_ptr + k);
    }
    acc = warp_sum64(acc);
    if (lane_id() == 0 && acc)
      atomicAdd(reinterpret_cast<unsigned long long *>(ops + p),
                static_cast<unsigned long long>(acc));
    if (bad) atomicOr(err, 1);
  }
}

__global__ void __launch_bounds__(kBT)
batch_pack_kernel(const rvsp_cuda_batch_item_t *__restrict__ items,
                  const rvsp_cuda_batch_offset_t *__restrict__ off, int32_t count,
                  bool with_structure, int32_t *__restrict__ a_rp,
                  int32_t *__restrict__ a_ci, float *__restrict__ a_v,
                  int32_t *__restrict__ b_rp, int32_t *__restrict__ b_ci,
                  float *__restrict__ b_v, int32_t *__restrict__ err) {
  const int32_t t0 = blockIdx.x * blockDim.x + threadIdx.x;
  const int32_t st = gridDim.x * blockDim.x;
  for (int32_t p = blockIdx.y; p < count; p += gridDim.y) {
    const rvsp_cuda_batch_item_t it = items[p];
    const rvsp_cuda_batch_offset_t o = off[p];
    int bad = 0;
    if (with_structure) {
      if (t0 == 0 && (it.a_row_ptr[0] != 0 || it.b_row_ptr[0] != 0)) bad |= 8;
      // Row pointers [0, rows] inclusive: a product's last entry and the
      // next product's first are the same value, written by both.
      for (int32_t r = t0; r <= it.a_rows; r += st) a_rp[o.a_row + r] = o.a_nnz + it.a_row_ptr[r];
      for (int32_t j = t0; j < it.a_nnz; j += st) {
        const int32_t k = __ldg(it.a_col_idx + j);
        if (static_cast<uint32_t>(k) >= static_cast<uint32_t>(it.b_rows)) bad |= 2;
        a_ci[o.a_nnz + j] = k + o.b_row;
      }
      for (int32_t r = t0; r <= it.b_rows; r += st) b_rp[o.b_row + r] = o.b_nnz + it.b_row_ptr[r];
      for (int32_t j = t0; j < it.b_nnz; j += st) {
        const int32_t c = __ldg(it.b_col_idx + j);
        if (static_cast<uint32_t>(c) >= static_cast<uint32_t>(it.b_cols)) bad |= 4;
        b_ci[o.b_nnz + j] = c;
      }
    }
    for (int32_t j = t0; j < it.a_nnz; j += st) a_v[o.a_nnz + j] = __ldg(it.a_values + j);
    for (int32_t j = t0; j < it.b_nnz; j += st) b_v[o.b_nnz + j] = __ldg(it.b_values + j);
    if (bad) atomicOr(err, bad);
  }
}

__global__ void __launch_bounds__(kBT)
batch_views_kernel(const rvsp_cuda_batch_item_t *__restrict__ items,
                   const rvsp_cuda_batch_offset_t *__restrict__ off,
                   const int64_t *__restrict__ crp_off, int32_t count,
                   const int32_t *__restrict__ c_rp, int32_t *__restrict__ out,
                   int32_t *__restrict__ base_out, int32_t *__restrict__ nnz_out) {
  const int32_t t0 = blockIdx.x * blockDim.x + threadIdx.x;
  const int32_t st = gridDim.x * blockDim.x;
  for (int32_t p = blockIdx.y; p < count; p += gridDim.y) {
    const int32_t rows = items[p].a_rows;
    const int32_t r0 = off[p].a_row;
    const int32_t base = c_rp[r0];
    int32_t *dst = out + crp_off[p];
    for (int32_t r = t0; r <= rows; r += st) dst[r] = c_rp[r0 + r] - base;
    if (t0 == 0) {
      base_out[p] = base;
      nnz_out[p] = c_rp[r0 + rows] - base;
    }
  }
}

rvsp_status_t status_of(cudaError_t e) {
  if (e == cudaSuccess) return RVSP_SUCCESS;
  return e == cudaErrorMemoryAllocation ? RVSP_ERROR_ALLOCATION_FAILED : RVSP_ERROR_DEVICE;
}

}  // namespace

}  // namespace rvsp

extern "C" {

rvsp_status_t rvsp_cuda_batch_entries(void *stream, rvsp_cuda_batch_item_t *items,
                                      int32_t count) {
  if (count < 0) return RVSP_ERROR_INVALID_ARGUMENT;
  if (count == 0) return RVSP_SUCCESS;
  if (!items) return RVSP_ERROR_NULL_POINTER;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  rvsp::batch_entries_kernel<<<(count + rvsp::kBT - 1) / rvsp::kBT, rvsp::kBT, 0, s>>>(
      items, count);
  return rvsp::status_of(cudaGetLastError());
}

rvsp_status_t rvsp_cuda_batch_op_counts(void *stream, const rvsp_cuda_batch_item_t *items,
                                        int32_t count, int64_t *ops, int32_t *err) {
  if (count < 0) return RVSP_ERROR_INVALID_ARGUMENT;
  if (count == 0) return RVSP_SUCCESS;
  if (!items || !ops || !err) return RVSP_ERROR_NULL_POINTER;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const dim3 grid(32, rvsp::grid_y(count));
  rvsp::batch_ops_kernel<<<grid, rvsp::kBT, 0, s>>>(items, count, ops, err);
  return rvsp::status_of(cudaGetLastError());
}

rvsp_status_t rvsp_cuda_batch_pack(void *stream, const rvsp_cuda_batch_item_t *items,
                                   const rvsp_cuda_batch_offset_t *off, int32_t count,
                                   int with_structure, int32_t *a_row_ptr,
                                   int32_t *a_col_idx, float *a_values,
                                   int32_t *b_row_ptr, int32_t *b_col_idx,
                                   float *b_values, int32_t *err) {
  if (count < 0) return RVSP_ERROR_INVALID_ARGUMENT;
  if (count == 0) return RVSP_SUCCESS;
  if (!items || !off || !a_values || !b_values || !err) return RVSP_ERROR_NULL_POINTER;
  if (with_structure && (!a_row_ptr || !a_col_idx || !b_row_ptr || !b_col_idx))
    return RVSP_ERROR_NULL_POINTER;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const dim3 grid(64, rvsp::grid_y(count));
  rvsp::batch_pack_kernel<<<grid, rvsp::kBT, 0, s>>>(items, off, count, with_structure != 0,
                                                     a_row_ptr, a_col_idx, a_values,
                                                     b_row_ptr, b_col_idx, b_values, err);
  return rvsp::status_of(cudaGetLastError());
}

rvsp_status_t rvsp_cuda_batch_views(void *stream, const rvsp_cuda_batch_item_t *items,
                                    const rvsp_cuda_batch_offset_t *off,
                                    const int64_t *crp_off, int32_t count,
                                    const int32_t *c_row_ptr, int32_t *c_rp_out,
                                    int32_t *base_out, int32_t *nnz_out) {
  if (count < 0) return RVSP_ERROR_INVALID_ARGUMENT;
  if (count == 0) return RVSP_SUCCESS;
  if (!items || !off || !crp_off || !c_row_ptr || !c_rp_out || !base_out || !nnz_out)
    return RVSP_ERROR_NULL_POINTER;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const dim3 grid(8, rvsp::grid_y(count));
  rvsp::batch_views_kernel<<<grid, rvsp::kBT, 0, s>>>(items, off, crp_off, count, c_row_ptr,
                                                      c_rp_out, base_out, nnz_out);
  return rvsp::status_of(cudaGetLastError());
}

}  // extern "C"
