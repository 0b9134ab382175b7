// The plan: device-resident analysis state of one product and the C-ABI
// entry points of rvsp_cuda.h that drive the kernel phases.
//
// Flow of rvsp_cuda_symbolic (the GPU form of rvsp_symbolic_count,
// rvsp_symbolic.c:13-86):
//   rowstats -> [host: symbolic class sizes] -> scatter rows by class ->
//   symbolic kernel per class -> scan + numeric classes ->
//   [host: total, numeric class sizes, status] -> scatter rows by class.
// Two host round trips, both for sizes the host must know (grid shapes and
// nnz(C), which the API returns).  rvsp_cuda_numeric then launches one kernel
// per non-empty numeric class with no host round trip.
#include <cuda_runtime.h>

#include <climits>
#include <cstring>
#include <new>
#include <vector>

#include "device_common.cuh"
#include "kernels.cuh"
#include "rvsp_cuda.h"

using namespace rvsp;

namespace {

template <class T>
struct DevArray {
  T *p = nullptr;
  size_t cap = 0;
  cudaError_t reserve(size_t n) {
    if (n <= cap && p) return cudaSuccess;
    release();
    if (n == 0) n = 1;
    cudaError_t e = cudaMalloc(reinterpret_cast<void **>(&p), n * sizeof(T));
    if (e != cudaSuccess) {
      p = nullptr;
      return e;
    }
    cap = n;
    return cudaSuccess;
  }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    cap = 0;
  }
};

rvsp_status_t map_cuda(cudaError_t e) {
  switch (e) {
    case cudaSuccess: return RVSP_SUCCESS;
    case cudaErrorMemoryAllocation: return RVSP_ERROR_ALLOCATION_FAILED;
    case cudaErrorNoDevice:
    case cudaErrorInsufficientDriver:
    case cudaErrorNoKernelImageForDevice:
    case cudaErrorInvalidDevice: return RVSP_ERROR_UNSUPPORTED_BACKEND;
    default: return RVSP_ERROR_DEVICE;
  }
}

// misc int32 words
constexpr int kSymCount = 0;
constexpr int kSymOff = kNumClasses;
constexpr int kSymFill = 2 * kNumClasses;
constexpr int kNumCount = 3 * kNumClasses;
constexpr int kNumOff = 4 * kNumClasses;
constexpr int kNumFill = 5 * kNumClasses;
constexpr int kStatus = 6 * kNumClasses;
constexpr int kLongCount = 6 * kNumClasses + 1;
constexpr int kMiscWords = 6 * kNumClasses + 2;

}  // namespace

struct rvsp_cuda_plan {
  int device = 0;
  int num_sms = 148;

  int analysed = 0;
  int32_t a_rows = 0, b_rows = 0, b_cols = 0;
  int64_t c_nnz = 0;

  DevArray<int64_t> ops;
  DevArray<uint8_t> cls;
  DevArray<int32_t> counts;
  DevArray<int32_t> rows_sym, rows_num, long_rows;
  DevArray<int32_t> misc;
  DevArray<int64_t> partials, total;
  DevArray<uint32_t> sym_bits;
  DevArray<unsigned long long> check;
  int32_t sym_bits_slots = 0;

  int32_t *h_misc = nullptr;  // pinned, kMiscWords
  int64_t *h_total = nullptr;  // pinned
  unsigned long long *h_check = nullptr;  // pinned

  int32_t sym_count[kNumClasses] = {};
  int32_t num_count[kNumClasses] = {};
  int32_t num_off[kNumClasses] = {};
  int32_t dense_slots = 0;
  size_t numeric_ws = 0;

  bool profiling = false;
  struct Pending {
    cudaEvent_t a, b;
    int phase;
    int launches;
  };
  std::vector<Pending> pending;
  std::vector<cudaEvent_t> pool;
  double ms[RVSP_PHASE_COUNT] = {};
  int64_t launches[RVSP_PHASE_COUNT] = {};

  cudaEvent_t take_event() {
    if (!pool.empty()) {
      cudaEvent_t e = pool.back();
      pool.pop_back();
      return e;
    }
    cudaEvent_t e = nullptr;
    cudaEventCreate(&e);
    return e;
  }
};

namespace {

struct PhaseScope {
  rvsp_cuda_plan *pl;
  cudaStream_t s;
  int phase;
  int launches = 0;
  cudaEvent_t a = nullptr;
  PhaseScope(rvsp_cuda_plan *p, cudaStream_t st, int ph) : pl(p), s(st), phase(ph) {
    if (pl->profiling) {
      a = pl->take_event();
      cudaEventRecord(a, s);
    }
  }
  ~PhaseScope() {
    if (pl->profiling && a) {
      cudaEvent_t b = pl->take_event();
      cudaEventRecord(b, s);
      pl->pending.push_back({a, b, phase, launches});
    }
  }
};

void resolve_pending(rvsp_cuda_plan *pl) {
  for (auto &q : pl->pending) {
    float t = 0.0f;
    if (cudaEventSynchronize(q.b) == cudaSuccess &&
        cudaEventElapsedTime(&t, q.a, q.b) == cudaSuccess) {
      pl->ms[q.phase] += t;
    }
    pl->launches[q.phase] += q.launches;
    pl->pool.push_back(q.a);
    pl->pool.push_back(q.b);
  }
  pl->pending.clear();
}

rvsp_status_t device_status_to_rvsp(int32_t st) {
  return st == kDevOk ? RVSP_SUCCESS : RVSP_ERROR_DEVICE;
}

}  // namespace

extern "C" {

rvsp_status_t rvsp_cuda_plan_create(rvsp_cuda_plan_t *plan) {
  if (!plan) return RVSP_ERROR_NULL_POINTER;
  *plan = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= 0) {
    cudaGetLastError();
    return RVSP_ERROR_UNSUPPORTED_BACKEND;
  }
  int dev = 0, major = 0, minor = 0, sms = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return RVSP_ERROR_UNSUPPORTED_BACKEND;
  cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev);
  cudaDeviceGetAttribute(&minor, cudaDevAttrComputeCapabilityMinor, dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (major != 10 || minor != 0) return RVSP_ERROR_UNSUPPORTED_BACKEND;
  rvsp_cuda_plan *p = new (std::nothrow) rvsp_cuda_plan();
  if (!p) return RVSP_ERROR_ALLOCATION_FAILED;
  p->device = dev;
  p->num_sms = sms > 0 ? sms : 148;
  cudaError_t e = p->misc.reserve(kMiscWords);
  if (e == cudaSuccess) e = p->total.reserve(1);
  if (e == cudaSuccess) e = p->check.reserve(1);
  if (e == cudaSuccess) e = cudaMallocHost(reinterpret_cast<void **>(&p->h_misc), kMiscWords * sizeof(int32_t));
  if (e == cudaSuccess) e = cudaMallocHost(reinterpret_cast<void **>(&p->h_total), sizeof(int64_t));
  if (e == cudaSuccess) e = cudaMallocHost(reinterpret_cast<void **>(&p->h_check), sizeof(unsigned long long));
  if (e == cudaSuccess) e = cudaMemset(p->misc.p, 0, kMiscWords * sizeof(int32_t));
  if (e != cudaSuccess) {
    rvsp_cuda_plan_destroy(p);
    return map_cuda(e);
  }
  *plan = p;
  return RVSP_SUCCESS;
}

void rvsp_cuda_plan_destroy(rvsp_cuda_plan_t p) {
  if (!p) return;
  resolve_pending(p);
  for (cudaEvent_t e : p->pool) cudaEventDestroy(e);
  p->ops.release();
  p->cls.release();
  p->counts.release();
  p->rows_sym.release();
  p->rows_num.release();
  p->long_rows.release();
  p->misc.release();
  p->partials.release();
  p->total.release();
  p->sym_bits.release();
  p->check.release();
  if (p->h_misc) cudaFreeHost(p->h_misc);
  if (p->h_total) cudaFreeHost(p->h_total);
  if (p->h_check) cudaFreeHost(p->h_check);
  delete p;
}

rvsp_status_t rvsp_cuda_symbolic(rvsp_cuda_plan_t p, void *stream, int32_t a_rows,
                                 int32_t b_rows, int32_t b_cols,
                                 const int32_t *a_row_ptr,
                                 const int32_t *a_col_idx,
                                 const int32_t *b_row_ptr,
                                 const int32_t *b_col_idx, int32_t *c_row_ptr,
                                 int64_t *c_nnz_out) {
  if (!p || !a_row_ptr || !a_col_idx || !b_row_ptr || !b_col_idx || !c_row_ptr ||
      !c_nnz_out)
    return RVSP_ERROR_NULL_POINTER;
  if (a_rows <= 0 || b_rows <= 0 || b_cols <= 0) return RVSP_ERROR_INVALID_ARGUMENT;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  p->analysed = 0;
  const size_t n = static_cast<size_t>(a_rows);

  cudaError_t e = p->ops.reserve(n);
  if (e == cudaSuccess) e = p->cls.reserve(n);
  if (e == cudaSuccess) e = p->counts.reserve(n);
  if (e == cudaSuccess) e = p->rows_sym.reserve(n);
  if (e == cudaSuccess) e = p->rows_num.reserve(n);
  if (e == cudaSuccess) e = p->long_rows.reserve(n);
  if (e == cudaSuccess) e = p->partials.reserve(scan_partials_bytes(a_rows) / sizeof(int64_t));
  if (e != cudaSuccess) return map_cuda(e);

  const Operands op{a_rows, b_cols, a_row_ptr, a_col_idx, nullptr,
                    b_row_ptr, b_col_idx, nullptr};
  int32_t *misc = p->misc.p;
  cudaMemsetAsync(misc, 0, kMiscWords * sizeof(int32_t), s);
  {
    PhaseScope ph(p, s, RVSP_PHASE_ROWSTATS);
    launch_rowstats(op, p->ops.p, p->cls.p, p->counts.p, misc + kSymCount,
                    p->long_rows.p, misc + kLongCount, a_rows, s);
    launch_rowstats_long(op, p->long_rows.p, misc + kLongCount, p->ops.p, p->cls.p,
                         p->counts.p, misc + kSymCount, p->num_sms, s);
    ph.launches = 2;
  }
  cudaMemcpyAsync(p->h_misc, misc, kNumClasses * sizeof(int32_t),
                  cudaMemcpyDeviceToHost, s);
  e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return map_cuda(e);
  int32_t sym_off[kNumClasses];
  int32_t off = 0;
  for (int c = 0; c < kNumClasses; ++c) {
    p->sym_count[c] = p->h_misc[kSymCount + c];
    sym_off[c] = off;
    if (c != kEmpty_) off += p->sym_count[c];
  }

  // Global bitmaps for dense symbolic rows when B is too wide for shared memory.
  const size_t bits_bytes = dense_slot_bits_bytes(b_cols);
  int32_t slots = 0;
  if (p->sym_count[kDense] > 0 && bits_bytes > 0) {
    slots = p->sym_count[kDense] < p->num_sms ? p->sym_count[kDense] : p->num_sms;
    const size_t words = bits_bytes / sizeof(uint32_t) * size_t(slots);
    if (words > p->sym_bits.cap) {
      e = p->sym_bits.reserve(words);
      if (e != cudaSuccess) return map_cuda(e);
      cudaMemsetAsync(p->sym_bits.p, 0, words * sizeof(uint32_t), s);
    }
    p->sym_bits_slots = slots;
  }
  {
    PhaseScope ph(p, s, RVSP_PHASE_SYMBOLIC);
    launch_class_offsets(misc + kSymCount, misc + kSymOff, s);
    launch_scatter_rows(a_rows, p->cls.p, misc + kSymOff, misc + kSymFill,
                        p->rows_sym.p, s);
    ph.launches = 2;
    for (int c = kEmpty_ + 1; c < kNumClasses; ++c) {
      if (p->sym_count[c] <= 0) continue;
      launch_symbolic_class(c, op, p->rows_sym.p + sym_off[c],
                            p->sym_count[c], p->counts.p, p->sym_bits.p, slots,
                            misc + kStatus, p->num_sms, s);
      ph.launches += 1;
    }
  }
  {
    PhaseScope ph(p, s, RVSP_PHASE_SCAN);
    launch_scan_and_class(a_rows, p->counts.p, p->ops.p, a_row_ptr, c_row_ptr,
                          p->partials.p,
                          p->total.p, p->cls.p, misc + kNumCount, s);
    ph.launches = 3;
  }
  cudaMemcpyAsync(p->h_misc + kNumCount, misc + kNumCount,
                  (kMiscWords - kNumCount) * sizeof(int32_t), cudaMemcpyDeviceToHost, s);
  cudaMemcpyAsync(p->h_total, p->total.p, sizeof(int64_t), cudaMemcpyDeviceToHost, s);
  e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return map_cuda(e);
  if (p->h_misc[kStatus] != kDevOk) {
    cudaMemsetAsync(misc + kStatus, 0, sizeof(int32_t), s);
    return RVSP_ERROR_DEVICE;
  }
  const int64_t total = *p->h_total;
  if (total > INT32_MAX) return RVSP_ERROR_ALLOCATION_FAILED;

  off = 0;
  for (int c = 0; c < kNumClasses; ++c) {
    p->num_count[c] = p->h_misc[kNumCount + c];
    p->num_off[c] = off;
    if (c != kEmpty_) off += p->num_count[c];
  }
  {
    PhaseScope ph(p, s, RVSP_PHASE_SCAN);
    launch_class_offsets(misc + kNumCount, misc + kNumOff, s);
    launch_scatter_rows(a_rows, p->cls.p, misc + kNumOff, misc + kNumFill,
                        p->rows_num.p, s);
    ph.launches = 2;
  }

  if (p->num_count[kDense] > 0) {
    p->dense_slots = p->num_count[kDense] < p->num_sms ? p->num_count[kDense] : p->num_sms;
    p->numeric_ws = size_t(p->dense_slots) *
                    (dense_slot_acc_bytes(b_cols) + dense_slot_bits_bytes(b_cols));
  } else {
    p->dense_slots = 0;
    p->numeric_ws = 0;
  }
  e = cudaGetLastError();
  if (e != cudaSuccess) return map_cuda(e);

  p->a_rows = a_rows;
  p->b_rows = b_rows;
  p->b_cols = b_cols;
  p->c_nnz = total;
  p->analysed = 1;
  *c_nnz_out = total;
  return RVSP_SUCCESS;
}

size_t rvsp_cuda_numeric_workspace_bytes(rvsp_cuda_plan_t p) {
  return (p && p->analysed) ? p->numeric_ws : 0;
}

rvsp_status_t rvsp_cuda_numeric(rvsp_cuda_plan_t p, void *stream,
                                const int32_t *a_row_ptr, const int32_t *a_col_idx,
                                const float *a_values, const int32_t *b_row_ptr,
                                const int32_t *b_col_idx, const float *b_values,
                                const int32_t *c_row_ptr, int32_t *c_col_idx,
                                float *c_values, int fill, void *workspace,
                                size_t workspace_bytes) {
  if (!p || !a_row_ptr || !a_col_idx || !a_values || !b_row_ptr || !b_col_idx ||
      !b_values || !c_row_ptr || !c_col_idx || !c_values)
    return RVSP_ERROR_NULL_POINTER;
  if (!p->analysed) return RVSP_ERROR_INVALID_ARGUMENT;
  if (p->numeric_ws > 0 && (!workspace || workspace_bytes < p->numeric_ws))
    return workspace ? RVSP_ERROR_INVALID_ARGUMENT : RVSP_ERROR_NULL_POINTER;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const Operands op{p->a_rows, p->b_cols, a_row_ptr, a_col_idx, a_values,
                    b_row_ptr, b_col_idx, b_values};
  float *dense_acc = static_cast<float *>(workspace);
  uint32_t *dense_bits = nullptr;
  if (p->numeric_ws > 0) {
    // The dense accumulators (and global bitmaps) must start zeroed; every
    // row leaves what it touched zeroed again, but the caller owns this
    // memory between calls, so clear it each time.
    cudaMemsetAsync(workspace, 0, p->numeric_ws, s);
    dense_bits = reinterpret_cast<uint32_t *>(
        static_cast<char *>(workspace) +
        size_t(p->dense_slots) * dense_slot_acc_bytes(p->b_cols));
  }
  {
    PhaseScope ph(p, s, RVSP_PHASE_NUMERIC);
    for (int c = kEmpty_ + 1; c < kNumClasses; ++c) {
      if (p->num_count[c] <= 0) continue;
      launch_numeric_class(c, op, p->ops.p, p->rows_num.p + p->num_off[c],
                           p->num_count[c], c_row_ptr, c_col_idx, c_values,
                           fill != 0, dense_acc, dense_bits, p->dense_slots,
                           p->misc.p + kStatus, p->num_sms, s);
      ph.launches += 1;
    }
  }
  return map_cuda(cudaGetLastError());
}

rvsp_status_t rvsp_cuda_op_counts(rvsp_cuda_plan_t p, void *stream,
                                  int64_t *host_out, int32_t n) {
  if (!p || !host_out) return RVSP_ERROR_NULL_POINTER;
  if (!p->analysed) return RVSP_ERROR_INVALID_ARGUMENT;
  if (n < p->a_rows) return RVSP_ERROR_INVALID_ARGUMENT;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  cudaError_t e = cudaMemcpyAsync(host_out, p->ops.p, size_t(p->a_rows) * sizeof(int64_t),
                                  cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  return map_cuda(e);
}

rvsp_status_t rvsp_cuda_plan_status(rvsp_cuda_plan_t p, void *stream) {
  if (!p) return RVSP_ERROR_NULL_POINTER;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  int32_t st = 0;
  cudaError_t e = cudaMemcpyAsync(&st, p->misc.p + kStatus, sizeof(int32_t),
                                  cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return map_cuda(e);
  if (st != kDevOk) {
    cudaMemsetAsync(p->misc.p + kStatus, 0, sizeof(int32_t), s);
    cudaStreamSynchronize(s);
  }
  return device_status_to_rvsp(st);
}

rvsp_status_t rvsp_cuda_csr_check(rvsp_cuda_plan_t p, void *stream, int32_t rows,
                                  int32_t cols, const int32_t *row_ptr,
                                  const int32_t *col_idx, int32_t nnz,
                                  int32_t *code_out, int32_t *bad_row_out) {
  if (!p || !code_out || !bad_row_out) return RVSP_ERROR_NULL_POINTER;
  *code_out = 1;  // malformed row pointer
  *bad_row_out = -1;
  if (!row_ptr || rows < 0 || cols < 0 || nnz < 0) return RVSP_SUCCESS;
  if (nnz > 0 && !col_idx) return RVSP_SUCCESS;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  cudaMemsetAsync(p->check.p, 0xff, sizeof(unsigned long long), s);
  {
    PhaseScope ph(p, s, RVSP_PHASE_CHECK);
    launch_csr_check(rows, cols, row_ptr, col_idx, nnz, p->check.p, s);
    ph.launches = 1;
  }
  cudaMemcpyAsync(p->h_check, p->check.p, sizeof(unsigned long long),
                  cudaMemcpyDeviceToHost, s);
  cudaError_t e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return map_cuda(e);
  const unsigned long long r = *p->h_check;
  if (r == ~0ull) {
    *code_out = 0;
    *bad_row_out = -1;
  } else {
    *code_out = static_cast<int32_t>(r & 0xffu);
    *bad_row_out = static_cast<int32_t>(r >> 8) - 1;
  }
  return RVSP_SUCCESS;
}

rvsp_status_t rvsp_cuda_plan_set_profiling(rvsp_cuda_plan_t p, int enable) {
  if (!p) return RVSP_ERROR_NULL_POINTER;
  p->profiling = enable != 0;
  return RVSP_SUCCESS;
}

rvsp_status_t rvsp_cuda_plan_phase_times(rvsp_cuda_plan_t p, double *ms_out,
                                         int64_t *launches_out, int32_t n,
                                         int reset) {
  if (!p) return RVSP_ERROR_NULL_POINTER;
  resolve_pending(p);
  for (int i = 0; i < n && i < RVSP_PHASE_COUNT; ++i) {
    if (ms_out) ms_out[i] = p->ms[i];
    if (launches_out) launches_out[i] = p->launches[i];
  }
  if (reset) {
    for (int i = 0; i < RVSP_PHASE_COUNT; ++i) {
      p->ms[i] = 0.0;
      p->launches[i] = 0;
    }
  }
  return RVSP_SUCCESS;
}

rvsp_status_t rvsp_cuda_plan_class_counts(rvsp_cuda_plan_t p, int32_t *sym_out,
                                          int32_t *num_out, int32_t n) {
  if (!p) return RVSP_ERROR_NULL_POINTER;
  for (int i = 0; i < n; ++i) {
    const bool in = i < kNumClasses;
    if (sym_out) sym_out[i] = in ? p->sym_count[i] : 0;
    if (num_out) num_out[i] = in ? p->num_count[i] : 0;
  }
  return RVSP_SUCCESS;
}

}  // extern "C"
