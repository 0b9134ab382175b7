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

#include <algorithm>
#include <climits>
#include <cstring>
#include <new>
#include <utility>
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

// Page-locked host memory, grown on demand and kept: the tile builds'
// transfers go through it (a copy from or to pageable memory is staged and
// synchronous, tens of microseconds each).
struct HostArray {
  char *p = nullptr;
  size_t cap = 0;
  cudaError_t reserve(size_t n) {
    if (n <= cap && p) return cudaSuccess;
    release();
    if (cudaMallocHost(reinterpret_cast<void **>(&p), n ? n : 1) != cudaSuccess) {
      p = nullptr;
      return cudaErrorMemoryAllocation;
    }
    cap = n;
    return cudaSuccess;
  }
  void release() {
    if (p) cudaFreeHost(p);
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
constexpr int kRetryCount = 6 * kNumClasses + 2;  // two: W1024, W2048 retry lists
constexpr int kShiftMembers = 6 * kNumClasses + 4;  // shift-class member rows
constexpr int kShiftNpat = 6 * kNumClasses + 5;     // shift-class pattern candidates
constexpr int kMiscWords = 6 * kNumClasses + 6;
// A map shared by at least this many rows gets a term table.
constexpr int32_t kPatMinShare = 16;
constexpr int kPatCountWords = 4 + kNumClasses;

}  // namespace

namespace rvsp {
// Row tiles over one set of term-table patterns (k_tile.cu): per pattern its
// tile table, B row lengths and shape; per row its pattern (pid, -1 for rows
// outside the set); the tiles and the pattern rows left to the warp-per-row
// table kernel (lo_rows / lo_ids); for the shift classes also every pattern
// row (all_rows / all_ids, for when tiles are off).
struct JitPattern {
  void *kernel = nullptr;
  DevArray<int4> tiles;
  DevArray<int32_t> prog;  // tile records (k_jit.cu)
  DevArray<int2> arange;   // per tile its A range
  DevArray<int32_t> head;  // the launch's tile queue
  int32_t n = 0, m = 0, stage_cap = 0, abuf_floats = 0, work_floats = 0;
  int grid = 0;
  void release() {
    tiles.release();
    prog.release();
    arange.release();
    head.release();
  }
};
struct TileBuild {
  std::vector<JitPattern> jit;   // patterns with their own kernel (k_jit.cu)
  std::vector<JitPattern> pool;  // device arrays of earlier builds, for reuse
  DevArray<int32_t> jwords;      // per chosen pattern: spans, record extent
  DevArray<int2> jgroups;        // per chosen pattern: its staging groups
  HostArray staging;             // host side of the builds' transfers
  int ready = 0;
  int32_t n_tiles = 0, n_lo = 0, stage = 0, aseg = 0, max_out = 0, b_nnz = 0;
  DevArray<uint16_t> tab, lens;
  DevArray<int4> desc, tiles;
  DevArray<int4> table;  // the tiles left to the table kernel, when patterns are compiled
  int32_t n_table = 0;
  DevArray<int32_t> pid, lo_rows, lo_ids, counts, all_rows, all_ids;
  void release() {
    tab.release();
    lens.release();
    desc.release();
    tiles.release();
    table.release();
    n_table = 0;
    pid.release();
    lo_rows.release();
    lo_ids.release();
    counts.release();
    all_rows.release();
    all_ids.release();
    for (auto &j : jit) j.release();
    for (auto &j : pool) j.release();
    jit.clear();
    pool.clear();
    jwords.release();
    jgroups.release();
    staging.release();
    ready = 0;
  }
};
}  // namespace rvsp

struct rvsp_cuda_plan {
  int device = 0;
  int num_sms = 148;

  int analysed = 0;
  int merge_policy = kMergeAuto;
  int32_t a_rows = 0, b_rows = 0, b_cols = 0;
  int64_t c_nnz = 0;

  DevArray<int64_t> ops;
  DevArray<uint8_t> cls;
  // Numeric classes from the scan queued before the class census (plain
  // symbolic with merge classes); swapped into cls when that scan is final.
  DevArray<uint8_t> cls_spec;
  DevArray<int32_t> counts;
  DevArray<int32_t> rows_sym, rows_num, long_rows;
  DevArray<int32_t> misc;
  DevArray<int64_t> partials, total;
  DevArray<uint32_t> sym_bits;
  DevArray<unsigned long long> check;
  DevArray<int32_t> check_long;  // count + list of the long rows the check met
  DevArray<int32_t> check_long_b;  // the same for B in rvsp_cuda_symbolic_checked
  int32_t sym_bits_slots = 0;

  int32_t *h_misc = nullptr;  // pinned, kMiscWords
  int64_t *h_total = nullptr;  // pinned
  unsigned long long *h_check = nullptr;  // pinned

  int32_t sym_count[kNumClasses] = {};
  int32_t num_count[kNumClasses] = {};
  int32_t num_off[kNumClasses] = {};
  int32_t dense_slots = 0;
  size_t numeric_ws = 0;
  int num_whole = -1;  // numeric class holding every row (no row list), or -1

  // Learned (fused) analysis: per-row capacity and slab slot, the slab with
  // every non-overflowed row's sorted columns and values, the overflow rows
  // grouped by numeric class, and the fingerprint of the values used.
  int learned = 0;
  DevArray<int32_t> cap;
  DevArray<int64_t> slab_off;
  DevArray<int32_t> slab_col;
  DevArray<float> slab_val;
  DevArray<int32_t> ovf_rows, ovf_sorted;
  DevArray<int32_t> big_rows;  // count + list of the rows compacted by whole blocks
  DevArray<uint8_t> ovf_cls;
  DevArray<char> fused_ws;
  DevArray<unsigned long long> vhash;
  unsigned long long *h_vhash = nullptr;  // pinned, 2 words
  unsigned long long est_hash = 0;
  int32_t n_ovf = 0;
  int32_t a_nnz = 0, b_nnz = 0;
  int32_t ovf_num_count[kNumClasses] = {};
  int32_t ovf_num_off[kNumClasses] = {};
  int64_t slab_total = 0;

  // Reuse map of the W<T> rows (k_reuse.cu), built for one C column array
  // (rmap_col) of the current analysis; rmap_state 0 = not tried, 1 = built,
  // -1 = not used (no W rows, over the memory budget, or a row too long).
  DevArray<uint16_t> rmap;
  DevArray<int64_t> rmap_off;
  DevArray<int32_t> rmap_ops;
  // Sharing of identical maps: per-row fingerprints, the table they meet in,
  // and a counter of the rows that read another row's map.
  DevArray<unsigned long long> rmap_key, rmap_tkey;
  DevArray<int32_t> rmap_trow, rmap_shared, rmap_canon, rmap_share_count;
  // Term tables of the shared maps (k_pattern.cu): per table its records,
  // offset and steps; the rows that use one (pat_rows, pat_ids) and, per W
  // class, the rows that keep the map (res_rows at res_off[c], res_count[c]).
  int pat_ready = 0;
  int32_t n_pat = 0, n_pat_rows = 0;
  int32_t res_off[kNumClasses] = {};
  int32_t res_count[kNumClasses] = {};
  DevArray<int32_t> pat_of, pat_canon, pat_cap, pat_steps, pat_rows, pat_ids, res_rows;
  // [0] tables, [1] table rows, [2 + c] map rows of class c, then the
  // tables' largest products and C row
  DevArray<int32_t> pat_counts;
  int32_t pat_max_ops = 0, pat_max_out = 0;
  DevArray<int64_t> pat_off;
  DevArray<uint32_t> pat_rec;
  // Row tiles of the table rows of shared maps (k_tile.cu).
  int tiles_enabled = 1;
  int pattern_kernels = 1;  // compile kernels for the largest patterns (k_jit.cu)
  TileBuild rt;
  // Shift classes (k_shift.cu): rows that are translates of a canonical row.
  // The probe sets the device flag sh_on; shift_active when the current
  // analysis has member rows (pattern in st.pid).  Their patterns' term
  // tables (sh_*) and row tiles (st) are built from the canonical rows' maps
  // on the first numeric call (shift_tables 1, or -1 when that failed).
  // Persistent numeric-only pass (k_persist.cu): merge rows per item (0: off)
  // and blocks per SM.
  int32_t persist_merge_rows = 0, persist_blocks = 2;
  DevArray<int32_t> persist_head;
  int shift_enabled = 1;
  int shift_active = 0;
  int shift_tables = 0;
  int32_t shift_members = 0, shift_npat = 0, shift_cap_pat = 0;
  int32_t sh_max_ops = 0, sh_max_out = 0;
  DevArray<int32_t> sh_on, sh_trow, sh_bcls, sh_rcls, sh_share, sh_pat_of, sh_pat_canon,
      sh_pat_cap, sh_pat_m, sh_steps, sh_counts;
  DevArray<unsigned long long> sh_probe, sh_bkey, sh_rkey, sh_tkey;
  DevArray<int64_t> sh_moff, sh_pat_off;
  DevArray<uint16_t> sh_map;
  DevArray<uint32_t> sh_rec;
  TileBuild st;
  const int32_t *rmap_col = nullptr;
  int rmap_state = 0;
  int64_t rmap_entries = 0;

  // Side streams of the numeric-only pass (created on first use; state 0
  // untried, 1 ready, -1 unavailable).
  static constexpr int kSide = 6;
  cudaStream_t side[kSide] = {};
  cudaEvent_t fork_ev = nullptr, join_ev[kSide] = {};
  int side_state = 0;

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

// The plan's two side streams, created on first use (at the highest stream
// priority, on the plan's device, never while `s` is being captured).
bool side_streams(rvsp_cuda_plan *p, cudaStream_t s) {
  if (p->side_state == 0) {
    int dev = -1;
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    if (cudaGetDevice(&dev) != cudaSuccess || dev != p->device ||
        cudaStreamIsCapturing(s, &cap) != cudaSuccess || cap != cudaStreamCaptureStatusNone) {
      cudaGetLastError();
      return false;
    }
    p->side_state = -1;
    int least = 0, greatest = 0;
    bool ok = cudaDeviceGetStreamPriorityRange(&least, &greatest) == cudaSuccess &&
              cudaEventCreateWithFlags(&p->fork_ev, cudaEventDisableTiming) == cudaSuccess;
    for (int i = 0; i < rvsp_cuda_plan::kSide && ok; ++i)
      ok = cudaStreamCreateWithPriority(&p->side[i], cudaStreamNonBlocking, greatest) ==
               cudaSuccess &&
           cudaEventCreateWithFlags(&p->join_ev[i], cudaEventDisableTiming) == cudaSuccess;
    if (ok) p->side_state = 1;
    else cudaGetLastError();
  }
  return p->side_state == 1;
}

// Streams of one numeric-only pass.  Its row groups (pattern kernels, table
// tiles, leftover rows, class kernels) write disjoint rows of C and only
// read A, B and the plan's tables, so all but the largest go to the side
// streams, forked from the caller's stream and joined back into it: the
// small launches, each bound by the latency of a few long rows, run beside
// the large one and beside each other instead of after one another.  main()
// is the caller's stream; next() hands out the side streams in turn
// (without side streams, the caller's stream).
struct Lanes {
  rvsp_cuda_plan *pl;
  cudaStream_t s;
  bool forked = false;
  int turn = 0;
  Lanes(rvsp_cuda_plan *p, cudaStream_t st, bool want) : pl(p), s(st) {
    if (!(want && side_streams(p, st) && cudaEventRecord(p->fork_ev, st) == cudaSuccess)) return;
    bool ok = true;
    for (int i = 0; i < rvsp_cuda_plan::kSide; ++i)
      ok = ok && cudaStreamWaitEvent(p->side[i], p->fork_ev, 0) == cudaSuccess;
    forked = ok;
  }
  cudaStream_t main() const { return s; }
  cudaStream_t next() {
    if (!forked) return s;
    const cudaStream_t x = pl->side[turn];
    turn = (turn + 1) % rvsp_cuda_plan::kSide;
    return x;
  }
  void join() {
    if (!forked) return;
    for (int i = 0; i < rvsp_cuda_plan::kSide; ++i) {
      cudaEventRecord(pl->join_ev[i], pl->side[i]);
      cudaStreamWaitEvent(s, pl->join_ev[i], 0);
    }
    forked = false;
  }
  ~Lanes() { join(); }
};

rvsp_status_t device_status_to_rvsp(int32_t st) {
  return st == kDevOk ? RVSP_SUCCESS : RVSP_ERROR_DEVICE;
}

// The class that holds every non-empty row, when there is exactly one and
// its kernel may also see the empty rows (merge kernels handle them; the
// others are used only when there are none).  Its rows then need no list.
int whole_matrix_class(const int32_t *count, int32_t a_rows) {
  int found = -1;
  for (int c = kEmpty_ + 1; c < kNumClasses; ++c) {
    if (count[c] <= 0) continue;
    if (found >= 0) return -1;
    found = c;
  }
  if (found < 0 || count[found] + count[kEmpty_] != a_rows) return -1;
  const bool merge = found == kM4 || found == kM8 || found == kM16;
  return (count[kEmpty_] == 0 || merge) ? found : -1;
}

// After the final scan (class counts of the numeric pass in h_misc): host
// offsets, the row lists (unless one class holds every row) and the dense
// workspace the numeric pass will need.
void finish_numeric_bins(rvsp_cuda_plan *p, int32_t a_rows, int32_t b_cols,
                         cudaStream_t s) {
  int32_t *misc = p->misc.p;
  int32_t off = 0;
  for (int c = 0; c < kNumClasses; ++c) {
    p->num_count[c] = p->h_misc[kNumCount + c];
    p->num_off[c] = off;
    if (c != kEmpty_) off += p->num_count[c];
  }
  p->num_whole = p->shift_active ? -1 : whole_matrix_class(p->num_count, a_rows);
  if (p->num_whole < 0) {
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
}

// Reserves (and zeroes when grown) the global bitmaps dense symbolic rows use
// when B is too wide for a shared-memory bitmap; returns the slot count.
cudaError_t ensure_sym_bits(rvsp_cuda_plan *p, int32_t dense_rows, int32_t b_cols,
                            cudaStream_t s, int32_t *slots_out) {
  *slots_out = 0;
  const size_t bits_bytes = dense_slot_bits_bytes(b_cols);
  if (dense_rows <= 0 || bits_bytes == 0) return cudaSuccess;
  const int32_t slots = dense_rows < p->num_sms ? dense_rows : p->num_sms;
  const size_t words = bits_bytes / sizeof(uint32_t) * size_t(slots);
  if (words > p->sym_bits.cap) {
    cudaError_t e = p->sym_bits.reserve(words);
    if (e != cudaSuccess) return e;
    cudaMemsetAsync(p->sym_bits.p, 0, words * sizeof(uint32_t), s);
  }
  p->sym_bits_slots = slots;
  *slots_out = slots;
  return cudaSuccess;
}

unsigned long long values_fingerprint_launch(rvsp_cuda_plan *p, const float *a_val,
                                             int64_t a_n, const float *b_val, int64_t b_n,
                                             cudaStream_t s) {
  cudaMemsetAsync(p->vhash.p, 0, sizeof(unsigned long long), s);
  launch_values_hash(a_val, a_n, 0x41ull, p->vhash.p, s);
  launch_values_hash(b_val, b_n, 0x42ull << 40, p->vhash.p, s);
  cudaMemcpyAsync(p->h_vhash, p->vhash.p, sizeof(unsigned long long),
                  cudaMemcpyDeviceToHost, s);
  return 0;
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
  if (e == cudaSuccess) e = p->check.reserve(2);
  if (e == cudaSuccess) e = cudaMallocHost(reinterpret_cast<void **>(&p->h_misc), kMiscWords * sizeof(int32_t));
  if (e == cudaSuccess) e = cudaMallocHost(reinterpret_cast<void **>(&p->h_total), sizeof(int64_t));
  if (e == cudaSuccess) e = cudaMallocHost(reinterpret_cast<void **>(&p->h_check), 2 * sizeof(unsigned long long));
  if (e == cudaSuccess) e = cudaMallocHost(reinterpret_cast<void **>(&p->h_vhash), 2 * sizeof(unsigned long long));
  if (e == cudaSuccess) e = p->vhash.reserve(2);
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
  for (int i = 0; i < rvsp_cuda_plan::kSide; ++i) {
    if (p->side[i]) cudaStreamDestroy(p->side[i]);
    if (p->join_ev[i]) cudaEventDestroy(p->join_ev[i]);
  }
  if (p->fork_ev) cudaEventDestroy(p->fork_ev);
  p->rmap.release();
  p->rmap_off.release();
  p->rmap_ops.release();
  p->rmap_key.release();
  p->rmap_tkey.release();
  p->rmap_trow.release();
  p->rmap_shared.release();
  p->rmap_canon.release();
  p->rmap_share_count.release();
  p->pat_of.release();
  p->pat_canon.release();
  p->pat_cap.release();
  p->pat_steps.release();
  p->pat_rows.release();
  p->pat_ids.release();
  p->res_rows.release();
  p->pat_counts.release();
  p->pat_off.release();
  p->pat_rec.release();
  p->rt.release();
  p->st.release();
  p->persist_head.release();
  for (auto *a : {&p->sh_on, &p->sh_trow, &p->sh_bcls, &p->sh_rcls, &p->sh_share,
                  &p->sh_pat_of, &p->sh_pat_canon, &p->sh_pat_cap, &p->sh_pat_m,
                  &p->sh_steps, &p->sh_counts})
    a->release();
  for (auto *a : {&p->sh_probe, &p->sh_bkey, &p->sh_rkey, &p->sh_tkey}) a->release();
  p->sh_moff.release();
  p->sh_pat_off.release();
  p->sh_map.release();
  p->sh_rec.release();
  p->ops.release();
  p->cls.release();
  p->cls_spec.release();
  p->counts.release();
  p->rows_sym.release();
  p->rows_num.release();
  p->long_rows.release();
  p->misc.release();
  p->partials.release();
  p->total.release();
  p->sym_bits.release();
  p->check.release();
  p->check_long.release();
  p->check_long_b.release();
  p->cap.release();
  p->slab_off.release();
  p->slab_col.release();
  p->slab_val.release();
  p->ovf_rows.release();
  p->ovf_sorted.release();
  p->ovf_cls.release();
  p->fused_ws.release();
  p->vhash.release();
  if (p->h_misc) cudaFreeHost(p->h_misc);
  if (p->h_total) cudaFreeHost(p->h_total);
  if (p->h_check) cudaFreeHost(p->h_check);
  if (p->h_vhash) cudaFreeHost(p->h_vhash);
  delete p;
}

namespace {

// Matrices of at least this many rows run the shift-class probe.
// The shift analysis runs by default (setting 1) on matrices of at least
// kShiftMinRows rows whose sampled rows average kShiftMinMeanOps products;
// setting 2 runs it on any matrix whose rows are translates.
constexpr int32_t kShiftMinRows = 32768;
constexpr int32_t kShiftMinMeanOps = 64;
int32_t shift_bar(const rvsp_cuda_plan *p) { return p->shift_enabled == 2 ? 0 : kShiftMinMeanOps; }
bool shift_size_ok(const rvsp_cuda_plan *p, int32_t a_rows) {
  return p->shift_enabled == 2 ? a_rows >= 64 : a_rows >= kShiftMinRows;
}

// Scratch of the shift-class analysis (k_shift.cu).  The key table is a
// power of two of at least twice the rows; a larger one kept from before is
// used whole.
cudaError_t reserve_shift(rvsp_cuda_plan *p, int32_t a_rows, int32_t b_rows) {
  const size_t n = static_cast<size_t>(a_rows), nb = static_cast<size_t>(b_rows);
  size_t tcap = 64;
  while (tcap < 2 * (n > nb ? n : nb)) tcap <<= 1;
  p->shift_cap_pat = static_cast<int32_t>(n / kPatMinShare + 1);
  const size_t cp = static_cast<size_t>(p->shift_cap_pat);
  cudaError_t e = p->sh_on.reserve(1);
  if (e == cudaSuccess) e = p->sh_probe.reserve(2 * size_t(shift_samples()));
  if (e == cudaSuccess) e = p->sh_bkey.reserve(nb);
  if (e == cudaSuccess) e = p->sh_rkey.reserve(n);
  if (e == cudaSuccess) e = p->sh_tkey.reserve(tcap);
  if (e == cudaSuccess) e = p->sh_trow.reserve(p->sh_tkey.cap);
  if (e == cudaSuccess) e = p->sh_bcls.reserve(nb);
  if (e == cudaSuccess) e = p->sh_rcls.reserve(n);
  if (e == cudaSuccess) e = p->sh_share.reserve(n);
  if (e == cudaSuccess) e = p->sh_pat_of.reserve(n);
  if (e == cudaSuccess) e = p->st.pid.reserve(n);
  if (e == cudaSuccess) e = p->sh_pat_canon.reserve(cp);
  if (e == cudaSuccess) e = p->sh_pat_cap.reserve(cp);
  if (e == cudaSuccess) e = p->sh_pat_m.reserve(cp);
  return e;
}

// The structure checks rvsp_cuda_symbolic_checked folds into the symbolic
// pass: A always, B unless it is A.
struct PreCheck {
  int32_t a_cols, a_nnz, b_nnz;
  bool check_b;
};

rvsp_status_t symbolic_impl(rvsp_cuda_plan_t p, cudaStream_t s, int32_t a_rows,
                            int32_t b_rows, int32_t b_cols, const int32_t *a_row_ptr,
                            const int32_t *a_col_idx, const int32_t *b_row_ptr,
                            const int32_t *b_col_idx, int32_t *c_row_ptr,
                            int64_t *c_nnz_out, const PreCheck *chk);
cudaError_t symbolic_rest(rvsp_cuda_plan *p, cudaStream_t s, const Operands &op,
                          int32_t a_rows, int32_t b_cols, const int32_t *a_row_ptr,
                          int32_t *c_row_ptr, const int32_t *sym_off, bool merge_done);

}  // namespace

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
  return symbolic_impl(p, static_cast<cudaStream_t>(stream), a_rows, b_rows, b_cols,
                       a_row_ptr, a_col_idx, b_row_ptr, b_col_idx, c_row_ptr, c_nnz_out,
                       nullptr);
}

rvsp_status_t rvsp_cuda_symbolic_checked(rvsp_cuda_plan_t p, void *stream, int32_t a_rows,
                                         int32_t a_cols, int32_t a_nnz, int32_t b_rows,
                                         int32_t b_cols, int32_t b_nnz,
                                         const int32_t *a_row_ptr, const int32_t *a_col_idx,
                                         const int32_t *b_row_ptr, const int32_t *b_col_idx,
                                         int check_b, int32_t *c_row_ptr,
                                         int64_t *c_nnz_out) {
  if (!p || !a_row_ptr || !a_col_idx || !b_row_ptr || !b_col_idx || !c_row_ptr ||
      !c_nnz_out)
    return RVSP_ERROR_NULL_POINTER;
  if (a_rows <= 0 || b_rows <= 0 || b_cols <= 0 || a_cols < 0 || a_nnz < 0 || b_nnz < 0)
    return RVSP_ERROR_INVALID_ARGUMENT;
  // A's columns index B's rows: a column the check lets through is < a_cols
  // = b_rows, so every pass after the verdict reads B's row pointers in
  // bounds (the row statistics bound it by b_rows as well).
  if (a_cols != b_rows) return RVSP_ERROR_INVALID_ARGUMENT;
  const PreCheck chk{a_cols, a_nnz, b_nnz, check_b != 0};
  return symbolic_impl(p, static_cast<cudaStream_t>(stream), a_rows, b_rows, b_cols,
                       a_row_ptr, a_col_idx, b_row_ptr, b_col_idx, c_row_ptr, c_nnz_out,
                       &chk);
}

namespace {

rvsp_status_t symbolic_impl(rvsp_cuda_plan_t p, cudaStream_t s, int32_t a_rows,
                            int32_t b_rows, int32_t b_cols, const int32_t *a_row_ptr,
                            const int32_t *a_col_idx, const int32_t *b_row_ptr,
                            const int32_t *b_col_idx, int32_t *c_row_ptr,
                            int64_t *c_nnz_out, const PreCheck *chk) {
  p->analysed = 0;
  p->rmap_state = 0;
  p->rmap_col = nullptr;
  const size_t n = static_cast<size_t>(a_rows);

  cudaError_t e = p->ops.reserve(n);
  if (e == cudaSuccess) e = p->cls.reserve(n);
  if (e == cudaSuccess) e = p->counts.reserve(n);
  if (e == cudaSuccess) e = p->rows_sym.reserve(n);
  if (e == cudaSuccess) e = p->rows_num.reserve(n);
  if (e == cudaSuccess) e = p->long_rows.reserve(n);
  if (e == cudaSuccess) e = p->partials.reserve(scan_partials_bytes(a_rows) / sizeof(int64_t));
  if (e == cudaSuccess && merge_allowed(p->merge_policy, a_rows)) e = p->cls_spec.reserve(n);
  if (e == cudaSuccess && chk)
    e = p->check_long.reserve(1 + size_t(check_long_rows_cap(a_rows, chk->a_nnz)));
  if (e == cudaSuccess && chk && chk->check_b)
    e = p->check_long_b.reserve(1 + size_t(check_long_rows_cap(b_rows, chk->b_nnz)));
  if (e != cudaSuccess) return map_cuda(e);

  Operands op{a_rows, b_cols, a_row_ptr, a_col_idx, nullptr,
              b_row_ptr, b_col_idx, nullptr,
              merge_allowed(p->merge_policy, a_rows)};
  if (chk) {
    // Checks of A (and B) run first; the row statistics after them are
    // bounded (they read nothing outside A's entries and B's row pointers),
    // and one host round trip brings back both the checks' verdicts and the
    // class sizes.  Nothing that depends on the structure runs before it.
    op.a_nnz = chk->a_nnz;
    op.b_rows = b_rows;
    cudaMemsetAsync(p->check.p, 0xff, 2 * sizeof(unsigned long long), s);
    cudaMemsetAsync(p->check_long.p, 0, sizeof(int32_t), s);
    if (chk->check_b) cudaMemsetAsync(p->check_long_b.p, 0, sizeof(int32_t), s);
    PhaseScope ph(p, s, RVSP_PHASE_CHECK);
    launch_csr_check(a_rows, chk->a_cols, a_row_ptr, a_col_idx, chk->a_nnz, p->check.p,
                     p->check_long.p, s);
    ph.launches = 2;
    if (chk->check_b) {
      launch_csr_check(b_rows, b_cols, b_row_ptr, b_col_idx, chk->b_nnz, p->check.p + 1,
                       p->check_long_b.p, s);
      ph.launches += 2;
    }
  }
  int32_t *misc = p->misc.p;
  cudaMemsetAsync(misc, 0, kMiscWords * sizeof(int32_t), s);
  CheckGuard guard;
  if (chk) {
    guard.w = p->check.p;
    guard.n = chk->check_b ? 2 : 1;
  }
  p->shift_active = 0;
  p->shift_tables = 0;
  p->shift_members = 0;
  p->shift_npat = 0;
  bool shift = p->shift_enabled && shift_size_ok(p, a_rows) &&
               reserve_shift(p, a_rows, b_rows) == cudaSuccess;
  if (!shift) cudaGetLastError();
  {
    PhaseScope ph(p, s, RVSP_PHASE_ROWSTATS);
    launch_rowstats(op, p->ops.p, p->cls.p, p->counts.p, misc + kSymCount,
                    p->long_rows.p, misc + kLongCount, a_rows, s);
    launch_rowstats_long(op, p->long_rows.p, misc + kLongCount, p->ops.p, p->cls.p,
                         p->counts.p, misc + kSymCount, p->num_sms, s);
    ph.launches = 2;
    if (shift) {
      // Shift classes: the probe decides on the device and one small read
      // brings the decision to the host, so a matrix without them queues
      // none of the analysis's passes (each a full grid that would only
      // read the flag and return).  Member rows leave the symbolic classes
      // (census recounted).
      launch_shift_decide(op, p->sh_probe.p, shift_bar(p), p->sh_on.p, guard, s);
      e = cudaMemcpyAsync(p->h_misc, p->sh_on.p, sizeof(int32_t), cudaMemcpyDeviceToHost, s);
      if (e == cudaSuccess) e = cudaStreamSynchronize(s);
      if (e != cudaSuccess) return map_cuda(e);
      shift = p->h_misc[0] != 0;
      ph.launches += 2;
    }
    if (shift) {
      launch_shift_classes(p->sh_on.p, op, b_rows, p->ops.p, p->sh_bkey.p, p->sh_rkey.p,
                           p->sh_tkey.p, p->sh_trow.p, p->sh_tkey.cap, p->sh_bcls.p,
                           p->sh_rcls.p, s);
      launch_shift_patterns(p->sh_on.p, op, p->sh_rcls.p, p->sh_share.p, kPatMinShare,
                            p->ops.p, p->sh_pat_of.p, p->sh_pat_canon.p, p->sh_pat_cap.p,
                            p->sh_pat_m.p, misc + kShiftNpat, p->shift_cap_pat, p->st.pid.p,
                            p->cls.p, misc + kShiftMembers, misc + kSymCount, p->num_sms, s);
      ph.launches += 18;
    }
  }
  const int32_t *skip = shift ? p->st.pid.p : nullptr;
  // Merge-class rows need no host-side census: their symbolic pass (one
  // launch per merge class over all rows, each skipping the other classes)
  // and the scan are queued at once, behind the check verdict, so a product
  // whose rows are all merge rows takes one host round trip.  When other
  // classes turn up, their pass and the scan follow the census.  The early
  // scan writes its numeric classes to cls_spec: the census-driven pass
  // still needs the symbolic classes in cls.
  const bool spec = op.merge_ok;
  if (spec) {
    {
      PhaseScope ph(p, s, RVSP_PHASE_SYMBOLIC);
      launch_merge_symbolic_all(op, p->cls.p, a_rows, p->counts.p, guard, s);
      ph.launches = 3;
    }
    {
      PhaseScope ph(p, s, RVSP_PHASE_SCAN);
      if (shift)
        launch_shift_copy_counts(p->sh_on.p, a_rows, p->st.pid.p, p->sh_rcls.p, p->counts.p, s);
      launch_scan_and_class(a_rows, p->counts.p, p->ops.p, a_row_ptr, c_row_ptr,
                            p->partials.p, p->total.p, p->cls_spec.p, misc + kNumCount,
                            op.merge_ok, s, guard, skip);
      ph.launches = shift ? 4 : 3;
    }
    cudaMemcpyAsync(p->h_misc, misc, kMiscWords * sizeof(int32_t), cudaMemcpyDeviceToHost, s);
    cudaMemcpyAsync(p->h_total, p->total.p, sizeof(int64_t), cudaMemcpyDeviceToHost, s);
  } else {
    cudaMemcpyAsync(p->h_misc, misc, kMiscWords * sizeof(int32_t), cudaMemcpyDeviceToHost, s);
  }
  if (chk)
    cudaMemcpyAsync(p->h_check, p->check.p, 2 * sizeof(unsigned long long),
                    cudaMemcpyDeviceToHost, s);
  e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return map_cuda(e);
  if (chk && (p->h_check[0] != ~0ull || (chk->check_b && p->h_check[1] != ~0ull)))
    return RVSP_ERROR_INVALID_CSR;  // not canonical: nothing ran on it
  if (shift) {
    p->shift_members = p->h_misc[kShiftMembers];
    p->shift_npat = p->h_misc[kShiftNpat] < p->shift_cap_pat ? p->h_misc[kShiftNpat]
                                                              : p->shift_cap_pat;
    p->shift_active = p->shift_members > 0;
  }
  int32_t sym_off[kNumClasses];
  int32_t off = 0;
  bool rest = !spec;  // classes left for the census-driven pass
  for (int c = 0; c < kNumClasses; ++c) {
    p->sym_count[c] = p->h_misc[kSymCount + c];
    sym_off[c] = off;
    if (c != kEmpty_) off += p->sym_count[c];
    if (c != kEmpty_ && !is_merge_class(c) && p->sym_count[c] > 0) rest = true;
  }
  if (rest) {
    e = symbolic_rest(p, s, op, a_rows, b_cols, a_row_ptr, c_row_ptr, sym_off, spec);
    if (e != cudaSuccess) return map_cuda(e);
  } else {
    std::swap(p->cls, p->cls_spec);  // the early scan's numeric classes
  }
  if (p->h_misc[kStatus] != kDevOk) {
    cudaMemsetAsync(misc + kStatus, 0, sizeof(int32_t), s);
    return RVSP_ERROR_DEVICE;
  }
  const int64_t total = *p->h_total;
  if (total > INT32_MAX) return RVSP_ERROR_ALLOCATION_FAILED;

  finish_numeric_bins(p, a_rows, b_cols, s);
  e = cudaGetLastError();
  if (e != cudaSuccess) return map_cuda(e);

  p->learned = 0;
  p->a_rows = a_rows;
  p->b_rows = b_rows;
  p->b_cols = b_cols;
  p->c_nnz = total;
  p->analysed = 1;
  *c_nnz_out = total;
  return RVSP_SUCCESS;
}

// The symbolic pass of the rows the census found outside the merge classes
// (all rows when merge_done is false), then the scan again, and the host
// copy of the counters and the total (one more round trip).
cudaError_t symbolic_rest(rvsp_cuda_plan *p, cudaStream_t s, const Operands &op,
                          int32_t a_rows, int32_t b_cols, const int32_t *a_row_ptr,
                          int32_t *c_row_ptr, const int32_t *sym_off, bool merge_done) {
  int32_t *misc = p->misc.p;
  cudaError_t e = cudaSuccess;
  // Global bitmaps for dense symbolic rows when B is too wide for shared memory.
  const size_t bits_bytes = dense_slot_bits_bytes(b_cols);
  int32_t slots = 0;
  if (p->sym_count[kDense] > 0 && bits_bytes > 0) {
    slots = p->sym_count[kDense] < p->num_sms ? p->sym_count[kDense] : p->num_sms;
    const size_t words = bits_bytes / sizeof(uint32_t) * size_t(slots);
    if (words > p->sym_bits.cap) {
      e = p->sym_bits.reserve(words);
      if (e != cudaSuccess) return e;
      cudaMemsetAsync(p->sym_bits.p, 0, words * sizeof(uint32_t), s);
    }
    p->sym_bits_slots = slots;
  }
  {
    PhaseScope ph(p, s, RVSP_PHASE_SYMBOLIC);
    // W1024 / W2048 rows count optimistically in a small table first; their
    // retry lists live in long_rows (free once the row statistics are done),
    // W1024's from 0, W2048's after it.
    auto launch_class = [&](int c, const int32_t *rows, int32_t nrows) {
      if (symbolic_optimistic_class(c)) {
        const int32_t base = c == kW1024 ? 0 : p->sym_count[kW1024];
        launch_symbolic_optimistic(c, op, rows, nrows, p->counts.p, p->long_rows.p + base,
                                   misc + kRetryCount + (c == kW1024 ? 0 : 1),
                                   misc + kStatus, p->num_sms, s);
        return 2;
      }
      launch_symbolic_class(c, op, rows, nrows, p->counts.p, p->sym_bits.p, slots,
                            misc + kStatus, p->num_sms, s);
      return 1;
    };
    // whole >= 0 is never a merge class here when merge_done (a class
    // outside them is non-empty).
    const int whole = p->shift_active ? -1 : whole_matrix_class(p->sym_count, a_rows);
    if (whole >= 0) {
      ph.launches = launch_class(whole, nullptr, a_rows);
    } else {
      launch_class_offsets(misc + kSymCount, misc + kSymOff, s);
      launch_scatter_rows(a_rows, p->cls.p, misc + kSymOff, misc + kSymFill,
                          p->rows_sym.p, s);
      ph.launches = 2;
      for (int c = kEmpty_ + 1; c < kNumClasses; ++c) {
        if (p->sym_count[c] <= 0 || (merge_done && is_merge_class(c))) continue;
        ph.launches += launch_class(c, p->rows_sym.p + sym_off[c], p->sym_count[c]);
      }
    }
  }
  if (merge_done)  // the first scan counted numeric classes already
    cudaMemsetAsync(misc + kNumCount, 0, kNumClasses * sizeof(int32_t), s);
  {
    PhaseScope ph(p, s, RVSP_PHASE_SCAN);
    const int32_t *skip = nullptr;
    if (p->shift_active) {
      launch_shift_copy_counts(p->sh_on.p, a_rows, p->st.pid.p, p->sh_rcls.p, p->counts.p, s);
      skip = p->st.pid.p;
    }
    launch_scan_and_class(a_rows, p->counts.p, p->ops.p, a_row_ptr, c_row_ptr,
                          p->partials.p,
                          p->total.p, p->cls.p, misc + kNumCount, op.merge_ok, s,
                          CheckGuard(), skip);
    ph.launches = skip ? 4 : 3;
  }
  cudaMemcpyAsync(p->h_misc + kNumCount, misc + kNumCount,
                  (kMiscWords - kNumCount) * sizeof(int32_t), cudaMemcpyDeviceToHost, s);
  cudaMemcpyAsync(p->h_total, p->total.p, sizeof(int64_t), cudaMemcpyDeviceToHost, s);
  return cudaStreamSynchronize(s);
}

}  // namespace

rvsp_status_t rvsp_cuda_learned_symbolic(
    rvsp_cuda_plan_t p, rvsp_mlp_t model, void *stream, int32_t a_rows, int32_t b_rows,
    int32_t b_cols, const int32_t *a_row_ptr, const int32_t *a_col_idx,
    const float *a_values, int32_t a_nnz, const int32_t *b_row_ptr,
    const int32_t *b_col_idx, const float *b_values, int32_t b_nnz,
    float capacity_scale, int32_t *c_row_ptr, int64_t *c_nnz_out) {
  if (!p || !model || !a_row_ptr || !a_col_idx || !a_values || !b_row_ptr ||
      !b_col_idx || !b_values || !c_row_ptr || !c_nnz_out)
    return RVSP_ERROR_NULL_POINTER;
  if (a_rows <= 0 || b_rows <= 0 || b_cols <= 0 || a_nnz < 0 || b_nnz < 0 ||
      !(capacity_scale > 0.0f))
    return RVSP_ERROR_INVALID_ARGUMENT;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  p->analysed = 0;
  p->learned = 0;
  p->rmap_state = 0;
  p->rmap_col = nullptr;
  p->shift_active = 0;
  p->shift_tables = 0;
  p->shift_members = 0;
  if (p->shift_enabled && shift_size_ok(p, a_rows)) {
    // Rows that are translates of a few canonical rows need no prediction:
    // their structure comes from the canonical rows.  When the probe finds
    // them common, the analysis is the shift-class one (symbolic_impl).
    if (reserve_shift(p, a_rows, b_rows) == cudaSuccess) {
      const Operands pop{a_rows, b_cols, a_row_ptr, a_col_idx, nullptr,
                         b_row_ptr, b_col_idx, nullptr, false};
      launch_shift_decide(pop, p->sh_probe.p, shift_bar(p), p->sh_on.p, CheckGuard(), s);
      cudaError_t e = cudaMemcpyAsync(p->h_misc, p->sh_on.p, sizeof(int32_t),
                                      cudaMemcpyDeviceToHost, s);
      if (e == cudaSuccess) e = cudaStreamSynchronize(s);
      if (e != cudaSuccess) return map_cuda(e);
      if (p->h_misc[0])
        return symbolic_impl(p, s, a_rows, b_rows, b_cols, a_row_ptr, a_col_idx, b_row_ptr,
                             b_col_idx, c_row_ptr, c_nnz_out, nullptr);
    } else {
      cudaGetLastError();
    }
  }
  const size_t n = static_cast<size_t>(a_rows);
  cudaError_t e = p->ops.reserve(n);
  if (e == cudaSuccess) e = p->cls.reserve(n);
  if (e == cudaSuccess) e = p->counts.reserve(n);
  if (e == cudaSuccess) e = p->rows_sym.reserve(n);
  if (e == cudaSuccess) e = p->rows_num.reserve(n);
  if (e == cudaSuccess) e = p->cap.reserve(n);
  if (e == cudaSuccess) e = p->slab_off.reserve(n);
  if (e == cudaSuccess) e = p->ovf_rows.reserve(n);
  if (e == cudaSuccess) e = p->big_rows.reserve(n + 1);
  if (e == cudaSuccess) e = p->partials.reserve(scan_partials_bytes(a_rows) / sizeof(int64_t));
  if (e != cudaSuccess) return map_cuda(e);

  const Operands op{a_rows, b_cols, a_row_ptr, a_col_idx, a_values,
                    b_row_ptr, b_col_idx, b_values,
                    merge_allowed(p->merge_policy, a_rows)};
  int32_t *misc = p->misc.p;
  cudaMemsetAsync(misc, 0, kMiscWords * sizeof(int32_t), s);
  // 1. Predict every row's class and capacity; slab offsets = scan of capacities.
  {
    PhaseScope ph(p, s, RVSP_PHASE_PREDICT);
    const float b_mean = static_cast<float>(b_nnz) / static_cast<float>(b_rows);
    launch_learned_plan(op, b_mean, mlp_device_params(model), capacity_scale,
                        op.merge_ok, p->ops.p, p->cls.p, p->cap.p,
                        p->counts.p, misc + kSymCount, p->num_sms, s);
    launch_scan_i64(a_rows, p->cap.p, p->slab_off.p, p->partials.p, p->total.p, s);
    ph.launches = 4;
  }
  cudaMemcpyAsync(p->h_misc, misc, kNumClasses * sizeof(int32_t), cudaMemcpyDeviceToHost, s);
  cudaMemcpyAsync(p->h_total, p->total.p, sizeof(int64_t), cudaMemcpyDeviceToHost, s);
  e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return map_cuda(e);
  int32_t pred_off[kNumClasses];
  int32_t off = 0;
  for (int c = 0; c < kNumClasses; ++c) {
    p->sym_count[c] = p->h_misc[kSymCount + c];
    pred_off[c] = off;
    if (c != kEmpty_) off += p->sym_count[c];
  }
  p->slab_total = *p->h_total;
  e = p->slab_col.reserve(size_t(p->slab_total));
  if (e == cudaSuccess) e = p->slab_val.reserve(size_t(p->slab_total));
  if (e != cudaSuccess) return map_cuda(e);
  // Dense rows of the fused pass use a plan-owned dense workspace.
  int32_t fslots = 0;
  float *facc = nullptr;
  uint32_t *fbits = nullptr;
  if (p->sym_count[kDense] > 0) {
    fslots = p->sym_count[kDense] < p->num_sms ? p->sym_count[kDense] : p->num_sms;
    const size_t acc_b = dense_slot_acc_bytes(b_cols), bits_b = dense_slot_bits_bytes(b_cols);
    const size_t need = size_t(fslots) * (acc_b + bits_b);
    e = p->fused_ws.reserve(need);
    if (e != cudaSuccess) return map_cuda(e);
    cudaMemsetAsync(p->fused_ws.p, 0, need, s);
    facc = reinterpret_cast<float *>(p->fused_ws.p);
    fbits = reinterpret_cast<uint32_t *>(p->fused_ws.p + size_t(fslots) * acc_b);
  }

  // 2. The fused pass: every row into its slab slot, or onto the overflow list.
  const FusedOut fo{p->slab_off.p, p->cap.p, p->counts.p, p->ovf_rows.p,
                    misc + kLongCount};
  {
    PhaseScope ph(p, s, RVSP_PHASE_FUSED);
    const int whole = whole_matrix_class(p->sym_count, a_rows);
    if (whole < 0) {
      launch_class_offsets(misc + kSymCount, misc + kSymOff, s);
      launch_scatter_rows(a_rows, p->cls.p, misc + kSymOff, misc + kSymFill,
                          p->rows_sym.p, s);
      ph.launches = 2;
    }
    for (int c = kEmpty_ + 1; c < kNumClasses; ++c) {
      if (p->sym_count[c] <= 0) continue;
      const bool all = c == whole;
      launch_numeric_class(c, op, p->ops.p, all ? nullptr : p->rows_sym.p + pred_off[c],
                           all ? a_rows : p->sym_count[c], nullptr, p->slab_col.p,
                           p->slab_val.p, true, facc, fbits, fslots, misc + kStatus,
                           p->num_sms, s, &fo);
      ph.launches += 1;
    }
  }
  // 3. Optimistic scan (valid when nothing overflowed) and the fingerprint of
  //    the values the fused pass used.
  {
    PhaseScope ph(p, s, RVSP_PHASE_SCAN);
    launch_scan_and_class(a_rows, p->counts.p, p->ops.p, a_row_ptr, c_row_ptr,
                          p->partials.p, p->total.p, p->cls.p, misc + kNumCount,
                            op.merge_ok, s);
    ph.launches = 3;
  }
  values_fingerprint_launch(p, a_values, a_nnz, b_values, b_nnz, s);
  cudaMemcpyAsync(p->h_misc + kNumCount, misc + kNumCount,
                  (kMiscWords - kNumCount) * sizeof(int32_t), cudaMemcpyDeviceToHost, s);
  cudaMemcpyAsync(p->h_total, p->total.p, sizeof(int64_t), cudaMemcpyDeviceToHost, s);
  e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return map_cuda(e);
  if (p->h_misc[kStatus] != kDevOk) {
    cudaMemsetAsync(misc + kStatus, 0, sizeof(int32_t), s);
    return RVSP_ERROR_DEVICE;
  }
  p->est_hash = p->h_vhash[0];
  p->n_ovf = p->h_misc[kLongCount];

  // 4. Overflowed rows: the plain symbolic pass, then the scan again.
  if (p->n_ovf > 0) {
    e = p->ovf_cls.reserve(size_t(p->n_ovf));
    if (e == cudaSuccess) e = p->ovf_sorted.reserve(size_t(p->n_ovf));
    if (e != cudaSuccess) return map_cuda(e);
    cudaMemsetAsync(misc + kSymCount, 0, 3 * kNumClasses * sizeof(int32_t), s);
    launch_list_classify(p->ovf_rows.p, p->n_ovf, p->ops.p, a_row_ptr, p->counts.p, b_cols,
                         false, p->ovf_cls.p, misc + kSymCount, s);
    cudaMemcpyAsync(p->h_misc, misc, kNumClasses * sizeof(int32_t), cudaMemcpyDeviceToHost, s);
    e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return map_cuda(e);
    int32_t ocount[kNumClasses], ooff[kNumClasses];
    off = 0;
    for (int c = 0; c < kNumClasses; ++c) {
      ocount[c] = p->h_misc[kSymCount + c];
      ooff[c] = off;
      if (c != kEmpty_) off += ocount[c];
    }
    int32_t slots = 0;
    e = ensure_sym_bits(p, ocount[kDense], b_cols, s, &slots);
    if (e != cudaSuccess) return map_cuda(e);
    {
      PhaseScope ph(p, s, RVSP_PHASE_SYMBOLIC);
      launch_class_offsets(misc + kSymCount, misc + kSymOff, s);
      launch_scatter_list(p->ovf_rows.p, p->n_ovf, p->ovf_cls.p, misc + kSymOff,
                          misc + kSymFill, p->rows_sym.p, s);
      ph.launches = 3;
      for (int c = kEmpty_ + 1; c < kNumClasses; ++c) {
        if (ocount[c] <= 0) continue;
        launch_symbolic_class(c, op, p->rows_sym.p + ooff[c], ocount[c], p->counts.p,
                              p->sym_bits.p, slots, misc + kStatus, p->num_sms, s);
        ph.launches += 1;
      }
    }
    {
      PhaseScope ph(p, s, RVSP_PHASE_SCAN);
      cudaMemsetAsync(misc + kNumCount, 0, kNumClasses * sizeof(int32_t), s);
      launch_scan_and_class(a_rows, p->counts.p, p->ops.p, a_row_ptr, c_row_ptr,
                            p->partials.p, p->total.p, p->cls.p, misc + kNumCount,
                            op.merge_ok, s);
      // The overflow rows by numeric class, for the first compute.
      cudaMemsetAsync(misc + kSymCount, 0, 3 * kNumClasses * sizeof(int32_t), s);
      launch_list_classify(p->ovf_rows.p, p->n_ovf, p->ops.p, a_row_ptr, p->counts.p,
                           b_cols, true, p->ovf_cls.p, misc + kSymCount, s);
      launch_class_offsets(misc + kSymCount, misc + kSymOff, s);
      launch_scatter_list(p->ovf_rows.p, p->n_ovf, p->ovf_cls.p, misc + kSymOff,
                          misc + kSymFill, p->ovf_sorted.p, s);
      ph.launches = 6;
    }
    cudaMemcpyAsync(p->h_misc, misc, kMiscWords * sizeof(int32_t), cudaMemcpyDeviceToHost, s);
    cudaMemcpyAsync(p->h_total, p->total.p, sizeof(int64_t), cudaMemcpyDeviceToHost, s);
    e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return map_cuda(e);
    if (p->h_misc[kStatus] != kDevOk) {
      cudaMemsetAsync(misc + kStatus, 0, sizeof(int32_t), s);
      return RVSP_ERROR_DEVICE;
    }
    off = 0;
    for (int c = 0; c < kNumClasses; ++c) {
      p->ovf_num_count[c] = p->h_misc[kSymCount + c];
      p->ovf_num_off[c] = off;
      if (c != kEmpty_) off += p->ovf_num_count[c];
    }
  }
  const int64_t total = *p->h_total;
  if (total > INT32_MAX) return RVSP_ERROR_ALLOCATION_FAILED;
  finish_numeric_bins(p, a_rows, b_cols, s);
  e = cudaGetLastError();
  if (e != cudaSuccess) return map_cuda(e);
  p->learned = 1;
  p->a_nnz = a_nnz;
  p->b_nnz = b_nnz;
  p->a_rows = a_rows;
  p->b_rows = b_rows;
  p->b_cols = b_cols;
  p->c_nnz = total;
  p->analysed = 1;
  *c_nnz_out = total;
  return RVSP_SUCCESS;
}

rvsp_status_t rvsp_cuda_plan_set_merge_policy(rvsp_cuda_plan_t p, int32_t policy) {
  if (!p) return RVSP_ERROR_NULL_POINTER;
  if (policy < kMergeAuto || policy > kMergeAlways) return RVSP_ERROR_INVALID_ARGUMENT;
  p->merge_policy = policy;
  return RVSP_SUCCESS;
}

rvsp_status_t rvsp_cuda_plan_set_row_tiles(rvsp_cuda_plan_t p, int32_t enable) {
  if (!p) return RVSP_ERROR_NULL_POINTER;
  if (enable != 0 && enable != 1) return RVSP_ERROR_INVALID_ARGUMENT;
  if (enable && !p->tiles_enabled) {
    // tiles were never built for the current reuse map: build it again
    p->rmap_state = 0;
    p->rmap_col = nullptr;
  }
  p->tiles_enabled = enable;
  return RVSP_SUCCESS;
}

rvsp_status_t rvsp_cuda_plan_set_persistent(rvsp_cuda_plan_t p, int32_t merge_rows,
                                           int32_t blocks_per_sm) {
  if (!p) return RVSP_ERROR_NULL_POINTER;
  if (merge_rows < 0 || merge_rows > kPersistThreads || merge_rows % 32 != 0 ||
      blocks_per_sm < 1 || blocks_per_sm > 4)
    return RVSP_ERROR_INVALID_ARGUMENT;
  p->persist_merge_rows = merge_rows;
  p->persist_blocks = blocks_per_sm;
  return RVSP_SUCCESS;
}

rvsp_status_t rvsp_cuda_plan_set_pattern_kernels(rvsp_cuda_plan_t p, int32_t enable) {
  if (!p) return RVSP_ERROR_NULL_POINTER;
  if (enable != 0 && enable != 1) return RVSP_ERROR_INVALID_ARGUMENT;
  if (enable != p->pattern_kernels) {
    // the tiles are built with or without pattern kernels: rebuild them
    p->rmap_state = 0;
    p->rmap_col = nullptr;
    if (p->shift_tables == 1) p->shift_tables = 0;
  }
  p->pattern_kernels = enable;
  return RVSP_SUCCESS;
}

int32_t rvsp_cuda_plan_pattern_kernel_rows(rvsp_cuda_plan_t p) {
  if (!p || !p->tiles_enabled) return 0;
  int32_t n = 0;
  if (p->rmap_state == 1 && p->pat_ready && p->rt.ready)
    for (const auto &j : p->rt.jit) n += 32 * j.n;
  if (p->shift_active && p->shift_tables == 1 && p->st.ready)
    for (const auto &j : p->st.jit) n += 32 * j.n;
  return n;
}

void rvsp_cuda_pattern_kernel_stats(int32_t *compiles, double *compile_ms) {
  jit_stats(compiles, compile_ms);
}

rvsp_status_t rvsp_cuda_plan_set_shift_classes(rvsp_cuda_plan_t p, int32_t enable) {
  if (!p) return RVSP_ERROR_NULL_POINTER;
  if (enable < 0 || enable > 2) return RVSP_ERROR_INVALID_ARGUMENT;
  p->shift_enabled = enable;
  return RVSP_SUCCESS;
}

int32_t rvsp_cuda_plan_shift_rows(rvsp_cuda_plan_t p) {
  return (p && p->analysed && p->shift_active) ? p->shift_members : 0;
}

int32_t rvsp_cuda_plan_tiled_rows(rvsp_cuda_plan_t p) {
  if (!p || !p->tiles_enabled) return 0;
  int32_t n = 0;
  if (p->rmap_state == 1 && p->pat_ready && p->rt.ready) n += p->n_pat_rows - p->rt.n_lo;
  if (p->shift_active && p->shift_tables == 1 && p->st.ready)
    n += p->shift_members - p->st.n_lo;
  return n;
}

int32_t rvsp_cuda_plan_overflow_rows(rvsp_cuda_plan_t p) {
  return (p && p->analysed && p->learned) ? p->n_ovf : 0;
}

size_t rvsp_cuda_numeric_workspace_bytes(rvsp_cuda_plan_t p) {
  return (p && p->analysed) ? p->numeric_ws : 0;
}

namespace {

// The reuse map may take at most this much device memory (and a quarter of
// what is free).
constexpr size_t kReuseMapMaxBytes = size_t(24) << 30;

// The tile tables may take at most this much device memory.
constexpr size_t kTileTablesMaxBytes = size_t(256) << 20;
// Patterns with at least this many tiles (of 32 rows) get a compiled kernel,
// the kJitMaxPatterns largest of them, when their rows have at most
// kJitMaxOut outputs (one register each).
constexpr int32_t kJitMinTiles = 128;
constexpr int kJitMaxPatterns = 12;
constexpr int32_t kJitMaxOut = 160;
// Largest B range (floats) one stage buffer of a pattern kernel takes.
constexpr int32_t kJitMaxSpan = 4096;

// Compiled kernels for the patterns that cover the most tiles.  The tile
// list is read back once to count each pattern's tiles and list them in row
// order; then, for all the chosen patterns at once, the union spans of runs
// of their A nonzeros are measured on a sample of their tiles (one round
// trip with their tables), the staging groups chosen and the kernels
// compiled side by side (k_jit.cu), their tile records built (one round
// trip for the records' A extents and every group's largest B range), and
// their tiles marked so the table kernel skips them (one round trip for the
// table kernel's own list).  A pattern whose compile fails stays on the
// table kernel.  The device arrays of earlier builds are kept and reused;
// every transfer goes through page-locked staging.  Synchronizes `s`.
cudaError_t build_pattern_kernels(rvsp_cuda_plan *p, cudaStream_t s, const Operands &op,
                                  int32_t npat, TileBuild &tb) {
  for (auto &j : tb.jit) tb.pool.push_back(j);
  tb.jit.clear();
  // per chosen pattern: spans (32 x kJitMaxGroup words), its records' A
  // extent and groups' B ranges
  constexpr size_t W = size_t(32 * kJitMaxGroup) + 2;
  const size_t KM = size_t(kJitMaxPatterns);
  const int32_t stride = tile_tab_stride();
  const size_t nt = static_cast<size_t>(tb.n_tiles), np = static_cast<size_t>(npat);
  // the staging layout: tiles read back, desc, lens, tables, sorted tile
  // lists, words, groups (16-byte aligned pieces)
  auto up16 = [](size_t x) { return (x + 15) & ~size_t(15); };
  const size_t o_tiles = 0, o_desc = o_tiles + up16(nt * sizeof(int4));
  const size_t o_lens = o_desc + up16(np * sizeof(int4));
  const size_t o_tabs = o_lens + up16(np * 32 * sizeof(uint16_t));
  const size_t o_lists = o_tabs + up16(KM * size_t(stride) * sizeof(uint16_t));
  const size_t o_words = o_lists + up16(nt * sizeof(int4));
  const size_t o_groups = o_words + up16(KM * W * sizeof(int32_t));
  const size_t total = o_groups + up16(KM * 32 * sizeof(int2));
  if (tb.staging.reserve(total) != cudaSuccess) {
    cudaGetLastError();
    return cudaSuccess;
  }
  int4 *const tiles = reinterpret_cast<int4 *>(tb.staging.p + o_tiles);
  int4 *const desc = reinterpret_cast<int4 *>(tb.staging.p + o_desc);
  uint16_t *const lens = reinterpret_cast<uint16_t *>(tb.staging.p + o_lens);
  uint16_t *const tabs = reinterpret_cast<uint16_t *>(tb.staging.p + o_tabs);
  int4 *const lists = reinterpret_cast<int4 *>(tb.staging.p + o_lists);
  int32_t *const words = reinterpret_cast<int32_t *>(tb.staging.p + o_words);
  int2 *const gh = reinterpret_cast<int2 *>(tb.staging.p + o_groups);
  cudaError_t e = cudaMemcpyAsync(tiles, tb.tiles.p, nt * sizeof(int4), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(desc, tb.desc.p, np * sizeof(int4), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(lens, tb.lens.p, np * 32 * sizeof(uint16_t), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return e;
  std::vector<int32_t> count(np, 0);
  for (size_t i = 0; i < nt; ++i)
    if (tiles[i].z >= 0 && tiles[i].z < npat) ++count[size_t(tiles[i].z)];
  std::vector<int32_t> order;
  for (int32_t id = 0; id < npat; ++id)
    if (count[size_t(id)] >= kJitMinTiles) order.push_back(id);
  std::sort(order.begin(), order.end(),
            [&](int32_t a, int32_t b) { return count[size_t(a)] > count[size_t(b)]; });
  if (order.size() > KM) order.resize(KM);
  if (order.empty()) return cudaSuccess;
  const size_t K = order.size();
  if (tb.jwords.reserve(K * W) != cudaSuccess || tb.jgroups.reserve(K * 32) != cudaSuccess) {
    cudaGetLastError();
    return cudaSuccess;
  }
  std::vector<JitPattern> cand(K);
  auto give_back = [&tb](JitPattern &jp) { tb.pool.push_back(jp); jp = JitPattern(); };
  // each chosen pattern's tiles in order of their first row (one tile per
  // chunk of 32 rows: a counting pass over the chunks), so that the
  // persistent warps, which take tiles in list order, work on neighbouring
  // rows at any one time and their B ranges stay in L2 between tiles
  std::vector<int32_t> kof(np, -1);
  for (size_t k = 0; k < K; ++k) kof[size_t(order[k])] = static_cast<int32_t>(k);
  std::vector<size_t> lbeg(K + 1, 0), lfill(K, 0);
  for (size_t k = 0; k < K; ++k) lbeg[k + 1] = lbeg[k] + size_t(count[size_t(order[k])]);
  {
    const int64_t nchunks = (int64_t(p->a_rows) + 31) / 32;
    std::vector<int32_t> at(static_cast<size_t>(nchunks), -1);
    for (size_t i = 0; i < nt; ++i) {
      const int64_t c = int64_t(tiles[i].x) / 32;
      if (c >= 0 && c < nchunks) at[size_t(c)] = static_cast<int32_t>(i);
    }
    for (const int32_t i : at) {
      if (i < 0) continue;
      const int4 &t = tiles[size_t(i)];
      if (t.z < 0 || t.z >= npat || kof[size_t(t.z)] < 0) continue;
      const size_t k = size_t(kof[size_t(t.z)]);
      lists[lbeg[k] + lfill[k]++] = t;
    }
  }
  for (size_t k = 0; k < K && e == cudaSuccess; ++k)
    e = cudaMemcpyAsync(tabs + k * size_t(stride), tb.tab.p + size_t(order[k]) * stride,
                        size_t(stride) * sizeof(uint16_t), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaMemsetAsync(tb.jwords.p, 0, K * W * sizeof(int32_t), s);
  // the patterns' span and record kernels are small and bound by latency:
  // they run side by side on the plan's side streams
  Lanes ln(p, s, true);
  for (size_t k = 0; k < K && e == cudaSuccess; ++k) {
    const int32_t id = order[k];
    JitPattern &jp = cand[k];
    // the device arrays of an earlier build: the smallest whose tile
    // capacity holds this pattern's tiles, else the largest (so that a
    // repeated analysis of the same structure allocates nothing)
    if (!tb.pool.empty()) {
      const size_t need = lfill[k];
      size_t best = 0;
      for (size_t q = 1; q < tb.pool.size(); ++q) {
        const size_t c = tb.pool[q].tiles.cap, bc = tb.pool[best].tiles.cap;
        const bool f = c >= need, bf = bc >= need;
        if ((f && (!bf || c < bc)) || (!f && !bf && c > bc)) best = q;
      }
      jp = tb.pool[best];
      tb.pool.erase(tb.pool.begin() + static_cast<std::ptrdiff_t>(best));
    }
    jp.n = static_cast<int32_t>(lfill[k]);
    if (jp.n <= 0 || jp.tiles.reserve(size_t(jp.n)) != cudaSuccess) {
      cudaGetLastError();
      give_back(jp);
      continue;
    }
    const cudaStream_t ks = k == 0 ? ln.main() : ln.next();
    e = cudaMemcpyAsync(jp.tiles.p, lists + lbeg[k], lfill[k] * sizeof(int4),
                        cudaMemcpyHostToDevice, ks);
    if (e != cudaSuccess) break;
    launch_jit_spans(jp.tiles.p, jp.n, tb.desc.p + id, tb.lens.p + size_t(id) * 32, op.a_rp,
                     op.a_col, op.b_rp, tb.jwords.p + k * W, p->num_sms, ks);
  }
  ln.join();
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(words, tb.jwords.p, K * W * sizeof(int32_t), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) {
    for (auto &c : cand) give_back(c);
    return e;
  }
  // requests for the patterns that can have a kernel
  std::vector<JitRequest> reqs(K);
  for (size_t k = 0; k < K; ++k) {
    JitPattern &jp = cand[k];
    const int4 d = desc[size_t(order[k])];
    if (!jp.tiles.p || d.x <= 0 || d.x > 32 || d.y <= 0 || d.y > kJitMaxOut) {
      give_back(jp);
      continue;
    }
    JitRequest &rq = reqs[k];
    rq.na = d.x;
    rq.m = d.y;
    const uint16_t *tab = tabs + k * size_t(stride);
    int32_t off = 0;
    for (int j = 0; j < d.x; ++j) {
      rq.len[j] = lens[size_t(order[k]) * 32 + j];
      for (int ee = 0; ee < rq.len[j]; ++ee) rq.slot.push_back(tab[size_t(off + ee)] & 0x7fff);
      off += (rq.len[j] + 7) & ~7;
    }
    int32_t need = 0;
    rq.groups = jit_groups(d.x, rq.len, words + k * W, kJitMaxSpan, &need);
    if (rq.groups.empty() || need <= 0 || need > kJitMaxSpan) {
      rq = JitRequest();
      give_back(jp);
      continue;
    }
    jp.m = d.y;
  }
  jit_pattern_kernels(reqs);
  // tile records of the compiled patterns (their maxima: the records' A
  // extent, then each group's largest B range over every tile)
  cudaMemsetAsync(tb.jwords.p, 0, K * W * sizeof(int32_t), s);
  std::vector<int32_t> rws(K, 0);
  Lanes lr(p, s, true);
  for (size_t k = 0; k < K; ++k) {
    JitPattern &jp = cand[k];
    const JitRequest &rq = reqs[k];
    if (!jp.tiles.p) continue;
    if (!rq.kernel) {
      give_back(jp);
      continue;
    }
    rws[k] = jit_record_words(rq.na, static_cast<int>(rq.groups.size()));
    if (jp.prog.reserve(size_t(jp.n) * size_t(rws[k])) != cudaSuccess ||
        jp.arange.reserve(size_t(jp.n)) != cudaSuccess || jp.head.reserve(1) != cudaSuccess) {
      cudaGetLastError();
      give_back(jp);
      continue;
    }
    for (size_t g = 0; g < rq.groups.size(); ++g)
      gh[k * 32 + g] = make_int2(rq.groups[g].first, rq.groups[g].second);
    const cudaStream_t ks = k == 0 ? lr.main() : lr.next();
    cudaMemcpyAsync(tb.jgroups.p + k * 32, gh + k * 32, rq.groups.size() * sizeof(int2),
                    cudaMemcpyHostToDevice, ks);
    launch_jit_programs(jp.tiles.p, jp.n, rq.na, rq.groups, tb.jgroups.p + k * 32,
                        tb.lens.p + size_t(order[k]) * 32, op.a_rp, op.a_col, op.b_rp,
                        jp.prog.p, jp.arange.p, tb.jwords.p + k * W, p->num_sms, ks);
  }
  lr.join();
  e = cudaMemcpyAsync(words, tb.jwords.p, K * W * sizeof(int32_t), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) {
    for (auto &c : cand) if (c.tiles.p) give_back(c);
    return e;
  }
  int dev_max = 0;
  cudaDeviceGetAttribute(&dev_max, cudaDevAttrMaxSharedMemoryPerBlockOptin, p->device);
  for (size_t k = 0; k < K; ++k) {
    JitPattern &jp = cand[k];
    if (!jp.tiles.p) continue;
    // the largest B range any tile's group reads (the sample only chose
    // the groups); past kJitMaxSpan the uint16 offsets would not hold
    int32_t need = 0;
    for (size_t g = 0; g < reqs[k].groups.size(); ++g)
      need = std::max(need, words[k * W + 1 + g]);
    if (need <= 0 || need > kJitMaxSpan) {
      give_back(jp);
      continue;
    }
    jit_layout(rws[k], words[k * W], need, jp.m, &jp.stage_cap, &jp.abuf_floats,
               &jp.work_floats);
    // two warps must fit one block's shared memory
    if (size_t(2) * size_t(jp.work_floats) * sizeof(float) > size_t(dev_max)) {
      give_back(jp);
      continue;
    }
    jp.grid = jit_grid(reqs[k].kernel, jp.n, jp.work_floats, jp.m, p->num_sms);
    jp.kernel = reqs[k].kernel;
    launch_mark_pattern(tb.desc.p, order[k], s);
    tb.jit.push_back(jp);
  }
  // the table kernel's own list: the tiles of the patterns left to it
  if (!tb.jit.empty() && tb.table.reserve(size_t(tb.n_tiles)) == cudaSuccess) {
    cudaMemsetAsync(tb.counts.p + 6, 0, sizeof(int32_t), s);
    launch_table_tiles(tb.tiles.p, tb.n_tiles, tb.desc.p, tb.table.p, tb.counts.p + 6, s);
    e = cudaMemcpyAsync(words, tb.counts.p + 6, sizeof(int32_t), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return e;
    tb.n_table = words[0];
  } else {
    cudaGetLastError();
  }
  return cudaGetLastError();
}
constexpr int kTileCountWords = 8;  // ntiles, leftovers, 3 maxima, list count, spare

// Row tiles of a set of table patterns (k_tile.cu): the per-pattern tile
// tables (from each pattern's canonical row map: moff[row], map), then tiles
// over chunks of 32 consecutive rows of tb.pid (the pattern of each row, -1
// elsewhere, filled by the caller) and the leftover list.  Leaves tb.ready 0
// (every pattern row on the warp-per-row kernel) when nothing is tiled.
// With `required` (the shift classes, whose rows have no other path) a
// failed allocation is an error, and the list of every pattern row is built
// too.  Synchronizes `s`.
cudaError_t build_row_tiles(rvsp_cuda_plan *p, cudaStream_t s, const Operands &op,
                            const int32_t *c_rp, int32_t npat, const int32_t *pat_canon,
                            const int32_t *psteps, const int64_t *moff, const uint16_t *map,
                            TileBuild &tb, bool required = false) {
  tb.ready = 0;
  tb.n_lo = 0;
  const size_t n = static_cast<size_t>(p->a_rows);
  const size_t tab_entries = size_t(npat) * size_t(tile_tab_stride());
  if (tb.tab.reserve(tab_entries) != cudaSuccess ||
      tb.lens.reserve(size_t(npat) * 32) != cudaSuccess ||
      tb.desc.reserve(size_t(npat)) != cudaSuccess ||
      tb.tiles.reserve((n + 31) / 32) != cudaSuccess ||
      tb.lo_rows.reserve(n) != cudaSuccess || tb.lo_ids.reserve(n) != cudaSuccess ||
      tb.counts.reserve(kTileCountWords) != cudaSuccess ||
      (required && (tb.all_rows.reserve(n) != cudaSuccess ||
                    tb.all_ids.reserve(n) != cudaSuccess))) {
    const cudaError_t err = cudaGetLastError();
    return required ? err : cudaSuccess;
  }
  int32_t b_nnz = 0;
  cudaError_t e = cudaMemcpyAsync(&b_nnz, op.b_rp + p->b_rows, sizeof(int32_t),
                                  cudaMemcpyDeviceToHost, s);
  if (e != cudaSuccess) return e;
  cudaMemsetAsync(tb.counts.p, 0, kTileCountWords * sizeof(int32_t), s);
  if (required)
    launch_tile_list(p->a_rows, tb.pid.p, tb.all_rows.p, tb.all_ids.p, tb.counts.p + 5, s);
  launch_tile_tab(npat, pat_canon, psteps, op.a_rp, op.a_col, op.b_rp, c_rp, moff, map,
                  tb.tab.p, tb.lens.p, tb.desc.p, s);
  launch_tile_build(p->a_rows, tb.pid.p, tb.desc.p, tb.lens.p, op.a_rp, op.a_col, op.b_rp,
                    c_rp, tb.tiles.p, tb.counts.p, tb.lo_rows.p, tb.lo_ids.p,
                    tb.counts.p + 1, tb.counts.p + 2, s);
  int32_t h[kTileCountWords] = {};
  e = cudaMemcpyAsync(h, tb.counts.p, sizeof(h), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return e;
  tb.n_lo = h[1];
  if (h[0] <= 0) return cudaSuccess;
  int32_t acc_rows = 0, work = 0, stage_cap = 0;
  const size_t per_warp = tile_smem_per_warp(h[2], h[3], h[4], &acc_rows, &work, &stage_cap);
  int dev_max = 0;
  cudaDeviceGetAttribute(&dev_max, cudaDevAttrMaxSharedMemoryPerBlockOptin, p->device);
  // (cannot happen: the tile limits keep one block under 140 KB)
  if (per_warp * kTileKernelWarps > size_t(dev_max))
    return required ? cudaErrorInvalidValue : cudaSuccess;
  tb.n_tiles = h[0];
  tb.stage = h[2];
  tb.aseg = h[3];
  tb.max_out = h[4];
  tb.b_nnz = b_nnz;
  tb.ready = 1;
  if (p->pattern_kernels) return build_pattern_kernels(p, s, op, npat, tb);
  return cudaSuccess;
}

// Builds the reuse map of the W<T> rows for the structure in c_col (written
// by an earlier fill).  Leaves rmap_state -1 when the map does not apply:
// no W rows, a row of more than INT32_MAX / 2 products, or over the memory
// budget.  Synchronizes s.
// Term tables for the maps that many rows share (k_pattern.cu), and the
// split of the W rows into table rows and map rows.  Leaves pat_ready 0 (all
// W rows on the map) when no map is shared widely enough or the tables would
// take more than an eighth of the map's bytes.  Synchronizes `s`.
cudaError_t build_term_tables(rvsp_cuda_plan *p, cudaStream_t s, const Operands &op,
                              const int32_t *c_rp, int64_t map_entries) {
  const size_t n = static_cast<size_t>(p->a_rows);
  cudaError_t e = p->pat_of.reserve(n);
  if (e == cudaSuccess) e = p->pat_canon.reserve(n);
  if (e == cudaSuccess) e = p->pat_cap.reserve(n);
  if (e == cudaSuccess) e = p->pat_counts.reserve(kPatCountWords);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return cudaSuccess;
  }
  cudaMemsetAsync(p->pat_of.p, 0xff, n * sizeof(int32_t), s);
  cudaMemsetAsync(p->pat_counts.p, 0, kPatCountWords * sizeof(int32_t), s);
  for (int c = kEmpty_ + 1; c < kNumClasses; ++c) {
    if (!map_class(c) || p->num_count[c] <= 0) continue;
    const bool whole = c == p->num_whole;
    launch_pat_select(whole ? nullptr : p->rows_num.p + p->num_off[c],
                      whole ? p->a_rows : p->num_count[c], p->rmap_canon.p,
                      p->rmap_share_count.p, kPatMinShare, op.a_rp, c_rp, p->rmap_ops.p,
                      p->pat_of.p, p->pat_canon.p, p->pat_cap.p, p->pat_counts.p,
                      p->pat_counts.p + 2 + kNumClasses, s);
  }
  int32_t npat = 0;
  e = cudaMemcpyAsync(&npat, p->pat_counts.p, sizeof(int32_t), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return e;
  if (npat <= 0) return cudaSuccess;
  e = p->pat_off.reserve(size_t(npat));
  if (e == cudaSuccess) e = p->pat_steps.reserve(size_t(npat));
  if (e != cudaSuccess) {
    cudaGetLastError();
    return cudaSuccess;
  }
  launch_scan_i64(npat, p->pat_cap.p, p->pat_off.p, p->partials.p, p->total.p, s);
  int64_t records = 0;
  e = cudaMemcpyAsync(&records, p->total.p, sizeof(int64_t), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return e;
  const int64_t budget = map_entries * int64_t(sizeof(uint16_t)) / 8;
  if (records <= 0 || records * int64_t(sizeof(uint32_t)) > budget) return cudaSuccess;
  if (p->pat_rec.reserve(size_t(records)) != cudaSuccess ||
      p->pat_rows.reserve(n) != cudaSuccess || p->pat_ids.reserve(n) != cudaSuccess ||
      p->res_rows.reserve(n) != cudaSuccess) {
    cudaGetLastError();
    return cudaSuccess;
  }
  launch_pat_build(npat, p->pat_canon.p, op.a_rp, op.a_col, op.b_rp, c_rp, p->rmap_off.p,
                   p->rmap.p, p->pat_off.p, p->pat_cap.p, p->pat_rec.p, p->pat_steps.p, s);
  // per-row pattern ids for the row tiles (skipped when they do not fit)
  const size_t tab_entries = size_t(npat) * size_t(tile_tab_stride());
  const bool tiles_fit = p->tiles_enabled &&
                         tab_entries * sizeof(uint16_t) <= kTileTablesMaxBytes &&
                         p->rt.pid.reserve(n) == cudaSuccess;
  if (!tiles_fit) cudaGetLastError();
  if (tiles_fit) cudaMemsetAsync(p->rt.pid.p, 0xff, n * sizeof(int32_t), s);
  int32_t off = 0;
  for (int c = kEmpty_ + 1; c < kNumClasses; ++c) {
    p->res_off[c] = off;
    if (!map_class(c) || p->num_count[c] <= 0) continue;
    const bool whole = c == p->num_whole;
    launch_pat_split(whole ? nullptr : p->rows_num.p + p->num_off[c],
                     whole ? p->a_rows : p->num_count[c], p->rmap_canon.p, p->pat_of.p,
                     p->pat_steps.p, op.a_rp, op.a_col, op.b_rp, p->pat_rows.p,
                     p->pat_ids.p, p->pat_counts.p + 1, p->res_rows.p + off,
                     p->pat_counts.p + 2 + c, tiles_fit ? p->rt.pid.p : nullptr, s);
    off += whole ? p->a_rows : p->num_count[c];
  }
  int32_t h[kPatCountWords] = {};
  e = cudaMemcpyAsync(h, p->pat_counts.p, sizeof(h), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return e;
  p->n_pat = npat;
  p->n_pat_rows = h[1];
  for (int c = 0; c < kNumClasses; ++c) p->res_count[c] = h[2 + c];
  p->pat_max_ops = h[2 + kNumClasses];
  p->pat_max_out = h[3 + kNumClasses];
  p->pat_ready = 1;
  p->rt.ready = 0;
  if (tiles_fit && p->n_pat_rows > 0) {
    e = build_row_tiles(p, s, op, c_rp, npat, p->pat_canon.p, p->pat_steps.p, p->rmap_off.p,
                        p->rmap.p, p->rt);
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

// Term tables and row tiles of the shift-class patterns, from the canonical
// rows' structure in C (c_rp, c_col): their maps (binary search in C's row),
// the warp-per-row tables (k_pattern.cu) and the row tiles of the member
// rows (k_tile.cu).  Every member row is then in a tile or on the leftover
// list.  Synchronizes `s`.
cudaError_t build_shift_tables(rvsp_cuda_plan *p, cudaStream_t s, const Operands &op,
                               const int32_t *c_rp, const int32_t *c_col) {
  p->shift_tables = -1;
  const int32_t npat = p->shift_npat;
  if (npat <= 0) return cudaErrorInvalidValue;
  const size_t n = static_cast<size_t>(p->a_rows);
  cudaError_t e = p->sh_moff.reserve(n);
  if (e == cudaSuccess) e = p->sh_map.reserve(size_t(npat) * size_t(shift_max_ops()));
  if (e == cudaSuccess) e = p->sh_pat_off.reserve(size_t(npat));
  if (e == cudaSuccess) e = p->sh_steps.reserve(size_t(npat));
  if (e == cudaSuccess) e = p->sh_counts.reserve(4);
  if (e != cudaSuccess) return e;
  launch_shift_canon_map(npat, p->sh_pat_canon.p, op, c_rp, c_col, p->sh_moff.p, p->sh_map.p,
                         s);
  launch_scan_i64(npat, p->sh_pat_cap.p, p->sh_pat_off.p, p->partials.p, p->total.p, s);
  cudaMemsetAsync(p->sh_counts.p, 0, 4 * sizeof(int32_t), s);
  launch_pat_maxima(npat, p->sh_pat_canon.p, p->sh_pat_m.p, p->ops.p, p->sh_counts.p, s);
  int64_t records = 0;
  int32_t maxima[4] = {};
  e = cudaMemcpyAsync(&records, p->total.p, sizeof(int64_t), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(maxima, p->sh_counts.p, sizeof(maxima), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return e;
  e = p->sh_rec.reserve(size_t(records > 0 ? records : 1));
  if (e != cudaSuccess) return e;
  launch_pat_build(npat, p->sh_pat_canon.p, op.a_rp, op.a_col, op.b_rp, c_rp, p->sh_moff.p,
                   p->sh_map.p, p->sh_pat_off.p, p->sh_pat_cap.p, p->sh_rec.p, p->sh_steps.p,
                   s);
  p->sh_max_ops = maxima[0];
  p->sh_max_out = maxima[1];
  e = build_row_tiles(p, s, op, c_rp, npat, p->sh_pat_canon.p, p->sh_steps.p, p->sh_moff.p,
                      p->sh_map.p, p->st, true);
  if (e != cudaSuccess) return e;
  p->shift_tables = 1;
  return cudaSuccess;
}

// The table kernel over the tiles of the patterns without a compiled
// kernel (every tile when none is compiled); returns the launches.
int launch_table_tile_kernel(const TileBuild &tb, const Operands &op, const int32_t *c_rp,
                             float *c_val, cudaStream_t s) {
  const bool own = !tb.jit.empty() && tb.table.p;
  const int32_t n = own ? tb.n_table : tb.n_tiles;
  if (n <= 0) return 0;
  launch_tile_numeric(op, tb.b_nnz, own ? tb.table.p : tb.tiles.p, n, tb.desc.p, tb.lens.p,
                      tb.tab.p, c_rp, c_val, tb.stage, tb.aseg, tb.max_out, s);
  return 1;
}

// Pattern kernels of a tile set (k_jit.cu); returns the launches.  The
// first (the pattern with the most tiles, persistent over every SM) goes to
// the caller's stream, the others to the side streams in turn.  The caller
// launches the others (main = false) with its other small launches before
// the first (main = true), so that they reach the SMs before the persistent
// kernel fills them.
int launch_pattern_kernels(const TileBuild &tb, const Operands &op, const int32_t *c_rp,
                           float *c_val, int32_t *status, Lanes &ln, bool main) {
  int launches = 0;
  for (size_t i = main ? 0 : 1; i < (main ? std::min<size_t>(1, tb.jit.size()) : tb.jit.size());
       ++i) {
    const auto &j = tb.jit[i];
    launch_pattern_kernel(j.kernel, op, j.prog.p, j.arange.p, j.n, c_rp, c_val, j.stage_cap,
                          j.abuf_floats, j.work_floats, j.grid, j.head.p, status,
                          i == 0 ? ln.main() : ln.next());
    ++launches;
  }
  return launches;
}

// Values of the shift-class member rows (tables built): row tiles, then the
// members no tile took through the warp-per-row table kernel; every member
// through that kernel when tiles are off.
int launch_shift_numeric(rvsp_cuda_plan *p, Lanes &ln, const Operands &op,
                         const int32_t *c_rp, float *c_val) {
  int launches = 0;
  if (p->st.ready && p->tiles_enabled) {
    launches += launch_table_tile_kernel(p->st, op, c_rp, c_val, ln.next());
    if (p->st.n_lo > 0) {
      launch_pat_numeric(op, p->ops.p, p->st.lo_rows.p, p->st.lo_ids.p, p->st.n_lo, c_rp,
                         c_val, p->sh_pat_off.p, p->sh_steps.p, p->sh_rec.p, p->sh_max_ops,
                         p->sh_max_out, ln.next());
      ++launches;
    }
    launches += launch_pattern_kernels(p->st, op, c_rp, c_val, p->misc.p + kStatus, ln, false);
    launches += launch_pattern_kernels(p->st, op, c_rp, c_val, p->misc.p + kStatus, ln, true);
  } else {
    launch_pat_numeric(op, p->ops.p, p->st.all_rows.p, p->st.all_ids.p, p->shift_members,
                       c_rp, c_val, p->sh_pat_off.p, p->sh_steps.p, p->sh_rec.p,
                       p->sh_max_ops, p->sh_max_out, ln.main());
    ++launches;
  }
  return launches;
}

cudaError_t build_reuse_map(rvsp_cuda_plan *p, cudaStream_t s, const Operands &op,
                            const int32_t *c_rp, const int32_t *c_col) {
  p->rmap_state = -1;
  p->rmap_col = nullptr;
  bool any = false;
  for (int c = kEmpty_ + 1; c < kNumClasses; ++c)
    any = any || (map_class(c) && p->num_count[c] > 0);
  if (!any) return cudaSuccess;
  const size_t n = static_cast<size_t>(p->a_rows);
  cudaError_t e = p->rmap_ops.reserve(n + 1);
  if (e == cudaSuccess) e = p->rmap_off.reserve(n);
  if (e != cudaSuccess) return e;
  cudaMemsetAsync(p->rmap_ops.p, 0, (n + 1) * sizeof(int32_t), s);
  for (int c = kEmpty_ + 1; c < kNumClasses; ++c) {
    if (!map_class(c) || p->num_count[c] <= 0) continue;
    const bool whole = c == p->num_whole;
    launch_map_ops(whole ? nullptr : p->rows_num.p + p->num_off[c],
                   whole ? p->a_rows : p->num_count[c], p->ops.p, p->rmap_ops.p,
                   p->rmap_ops.p + n, s);
  }
  launch_scan_i64(p->a_rows, p->rmap_ops.p, p->rmap_off.p, p->partials.p, p->total.p, s);
  int32_t too_long = 0;
  int64_t entries = 0;
  e = cudaMemcpyAsync(&entries, p->total.p, sizeof(int64_t), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(&too_long, p->rmap_ops.p + n, sizeof(int32_t), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return e;
  const size_t bytes = static_cast<size_t>(entries) * sizeof(uint16_t);
  if (too_long || entries <= 0 || bytes > kReuseMapMaxBytes) return cudaSuccess;
  // the free-memory bound only matters when the map must grow (a repeated
  // analysis of the same structure reuses its allocation without asking
  // the driver)
  if (static_cast<size_t>(entries) > p->rmap.cap) {
    size_t free_b = 0, total_b = 0;
    if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) return cudaGetLastError();
    if (bytes > free_b / 4) return cudaSuccess;
  }
  if (p->rmap.reserve(static_cast<size_t>(entries)) != cudaSuccess) {
    cudaGetLastError();  // out of memory: keep the hash path
    return cudaSuccess;
  }
  // Fingerprints for sharing identical maps (skipped when the table does not
  // fit: every row then keeps its own map).
  int64_t map_rows = 0;
  for (int c = kEmpty_ + 1; c < kNumClasses; ++c)
    if (map_class(c) && p->num_count[c] > 0) map_rows += p->num_count[c];
  size_t tcap = 64;
  while (tcap < size_t(2 * map_rows)) tcap <<= 1;
  bool dedup = p->rmap_key.reserve(n) == cudaSuccess &&
               p->rmap_tkey.reserve(tcap) == cudaSuccess &&
               p->rmap_trow.reserve(tcap) == cudaSuccess &&
               p->rmap_shared.reserve(1) == cudaSuccess &&
               p->rmap_canon.reserve(n) == cudaSuccess &&
               p->rmap_share_count.reserve(n) == cudaSuccess;
  if (!dedup) {
    cudaGetLastError();
    if (p->rmap_shared.p) cudaMemsetAsync(p->rmap_shared.p, 0, sizeof(int32_t), s);
  }
  for (int c = kEmpty_ + 1; c < kNumClasses; ++c) {
    if (!map_class(c) || p->num_count[c] <= 0) continue;
    const bool whole = c == p->num_whole;
    launch_map_build(c, op, whole ? nullptr : p->rows_num.p + p->num_off[c],
                     whole ? p->a_rows : p->num_count[c], c_rp, c_col, p->rmap_off.p,
                     p->rmap.p, dedup ? p->rmap_key.p : nullptr, p->misc.p + kStatus, s);
  }
  if (dedup) {
    const unsigned long long mask = tcap - 1;
    cudaMemsetAsync(p->rmap_tkey.p, 0, tcap * sizeof(unsigned long long), s);
    cudaMemsetAsync(p->rmap_trow.p, 0x7f, tcap * sizeof(int32_t), s);
    cudaMemsetAsync(p->rmap_shared.p, 0, sizeof(int32_t), s);
    cudaMemsetAsync(p->rmap_share_count.p, 0, n * sizeof(int32_t), s);
    for (int pass = 0; pass < 2; ++pass) {
      for (int c = kEmpty_ + 1; c < kNumClasses; ++c) {
        if (!map_class(c) || p->num_count[c] <= 0) continue;
        const bool whole = c == p->num_whole;
        const int32_t *rows = whole ? nullptr : p->rows_num.p + p->num_off[c];
        const int32_t nrows = whole ? p->a_rows : p->num_count[c];
        if (pass == 0)
          launch_map_dedup_insert(rows, nrows, p->rmap_key.p, p->rmap_tkey.p,
                                  p->rmap_trow.p, mask, s);
        else
          launch_map_dedup_resolve(rows, nrows, p->rmap_key.p, p->rmap_tkey.p,
                                   p->rmap_trow.p, mask, c_rp, p->rmap_ops.p,
                                   p->rmap_off.p, p->rmap.p, p->rmap_shared.p,
                                   p->rmap_canon.p, p->rmap_share_count.p, s);
      }
    }
  }
  p->pat_ready = 0;
  if (dedup) {
    e = build_term_tables(p, s, op, c_rp, entries);
    if (e != cudaSuccess) return e;
  }
  p->rmap_state = 1;
  p->rmap_col = c_col;
  p->rmap_entries = entries;
  return cudaGetLastError();
}

}  // namespace

rvsp_status_t rvsp_cuda_plan_prepare_reuse(rvsp_cuda_plan_t p, void *stream,
                                           const int32_t *a_row_ptr, const int32_t *a_col_idx,
                                           const int32_t *b_row_ptr, const int32_t *b_col_idx,
                                           const int32_t *c_row_ptr, const int32_t *c_col_idx,
                                           int64_t *map_entries_out) {
  if (!p || !a_row_ptr || !a_col_idx || !b_row_ptr || !b_col_idx || !c_row_ptr ||
      !c_col_idx)
    return RVSP_ERROR_NULL_POINTER;
  if (!p->analysed) return RVSP_ERROR_INVALID_ARGUMENT;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const Operands op{p->a_rows, p->b_cols, a_row_ptr, a_col_idx, nullptr,
                    b_row_ptr, b_col_idx, nullptr,
                    merge_allowed(p->merge_policy, p->a_rows)};
  const cudaError_t e = build_reuse_map(p, s, op, c_row_ptr, c_col_idx);
  if (map_entries_out) *map_entries_out = p->rmap_state == 1 ? p->rmap_entries : 0;
  return map_cuda(e);
}

rvsp_status_t rvsp_cuda_plan_reuse_shared_rows(rvsp_cuda_plan_t p, void *stream,
                                               int32_t *shared_rows_out) {
  if (!p || !shared_rows_out) return RVSP_ERROR_NULL_POINTER;
  *shared_rows_out = 0;
  if (p->rmap_state != 1 || !p->rmap_shared.p) return RVSP_SUCCESS;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  cudaError_t e = cudaMemcpyAsync(shared_rows_out, p->rmap_shared.p, sizeof(int32_t),
                                  cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  return map_cuda(e);
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
                    b_row_ptr, b_col_idx, b_values,
                    merge_allowed(p->merge_policy, p->a_rows)};
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
  if (p->learned && fill) {
    // The fused pass already holds every non-overflowed row, sorted, with
    // its values: copy them; the overflowed rows take the plain fill.
    {
      PhaseScope ph(p, s, RVSP_PHASE_COMPACT);
      launch_compact(p->a_rows, p->counts.p, p->slab_off.p, c_row_ptr, p->slab_col.p,
                     p->slab_val.p, c_col_idx, c_values, true, p->big_rows.p,
                     p->num_sms, s);
      ph.launches = 2;
      for (int c = kEmpty_ + 1; c < kNumClasses && p->n_ovf > 0; ++c) {
        if (p->ovf_num_count[c] <= 0) continue;
        launch_numeric_class(c, op, p->ops.p, p->ovf_sorted.p + p->ovf_num_off[c],
                             p->ovf_num_count[c], c_row_ptr, c_col_idx, c_values, true,
                             dense_acc, dense_bits, p->dense_slots, p->misc.p + kStatus,
                             p->num_sms, s);
        ph.launches += 1;
      }
    }
    // Those values are the ones A and B held at estimation; if they changed
    // since, recompute every value with the structure now in C.
    values_fingerprint_launch(p, a_values, p->a_nnz, b_values, p->b_nnz, s);
    cudaError_t e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return map_cuda(e);
    if (p->h_vhash[0] == p->est_hash) return map_cuda(cudaGetLastError());
    fill = 0;
  }
  if (fill == 0 && (p->rmap_state == 0 || (p->rmap_state == 1 && p->rmap_col != c_col_idx))) {
    // First numeric-only call on this structure: build the reuse map, unless
    // the stream is being captured (building synchronizes).
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(s, &cap) == cudaSuccess && cap == cudaStreamCaptureStatusNone) {
      const cudaError_t e = build_reuse_map(p, s, op, c_row_ptr, c_col_idx);
      if (e != cudaSuccess) return map_cuda(e);
    }
  }
  const bool use_map = fill == 0 && p->rmap_state == 1 && p->rmap_col == c_col_idx;
  // numeric-only with every table in place: the row groups run side by side
  Lanes ln(p, s, use_map && (!p->shift_active || p->shift_tables == 1));
  bool rt_main = false;  // the largest shared-map pattern kernel, launched last
  {
    PhaseScope ph(p, s, RVSP_PHASE_NUMERIC);
    if (use_map && p->pat_ready && p->n_pat_rows > 0) {
      if (p->rt.ready && p->tiles_enabled) {
        ph.launches += launch_table_tile_kernel(p->rt, op, c_row_ptr, c_values, ln.next());
        ph.launches += launch_pattern_kernels(p->rt, op, c_row_ptr, c_values,
                                              p->misc.p + kStatus, ln, false);
        rt_main = true;
        if (p->rt.n_lo > 0) {
          launch_pat_numeric(op, p->ops.p, p->rt.lo_rows.p, p->rt.lo_ids.p, p->rt.n_lo,
                             c_row_ptr, c_values, p->pat_off.p, p->pat_steps.p, p->pat_rec.p,
                             p->pat_max_ops, p->pat_max_out, ln.next());
          ph.launches += 1;
        }
      } else {
        launch_pat_numeric(op, p->ops.p, p->pat_rows.p, p->pat_ids.p, p->n_pat_rows,
                           c_row_ptr, c_values, p->pat_off.p, p->pat_steps.p, p->pat_rec.p,
                           p->pat_max_ops, p->pat_max_out, ln.main());
        ph.launches += 1;
      }
    }
    // Persistent pass: the merge and map rows in one launch over a queue of
    // row bins, heaviest class first.
    const bool persist = use_map && p->persist_merge_rows > 0 &&
                         p->persist_head.reserve(1) == cudaSuccess;
    if (persist) {
      PersistPlan pp;
      int32_t max_out = 0;
      const int order[] = {kW2048, kW1024, kW512, kW256, kW128, kW64, kM16, kM8, kM4};
      for (int c : order) {
        if (p->num_count[c] <= 0) continue;
        const bool whole = c == p->num_whole;
        PersistSeg g;
        g.cls = c;
        if (map_class(c) && p->pat_ready) {
          g.rows = p->res_rows.p + p->res_off[c];
          g.count = p->res_count[c];
        } else {
          g.rows = whole ? nullptr : p->rows_num.p + p->num_off[c];
          g.count = whole ? p->a_rows : p->num_count[c];
        }
        if (g.count <= 0) continue;
        g.per_item = map_class(c) ? kPersistThreads / 32 : p->persist_merge_rows;
        g.item0 = pp.n_items;
        pp.seg[pp.nseg++] = g;
        pp.n_items += (g.count + g.per_item - 1) / g.per_item;
        if (map_class(c) && max_out == 0) max_out = 1 << (class_log2(c) - 1);
      }
      launch_persist_numeric(op, p->ops.p, pp, p->persist_head.p, c_row_ptr, c_values,
                             p->rmap_off.p, p->rmap.p, p->misc.p + kStatus, max_out,
                             p->persist_blocks, p->num_sms, ln.next());
      ph.launches += 2;
    } else {
      cudaGetLastError();
    }
    for (int c = kEmpty_ + 1; c < kNumClasses; ++c) {
      if (p->num_count[c] <= 0) continue;
      if (persist && persist_class(c)) continue;
      const bool whole = c == p->num_whole;
      const int32_t *rows = whole ? nullptr : p->rows_num.p + p->num_off[c];
      const int32_t nrows = whole ? p->a_rows : p->num_count[c];
      if (use_map && map_class(c) && p->pat_ready) {
        if (p->res_count[c] > 0)
          launch_map_numeric(c, op, p->ops.p, p->res_rows.p + p->res_off[c],
                             p->res_count[c], c_row_ptr, c_values, p->rmap_off.p,
                             p->rmap.p, p->misc.p + kStatus, ln.next());
      } else if (use_map && map_class(c))
        launch_map_numeric(c, op, p->ops.p, rows, nrows, c_row_ptr, c_values,
                           p->rmap_off.p, p->rmap.p, p->misc.p + kStatus, ln.next());
      else
        launch_numeric_class(c, op, p->ops.p, rows, nrows, c_row_ptr, c_col_idx, c_values,
                             fill != 0, dense_acc, dense_bits, p->dense_slots,
                             p->misc.p + kStatus, p->num_sms, ln.next());
      ph.launches += 1;
    }
    if (rt_main)
      ph.launches += launch_pattern_kernels(p->rt, op, c_row_ptr, c_values, p->misc.p + kStatus,
                                            ln, true);
    if (!p->shift_active) ln.join();
  }
  if (p->shift_active) {
    // Shift-class members: columns by translation of their canonical rows
    // (filled above), values from the canonical rows' term tables.
    if (fill) {
      PhaseScope ph(p, s, RVSP_PHASE_NUMERIC);
      launch_shift_fill(p->a_rows, p->st.pid.p, p->sh_rcls.p, c_row_ptr, c_col_idx, s);
      ph.launches = 1;
    }
    if (p->shift_tables == 0) {
      cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
      if (cudaStreamIsCapturing(s, &cap) != cudaSuccess || cap != cudaStreamCaptureStatusNone)
        return RVSP_ERROR_INVALID_ARGUMENT;  // building synchronizes: not under capture
      const cudaError_t e = build_shift_tables(p, s, op, c_row_ptr, c_col_idx);
      if (e != cudaSuccess) return map_cuda(e);
    }
    if (p->shift_tables != 1) return RVSP_ERROR_DEVICE;
    PhaseScope ph(p, s, RVSP_PHASE_NUMERIC);
    ph.launches = launch_shift_numeric(p, ln, op, c_row_ptr, c_values);
    ln.join();
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
  cudaError_t re = p->check_long.reserve(1 + size_t(check_long_rows_cap(rows, nnz)));
  if (re != cudaSuccess) return map_cuda(re);
  cudaMemsetAsync(p->check.p, 0xff, sizeof(unsigned long long), s);
  cudaMemsetAsync(p->check_long.p, 0, sizeof(int32_t), s);
  {
    PhaseScope ph(p, s, RVSP_PHASE_CHECK);
    launch_csr_check(rows, cols, row_ptr, col_idx, nnz, p->check.p, p->check_long.p, s);
    ph.launches = 2;
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
