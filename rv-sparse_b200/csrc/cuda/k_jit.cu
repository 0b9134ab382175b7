// Pattern kernels: row tiles of one term pattern, compiled for that pattern.
//
// The row-tile kernel (k_tile.cu) reads each product's output position from
// a table, so its accumulators must be addressable: a shared-memory column
// per lane, which costs three shared accesses and several integer
// instructions per product and, at about 16 KB a warp, caps the SM at a few
// warps.  When one pattern covers many rows (the interior of a stencil), this
// file writes CUDA source for that pattern alone -- its A length, B row
// lengths and every product's position are constants -- and compiles it with
// NVRTC for the GPU in use.  Each lane keeps its row's outputs in registers
// (c0 ... c{m-1}, named statically), so a product is one shared load of b, a
// multiply and an add.  One warp takes one tile (up to 32 consecutive rows of
// the pattern, one per lane):
//
//   A segment: the tile's A values and, per A nonzero, the start of its B row
//   (b_rp[a_col]) into shared memory;
//   the A nonzeros are cut into groups whose B spans overlap (in a stencil
//   the three x-neighbours of a row read B rows one apart, so the tile's
//   three spans share all but two rows; the grouping is chosen when the
//   kernel is built, from the largest union span over the pattern's tiles);
//   per group, the union of the lanes' B rows is one contiguous range of B
//   values, copied into shared memory by one bulk copy (cp.async.bulk, the
//   copy engine; its completion is counted on an mbarrier), one group ahead
//   of the arithmetic (two buffers);
//   for each A nonzero j of the group (ascending) and entry e of B row k_j:
//     c[q(j,e)] = fl(c[q(j,e)] + fl(a_j * b[k_j][e]))   (q a constant)
//
// and the outputs go to C through shared memory: when the tile's rows are
// one run of consecutive rows, their C rows are one contiguous block (equal
// lengths), which is written by one bulk store (plain stores for the ends
// outside whole 16-byte units); otherwise row by row, coalesced.  Accumulators start from a
// run-time +0.0f (a kernel argument, so no compiler can fold 0 + p to p:
// +0 + -0 must give +0) and every product and sum is rounded separately
// (__fmul_rn, __fadd_rn, -fmad=false), in ascending A-nonzero order: the
// reference's order and rounding (gustavson_core_f32.inc:31-62,
// accum_scalar_f32.c:20-71), so values equal the table kernel's bit for bit.
//
// A bulk copy moves whole 16-byte units: the range is widened to the units
// that hold its first and last B values.  Every unit read holds at least one
// B value of the range, so no copy reads outside the pages of B's values,
// and the B index of the first staged float is recorded per buffer.  Each
// wait on an mbarrier is bounded (about a second of clock cycles); a wait
// that runs out makes the warp wait, again bounded, for the copies it has in
// flight, record kDevWaitTimeout in the status word and return.
//
// NVRTC is opened at run time (dlopen of libnvrtc.so.12); without it, or if
// a compile fails, the pattern stays on the table kernel.  The patterns of
// one structure compile side by side, one host thread each.  Compiled
// kernels are kept for the life of the process, keyed by the pattern's
// numbers and the architecture: a pattern is compiled once per process, and
// a cached one is not even turned into source again.
#include <cuda_runtime.h>
#include <dlfcn.h>
#include <nvrtc.h>

#include <algorithm>
#include <chrono>
#include <climits>
#include <cstdio>
#include <map>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "device_common.cuh"
#include "kernels.cuh"

namespace rvsp {

namespace {

constexpr int kJitThreads = 64;  // two warps (tiles) per block

// ---- NVRTC, opened on first use ---------------------------------------------
struct Nvrtc {
  bool tried = false, ok = false;
  nvrtcResult (*create)(nvrtcProgram *, const char *, const char *, int, const char *const *,
                        const char *const *) = nullptr;
  nvrtcResult (*compile)(nvrtcProgram, int, const char *const *) = nullptr;
  nvrtcResult (*cubin_size)(nvrtcProgram, size_t *) = nullptr;
  nvrtcResult (*cubin)(nvrtcProgram, char *) = nullptr;
  nvrtcResult (*destroy)(nvrtcProgram *) = nullptr;
};

std::mutex g_mutex;
Nvrtc g_nvrtc;
std::map<std::string, cudaKernel_t> g_cache;  // pattern key -> kernel
int g_compiles = 0;
double g_compile_ms = 0.0;

bool open_nvrtc() {
  if (g_nvrtc.tried) return g_nvrtc.ok;
  g_nvrtc.tried = true;
  const char *names[] = {"libnvrtc.so.12", "libnvrtc.so", "/usr/local/cuda/lib64/libnvrtc.so.12"};
  void *h = nullptr;
  for (const char *n : names)
    if ((h = dlopen(n, RTLD_NOW | RTLD_LOCAL)) != nullptr) break;
  if (!h) return false;
  g_nvrtc.create = reinterpret_cast<decltype(g_nvrtc.create)>(dlsym(h, "nvrtcCreateProgram"));
  g_nvrtc.compile = reinterpret_cast<decltype(g_nvrtc.compile)>(dlsym(h, "nvrtcCompileProgram"));
  g_nvrtc.cubin_size = reinterpret_cast<decltype(g_nvrtc.cubin_size)>(dlsym(h, "nvrtcGetCUBINSize"));
  g_nvrtc.cubin = reinterpret_cast<decltype(g_nvrtc.cubin)>(dlsym(h, "nvrtcGetCUBIN"));
  g_nvrtc.destroy = reinterpret_cast<decltype(g_nvrtc.destroy)>(dlsym(h, "nvrtcDestroyProgram"));
  g_nvrtc.ok = g_nvrtc.create && g_nvrtc.compile && g_nvrtc.cubin_size && g_nvrtc.cubin &&
               g_nvrtc.destroy;
  return g_nvrtc.ok;
}

// ---- the generated source ---------------------------------------------------
// The helpers of every pattern kernel: mbarrier init / bounded wait, the
// bulk copies of a B range and of a tile's record and A values, the bulk
// store of a C block.
const char *kPrelude = R"(
typedef unsigned int u32;
typedef unsigned long long u64;
typedef unsigned short u16;
#define FULL 0xffffffffu
// Two products and sums in one f32x2 multiply and one f32x2 add, each half
// rounded to nearest like __fmul_rn / __fadd_rn (never fused):
// (c0, c1) = (c0 + a * b0, c1 + a * b1), a2 holding a in both halves.
__device__ __forceinline__ u64 pk2(float a) {
  u64 r;
  asm("mov.b64 %0, {%1, %1};" : "=l"(r) : "f"(a));
  return r;
}
__device__ __forceinline__ void muladd2(float &c0, float &c1, u64 a2, float b0, float b1) {
  u64 acc, b, p;
  asm("mov.b64 %0, {%1, %2};" : "=l"(acc) : "f"(c0), "f"(c1));
  asm("mov.b64 %0, {%1, %2};" : "=l"(b) : "f"(b0), "f"(b1));
  asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(p) : "l"(a2), "l"(b));
  asm("add.rn.f32x2 %0, %1, %2;" : "=l"(acc) : "l"(acc), "l"(p));
  asm("mov.b64 {%0, %1}, %2;" : "=f"(c0), "=f"(c1) : "l"(acc));
}
__device__ __forceinline__ u32 saddr(const void *p) { return (u32)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void bar_init(u32 bar) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(bar) : "memory");
}
__device__ __forceinline__ bool bar_try(u32 bar, u32 ph) {
  u32 ok;
  asm volatile("{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
               " selp.u32 %0, 1, 0, p;\n}\n" : "=r"(ok) : "r"(bar), "r"(ph) : "memory");
  return ok != 0u;
}
// Waits for phase ph of the mbarrier; false after about 2^31 clock cycles.
__device__ __forceinline__ bool bar_wait(u32 bar, u32 ph) {
  if (bar_try(bar, ph)) return true;
  const long long t0 = clock64();
  while (!bar_try(bar, ph))
    if (clock64() - t0 > (1ll << 31)) return false;
  return true;
}
// L2 policies: B ranges are read by up to nine tiles (kept: evict_last);
// tile records, A values and C blocks pass through once (evict_first).
__device__ __forceinline__ u64 policy_keep() {
  u64 p;
  asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;\n" : "=l"(p));
  return p;
}
__device__ __forceinline__ u64 policy_stream() {
  u64 p;
  asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;\n" : "=l"(p));
  return p;
}
__device__ __forceinline__ void bulk_load(void *dst, u64 src, u32 bytes, u32 bar, u64 pol) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes.L2::cache_hint"
               " [%0], [%1], %2, [%3], %4;\n"
               ::"r"(saddr(dst)), "l"(src), "r"(bytes), "r"(bar), "l"(pol) : "memory");
}
__device__ __forceinline__ void expect(u32 bar, u32 bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n"
               ::"r"(bar), "r"(bytes) : "memory");
}
// Lane 0 copies B values [lo, hi) (widened to whole 16-byte units) to dst,
// completing on bar.  Returns the position in dst of B value lo.
__device__ __forceinline__ int stage(float *dst, const float *b_val, int lo, int hi, u32 bar,
                                     int lane, u64 pol) {
  const u64 g0 = (u64)(b_val + lo);
  if (lane == 0) {
    const u64 a0 = g0 & ~15ull;
    const u64 a1 = ((u64)(b_val + hi) + 15ull) & ~15ull;
    expect(bar, (u32)(a1 - a0));
    bulk_load(dst, a0, (u32)(a1 - a0), bar, pol);
  }
  return (int)((g0 & 15ull) >> 2);
}
// Lane 0 copies a tile's record (rwords words of prog) to dst and its A
// values a_val[r.x, r.x + r.y) (widened to 16-byte units) after it,
// completing on bar.
__device__ __forceinline__ void stage_tile(float *dst, const int *prog, int rwords, int2 r,
                                           int tile, const float *a_val, u32 bar, int lane,
                                           u64 pol) {
  if (lane == 0) {
    const u64 a0 = (u64)(a_val + r.x) & ~15ull;
    const u64 a1 = ((u64)(a_val + r.x + r.y) + 15ull) & ~15ull;
    const u32 rb = (u32)rwords * 4u, ab = r.y > 0 ? (u32)(a1 - a0) : 0u;
    expect(bar, rb + ab);
    bulk_load(dst, (u64)(prog + (size_t)tile * rwords), rb, bar, pol);
    if (ab) bulk_load(dst + rwords, a0, ab, bar, pol);
  }
}
// The next tile of the launch's queue (head zeroed before the launch).
__device__ __forceinline__ int take(int *head, int lane) {
  int t = 0;
  if (lane == 0) t = atomicAdd(head, 1);
  return __shfl_sync(FULL, t, 0);
}
__device__ __forceinline__ void store_block(float *g, const float *s, int bytes, u64 pol) {
  asm volatile("cp.async.bulk.global.shared::cta.bulk_group.L2::cache_hint [%0], [%1], %2, %3;\n"
               ::"l"(g), "r"(saddr(s)), "r"(bytes), "l"(pol) : "memory");
  asm volatile("cp.async.bulk.commit_group;\n" ::: "memory");
  asm volatile("cp.async.bulk.wait_group.read 0;\n" ::: "memory");
}
)";

// Registers of a pattern kernel with m outputs: the m accumulators and
// about 19 for addresses and staged b values in flight, then raised to the
// most that keeps as many warps per scheduler (a quarter of the SM's 64K
// registers, allocated in units of 256 per warp): 168 at m = 125, 3 warps.
int pattern_regs(int m) {
  int r = (m + 19 + 7) & ~7;
  r = r < 64 ? 64 : r > 255 ? 255 : r;
  const int per_sched = 16384 / (((r * 32) + 255) & ~255);
  int up = (16384 / per_sched / 32) & ~7;
  return up > 255 ? 255 : up < r ? r : up;
}

// Accumulator pairs of a pattern kernel: outputs (2p + par, 2p + 1 + par),
// for the parity par under which the most products of one A nonzero reach
// both outputs of a pair (each such two products take one f32x2 multiply
// and one f32x2 add).  Each output still sums its products in ascending
// A-nonzero order.
int pair_parity(int na, const int *len, const std::vector<int> &slot, int m) {
  int count[2] = {0, 0};
  std::vector<char> hit(size_t(m), 0);
  size_t t = 0;
  for (int j = 0; j < na; ++j) {
    std::fill(hit.begin(), hit.end(), 0);
    for (int e = 0; e < len[j]; ++e) hit[size_t(slot[t + size_t(e)])] = 1;
    for (int q = 0; q + 1 < m; ++q)
      if (hit[size_t(q)] && hit[size_t(q) + 1]) ++count[q & 1];
    t += size_t(len[j]);
  }
  return count[1] > count[0] ? 1 : 0;
}

// Words of a tile record (see jit_record_words).
int record_words(int na, int ngroups) { return (4 + 2 * ngroups + 16 + 16 * na + 3) & ~3; }

// Source of the kernel for one pattern: na A nonzeros with B row lengths
// len[j], slot[t] the output position of flattened product t (in j, e
// order), m outputs, and the groups of A nonzeros staged together
// ([first, end) ranges over j, in order, covering every j with len > 0).
//
// The kernel is persistent: each warp takes tiles from the launch's queue
// (an atomic counter), so warps that start late take fewer.
// Per warp, shared memory holds two tile buffers (record + A values) around
// two B stage buffers: [tile 0 | stage 0 | stage 1 | tile 1].  While a tile
// is computed, the next tile's record and A values are copied into the other
// tile buffer; the outputs of a tile go out through its own tile buffer and
// the stage buffers (one contiguous region either way), 16 rows at a time.
std::string pattern_source(int na, const int *len, const std::vector<int> &slot, int m,
                           const std::vector<std::pair<int, int>> &groups) {
  std::string s(kPrelude);
  char buf[1024];
  const int ms = (m & 1) ? m : m + 1;  // odd row stride: conflict-free stores
  const int ng = static_cast<int>(groups.size());
  const int rw = record_words(na, ng);
  const int aoff_w = 4 + 2 * ng, d_w = aoff_w + 16;
  // the next tile's copies go out with group mid's, late enough that the
  // next tile's number (an atomic on the queue head) and A range are in
  const int mid = ng / 2;
  std::vector<int> t_of(size_t(na) + 1, 0);
  for (int j = 0; j < na; ++j) t_of[size_t(j) + 1] = t_of[size_t(j)] + len[j];
  const int par = pair_parity(na, len, slot, m);
  snprintf(buf, sizeof(buf), "#define RW %d\n#define M %d\n#define MS %d\n", rw, m, ms);
  s += buf;
  snprintf(buf, sizeof(buf), "extern \"C\" __global__ void __maxnreg__(%d)\n", pattern_regs(m));
  s += buf;
  s += "rvsp_pattern_tiles(const int *__restrict__ prog, const int2 *__restrict__ arange,\n"
       "    int ntiles, const float *__restrict__ a_val, const float *__restrict__ b_val,\n"
       "    const int *__restrict__ c_rp, float *__restrict__ c_val, int stage_cap,\n"
       "    int abuf_floats, int work_floats, float zero, int *__restrict__ head,\n"
       "    int *__restrict__ status) {\n"
       "  extern __shared__ __align__(16) float sm[];\n"
       "  __shared__ __align__(8) u64 bars[8];\n"
       "  const int wib = threadIdx.x >> 5, lane = threadIdx.x & 31;\n"
       "  float *const work = sm + wib * work_floats;\n"
       "  float *const sb0 = work + abuf_floats;\n"
       "  float *const sb1 = sb0 + stage_cap;\n"
       "  float *const tb1 = sb1 + stage_cap;\n"
       "  int tile = take(head, lane);\n"
       "  if (tile >= ntiles) return;\n"
       "  const u32 bar0 = saddr(&bars[4 * wib]), bar1 = bar0 + 8u;\n"
       "  const u32 bara0 = bar0 + 16u, bara1 = bar0 + 24u;\n"
       "  if (lane == 0) {\n"
       "    bar_init(bar0); bar_init(bar1); bar_init(bara0); bar_init(bara1);\n"
       "    asm volatile(\"fence.mbarrier_init.release.cluster;\\n\" ::: \"memory\");\n"
       "  }\n"
       "  __syncwarp();\n"
       "  u32 pb0 = 0u, pb1 = 0u, pa0 = 0u, pa1 = 0u;\n"
       "  const u64 keep = policy_keep(), once = policy_stream();\n"
       "  // lane 0 holds the ticket of the tile after this one, requested a\n"
       "  // tile ahead so that its atomic is back when the number is needed\n"
       "  int ticket = lane == 0 ? atomicAdd(head, 1) : 0;\n"
       "  stage_tile(work, prog, RW, __ldg(arange + tile), tile, a_val, bara0, lane, once);\n"
       "  for (int it = 0; tile < ntiles; ++it) {\n"
       "    const bool odd = (it & 1) != 0;\n"
       "    float *const ab = odd ? tb1 : work;\n"
       "    float *const nb = odd ? work : tb1;\n"
       "    float *const region = odd ? sb0 : work;\n"
       "    const u32 bara = odd ? bara1 : bara0, barn = odd ? bara0 : bara1;\n"
       "    const u32 pa = odd ? pa1 : pa0, pn = odd ? pa0 : pa1;\n"
       "    const int nxt = __shfl_sync(FULL, ticket, 0);\n"
       "    if (lane == 0 && nxt < ntiles) ticket = atomicAdd(head, 1);\n"
       "    const int2 nr = nxt < ntiles ? __ldg(arange + nxt) : make_int2(0, 0);\n"
       "    if (!__all_sync(FULL, bar_wait(bara, pa))) {\n"
       "      bar_wait(bara, pa);\n"
       "      if (lane == 0) atomicCAS(status, 0, 5);\n"
       "      return;\n"
       "    }\n"
       "    if (odd) pa1 ^= 1u; else pa0 ^= 1u;\n"
       "    const int *const rec = (const int *)ab;\n"
       "    const int row0 = rec[0];\n"
       "    const u32 mask = (u32)rec[1];\n"
       "    const bool active = ((mask >> lane) & 1u) != 0u;\n"
       "    const int cs = active ? __ldg(c_rp + row0 + lane) : 0;\n"
       "    const float *const sa = ab + RW + (int)(((u64)(a_val + rec[2]) & 15ull) >> 2) +\n"
       "                            (int)((const u16 *)(rec + ";
  snprintf(buf, sizeof(buf), "%d))[lane];\n    const u16 *const dd = (const u16 *)(rec + %d) + lane;\n",
           aoff_w, d_w);
  s += buf;
  for (int q = 0; q < m; ++q) {
    snprintf(buf, sizeof(buf), "    float c%d = zero;\n", q);
    s += buf;
  }
  s += "    int cb0 = stage(sb0, b_val, rec[4], rec[5], bar0, lane, keep), cb1 = 0;\n";
  for (int g = 0; g < ng; ++g) {
    const int b = g & 1;
    if (g + 1 < ng) {
      snprintf(buf, sizeof(buf),
               "    cb%d = stage(sb%d, b_val, rec[%d], rec[%d], bar%d, lane, keep);\n",
               (g + 1) & 1, (g + 1) & 1, 4 + 2 * (g + 1), 5 + 2 * (g + 1), (g + 1) & 1);
      s += buf;
    }
    if (g == mid) s += "    if (nxt < ntiles) stage_tile(nb, prog, RW, nr, nxt, a_val, barn, lane, once);\n";
    // bounded wait; on a timeout wait (bounded) for the copies still out
    snprintf(buf, sizeof(buf), "    if (!__all_sync(FULL, bar_wait(bar%d, pb%d))) {\n", b, b);
    s += buf;
    snprintf(buf, sizeof(buf), "      bar_wait(bar%d, pb%d);\n", b, b);
    s += buf;
    if (g + 1 < ng) {
      snprintf(buf, sizeof(buf), "      bar_wait(bar%d, pb%d);\n", (g + 1) & 1, (g + 1) & 1);
      s += buf;
    }
    if (g >= mid) s += "      if (nxt < ntiles) bar_wait(barn, pn);\n";
    s += "      if (lane == 0) atomicCAS(status, 0, 5);\n      return;\n    }\n";
    snprintf(buf, sizeof(buf), "    pb%d ^= 1u;\n    {\n      const float *const sbb = sb%d + cb%d;\n",
             b, b, b);
    s += buf;
    for (int j = groups[size_t(g)].first; j < groups[size_t(g)].second; ++j) {
      if (len[j] == 0) continue;
      snprintf(buf, sizeof(buf),
               "      {\n        const float a = sa[%d];\n"
               "        const float *const st = sbb + dd[%d];\n"
               "        const u64 a2 = pk2(a);\n",
               j, j * 32);
      s += buf;
      // e of each output this A nonzero reaches (its B row's columns are
      // distinct, so at most one), then the pairs in one f32x2 step each
      std::vector<int> e_of(size_t(m), -1);
      for (int e = 0; e < len[j]; ++e) e_of[size_t(slot[size_t(t_of[size_t(j)] + e)])] = e;
      for (int e = 0; e < len[j]; ++e) {
        const int q = slot[size_t(t_of[size_t(j)] + e)];
        const int mate = ((q - par) & 1) == 0 ? q + 1 : q - 1;
        const int em = mate >= 0 && mate < m ? e_of[size_t(mate)] : -1;
        if (em < 0)
          snprintf(buf, sizeof(buf), "        c%d = __fadd_rn(c%d, __fmul_rn(a, st[%d]));\n", q,
                   q, e);
        else if (q < mate)
          snprintf(buf, sizeof(buf), "        muladd2(c%d, c%d, a2, st[%d], st[%d]);\n", q, mate,
                   e, em);
        else
          continue;
        s += buf;
      }
      s += "      }\n";
    }
    s += "    }\n    __syncwarp();\n";
  }
  // outputs, 16 rows at a time: the active lanes' rows in lane order at
  // region[sh + (rank - base) * MS]; when the active lanes are one run of
  // consecutive rows their C rows are one block (equal lengths), aligned by
  // sh and written by one bulk store
  snprintf(buf, sizeof(buf),
           "    const int first = __ffs(mask) - 1, nact = __popc(mask);\n"
           "    const bool contig = %s (mask >> first) == (nact == 32 ? FULL : (1u << nact) - 1u);\n"
           "    const int rank = __popc(mask & ((1u << lane) - 1u));\n"
           "    const int cs0 = __shfl_sync(FULL, cs, first);\n"
           "    for (int base = 0; base < nact; base += 16) {\n"
           "      const int cnt = nact - base < 16 ? nact - base : 16;\n"
           "      const int sh = contig ? (int)(((u64)(c_val + cs0 + base * M) & 15ull) >> 2) : 0;\n"
           "      if (active && rank >= base && rank < base + 16) {\n"
           "        float *const o = region + sh + (rank - base) * MS;\n",
           ms == m ? "" : "false &&");
  s += buf;
  for (int q = 0; q < m; ++q) {
    snprintf(buf, sizeof(buf), "        o[%d] = c%d;\n", q, q);
    s += buf;
  }
  s += "      }\n"
       "      if (contig) {\n"
       "        asm volatile(\"fence.proxy.async.shared::cta;\\n\" ::: \"memory\");\n"
       "        __syncwarp();\n"
       "        float *const g = c_val + cs0 + base * M;\n"
       "        const int total = cnt * M;\n"
       "        const int head = min((4 - sh) & 3, total);\n"
       "        const int body = (total - head) & ~3;\n"
       "        if (lane < head) g[lane] = region[sh + lane];\n"
       "        if (head + body + lane < total) g[head + body + lane] = region[sh + head + body + lane];\n"
       "        if (lane == 0 && body > 0) store_block(g + head, region + sh + head, body * 4, once);\n"
       "      } else {\n"
       "        __syncwarp();\n"
       "        int k = 0;\n"
       "        for (u32 mm = mask; mm; mm &= mm - 1u, ++k) {\n"
       "          const int cb = __shfl_sync(FULL, cs, __ffs(mm) - 1);\n"
       "          if (k >= base && k < base + 16) {\n"
       "            const float *const src = region + (k - base) * MS;\n"
       "            for (int q = lane; q < M; q += 32) c_val[cb + q] = src[q];\n"
       "          }\n"
       "        }\n"
       "      }\n"
       "      __syncwarp();\n"
       "    }\n"
       "    tile = nxt;\n"
       "  }\n"
       "}\n";
  return s;
}

// NVRTC compile of `src` into a cubin for `arch` (empty on failure).  Makes
// no CUDA call, so several run at once on their own threads.
std::vector<char> compile_cubin(const std::string &src, const std::string &arch) {
  std::vector<char> bin;
  nvrtcProgram prog = nullptr;
  if (g_nvrtc.create(&prog, src.c_str(), "rvsp_pattern.cu", 0, nullptr, nullptr) !=
      NVRTC_SUCCESS)
    return bin;
  const char *opts[] = {arch.c_str(), "-fmad=false", "--std=c++17", "-default-device"};
  size_t n = 0;
  if (g_nvrtc.compile(prog, 4, opts) == NVRTC_SUCCESS &&
      g_nvrtc.cubin_size(prog, &n) == NVRTC_SUCCESS && n > 0) {
    bin.resize(n);
    if (g_nvrtc.cubin(prog, bin.data()) != NVRTC_SUCCESS) bin.clear();
  }
  g_nvrtc.destroy(&prog);
  return bin;
}

// The architecture string of the current device (`--gpu-architecture=sm_XYa`).
std::string current_arch() {
  int dev = 0, major = 0, minor = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev);
  cudaDeviceGetAttribute(&minor, cudaDevAttrComputeCapabilityMinor, dev);
  return "--gpu-architecture=sm_" + std::to_string(major) + std::to_string(minor) + "a";
}

// The kernels for `keys` (nullptr where a compile failed): cached ones at
// once; for the others source(i) is generated and compiled side by side,
// one thread each, then loaded on the calling thread (whose device is the
// plan's).  A key names everything its source depends on, so a cached
// pattern costs no source generation.
template <class Source>
void kernels_for(const std::vector<std::string> &keys, const Source &source,
                 std::vector<cudaKernel_t> &out) {
  out.assign(keys.size(), nullptr);
  std::vector<size_t> todo;
  {
    std::lock_guard<std::mutex> lock(g_mutex);
    for (size_t i = 0; i < keys.size(); ++i) {
      auto it = g_cache.find(keys[i]);
      if (it != g_cache.end()) out[i] = it->second;
      else todo.push_back(i);
    }
    if (todo.empty() || !open_nvrtc()) return;
  }
  const std::string arch = current_arch();
  const auto t0 = std::chrono::steady_clock::now();
  std::vector<std::vector<char>> bins(todo.size());
  std::vector<std::thread> threads;
  for (size_t k = 0; k < todo.size(); ++k) {
    auto work = [&bins, &source, &todo, &arch, k] {
      bins[k] = compile_cubin(source(todo[k]), arch);
    };
    try {
      threads.emplace_back(work);
    } catch (...) {  // no thread: compile here
      work();
    }
  }
  for (auto &t : threads) t.join();
  std::lock_guard<std::mutex> lock(g_mutex);
  for (size_t k = 0; k < todo.size(); ++k) {
    cudaKernel_t kern = nullptr;
    cudaLibrary_t lib = nullptr;
    if (!bins[k].empty() &&
        (cudaLibraryLoadData(&lib, bins[k].data(), nullptr, nullptr, 0, nullptr, nullptr, 0) !=
             cudaSuccess ||
         cudaLibraryGetKernel(&kern, lib, "rvsp_pattern_tiles") != cudaSuccess))
      kern = nullptr;
    cudaGetLastError();
    // a failure is remembered too: the table kernel keeps the pattern
    g_cache[keys[todo[k]]] = kern;
    out[todo[k]] = kern;
    ++g_compiles;
  }
  g_compile_ms += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0)
                      .count();
}

// Warps per block of the span and record kernels, and the A entries of one
// tile's segment they stage in shared memory (a longer segment's B row
// starts are read from global memory instead; 4 KB a warp and at most 64
// registers keep 32 warps an SM resident, these kernels being bound by load
// latency).
constexpr int kBuildWarps = 4;
constexpr int kBuildSeg = 1024;

// The start of B row a_col[seg0 + i], for every i < seg, into sb[i]: loads
// of a_col coalesced across the lanes, 512 entries at a time (16 loads a
// lane in flight, then their 16 gathers of b_rp).
__device__ __forceinline__ void stage_b_starts(int32_t *sb, int32_t seg0, int32_t seg,
                                               const int32_t *__restrict__ a_col,
                                               const int32_t *__restrict__ b_rp, int lane) {
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
  __syncwarp();
}

// The start of the B row of segment entry i: staged, or read through a_col.
__device__ __forceinline__ int32_t b_start(const int32_t *sb, bool staged, int32_t seg0,
                                           int32_t i, const int32_t *__restrict__ a_col,
                                           const int32_t *__restrict__ b_rp) {
  return staged ? sb[i] : __ldg(b_rp + __ldg(a_col + seg0 + i));
}

// A tile's segment: from the first active row's first A nonzero to the last
// active row's end.
__device__ __forceinline__ void tile_segment(const int4 &t, const int32_t *__restrict__ a_rp,
                                             int32_t *seg0, int32_t *seg) {
  const uint32_t mask = static_cast<uint32_t>(t.y);
  const int first = __ffs(static_cast<int>(mask)) - 1, last = 31 - __clz(static_cast<int>(mask));
  *seg0 = a_rp[t.x + first];
  *seg = a_rp[t.x + last + 1] - *seg0;
}

// Union spans of a sample of a pattern's tiles (every stride-th; warp per
// tile, grid-stride): for every A nonzero j0 and run length g in
// [1, kJitMaxGroup], span[j0 * kJitMaxGroup + g - 1] = the largest, over the
// sample, of (end of the last B value - first B value) that the tile's rows
// read for A nonzeros j0 .. j0 + g - 1.  A nonzero with an empty B row reads
// nothing.  The grouping is chosen from these; the tile records then measure
// every tile's ranges.  span zeroed by the caller.
__global__ void __launch_bounds__(kBuildWarps * 32, 8)
span_kernel(const int4 *__restrict__ tiles, int32_t ntiles, int32_t stride,
            const int4 *__restrict__ desc,
            const uint16_t *__restrict__ lens, const int32_t *__restrict__ a_rp,
            const int32_t *__restrict__ a_col, const int32_t *__restrict__ b_rp,
            int32_t *__restrict__ span) {
  __shared__ int32_t sseg[kBuildWarps][kBuildSeg];
  __shared__ int32_t slo[kBuildWarps][32], shi[kBuildWarps][32], slen[32];
  const int wib = threadIdx.x >> 5, lane = lane_id();
  const int32_t na = desc->x;  // A nonzeros of the pattern
  if (na <= 0 || na > 32) return;
  if (threadIdx.x < 32) slen[threadIdx.x] = threadIdx.x < na ? lens[threadIdx.x] : 0;
  __syncthreads();
  int32_t um[kJitMaxGroup];
#pragma unroll
  for (int g = 0; g < kJitMaxGroup; ++g) um[g] = 0;
  for (int64_t w = int64_t(blockIdx.x) * kBuildWarps + wib; w * stride < ntiles;
       w += int64_t(gridDim.x) * kBuildWarps) {
    const int4 t = tiles[w * stride];
    const bool active = ((static_cast<uint32_t>(t.y) >> lane) & 1u) != 0u;
    int32_t seg0 = 0, seg = 0;
    tile_segment(t, a_rp, &seg0, &seg);
    const int32_t p = active ? a_rp[t.x + lane] - seg0 : 0;
    const bool staged = seg <= kBuildSeg;
    if (staged) stage_b_starts(sseg[wib], seg0, seg, a_col, b_rp, lane);
    for (int32_t j = 0; j < na; ++j) {
      const bool use = active && slen[j] > 0 && p + j < seg;
      const int32_t r = use ? b_start(sseg[wib], staged, seg0, p + j, a_col, b_rp) : 0;
      const int32_t lo = __reduce_min_sync(kFull, use ? r : INT_MAX);
      const int32_t hi = __reduce_max_sync(kFull, use ? r + slen[j] : INT_MIN);
      if (lane == 0) {
        slo[wib][j] = lo;
        shi[wib][j] = hi;
      }
    }
    __syncwarp();
    if (lane < na) {
      int32_t lo = INT_MAX, hi = INT_MIN;
#pragma unroll
      for (int g = 0; g < kJitMaxGroup; ++g) {
        if (lane + g < na) {
          lo = min(lo, slo[wib][lane + g]);
          hi = max(hi, shi[wib][lane + g]);
          if (hi > lo) um[g] = max(um[g], hi - lo);
        }
      }
    }
    __syncwarp();
  }
  if (lane < na) {
#pragma unroll
    for (int g = 0; g < kJitMaxGroup; ++g)
      if (um[g] > 0) atomicMax(span + lane * kJitMaxGroup + g, um[g]);
  }
}

// Tile records of one pattern (warp per tile, grid-stride), rw words each:
//   [0] first row of the tile, [1] lane mask, [2] A index of the first active
//   row's first nonzero, [3] A entries from there to the last active row's
//   end;  [4 + 2g], [5 + 2g]: the B range [lo, hi) that group g stages;
//   then 32 uint16 A offsets (lane's first nonzero - [2]) and, per A nonzero
//   j and lane, the uint16 offset of the lane's B row k_j from its group's
//   lo (0 for inactive lanes and empty B rows).
// arange[tile] = ([2], [3]); maxima[0] = the largest [3], maxima[1 + g] =
// the largest B range of group g.  Structure only: built once per
// structure, read by every numeric-only repeat.
__global__ void __launch_bounds__(kBuildWarps * 32, 8)
program_kernel(const int4 *__restrict__ tiles, int32_t ntiles, int32_t na, int32_t ngroups,
               const int2 *__restrict__ groups, const uint16_t *__restrict__ lens,
               const int32_t *__restrict__ a_rp, const int32_t *__restrict__ a_col,
               const int32_t *__restrict__ b_rp, int32_t rw, int32_t *__restrict__ prog,
               int2 *__restrict__ arange, int32_t *__restrict__ maxima) {
  __shared__ int32_t sseg[kBuildWarps][kBuildSeg];
  __shared__ int32_t slen[32];
  const int wib = threadIdx.x >> 5, lane = lane_id();
  if (threadIdx.x < 32) slen[threadIdx.x] = threadIdx.x < na ? lens[threadIdx.x] : 0;
  __syncthreads();
  // the warp's maxima over its tiles (the A extent; lane g: group g's B
  // range), merged into maxima once at the end
  int32_t mine = 0, segmax = 0;
  for (int64_t w = int64_t(blockIdx.x) * kBuildWarps + wib; w < ntiles;
       w += int64_t(gridDim.x) * kBuildWarps) {
    const int4 t = tiles[w];
    const bool active = ((static_cast<uint32_t>(t.y) >> lane) & 1u) != 0u;
    int32_t seg0 = 0, seg = 0;
    tile_segment(t, a_rp, &seg0, &seg);
    const int32_t p = active ? a_rp[t.x + lane] - seg0 : 0;
    const bool staged = seg <= kBuildSeg;
    if (staged) stage_b_starts(sseg[wib], seg0, seg, a_col, b_rp, lane);
    int32_t *const rec = prog + w * rw;
    if (lane == 0) {
      rec[0] = t.x;
      rec[1] = t.y;
      rec[2] = seg0;
      rec[3] = seg;
      arange[w] = make_int2(seg0, seg);
    }
    segmax = max(segmax, seg);
    uint16_t *const aoff = reinterpret_cast<uint16_t *>(rec + 4 + 2 * ngroups);
    uint16_t *const d = aoff + 32;
    aoff[lane] = static_cast<uint16_t>(p);
    for (int32_t g = 0; g < ngroups; ++g) {
      const int2 gr = groups[g];
      int32_t lo = INT_MAX, hi = INT_MIN;
      for (int32_t j = gr.x; j < gr.y; ++j) {
        if (active && slen[j] > 0 && p + j < seg) {
          const int32_t r = b_start(sseg[wib], staged, seg0, p + j, a_col, b_rp);
          lo = min(lo, r);
          hi = max(hi, r + slen[j]);
        }
      }
      lo = __reduce_min_sync(kFull, lo);
      hi = __reduce_max_sync(kFull, hi);
      if (lane == 0) {
        rec[4 + 2 * g] = lo;
        rec[5 + 2 * g] = hi;
      }
      if (lane == g) mine = max(mine, hi - lo);
      for (int32_t j = gr.x; j < gr.y; ++j) {
        const bool use = active && slen[j] > 0 && p + j < seg;
        d[j * 32 + lane] = static_cast<uint16_t>(
            use ? b_start(sseg[wib], staged, seg0, p + j, a_col, b_rp) - lo : 0);
      }
    }
    __syncwarp();
  }
  if (lane == 0 && segmax > 0) atomicMax(maxima, segmax);
  if (lane < ngroups && mine > 0) atomicMax(maxima + 1 + lane, mine);
}

// desc[pid].w = 1: the table kernel leaves the pattern's tiles alone.
__global__ void mark_pattern_kernel(int4 *desc, int32_t pid) { desc[pid].w = 1; }

// The tiles the table kernel keeps (pattern not marked), in order of
// arrival (count at *n, zeroed by the caller).
__global__ void __launch_bounds__(256)
table_tiles_kernel(const int4 *__restrict__ tiles, int32_t ntiles,
                   const int4 *__restrict__ desc, int4 *__restrict__ out,
                   int32_t *__restrict__ n) {
  const int32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  int4 t = make_int4(0, 0, 0, 0);
  bool take = false;
  if (i < ntiles) {
    t = tiles[i];
    take = desc[t.z].w == 0;
  }
  const unsigned b = __ballot_sync(kFull, take);
  if (!b) return;
  int32_t base = 0;
  if (lane_id() == 0) base = atomicAdd(n, __popc(b));
  base = __shfl_sync(kFull, base, 0);
  if (take) out[base + __popc(b & lanemask_lt())] = t;
}

}  // namespace

void jit_stats(int32_t *compiles, double *ms) {
  std::lock_guard<std::mutex> lock(g_mutex);
  if (compiles) *compiles = g_compiles;
  if (ms) *ms = g_compile_ms;
}

int jit_pattern_kernels(std::vector<JitRequest> &reqs) {
  std::vector<std::string> keys;
  std::vector<size_t> idx;
  const std::string arch = current_arch();
  for (size_t i = 0; i < reqs.size(); ++i) {
    JitRequest &r = reqs[i];
    r.kernel = nullptr;
    if (r.na <= 0 || r.na > 32 || r.m <= 0 || r.groups.empty()) continue;
    // the key: architecture, generator version and the pattern's numbers
    std::vector<int32_t> w = {5, r.na, r.m, static_cast<int32_t>(r.groups.size())};
    w.insert(w.end(), r.len, r.len + r.na);
    for (const auto &g : r.groups) {
      w.push_back(g.first);
      w.push_back(g.second);
    }
    w.insert(w.end(), r.slot.begin(), r.slot.end());
    std::string key = arch;
    key.append(reinterpret_cast<const char *>(w.data()), w.size() * sizeof(int32_t));
    keys.push_back(std::move(key));
    idx.push_back(i);
  }
  std::vector<cudaKernel_t> ks;
  kernels_for(keys,
              [&reqs, &idx](size_t k) {
                const JitRequest &r = reqs[idx[k]];
                return pattern_source(r.na, r.len, r.slot, r.m, r.groups);
              },
              ks);
  int ok = 0;
  for (size_t k = 0; k < idx.size(); ++k) {
    reqs[idx[k]].kernel = reinterpret_cast<void *>(ks[k]);
    ok += ks[k] != nullptr;
  }
  return ok;
}

std::vector<std::pair<int, int>> jit_groups(int na, const int *len, const int32_t *span,
                                            int32_t max_span, int32_t *stage_need) {
  std::vector<std::pair<int, int>> groups;
  int32_t need = 0;
  auto at = [&](int j0, int g) { return span[j0 * kJitMaxGroup + g - 1]; };
  for (int j = 0; j < na;) {
    if (len[j] == 0) {
      ++j;
      continue;
    }
    int g = 1;
    // grow the group while the next nonempty A nonzero adds less than half
    // of its own span to the union
    while (g < kJitMaxGroup && j + g < na) {
      if (len[j + g] == 0) {
        ++g;
        continue;
      }
      const int32_t cur = at(j, g), nxt = at(j, g + 1), own = at(j + g, 1);
      if (nxt > max_span || 2 * (nxt - cur) > own) break;
      ++g;
    }
    // trailing empty A nonzeros belong to no group
    int end = j + g;
    while (end > j + 1 && len[end - 1] == 0) --end;
    groups.emplace_back(j, end);
    need = need > at(j, end - j) ? need : at(j, end - j);
    j = j + g;
  }
  *stage_need = need;
  return groups;
}

void launch_jit_spans(const int4 *tiles, int32_t ntiles, const int4 *desc, const uint16_t *lens,
                      const int32_t *a_rp, const int32_t *a_col, const int32_t *b_rp,
                      int32_t *span, int num_sms, cudaStream_t s) {
  if (ntiles <= 0) return;
  // a sample of at most about 1024 tiles spread over the list
  const int32_t stride = ntiles > 1024 ? ntiles / 1024 : 1;
  const int64_t sampled = (int64_t(ntiles) + stride - 1) / stride;
  int64_t grid = (sampled + kBuildWarps - 1) / kBuildWarps;
  const int64_t cap = int64_t(num_sms > 0 ? num_sms : 148) * 8;
  if (grid > cap) grid = cap;
  span_kernel<<<static_cast<unsigned>(grid), kBuildWarps * 32, 0, s>>>(
      tiles, ntiles, stride, desc, lens, a_rp, a_col, b_rp, span);
}

void launch_mark_pattern(int4 *desc, int32_t pid, cudaStream_t s) {
  mark_pattern_kernel<<<1, 1, 0, s>>>(desc, pid);
}

void launch_table_tiles(const int4 *tiles, int32_t ntiles, const int4 *desc, int4 *out,
                        int32_t *n, cudaStream_t s) {
  if (ntiles <= 0) return;
  table_tiles_kernel<<<(ntiles + 255) / 256, 256, 0, s>>>(tiles, ntiles, desc, out, n);
}

int32_t jit_record_words(int na, int ngroups) { return record_words(na, ngroups); }

void launch_jit_programs(const int4 *tiles, int32_t ntiles, int32_t na,
                         const std::vector<std::pair<int, int>> &groups, const int2 *groups_dev,
                         const uint16_t *lens, const int32_t *a_rp, const int32_t *a_col,
                         const int32_t *b_rp, int32_t *prog, int2 *arange, int32_t *maxima,
                         int num_sms, cudaStream_t s) {
  if (ntiles <= 0) return;
  const int32_t rw = record_words(na, static_cast<int>(groups.size()));
  cudaMemsetAsync(prog, 0, size_t(ntiles) * size_t(rw) * sizeof(int32_t), s);
  int64_t grid = (int64_t(ntiles) + kBuildWarps - 1) / kBuildWarps;
  const int64_t cap = int64_t(num_sms > 0 ? num_sms : 148) * 8;
  if (grid > cap) grid = cap;
  program_kernel<<<static_cast<unsigned>(grid), kBuildWarps * 32, 0, s>>>(
      tiles, ntiles, na, static_cast<int32_t>(groups.size()), groups_dev, lens, a_rp, a_col,
      b_rp, rw, prog, arange, maxima);
}

void jit_layout(int32_t rw, int32_t seg_max, int32_t need, int32_t m, int32_t *stage_cap,
                int32_t *abuf_floats, int32_t *work_floats) {
  const int32_t ms = (m & 1) ? m : m + 1;
  // a tile buffer: the record, then A values widened by up to 3 floats at
  // each end; a stage buffer: a B range widened the same way
  const int32_t ab = (rw + seg_max + 8 + 3) & ~3;
  int32_t sc = (need + 8 + 3) & ~3;
  // the output region (one tile buffer and both stage buffers) holds 16 rows
  if (ab + 2 * sc < 16 * ms + 4) sc = ((16 * ms + 4 - ab + 1) / 2 + 3) & ~3;
  *stage_cap = sc;
  *abuf_floats = ab;
  *work_floats = 2 * ab + 2 * sc;
}

int jit_grid(void *kernel, int32_t ntiles, int32_t work_floats, int32_t m, int num_sms) {
  (void)kernel;
  // registers: a quarter of the SM's file per scheduler, 256-register units
  // per warp; shared memory: the SM's total with 1 KB reserved per block
  const int warp_regs = ((pattern_regs(m) * 32) + 255) & ~255;
  const int by_regs = (4 * (16384 / warp_regs)) / (kJitThreads / 32);
  int dev = 0, sm_bytes = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sm_bytes, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev);
  const size_t block_bytes =
      size_t(kJitThreads / 32) * size_t(work_floats) * sizeof(float) + 64 + 1024;
  int by_smem = sm_bytes > 0 ? static_cast<int>(size_t(sm_bytes) / block_bytes) : 1;
  int per_sm = by_regs < by_smem ? by_regs : by_smem;
  if (per_sm < 1) per_sm = 1;
  if (per_sm > 16) per_sm = 16;
  const int64_t want = (int64_t(ntiles) + 1) / 2;
  const int64_t cap = int64_t(num_sms > 0 ? num_sms : 148) * per_sm;
  return static_cast<int>(want < cap ? want : cap);
}

cudaError_t launch_pattern_kernel(void *kernel, const Operands &op, const int32_t *prog,
                                  const int2 *arange, int32_t ntiles, const int32_t *c_rp,
                                  float *c_val, int32_t stage_cap, int32_t abuf_floats,
                                  int32_t work_floats, int grid, int32_t *head,
                                  int32_t *status, cudaStream_t s) {
  if (ntiles <= 0 || grid <= 0) return cudaSuccess;
  cudaError_t e = cudaMemsetAsync(head, 0, sizeof(int32_t), s);
  if (e != cudaSuccess) return e;
  const size_t smem = size_t(kJitThreads / 32) * size_t(work_floats) * sizeof(float);
  int dev = 0;
  cudaGetDevice(&dev);
  cudaKernel_t k = reinterpret_cast<cudaKernel_t>(kernel);
  e = cudaKernelSetAttributeForDevice(
      k, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem), dev);
  if (e != cudaSuccess) return e;
  float zero = 0.0f;
  const int32_t *pr = prog;
  const int2 *ar = arange;
  int32_t nt = ntiles;
  const float *a_val = op.a_val, *b_val = op.b_val;
  int32_t sc = stage_cap, abf = abuf_floats, wf = work_floats;
  int32_t *hd = head, *st = status;
  void *args[] = {&pr, &ar, &nt, &a_val, &b_val, &c_rp, &c_val, &sc, &abf, &wf, &zero, &hd, &st};
  return cudaLaunchKernel(reinterpret_cast<const void *>(k), dim3(static_cast<unsigned>(grid)),
                          dim3(kJitThreads), args, smem, s);
}

}  // namespace rvsp
