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
// multiply and an add:
//
//   for each A nonzero j (ascending, unrolled): stage the lanes' B span (as in
//   k_tile.cu, two buffers, cp.async);  c[q(j,e)] = fl(c[q(j,e)] + fl(a_j * b))
//   for every entry e of B row k_j (unrolled, q(j,e) a constant);
//
// and the rows go to C through shared memory in coalesced chunks of 32
// positions.  Accumulators start from a run-time +0.0f (a kernel argument,
// so no compiler can fold 0 + p to p: +0 + -0 must give +0) and every
// product and sum is rounded separately (__fmul_rn, __fadd_rn, -fmad=false),
// in ascending A-nonzero order: the reference's order and rounding
// (gustavson_core_f32.inc:31-62, accum_scalar_f32.c:20-71), so values equal
// the table kernel's bit for bit.
//
// NVRTC is opened at run time (dlopen of libnvrtc.so.12); without it, or if
// a compile fails, the pattern stays on the table kernel.  Compiled kernels
// are kept for the life of the process, keyed by their source text, so a
// pattern is compiled once per process.
#include <cuda_runtime.h>
#include <dlfcn.h>
#include <nvrtc.h>

#include <chrono>
#include <cstdio>
#include <map>
#include <mutex>
#include <string>
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
std::map<std::string, cudaKernel_t> g_cache;  // source text -> kernel
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
const char *kPrelude = R"(
typedef unsigned int u32;
#define FULL 0xffffffffu
__device__ __forceinline__ void cpa16(float *s, const float *g) {
  const u32 a = (u32)__cvta_generic_to_shared(s);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(a), "l"(g) : "memory");
}
__device__ __forceinline__ void cpa4(float *s, const float *g) {
  const u32 a = (u32)__cvta_generic_to_shared(s);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(a), "l"(g) : "memory");
}
__device__ __forceinline__ void cpa_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cpa_wait1() { asm volatile("cp.async.wait_group 1;\n" ::: "memory"); }
__device__ __forceinline__ void cpa_wait0() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }
// B values [lo, hi) into dst; returns the B index dst[0] stands for.
__device__ __forceinline__ int stage_span(float *dst, const float *__restrict__ b_val, int lo,
                                          int hi, int b_nnz, bool al, int lane) {
  if (al) {
    const int c0 = lo & ~3;
    const int chunks = (hi - c0 + 3) >> 2;
    for (int c = lane; c < chunks; c += 32) {
      const int g = c0 + 4 * c;
      if (g + 4 <= b_nnz) cpa16(dst + 4 * c, b_val + g);
      else for (int x = g; x < hi; ++x) cpa4(dst + (x - c0), b_val + x);
    }
    return c0;
  }
  for (int x = lo + lane; x < hi; x += 32) cpa4(dst + (x - lo), b_val + x);
  return lo;
}
)";

// Source of the kernel for one pattern: na A nonzeros with B row lengths
// len[j], slot[t] the output position of flattened product t, m outputs.
std::string pattern_source(int na, const int *len, const std::vector<int> &slot, int m) {
  std::string s(kPrelude);
  char buf[1024];
  s += "extern \"C\" __global__ void __launch_bounds__(64)\n"
       "rvsp_pattern_tiles(const int4 *__restrict__ tiles, int ntiles,\n"
       "    const int *__restrict__ a_rp, const int *__restrict__ a_col,\n"
       "    const float *__restrict__ a_val, const int *__restrict__ b_rp,\n"
       "    const float *__restrict__ b_val, int b_nnz, const int *__restrict__ c_rp,\n"
       "    float *__restrict__ c_val, int stage_cap, int work_floats, float zero) {\n"
       "  extern __shared__ __align__(16) float sm[];\n"
       "  const int wib = threadIdx.x >> 5, lane = threadIdx.x & 31;\n"
       "  float *const work = sm + wib * work_floats;\n"
       "  const int w = blockIdx.x * 2 + wib;\n"
       "  if (w >= ntiles) return;\n"
       "  const int4 t = tiles[w];\n"
       "  const int row0 = t.x;\n"
       "  const u32 mask = (u32)t.y;\n"
       "  const bool active = (mask >> lane) & 1u;\n"
       "  const int row = row0 + lane;\n"
       "  const bool al = (((unsigned long long)b_val) & 15ull) == 0;\n"
       "  const int seg0 = a_rp[row0];\n"
       "  int my_p = 0, cs = 0;\n"
       "  if (active) { my_p = a_rp[row] - seg0; cs = c_rp[row]; }\n"
       "  const int seg = a_rp[__reduce_max_sync(FULL, active ? row : row0) + 1] - seg0;\n"
       "  {\n"
       "    int *scol = (int *)work; float *sval = work + seg;\n"
       "    for (int i = lane; i < seg; i += 32) {\n"
       "      scol[i] = __ldg(a_col + seg0 + i); sval[i] = __ldg(a_val + seg0 + i);\n"
       "    }\n"
       "  }\n"
       "  __syncwarp();\n";
  snprintf(buf, sizeof(buf), "  float av[%d]; int rp[%d];\n", na, na);
  s += buf;
  snprintf(buf, sizeof(buf),
           "  {\n    const int *scol = (const int *)work; const float *sval = work + seg;\n"
           "#pragma unroll\n    for (int j = 0; j < %d; ++j) {\n"
           "      av[j] = 0.0f; rp[j] = 0;\n"
           "      if (active) { av[j] = sval[my_p + j]; rp[j] = __ldg(b_rp + scol[my_p + j]); }\n"
           "    }\n  }\n  __syncwarp();\n",
           na);
  s += buf;
  // accumulators
  for (int q = 0; q < m; ++q) {
    snprintf(buf, sizeof(buf), "  float c%d = zero;\n", q);
    s += buf;
  }
  s += "  int cb0 = 0, cb1 = 0;\n";
  snprintf(buf, sizeof(buf),
           "  { const int lo = __reduce_min_sync(FULL, active ? rp[0] : 0x7fffffff);\n"
           "    const int hi = __reduce_max_sync(FULL, active ? rp[0] + %d : (int)0x80000000);\n"
           "    cb0 = stage_span(work, b_val, lo, hi, b_nnz, al, lane); cpa_commit(); }\n",
           len[0]);
  s += buf;
  int t0 = 0;
  for (int j = 0; j < na; ++j) {
    s += "  {\n";
    if (j + 1 < na) {
      snprintf(buf, sizeof(buf),
               "    const int lo = __reduce_min_sync(FULL, active ? rp[%d] : 0x7fffffff);\n"
               "    const int hi = __reduce_max_sync(FULL, active ? rp[%d] + %d : (int)0x80000000);\n"
               "    cb%d = stage_span(work + %d * stage_cap, b_val, lo, hi, b_nnz, al, lane);\n"
               "    cpa_commit(); cpa_wait1();\n",
               j + 1, j + 1, len[j + 1], (j + 1) & 1, (j + 1) & 1);
      s += buf;
    } else {
      s += "    cpa_wait0();\n";
    }
    snprintf(buf, sizeof(buf),
             "    __syncwarp();\n"
             "    const float *st = work + %d * stage_cap + (active ? rp[%d] - cb%d : 0);\n"
             "    const float a = av[%d];\n",
             j & 1, j, j & 1, j);
    s += buf;
    for (int e = 0; e < len[j]; ++e) {
      const int q = slot[size_t(t0 + e)];
      snprintf(buf, sizeof(buf), "    c%d = __fadd_rn(c%d, __fmul_rn(a, st[%d]));\n", q, q, e);
      s += buf;
    }
    s += "    __syncwarp();\n  }\n";
    t0 += len[j];
  }
  // output: chunks of 32 positions through shared memory, coalesced per row
  for (int q0 = 0; q0 < m; q0 += 32) {
    const int cl = m - q0 < 32 ? m - q0 : 32;
    s += "  {\n";
    for (int q = q0; q < q0 + cl; ++q) {
      snprintf(buf, sizeof(buf), "    work[%d * 33 + lane] = c%d;\n", q - q0, q);
      s += buf;
    }
    snprintf(buf, sizeof(buf),
             "    __syncwarp();\n"
             "    for (int r = 0; r < 32; ++r) {\n"
             "      const int base = __shfl_sync(FULL, cs, r);\n"
             "      if (((mask >> r) & 1u) && lane < %d) c_val[base + %d + lane] = work[lane * 33 + r];\n"
             "    }\n"
             "    __syncwarp();\n  }\n",
             cl, q0);
    s += buf;
  }
  s += "}\n";
  return s;
}

// Compiles (or finds) the kernel of `src`.  Returns nullptr on failure.
cudaKernel_t kernel_for(const std::string &src) {
  std::lock_guard<std::mutex> lock(g_mutex);
  auto it = g_cache.find(src);
  if (it != g_cache.end()) return it->second;
  if (!open_nvrtc()) return nullptr;
  int dev = 0, major = 0, minor = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev);
  cudaDeviceGetAttribute(&minor, cudaDevAttrComputeCapabilityMinor, dev);
  char arch[64];
  snprintf(arch, sizeof(arch), "--gpu-architecture=sm_%d%da", major, minor);
  const auto t0 = std::chrono::steady_clock::now();
  nvrtcProgram prog = nullptr;
  cudaKernel_t k = nullptr;
  if (g_nvrtc.create(&prog, src.c_str(), "rvsp_pattern.cu", 0, nullptr, nullptr) ==
      NVRTC_SUCCESS) {
    const char *opts[] = {arch, "-fmad=false", "--std=c++17", "-default-device"};
    size_t n = 0;
    if (g_nvrtc.compile(prog, 4, opts) == NVRTC_SUCCESS &&
        g_nvrtc.cubin_size(prog, &n) == NVRTC_SUCCESS && n > 0) {
      std::vector<char> bin(n);
      cudaLibrary_t lib = nullptr;
      if (g_nvrtc.cubin(prog, bin.data()) == NVRTC_SUCCESS &&
          cudaLibraryLoadData(&lib, bin.data(), nullptr, nullptr, 0, nullptr, nullptr, 0) ==
              cudaSuccess &&
          cudaLibraryGetKernel(&k, lib, "rvsp_pattern_tiles") != cudaSuccess)
        k = nullptr;
    }
    g_nvrtc.destroy(&prog);
  }
  cudaGetLastError();
  g_compile_ms += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0)
                      .count();
  ++g_compiles;
  g_cache[src] = k;  // a failure is remembered too: the table kernel keeps the pattern
  return k;
}

// tiles of pattern pid, in order (count at *n, zeroed by the caller)
__global__ void __launch_bounds__(256)
tile_select_kernel(const int4 *__restrict__ tiles, int32_t ntiles, int32_t pid,
                   int4 *__restrict__ out, int32_t *__restrict__ n) {
  const int32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  const bool take = i < ntiles && tiles[i].z == pid;
  const unsigned b = __ballot_sync(kFull, take);
  if (!b) return;
  int32_t base = 0;
  if (lane_id() == 0) base = atomicAdd(n, __popc(b));
  base = __shfl_sync(kFull, base, 0);
  if (take) out[base + __popc(b & lanemask_lt())] = tiles[i];
}

// desc[pid].w = 1: the table kernel leaves the pattern's tiles alone.
__global__ void mark_pattern_kernel(int4 *desc, int32_t pid) { desc[pid].w = 1; }

}  // namespace

void jit_stats(int32_t *compiles, double *ms) {
  std::lock_guard<std::mutex> lock(g_mutex);
  if (compiles) *compiles = g_compiles;
  if (ms) *ms = g_compile_ms;
}

int jit_pattern_kernel(int na, const int *len, const std::vector<int> &slot, int m,
                       void **kernel_out) {
  if (na <= 0 || m <= 0) return 0;
  const cudaKernel_t k = kernel_for(pattern_source(na, len, slot, m));
  *kernel_out = reinterpret_cast<void *>(k);
  return k != nullptr;
}

void launch_tile_select(const int4 *tiles, int32_t ntiles, int32_t pid, int4 *out, int32_t *n,
                        cudaStream_t s) {
  if (ntiles <= 0) return;
  tile_select_kernel<<<(ntiles + 255) / 256, 256, 0, s>>>(tiles, ntiles, pid, out, n);
}

void launch_mark_pattern(int4 *desc, int32_t pid, cudaStream_t s) {
  mark_pattern_kernel<<<1, 1, 0, s>>>(desc, pid);
}

cudaError_t launch_pattern_kernel(void *kernel, const Operands &op, int32_t b_nnz,
                                  const int4 *tiles, int32_t ntiles, const int32_t *c_rp,
                                  float *c_val, int32_t stage_cap, int32_t work_floats,
                                  cudaStream_t s) {
  if (ntiles <= 0) return cudaSuccess;
  const size_t smem = size_t(kJitThreads / 32) * size_t(work_floats) * sizeof(float);
  int dev = 0;
  cudaGetDevice(&dev);
  cudaKernel_t k = reinterpret_cast<cudaKernel_t>(kernel);
  cudaError_t e = cudaKernelSetAttributeForDevice(
      k, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem), dev);
  if (e != cudaSuccess) return e;
  float zero = 0.0f;
  const int4 *t = tiles;
  int32_t nt = ntiles;
  const int32_t *a_rp = op.a_rp, *a_col = op.a_col, *b_rp = op.b_rp;
  const float *a_val = op.a_val, *b_val = op.b_val;
  int32_t bn = b_nnz, sc = stage_cap, wf = work_floats;
  void *args[] = {&t, &nt, &a_rp, &a_col, &a_val, &b_rp, &b_val, &bn, &c_rp, &c_val, &sc,
                  &wf, &zero};
  const unsigned grid = static_cast<unsigned>((int64_t(ntiles) + 1) / 2);
  return cudaLaunchKernel(reinterpret_cast<const void *>(k), dim3(grid), dim3(kJitThreads),
                          args, smem, s);
}

}  // namespace rvsp
