// The row-binning MLP: features, inference, and training on the GPU.
//
// Network: 8 row features -> 32 (ReLU) -> 32 (ReLU) -> 2, FP32, CUDA cores
// (1.4 k parameters; nothing here is big enough for tensor cores).
//   output 0: predicted log2(1 + nnz of the output row)
//   output 1: logit of the accumulator class (1 = the merge kernel is the
//             faster accumulator for this row, 0 = the warp hash)
// Loss per sample: (y0 - t0)^2 + BCE(sigmoid(y1), t1), averaged over the
// batch.  Training is Adam over mini-batches; every kernel is hand-written:
// mlp_forward_train_kernel (activations), mlp_backward_kernel (gradients,
// reduced per block and added with atomics), mlp_adam_kernel (update).
//
// Features of row i (all from A's structure and B's row pointers / first and
// last columns; log2(1 + x) each):
//   f0 nnz(A row)       f1 ops = sum |B row k|       f2 max |B row k|
//   f3 ops / nnz        f4 column span of the row's products (last - first + 1)
//   f5 min(ops, span)   f6 b_cols                   f7 mean |B row| of B
// Inputs are standardised with the per-feature mean and standard deviation
// stored in the model (set from the training data, not trained).
#include <cuda_runtime.h>

#include <cmath>
#include <climits>
#include <cstdint>

#include "device_common.cuh"
#include "kernels.cuh"

namespace rvsp {

namespace {

constexpr int kThreads = 256;

__device__ __forceinline__ float lg(float x) { return log2f(1.0f + x); }

// Features of one row, reduced over the row's A nonzeros by one warp.
// Returns, on every lane, the 8 raw features; also ops (int64) and ub.
struct RowFeat {
  float f[kMlpIn];
  long long ops;
};

__device__ __forceinline__ RowFeat warp_row_features(const Operands &op, int32_t row,
                                                      float b_mean_len) {
  const int lane = lane_id();
  const int32_t p0 = op.a_rp[row], p1 = op.a_rp[row + 1];
  long long ops = 0;
  int maxlen = 0, lo = INT_MAX, hi = -1;
  for (int32_t p = p0 + lane; p < p1; p += 32) {
    const int32_t k = __ldg(op.a_col + p);
    const int32_t b0 = __ldg(op.b_rp + k), b1 = __ldg(op.b_rp + k + 1);
    const int len = b1 - b0;
    ops += len;
    maxlen = max(maxlen, len);
    if (len > 0) {
      lo = min(lo, __ldg(op.b_col + b0));
      hi = max(hi, __ldg(op.b_col + b1 - 1));
    }
  }
  ops = warp_sum64(ops);
  maxlen = warp_max(maxlen);
  lo = warp_min(lo);
  hi = warp_max(hi);
  RowFeat r;
  const float nnz = static_cast<float>(p1 - p0);
  const float fops = static_cast<float>(ops);
  const float span = hi >= lo ? static_cast<float>(hi - lo + 1) : 0.0f;
  r.f[0] = lg(nnz);
  r.f[1] = lg(fops);
  r.f[2] = lg(static_cast<float>(maxlen));
  r.f[3] = lg(nnz > 0 ? fops / nnz : 0.0f);
  r.f[4] = lg(span);
  r.f[5] = lg(fminf(fops, span));
  r.f[6] = lg(static_cast<float>(op.b_cols));
  r.f[7] = lg(b_mean_len);
  r.ops = ops;
  return r;
}

// y = MLP(x) with the hidden units spread over the 32 lanes (unit j on lane
// j); every lane returns both outputs.  P holds the parameters in the layout
// of MlpLayout (shared memory).
// Copies the parameters into shared memory with W1 and W2 transposed
// (W1T[i][j] at kW1 + i * 32 + j, W2T[k][j] at kW2 + k * 32 + j), so that in
// warp_mlp lane j's reads of row j fall in 32 different banks.
__device__ __forceinline__ void load_params_transposed(float *P,
                                                       const float *__restrict__ params) {
  for (int i = threadIdx.x; i < kMlpParams; i += blockDim.x) {
    float v = params[i];
    int at = i;
    if (i >= kW1 && i < kB1) {
      const int j = (i - kW1) / kMlpIn, c = (i - kW1) % kMlpIn;
      at = kW1 + c * kMlpHidden + j;
    } else if (i >= kW2 && i < kB2) {
      const int j = (i - kW2) / kMlpHidden, c = (i - kW2) % kMlpHidden;
      at = kW2 + c * kMlpHidden + j;
    }
    P[at] = v;
  }
}

// Forward pass of one row on one warp (lane j = hidden unit j), with P laid
// out by load_params_transposed.
__device__ __forceinline__ void warp_mlp(const float *P, const float *x, float &y0,
                                         float &y1) {
  const int j = lane_id();
  float a = P[kB1 + j];
#pragma unroll
  for (int i = 0; i < kMlpIn; ++i) a = fmaf(P[kW1 + i * kMlpHidden + j], x[i], a);
  const float h1 = fmaxf(a, 0.0f);
  float b = P[kB2 + j];
#pragma unroll
  for (int k = 0; k < kMlpHidden; ++k)
    b = fmaf(P[kW2 + k * kMlpHidden + j], __shfl_sync(kFull, h1, k), b);
  const float h2 = fmaxf(b, 0.0f);
  float o0 = P[kW3 + j] * h2;
  float o1 = P[kW3 + kMlpHidden + j] * h2;
#pragma unroll
  for (int s = 16; s > 0; s >>= 1) {
    o0 += __shfl_xor_sync(kFull, o0, s);
    o1 += __shfl_xor_sync(kFull, o1, s);
  }
  y0 = o0 + P[kB3];
  y1 = o1 + P[kB3 + 1];
}

// Training / harvest: raw features of every row (n x 8, row-major) and the
// op counts.  One warp per row.
__global__ void __launch_bounds__(kThreads)
features_kernel(Operands op, float b_mean_len, float *__restrict__ feat,
                int64_t *__restrict__ ops_out) {
  const int warps = (gridDim.x * blockDim.x) >> 5;
  for (int32_t row = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; row < op.a_rows;
       row += warps) {
    const RowFeat r = warp_row_features(op, row, b_mean_len);
    const int lane = lane_id();
    if (lane < kMlpIn) feat[size_t(row) * kMlpIn + lane] = r.f[lane];
    if (lane == 0 && ops_out) ops_out[row] = r.ops;
  }
}

// Inference: features -> standardise -> MLP -> per-row prediction.
// pred[row] = (y0, y1); ops[row] = op count.
__global__ void __launch_bounds__(kThreads)
predict_kernel(Operands op, float b_mean_len, const float *__restrict__ params,
               float2 *__restrict__ pred, int64_t *__restrict__ ops_out) {
  __shared__ float P[kMlpParamsPad];
  load_params_transposed(P, params);
  __syncthreads();
  const int warps = (gridDim.x * blockDim.x) >> 5;
  for (int32_t row = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; row < op.a_rows;
       row += warps) {
    const RowFeat r = warp_row_features(op, row, b_mean_len);
    float x[kMlpIn];
#pragma unroll
    for (int i = 0; i < kMlpIn; ++i) x[i] = (r.f[i] - P[kMu + i]) * P[kInvSd + i];
    float y0, y1;
    warp_mlp(P, x, y0, y1);
    if (lane_id() == 0) {
      pred[row] = make_float2(y0, y1);
      if (ops_out) ops_out[row] = r.ops;
    }
  }
}

// Learned binning of every row for the fused pass (one warp per row):
// features -> MLP -> (class, slab capacity).
//   no products                          EMPTY, capacity 0, counts[row] = 0
//   merge-eligible and output 1 > 0      M<K>, capacity = ops (exact bound)
//   otherwise                            capacity = min(ub, ceil(scale *
//     (2^y0 - 1)) + kCapPad) with ub = min(ops, b_cols); warp hash with
//     T >= 2 capacity slots up to 2048, the 8192-slot block hash up to 4096,
//     else DENSE with capacity ub (never overflows).
// A row whose nnz exceeds its capacity is caught by the fused kernel and
// redone by the plain two-pass path.
constexpr int kCapPad = 16;
constexpr int kThreadRowNnz = 32;  // rows up to this many A nonzeros: a thread each

__global__ void __launch_bounds__(kThreads)
learned_plan_kernel(Operands op, float b_mean_len, const float *__restrict__ params,
                    float scale, bool merge_ok, int64_t *__restrict__ ops_out,
                    uint8_t *__restrict__ cls_out, int32_t *__restrict__ cap_out,
                    int32_t *__restrict__ counts, int32_t *__restrict__ class_count) {
  __shared__ float P[kMlpParamsPad];
  __shared__ int32_t s_cnt[kNumClasses];
  load_params_transposed(P, params);
  for (int c = threadIdx.x; c < kNumClasses; c += blockDim.x) s_cnt[c] = 0;
  __syncthreads();
  auto decide = [&](int32_t row, int32_t nnz, long long ops, float y0, float y1) {
    const long long ub = ops < op.b_cols ? ops : op.b_cols;
    int c;
    long long cap;
    if (ops == 0) {
      c = kEmpty_;
      cap = 0;
      counts[row] = 0;
    } else if (merge_ok && nnz <= kMergeMaxNnz && ops <= kMergeMaxOps && y1 > 0.0f) {
      c = nnz <= 4 ? kM4 : nnz <= 8 ? kM8 : kM16;
      cap = ops;
    } else {
      const float mhat = exp2f(fminf(y0, 40.0f)) - 1.0f;
      const float want = ceilf(scale * fmaxf(mhat, 0.0f)) + kCapPad;
      cap = want >= static_cast<float>(ub) ? ub : static_cast<long long>(want);
      if (cap < 1) cap = 1;
      c = classify_row(nnz, ops, cap, false);
      if (c == kDense) cap = ub;
    }
    ops_out[row] = ops;
    cls_out[row] = static_cast<uint8_t>(c);
    cap_out[row] = static_cast<int32_t>(cap);
    atomicAdd(&s_cnt[c], 1);
  };
  // Rows of at most kThreadRowNnz A nonzeros: one thread each, features and
  // MLP in registers (every thread reads the same weight at the same time, a
  // shared-memory broadcast).  Their loads all start at once instead of one
  // row after another on a warp.
  const int32_t tstride = gridDim.x * blockDim.x;
  for (int32_t row = blockIdx.x * blockDim.x + threadIdx.x; row < op.a_rows; row += tstride) {
    const int32_t p0 = op.a_rp[row], p1 = op.a_rp[row + 1];
    if (p1 - p0 > kThreadRowNnz) continue;
    long long ops = 0;
    int maxlen = 0, lo = INT_MAX, hi = -1;
    for (int32_t p = p0; p < p1; ++p) {
      const int32_t k = __ldg(op.a_col + p);
      const int32_t b0 = __ldg(op.b_rp + k), b1 = __ldg(op.b_rp + k + 1);
      const int len = b1 - b0;
      ops += len;
      maxlen = max(maxlen, len);
      if (len > 0) {
        lo = min(lo, __ldg(op.b_col + b0));
        hi = max(hi, __ldg(op.b_col + b1 - 1));
      }
    }
    const float nnz = static_cast<float>(p1 - p0), fops = static_cast<float>(ops);
    const float span = hi >= lo ? static_cast<float>(hi - lo + 1) : 0.0f;
    float f[kMlpIn] = {lg(nnz), lg(fops), lg(static_cast<float>(maxlen)),
                       lg(nnz > 0 ? fops / nnz : 0.0f), lg(span), lg(fminf(fops, span)),
                       lg(static_cast<float>(op.b_cols)), lg(b_mean_len)};
#pragma unroll
    for (int i = 0; i < kMlpIn; ++i) f[i] = (f[i] - P[kMu + i]) * P[kInvSd + i];
    float h1[kMlpHidden];
#pragma unroll
    for (int j = 0; j < kMlpHidden; ++j) {
      float a = P[kB1 + j];
#pragma unroll
      for (int i = 0; i < kMlpIn; ++i) a = fmaf(P[kW1 + i * kMlpHidden + j], f[i], a);
      h1[j] = fmaxf(a, 0.0f);
    }
    float y0 = P[kB3], y1 = P[kB3 + 1];
#pragma unroll 4
    for (int j = 0; j < kMlpHidden; ++j) {
      float b = P[kB2 + j];
#pragma unroll
      for (int k = 0; k < kMlpHidden; ++k) b = fmaf(P[kW2 + k * kMlpHidden + j], h1[k], b);
      const float h2 = fmaxf(b, 0.0f);
      y0 = fmaf(P[kW3 + j], h2, y0);
      y1 = fmaf(P[kW3 + kMlpHidden + j], h2, y1);
    }
    decide(row, p1 - p0, ops, y0, y1);
  }
  // Longer rows: one warp each (features over the lanes, hidden unit j on
  // lane j), found 32 rows at a time.
  const int32_t wstride = tstride >> 5;
  const int lane = lane_id();
  for (int32_t base = ((blockIdx.x * blockDim.x + threadIdx.x) >> 5) * 32; base < op.a_rows;
       base += wstride * 32) {
    const int32_t mine = base + lane;
    const bool longrow =
        mine < op.a_rows && op.a_rp[mine + 1] - op.a_rp[mine] > kThreadRowNnz;
    unsigned todo = __ballot_sync(kFull, longrow);
    while (todo) {
      const int32_t row = base + __ffs(todo) - 1;
      todo &= todo - 1u;
      const RowFeat r = warp_row_features(op, row, b_mean_len);
      float x[kMlpIn];
#pragma unroll
      for (int i = 0; i < kMlpIn; ++i) x[i] = (r.f[i] - P[kMu + i]) * P[kInvSd + i];
      float y0, y1;
      warp_mlp(P, x, y0, y1);
      if (lane == 0) decide(row, op.a_rp[row + 1] - op.a_rp[row], r.ops, y0, y1);
    }
  }
  __syncthreads();
  for (int c = threadIdx.x; c < kNumClasses; c += blockDim.x)
    if (s_cnt[c]) atomicAdd(&class_count[c], s_cnt[c]);
}

// ---- training ----------------------------------------------------------------
// One block per tile of kTile samples.  The tile's activations live in
// shared memory and every step is a small matrix product over the tile:
//   forward   H1 = relu(X W1^T + b1), H2 = relu(H1 W2^T + b2), Y = H2 W3^T + b3
//   dL/dY     dY0 = 2 (y0 - t0) / N,  dY1 = (sigmoid(y1) - t1) / N
//   backward  D2 = (dY W3) . [H2 > 0],  D1 = (D2 W2) . [H1 > 0]
//   gradients dW3 = dY^T H2, dW2 = D2^T H1, dW1 = D1^T X, db = column sums
// Each gradient entry is summed over the tile by one thread, then added to
// the global gradient (one atomic per entry per block).  N is the batch size.

constexpr int kTile = 64;

__global__ void __launch_bounds__(kThreads)
mlp_grad_kernel(const float *__restrict__ params, const float *__restrict__ feat,
                const float *__restrict__ target, int32_t n, int32_t n_total,
                float *__restrict__ grad, float *__restrict__ loss_sum) {
  __shared__ float P[kMlpParamsPad];
  __shared__ float X[kTile][kMlpIn];
  __shared__ float H1[kTile][kMlpHidden + 1];
  __shared__ float H2[kTile][kMlpHidden + 1];
  __shared__ float D1[kTile][kMlpHidden + 1];
  __shared__ float D2[kTile][kMlpHidden + 1];
  __shared__ float DY[kTile][kMlpOut];
  __shared__ float s_loss;
  const int tid = threadIdx.x;
  for (int i = tid; i < kMlpParamsPad; i += blockDim.x)
    P[i] = i < kMlpParams ? params[i] : 0.0f;
  if (tid == 0) s_loss = 0.0f;
  const int32_t base = blockIdx.x * kTile;
  const int cnt = min(kTile, n - base);
  __syncthreads();
  for (int e = tid; e < kTile * kMlpIn; e += blockDim.x) {
    const int s = e / kMlpIn, i = e % kMlpIn;
    X[s][i] = s < cnt ? (feat[size_t(base + s) * kMlpIn + i] - P[kMu + i]) * P[kInvSd + i]
                      : 0.0f;
  }
  __syncthreads();
  for (int e = tid; e < kTile * kMlpHidden; e += blockDim.x) {
    const int s = e / kMlpHidden, j = e % kMlpHidden;
    float a = P[kB1 + j];
#pragma unroll
    for (int i = 0; i < kMlpIn; ++i) a = fmaf(P[kW1 + j * kMlpIn + i], X[s][i], a);
    H1[s][j] = fmaxf(a, 0.0f);
  }
  __syncthreads();
  for (int e = tid; e < kTile * kMlpHidden; e += blockDim.x) {
    const int s = e / kMlpHidden, j = e % kMlpHidden;
    float b = P[kB2 + j];
#pragma unroll
    for (int k = 0; k < kMlpHidden; ++k) b = fmaf(P[kW2 + j * kMlpHidden + k], H1[s][k], b);
    H2[s][j] = fmaxf(b, 0.0f);
  }
  __syncthreads();
  const float inv_n = 1.0f / static_cast<float>(n_total);
  if (tid < kTile) {
    const int s = tid;
    float d0 = 0.0f, d1 = 0.0f, l = 0.0f;
    if (s < cnt) {
      float y0 = P[kB3], y1 = P[kB3 + 1];
#pragma unroll
      for (int j = 0; j < kMlpHidden; ++j) {
        y0 = fmaf(P[kW3 + j], H2[s][j], y0);
        y1 = fmaf(P[kW3 + kMlpHidden + j], H2[s][j], y1);
      }
      const float t0 = target[2 * size_t(base + s)], t1 = target[2 * size_t(base + s) + 1];
      const float e0 = y0 - t0;
      // stable BCE-with-logits: log(1 + exp(-|y|)) + max(y, 0) - y t
      l = e0 * e0 + log1pf(expf(-fabsf(y1))) + fmaxf(y1, 0.0f) - y1 * t1;
      d0 = 2.0f * e0 * inv_n;
      d1 = (1.0f / (1.0f + expf(-y1)) - t1) * inv_n;
    }
    DY[s][0] = d0;
    DY[s][1] = d1;
    l = warp_sum_f(l);
    if (lane_id() == 0) atomicAdd(&s_loss, l * inv_n);
  }
  __syncthreads();
  for (int e = tid; e < kTile * kMlpHidden; e += blockDim.x) {
    const int s = e / kMlpHidden, j = e % kMlpHidden;
    const float g = DY[s][0] * P[kW3 + j] + DY[s][1] * P[kW3 + kMlpHidden + j];
    D2[s][j] = H2[s][j] > 0.0f ? g : 0.0f;
  }
  __syncthreads();
  for (int e = tid; e < kTile * kMlpHidden; e += blockDim.x) {
    const int s = e / kMlpHidden, k = e % kMlpHidden;
    float g = 0.0f;
#pragma unroll
    for (int j = 0; j < kMlpHidden; ++j) g = fmaf(P[kW2 + j * kMlpHidden + k], D2[s][j], g);
    D1[s][k] = H1[s][k] > 0.0f ? g : 0.0f;
  }
  __syncthreads();
  for (int q = tid; q < kMlpTrained; q += blockDim.x) {
    float acc = 0.0f;
    if (q < kB1) {  // W1[k][i]
      const int k = q / kMlpIn, i = q % kMlpIn;
      for (int s = 0; s < cnt; ++s) acc = fmaf(D1[s][k], X[s][i], acc);
    } else if (q < kW2) {  // b1[k]
      const int k = q - kB1;
      for (int s = 0; s < cnt; ++s) acc += D1[s][k];
    } else if (q < kB2) {  // W2[j][k]
      const int j = (q - kW2) / kMlpHidden, k = (q - kW2) % kMlpHidden;
      for (int s = 0; s < cnt; ++s) acc = fmaf(D2[s][j], H1[s][k], acc);
    } else if (q < kW3) {  // b2[j]
      const int j = q - kB2;
      for (int s = 0; s < cnt; ++s) acc += D2[s][j];
    } else if (q < kB3) {  // W3[o][j]
      const int o = (q - kW3) / kMlpHidden, j = (q - kW3) % kMlpHidden;
      for (int s = 0; s < cnt; ++s) acc = fmaf(DY[s][o], H2[s][j], acc);
    } else {  // b3[o]
      const int o = q - kB3;
      for (int s = 0; s < cnt; ++s) acc += DY[s][o];
    }
    atomicAdd(&grad[q], acc);
  }
  if (tid == 0) atomicAdd(loss_sum, s_loss);
}

// Adam on the trained parameters [0, kMlpTrained); step is 1-based.
__global__ void mlp_adam_kernel(float *__restrict__ params,
                                const float *__restrict__ grad,
                                float *__restrict__ m, float *__restrict__ v,
                                float lr, float b1, float b2, float eps, int step) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= kMlpTrained) return;
  const float g = grad[i];
  const float mi = b1 * m[i] + (1.0f - b1) * g;
  const float vi = b2 * v[i] + (1.0f - b2) * g * g;
  m[i] = mi;
  v[i] = vi;
  const float mh = mi / (1.0f - powf(b1, static_cast<float>(step)));
  const float vh = vi / (1.0f - powf(b2, static_cast<float>(step)));
  params[i] -= lr * mh / (sqrtf(vh) + eps);
}

}  // namespace

void launch_features(const Operands &op, float b_mean_len, float *feat,
                     int64_t *ops, int num_sms, cudaStream_t s) {
  const int grid = num_sms * 8;
  features_kernel<<<grid, kThreads, 0, s>>>(op, b_mean_len, feat, ops);
}

void launch_predict(const Operands &op, float b_mean_len, const float *params,
                    float2 *pred, int64_t *ops, int num_sms, cudaStream_t s) {
  const int grid = num_sms * 8;
  predict_kernel<<<grid, kThreads, 0, s>>>(op, b_mean_len, params, pred, ops);
}

void launch_learned_plan(const Operands &op, float b_mean_len, const float *params,
                         float scale, bool merge_ok, int64_t *ops, uint8_t *cls,
                         int32_t *cap, int32_t *counts, int32_t *class_count,
                         int num_sms, cudaStream_t s) {
  const int grid = num_sms * 8;
  learned_plan_kernel<<<grid, kThreads, 0, s>>>(op, b_mean_len, params, scale, merge_ok,
                                                ops, cls, cap, counts, class_count);
}

void launch_mlp_grad(const float *params, const float *feat, const float *target,
                     int32_t n, int32_t n_total, float *grad, float *loss_sum,
                     cudaStream_t s) {
  const int grid = (n + kTile - 1) / kTile;
  mlp_grad_kernel<<<grid, kThreads, 0, s>>>(params, feat, target, n, n_total, grad,
                                            loss_sum);
}

void launch_mlp_adam(float *params, const float *grad, float *m, float *v, float lr,
                     float b1, float b2, float eps, int step, cudaStream_t s) {
  mlp_adam_kernel<<<(kMlpTrained + 255) / 256, 256, 0, s>>>(params, grad, m, v, lr,
                                                            b1, b2, eps, step);
}

}  // namespace rvsp
