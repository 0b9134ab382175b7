// The row-binning model object (rvsp_mlp_t) and its C-ABI: parameters,
// features, gradients, training, inference and the weight file.
//
// File format (little endian): "RVSPMLP1", u32 version = 1, u32 in = 8,
// u32 hidden = 32, u32 out = 2, u32 feature schema = 1, u64 seed, then the
// 1426 float parameters in the layout of kernels.cuh (trained weights, then
// the per-feature mean and 1/sd).
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <new>
#include <vector>

#include "kernels.cuh"
#include "rvsp_cuda.h"

using namespace rvsp;

struct rvsp_mlp {
  float *params = nullptr;  // device, kMlpParamsPad
  float *grad = nullptr;    // device, kMlpTrained
  float *m = nullptr;       // Adam moments
  float *v = nullptr;
  float *loss = nullptr;    // device scalar
  int num_sms = 148;
  uint64_t seed = 0;
  int step = 0;
};

namespace {

constexpr char kMagic[8] = {'R', 'V', 'S', 'P', 'M', 'L', 'P', '1'};
constexpr uint32_t kVersion = 1, kSchema = 1;

rvsp_status_t map_err(cudaError_t e) {
  if (e == cudaSuccess) return RVSP_SUCCESS;
  cudaGetLastError();
  return e == cudaErrorMemoryAllocation ? RVSP_ERROR_ALLOCATION_FAILED : RVSP_ERROR_DEVICE;
}

uint64_t splitmix64(uint64_t &s) {
  uint64_t z = (s += 0x9E3779B97F4A7C15ull);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

// He-uniform initial weights, zero biases, identity standardisation.
void init_params(std::vector<float> &p, uint64_t seed) {
  p.assign(kMlpParamsPad, 0.0f);
  uint64_t s = seed;
  auto uni = [&](float bound) {
    const double u = static_cast<double>(splitmix64(s) >> 11) * (1.0 / 9007199254740992.0);
    return static_cast<float>((2.0 * u - 1.0) * bound);
  };
  const float b1 = std::sqrt(6.0f / kMlpIn), b2 = std::sqrt(6.0f / kMlpHidden);
  for (int i = 0; i < kMlpHidden * kMlpIn; ++i) p[kW1 + i] = uni(b1);
  for (int i = 0; i < kMlpHidden * kMlpHidden; ++i) p[kW2 + i] = uni(b2);
  for (int i = 0; i < kMlpOut * kMlpHidden; ++i) p[kW3 + i] = uni(b2);
  for (int i = 0; i < kMlpIn; ++i) p[kInvSd + i] = 1.0f;
}

float mean_b_row_len(int32_t b_rows, const int32_t *b_row_ptr, cudaStream_t s) {
  int32_t last = 0;
  cudaMemcpyAsync(&last, b_row_ptr + b_rows, sizeof(int32_t), cudaMemcpyDeviceToHost, s);
  cudaStreamSynchronize(s);
  return b_rows > 0 ? static_cast<float>(last) / static_cast<float>(b_rows) : 0.0f;
}

}  // namespace

namespace rvsp {
// Used by the plan's learned path.
const float *mlp_device_params(const rvsp_mlp *m) { return m ? m->params : nullptr; }
float mlp_mean_b_row_len(int32_t b_rows, const int32_t *b_row_ptr, cudaStream_t s) {
  return mean_b_row_len(b_rows, b_row_ptr, s);
}
}  // namespace rvsp

extern "C" {

rvsp_status_t rvsp_mlp_create(rvsp_mlp_t *model, uint64_t seed) {
  if (!model) return RVSP_ERROR_NULL_POINTER;
  *model = nullptr;
  int dev = 0, major = 0, sms = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) {
    cudaGetLastError();
    return RVSP_ERROR_UNSUPPORTED_BACKEND;
  }
  cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (major != 10) return RVSP_ERROR_UNSUPPORTED_BACKEND;
  rvsp_mlp *m = new (std::nothrow) rvsp_mlp();
  if (!m) return RVSP_ERROR_ALLOCATION_FAILED;
  m->num_sms = sms > 0 ? sms : 148;
  m->seed = seed;
  cudaError_t e = cudaMalloc(&m->params, kMlpParamsPad * sizeof(float));
  if (e == cudaSuccess) e = cudaMalloc(&m->grad, kMlpTrained * sizeof(float));
  if (e == cudaSuccess) e = cudaMalloc(&m->m, kMlpTrained * sizeof(float));
  if (e == cudaSuccess) e = cudaMalloc(&m->v, kMlpTrained * sizeof(float));
  if (e == cudaSuccess) e = cudaMalloc(&m->loss, sizeof(float));
  std::vector<float> p;
  init_params(p, seed);
  if (e == cudaSuccess)
    e = cudaMemcpy(m->params, p.data(), kMlpParamsPad * sizeof(float), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemset(m->m, 0, kMlpTrained * sizeof(float));
  if (e == cudaSuccess) e = cudaMemset(m->v, 0, kMlpTrained * sizeof(float));
  if (e != cudaSuccess) {
    rvsp_mlp_destroy(m);
    return map_err(e);
  }
  *model = m;
  return RVSP_SUCCESS;
}

void rvsp_mlp_destroy(rvsp_mlp_t m) {
  if (!m) return;
  cudaFree(m->params);
  cudaFree(m->grad);
  cudaFree(m->m);
  cudaFree(m->v);
  cudaFree(m->loss);
  delete m;
}

rvsp_status_t rvsp_mlp_get_params(rvsp_mlp_t m, float *host_out, int32_t n) {
  if (!m || !host_out) return RVSP_ERROR_NULL_POINTER;
  if (n < kMlpParams) return RVSP_ERROR_INVALID_ARGUMENT;
  return map_err(cudaMemcpy(host_out, m->params, kMlpParams * sizeof(float),
                            cudaMemcpyDeviceToHost));
}

rvsp_status_t rvsp_mlp_set_params(rvsp_mlp_t m, const float *host_in, int32_t n) {
  if (!m || !host_in) return RVSP_ERROR_NULL_POINTER;
  if (n < kMlpParams) return RVSP_ERROR_INVALID_ARGUMENT;
  m->step = 0;
  cudaMemset(m->m, 0, kMlpTrained * sizeof(float));
  cudaMemset(m->v, 0, kMlpTrained * sizeof(float));
  return map_err(cudaMemcpy(m->params, host_in, kMlpParams * sizeof(float),
                            cudaMemcpyHostToDevice));
}

rvsp_status_t rvsp_mlp_features(void *stream, int32_t a_rows, int32_t b_rows,
                                int32_t b_cols, const int32_t *a_row_ptr,
                                const int32_t *a_col_idx, const int32_t *b_row_ptr,
                                const int32_t *b_col_idx, float *features_out,
                                int64_t *op_counts_out) {
  if (!a_row_ptr || !a_col_idx || !b_row_ptr || !b_col_idx || !features_out)
    return RVSP_ERROR_NULL_POINTER;
  if (a_rows <= 0 || b_rows <= 0 || b_cols <= 0) return RVSP_ERROR_INVALID_ARGUMENT;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const Operands op{a_rows, b_cols, a_row_ptr, a_col_idx, nullptr,
                    b_row_ptr, b_col_idx, nullptr};
  launch_features(op, mean_b_row_len(b_rows, b_row_ptr, s), features_out, op_counts_out,
                  sms, s);
  return map_err(cudaGetLastError());
}

rvsp_status_t rvsp_mlp_gradient(rvsp_mlp_t m, void *stream, const float *features,
                                const float *targets, int32_t n, float *grad_host_out,
                                float *loss_out) {
  if (!m || !features || !targets || !grad_host_out || !loss_out)
    return RVSP_ERROR_NULL_POINTER;
  if (n <= 0) return RVSP_ERROR_INVALID_ARGUMENT;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  cudaMemsetAsync(m->grad, 0, kMlpTrained * sizeof(float), s);
  cudaMemsetAsync(m->loss, 0, sizeof(float), s);
  launch_mlp_grad(m->params, features, targets, n, n, m->grad, m->loss, s);
  cudaError_t e = cudaMemcpyAsync(grad_host_out, m->grad, kMlpTrained * sizeof(float),
                                  cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(loss_out, m->loss, sizeof(float), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  return map_err(e);
}

rvsp_status_t rvsp_mlp_train(rvsp_mlp_t m, void *stream, const float *features,
                             const float *targets, int32_t n, int32_t batch,
                             int32_t epochs, float lr, float *loss_history) {
  if (!m || !features || !targets) return RVSP_ERROR_NULL_POINTER;
  if (n <= 0 || batch <= 0 || epochs <= 0 || !(lr > 0.0f)) return RVSP_ERROR_INVALID_ARGUMENT;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  // One loss slot per batch, read back once per epoch.
  const int32_t nbatch = (n + batch - 1) / batch;
  float *batch_loss = nullptr;
  cudaError_t e = cudaMalloc(&batch_loss, size_t(nbatch) * sizeof(float));
  if (e != cudaSuccess) return map_err(e);
  std::vector<float> host_loss(nbatch);
  for (int ep = 0; ep < epochs && e == cudaSuccess; ++ep) {
    cudaMemsetAsync(batch_loss, 0, size_t(nbatch) * sizeof(float), s);
    for (int32_t b = 0; b < nbatch; ++b) {
      const int32_t b0 = b * batch;
      const int32_t nb = n - b0 < batch ? n - b0 : batch;
      cudaMemsetAsync(m->grad, 0, kMlpTrained * sizeof(float), s);
      launch_mlp_grad(m->params, features + size_t(b0) * kMlpIn,
                      targets + size_t(b0) * kMlpOut, nb, nb, m->grad, batch_loss + b, s);
      launch_mlp_adam(m->params, m->grad, m->m, m->v, lr, 0.9f, 0.999f, 1e-8f,
                      ++m->step, s);
    }
    if (loss_history) {
      e = cudaMemcpyAsync(host_loss.data(), batch_loss, size_t(nbatch) * sizeof(float),
                          cudaMemcpyDeviceToHost, s);
      if (e == cudaSuccess) e = cudaStreamSynchronize(s);
      double sum = 0.0;
      for (int32_t b = 0; b < nbatch; ++b) {
        const int32_t nb = n - b * batch < batch ? n - b * batch : batch;
        sum += static_cast<double>(host_loss[b]) * nb;
      }
      loss_history[ep] = static_cast<float>(sum / n);
    }
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e == cudaSuccess) e = cudaGetLastError();
  cudaFree(batch_loss);
  return map_err(e);
}

rvsp_status_t rvsp_mlp_predict(rvsp_mlp_t m, void *stream, int32_t a_rows, int32_t b_rows,
                               int32_t b_cols, const int32_t *a_row_ptr,
                               const int32_t *a_col_idx, const int32_t *b_row_ptr,
                               const int32_t *b_col_idx, float *pred_out) {
  if (!m || !a_row_ptr || !a_col_idx || !b_row_ptr || !b_col_idx || !pred_out)
    return RVSP_ERROR_NULL_POINTER;
  if (a_rows <= 0 || b_rows <= 0 || b_cols <= 0) return RVSP_ERROR_INVALID_ARGUMENT;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const Operands op{a_rows, b_cols, a_row_ptr, a_col_idx, nullptr,
                    b_row_ptr, b_col_idx, nullptr};
  launch_predict(op, mean_b_row_len(b_rows, b_row_ptr, s), m->params,
                 reinterpret_cast<float2 *>(pred_out), nullptr, m->num_sms, s);
  return map_err(cudaGetLastError());
}

rvsp_status_t rvsp_mlp_save(rvsp_mlp_t m, const char *path) {
  if (!m || !path) return RVSP_ERROR_NULL_POINTER;
  std::vector<float> p(kMlpParams);
  rvsp_status_t st = rvsp_mlp_get_params(m, p.data(), kMlpParams);
  if (st != RVSP_SUCCESS) return st;
  FILE *f = std::fopen(path, "wb");
  if (!f) return RVSP_ERROR_INVALID_ARGUMENT;
  const uint32_t hdr[5] = {kVersion, kMlpIn, kMlpHidden, kMlpOut, kSchema};
  bool ok = std::fwrite(kMagic, 1, 8, f) == 8 && std::fwrite(hdr, 4, 5, f) == 5 &&
            std::fwrite(&m->seed, 8, 1, f) == 1 &&
            std::fwrite(p.data(), 4, kMlpParams, f) == size_t(kMlpParams);
  ok = (std::fclose(f) == 0) && ok;
  return ok ? RVSP_SUCCESS : RVSP_ERROR_INVALID_ARGUMENT;
}

rvsp_status_t rvsp_mlp_load(rvsp_mlp_t m, const char *path) {
  if (!m || !path) return RVSP_ERROR_NULL_POINTER;
  FILE *f = std::fopen(path, "rb");
  if (!f) return RVSP_ERROR_INVALID_ARGUMENT;
  char magic[8];
  uint32_t hdr[5];
  uint64_t seed = 0;
  std::vector<float> p(kMlpParams);
  bool ok = std::fread(magic, 1, 8, f) == 8 && std::memcmp(magic, kMagic, 8) == 0 &&
            std::fread(hdr, 4, 5, f) == 5 && hdr[0] == kVersion && hdr[1] == kMlpIn &&
            hdr[2] == kMlpHidden && hdr[3] == kMlpOut && hdr[4] == kSchema &&
            std::fread(&seed, 8, 1, f) == 1 &&
            std::fread(p.data(), 4, kMlpParams, f) == size_t(kMlpParams);
  std::fclose(f);
  if (!ok) return RVSP_ERROR_INVALID_ARGUMENT;
  m->seed = seed;
  return rvsp_mlp_set_params(m, p.data(), kMlpParams);
}

int32_t rvsp_mlp_num_params(void) { return kMlpParams; }

}  // extern "C"
