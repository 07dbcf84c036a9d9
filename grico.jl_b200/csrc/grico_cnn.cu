// C ABI of the learned-smoother network primitives: 3x3x3 convolutions (forward, backward
// data, backward weight), ReLU backward, masked mean squared error and Adam.  All pointers are
// device pointers; every call is asynchronous on the given stream (NULL: the legacy stream).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <mutex>
#include <string>

#include "cnn_kernels.cuh"
#include "cnn_tc.cuh"
#include "grico_host.h"
#include "grico_mg_internal.h"
#include "vector_kernels.cuh"

using namespace grico;

namespace {

cudaStream_t as_stream(void* s) { return static_cast<cudaStream_t>(s); }

bool conv_args_ok(int B, int Ci, int Co, int Z, int Y, int X) {
  return B > 0 && Ci > 0 && Co > 0 && Z > 0 && Y > 0 && X > 0 && B <= 65535 && Co <= 65535 * kConvCo;
}

dim3 conv_grid(int B, int Co, int Z, int Y, int X) {
  const int tiles = ((X + kConvTile - 1) / kConvTile) * ((Y + kConvTile - 1) / kConvTile) *
                    ((Z + kConvTile - 1) / kConvTile);
  return dim3(tiles, (Co + kConvCo - 1) / kConvCo, B);
}

int launch_status(const char* what) {
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    set_error(std::string(what) + ": " + cudaGetErrorString(e));
    return GRICO_ERR_CUDA;
  }
  return GRICO_OK;
}

}  // namespace

// error flag of the tensor-core convolution (an mbarrier wait that gave up); one per device,
// its address resolved on the first call on that device
static __device__ int g_conv_tc_err;

namespace {

std::mutex g_conv_tc_mutex;
int* g_conv_tc_err_ptr[64] = {nullptr};

int conv_tc_err_ptr(int** out) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) {
    cudaGetLastError();
    set_error("tensor-core convolution: no current CUDA device");
    return GRICO_ERR_CUDA;
  }
  std::lock_guard<std::mutex> lock(g_conv_tc_mutex);
  if (!g_conv_tc_err_ptr[dev]) {
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, g_conv_tc_err) != cudaSuccess) {
      set_error(std::string("tensor-core convolution: ") + cudaGetErrorString(cudaGetLastError()));
      return GRICO_ERR_CUDA;
    }
    g_conv_tc_err_ptr[dev] = static_cast<int*>(p);
  }
  *out = g_conv_tc_err_ptr[dev];
  return GRICO_OK;
}

}  // namespace

namespace grico {

int tc_error_flag(int** out) { return conv_tc_err_ptr(out); }

int conv_tc_forward(const void* x, const void* wp, const float* bias, void* y, int out_cf, int B, int Ci, int Co,
                    int Z, int Y, int X, int relu, cudaStream_t st) {
  int* err = nullptr;
  if (int rc = conv_tc_err_ptr(&err)) return rc;
  void (*kern)(const __nv_bfloat16*, const __nv_bfloat16*, const float*, void*, int, int, int, int, int, int, int,
               int, int*) = nullptr;
  switch (Ci) {
    case 16: kern = tc::conv3d_cl_tc<2>; break;
    case 32: kern = tc::conv3d_cl_tc<4>; break;
    case 48: kern = tc::conv3d_cl_tc<6>; break;
    case 64: kern = tc::conv3d_cl_tc<8>; break;
    default: set_error("grico_conv3d_forward_tc: Ci must be 16, 32, 48 or 64"); return GRICO_ERR_INVALID;
  }
  const size_t smem = tc::conv_tc_smem_bytes(Ci, Co);
  if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)) != cudaSuccess ||
      cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout, 100) != cudaSuccess)
    return launch_status("grico_conv3d_forward_tc");
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, tc::kThreads, smem) != cudaSuccess || per_sm < 1)
    return launch_status("grico_conv3d_forward_tc");
  int dev = 0, sms = 1, smem_sm = 0, regs_sm = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev);
  cudaDeviceGetAttribute(&regs_sm, cudaDevAttrMaxRegistersPerMultiprocessor, dev);
  cudaFuncAttributes fa{};
  if (cudaFuncGetAttributes(&fa, kern) == cudaSuccess && fa.numRegs > 0) {
    // the occupancy query can answer 1 for two CTAs that fit (the carveout it assumes); the
    // persistent grid does not rely on co-residency, so take the larger of the two estimates
    const int by_smem = smem_sm / int(smem + fa.sharedSizeBytes + 1024);
    const int by_regs = regs_sm / (fa.numRegs * tc::kThreads);
    per_sm = std::max(per_sm, std::min({by_smem, by_regs, 2048 / tc::kThreads}));
  }
  per_sm = std::max(1, std::min<int>(per_sm, int(512 / tc::conv_tc_tmem_cols(Co))));  // TMEM: 512 columns per SM
  const int ctas = per_sm * sms;
  const int seglen = tc::conv_tc_seglen(B, Z, Y, X, ctas);
  const int64_t items = int64_t(B) * ((Y + tc::kTY - 1) / tc::kTY) * ((X + tc::kTX - 1) / tc::kTX) *
                        ((Z + seglen - 1) / seglen);
  const int grid = int(std::min<int64_t>(items, ctas));
  kern<<<grid, tc::kThreads, smem, st>>>(static_cast<const __nv_bfloat16*>(x), static_cast<const __nv_bfloat16*>(wp),
                                         bias, y, out_cf, B, Co, Z, Y, X, seglen, relu, err);
  return launch_status("grico_conv3d_forward_tc");
}

int conv_tc_pack(const float* w, int Ci, int Co, void* wp, cudaStream_t st) {
  const int n = 27 * Ci * tc::conv_tc_npad(Co);
  tc::conv_tc_pack_weights<<<std::min((n + 255) / 256, 1024), 256, 0, st>>>(w, static_cast<__nv_bfloat16*>(wp), Ci,
                                                                             Co, tc::conv_tc_npad(Co));
  return launch_status("grico_conv3d_pack_weights_tc");
}

}  // namespace grico

namespace {

}  // namespace

extern "C" {

int grico_conv3d_forward(const void* x, int x_bf16, const float* w, const float* bias, void* y, int y_bf16, int B,
                         int Ci, int Co, int Z, int Y, int X, int relu, void* stream) {
  if (!x || !w || !y || !conv_args_ok(B, Ci, Co, Z, Y, X)) {
    set_error("grico_conv3d_forward: invalid argument");
    return GRICO_ERR_INVALID;
  }
  const dim3 grid = conv_grid(B, Co, Z, Y, X);
  cudaStream_t st = as_stream(stream);
  if (!x_bf16 && !y_bf16)
    conv3d_fwd<float, float><<<grid, 512, 0, st>>>(static_cast<const float*>(x), w, bias, static_cast<float*>(y), Ci, Co, Z, Y, X, relu);
  else if (!x_bf16 && y_bf16)
    conv3d_fwd<float, __nv_bfloat16><<<grid, 512, 0, st>>>(static_cast<const float*>(x), w, bias,
                                                           static_cast<__nv_bfloat16*>(y), Ci, Co, Z, Y, X, relu);
  else if (x_bf16 && y_bf16)
    conv3d_fwd<__nv_bfloat16, __nv_bfloat16><<<grid, 512, 0, st>>>(static_cast<const __nv_bfloat16*>(x), w, bias,
                                                                   static_cast<__nv_bfloat16*>(y), Ci, Co, Z, Y, X, relu);
  else
    conv3d_fwd<__nv_bfloat16, float><<<grid, 512, 0, st>>>(static_cast<const __nv_bfloat16*>(x), w, bias,
                                                           static_cast<float*>(y), Ci, Co, Z, Y, X, relu);
  return launch_status("grico_conv3d_forward");
}

// gx = conv^T(gy, w); wt: caller scratch of Co*Ci*27 floats for the flipped, transposed weights
int grico_conv3d_backward_data(const float* gy, const float* w, float* wt, float* gx, int B, int Ci, int Co, int Z,
                               int Y, int X, void* stream) {
  if (!gy || !w || !wt || !gx || !conv_args_ok(B, Co, Ci, Z, Y, X)) {
    set_error("grico_conv3d_backward_data: invalid argument");
    return GRICO_ERR_INVALID;
  }
  cudaStream_t st = as_stream(stream);
  conv3d_flip_transpose<<<64, 256, 0, st>>>(w, wt, Ci, Co);
  conv3d_fwd<float, float><<<conv_grid(B, Ci, Z, Y, X), 512, 0, st>>>(gy, wt, nullptr, gx, Co, Ci, Z, Y, X, 0);
  return launch_status("grico_conv3d_backward_data");
}

int grico_conv3d_backward_weight(const float* x, const float* gy, float* gw, float* gb, int B, int Ci, int Co, int Z,
                                 int Y, int X, void* stream) {
  if (!x || !gy || !gw || !conv_args_ok(B, Ci, Co, Z, Y, X) || Ci > 65535) {
    set_error("grico_conv3d_backward_weight: invalid argument");
    return GRICO_ERR_INVALID;
  }
  conv3d_bwd_weight<<<dim3(Ci, Co), 256, 0, as_stream(stream)>>>(x, gy, gw, gb, B, Ci, Co, Z, Y, X);
  return launch_status("grico_conv3d_backward_weight");
}

int grico_relu_backward(const float* y, float* g, int64_t n, void* stream) {
  if (!y || !g || n < 0) return GRICO_ERR_INVALID;
  if (n == 0) return GRICO_OK;
  relu_backward<<<int(std::min<int64_t>((n + 255) / 256, 148 * 16)), 256, 0, as_stream(stream)>>>(y, g, n);
  return launch_status("grico_relu_backward");
}

// g = d/dp of sum(m (p - t)^2) / count; loss (device double) = that sum / count.
// partial: caller scratch of kRedBlocks doubles.
int grico_mse_grad(const float* p, const float* t, const float* mask, float* g, int64_t n, double count,
                   double* partial, double* loss, void* stream) {
  if (!p || !t || !g || !partial || !loss || n <= 0 || !(count > 0)) return GRICO_ERR_INVALID;
  cudaStream_t st = as_stream(stream);
  mse_grad<<<kRedBlocks, 256, 0, st>>>(p, t, mask, g, n, float(1.0 / count), partial);
  reduce_final<<<1, kRedThreads, 0, st>>>(partial, kRedBlocks, loss);
  scale_scalar<<<1, 1, 0, st>>>(loss, 1.0 / count);
  return launch_status("grico_mse_grad");
}

int grico_adam_step(float* w, const float* g, float* m, float* v, int64_t n, float lr, float beta1, float beta2,
                    int step, float eps, void* stream) {
  if (!w || !g || !m || !v || n < 0 || step < 1) return GRICO_ERR_INVALID;
  if (n == 0) return GRICO_OK;
  const float c1 = 1.0f - std::pow(beta1, float(step));
  const float c2 = 1.0f - std::pow(beta2, float(step));
  adam_step<<<int(std::min<int64_t>((n + 255) / 256, 148 * 16)), 256, 0, as_stream(stream)>>>(w, g, m, v, n, lr, beta1,
                                                                                            beta2, c1, c2, eps);
  return launch_status("grico_adam_step");
}

// grid <- reduced vector (idx[g] = reduced dof of grid point g or -1), FP32
int grico_grid_gather(const int64_t* idx, int64_t n_grid, const float* src, float scale, float* dst, void* stream) {
  if (!idx || !src || !dst || n_grid < 0) return GRICO_ERR_INVALID;
  if (n_grid == 0) return GRICO_OK;
  grid_gather<float, float><<<int(std::min<int64_t>((n_grid + 255) / 256, 148 * 16)), 256, 0, as_stream(stream)>>>(
      idx, n_grid, src, scale, nullptr, dst);
  return launch_status("grico_grid_gather");
}

// reduced vector += scale * grid, FP32
int grico_grid_scatter_add(const int64_t* idx, int64_t n_grid, const float* src, float scale, float* dst,
                           void* stream) {
  if (!idx || !src || !dst || n_grid < 0) return GRICO_ERR_INVALID;
  if (n_grid == 0) return GRICO_OK;
  grid_scatter_add<float, float><<<int(std::min<int64_t>((n_grid + 255) / 256, 148 * 16)), 256, 0, as_stream(stream)>>>(
      idx, n_grid, src, scale, nullptr, dst);
  return launch_status("grico_grid_scatter_add");
}

// out = w (r - ar), *sum = sum w (r - ar)^2 (device double); partial: scratch of 592 doubles
int grico_weighted_residual(const float* r, const float* ar, const float* w, float* out, int64_t n, double* partial,
                            double* sum, void* stream) {
  if (!r || !ar || !w || !out || !partial || !sum || n <= 0) return GRICO_ERR_INVALID;
  cudaStream_t st = as_stream(stream);
  weighted_residual<float><<<kRedBlocks, 256, 0, st>>>(r, ar, w, out, n, partial);
  reduce_final<<<1, kRedThreads, 0, st>>>(partial, kRedBlocks, sum);
  return launch_status("grico_weighted_residual");
}

// Bytes of the packed BF16 weights of the tensor-core convolution (Ci, Co), or -1 when the
// shape is not served.
int64_t grico_conv_tc_weight_bytes(int Ci, int Co) {
  return tc::conv_tc_supported(Ci, Co) ? int64_t(tc::conv_tc_weight_bytes(Ci, Co)) : -1;
}

// FP32 weights [Co][Ci][27] -> packed BF16 weights (grico_conv_tc_weight_bytes bytes at wp).
int grico_conv3d_pack_weights_tc(const float* w, int Ci, int Co, void* wp, void* stream) {
  if (!w || !wp || !tc::conv_tc_supported(Ci, Co)) {
    set_error("grico_conv3d_pack_weights_tc: invalid argument (Ci 16, 32, 48 or 64, Co up to 128)");
    return GRICO_ERR_INVALID;
  }
  return conv_tc_pack(w, Ci, Co, wp, as_stream(stream));
}

// Tensor-core forward convolution (tcgen05.mma, BF16 operands, FP32 accumulation): x BF16
// channels-last [B][Z][Y][X][Ci], wp packed weights, y BF16 channels-last [B][Z][Y][X][Co]
// (y_layout 0) or FP32 [B][Co][Z][Y][X] (y_layout 1).
int grico_conv3d_forward_tc(const void* x, const void* wp, const float* bias, void* y, int y_layout, int B, int Ci,
                            int Co, int Z, int Y, int X, int relu, void* stream) {
  const bool aligned = (reinterpret_cast<uintptr_t>(x) % 16 == 0) && (reinterpret_cast<uintptr_t>(wp) % 16 == 0) &&
                       (y_layout == 1 || reinterpret_cast<uintptr_t>(y) % 16 == 0);
  if (!x || !wp || !y || !aligned || (y_layout != 0 && y_layout != 1) || !conv_args_ok(B, Ci, Co, Z, Y, X) ||
      !tc::conv_tc_supported(Ci, Co) || (y_layout == 0 && Co % 8 != 0)) {
    set_error("grico_conv3d_forward_tc: invalid argument (Ci 16, 32, 48 or 64, Co up to 128 and a multiple of 8 for "
              "channels-last output, 16-byte aligned buffers)");
    return GRICO_ERR_INVALID;
  }
  return conv_tc_forward(x, wp, bias, y, y_layout, B, Ci, Co, Z, Y, X, relu, as_stream(stream));
}

// Synchronises `stream` and reports (then clears) a bounded wait of a tensor-core kernel (the
// convolutions and the FP32 apply of uniform batches) that gave up on this device:
// GRICO_ERR_TIMEOUT, else GRICO_OK.
int grico_tc_status(void* stream) {
  int* err = nullptr;
  if (int rc = conv_tc_err_ptr(&err)) return rc;
  cudaStream_t st = as_stream(stream);
  int h = 0;
  if (cudaMemcpyAsync(&h, err, sizeof(int), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
      cudaStreamSynchronize(st) != cudaSuccess)
    return launch_status("grico_conv_tc_status");
  if (h) {
    const int zero = 0;
    cudaMemcpyAsync(err, &zero, sizeof(int), cudaMemcpyHostToDevice, st);
    cudaStreamSynchronize(st);
    set_error("a tensor-core kernel's bounded wait gave up");
    return GRICO_ERR_TIMEOUT;
  }
  return GRICO_OK;
}

int grico_conv_tc_status(void* stream) { return grico_tc_status(stream); }

}  // extern "C"
