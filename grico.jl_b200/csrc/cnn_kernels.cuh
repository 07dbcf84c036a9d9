// 3-D convolution kernels of the learned smoother (3x3x3 kernels, zero padding, stride 1).
//
// Tensors are [batch][channel][z][y][x].  The forward kernel gives each block an 8x8x8 tile of
// output voxels and a group of CO_TILE output channels; per input channel it stages the 10^3
// halo tile and the CO_TILE x 27 weights in shared memory and every thread accumulates its
// voxel for all CO_TILE channels (27 * CO_TILE FMAs per staged value).  Activations may be
// stored in BF16 (TIn/TOut); arithmetic is FP32.  Backward-data reuses the forward kernel with
// the transposed, spatially flipped weights; backward-weight reduces grad_y * x over the
// batch and the voxels with one block per (output channel, input channel) pair.
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace grico {

constexpr int kConvTile = 8;
constexpr int kConvHalo = kConvTile + 2;
constexpr int kConvCo = 8;

template <typename T>
__device__ __forceinline__ float to_f(T v) { return float(v); }
template <>
__device__ __forceinline__ float to_f<__nv_bfloat16>(__nv_bfloat16 v) { return __bfloat162float(v); }
template <typename T>
__device__ __forceinline__ T from_f(float v) { return T(v); }
template <>
__device__ __forceinline__ __nv_bfloat16 from_f<__nv_bfloat16>(float v) { return __float2bfloat16(v); }

// y[b, co, v] = act(bias[co] + sum_{ci,k} w[co, ci, k] x[b, ci, v + off(k)])
// grid: (tiles_x * tiles_y * tiles_z, ceil(Co / kConvCo), B); block: 512 threads.
template <typename TIn, typename TOut>
__global__ void __launch_bounds__(512) conv3d_fwd(const TIn* __restrict__ x, const float* __restrict__ w,
                                                  const float* __restrict__ bias, TOut* __restrict__ y, int Ci,
                                                  int Co, int Z, int Y, int X, int relu) {
  __shared__ float xs[kConvHalo * kConvHalo * kConvHalo];
  __shared__ float ws[kConvCo * 27];
  const int tx = (X + kConvTile - 1) / kConvTile, ty = (Y + kConvTile - 1) / kConvTile;
  const int tile = blockIdx.x;
  const int bx = (tile % tx) * kConvTile, by = ((tile / tx) % ty) * kConvTile, bz = (tile / (tx * ty)) * kConvTile;
  const int co0 = blockIdx.y * kConvCo;
  const int b = blockIdx.z;
  const int lx = threadIdx.x % kConvTile, ly = (threadIdx.x / kConvTile) % kConvTile, lz = threadIdx.x / (kConvTile * kConvTile);
  const int vx = bx + lx, vy = by + ly, vz = bz + lz;
  const int64_t vol = int64_t(Z) * Y * X;
  float acc[kConvCo];
#pragma unroll
  for (int c = 0; c < kConvCo; ++c) acc[c] = (co0 + c < Co && bias) ? bias[co0 + c] : 0.0f;
  for (int ci = 0; ci < Ci; ++ci) {
    const TIn* xc = x + (int64_t(b) * Ci + ci) * vol;
    for (int t = threadIdx.x; t < kConvHalo * kConvHalo * kConvHalo; t += blockDim.x) {
      const int hx = t % kConvHalo, hy = (t / kConvHalo) % kConvHalo, hz = t / (kConvHalo * kConvHalo);
      const int gx = bx + hx - 1, gy = by + hy - 1, gz = bz + hz - 1;
      const bool in = gx >= 0 && gx < X && gy >= 0 && gy < Y && gz >= 0 && gz < Z;
      xs[t] = in ? to_f(xc[(int64_t(gz) * Y + gy) * X + gx]) : 0.0f;
    }
    for (int t = threadIdx.x; t < kConvCo * 27; t += blockDim.x) {
      const int c = t / 27, k = t % 27;
      ws[t] = co0 + c < Co ? w[(int64_t(co0 + c) * Ci + ci) * 27 + k] : 0.0f;
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < 27; ++k) {
      const int kx = k % 3, ky = (k / 3) % 3, kz = k / 9;
      const float v = xs[((lz + kz) * kConvHalo + (ly + ky)) * kConvHalo + (lx + kx)];
#pragma unroll
      for (int c = 0; c < kConvCo; ++c) acc[c] += ws[c * 27 + k] * v;
    }
    __syncthreads();
  }
  if (vx < X && vy < Y && vz < Z) {
#pragma unroll
    for (int c = 0; c < kConvCo; ++c) {
      if (co0 + c >= Co) break;
      float v = acc[c];
      if (relu) v = v > 0.0f ? v : 0.0f;
      y[(int64_t(b) * Co + co0 + c) * vol + (int64_t(vz) * Y + vy) * X + vx] = from_f<TOut>(v);
    }
  }
}

// wt[ci, co, 26 - k] = w[co, ci, k]: the weights of the backward-data convolution
static __global__ void conv3d_flip_transpose(const float* __restrict__ w, float* __restrict__ wt, int Ci, int Co) {
  const int64_t n = int64_t(Co) * Ci * 27;
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) {
    const int k = int(i % 27);
    const int64_t r = i / 27;
    const int ci = int(r % Ci), co = int(r / Ci);
    wt[(int64_t(ci) * Co + co) * 27 + (26 - k)] = w[i];
  }
}

// gw[co, ci, k] (+)= sum_{b, v} gy[b, co, v] x[b, ci, v + off(k)];  gb[co] (+)= sum gy
// grid: (Ci, Co); block: 256 threads, each owning strided voxels; block reduction per tap.
static __global__ void __launch_bounds__(256) conv3d_bwd_weight(const float* __restrict__ x, const float* __restrict__ gy,
                                                         float* __restrict__ gw, float* __restrict__ gb, int B,
                                                         int Ci, int Co, int Z, int Y, int X) {
  const int ci = blockIdx.x, co = blockIdx.y;
  const int64_t vol = int64_t(Z) * Y * X;
  float acc[28];
#pragma unroll
  for (int k = 0; k < 28; ++k) acc[k] = 0.0f;
  for (int b = 0; b < B; ++b) {
    const float* xc = x + (int64_t(b) * Ci + ci) * vol;
    const float* g = gy + (int64_t(b) * Co + co) * vol;
    for (int64_t v = threadIdx.x; v < vol; v += blockDim.x) {
      const float gv = g[v];
      if (gv == 0.0f) continue;
      const int vx = int(v % X), vy = int((v / X) % Y), vz = int(v / (int64_t(X) * Y));
#pragma unroll
      for (int k = 0; k < 27; ++k) {
        const int sx = vx + k % 3 - 1, sy = vy + (k / 3) % 3 - 1, sz = vz + k / 9 - 1;
        if (sx >= 0 && sx < X && sy >= 0 && sy < Y && sz >= 0 && sz < Z)
          acc[k] += gv * xc[(int64_t(sz) * Y + sy) * X + sx];
      }
      acc[27] += gv;
    }
  }
  __shared__ float red[8][28];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < 28; ++k) {
    float s = acc[k];
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (lane == 0) red[warp][k] = s;
  }
  __syncthreads();
  if (threadIdx.x < 28) {
    float s = 0.0f;
    for (int wi = 0; wi < 8; ++wi) s += red[wi][threadIdx.x];
    if (threadIdx.x < 27) gw[(int64_t(co) * Ci + ci) * 27 + threadIdx.x] = s;
    else if (ci == 0 && gb) gb[co] = s;
  }
}

// g *= (y > 0): ReLU backward with the stored post-activation values
static __global__ void relu_backward(const float* __restrict__ y, float* __restrict__ g, int64_t n) {
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x)
    if (!(y[i] > 0.0f)) g[i] = 0.0f;
}

// g = 2 (p - t) m / count and partial sums of m (p - t)^2 (masked mean squared error)
static __global__ void mse_grad(const float* __restrict__ p, const float* __restrict__ t, const float* __restrict__ m,
                         float* __restrict__ g, int64_t n, float inv_count, double* __restrict__ partial) {
  __shared__ double sh[256];
  double s = 0.0;
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) {
    const float mi = m ? m[i] : 1.0f;
    const float d = (p[i] - t[i]) * mi;
    g[i] = 2.0f * d * inv_count;
    s += double(d) * double(d);
  }
  sh[threadIdx.x] = s;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) sh[threadIdx.x] += sh[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) partial[blockIdx.x] = sh[0];
}

static __global__ void scale_scalar(double* s, double f) { *s *= f; }

// Adam step (D. P. Kingma and J. Ba, arXiv:1412.6980) with bias correction factors c1, c2
static __global__ void adam_step(float* __restrict__ w, const float* __restrict__ g, float* __restrict__ m,
                          float* __restrict__ v, int64_t n, float lr, float b1, float b2, float c1, float c2,
                          float eps) {
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) {
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.0f - b1) * gi;
    const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    w[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
  }
}

// dst[g] = src[idx[g]] * scale * (scale_dev ? *scale_dev : 1) for idx[g] >= 0, else 0
template <typename TS, typename TD>
__global__ void grid_gather(const int64_t* __restrict__ idx, int64_t n_grid, const TS* __restrict__ src, float scale,
                            const double* __restrict__ scale_dev, TD* __restrict__ dst) {
  const float s = scale * (scale_dev ? float(*scale_dev) : 1.0f);
  for (int64_t g = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; g < n_grid; g += int64_t(gridDim.x) * blockDim.x) {
    const int64_t i = idx[g];
    dst[g] = from_f<TD>(i >= 0 ? float(src[i]) * s : 0.0f);
  }
}

// the same into channel 0 of a channels-last grid: dst[g * stride]
template <typename TS, typename TD>
__global__ void grid_gather_strided(const int64_t* __restrict__ idx, int64_t n_grid, const TS* __restrict__ src,
                                    float scale, const double* __restrict__ scale_dev, TD* __restrict__ dst,
                                    int stride) {
  const float s = scale * (scale_dev ? float(*scale_dev) : 1.0f);
  for (int64_t g = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; g < n_grid; g += int64_t(gridDim.x) * blockDim.x) {
    const int64_t i = idx[g];
    dst[g * stride] = from_f<TD>(i >= 0 ? float(src[i]) * s : 0.0f);
  }
}

// dst[idx[g]] += src[g] * scale * (scale_dev ? *scale_dev : 1) (each dof appears once in the grid)
template <typename TS, typename TD>
__global__ void grid_scatter_add(const int64_t* __restrict__ idx, int64_t n_grid, const TS* __restrict__ src,
                                 float scale, const double* __restrict__ scale_dev, TD* __restrict__ dst) {
  const float s = scale * (scale_dev ? float(*scale_dev) : 1.0f);
  for (int64_t g = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; g < n_grid; g += int64_t(gridDim.x) * blockDim.x) {
    const int64_t i = idx[g];
    if (i >= 0) dst[i] += TD(to_f(src[g]) * s);
  }
}

// out = w (r - ar); partial sums of w (r - ar)^2
template <typename T>
__global__ void weighted_residual(const T* __restrict__ r, const T* __restrict__ ar, const T* __restrict__ w,
                                  T* __restrict__ out, int64_t n, double* __restrict__ partial) {
  __shared__ double sh[256];
  double s = 0.0;
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) {
    const double d = double(r[i]) - double(ar[i]);
    out[i] = T(double(w[i]) * d);
    s += double(w[i]) * d * d;
  }
  sh[threadIdx.x] = s;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) sh[threadIdx.x] += sh[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) partial[blockIdx.x] = sh[0];
}

}  // namespace grico
