// Vector kernels of the reduced Krylov solvers (solve.jl:761-817): dots with a deterministic
// two-stage reduction, fused CG updates and the Jacobi scaling.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace grico {

constexpr int kRedThreads = 256;
constexpr int kRedBlocks = 592;  // 4 x 148 SMs

template <typename T>
__device__ __forceinline__ double block_sum(double v, double* sh) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) sh[warp] = v;
  __syncthreads();
  v = threadIdx.x < (blockDim.x >> 5) ? sh[lane] : 0.0;
  if (warp == 0)
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}

// partial[block] = sum_i a[i]*b[i]
template <typename T>
static __global__ void dot_partial(const T* __restrict__ a, const T* __restrict__ b, int64_t n, double* __restrict__ partial) {
  __shared__ double sh[32];
  double s = 0.0;
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x)
    s += double(a[i]) * double(b[i]);
  s = block_sum<T>(s, sh);
  if (threadIdx.x == 0) partial[blockIdx.x] = s;
}

static __global__ void reduce_final(const double* __restrict__ partial, int count, double* __restrict__ out) {
  __shared__ double sh[32];
  double s = 0.0;
  for (int i = threadIdx.x; i < count; i += blockDim.x) s += partial[i];
  s = block_sum<double>(s, sh);
  if (threadIdx.x == 0) *out = s;
}

// x += alpha p ; r -= alpha q ; partial = sum r*r
static __global__ void cg_update_xr(double* __restrict__ x, double* __restrict__ r, const double* __restrict__ p,
                             const double* __restrict__ q, const double* __restrict__ scal, int64_t n,
                             double* __restrict__ partial) {
  __shared__ double sh[32];
  if (!(scal[1] > 0.0)) {  // breakdown: keep x and r, the host reports it
    if (threadIdx.x == 0) partial[blockIdx.x] = 0.0;
    return;
  }
  const double alpha = scal[0] / scal[1];  // rz / pAp
  double s = 0.0;
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) {
    x[i] += alpha * p[i];
    double ri = r[i] - alpha * q[i];
    r[i] = ri;
    s += ri * ri;
  }
  s = block_sum<double>(s, sh);
  if (threadIdx.x == 0) partial[blockIdx.x] = s;
}

// z = dinv .* r (dinv == nullptr => identity); partial = sum r*z
static __global__ void jacobi_dot(const double* __restrict__ r, const double* __restrict__ dinv, double* __restrict__ z,
                           int64_t n, double* __restrict__ partial) {
  __shared__ double sh[32];
  double s = 0.0;
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) {
    double zi = dinv ? dinv[i] * r[i] : r[i];
    z[i] = zi;
    s += r[i] * zi;
  }
  s = block_sum<double>(s, sh);
  if (threadIdx.x == 0) partial[blockIdx.x] = s;
}

// p = z + (rz_new / rz_old) p
static __global__ void cg_direction(double* __restrict__ p, const double* __restrict__ z, const double* __restrict__ rz_new,
                             const double* __restrict__ rz_old, int64_t n) {
  const double beta = rz_new[0] / rz_old[0];
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x)
    p[i] = z[i] + beta * p[i];
}

template <typename T>
static __global__ void fill_kernel(T* __restrict__ y, int64_t n, T v) {
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) y[i] = v;
}

// y = a*x + b*y; with b == 0, y is not read (it may be fresh memory holding NaN bit patterns,
// and 0 * NaN is NaN)
template <typename T>
static __global__ void axpby_kernel(T a, const T* __restrict__ x, T b, T* __restrict__ y, int64_t n) {
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x)
    y[i] = b == T(0) ? a * x[i] : a * x[i] + b * y[i];
}

// z = w .* r
template <typename T>
static __global__ void scale_kernel(const T* __restrict__ w, const T* __restrict__ r, T* __restrict__ z, int64_t n) {
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x)
    z[i] = w[i] * r[i];
}

// Constraint rows of the full layout (assembly.jl:1893-1920): fixed rows copy x, affine
// relation rows evaluate x[p] - sum c x[j].
template <typename T>
static __global__ void constraint_action(const int64_t* __restrict__ fixed, int64_t n_fixed, const int64_t* __restrict__ piv,
                                  const int64_t* __restrict__ off, const int64_t* __restrict__ idx,
                                  const double* __restrict__ coef, int64_t n_rel, const T* __restrict__ x,
                                  T* __restrict__ y, int64_t n_vec) {
  const int rhs = blockIdx.y;
  x += rhs * n_vec;
  y += rhs * n_vec;
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n_fixed + n_rel;
       i += int64_t(gridDim.x) * blockDim.x) {
    if (i < n_fixed) {
      y[fixed[i]] = x[fixed[i]];
    } else {
      int64_t r = i - n_fixed;
      T v = x[piv[r]];
      for (int64_t t = off[r]; t < off[r + 1]; ++t) v -= T(coef[t]) * x[idx[t]];
      y[piv[r]] = v;
    }
  }
}

// constraint right-hand sides: b[fixed] = fixed value, b[pivot] = relation rhs
static __global__ void constraint_rhs(const int64_t* __restrict__ fixed, const double* __restrict__ fixed_vals,
                                      int64_t n_fixed, const int64_t* __restrict__ piv,
                                      const double* __restrict__ rel_rhs, int64_t n_rel, double* __restrict__ b) {
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n_fixed + n_rel;
       i += int64_t(gridDim.x) * blockDim.x) {
    if (i < n_fixed) b[fixed[i]] = fixed_vals[i];
    else b[piv[i - n_fixed]] = rel_rhs[i - n_fixed];
  }
}

// u_full = shift + P u_red (CSR rows per full dof)
static __global__ void expand_reduced(const int64_t* __restrict__ off, const int64_t* __restrict__ idx,
                               const double* __restrict__ coef, const double* __restrict__ shift,
                               const double* __restrict__ ured, double* __restrict__ ufull, int64_t n_full) {
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n_full; i += int64_t(gridDim.x) * blockDim.x) {
    double v = shift ? shift[i] : 0.0;
    for (int64_t t = off[i]; t < off[i + 1]; ++t) v += coef[t] * ured[idx[t]];
    ufull[i] = v;
  }
}

// y_red += P^T y_full
static __global__ void project_reduced(const int64_t* __restrict__ off, const int64_t* __restrict__ idx,
                                const double* __restrict__ coef, const double* __restrict__ yfull,
                                double* __restrict__ yred, int64_t n_full) {
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n_full; i += int64_t(gridDim.x) * blockDim.x) {
    double v = yfull[i];
    for (int64_t t = off[i]; t < off[i + 1]; ++t) atomicAdd(yred + idx[t], coef[t] * v);
  }
}

// dinv = 1/diag with a non-finite/zero check flag (solve.jl:740-748)
static __global__ void invert_diagonal(const double* __restrict__ d, double* __restrict__ dinv, int64_t n, int* __restrict__ bad) {
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) {
    double v = d[i];
    if (!(v > 0.0 || v < 0.0) || !isfinite(v)) {
      atomicExch(bad, 1);
      dinv[i] = 0.0;
    } else {
      dinv[i] = 1.0 / v;
    }
  }
}

// y[idx[k]] += val[k]
static __global__ void add_sparse(const int64_t* __restrict__ idx, const double* __restrict__ val, int64_t n,
                                  double* __restrict__ y) {
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x)
    atomicAdd(y + idx[i], val[i]);
}

}  // namespace grico

namespace grico {
// y += sign * (*coef) * x  (coefficient read from device memory, no host round trip)
static __global__ void axpy_dev(double* __restrict__ y, const double* __restrict__ x, const double* __restrict__ coef,
                                double sign, int64_t n) {
  const double a = sign * coef[0];
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x)
    y[i] += a * x[i];
}
}  // namespace grico
