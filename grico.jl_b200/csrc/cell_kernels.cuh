// Sum-factorized matrix-free cell kernels for sm_100a.
//
// Semantics follow Grico.jl's accumulator cell apply for TestChannels(mass*u, kappa*k(x)*∇u)
// on axis-aligned affine cells (accumulators.jl:1003-1020, 1955-2013): gather the local
// coefficients through the cell's term map (assembly.jl:1751-1771), interpolate value and
// gradient at the tensor Gauss points, weight by ŵ·det J, project back and scatter
// (assembly.jl:1788-1803).
//
// Schedule (differs from the reference's D + D² contractions, same result up to rounding):
// interpolate modes -> points with the 1-D basis table B (n x q) once per axis, take
// reference derivatives at the points with the q x q collocation matrix D of the Gauss
// points (exact because q >= p+1), apply the pointwise flux, and run the transposed
// sequence.  That is 2·D contractions each way instead of D + D².
//
// Thread layout, 3-D: one thread per (x, y) point column, the z column held in registers;
// contractions along z are register-only, along x and y through shared memory.  CPB cells
// share a block.  Accumulation into the global result uses atomicAdd (the reference's
// colouring only makes its CPU scatter race-free; the GPU sums in arbitrary order, which
// changes results at the rounding level only).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace grico {

struct BatchView {
  int32_t n_cells;
  const int32_t* map;        // [n_cells*nbox]
  const double* coef;        // nullable
  const int64_t* tail_off;
  const int32_t* tail_idx;
  const double* tail_coef;
  const double* h;           // [n_cells*dim]
  const double* kappa_pts;   // nullable [n_cells*nq]
  const double* B;           // [n*q]   B[i*q+p] = psi_i(xi_p)
  const double* D;           // [q*q]   D[p*q+l] = L_l'(xi_p)
  const double* W;           // [q]     reference Gauss weights
  const double* G;           // [n*q]   reference derivative table psi_i'(xi_p)
  const uint8_t* skip;       // nullable: cells excluded from the diagonal kernel
  const double* mass_pts;    // nullable [n_cells*nq]: pointwise mass added to the constant mass
  // long tails, operator apply: the expansions are summed by tail_gather before the cell kernel
  // (tail_x[rhs * n_tail + k]) and spread by tail_scatter after it (the kernel adds into tail_y,
  // zeroed before; entries with the same expansion share a tail)
  const void* tail_x = nullptr;
  void* tail_y = nullptr;
  int64_t n_tail = 0;
  // deterministic apply: the kernels store every entry's local result at
  // local_out[rhs * local_stride + e] instead of adding it into y (det_gather sums them)
  void* local_out = nullptr;
  int64_t local_stride = 0;
};

template <typename T>
__device__ __forceinline__ T gather_entry(const BatchView& b, int64_t e, const T* __restrict__ x) {
  int v = __ldg(b.map + e);
  if (v >= 0) return b.coef ? T(__ldg(b.coef + e)) * x[v] : x[v];
  if (v == -1) return T(0);
  int64_t k = -(int64_t(v) + 2);
  if (b.tail_x) return static_cast<const T*>(b.tail_x)[blockIdx.y * b.n_tail + k];
  T s = T(0);
  for (int64_t t = b.tail_off[k]; t < b.tail_off[k + 1]; ++t) s += T(b.tail_coef[t]) * x[b.tail_idx[t]];
  return s;
}

template <typename T>
__device__ __forceinline__ void scatter_entry(const BatchView& b, int64_t e, T val, T* __restrict__ y) {
  if (b.local_out) {
    static_cast<T*>(b.local_out)[blockIdx.y * b.local_stride + e] = val;
    return;
  }
  int v = __ldg(b.map + e);
  if (v >= 0) {
    atomicAdd(y + v, b.coef ? T(__ldg(b.coef + e)) * val : val);
    return;
  }
  if (v == -1) return;
  int64_t k = -(int64_t(v) + 2);
  if (b.tail_y) {
    atomicAdd(static_cast<T*>(b.tail_y) + blockIdx.y * b.n_tail + k, val);  // entries may share a tail
    return;
  }
  for (int64_t t = b.tail_off[k]; t < b.tail_off[k + 1]; ++t) atomicAdd(y + b.tail_idx[t], T(b.tail_coef[t]) * val);
}

// xt[r * n_tail + k] = sum_t coef[t] x[r * n_vec + idx[t]] over the terms of tail k (rhs r =
// blockIdx.y): one warp per tail, lanes over its terms, a shuffle reduction
template <typename T>
__global__ void tail_gather(const int64_t* __restrict__ off, const int32_t* __restrict__ idx,
                            const double* __restrict__ coef, int64_t n_tail, const T* __restrict__ x, int64_t n_vec,
                            T* __restrict__ xt, T* __restrict__ yt) {
  const int lane = threadIdx.x % 32;
  const int64_t nw = int64_t(gridDim.x) * blockDim.x / 32;
  x += blockIdx.y * n_vec;
  xt += blockIdx.y * n_tail;
  yt += blockIdx.y * n_tail;
  for (int64_t k = (blockIdx.x * int64_t(blockDim.x) + threadIdx.x) / 32; k < n_tail; k += nw) {
    T s = T(0);
    for (int64_t t = off[k] + lane; t < off[k + 1]; t += 32) s += T(coef[t]) * x[idx[t]];
#pragma unroll
    for (int d = 16; d > 0; d /= 2) s += __shfl_down_sync(0xffffffffu, s, d);
    if (lane == 0) {
      xt[k] = s;
      yt[k] = T(0);  // the cell kernel adds the results of the tail's entries here
    }
  }
}

// Tail segments of at most kTailSeg terms, for nrhs <= 32 right-hand sides at once: one warp per
// segment, lane r = right-hand side, so each term's index and coefficient are read once for
// all columns and a long expansion is spread over many warps.  The gather adds its partial sum
// to xt (zeroed before); the scatter spreads yt over the segment's terms.
constexpr int kTailSeg = 16;

template <typename T>
__global__ void tail_gather_seg(const int32_t* __restrict__ seg_k, const int64_t* __restrict__ seg_t, int64_t n_seg,
                                const int64_t* __restrict__ off, const int32_t* __restrict__ idx,
                                const double* __restrict__ coef, int64_t n_tail, const T* __restrict__ x,
                                int64_t n_vec, T* __restrict__ xt, T* __restrict__ yt, int nrhs) {
  const int lane = threadIdx.x % 32;
  const bool on = lane < nrhs;
  const int64_t nw = int64_t(gridDim.x) * blockDim.x / 32;
  const T* xr = x + (on ? lane : 0) * n_vec;
  for (int64_t sg = (blockIdx.x * int64_t(blockDim.x) + threadIdx.x) / 32; sg < n_seg; sg += nw) {
    const int32_t k = seg_k[sg];
    const int64_t t0 = seg_t[sg], t1 = min(t0 + kTailSeg, off[k + 1]);
    T acc = T(0);
#pragma unroll
    for (int u = 0; u < kTailSeg; ++u) {
      const int64_t t = t0 + u;
      if (t < t1 && on) acc += T(__ldg(coef + t)) * xr[__ldg(idx + t)];
    }
    if (on) {
      atomicAdd(xt + lane * n_tail + k, acc);
      if (t0 == off[k]) yt[lane * n_tail + k] = T(0);  // the tail's first segment clears its result slot
    }
  }
}

template <typename T>
__global__ void tail_scatter_seg(const int32_t* __restrict__ seg_k, const int64_t* __restrict__ seg_t, int64_t n_seg,
                                 const int64_t* __restrict__ off, const int32_t* __restrict__ idx,
                                 const double* __restrict__ coef, int64_t n_tail, const T* __restrict__ yt,
                                 T* __restrict__ y, int64_t n_vec, int nrhs) {
  const int lane = threadIdx.x % 32;
  const bool on = lane < nrhs;
  const int64_t nw = int64_t(gridDim.x) * blockDim.x / 32;
  T* yr = y + (on ? lane : 0) * n_vec;
  for (int64_t sg = (blockIdx.x * int64_t(blockDim.x) + threadIdx.x) / 32; sg < n_seg; sg += nw) {
    const int32_t k = seg_k[sg];
    const int64_t t0 = seg_t[sg], t1 = min(t0 + kTailSeg, off[k + 1]);
    const T v = on ? yt[lane * n_tail + k] : T(0);
#pragma unroll
    for (int u = 0; u < kTailSeg; ++u) {
      const int64_t t = t0 + u;
      if (t < t1 && on) atomicAdd(yr + __ldg(idx + t), T(__ldg(coef + t)) * v);
    }
  }
}

// y[r * n_vec + idx[t]] += coef[t] yt[r * n_tail + k] over the terms of tail k: one warp per tail
template <typename T>
__global__ void tail_scatter(const int64_t* __restrict__ off, const int32_t* __restrict__ idx,
                             const double* __restrict__ coef, int64_t n_tail, const T* __restrict__ yt, T* __restrict__ y,
                             int64_t n_vec) {
  const int lane = threadIdx.x % 32;
  const int64_t nw = int64_t(gridDim.x) * blockDim.x / 32;
  y += blockIdx.y * n_vec;
  yt += blockIdx.y * n_tail;
  for (int64_t k = (blockIdx.x * int64_t(blockDim.x) + threadIdx.x) / 32; k < n_tail; k += nw) {
    const T v = yt[k];
    for (int64_t t = off[k] + lane; t < off[k + 1]; t += 32) atomicAdd(y + idx[t], T(coef[t]) * v);
  }
}

// Deterministic sum of the stored local results: y[r * n_vec + d] = sum over the row d of the
// gather CSR (in its fixed order) of coef[k] local[r * stride + pos[k]]
template <typename T>
__global__ void det_gather(const int64_t* __restrict__ off, const int32_t* __restrict__ pos,
                           const double* __restrict__ coef, int64_t n, const T* __restrict__ local, int64_t stride,
                           T* __restrict__ y, int64_t n_vec) {
  local += blockIdx.y * stride;
  y += blockIdx.y * n_vec;
  for (int64_t d = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; d < n; d += int64_t(gridDim.x) * blockDim.x) {
    T s = T(0);
    for (int64_t k = off[d]; k < off[d + 1]; ++k) s += T(coef[k]) * local[pos[k]];
    y[d] = s;
  }
}

// 1-D tables of one (n, q) signature, passed by value so that fully unrolled contractions read
// them as constant-bank operands instead of shared-memory loads.
template <int N, int Q, typename T>
struct Tables1D {
  T B[N * Q];  // B[i*Q+p] = psi_i(xi_p)
  T D[Q * Q];  // D[p*Q+l] = L_l'(xi_p)
  T W[Q];      // Gauss weights
};

// mode: 0 = operator apply, 1 = load (rhs) from tabulated source values at the points.
//
// One cell is handled by Q*Q threads; every contraction step gives each thread one whole line
// of the cell's Q^3 point box along the contracted axis (z-lines: thread (x, y); y-lines:
// thread (x, z); x-lines: thread (y, z)), so a step costs one line of shared-memory loads and
// stores per thread for N*Q (or Q*Q) FMAs.  Three buffers per cell hold u / r, the x-flux and
// the y-flux.  Sequence: z, y, x interpolation; x derivative; y derivative; z derivative and
// the pointwise flux on z-lines; transposed z, y, x derivatives; transposed x, y, z
// interpolation; scatter.
template <int N, int Q, int CPB, typename T>
__global__ void __launch_bounds__(Q* Q* CPB) cell_apply_3d(BatchView b, const Tables1D<N, Q, T> tab,
                                                           const T* __restrict__ x, T* __restrict__ y,
                                                           int64_t n_vec, T mass, T kappa, int mode,
                                                           const double* __restrict__ src) {
  constexpr int Q3 = Q * Q * Q;
  constexpr int NB = N * N * N;
  constexpr int PITCH = Q3 | 1;  // odd per-cell pitch spreads cells over the banks
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* smem = reinterpret_cast<T*>(smem_raw);
  const int c = threadIdx.y;
  T* S0 = smem + (3 * c + 0) * PITCH;
  T* S1 = smem + (3 * c + 1) * PITCH;
  T* S2 = smem + (3 * c + 2) * PITCH;
  const int ta = threadIdx.x % Q, tb = threadIdx.x / Q;
  const int64_t cell = int64_t(blockIdx.x) * CPB + c;
  const bool act = cell < b.n_cells;
  x += blockIdx.y * n_vec;
  y += blockIdx.y * n_vec;
  auto at = [](int ix, int iy, int iz) { return ix + Q * (iy + Q * iz); };

  T h0 = T(1), h1 = T(1), h2 = T(1);
  if (act) {
    h0 = T(b.h[cell * 3 + 0]);
    h1 = T(b.h[cell * 3 + 1]);
    h2 = T(b.h[cell * 3 + 2]);
  }
  const T sx = T(2) / h0, sy = T(2) / h1, sz = T(2) / h2;
  const T detJ = h0 * h1 * h2 * T(0.125);
  T line[Q], out[Q];

  if (mode != 1) {
    // 1. gather + z interpolation on z-lines (x = ta < N, y = tb < N)
    if (ta < N && tb < N) {
      T in[N];
#pragma unroll
      for (int k = 0; k < N; ++k) in[k] = act ? gather_entry<T>(b, cell * NB + ta + N * (tb + N * k), x) : T(0);
#pragma unroll
      for (int q = 0; q < Q; ++q) {
        T s = T(0);
#pragma unroll
        for (int k = 0; k < N; ++k) s += tab.B[k * Q + q] * in[k];
        S0[at(ta, tb, q)] = s;
      }
    }
    __syncthreads();
    // 2. y interpolation on y-lines (x = ta < N, z = tb)
    if (ta < N) {
#pragma unroll
      for (int j = 0; j < N; ++j) line[j] = S0[at(ta, j, tb)];
#pragma unroll
      for (int q = 0; q < Q; ++q) {
        T s = T(0);
#pragma unroll
        for (int j = 0; j < N; ++j) s += tab.B[j * Q + q] * line[j];
        out[q] = s;
      }
#pragma unroll
      for (int q = 0; q < Q; ++q) S0[at(ta, q, tb)] = out[q];
    }
    __syncthreads();
    // 3. x interpolation and x derivative on x-lines (y = ta, z = tb)
    {
#pragma unroll
      for (int i = 0; i < N; ++i) line[i] = S0[at(i, ta, tb)];
#pragma unroll
      for (int q = 0; q < Q; ++q) {
        T s = T(0);
#pragma unroll
        for (int i = 0; i < N; ++i) s += tab.B[i * Q + q] * line[i];
        out[q] = s;
      }
#pragma unroll
      for (int q = 0; q < Q; ++q) {
        T s = T(0);
#pragma unroll
        for (int l = 0; l < Q; ++l) s += tab.D[q * Q + l] * out[l];
        S0[at(q, ta, tb)] = out[q];
        S2[at(q, ta, tb)] = s;
      }
    }
    __syncthreads();
    // 4. y derivative on y-lines (x = ta, z = tb)
    {
#pragma unroll
      for (int l = 0; l < Q; ++l) line[l] = S0[at(ta, l, tb)];
#pragma unroll
      for (int q = 0; q < Q; ++q) {
        T s = T(0);
#pragma unroll
        for (int l = 0; l < Q; ++l) s += tab.D[q * Q + l] * line[l];
        S1[at(ta, q, tb)] = s;
      }
    }
    __syncthreads();
  }
  // 5. z derivative, pointwise flux and transposed z derivative on z-lines (x = ta, y = tb)
  {
    const T wxy = tab.W[ta] * tab.W[tb] * detJ;
    if (mode == 1) {
#pragma unroll
      for (int q = 0; q < Q; ++q) {
        const T f = act && src ? T(src[cell * Q3 + at(ta, tb, q)]) : T(0);
        S0[at(ta, tb, q)] = wxy * tab.W[q] * f;
      }
    } else {
      T u[Q], dz[Q];
#pragma unroll
      for (int l = 0; l < Q; ++l) u[l] = S0[at(ta, tb, l)];
#pragma unroll
      for (int q = 0; q < Q; ++q) {
        T s = T(0);
#pragma unroll
        for (int l = 0; l < Q; ++l) s += tab.D[q * Q + l] * u[l];
        dz[q] = s;
      }
#pragma unroll
      for (int q = 0; q < Q; ++q) {
        const int p = at(ta, tb, q);
        const T w = wxy * tab.W[q];
        T k = kappa;
        if (b.kappa_pts && act) k *= T(b.kappa_pts[cell * Q3 + p]);
        const T wk = w * k;
        S2[p] = S2[p] * (wk * sx * sx);
        S1[p] = S1[p] * (wk * sy * sy);
        dz[q] *= wk * sz * sz;
        u[q] *= w * (b.mass_pts && act ? mass + T(b.mass_pts[cell * Q3 + p]) : mass);
      }
#pragma unroll
      for (int l = 0; l < Q; ++l) {
        T s = u[l];
#pragma unroll
        for (int q = 0; q < Q; ++q) s += tab.D[q * Q + l] * dz[q];
        S0[at(ta, tb, l)] = s;
      }
    }
  }
  __syncthreads();
  if (mode != 1) {
    // 6. transposed y derivative on y-lines (x = ta, z = tb)
    {
#pragma unroll
      for (int q = 0; q < Q; ++q) line[q] = S1[at(ta, q, tb)];
#pragma unroll
      for (int l = 0; l < Q; ++l) {
        T s = S0[at(ta, l, tb)];
#pragma unroll
        for (int q = 0; q < Q; ++q) s += tab.D[q * Q + l] * line[q];
        S0[at(ta, l, tb)] = s;
      }
    }
    __syncthreads();
  }
  // 7. transposed x derivative and transposed x interpolation on x-lines (y = ta, z = tb)
  {
#pragma unroll
    for (int l = 0; l < Q; ++l) out[l] = S0[at(l, ta, tb)];
    if (mode != 1) {
#pragma unroll
      for (int q = 0; q < Q; ++q) line[q] = S2[at(q, ta, tb)];
#pragma unroll
      for (int l = 0; l < Q; ++l) {
        T s = out[l];
#pragma unroll
        for (int q = 0; q < Q; ++q) s += tab.D[q * Q + l] * line[q];
        out[l] = s;
      }
    }
#pragma unroll
    for (int i = 0; i < N; ++i) {
      T s = T(0);
#pragma unroll
      for (int q = 0; q < Q; ++q) s += tab.B[i * Q + q] * out[q];
      S0[at(i, ta, tb)] = s;
    }
  }
  __syncthreads();
  // 8. transposed y interpolation on y-lines (x = ta < N, z = tb)
  if (ta < N) {
#pragma unroll
    for (int q = 0; q < Q; ++q) line[q] = S0[at(ta, q, tb)];
#pragma unroll
    for (int j = 0; j < N; ++j) {
      T s = T(0);
#pragma unroll
      for (int q = 0; q < Q; ++q) s += tab.B[j * Q + q] * line[q];
      S0[at(ta, j, tb)] = s;
    }
  }
  __syncthreads();
  // 9. transposed z interpolation on z-lines (x = ta < N, y = tb < N) and scatter
  if (act && ta < N && tb < N) {
#pragma unroll
    for (int q = 0; q < Q; ++q) line[q] = S0[at(ta, tb, q)];
#pragma unroll
    for (int k = 0; k < N; ++k) {
      T s = T(0);
#pragma unroll
      for (int q = 0; q < Q; ++q) s += tab.B[k * Q + q] * line[q];
      scatter_entry<T>(b, cell * NB + ta + N * (tb + N * k), s, y);
    }
  }
}

template <int N, int Q, int CPB, typename T>
__global__ void __launch_bounds__(Q* CPB) cell_apply_2d(BatchView b, const T* __restrict__ x, T* __restrict__ y,
                                                        int64_t n_vec, T mass, T kappa, int mode,
                                                        const double* __restrict__ src) {
  constexpr int Q2 = Q * Q;
  constexpr int NB = N * N;
  __shared__ T sB[N * Q], sD[Q * Q], sW[Q];
  __shared__ T S0[CPB][Q2];
  const int tid = threadIdx.x + threadIdx.y * blockDim.x;
  for (int i = tid; i < N * Q; i += blockDim.x * blockDim.y) sB[i] = T(b.B[i]);
  for (int i = tid; i < Q * Q; i += blockDim.x * blockDim.y) sD[i] = T(b.D[i]);
  for (int i = tid; i < Q; i += blockDim.x * blockDim.y) sW[i] = T(b.W[i]);
  const int tx = threadIdx.x, c = threadIdx.y;
  const int64_t cell = int64_t(blockIdx.x) * CPB + c;
  const bool act = cell < b.n_cells;
  const int rhs = blockIdx.y;
  x += rhs * n_vec;
  y += rhs * n_vec;
  T* s0 = S0[c];
  __syncthreads();
  T h0 = 1, h1 = 1;
  if (act) {
    h0 = T(b.h[cell * 2 + 0]);
    h1 = T(b.h[cell * 2 + 1]);
  }
  const T sx = T(2) / h0, sy = T(2) / h1;
  const T detJ = h0 * h1 * T(0.25);
  T u[Q], dx[Q], dy[Q];
  if (mode != 1) {
    if (act && tx < N) {
      T reg[N];
#pragma unroll
      for (int k = 0; k < N; ++k) reg[k] = gather_entry<T>(b, cell * NB + tx + N * k, x);
#pragma unroll
      for (int q = 0; q < Q; ++q) {
        T s = T(0);
#pragma unroll
        for (int k = 0; k < N; ++k) s += sB[k * Q + q] * reg[k];
        s0[tx + Q * q] = s;
      }
    }
    __syncthreads();
#pragma unroll
    for (int q = 0; q < Q; ++q) {
      T s = T(0);
#pragma unroll
      for (int i = 0; i < N; ++i) s += sB[i * Q + tx] * s0[i + Q * q];
      u[q] = s;
    }
#pragma unroll
    for (int q = 0; q < Q; ++q) {
      T s = T(0);
#pragma unroll
      for (int l = 0; l < Q; ++l) s += sD[q * Q + l] * u[l];
      dy[q] = s;
    }
    __syncthreads();
#pragma unroll
    for (int q = 0; q < Q; ++q) s0[tx + Q * q] = u[q];
    __syncthreads();
#pragma unroll
    for (int q = 0; q < Q; ++q) {
      T s = T(0);
#pragma unroll
      for (int l = 0; l < Q; ++l) s += sD[tx * Q + l] * s0[l + Q * q];
      dx[q] = s;
    }
  }
  T r[Q];
#pragma unroll
  for (int q = 0; q < Q; ++q) {
    const T w = sW[tx] * sW[q] * detJ;
    if (mode == 1) {
      T f = act && src ? T(src[cell * Q2 + tx + Q * q]) : T(0);
      r[q] = w * f;
    } else {
      T k = kappa;
      if (b.kappa_pts && act) k *= T(b.kappa_pts[cell * Q2 + tx + Q * q]);
      r[q] = w * (b.mass_pts && act ? mass + T(b.mass_pts[cell * Q2 + tx + Q * q]) : mass) * u[q];
      dx[q] *= w * k * sx * sx;
      dy[q] *= w * k * sy * sy;
    }
  }
  if (mode != 1) {
    __syncthreads();
#pragma unroll
    for (int q = 0; q < Q; ++q) s0[tx + Q * q] = dx[q];
    __syncthreads();
#pragma unroll
    for (int l = 0; l < Q; ++l) {
      T s = r[l];
#pragma unroll
      for (int q = 0; q < Q; ++q) s += sD[q * Q + l] * dy[q] + sD[q * Q + tx] * s0[q + Q * l];
      r[l] = s;
    }
  }
  __syncthreads();
#pragma unroll
  for (int q = 0; q < Q; ++q) s0[tx + Q * q] = r[q];
  __syncthreads();
  if (act && tx < N) {
    T t[Q];
#pragma unroll
    for (int q = 0; q < Q; ++q) {
      T s = T(0);
#pragma unroll
      for (int p = 0; p < Q; ++p) s += sB[tx * Q + p] * s0[p + Q * q];
      t[q] = s;
    }
#pragma unroll
    for (int k = 0; k < N; ++k) {
      T s = T(0);
#pragma unroll
      for (int q = 0; q < Q; ++q) s += sB[k * Q + q] * t[q];
      scatter_entry<T>(b, cell * NB + tx + N * k, s, y);
    }
  }
}

// Generic tensor-table kernel for any dimension 1..3 and any (n, q) — one block per cell,
// threads over points then over modes; O(n^D q^D D) per cell.  Used for 1-D, q < p+1, as the
// diagonal kernel (mode 3: local diagonal sum of squared shape products) and to evaluate the
// field at the quadrature points (mode 4: y[cell * nq + p] = u(x_p), nothing projected).
template <typename T>
__global__ void cell_apply_generic(BatchView b, int dim, int n0, int n1, int n2, int q0, int q1, int q2,
                                   const T* __restrict__ x, T* __restrict__ y, int64_t n_vec, T mass, T kappa,
                                   int mode, const double* __restrict__ src) {
  extern __shared__ unsigned char smem_raw[];
  T* sm = reinterpret_cast<T*>(smem_raw);
  const int q[3] = {q0, q1, q2};
  const int nb = n0 * n1 * n2, nq = q0 * q1 * q2;
  T* xl = sm;            // nb
  T* flux = xl + nb;     // (dim+1)*nq
  const int64_t cell = blockIdx.x;
  if (mode == 3 && b.skip && b.skip[cell]) return;
  const int rhs = blockIdx.y;
  x += rhs * n_vec;
  y += rhs * n_vec;
  const int nmax = max(n0, max(n1, n2)), qmax = max(q0, max(q1, q2));
  // tables are stored with per-axis stride nmax*qmax: B[a][i*q[a]+p]
  T hs[3] = {1, 1, 1};
  T detJ = 1;
  for (int a = 0; a < dim; ++a) {
    hs[a] = T(b.h[cell * dim + a]);
    detJ *= hs[a] * T(0.5);
  }
  auto Bv = [&](int a, int i, int p) { return T(b.B[a * nmax * qmax + i * q[a] + p]); };
  auto Gv = [&](int a, int i, int p) { return T(b.G[a * nmax * qmax + i * q[a] + p]) * (T(2) / hs[a]); };
  auto Wv = [&](int a, int p) { return T(b.W[a * qmax + p]); };
  if (mode == 0 || mode == 4) {
    for (int i = threadIdx.x; i < nb; i += blockDim.x) xl[i] = gather_entry<T>(b, cell * nb + i, x);
    __syncthreads();
  }
  if (mode != 3) {
    for (int p = threadIdx.x; p < nq; p += blockDim.x) {
      int pi[3] = {p % q0, (p / q0) % q1, p / (q0 * q1)};
      T w = detJ;
      for (int a = 0; a < dim; ++a) w *= Wv(a, pi[a]);
      if (mode == 1) {
        flux[p] = w * (src ? T(src[cell * nq + p]) : T(0));
        for (int a = 0; a < dim; ++a) flux[(a + 1) * nq + p] = T(0);
        continue;
      }
      T uval = 0, g[3] = {0, 0, 0};
      for (int i = 0; i < nb; ++i) {
        int mi[3] = {i % n0, (i / n0) % n1, i / (n0 * n1)};
        T bv[3] = {1, 1, 1};
        for (int a = 0; a < dim; ++a) bv[a] = Bv(a, mi[a], pi[a]);
        T prod = bv[0] * bv[1] * bv[2];
        uval += xl[i] * prod;
        for (int a = 0; a < dim; ++a) {
          T gg = Gv(a, mi[a], pi[a]);
          for (int e = 0; e < dim; ++e)
            if (e != a) gg *= bv[e];
          g[a] += xl[i] * gg;
        }
      }
      if (mode == 4) {  // u at the point
        y[cell * nq + p] = uval;
        continue;
      }
      T k = kappa;
      if (b.kappa_pts) k *= T(b.kappa_pts[cell * nq + p]);
      flux[p] = w * (b.mass_pts ? mass + T(b.mass_pts[cell * nq + p]) : mass) * uval;
      for (int a = 0; a < dim; ++a) flux[(a + 1) * nq + p] = w * k * g[a];
    }
    __syncthreads();
  }
  if (mode == 4) return;
  for (int i = threadIdx.x; i < nb; i += blockDim.x) {
    int mi[3] = {i % n0, (i / n0) % n1, i / (n0 * n1)};
    T acc = 0;
    for (int p = 0; p < nq; ++p) {
      int pi[3] = {p % q0, (p / q0) % q1, p / (q0 * q1)};
      T bv[3] = {1, 1, 1};
      for (int a = 0; a < dim; ++a) bv[a] = Bv(a, mi[a], pi[a]);
      T prod = bv[0] * bv[1] * bv[2];
      if (mode == 3) {
        T w = detJ;
        for (int a = 0; a < dim; ++a) w *= Wv(a, pi[a]);
        T k = kappa;
        if (b.kappa_pts) k *= T(b.kappa_pts[cell * nq + p]);
        T s = (b.mass_pts ? mass + T(b.mass_pts[cell * nq + p]) : mass) * prod * prod;
        for (int a = 0; a < dim; ++a) {
          T gg = Gv(a, mi[a], pi[a]);
          for (int e = 0; e < dim; ++e)
            if (e != a) gg *= bv[e];
          s += k * gg * gg;
        }
        acc += w * s;
        continue;
      }
      acc += flux[p] * prod;
      for (int a = 0; a < dim; ++a) {
        T gg = Gv(a, mi[a], pi[a]);
        for (int e = 0; e < dim; ++e)
          if (e != a) gg *= bv[e];
        acc += flux[(a + 1) * nq + p] * gg;
      }
    }
    if (mode == 3) {
      // diagonal: coefficient squared scatter (assembly.jl:1811-1825)
      int v = b.map[cell * nb + i];
      if (v >= 0) {
        T cc = b.coef ? T(b.coef[cell * nb + i]) : T(1);
        atomicAdd(y + v, cc * cc * acc);
      } else if (v <= -2) {
        int64_t kk = -(int64_t(v) + 2);
        for (int64_t t = b.tail_off[kk]; t < b.tail_off[kk + 1]; ++t) {
          T cc = T(b.tail_coef[t]);
          atomicAdd(y + b.tail_idx[t], cc * cc * acc);
        }
      }
    } else {
      scatter_entry<T>(b, cell * nb + i, acc, y);
    }
  }
}

}  // namespace grico

namespace grico {

// Point-quadrature items: one cell's modes evaluated at an arbitrary list of reference points.
// Covers non-tensor cells (finite-cell cut cells, accumulators.jl:1022-1054), boundary faces
// and embedded surfaces (_accumulate_one_sided_apply_basis!, accumulators.jl:1133-1161).
// kind 1 (cell):    TestChannels(mass*u, kappa*k(x)*grad u)
// kind 2 (nitsche): TestChannels(-du/dn + eta*u, -u*n)   (symmetric Nitsche, driver.jl:52-62)
struct PointView {
  int32_t n_items;
  int kind;
  int n[3];
  const int32_t* map;
  const double* coef;
  const int64_t* tail_off;
  const int32_t* tail_idx;
  const double* tail_coef;
  const double* h;         // [n_items*dim]
  const int64_t* pt_off;   // [n_items+1]
  const double* ref;       // [n_points*dim]
  const double* w;         // [n_points]
  const double* nrm;       // [n_points*dim] or null
  const double* eta;       // [n_items] or null
  const double* kpts;      // [n_points] or null
  const uint8_t* skip;     // nullable: items excluded from the diagonal kernel (host computes them)
  // GRICO_ITEM_INTERFACE: plus-side modes per axis, reference points, cell sizes, normal axis
  int np[3];
  const double* ref_p;     // [n_points*dim]
  const double* h_p;       // [n_items*dim]
  const int32_t* axis;     // [n_items]
  void* local_out;         // deterministic apply (BatchView::local_out)
  int64_t local_stride;
};

constexpr int kPointChunk = 32;
constexpr int kPointThreads = 128;
constexpr int kPointWarps = kPointThreads / 32;
constexpr int kMaxModes = 6;  // modes per thread: box <= 768

// psi_0..psi_p and derivatives at x (polynomials.jl:403-434) on the device
template <typename T>
__device__ void fe_basis_dev(T x, int p, T* v, T* d) {
  if (p == 0) {
    v[0] = T(1);
    d[0] = T(0);
    return;
  }
  T pm2 = T(1), pm1 = x;  // P_{k-2}, P_{k-1}
  v[0] = T(0.5) * (T(1) - x);
  v[1] = T(0.5) * (T(1) + x);
  d[0] = T(-0.5);
  d[1] = T(0.5);
  for (int k = 2; k <= p; ++k) {
    const T inv_k = T(1) / T(k);
    const T pk = T(2 * k - 1) * inv_k * x * pm1 - T(k - 1) * inv_k * pm2;
    v[k] = (pk - pm2) / sqrt(T(4 * k - 2));
    d[k] = sqrt(T(2 * k - 1) / T(2)) * pm1;
    pm2 = pm1;
    pm1 = pk;
  }
}

// value and gradient of box mode (m0, m1, m2) at chunk point pp from the staged 1-D tables
template <typename T, int D>
__device__ __forceinline__ void mode_value_grad(const T* tv, const T* td, int nmax, int pp, const int* mi, T& phi,
                                                T* grad) {
  T v[D], g[D];
#pragma unroll
  for (int a = 0; a < D; ++a) {
    v[a] = tv[(pp * D + a) * nmax + mi[a]];
    g[a] = td[(pp * D + a) * nmax + mi[a]];
  }
  phi = v[0];
#pragma unroll
  for (int a = 1; a < D; ++a) phi *= v[a];
#pragma unroll
  for (int a = 0; a < D; ++a) {
    T gg = g[a];
#pragma unroll
    for (int e = 0; e < D; ++e)
      if (e != a) gg *= v[e];
    grad[a] = gg;
  }
}

// mode: 0 apply, 1 rhs (src per point), 3 local diagonal.  One block per item (blockIdx.x)
// and right-hand side (blockIdx.y); points are staged in chunks of kPointChunk: 1-D tables per
// (point, axis), then one warp per point reduces u and grad u over the modes, then one thread
// per mode projects the point fluxes.
template <typename T, int D>
__global__ void __launch_bounds__(kPointThreads) point_apply(PointView b, const T* __restrict__ x, T* __restrict__ y,
                                                             int64_t n_vec, T mass, T kappa, int mode,
                                                             const double* __restrict__ src) {
  extern __shared__ unsigned char smem_raw[];
  int nn[3] = {b.n[0], D > 1 ? b.n[1] : 1, D > 2 ? b.n[2] : 1};
  const int nb = nn[0] * nn[1] * nn[2];
  const int nmax = max(nn[0], max(nn[1], nn[2]));
  T* xl = reinterpret_cast<T*>(smem_raw);                       // nb
  T* tv = xl + nb;                                               // [chunk][D][nmax] values
  T* td = tv + kPointChunk * D * nmax;                           // [chunk][D][nmax] derivatives
  T* fl = td + kPointChunk * D * nmax;                           // [chunk][D+1] flux
  const int64_t item = blockIdx.x;
  if (mode == 3 && b.skip && b.skip[item]) return;
  x += blockIdx.y * n_vec;
  y += blockIdx.y * n_vec;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  T scale[D];
#pragma unroll
  for (int a = 0; a < D; ++a) scale[a] = T(2) / T(b.h[item * D + a]);
  const T eta = b.eta ? T(b.eta[item]) : T(0);
  BatchView bv;
  bv.n_cells = b.n_items;
  bv.map = b.map;
  bv.coef = b.coef;
  bv.tail_off = b.tail_off;
  bv.tail_idx = b.tail_idx;
  bv.tail_coef = b.tail_coef;
  bv.local_out = b.local_out;
  bv.local_stride = b.local_stride;
  if (mode == 0)
    for (int i = threadIdx.x; i < nb; i += blockDim.x) xl[i] = gather_entry<T>(bv, item * nb + i, x);
  T acc[kMaxModes];
#pragma unroll
  for (int k = 0; k < kMaxModes; ++k) acc[k] = T(0);
  const int64_t p_begin = b.pt_off[item], p_end = b.pt_off[item + 1];
  for (int64_t p0 = p_begin; p0 < p_end; p0 += kPointChunk) {
    const int cnt = int(p_end - p0 < int64_t(kPointChunk) ? p_end - p0 : int64_t(kPointChunk));
    __syncthreads();
    for (int t = threadIdx.x; t < cnt * D; t += blockDim.x) {
      const int pp = t / D, a = t - pp * D;
      T* v = tv + (pp * D + a) * nmax;
      T* d = td + (pp * D + a) * nmax;
      fe_basis_dev<T>(T(b.ref[(p0 + pp) * D + a]), nn[a] - 1, v, d);
      for (int i = 0; i < nn[a]; ++i) d[i] *= scale[a];
    }
    __syncthreads();
    if (mode == 1) {
      for (int pp = threadIdx.x; pp < cnt; pp += blockDim.x) {
        const int64_t pg = p0 + pp;
        const T w = T(b.w[pg]);
        const T g = src ? T(src[pg]) : T(0);
        if (b.kind == 2) {
          fl[pp * (D + 1)] = w * eta * g;
#pragma unroll
          for (int a = 0; a < D; ++a) fl[pp * (D + 1) + 1 + a] = -w * g * T(b.nrm[pg * D + a]);
        } else {
          fl[pp * (D + 1)] = w * g;
#pragma unroll
          for (int a = 0; a < D; ++a) fl[pp * (D + 1) + 1 + a] = T(0);
        }
      }
      __syncthreads();
    } else if (mode == 0) {
      for (int pp = warp; pp < cnt; pp += kPointWarps) {
        T u = T(0), g[D];
#pragma unroll
        for (int a = 0; a < D; ++a) g[a] = T(0);
        for (int i = lane; i < nb; i += 32) {
          const int mi[3] = {i % nn[0], (i / nn[0]) % nn[1], i / (nn[0] * nn[1])};
          T phi, grad[D];
          mode_value_grad<T, D>(tv, td, nmax, pp, mi, phi, grad);
          const T xi = xl[i];
          u += xi * phi;
#pragma unroll
          for (int a = 0; a < D; ++a) g[a] += xi * grad[a];
        }
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) {
          u += __shfl_xor_sync(0xffffffffu, u, off);
#pragma unroll
          for (int a = 0; a < D; ++a) g[a] += __shfl_xor_sync(0xffffffffu, g[a], off);
        }
        if (lane == 0) {
          const int64_t pg = p0 + pp;
          const T w = T(b.w[pg]);
          if (b.kind == 2) {
            T dn = T(0);
#pragma unroll
            for (int a = 0; a < D; ++a) dn += g[a] * T(b.nrm[pg * D + a]);
            fl[pp * (D + 1)] = w * (-dn + eta * u);
#pragma unroll
            for (int a = 0; a < D; ++a) fl[pp * (D + 1) + 1 + a] = -w * u * T(b.nrm[pg * D + a]);
          } else {
            const T k = b.kpts ? kappa * T(b.kpts[pg]) : kappa;
            fl[pp * (D + 1)] = w * mass * u;
#pragma unroll
            for (int a = 0; a < D; ++a) fl[pp * (D + 1) + 1 + a] = w * k * g[a];
          }
        }
      }
      __syncthreads();
    }
#pragma unroll
    for (int k = 0; k < kMaxModes; ++k) {
      const int i = threadIdx.x + k * blockDim.x;
      if (i >= nb) break;
      const int mi[3] = {i % nn[0], (i / nn[0]) % nn[1], i / (nn[0] * nn[1])};
      T s = T(0);
      for (int pp = 0; pp < cnt; ++pp) {
        T phi, grad[D];
        mode_value_grad<T, D>(tv, td, nmax, pp, mi, phi, grad);
        if (mode == 3) {
          const int64_t pg = p0 + pp;
          const T w = T(b.w[pg]);
          if (b.kind == 2) {
            T dn = T(0);
#pragma unroll
            for (int a = 0; a < D; ++a) dn += grad[a] * T(b.nrm[pg * D + a]);
            s += w * (eta * phi * phi - T(2) * phi * dn);
          } else {
            const T kk = b.kpts ? kappa * T(b.kpts[pg]) : kappa;
            T gg = T(0);
#pragma unroll
            for (int a = 0; a < D; ++a) gg += grad[a] * grad[a];
            s += w * (mass * phi * phi + kk * gg);
          }
        } else {
          s += fl[pp * (D + 1)] * phi;
#pragma unroll
          for (int a = 0; a < D; ++a) s += fl[pp * (D + 1) + 1 + a] * grad[a];
        }
      }
      acc[k] += s;
    }
  }
#pragma unroll
  for (int k = 0; k < kMaxModes; ++k) {
    const int i = threadIdx.x + k * blockDim.x;
    if (i >= nb) break;
    if (mode == 3) {
      const int v = b.map[item * nb + i];
      if (v >= 0) {
        const T c = b.coef ? T(b.coef[item * nb + i]) : T(1);
        atomicAdd(y + v, c * c * acc[k]);
      }
    } else {
      scatter_entry<T>(bv, item * nb + i, acc[k], y);
    }
  }
}

constexpr int kIfaceModes = 8;  // modes per thread: minus + plus boxes <= 1024

// value and normal derivative (along axis ax) of box mode mi at chunk point pp
template <typename T, int D>
__device__ __forceinline__ void mode_value_dn(const T* tv, const T* td, int nmax, int pp, const int* mi, int ax,
                                              T& phi, T& dn) {
  phi = T(1);
  dn = T(1);
#pragma unroll
  for (int a = 0; a < D; ++a) {
    const T v = tv[(pp * D + a) * nmax + mi[a]];
    phi *= v;
    dn *= a == ax ? td[(pp * D + a) * nmax + mi[a]] : v;
  }
}

// Symmetric interior-penalty interface items (GRICO_ITEM_INTERFACE; interface_apply!,
// accumulators.jl:1576-1616, with the SIPG form of benchmark/sine_poisson_sipg.jl:54-95).
// mode 0 apply, 3 local diagonal (interface_diagonal!, sine_poisson_sipg.jl:97-123); there is
// no load term.  One block per interface: both cells' local coefficients are gathered into
// shared memory, points are staged in chunks with 1-D tables of both sides, one warp per point
// forms the two traces u-, u+, du-/dn, du+/dn, and one thread per mode projects
//   minus test mode: w (sigma J - {du/dn}) phi + w (-J/2) dphi/dn,
//   plus test mode: -w (sigma J - {du/dn}) phi + w (-J/2) dphi/dn,   J = u- - u+.
template <typename T, int D>
__global__ void __launch_bounds__(kPointThreads) interface_apply(PointView b, const T* __restrict__ x,
                                                                 T* __restrict__ y, int64_t n_vec, int mode) {
  extern __shared__ unsigned char smem_raw[];
  const int nm[3] = {b.n[0], D > 1 ? b.n[1] : 1, D > 2 ? b.n[2] : 1};
  const int npl[3] = {b.np[0], D > 1 ? b.np[1] : 1, D > 2 ? b.np[2] : 1};
  const int nbm = nm[0] * nm[1] * nm[2], nbp = npl[0] * npl[1] * npl[2], nb = nbm + nbp;
  const int nmax = max(max(nm[0], max(nm[1], nm[2])), max(npl[0], max(npl[1], npl[2])));
  T* xl = reinterpret_cast<T*>(smem_raw);       // nb
  T* tvm = xl + nb;                              // [chunk][D][nmax] minus values
  T* tdm = tvm + kPointChunk * D * nmax;         // minus derivatives (physical)
  T* tvp = tdm + kPointChunk * D * nmax;         // plus values
  T* tdp = tvp + kPointChunk * D * nmax;         // plus derivatives (physical)
  T* fl = tdp + kPointChunk * D * nmax;          // [chunk][2] value and normal-derivative coefficients
  const int64_t item = blockIdx.x;
  if (mode == 1 || (mode == 3 && b.skip && b.skip[item])) return;
  x += blockIdx.y * n_vec;
  y += blockIdx.y * n_vec;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int ax = b.axis[item];
  T sm[D], sp[D];
#pragma unroll
  for (int a = 0; a < D; ++a) {
    sm[a] = T(2) / T(b.h[item * D + a]);
    sp[a] = T(2) / T(b.h_p[item * D + a]);
  }
  const T sigma = T(b.eta[item]);
  BatchView bv;
  bv.n_cells = b.n_items;
  bv.map = b.map;
  bv.coef = b.coef;
  bv.tail_off = b.tail_off;
  bv.tail_idx = b.tail_idx;
  bv.tail_coef = b.tail_coef;
  bv.local_out = b.local_out;
  bv.local_stride = b.local_stride;
  if (mode == 0)
    for (int i = threadIdx.x; i < nb; i += blockDim.x) xl[i] = gather_entry<T>(bv, item * nb + i, x);
  T acc[kIfaceModes];
#pragma unroll
  for (int k = 0; k < kIfaceModes; ++k) acc[k] = T(0);
  const int64_t p_begin = b.pt_off[item], p_end = b.pt_off[item + 1];
  for (int64_t p0 = p_begin; p0 < p_end; p0 += kPointChunk) {
    const int cnt = int(p_end - p0 < int64_t(kPointChunk) ? p_end - p0 : int64_t(kPointChunk));
    __syncthreads();
    for (int t = threadIdx.x; t < 2 * cnt * D; t += blockDim.x) {
      const int side = t / (cnt * D), r = t - side * cnt * D, pp = r / D, a = r - pp * D;
      const int deg = (side ? npl[a] : nm[a]) - 1;
      T* v = (side ? tvp : tvm) + (pp * D + a) * nmax;
      T* d = (side ? tdp : tdm) + (pp * D + a) * nmax;
      fe_basis_dev<T>(T((side ? b.ref_p : b.ref)[(p0 + pp) * D + a]), deg, v, d);
      const T sc = side ? sp[a] : sm[a];
      for (int i = 0; i <= deg; ++i) d[i] *= sc;
    }
    __syncthreads();
    if (mode == 0) {
      for (int pp = warp; pp < cnt; pp += kPointWarps) {
        T um = T(0), dm = T(0), up = T(0), dp = T(0);
        for (int i = lane; i < nb; i += 32) {
          const bool plus = i >= nbm;
          const int li = plus ? i - nbm : i;
          const int* nn = plus ? npl : nm;
          const int mi[3] = {li % nn[0], (li / nn[0]) % nn[1], li / (nn[0] * nn[1])};
          T phi, dn;
          mode_value_dn<T, D>(plus ? tvp : tvm, plus ? tdp : tdm, nmax, pp, mi, ax, phi, dn);
          const T xi = xl[i];
          if (plus) {
            up += xi * phi;
            dp += xi * dn;
          } else {
            um += xi * phi;
            dm += xi * dn;
          }
        }
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) {
          um += __shfl_xor_sync(0xffffffffu, um, off);
          dm += __shfl_xor_sync(0xffffffffu, dm, off);
          up += __shfl_xor_sync(0xffffffffu, up, off);
          dp += __shfl_xor_sync(0xffffffffu, dp, off);
        }
        if (lane == 0) {
          const T w = T(b.w[p0 + pp]);
          const T jump = um - up;
          const T avg = T(0.5) * (dm + dp);
          fl[pp * 2] = w * (sigma * jump - avg);
          fl[pp * 2 + 1] = -T(0.5) * w * jump;
        }
      }
      __syncthreads();
    }
#pragma unroll
    for (int k = 0; k < kIfaceModes; ++k) {
      const int i = threadIdx.x + k * blockDim.x;
      if (i >= nb) break;
      const bool plus = i >= nbm;
      const int li = plus ? i - nbm : i;
      const int* nn = plus ? npl : nm;
      const int mi[3] = {li % nn[0], (li / nn[0]) % nn[1], li / (nn[0] * nn[1])};
      T s = T(0);
      for (int pp = 0; pp < cnt; ++pp) {
        T phi, dn;
        mode_value_dn<T, D>(plus ? tvp : tvm, plus ? tdp : tdm, nmax, pp, mi, ax, phi, dn);
        if (mode == 3) {
          const T w = T(b.w[p0 + pp]);
          s += w * (sigma * phi * phi + (plus ? phi * dn : -phi * dn));
        } else {
          s += (plus ? -fl[pp * 2] : fl[pp * 2]) * phi + fl[pp * 2 + 1] * dn;
        }
      }
      acc[k] += s;
    }
  }
#pragma unroll
  for (int k = 0; k < kIfaceModes; ++k) {
    const int i = threadIdx.x + k * blockDim.x;
    if (i >= nb) break;
    if (mode == 3) {
      const int v = b.map[item * nb + i];
      if (v >= 0) {
        const T c = b.coef ? T(b.coef[item * nb + i]) : T(1);
        atomicAdd(y + v, c * c * acc[k]);
      }
    } else {
      scatter_entry<T>(bv, item * nb + i, acc[k], y);
    }
  }
}

// Sum-factorised SIPG interface apply (same result as interface_apply, mode 0).  An item's points
// form a tensor grid over the tangential axes t1 < t2 (t1 fastest, q1 x q2 points) with one
// normal coordinate per side; sf_q holds (q1, q2) and sf_x the 1-D coordinates per item:
// [side][t1 (q1) | t2 (q2) | normal].  Per side: the normal contraction gives the trace and the
// normal derivative on the n1 x n2 tangential modes, two tangential contractions give them at
// the points, the flux w (sigma J - {du/dn}) and -w J / 2 (J = u- - u+) is formed per point,
// and the transposed contractions project it back: O(n^3 + n^2 q + n q^2) per side instead of
// q^2 n^3 mode evaluations.
template <typename T, int D, int G>
__global__ void __launch_bounds__(kPointThreads) interface_apply_sf(PointView b, const int32_t* __restrict__ sf_q,
                                                                    const double* __restrict__ sf_x, int sf_stride,
                                                                    const T* __restrict__ x, T* __restrict__ y,
                                                                    int64_t n_vec, int64_t item_elems) {
  // G threads per interface: a warp (32, kPointThreads / 32 interfaces per block, warp barriers)
  // or the whole block (kPointThreads)
  static_assert(G == 32 || G == kPointThreads, "one warp or one block per interface");
  extern __shared__ unsigned char smem_raw[];
  const int64_t item = int64_t(blockIdx.x) * (kPointThreads / G) + threadIdx.x / G;
  if (item >= b.n_items) return;  // only warp barriers follow when G == 32
  auto sync = [] {
    if constexpr (G == 32) __syncwarp();
    else __syncthreads();
  };
  x += blockIdx.y * n_vec;
  y += blockIdx.y * n_vec;
  const int ax = b.axis[item];
  const int t1 = ax == 0 ? 1 : 0, t2 = D == 3 ? (ax == 2 ? 1 : 2) : -1;
  const int q1 = sf_q[2 * item], q2 = sf_q[2 * item + 1];
  const int Qm = q1 > q2 ? q1 : q2;
  int nn[2][3];
  for (int a = 0; a < 3; ++a) {
    nn[0][a] = a < D ? b.n[a] : 1;
    nn[1][a] = a < D ? b.np[a] : 1;
  }
  const int nbm = nn[0][0] * nn[0][1] * nn[0][2], nb = nbm + nn[1][0] * nn[1][1] * nn[1][2];
  int nmax = 1;
  for (int s = 0; s < 2; ++s)
    for (int a = 0; a < D; ++a) nmax = nn[s][a] > nmax ? nn[s][a] : nmax;
  const int P = q1 * q2;
  // shared memory (T): local modes; per side Vn, Dn [nmax], V1 [nmax x Qm], V2 [nmax x Qm],
  // U/Dv [nmax x nmax], W/WD [Qm x nmax]; traces at the points u[2][P], d[2][P]; flux F0, F1 [P]
  T* xl = reinterpret_cast<T*>(smem_raw) + (threadIdx.x / G) * item_elems;
  T* base = xl + nb;
  const int per_side = 2 * nmax + 2 * nmax * Qm + 2 * nmax * nmax + 2 * Qm * nmax;
  auto Vn = [&](int s) { return base + s * per_side; };
  auto Dn = [&](int s) { return base + s * per_side + nmax; };
  auto V1 = [&](int s) { return base + s * per_side + 2 * nmax; };
  auto V2 = [&](int s) { return base + s * per_side + 2 * nmax + nmax * Qm; };
  auto U0 = [&](int s) { return base + s * per_side + 2 * nmax + 2 * nmax * Qm; };
  auto UD = [&](int s) { return base + s * per_side + 2 * nmax + 2 * nmax * Qm + nmax * nmax; };
  auto W0 = [&](int s) { return base + s * per_side + 2 * nmax + 2 * nmax * Qm + 2 * nmax * nmax; };
  auto WD = [&](int s) { return base + s * per_side + 2 * nmax + 2 * nmax * Qm + 2 * nmax * nmax + Qm * nmax; };
  T* tr = base + 2 * per_side;  // u[s][p] at tr + s * P, d[s][p] at tr + (2 + s) * P
  T* F0 = tr + 4 * P;
  T* F1 = F0 + P;
  const int tid = threadIdx.x % G, nt = G;

  BatchView bv;
  bv.n_cells = b.n_items;
  bv.map = b.map;
  bv.coef = b.coef;
  bv.tail_off = b.tail_off;
  bv.tail_idx = b.tail_idx;
  bv.tail_coef = b.tail_coef;
  bv.local_out = b.local_out;
  bv.local_stride = b.local_stride;
  for (int i = tid; i < nb; i += nt) xl[i] = gather_entry<T>(bv, item * nb + i, x);
  // 1-D tables: normal values and physical normal derivatives, tangential values
  const double* cx = sf_x + item * int64_t(sf_stride);
  for (int t = tid; t < 2 * (1 + q1 + q2); t += nt) {
    const int s = t / (1 + q1 + q2), r = t % (1 + q1 + q2);
    T v[16], d[16];
    const double* c = cx + s * (q1 + q2 + 1);
    if (r == 0) {
      const int deg = nn[s][ax] - 1;
      fe_basis_dev<T>(T(c[q1 + q2]), deg, v, d);
      const T sc = T(2) / T((s ? b.h_p : b.h)[item * D + ax]);
      for (int i = 0; i <= deg; ++i) {
        Vn(s)[i] = v[i];
        Dn(s)[i] = d[i] * sc;
      }
    } else if (r <= q1) {
      const int deg = nn[s][t1] - 1;
      fe_basis_dev<T>(T(c[r - 1]), deg, v, d);
      for (int i = 0; i <= deg; ++i) V1(s)[i * Qm + (r - 1)] = v[i];
    } else {
      const int deg = D == 3 ? nn[s][t2] - 1 : 0;
      if (D == 3) fe_basis_dev<T>(T(c[r - 1]), deg, v, d);
      else v[0] = T(1);
      for (int i = 0; i <= deg; ++i) V2(s)[i * Qm + (r - 1 - q1)] = v[i];
    }
  }
  sync();
  auto box = [&](int s, int ia, int i1, int i2) {
    int mi[3] = {0, 0, 0};
    mi[ax] = ia;
    mi[t1] = i1;
    if (D == 3) mi[t2] = i2;
    return (s ? nbm : 0) + mi[0] + nn[s][0] * (mi[1] + nn[s][1] * mi[2]);
  };
  auto n2of = [&](int s) { return D == 3 ? nn[s][t2] : 1; };
  // A: normal contraction -> U0, UD [i1 * nmax + i2]
  for (int t = tid; t < 2 * nmax * nmax; t += nt) {
    const int s = t / (nmax * nmax), i1 = (t / nmax) % nmax, i2 = t % nmax;
    if (i1 >= nn[s][t1] || i2 >= n2of(s)) continue;
    T u = T(0), du = T(0);
    for (int ia = 0; ia < nn[s][ax]; ++ia) {
      const T xv = xl[box(s, ia, i1, i2)];
      u += xv * Vn(s)[ia];
      du += xv * Dn(s)[ia];
    }
    U0(s)[i1 * nmax + i2] = u;
    UD(s)[i1 * nmax + i2] = du;
  }
  sync();
  // B: t1 contraction -> W0, WD [p1 * nmax + i2]
  for (int t = tid; t < 2 * q1 * nmax; t += nt) {
    const int s = t / (q1 * nmax), p1 = (t / nmax) % q1, i2 = t % nmax;
    if (i2 >= n2of(s)) continue;
    T u = T(0), du = T(0);
    for (int i1 = 0; i1 < nn[s][t1]; ++i1) {
      const T v = V1(s)[i1 * Qm + p1];
      u += U0(s)[i1 * nmax + i2] * v;
      du += UD(s)[i1 * nmax + i2] * v;
    }
    W0(s)[p1 * nmax + i2] = u;
    WD(s)[p1 * nmax + i2] = du;
  }
  sync();
  // C: t2 contraction -> traces at the points p = p1 + q1 p2
  for (int t = tid; t < 2 * P; t += nt) {
    const int s = t / P, p = t % P, p1 = p % q1, p2 = p / q1;
    T u = T(0), du = T(0);
    for (int i2 = 0; i2 < n2of(s); ++i2) {
      const T v = V2(s)[i2 * Qm + p2];
      u += W0(s)[p1 * nmax + i2] * v;
      du += WD(s)[p1 * nmax + i2] * v;
    }
    tr[s * P + p] = u;
    tr[(2 + s) * P + p] = du;
  }
  sync();
  const T sigma = T(b.eta[item]);
  const int64_t p0 = b.pt_off[item];
  for (int p = tid; p < P; p += nt) {
    const T w = T(b.w[p0 + p]);
    const T jump = tr[p] - tr[P + p];
    const T avg = T(0.5) * (tr[2 * P + p] + tr[3 * P + p]);
    F0[p] = w * (sigma * jump - avg);
    F1[p] = -T(0.5) * w * jump;
  }
  sync();
  // C^T: sum over p2 -> W0 (F0 with the side's sign), WD (F1)
  for (int t = tid; t < 2 * q1 * nmax; t += nt) {
    const int s = t / (q1 * nmax), p1 = (t / nmax) % q1, i2 = t % nmax;
    if (i2 >= n2of(s)) continue;
    T g0 = T(0), g1 = T(0);
    for (int p2 = 0; p2 < q2; ++p2) {
      const T v = V2(s)[i2 * Qm + p2];
      g0 += F0[p1 + q1 * p2] * v;
      g1 += F1[p1 + q1 * p2] * v;
    }
    W0(s)[p1 * nmax + i2] = s ? -g0 : g0;
    WD(s)[p1 * nmax + i2] = g1;
  }
  sync();
  // B^T: sum over p1 -> U0, UD
  for (int t = tid; t < 2 * nmax * nmax; t += nt) {
    const int s = t / (nmax * nmax), i1 = (t / nmax) % nmax, i2 = t % nmax;
    if (i1 >= nn[s][t1] || i2 >= n2of(s)) continue;
    T h0 = T(0), h1 = T(0);
    for (int p1 = 0; p1 < q1; ++p1) {
      const T v = V1(s)[i1 * Qm + p1];
      h0 += W0(s)[p1 * nmax + i2] * v;
      h1 += WD(s)[p1 * nmax + i2] * v;
    }
    U0(s)[i1 * nmax + i2] = h0;
    UD(s)[i1 * nmax + i2] = h1;
  }
  sync();
  // A^T and scatter: y_i = Vn[ia] H0[i1, i2] + Dn[ia] H1[i1, i2]
  for (int i = tid; i < nb; i += nt) {
    const int s = i >= nbm ? 1 : 0, li = s ? i - nbm : i;
    const int mi[3] = {li % nn[s][0], (li / nn[s][0]) % nn[s][1], li / (nn[s][0] * nn[s][1])};
    const int ia = mi[ax], i1 = mi[t1], i2 = D == 3 ? mi[t2] : 0;
    const T val = Vn(s)[ia] * U0(s)[i1 * nmax + i2] + Dn(s)[ia] * UD(s)[i1 * nmax + i2];
    scatter_entry<T>(bv, item * nb + i, val, y);
  }
}

// shared memory of interface_apply_sf for mode counts up to nmax per axis and qm points per
// tangential axis (q1 q2 <= pmax points)
inline size_t interface_sf_smem(int nb, int nmax, int qm, int pmax, size_t elem) {
  const size_t per_side = 2 * size_t(nmax) + 2 * size_t(nmax) * qm + 2 * size_t(nmax) * nmax + 2 * size_t(qm) * nmax;
  return elem * (size_t(nb) + 2 * per_side + 6 * size_t(pmax));
}

}  // namespace grico

namespace grico {

// Finite-cell cut cells as lists of octree subcells.  The candidate rule of a cut cell
// (regions.jl:477-510, 759-792) is the union of the cell's tensor rule mapped onto inside
// subcells and onto terminal cut subcells with the points of positive classifier value
// dropped, so each subcell is a tensor-product cell of its own: the 1-D basis tables at the
// subcell's Gauss points depend only on its level and position, and sum factorisation applies.
// One block per cut cell; each warp takes whole subcells and accumulates into its own copy of
// the local result, the copies are summed and scattered once per cell.
struct SubcellView {
  int32_t n_items;
  const int32_t* map;
  const double* coef;
  const int64_t* tail_off;
  const int32_t* tail_idx;
  const double* tail_coef;
  const double* h;          // [n_items*dim]
  const int64_t* sub_off;   // [n_items+1]
  const int32_t* level;     // [n_sub]
  const int32_t* pos;       // [n_sub*dim]
  const uint64_t* mask;     // [n_sub]: bit p keeps tensor point p (axis 1 fastest)
  const double* ws;         // [n_sub]: weight factor (2^(-dim*level) times the measure factor)
  const double* kpts;       // [n_sub*Q^dim] or null
  const uint8_t* skip;      // diagonal kernel skips these items (host computes them)
  void* local_out;          // deterministic apply (BatchView::local_out)
  int64_t local_stride;
};

template <int Q, typename T>
struct SubTables {
  T eta[Q];     // Gauss points
  T W[Q];       // Gauss weights
  T Dm[Q * Q];  // Dm[p*Q+l] = L_l'(eta_p), collocation derivative
};

constexpr int kSubThreads = 128;
constexpr int kSubWarps = kSubThreads / 32;

template <int D, int N, int Q>
struct SubSizes {
  static constexpr int NB = D == 3 ? N * N * N : N * N;
  static constexpr int QP = D == 3 ? Q * Q * Q : Q * Q;
  static constexpr int A1 = D == 3 ? N * N * Q : 1;  // after the z stage
  static constexpr int A2 = D == 3 ? N * Q * Q : N * Q;
  // per-warp scratch: value and derivative tables, A1, A2, U, G[D], R, local result (last)
  static constexpr int WARP = 2 * D * N * Q + A1 + A2 + QP * (D + 2) + NB;
};

// mode: 0 apply, 1 rhs (src[n_sub*QP] at the subcell points), 3 local diagonal
template <typename T, int D, int N, int Q>
__global__ void __launch_bounds__(kSubThreads) subcell_apply(SubcellView b, const SubTables<Q, T> tab,
                                                            const T* __restrict__ x, T* __restrict__ y, int64_t n_vec,
                                                            T mass, T kappa, int mode, const double* __restrict__ src) {
  using S = SubSizes<D, N, Q>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* xl = reinterpret_cast<T*>(smem_raw);  // NB, shared by the warps
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  T* tb = xl + S::NB + warp * S::WARP;  // [D][N*Q] values at the subcell points
  T* td = tb + D * N * Q;               // [D][N*Q] physical derivatives (diagonal only)
  T* a1 = td + D * N * Q;
  T* a2 = a1 + S::A1;
  T* U = a2 + S::A2;
  T* G = U + S::QP;                     // [D][QP]
  T* R = G + D * S::QP;
  T* yl = R + S::QP;                    // NB
  const int64_t item = blockIdx.x;
  if (mode == 3 && b.skip && b.skip[item]) return;
  x += blockIdx.y * n_vec;
  y += blockIdx.y * n_vec;
  BatchView bv;
  bv.n_cells = b.n_items;
  bv.map = b.map;
  bv.coef = b.coef;
  bv.tail_off = b.tail_off;
  bv.tail_idx = b.tail_idx;
  bv.tail_coef = b.tail_coef;
  bv.local_out = b.local_out;
  bv.local_stride = b.local_stride;
  if (mode == 0)
    for (int i = threadIdx.x; i < S::NB; i += blockDim.x) xl[i] = gather_entry<T>(bv, item * S::NB + i, x);
  for (int i = lane; i < S::NB; i += 32) yl[i] = T(0);
  T hs[D];
  T det = T(1);
#pragma unroll
  for (int a = 0; a < D; ++a) {
    hs[a] = T(b.h[item * D + a]);
    det *= T(0.5) * hs[a];
  }
  __syncthreads();
  const int64_t s_begin = b.sub_off[item], s_end = b.sub_off[item + 1];
  for (int64_t s = s_begin + warp; s < s_end; s += kSubWarps) {
    const int lev = b.level[s];
    const T half = ldexp(T(1), -lev);
    T sc[D];  // d/dx = (1 / half) * (2 / h) d/d eta
#pragma unroll
    for (int a = 0; a < D; ++a) sc[a] = T(2) / (hs[a] * half);
    const uint64_t msk = b.mask[s];
    const T wsub = T(b.ws[s]) * det;
    // 1-D tables at the subcell's Gauss points
    for (int t = lane; t < D * Q; t += 32) {
      const int a = t / Q, j = t - a * Q;
      const T c = T(-1) + T(2 * b.pos[s * D + a] + 1) * half;
      T v[N], dv[N];
      fe_basis_dev<T>(c + half * tab.eta[j], N - 1, v, dv);
#pragma unroll
      for (int m = 0; m < N; ++m) {
        tb[a * N * Q + m * Q + j] = v[m];
        td[a * N * Q + m * Q + j] = dv[m] * T(2) / hs[a];
      }
    }
    __syncwarp();
    const T* Bx = tb;
    const T* By = tb + N * Q;
    const T* Bz = tb + 2 * N * Q;
    if (mode == 3) {
      // local diagonal: sum_p w_p (mass phi_i^2 + k |grad phi_i|^2) for the lane's modes
      for (int i = lane; i < S::NB; i += 32) {
        const int mi[3] = {i % N, (i / N) % N, D == 3 ? i / (N * N) : 0};
        T acc = T(0);
        for (int p = 0; p < S::QP; ++p) {
          if (!((msk >> p) & 1ull)) continue;
          const int pq[3] = {p % Q, (p / Q) % Q, D == 3 ? p / (Q * Q) : 0};
          T v[D], g[D];
#pragma unroll
          for (int a = 0; a < D; ++a) {
            v[a] = tb[a * N * Q + mi[a] * Q + pq[a]];
            g[a] = td[a * N * Q + mi[a] * Q + pq[a]];
          }
          T w = wsub;
#pragma unroll
          for (int a = 0; a < D; ++a) w *= tab.W[pq[a]];
          T phi = T(1), gg = T(0);
#pragma unroll
          for (int a = 0; a < D; ++a) phi *= v[a];
#pragma unroll
          for (int a = 0; a < D; ++a) {
            T ga = g[a];
#pragma unroll
            for (int e = 0; e < D; ++e)
              if (e != a) ga *= v[e];
            gg += ga * ga;
          }
          const T k = b.kpts ? kappa * T(b.kpts[s * S::QP + p]) : kappa;
          acc += w * (mass * phi * phi + k * gg);
        }
        yl[i] += acc;
      }
      __syncwarp();
      continue;
    }
    if (mode == 0) {
      // interpolation: (z), y, x stages
      const T* in = xl;
      if constexpr (D == 3) {
        for (int o = lane; o < S::A1; o += 32) {
          const int i = o % N, j = (o / N) % N, kq = o / (N * N);
          T acc = T(0);
#pragma unroll
          for (int k = 0; k < N; ++k) acc += Bz[k * Q + kq] * xl[i + N * (j + N * k)];
          a1[o] = acc;
        }
        __syncwarp();
        in = a1;
      }
      for (int o = lane; o < S::A2; o += 32) {
        const int i = o % N, jq = (o / N) % Q, kq = D == 3 ? o / (N * Q) : 0;
        T acc = T(0);
#pragma unroll
        for (int j = 0; j < N; ++j) acc += By[j * Q + jq] * in[i + N * (j + N * kq)];
        a2[o] = acc;
      }
      __syncwarp();
      for (int o = lane; o < S::QP; o += 32) {
        const int iq = o % Q, rest = o / Q;
        T acc = T(0);
#pragma unroll
        for (int i = 0; i < N; ++i) acc += Bx[i * Q + iq] * a2[i + N * rest];
        U[o] = acc;
      }
      __syncwarp();
      // collocation derivatives and the pointwise flux
      for (int o = lane; o < S::QP; o += 32) {
        const int pq[3] = {o % Q, (o / Q) % Q, D == 3 ? o / (Q * Q) : 0};
        T w = ((msk >> o) & 1ull) ? wsub : T(0);
#pragma unroll
        for (int a = 0; a < D; ++a) w *= tab.W[pq[a]];
        const T k = b.kpts ? kappa * T(b.kpts[s * S::QP + o]) : kappa;
        T g[D];
#pragma unroll
        for (int a = 0; a < D; ++a) {
          const int stride = a == 0 ? 1 : (a == 1 ? Q : Q * Q);
          const int base = o - pq[a] * stride;
          T acc = T(0);
#pragma unroll
          for (int l = 0; l < Q; ++l) acc += tab.Dm[pq[a] * Q + l] * U[base + l * stride];
          g[a] = acc * sc[a];
        }
        R[o] = w * mass * U[o];
#pragma unroll
        for (int a = 0; a < D; ++a) G[a * S::QP + o] = w * k * g[a];
      }
    } else {
      for (int o = lane; o < S::QP; o += 32) {
        const int pq[3] = {o % Q, (o / Q) % Q, D == 3 ? o / (Q * Q) : 0};
        T w = ((msk >> o) & 1ull) ? wsub : T(0);
#pragma unroll
        for (int a = 0; a < D; ++a) w *= tab.W[pq[a]];
        R[o] = src ? w * T(src[s * S::QP + o]) : T(0);
      }
    }
    __syncwarp();
    // transposed collocation derivatives into U (values only for the load)
    if (mode == 0) {
      for (int o = lane; o < S::QP; o += 32) {
        const int pq[3] = {o % Q, (o / Q) % Q, D == 3 ? o / (Q * Q) : 0};
        T acc = R[o];
#pragma unroll
        for (int a = 0; a < D; ++a) {
          const int stride = a == 0 ? 1 : (a == 1 ? Q : Q * Q);
          const int base = o - pq[a] * stride;
          T s2 = T(0);
#pragma unroll
          for (int l = 0; l < Q; ++l) s2 += tab.Dm[l * Q + pq[a]] * G[a * S::QP + base + l * stride];
          acc += s2 * sc[a];
        }
        U[o] = acc;
      }
    } else {
      for (int o = lane; o < S::QP; o += 32) U[o] = R[o];
    }
    __syncwarp();
    // transposed interpolation: x, y, (z) stages into the warp's local result
    for (int o = lane; o < S::A2; o += 32) {
      const int i = o % N, rest = o / N;
      T acc = T(0);
#pragma unroll
      for (int iq = 0; iq < Q; ++iq) acc += Bx[i * Q + iq] * U[iq + Q * rest];
      a2[o] = acc;
    }
    __syncwarp();
    if constexpr (D == 3) {
      for (int o = lane; o < S::A1; o += 32) {
        const int i = o % N, j = (o / N) % N, kq = o / (N * N);
        T acc = T(0);
#pragma unroll
        for (int jq = 0; jq < Q; ++jq) acc += By[j * Q + jq] * a2[i + N * (jq + Q * kq)];
        a1[o] = acc;
      }
      __syncwarp();
      for (int o = lane; o < S::NB; o += 32) {
        const int i = o % N, j = (o / N) % N, k = o / (N * N);
        T acc = T(0);
#pragma unroll
        for (int kq = 0; kq < Q; ++kq) acc += Bz[k * Q + kq] * a1[i + N * (j + N * kq)];
        yl[o] += acc;
      }
    } else {
      for (int o = lane; o < S::NB; o += 32) {
        const int i = o % N, j = o / N;
        T acc = T(0);
#pragma unroll
        for (int jq = 0; jq < Q; ++jq) acc += By[j * Q + jq] * a2[i + N * jq];
        yl[o] += acc;
      }
    }
    __syncwarp();
  }
  __syncthreads();
  // sum the warps' local results (the last NB entries of each warp's scratch) and scatter once
  for (int i = threadIdx.x; i < S::NB; i += blockDim.x) {
    T acc = T(0);
#pragma unroll
    for (int w = 0; w < kSubWarps; ++w) acc += xl[S::NB + w * S::WARP + S::WARP - S::NB + i];
    if (mode == 3) {
      const int v = b.map[item * S::NB + i];
      if (v >= 0) {
        const T c = b.coef ? T(b.coef[item * S::NB + i]) : T(1);
        atomicAdd(y + v, c * c * acc);
      }
    } else {
      scatter_entry<T>(bv, item * S::NB + i, acc, y);
    }
  }
}

}  // namespace grico
