// hp geometric multigrid V-cycle on the device (multigrid.jl:858-1087).
//
// Levels are device plans (coarse -> fine).  Transfers are the reduced-space prolongations
// P_l (coarse -> fine, CSR over fine rows); restriction uses the explicit transpose (CSR over
// coarse rows) so both directions are gathers without atomics.  Smoothers:
//   * damped Jacobi x += w D^-1 (b - A x)   — the reference's SPD smoother (multigrid.jl:943-956)
//   * Chebyshev-Jacobi of a given degree on [lambda_max*lower, 1.2*lambda_max] of D^-1 A, with
//     lambda_max from a power iteration at set-up — no reference counterpart.
//   * fixed-step right-Jacobi-preconditioned GMRES (multigrid.jl:963-1056) for non-SPD levels:
//     Arnoldi with modified Gram-Schmidt, Givens rotations and the back substitution run on the
//     device (one thread for the small Hessenberg work), so the V-cycle needs no host round trip.
// The coarsest level is solved in FP64 with the dense Cholesky factor of its reduced matrix
// (common.jl:272-330); the factor is inverted once on the host and applied as a dense
// matrix-vector product.
//
// Working precision: with GRICO_PREC_FP32 every level below the caller (smoother applies,
// residuals, transfers, Chebyshev/Jacobi updates) runs in FP32 on FP32 copies of D^-1 and of
// the transfer values; the caller's residual and correction stay FP64 (the outer Krylov
// iteration owns them) and the coarsest solve stays FP64.
#include <cuda_runtime.h>

#include <atomic>
#include <cmath>
#include <memory>
#include <vector>

#include "grico_host.h"
#include "grico_mg_internal.h"
#include "grico_plan_internal.h"
#include "vector_kernels.cuh"
#include "cnn_kernels.cuh"

// input channels of the tensor-core network: the 2 inputs padded to one K = 16 step
constexpr int kTcIn = 16;

struct GricoMultigrid {
  struct Transfer {
    int64_t nf = 0, nc = 0;
    grico::DevBuf p_off, p_idx, p_val;  // fine rows
    grico::DevBuf r_off, r_idx, r_val;  // coarse rows (transpose)
    grico::DevBuf p_val32, r_val32;     // FP32 copies (FP32 working precision)
  };
  std::vector<GricoPlan*> levels;
  std::vector<Transfer> xfer;
  std::vector<grico::DevBuf> dinv, b, x, r, t, d;           // FP64 level vectors
  std::vector<grico::DevBuf> dinv32, b32, x32, r32, t32, d32;  // FP32 level vectors
  grico::DevBuf coarse_b, coarse_x;                         // FP64 coarse solve in FP32 mode
  std::vector<double> lmax;
  grico::DevBuf coarse_inv;
  int64_t n0 = 0;
  GricoMGOptions opts{};
  cudaStream_t stream = nullptr;
  grico::DevBuf io_r, io_z;
  uint64_t identity = 0;  // see mg_identity
  // GMRES smoother: per smoothed level the Krylov basis V [(m+1) x n] and the preconditioned
  // directions Z [m x n] in the working precision; one small FP64 workspace shared by all levels
  std::vector<grico::DevBuf> gm_v, gm_z;
  grico::DevBuf gm_ws;
  // learned smoother sweep on one level (see learned_sweep)
  struct Learned {
    int level = -1;
    int nx = 0, ny = 0, nz = 0;
    int64_t n_grid = 0;
    double omega = 1.0;
    std::vector<int> ch;                 // channels at each layer boundary
    std::vector<grico::DevBuf> w, bias;  // FP32 weights [co][ci][27] and biases per layer
    grico::DevBuf idx;                   // grid point -> reduced dof (or -1)
    grico::DevBuf in, act0, act1;        // BF16 network input (channel 1: log coefficient) and activations
    // tensor-core path (every layer served by tcgen05): channels-last activations, the input
    // padded to kTcIn channels (0: residual, 1: log coefficient, others zero), packed weights
    bool tc = false;
    std::vector<grico::DevBuf> wp;
    grico::DevBuf out;                   // FP32 network output grid
    grico::DevBuf xn, tn, z;             // candidate iterate, its operator image, D^-1 r (level precision)
    grico::DevBuf stats;                 // [sweeps, accepted sweeps]
  } learned;
};

namespace grico {

namespace {

template <typename T>
__global__ void csr_gather(const int64_t* __restrict__ off, const int64_t* __restrict__ idx,
                           const T* __restrict__ val, const T* __restrict__ x, T* __restrict__ y,
                           int64_t nrows, int accumulate) {
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < nrows; i += int64_t(gridDim.x) * blockDim.x) {
    T s = T(0);
    for (int64_t t = off[i]; t < off[i + 1]; ++t) s += val[t] * x[idx[t]];
    y[i] = accumulate ? y[i] + s : s;
  }
}

// x += w * dinv * (b - ax)
// The smoothing kernels below read the level's operator product ax once; with `clear` they
// leave zeros in its place, so the next apply into that buffer need not zero it first.
template <typename T>
__global__ void jacobi_smooth(T* __restrict__ x, const T* __restrict__ b, T* __restrict__ ax,
                              const T* __restrict__ dinv, T w, int64_t n, bool clear) {
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) {
    x[i] += w * dinv[i] * (b[i] - ax[i]);
    if (clear) ax[i] = T(0);
  }
}

// First smoothing step from x = 0, whose apply is skipped: A 0 = 0, so b - ax is b and the
// damped-Jacobi step x += w dinv (b - ax) becomes x = w dinv b (the same values, bit for bit)
template <typename T>
__global__ void jacobi_from_zero(T* __restrict__ x, const T* __restrict__ b, const T* __restrict__ dinv, T w,
                                 T* __restrict__ clear, int64_t n) {
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) {
    x[i] = T(0) + w * dinv[i] * b[i];
    if (clear) clear[i] = T(0);
  }
}

// d = c1*d + c2*dinv*(b - ax); x += d
template <typename T>
__global__ void chebyshev_step(T* __restrict__ x, T* __restrict__ d, const T* __restrict__ b,
                               T* __restrict__ ax, const T* __restrict__ dinv, T c1, T c2, int64_t n, bool clear) {
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) {
    // the first step must not read d: fresh device memory may hold NaN bit patterns
    T di = (c1 != T(0) ? c1 * d[i] : T(0)) + c2 * dinv[i] * (b[i] - ax[i]);
    d[i] = di;
    x[i] += di;
    if (clear) ax[i] = T(0);
  }
}

// First Chebyshev step from x = 0 (apply skipped, as for jacobi_from_zero): d = x = c2 dinv b
template <typename T>
__global__ void chebyshev_from_zero(T* __restrict__ x, T* __restrict__ d, const T* __restrict__ b,
                                    const T* __restrict__ dinv, T c2, T* __restrict__ clear, int64_t n) {
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) {
    const T di = T(0) + c2 * dinv[i] * b[i];
    d[i] = di;
    x[i] = T(0) + di;
    if (clear) clear[i] = T(0);
  }
}

// Three-term Chebyshev step: nxt = x_k + c1 (x_k - x_{k-1}) + c2 dinv (b - A x_k), with x_k in
// `cur` and x_{k-1} in `nxt` (overwritten).  cur_zero: x_k = 0 (not read, and ax == nullptr:
// no apply); prev_zero: x_{k-1} = 0 (not read); c1 == 0 reads no x_{k-1} either.  With `clear`
// the product ax is zeroed after the read; `clear_t` (when ax is null) is zeroed instead.
template <typename T>
__global__ void chebyshev3_step(T* __restrict__ nxt, const T* __restrict__ cur, const T* __restrict__ b,
                                T* __restrict__ ax, const T* __restrict__ dinv, T c1, T c2, int64_t n,
                                bool cur_zero, bool prev_zero, bool clear, T* __restrict__ clear_t) {
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) {
    const T xk = cur_zero ? T(0) : cur[i];
    const T r = ax ? b[i] - ax[i] : b[i];
    const T prev = (c1 != T(0) && !prev_zero) ? nxt[i] : T(0);
    nxt[i] = xk + (c1 != T(0) ? c1 * (xk - prev) : T(0)) + c2 * dinv[i] * r;
    if (clear && ax) ax[i] = T(0);
    if (clear_t) clear_t[i] = T(0);
  }
}

// r = b - ax (ax cleared after the read with `clear`)
template <typename T>
__global__ void residual_kernel(T* __restrict__ r, const T* __restrict__ b, T* __restrict__ ax, int64_t n,
                                bool clear = false) {
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) {
    r[i] = b[i] - ax[i];
    if (clear) ax[i] = T(0);
  }
}

template <typename S, typename D>
__global__ void cast_kernel(const S* __restrict__ x, D* __restrict__ y, int64_t n) {
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x)
    y[i] = D(x[i]);
}

// y = M x for a dense row-major n x n matrix (one warp per row)
__global__ void dense_matvec(const double* __restrict__ M, const double* __restrict__ x, double* __restrict__ y, int64_t n) {
  const int lane = threadIdx.x & 31;
  const int64_t row = (blockIdx.x * int64_t(blockDim.x) + threadIdx.x) >> 5;
  if (row >= n) return;
  double s = 0.0;
  for (int64_t j = lane; j < n; j += 32) s += M[row * n + j] * x[j];
  for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  if (lane == 0) y[row] = s;
}

int blocks(int64_t n) { return int(std::min<int64_t>((n + 255) / 256, 148 * 8)); }

// Dense Cholesky A = L L^T in place (lower triangle), restating common.jl:272-300.
bool cholesky(std::vector<double>& a, int64_t n) {
  for (int64_t j = 0; j < n; ++j) {
    double s = a[j * n + j];
    for (int64_t k = 0; k < j; ++k) s -= a[j * n + k] * a[j * n + k];
    if (!(s > 0.0) || !std::isfinite(s)) return false;
    double ljj = std::sqrt(s);
    a[j * n + j] = ljj;
    for (int64_t i = j + 1; i < n; ++i) {
      double v = a[i * n + j];
      for (int64_t k = 0; k < j; ++k) v -= a[i * n + k] * a[j * n + k];
      a[i * n + j] = v / ljj;
    }
  }
  return true;
}

// Solve L L^T x = b on the host (common.jl:302-330)
void cholesky_solve(const std::vector<double>& l, int64_t n, std::vector<double>& x) {
  for (int64_t i = 0; i < n; ++i) {
    double v = x[i];
    for (int64_t k = 0; k < i; ++k) v -= l[i * n + k] * x[k];
    x[i] = v / l[i * n + i];
  }
  for (int64_t i = n - 1; i >= 0; --i) {
    double v = x[i];
    for (int64_t k = i + 1; k < n; ++k) v -= l[k * n + i] * x[k];
    x[i] = v / l[i * n + i];
  }
}

template <typename T>
struct LevelBufs;
template <>
struct LevelBufs<double> {
  static double* b(GricoMultigrid* m, int l) { return m->b[l].get<double>(); }
  static double* x(GricoMultigrid* m, int l) { return m->x[l].get<double>(); }
  static double* r(GricoMultigrid* m, int l) { return m->r[l].get<double>(); }
  static double* t(GricoMultigrid* m, int l) { return m->t[l].get<double>(); }
  static double* d(GricoMultigrid* m, int l) { return m->d[l].get<double>(); }
  static const double* dinv(GricoMultigrid* m, int l) { return m->dinv[l].get<double>(); }
  static const double* pval(GricoMultigrid::Transfer& X) { return X.p_val.get<double>(); }
  static const double* rval(GricoMultigrid::Transfer& X) { return X.r_val.get<double>(); }
};
template <>
struct LevelBufs<float> {
  static float* b(GricoMultigrid* m, int l) { return m->b32[l].get<float>(); }
  static float* x(GricoMultigrid* m, int l) { return m->x32[l].get<float>(); }
  static float* r(GricoMultigrid* m, int l) { return m->r32[l].get<float>(); }
  static float* t(GricoMultigrid* m, int l) { return m->t32[l].get<float>(); }
  static float* d(GricoMultigrid* m, int l) { return m->d32[l].get<float>(); }
  static const float* dinv(GricoMultigrid* m, int l) { return m->dinv32[l].get<float>(); }
  static const float* pval(GricoMultigrid::Transfer& X) { return X.p_val32.get<float>(); }
  static const float* rval(GricoMultigrid::Transfer& X) { return X.r_val32.get<float>(); }
};

template <typename T>
void level_apply(GricoMultigrid* mg, int l, const T* x, T* y, cudaStream_t st, bool y_zero = false) {
  run_apply<T>(mg->levels[l], true, x, y, 1, st, y_zero);
}

template <typename T>
void smooth_gmres(GricoMultigrid* mg, int l, T* x, const T* b, int steps, cudaStream_t st);

// x_zero: x holds no values yet and is taken as zero (Jacobi and Chebyshev only; the caller
// zeroes x for the GMRES smoother), so the first step skips its apply of x.
// t_zero (optional): whether the level's product buffer t holds zeros, kept up to date; the
// Jacobi and Chebyshev steps then clear t as they read it, and the next apply skips zeroing it.
template <typename T>
void smooth(GricoMultigrid* mg, int l, T* x, const T* b, int steps, cudaStream_t st, bool x_zero = false,
            bool* t_zero = nullptr) {
  using B = LevelBufs<T>;
  const int64_t n = mg->levels[l]->n_red;
  T* t = B::t(mg, l);
  const T* dinv = B::dinv(mg, l);
  if (steps <= 0) return;
  if (mg->opts.smoother == GRICO_SMOOTHER_GMRES) {
    smooth_gmres<T>(mg, l, x, b, steps, st);
    if (t_zero) *t_zero = false;
    return;
  }
  const bool clear = t_zero != nullptr;
  auto apply_t = [&](const T* v) {
    level_apply<T>(mg, l, v, t, st, clear && *t_zero);
    if (clear) *t_zero = false;
  };
  if (mg->opts.smoother == GRICO_SMOOTHER_JACOBI) {
    for (int s = 0; s < steps; ++s) {
      if (s == 0 && x_zero) {
        jacobi_from_zero<T><<<blocks(n), 256, 0, st>>>(x, b, dinv, T(mg->opts.jacobi_omega),
                                                       clear && !*t_zero ? t : nullptr, n);
      } else {
        apply_t(x);
        jacobi_smooth<T><<<blocks(n), 256, 0, st>>>(x, b, t, dinv, T(mg->opts.jacobi_omega), n, clear);
      }
      if (clear) *t_zero = true;
    }
    return;
  }
  const double lmax = 1.2 * mg->lmax[l];
  const double lmin = lmax * mg->opts.chebyshev_lower;
  const double theta = 0.5 * (lmax + lmin), delta = 0.5 * (lmax - lmin);
  const double sigma = theta / delta;
  T* d = B::d(mg, l);
  const int degree = mg->opts.chebyshev_degree;
  if (degree % 2 == 0) {
    // Even degree: the three-term form x_{k+1} = x_k + c1 (x_k - x_{k-1}) + c2 D^-1 (b - A x_k)
    // (the same recurrence, d_k = x_{k+1} - x_k), the iterates alternating between x and d, so
    // each step streams x_k, x_{k-1}, b, A x_k and D^-1 and writes x_{k+1}: one vector fewer
    // than the update form, and the sweep's last iterate lands in x.
    for (int s = 0; s < steps; ++s) {
      double rho_old = 1.0 / sigma;
      for (int k = 0; k < degree; ++k) {
        T* cur = (k % 2 == 0) ? x : d;
        T* nxt = (k % 2 == 0) ? d : x;
        const bool cur_zero = s == 0 && k == 0 && x_zero;
        const bool prev_zero = s == 0 && k == 1 && x_zero;
        if (!cur_zero) apply_t(cur);
        double c1 = 0.0, c2 = 1.0 / theta;
        if (k > 0) {
          const double rho = 1.0 / (2.0 * sigma - rho_old);
          c1 = rho * rho_old;
          c2 = 2.0 * rho / delta;
          rho_old = rho;
        }
        chebyshev3_step<T><<<blocks(n), 256, 0, st>>>(nxt, cur, b, cur_zero ? nullptr : t, dinv, T(c1), T(c2), n,
                                                      cur_zero, prev_zero, clear,
                                                      cur_zero && clear && !*t_zero ? t : nullptr);
        if (clear) *t_zero = true;
      }
    }
    return;
  }
  for (int s = 0; s < steps; ++s) {
    double rho_old = 1.0 / sigma;
    for (int k = 0; k < degree; ++k) {
      if (s == 0 && k == 0 && x_zero) {
        chebyshev_from_zero<T><<<blocks(n), 256, 0, st>>>(x, d, b, dinv, T(1.0 / theta),
                                                          clear && !*t_zero ? t : nullptr, n);
        if (clear) *t_zero = true;
        continue;
      }
      apply_t(x);
      if (k == 0) {
        chebyshev_step<T><<<blocks(n), 256, 0, st>>>(x, d, b, t, dinv, T(0), T(1.0 / theta), n, clear);
      } else {
        const double rho = 1.0 / (2.0 * sigma - rho_old);
        chebyshev_step<T><<<blocks(n), 256, 0, st>>>(x, d, b, t, dinv, T(rho * rho_old), T(2.0 * rho / delta), n,
                                                     clear);
        rho_old = rho;
      }
      if (clear) *t_zero = true;
    }
  }
}

// ---- GMRES smoother (multigrid.jl:963-1056) ----
// Small FP64 workspace: scalars, then H ((m+1) x m, column-major), g (m+1), cs, sn, y (m each).
enum GmresScalar { kGmBeta = 0, kGmNrm2 = 1, kGmNrm = 2, kGmStop = 3, kGmInner = 4, kGmSingular = 5, kGmScalars = 8 };
inline size_t gmres_ws_doubles(int m) { return size_t(kGmScalars) + size_t(m + 1) * m + size_t(m + 1) + 3 * size_t(m); }

// ws[kGmBeta] holds ||r||^2 on entry and beta = ||r|| on exit: g = (beta, 0, ...), H = 0; stop
// when beta == 0 (the smoother then leaves x unchanged, multigrid.jl:972)
__global__ void gm_start(double* ws, int m) {
  double* H = ws + kGmScalars;
  double* g = H + (m + 1) * m;
  for (int i = threadIdx.x; i < (m + 1) * m; i += blockDim.x) H[i] = 0.0;
  for (int i = threadIdx.x; i < m + 1; i += blockDim.x) g[i] = 0.0;
  if (threadIdx.x == 0) {
    const double beta = sqrt(ws[kGmBeta]);
    g[0] = beta;
    ws[kGmStop] = beta > 0.0 ? 0.0 : 1.0;
    ws[kGmInner] = 0.0;
    ws[kGmBeta] = beta;
  }
}

// ws[kGmNrm] = ||w|| from ws[kGmNrm2]
__global__ void gm_sqrt_into(double* ws) { ws[kGmNrm] = sqrt(ws[kGmNrm2]); }

// dst = src / *s (0 when *s == 0); the reference divides element by element
template <typename T>
__global__ void gm_divide(const T* __restrict__ src, T* __restrict__ dst, const double* __restrict__ s, int64_t n) {
  const double d = *s;
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x)
    dst[i] = d > 0.0 ? T(double(src[i]) / d) : T(0);
}

// w -= c v with c a device scalar (modified Gram-Schmidt step)
template <typename T>
__global__ void gm_axpy_neg(T* __restrict__ w, const T* __restrict__ v, const double* __restrict__ c, int64_t n) {
  const T a = T(*c);
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x)
    w[i] -= a * v[i];
}

// H[j+1, j] = ||w||, then the previous rotations, the new rotation of column j and its action
// on g (solve.jl:544-576); records the inner count and stops after a zero norm
__global__ void gm_givens(double* ws, int m, int j) {
  if (ws[kGmStop] != 0.0) return;
  double* H = ws + kGmScalars;
  double* g = H + (m + 1) * m;
  double* cs = g + (m + 1);
  double* sn = cs + m;
  double* col = H + size_t(m + 1) * j;
  const double nrm = ws[kGmNrm];
  col[j + 1] = nrm;
  for (int i = 0; i < j; ++i) {
    const double a = col[i], b = col[i + 1];
    col[i] = cs[i] * a + sn[i] * b;
    col[i + 1] = -sn[i] * a + cs[i] * b;
  }
  const double scale = hypot(col[j], col[j + 1]);
  const double c = scale == 0.0 ? 1.0 : col[j] / scale, s = scale == 0.0 ? 0.0 : col[j + 1] / scale;
  cs[j] = c;
  sn[j] = s;
  const double a = col[j], b = col[j + 1];
  col[j] = c * a + s * b;
  col[j + 1] = -s * a + c * b;
  const double ga = g[j], gb = g[j + 1];
  g[j] = c * ga + s * gb;
  g[j + 1] = -s * ga + c * gb;
  ws[kGmInner] = double(j + 1);
  if (nrm == 0.0) ws[kGmStop] = 1.0;
}

// back substitution of the rotated Hessenberg system; a zero or non-finite diagonal (the
// reference's ArgumentError, multigrid.jl:1048-1051) counts in ws[kGmSingular] and skips the update
__global__ void gm_solve(double* ws, int m) {
  double* H = ws + kGmScalars;
  double* g = H + (m + 1) * m;
  double* y = g + (m + 1) + 2 * m;
  const int inner = int(ws[kGmInner]);
  for (int row = inner - 1; row >= 0; --row) {
    double v = g[row];
    for (int col = row + 1; col < inner; ++col) v -= H[size_t(m + 1) * col + row] * y[col];
    const double d = H[size_t(m + 1) * row + row];
    if (!isfinite(d) || d == 0.0) {
      ws[kGmSingular] += 1.0;
      ws[kGmInner] = 0.0;
      return;
    }
    y[row] = v / d;
  }
}

// x += omega y_j z_j for j < inner, one column after the other
template <typename T>
__global__ void gm_update(T* __restrict__ x, const T* __restrict__ Z, const double* __restrict__ ws, int m, double omega,
                          int64_t n) {
  const double* y = ws + kGmScalars + (m + 1) * m + (m + 1) + 2 * m;
  const int inner = int(ws[kGmInner]);
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) {
    T xi = x[i];
    for (int j = 0; j < inner; ++j) {
      const T a = T(omega * y[j]);
      if (a != T(0)) xi += a * Z[size_t(j) * n + i];
    }
    x[i] = xi;
  }
}

template <typename T>
void smooth_gmres(GricoMultigrid* mg, int l, T* x, const T* b, int steps, cudaStream_t st) {
  using B = LevelBufs<T>;
  const int64_t n = mg->levels[l]->n_red;
  const int m = mg->opts.smoother_restart;
  const int count = int(std::min<int64_t>(std::min(steps, m), n));
  if (count <= 0) return;
  T* t = B::t(mg, l);
  T* r = B::r(mg, l);
  const T* dinv = B::dinv(mg, l);
  T* V = mg->gm_v[l].get<T>();
  T* Z = mg->gm_z[l].get<T>();
  double* ws = mg->gm_ws.get<double>();
  double* H = ws + kGmScalars;
  double* partial = mg->levels[l]->partial.get<double>();
  level_apply<T>(mg, l, x, t, st);
  residual_kernel<T><<<blocks(n), 256, 0, st>>>(r, b, t, n);
  dot_partial<T><<<kRedBlocks, kRedThreads, 0, st>>>(r, r, n, partial);
  reduce_final<<<1, kRedThreads, 0, st>>>(partial, kRedBlocks, ws + kGmBeta);
  gm_start<<<1, 128, 0, st>>>(ws, m);
  gm_divide<T><<<blocks(n), 256, 0, st>>>(r, V, ws + kGmBeta, n);
  for (int j = 0; j < count; ++j) {
    T* vj = V + size_t(j) * n;
    T* zj = Z + size_t(j) * n;
    scale_kernel<T><<<blocks(n), 256, 0, st>>>(dinv, vj, zj, n);  // z = D^-1 v
    level_apply<T>(mg, l, zj, t, st);                              // w = A z
    for (int i = 0; i <= j; ++i) {
      const T* vi = V + size_t(i) * n;
      double* hij = H + size_t(m + 1) * j + i;
      dot_partial<T><<<kRedBlocks, kRedThreads, 0, st>>>(t, vi, n, partial);
      reduce_final<<<1, kRedThreads, 0, st>>>(partial, kRedBlocks, hij);
      gm_axpy_neg<T><<<blocks(n), 256, 0, st>>>(t, vi, hij, n);
    }
    dot_partial<T><<<kRedBlocks, kRedThreads, 0, st>>>(t, t, n, partial);
    reduce_final<<<1, kRedThreads, 0, st>>>(partial, kRedBlocks, ws + kGmNrm2);
    gm_sqrt_into<<<1, 1, 0, st>>>(ws);
    gm_divide<T><<<blocks(n), 256, 0, st>>>(t, V + size_t(j + 1) * n, ws + kGmNrm, n);
    gm_givens<<<1, 1, 0, st>>>(ws, m, j);
  }
  gm_solve<<<1, 1, 0, st>>>(ws, m);
  gm_update<T><<<blocks(n), 256, 0, st>>>(x, Z, ws, m, mg->opts.jacobi_omega, n);
}

void coarse_solve(GricoMultigrid* mg, double* x, const double* b, cudaStream_t st) {
  const int64_t n = mg->levels[0]->n_red;
  if (n > 0) dense_matvec<<<int((n * 32 + 255) / 256), 256, 0, st>>>(mg->coarse_inv.get<double>(), b, x, n);
}

void coarse_solve(GricoMultigrid* mg, float* x, const float* b, cudaStream_t st) {
  // the coarsest solve stays FP64
  const int64_t n = mg->levels[0]->n_red;
  if (n == 0) return;
  cast_kernel<float, double><<<blocks(n), 256, 0, st>>>(b, mg->coarse_b.get<double>(), n);
  coarse_solve(mg, mg->coarse_x.get<double>(), mg->coarse_b.get<double>(), st);
  cast_kernel<double, float><<<blocks(n), 256, 0, st>>>(mg->coarse_x.get<double>(), x, n);
}

// s[1] = sqrt(s[0] / n) (the D^-1-weighted residual scale), s[2] = 1 / s[1] (0 if s[1] == 0)
__global__ void residual_scale(double* s, int64_t n) {
  const double sig = sqrt(s[0] / double(n > 0 ? n : 1));
  s[1] = sig;
  s[2] = sig > 0.0 ? 1.0 / sig : 0.0;
}

// accept the candidate iterate when its weighted residual norm is smaller
template <typename T>
__global__ void select_iterate(T* __restrict__ x, const T* __restrict__ xn, int64_t n, const double* __restrict__ s_old,
                               const double* __restrict__ s_new, unsigned long long* __restrict__ stats) {
  const bool accept = *s_new < *s_old;
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    stats[0] += 1;
    if (accept) stats[1] += 1;
  }
  if (!accept) return;
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x)
    x[i] = xn[i];
}

template <typename T>
T* lbuf(grico::DevBuf& b) { return b.get<T>(); }

// One learned smoother sweep on level l: r = b - A x, c = sigma * N(D^-1 r / sigma, log a) on the
// level's grid, x_new = x + omega c, kept only if ||b - A x_new||_{D^-1} < ||r||_{D^-1}, so the
// true residual judges every sweep and the plain iterate is the fallback.
template <typename T>
void learned_sweep(GricoMultigrid* mg, int l, T* x, const T* b, cudaStream_t st) {
  using B = LevelBufs<T>;
  auto& L = mg->learned;
  const int64_t n = mg->levels[l]->n_red;
  T* t = B::t(mg, l);
  T* r = B::r(mg, l);
  const T* dinv = B::dinv(mg, l);
  double* sc = mg->levels[l]->scalars.get<double>() + 8;  // [0] old norm^2, [1] sigma, [2] 1/sigma, [3] new norm^2
  double* partial = mg->levels[l]->partial.get<double>();
  level_apply<T>(mg, l, x, t, st);
  weighted_residual<T><<<kRedBlocks, 256, 0, st>>>(b, t, dinv, lbuf<T>(L.z), n, partial);  // z = D^-1 r
  reduce_final<<<1, kRedThreads, 0, st>>>(partial, kRedBlocks, sc);
  residual_scale<<<1, 1, 0, st>>>(sc, n);
  const int gb = int(std::min<int64_t>((L.n_grid + 255) / 256, 148 * 16));
  __nv_bfloat16* in = L.in.get<__nv_bfloat16>();
  const int nl = int(L.w.size());
  if (L.tc) {
    grid_gather_strided<T, __nv_bfloat16><<<gb, 256, 0, st>>>(L.idx.get<int64_t>(), L.n_grid, lbuf<T>(L.z), 1.0f,
                                                               sc + 2, in, kTcIn);
    const void* src = in;
    for (int k = 0; k < nl; ++k) {
      const int ci = k == 0 ? kTcIn : L.ch[k], co = L.ch[k + 1];
      const bool last = k + 1 == nl;
      void* dst = last ? L.out.ptr : ((k % 2 == 0) ? L.act0.ptr : L.act1.ptr);
      conv_tc_forward(src, L.wp[k].ptr, L.bias[k].get<float>(), dst, last ? 1 : 0, 1, ci, co, L.nz, L.ny, L.nx,
                      last ? 0 : 1, st);
      src = dst;
    }
  } else {
    grid_gather<T, __nv_bfloat16><<<gb, 256, 0, st>>>(L.idx.get<int64_t>(), L.n_grid, lbuf<T>(L.z), 1.0f, sc + 2, in);
    const __nv_bfloat16* src = in;
    for (int k = 0; k < nl; ++k) {
      const int ci = L.ch[k], co = L.ch[k + 1];
      const int tiles = ((L.nx + kConvTile - 1) / kConvTile) * ((L.ny + kConvTile - 1) / kConvTile) *
                        ((L.nz + kConvTile - 1) / kConvTile);
      const dim3 grid(tiles, (co + kConvCo - 1) / kConvCo, 1);
      if (k + 1 < nl) {
        __nv_bfloat16* dst = (k % 2 == 0) ? L.act0.get<__nv_bfloat16>() : L.act1.get<__nv_bfloat16>();
        conv3d_fwd<__nv_bfloat16, __nv_bfloat16><<<grid, 512, 0, st>>>(src, L.w[k].get<float>(), L.bias[k].get<float>(),
                                                                       dst, ci, co, L.nz, L.ny, L.nx, 1);
        src = dst;
      } else {
        conv3d_fwd<__nv_bfloat16, float><<<grid, 512, 0, st>>>(src, L.w[k].get<float>(), L.bias[k].get<float>(),
                                                               L.out.get<float>(), ci, co, L.nz, L.ny, L.nx, 0);
      }
    }
  }
  T* xn = lbuf<T>(L.xn);
  cudaMemcpyAsync(xn, x, sizeof(T) * n, cudaMemcpyDeviceToDevice, st);
  grid_scatter_add<float, T><<<gb, 256, 0, st>>>(L.idx.get<int64_t>(), L.n_grid, L.out.get<float>(), float(L.omega),
                                                 sc + 1, xn);
  T* tn = lbuf<T>(L.tn);
  level_apply<T>(mg, l, xn, tn, st);
  weighted_residual<T><<<kRedBlocks, 256, 0, st>>>(b, tn, dinv, lbuf<T>(L.z), n, partial);
  reduce_final<<<1, kRedThreads, 0, st>>>(partial, kRedBlocks, sc + 3);
  select_iterate<T><<<blocks(n), 256, 0, st>>>(x, xn, n, sc, sc + 3, L.stats.get<unsigned long long>());
}

template <typename T>
void vcycle(GricoMultigrid* mg, int l, T* x, const T* b, cudaStream_t st) {
  using B = LevelBufs<T>;
  const int64_t n = mg->levels[l]->n_red;
  if (l == 0) {
    coarse_solve(mg, x, b, st);
    return;
  }
  // the learned sweep replaces the last pre-smoothing step on its level
  const bool learned = mg->learned.level == l;
  const int pre = learned ? std::max(mg->opts.pre_steps - 1, 0) : mg->opts.pre_steps;
  // x starts at zero; Jacobi and Chebyshev take that as given in their first step instead of
  // applying the operator to a zeroed vector
  const bool from_zero = pre > 0 && mg->opts.smoother != GRICO_SMOOTHER_GMRES;
  if (!from_zero) cudaMemsetAsync(x, 0, sizeof(T) * n, st);
  // t (the level's product buffer) is cleared by the passes that read it, from the first
  // smoothing step on, so the applies of this level skip zeroing it
  bool t_zero = false;
  smooth<T>(mg, l, x, b, pre, st, from_zero, &t_zero);
  if (learned) {
    learned_sweep<T>(mg, l, x, b, st);
    t_zero = false;
  }
  T* t = B::t(mg, l);
  T* r = B::r(mg, l);
  level_apply<T>(mg, l, x, t, st, t_zero);
  residual_kernel<T><<<blocks(n), 256, 0, st>>>(r, b, t, n, true);
  t_zero = true;
  auto& X = mg->xfer[l - 1];
  T* bc = B::b(mg, l - 1);
  T* xc = B::x(mg, l - 1);
  csr_gather<T><<<blocks(X.nc), 256, 0, st>>>(X.r_off.get<int64_t>(), X.r_idx.get<int64_t>(), B::rval(X), r, bc, X.nc, 0);
  vcycle<T>(mg, l - 1, xc, bc, st);
  csr_gather<T><<<blocks(X.nf), 256, 0, st>>>(X.p_off.get<int64_t>(), X.p_idx.get<int64_t>(), B::pval(X), xc, x, X.nf, 1);
  smooth<T>(mg, l, x, b, mg->opts.post_steps, st, false, &t_zero);
}

}  // namespace

int mg_vcycle_device(GricoMultigrid* mg, const double* r, double* z, cudaStream_t st) {
  if (!mg) return GRICO_ERR_INVALID;
  const int L = int(mg->levels.size());
  if (mg->opts.precision == GRICO_PREC_FP32) {
    const int64_t n = mg->levels[L - 1]->n_red;
    float* b32 = mg->b32[L - 1].get<float>();
    float* x32 = mg->x32[L - 1].get<float>();
    cast_kernel<double, float><<<blocks(n), 256, 0, st>>>(r, b32, n);
    vcycle<float>(mg, L - 1, x32, b32, st);
    cast_kernel<float, double><<<blocks(n), 256, 0, st>>>(x32, z, n);
  } else {
    vcycle<double>(mg, L - 1, z, r, st);
  }
  return cuda_ok(cudaGetLastError(), "vcycle") ? GRICO_OK : GRICO_ERR_CUDA;
}

int mg_smoother(const GricoMultigrid* mg) { return mg ? mg->opts.smoother : -1; }

namespace {
std::atomic<uint64_t> g_mg_identity{1};
}
uint64_t mg_identity(const GricoMultigrid* mg) { return mg ? mg->identity : 0; }

uint64_t mg_epoch(const GricoMultigrid* mg) {
  uint64_t e = 0;
  if (mg)
    for (const GricoPlan* L : mg->levels) e += L->epoch;
  return e;
}

int prepare_jacobi(GricoPlan* P, cudaStream_t st);

}  // namespace grico

using namespace grico;

extern "C" {

int grico_mg_create(GricoPlan* const* levels, int nlevels, const GricoTransferDesc* transfers,
                    const double* coarse_matrix, const GricoMGOptions* opts, GricoMultigrid** out) {
  if (!levels || nlevels < 1 || !opts || !out || (nlevels > 1 && !transfers)) {
    set_error("grico_mg_create: invalid argument");
    return GRICO_ERR_INVALID;
  }
  if (opts->smoother != GRICO_SMOOTHER_JACOBI && opts->smoother != GRICO_SMOOTHER_CHEBYSHEV &&
      opts->smoother != GRICO_SMOOTHER_GMRES) {
    set_error("grico_mg_create: unknown smoother");
    return GRICO_ERR_INVALID;
  }
  if (opts->smoother == GRICO_SMOOTHER_GMRES &&
      (opts->smoother_restart < 1 || opts->smoother_restart > 64 ||
       opts->smoother_restart < std::max(opts->pre_steps, opts->post_steps))) {
    // multigrid.jl:352-358
    set_error("grico_mg_create: the GMRES smoother needs 1 <= smoother_restart <= 64 and smoother_restart >= "
              "max(pre_steps, post_steps)");
    return GRICO_ERR_INVALID;
  }
  if (opts->smoother == GRICO_SMOOTHER_CHEBYSHEV && (opts->chebyshev_degree < 1 || !(opts->chebyshev_lower > 0.0 && opts->chebyshev_lower < 1.0))) {
    set_error("grico_mg_create: Chebyshev degree must be >= 1 and the lower bound fraction in (0,1)");
    return GRICO_ERR_INVALID;
  }
  if (opts->precision != GRICO_PREC_FP64 && opts->precision != GRICO_PREC_FP32) {
    set_error("grico_mg_create: precision must be GRICO_PREC_FP64 or GRICO_PREC_FP32");
    return GRICO_ERR_INVALID;
  }
  std::unique_ptr<GricoMultigrid> mg(new GricoMultigrid());
  mg->opts = *opts;
  mg->identity = g_mg_identity.fetch_add(1);
  const bool fp32 = opts->precision == GRICO_PREC_FP32;
  mg->stream = levels[nlevels - 1]->stream;
  cudaStream_t st = mg->stream;
  for (int l = 0; l < nlevels; ++l) {
    if (!levels[l]) { set_error("grico_mg_create: null level"); return GRICO_ERR_INVALID; }
    mg->levels.push_back(levels[l]);
  }
  mg->dinv.resize(nlevels);
  mg->b.resize(nlevels);
  mg->x.resize(nlevels);
  mg->r.resize(nlevels);
  mg->t.resize(nlevels);
  mg->d.resize(nlevels);
  mg->lmax.assign(nlevels, 0.0);
  if (fp32) {
    mg->dinv32.resize(nlevels);
    mg->b32.resize(nlevels);
    mg->x32.resize(nlevels);
    mg->r32.resize(nlevels);
    mg->t32.resize(nlevels);
    mg->d32.resize(nlevels);
  }
  for (int l = 0; l < nlevels; ++l) {
    const int64_t n = std::max<int64_t>(levels[l]->n_red, 1);
    if (!mg->b[l].alloc(8 * n) || !mg->x[l].alloc(8 * n) || !mg->r[l].alloc(8 * n) || !mg->t[l].alloc(8 * n) ||
        !mg->d[l].alloc(8 * n))
      return GRICO_ERR_CUDA;
    if (l > 0) {
      int rc = prepare_jacobi(levels[l], st);
      if (rc) return rc;
      if (!mg->dinv[l].alloc(8 * n)) return GRICO_ERR_CUDA;
      cudaMemcpyAsync(mg->dinv[l].ptr, levels[l]->w_dinv.ptr, 8 * levels[l]->n_red, cudaMemcpyDeviceToDevice, st);
    }
    if (fp32) {
      if (!mg->b32[l].alloc(4 * n) || !mg->x32[l].alloc(4 * n) || !mg->r32[l].alloc(4 * n) ||
          !mg->t32[l].alloc(4 * n) || !mg->d32[l].alloc(4 * n) || !mg->dinv32[l].alloc(4 * n))
        return GRICO_ERR_CUDA;
      if (l > 0)
        cast_kernel<double, float><<<blocks(n), 256, 0, st>>>(mg->dinv[l].get<double>(), mg->dinv32[l].get<float>(),
                                                              levels[l]->n_red);
    }
  }
  if (fp32) {
    const int64_t n0 = std::max<int64_t>(levels[0]->n_red, 1);
    if (!mg->coarse_b.alloc(8 * n0) || !mg->coarse_x.alloc(8 * n0)) return GRICO_ERR_CUDA;
  }
  for (int l = 0; l + 1 < nlevels; ++l) {
    const GricoTransferDesc& T = transfers[l];
    if (T.n_fine != levels[l + 1]->n_red || T.n_coarse != levels[l]->n_red) {
      set_error("grico_mg_create: transfer sizes do not match the level plans");
      return GRICO_ERR_INVALID;
    }
    GricoMultigrid::Transfer X;
    X.nf = T.n_fine;
    X.nc = T.n_coarse;
    const int64_t nnz = T.row_offsets[T.n_fine];
    for (int64_t k = 0; k < nnz; ++k)
      if (T.col_index[k] < 0 || T.col_index[k] >= T.n_coarse) { set_error("transfer column out of range"); return GRICO_ERR_INVALID; }
    // transpose on the host (coarse rows), keeping fine-row order inside each coarse row
    std::vector<int64_t> roff(T.n_coarse + 1, 0), ridx(nnz);
    std::vector<double> rval(nnz);
    for (int64_t k = 0; k < nnz; ++k) roff[T.col_index[k] + 1]++;
    for (int64_t c = 0; c < T.n_coarse; ++c) roff[c + 1] += roff[c];
    std::vector<int64_t> fill(roff.begin(), roff.end() - 1);
    for (int64_t f = 0; f < T.n_fine; ++f)
      for (int64_t k = T.row_offsets[f]; k < T.row_offsets[f + 1]; ++k) {
        int64_t pos = fill[T.col_index[k]]++;
        ridx[pos] = f;
        rval[pos] = T.values[k];
      }
    bool ok = X.p_off.upload(T.row_offsets, size_t(T.n_fine + 1)) && X.p_idx.upload(T.col_index, size_t(nnz)) &&
              X.p_val.upload(T.values, size_t(nnz)) && X.r_off.upload(roff) && X.r_idx.upload(ridx) &&
              X.r_val.upload(rval);
    if (ok && fp32) {
      std::vector<float> pv(T.values, T.values + nnz), rv(rval.begin(), rval.end());
      ok = X.p_val32.upload(pv) && X.r_val32.upload(rv);
    }
    if (!ok) return GRICO_ERR_CUDA;
    mg->xfer.push_back(std::move(X));
  }
  // coarse matrix: given, or assembled by probing the coarsest reduced operator
  const int64_t n0 = levels[0]->n_red;
  mg->n0 = n0;
  if (n0 > 4096) { set_error("coarse level too large for the dense Cholesky solve (n > 4096)"); return GRICO_ERR_INVALID; }
  std::vector<double> A(n0 * n0, 0.0);
  if (coarse_matrix) {
    std::copy(coarse_matrix, coarse_matrix + n0 * n0, A.begin());
  } else if (n0 > 0) {
    DevBuf e, col;
    if (!e.alloc(8 * n0) || !col.alloc(8 * n0)) return GRICO_ERR_CUDA;
    std::vector<double> h(n0);
    for (int64_t j = 0; j < n0; ++j) {
      cudaMemsetAsync(e.ptr, 0, 8 * n0, st);
      double one = 1.0;
      cudaMemcpyAsync(e.get<double>() + j, &one, 8, cudaMemcpyHostToDevice, st);
      run_apply<double>(levels[0], true, e.get<double>(), col.get<double>(), 1, st);
      cudaMemcpyAsync(h.data(), col.ptr, 8 * n0, cudaMemcpyDeviceToHost, st);
      cudaStreamSynchronize(st);
      for (int64_t i = 0; i < n0; ++i) A[i * n0 + j] = h[i];
    }
  }
  if (n0 > 0) {
    // symmetrize check (multigrid.jl:400-420) then factor
    double scale = 0.0;
    for (double v : A) scale = std::max(scale, std::fabs(v));
    for (int64_t i = 0; i < n0; ++i)
      for (int64_t j = i + 1; j < n0; ++j)
        if (std::fabs(A[i * n0 + j] - A[j * n0 + i]) > 1.4901161193847656e-08 * scale) {
          set_error("declared SPD coarse multigrid matrix is not numerically symmetric");
          return GRICO_ERR_INVALID;
        }
    std::vector<double> Lf = A;
    if (!cholesky(Lf, n0)) { set_error("declared SPD coarse multigrid matrix is not positive definite"); return GRICO_ERR_INVALID; }
    std::vector<double> inv(n0 * n0);
    std::vector<double> col(n0);
    for (int64_t j = 0; j < n0; ++j) {
      std::fill(col.begin(), col.end(), 0.0);
      col[j] = 1.0;
      cholesky_solve(Lf, n0, col);
      for (int64_t i = 0; i < n0; ++i) inv[i * n0 + j] = col[i];
    }
    if (!mg->coarse_inv.upload(inv)) return GRICO_ERR_CUDA;
  }
  // GMRES smoother workspaces (multigrid.jl:163-176, 360-365)
  if (opts->smoother == GRICO_SMOOTHER_GMRES) {
    const int m = opts->smoother_restart;
    const size_t es = fp32 ? sizeof(float) : sizeof(double);
    mg->gm_v.resize(size_t(nlevels));
    mg->gm_z.resize(size_t(nlevels));
    for (int l = 1; l < nlevels; ++l) {
      const size_t n = size_t(std::max<int64_t>(levels[l]->n_red, 1));
      if (!mg->gm_v[size_t(l)].alloc(es * n * size_t(m + 1)) || !mg->gm_z[size_t(l)].alloc(es * n * size_t(m)))
        return GRICO_ERR_CUDA;
    }
    if (!mg->gm_ws.alloc(sizeof(double) * gmres_ws_doubles(m))) return GRICO_ERR_CUDA;
    cudaMemsetAsync(mg->gm_ws.ptr, 0, sizeof(double) * gmres_ws_doubles(m), st);
  }
  // Chebyshev: lambda_max(D^-1 A) per smoothed level by power iteration
  if (opts->smoother == GRICO_SMOOTHER_CHEBYSHEV) {
    for (int l = 1; l < nlevels; ++l) {
      const int64_t n = levels[l]->n_red;
      if (n == 0) continue;
      std::vector<double> v(n);
      uint64_t s = 0x9e3779b97f4a7c15ull + uint64_t(l);
      for (int64_t i = 0; i < n; ++i) {
        s ^= s << 13; s ^= s >> 7; s ^= s << 17;
        v[i] = 0.5 + double(s % 1000003) / 1000003.0;
      }
      double* x = mg->x[l].get<double>();
      double* t = mg->t[l].get<double>();
      cudaMemcpyAsync(x, v.data(), 8 * n, cudaMemcpyHostToDevice, st);
      double lam = 0.0;
      for (int it = 0; it < 20; ++it) {
        run_apply<double>(levels[l], true, x, t, 1, st);
        scale_kernel<double><<<blocks(n), 256, 0, st>>>(mg->dinv[l].get<double>(), t, t, n);
        double* sc_dev = levels[l]->scalars.get<double>() + 12;
        dot_partial<double><<<kRedBlocks, kRedThreads, 0, st>>>(t, t, n, levels[l]->partial.get<double>());
        reduce_final<<<1, kRedThreads, 0, st>>>(levels[l]->partial.get<double>(), kRedBlocks, sc_dev);
        dot_partial<double><<<kRedBlocks, kRedThreads, 0, st>>>(x, x, n, levels[l]->partial.get<double>());
        reduce_final<<<1, kRedThreads, 0, st>>>(levels[l]->partial.get<double>(), kRedBlocks, sc_dev + 1);
        double sc[2];
        cudaMemcpyAsync(sc, sc_dev, 16, cudaMemcpyDeviceToHost, st);
        cudaStreamSynchronize(st);
        const double tn = std::sqrt(sc[0]), xn = std::sqrt(sc[1]);
        if (!(tn > 0.0) || !(xn > 0.0)) break;
        lam = tn / xn;  // power-iteration estimate of the spectral radius of D^-1 A
        axpby_kernel<double><<<blocks(n), 256, 0, st>>>(1.0 / tn, t, 0.0, x, n);
      }
      mg->lmax[l] = lam;
    }
  }
  if (!cuda_ok(cudaStreamSynchronize(st), "mg create")) return GRICO_ERR_CUDA;
  *out = mg.release();
  return GRICO_OK;
}

int grico_mg_destroy(GricoMultigrid* mg) {
  delete mg;
  return GRICO_OK;
}

int grico_mg_vcycle(GricoMultigrid* mg, const double* r, double* z, int flags) {
  if (!mg || !r || !z) return GRICO_ERR_INVALID;
  cudaStream_t st = mg->stream;
  const int64_t n = mg->levels.back()->n_red;
  const double* rd = r;
  double* zd = z;
  if (flags & GRICO_FLAG_HOST_POINTERS) {
    if (!mg->io_r.ensure(8 * std::max<int64_t>(n, 1)) || !mg->io_z.ensure(8 * std::max<int64_t>(n, 1))) return GRICO_ERR_CUDA;
    cudaMemcpyAsync(mg->io_r.ptr, r, 8 * n, cudaMemcpyHostToDevice, st);
    rd = mg->io_r.get<double>();
    zd = mg->io_z.get<double>();
  }
  int rc = mg_vcycle_device(mg, rd, zd, st);
  if (rc) return rc;
  if (flags & GRICO_FLAG_HOST_POINTERS) cudaMemcpyAsync(z, zd, 8 * n, cudaMemcpyDeviceToHost, st);
  return cuda_ok(cudaStreamSynchronize(st), "vcycle") ? GRICO_OK : GRICO_ERR_CUDA;
}

int grico_mg_set_learned(GricoMultigrid* mg, const GricoLearnedDesc* d) {
  if (mg) mg->identity = g_mg_identity.fetch_add(1);  // the V-cycle changes
  if (!mg) return GRICO_ERR_INVALID;
  if (!d) {
    mg->learned = GricoMultigrid::Learned{};
    return GRICO_OK;
  }
  const int nlev = int(mg->levels.size());
  if (d->level < 1 || d->level >= nlev || d->nx < 1 || d->ny < 1 || d->nz < 1 || d->n_layers < 1 || !d->channels ||
      !d->weights || !d->biases || !d->grid_index || !d->grid_log_coefficient) {
    set_error("grico_mg_set_learned: invalid descriptor (the level must be a smoothed level, 1..levels-1)");
    return GRICO_ERR_INVALID;
  }
  if (d->channels[0] != 2 || d->channels[d->n_layers] != 1) {
    set_error("grico_mg_set_learned: the network maps 2 input channels (residual, log coefficient) to 1");
    return GRICO_ERR_INVALID;
  }
  const int64_t ng = int64_t(d->nx) * d->ny * d->nz;
  const int64_t n = mg->levels[d->level]->n_red;
  for (int64_t g = 0; g < ng; ++g)
    if (d->grid_index[g] < -1 || d->grid_index[g] >= n) {
      set_error("grico_mg_set_learned: grid index out of range");
      return GRICO_ERR_INVALID;
    }
  GricoMultigrid::Learned L;
  L.level = d->level;
  L.nx = d->nx;
  L.ny = d->ny;
  L.nz = d->nz;
  L.n_grid = ng;
  L.omega = d->omega;
  int maxc = 1;
  for (int k = 0; k <= d->n_layers; ++k) {
    if (d->channels[k] < 1 || d->channels[k] > 1024) { set_error("grico_mg_set_learned: bad channel count"); return GRICO_ERR_INVALID; }
    L.ch.push_back(d->channels[k]);
    maxc = std::max(maxc, d->channels[k]);
  }
  bool ok = L.idx.upload(d->grid_index, size_t(ng));
  L.w.resize(d->n_layers);
  L.bias.resize(d->n_layers);
  for (int k = 0; k < d->n_layers && ok; ++k)
    ok = L.w[k].upload(d->weights[k], size_t(L.ch[k + 1]) * L.ch[k] * 27) && L.bias[k].upload(d->biases[k], size_t(L.ch[k + 1]));
  // every layer on the tensor cores when the shapes allow: hidden widths multiples of 16 up to 128
  L.tc = true;
  for (int k = 0; k < d->n_layers; ++k) {
    const int ci = k == 0 ? kTcIn : L.ch[k], co = L.ch[k + 1];
    if (grico_conv_tc_weight_bytes(ci, co) < 0 || (k + 1 < d->n_layers && co % 16 != 0)) L.tc = false;
  }
  if (L.tc) {
    L.wp.resize(d->n_layers);
    for (int k = 0; k < d->n_layers && ok; ++k) {
      const int ci = k == 0 ? kTcIn : L.ch[k], co = L.ch[k + 1];
      grico::DevBuf padded;  // first layer: [co][kTcIn][27] with zero weights on the padding channels
      const float* wsrc = L.w[k].get<float>();
      if (k == 0) {
        std::vector<float> wpad(size_t(co) * kTcIn * 27, 0.0f);
        for (int o = 0; o < co; ++o)
          for (int i = 0; i < L.ch[0]; ++i)
            for (int t = 0; t < 27; ++t) wpad[(size_t(o) * kTcIn + i) * 27 + t] = d->weights[0][(size_t(o) * L.ch[0] + i) * 27 + t];
        ok = padded.upload(wpad.data(), wpad.size());
        wsrc = padded.get<float>();
      }
      ok = ok && L.wp[k].alloc(size_t(grico_conv_tc_weight_bytes(ci, co))) &&
           grico::conv_tc_pack(wsrc, ci, co, L.wp[k].ptr, mg->stream) == GRICO_OK &&
           cuda_ok(cudaStreamSynchronize(mg->stream), "pack learned weights");
    }
  }
  const int in_ch = L.tc ? kTcIn : 2;
  std::vector<__nv_bfloat16> coef(size_t(in_ch) * ng, __float2bfloat16(0.0f));
  // channel 1 of the input: channel-first [2][grid] or channels-last [grid][kTcIn]
  for (int64_t g = 0; g < ng; ++g)
    coef[L.tc ? g * kTcIn + 1 : ng + g] = __float2bfloat16(d->grid_log_coefficient[g]);
  const size_t vb = (mg->opts.precision == GRICO_PREC_FP32 ? 4 : 8) * size_t(std::max<int64_t>(n, 1));
  ok = ok && L.in.alloc(size_t(in_ch) * sizeof(__nv_bfloat16) * ng) && L.act0.alloc(sizeof(__nv_bfloat16) * maxc * ng) &&
       L.act1.alloc(sizeof(__nv_bfloat16) * maxc * ng) && L.out.alloc(sizeof(float) * ng) && L.xn.alloc(vb) &&
       L.tn.alloc(vb) && L.z.alloc(vb) && L.stats.alloc(2 * sizeof(unsigned long long));
  if (!ok) return GRICO_ERR_CUDA;
  cudaMemsetAsync(L.stats.ptr, 0, 2 * sizeof(unsigned long long), mg->stream);
  cudaMemcpyAsync(L.in.ptr, coef.data(), sizeof(__nv_bfloat16) * coef.size(), cudaMemcpyHostToDevice, mg->stream);
  if (!cuda_ok(cudaStreamSynchronize(mg->stream), "set learned")) return GRICO_ERR_CUDA;
  mg->learned = std::move(L);
  return GRICO_OK;
}

int grico_mg_learned_stats(GricoMultigrid* mg, int64_t* sweeps, int64_t* accepted) {
  if (!mg || mg->learned.level < 0) return GRICO_ERR_INVALID;
  unsigned long long h[2] = {0, 0};
  cudaMemcpyAsync(h, mg->learned.stats.ptr, sizeof(h), cudaMemcpyDeviceToHost, mg->stream);
  if (!cuda_ok(cudaStreamSynchronize(mg->stream), "learned stats")) return GRICO_ERR_CUDA;
  if (sweeps) *sweeps = int64_t(h[0]);
  if (accepted) *accepted = int64_t(h[1]);
  return GRICO_OK;
}

double grico_mg_lambda_max(GricoMultigrid* mg, int level) {
  if (!mg || level < 0 || level >= int(mg->lmax.size())) return -1.0;
  return mg->lmax[level];
}

}  // extern "C"
