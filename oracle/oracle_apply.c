/*
 * CPU oracle kernels — TEST INFRASTRUCTURE ONLY (parity checker and timed CPU baseline).
 *
 * Restates the reference's full-tensor cell apply for TestChannels(mass*u, kappa*k(x)*grad u):
 *   _accumulate_cell_accumulator_tensor_project!   accumulators.jl:1955-2013
 *   tensor_box_interpolate! / tensor_box_gradient! integration.jl:1184-1264 (D + D^2 contractions)
 *   tensor_box_project! / _project_gradient!       integration.jl:1315-1399 (transposes)
 *   gather / masked scatter                        assembly.jl:1751-1803
 * and the coloured, threaded traversal of _apply_pass! (assembly.jl:1350-1374): colours run in
 * sequence, the items of one colour are split over the threads (OpenMP static schedule in place
 * of Polyester's @batch per=thread).  Maps are single-term (conforming meshes); `map[e] < 0`
 * marks an inactive mode.
 */
#include <math.h>
#include <omp.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define MAXN 12

/* out[i..] = sum_k tab[k, i] in[... k ...] along one axis of a (n0,n1,n2) box; tab is [nin x nout]
 * row-major; axis a contracts nin -> nout. */
static void contract(const double* in, double* out, const int* shape_in, int axis, const double* tab, int nout,
                     int transpose) {
  int s[3] = {shape_in[0], shape_in[1], shape_in[2]};
  int nin = s[axis];
  int so[3] = {s[0], s[1], s[2]};
  so[axis] = nout;
  /* strides: axis 0 fastest */
  int stride_in = axis == 0 ? 1 : (axis == 1 ? s[0] : s[0] * s[1]);
  int stride_out = axis == 0 ? 1 : (axis == 1 ? so[0] : so[0] * so[1]);
  int outer = 1, inner = 1;
  for (int b = 0; b < axis; ++b) inner *= s[b];
  for (int b = axis + 1; b < 3; ++b) outer *= s[b];
  for (int o = 0; o < outer; ++o)
    for (int i = 0; i < inner; ++i) {
      const double* src = in + (int64_t)o * nin * inner + i;
      double* dst = out + (int64_t)o * nout * inner + i;
      for (int q = 0; q < nout; ++q) {
        double acc = 0.0;
        for (int k = 0; k < nin; ++k) acc += (transpose ? tab[q * nin + k] : tab[k * nout + q]) * src[k * stride_in];
        dst[q * stride_out] = acc;
      }
    }
  (void)stride_out;
}

/*
 * Apply the cell operator of `ncells` cells listed in `order` (colour ranges `color_off`).
 * B, G: [n x q] 1-D tables (values, reference derivatives); W: [q] weights; h: [ncells x dim];
 * map: [ncells x n^dim] single-term global indices (<0 inactive); kappa_pts: NULL or [ncells x q^dim].
 */
void oracle_tensor_apply(int dim, int n, int q, int64_t ncells, const int32_t* map, const double* h,
                         const double* B, const double* G, const double* W, double mass, double kappa,
                         const double* kappa_pts, int ncolors, const int64_t* color_off, const int64_t* order,
                         const double* x, double* y, int nthreads) {
  const int nb = dim == 3 ? n * n * n : (dim == 2 ? n * n : n);
  const int nq = dim == 3 ? q * q * q : (dim == 2 ? q * q : q);
  if (nthreads > 0) omp_set_num_threads(nthreads);
  for (int c = 0; c < ncolors; ++c) {
#pragma omp parallel
    {
      double xl[MAXN * MAXN * MAXN], u[MAXN * MAXN * MAXN], t1[MAXN * MAXN * MAXN], t2[MAXN * MAXN * MAXN];
      double g[3][MAXN * MAXN * MAXN], yl[MAXN * MAXN * MAXN];
      /* J^-1-scaled derivative tables per axis are formed per cell */
      double Gs[3][MAXN * MAXN];
#pragma omp for schedule(static)
      for (int64_t it = color_off[c]; it < color_off[c + 1]; ++it) {
        const int64_t cell = order[it];
        const int32_t* m = map + cell * nb;
        for (int i = 0; i < nb; ++i) xl[i] = m[i] >= 0 ? x[m[i]] : 0.0;
        double detJ = 1.0, sc[3] = {1, 1, 1};
        for (int a = 0; a < dim; ++a) {
          detJ *= 0.5 * h[cell * dim + a];
          sc[a] = 2.0 / h[cell * dim + a];
          for (int k = 0; k < n * q; ++k) Gs[a][k] = sc[a] * G[k];
        }
        int shape_n[3] = {n, dim >= 2 ? n : 1, dim >= 3 ? n : 1};
        /* values: B on every axis (tensor_box_interpolate!) */
        {
          int s[3] = {shape_n[0], shape_n[1], shape_n[2]};
          const double* src = xl;
          double* bufs[2] = {t1, t2};
          for (int a = 0; a < dim; ++a) {
            double* dst = (a == dim - 1) ? u : bufs[a % 2];
            contract(src, dst, s, a, B, q, 0);
            s[a] = q;
            src = dst;
          }
        }
        /* gradient: for each component axis a, G on a and B elsewhere (tensor_box_gradient!) */
        for (int ga = 0; ga < dim; ++ga) {
          int s[3] = {shape_n[0], shape_n[1], shape_n[2]};
          const double* src = xl;
          double* bufs[2] = {t1, t2};
          for (int a = 0; a < dim; ++a) {
            double* dst = (a == dim - 1) ? g[ga] : bufs[a % 2];
            contract(src, dst, s, a, a == ga ? Gs[a] : B, q, 0);
            s[a] = q;
            src = dst;
          }
        }
        /* pointwise accumulator: w*mass*u and w*kappa*grad u */
        for (int p = 0; p < nq; ++p) {
          int i0 = p % q, i1 = (p / q) % q, i2 = p / (q * q);
          double w = detJ * W[i0] * (dim >= 2 ? W[i1] : 1.0) * (dim >= 3 ? W[i2] : 1.0);
          double k = kappa * (kappa_pts ? kappa_pts[cell * nq + p] : 1.0);
          u[p] *= w * mass;
          for (int a = 0; a < dim; ++a) g[a][p] *= w * k;
        }
        /* project values and gradients back (transposed contractions) and sum */
        memset(yl, 0, sizeof(double) * nb);
        for (int comp = -1; comp < dim; ++comp) {
          int s[3] = {dim >= 1 ? q : 1, dim >= 2 ? q : 1, dim >= 3 ? q : 1};
          const double* src = comp < 0 ? u : g[comp];
          double* bufs[2] = {t1, t2};
          double tmp[MAXN * MAXN * MAXN];
          for (int a = 0; a < dim; ++a) {
            double* dst = (a == dim - 1) ? tmp : bufs[a % 2];
            /* tab is [n x q]; transpose contraction maps q -> n with tab[k*q + p] */
            const double* tab = (comp == a) ? Gs[a] : B;
            int nout = n;
            int sin_[3] = {s[0], s[1], s[2]};
            int stride_in = a == 0 ? 1 : (a == 1 ? sin_[0] : sin_[0] * sin_[1]);
            int inner = 1, outer = 1;
            for (int b = 0; b < a; ++b) inner *= sin_[b];
            for (int b = a + 1; b < 3; ++b) outer *= sin_[b];
            for (int o = 0; o < outer; ++o)
              for (int i = 0; i < inner; ++i) {
                const double* sp = src + (int64_t)o * sin_[a] * inner + i;
                double* dp = dst + (int64_t)o * nout * inner + i;
                for (int kk = 0; kk < nout; ++kk) {
                  double acc = 0.0;
                  for (int pp = 0; pp < sin_[a]; ++pp) acc += tab[kk * q + pp] * sp[pp * stride_in];
                  dp[kk * inner] = acc;
                }
              }
            s[a] = n;
            src = dst;
          }
          for (int i = 0; i < nb; ++i) yl[i] += tmp[i];
        }
        for (int i = 0; i < nb; ++i)
          if (m[i] >= 0 && yl[i] != 0.0) y[m[i]] += yl[i];
      }
    }
  }
}

int oracle_max_threads(void) { return omp_get_max_threads(); }
