// Thread-per-plane 3-D tensor-cell apply: the operator of cell_apply_3d_pipe (plain maps,
// constant coefficients, even-odd contractions) with far less shared-memory traffic.
//
// A block is one warp holding CPB = 32 / Q cells; lane (c, r) owns plane r of cell c.  In the
// "plane" layout a lane holds the Q x Q values of one z-plane of its cell in registers, so the x
// and y contractions run without any exchange; in the "slab" layout it holds one y-slab
// (z x x values), where the z and x contractions run in registers.  A cell's box changes layout
// through shared memory four times per apply:
//
//   plane (z-mode k):  modes -> x interpolation -> y interpolation          (registers)
//   slab  (y-point j): z interpolation; u, x- and z-fluxes and their transposed derivatives,
//                      plus the mass term: R = m u + Dx^T fx + Dz^T fz      (registers)
//   plane (z-point q): y-flux and Dy^T, then transposed y and x interpolation (registers)
//   slab  (y-mode j):  transposed z interpolation, then the scatter
//
// i.e. about 10 shared-memory accesses per point and apply instead of about 17 for the
// line-per-thread kernel (one line per contraction step), and six __syncwarp barriers instead
// of nine block barriers.  The gather is pipelined as in cell_apply_3d_pipe: while a warp
// computes group g, cp.async copies of x[map] for group g + G land in the stage and the map
// entries of group g + 2G land in a map stage.  The scatter re-reads its map entries from
// global memory (cached: they were staged two groups earlier).
//
// Shared-memory pitches: element (x, y, z) of cell c sits at c * cp + z * pz + y * Q + x in the
// work buffers and the mode stage.  The host searches pz and cp so that the 16 lanes of every
// half warp (8-byte elements; 32 lanes for 4-byte elements) hit different bank pairs in both the
// plane access (lane offsets c cp + r pz) and the slab access (c cp + r Q), and the map-stage
// pitch mp likewise for plane reads of int entries.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <vector>

#include "cell_pipe.cuh"

namespace grico {

struct PlaneLayout {
  int pz, cp, mp;
};

template <int Q>
struct PlaneShape {
  static constexpr int CPB = 32 / Q;  // cells per warp
  static constexpr int NT = CPB * Q;  // active lanes
};

namespace plane_detail {

// wavefronts of one access: lanes in windows of W, each window costs the largest number of
// distinct addresses sharing a bank residue
inline int wavefronts(const std::vector<long>& addr, int W) {
  int total = 0;
  for (size_t w0 = 0; w0 < addr.size(); w0 += size_t(W)) {
    std::vector<std::vector<long>> by(static_cast<size_t>(W));
    for (size_t l = w0; l < std::min(addr.size(), w0 + size_t(W)); ++l) {
      auto& v = by[size_t(addr[l] % W)];
      if (std::find(v.begin(), v.end(), addr[l]) == v.end()) v.push_back(addr[l]);
    }
    size_t worst = 0;
    for (auto& v : by) worst = std::max(worst, v.size());
    total += int(worst);
  }
  return total;
}

}  // namespace plane_detail

// Pitches of the plane kernel for (N, Q) and element size `elem` (4 or 8 bytes).
inline PlaneLayout make_plane_layout(int N, int Q, int elem) {
  using plane_detail::wavefronts;
  const int CPB = 32 / Q, NT = CPB * Q, W = 128 / elem;
  PlaneLayout best{Q * Q, Q * Q * Q, N * N * N};
  int best_cost = -1;
  std::vector<long> pl(static_cast<size_t>(NT)), sl(static_cast<size_t>(NT));
  for (int pz = Q * Q; pz < Q * Q + W; ++pz)
    for (int cp = pz * Q; cp < pz * Q + 2 * W; ++cp) {
      for (int t = 0; t < NT; ++t) {
        pl[size_t(t)] = long(t / Q) * cp + long(t % Q) * pz;
        sl[size_t(t)] = long(t / Q) * cp + long(t % Q) * Q;
      }
      const int cost = wavefronts(pl, W) + wavefronts(sl, W);
      if (best_cost < 0 || cost < best_cost) {
        best_cost = cost;
        best.pz = pz;
        best.cp = cp;
      }
    }
  // map stage: lane (c, k < N) reads the N^2 entries of mode plane k at c mp + k N^2 + e
  int best_m = -1;
  std::vector<long> ml;
  for (int mp = N * N * N; mp < N * N * N + 32; ++mp) {
    ml.clear();
    for (int t = 0; t < NT; ++t)
      if (t % Q < N) ml.push_back(long(t / Q) * mp + long(t % Q) * N * N);
    const int cost = wavefronts(ml, 32);
    if (best_m < 0 || cost < best_m) {
      best_m = cost;
      best.mp = mp;
    }
  }
  return best;
}

// staged cell sizes [CPB][4] and flux scales [CPB][4] (doubles), work buffers A and B and the
// mode stage (CPB * cp elements each), the map stage (CPB * mp ints)
inline size_t plane_smem_bytes(int CPB, const PlaneLayout& L, int elem) {
  return size_t(CPB) * 8 * 8 + size_t(3) * CPB * L.cp * elem + size_t(CPB) * L.mp * 4;
}

template <int N, int Q, typename T>
__global__ void __launch_bounds__(32) cell_apply_3d_plane(BatchView b, const Tables1D<N, Q, T> tab,
                                                          const TablesEO<N, Q, T> eo, const PlaneLayout lay,
                                                          const T* __restrict__ x, T* __restrict__ y, int64_t n_vec,
                                                          T mass, T kappa) {
  constexpr int CPB = PlaneShape<Q>::CPB;
  constexpr int NB = N * N * N;
  const int PZ = lay.pz, CP = lay.cp, MP = lay.mp;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double* hst = reinterpret_cast<double*>(smem_raw);   // [CPB][4] staged cell sizes
  double* scl = hst + CPB * 4;                          // [CPB][4] detJ sx^2, detJ sy^2, detJ sz^2, detJ
  T* bufA = reinterpret_cast<T*>(scl + CPB * 4);        // [CPB][cp]
  T* bufB = bufA + CPB * CP;                            // [CPB][cp]
  T* xst = bufB + CPB * CP;                             // [CPB][cp] staged modes of the next group
  int* mst = reinterpret_cast<int*>(xst + CPB * CP);    // [CPB][mp] staged map entries
  const int lane = threadIdx.x;
  const int c = lane / Q, r = lane % Q;
  const bool act = c < CPB;
  const int cb = c * CP;
  x += blockIdx.y * n_vec;
  y += blockIdx.y * n_vec;
  const int64_t n_groups = (int64_t(b.n_cells) + CPB - 1) / CPB;
  const int64_t G = gridDim.x;

  // map entries of mode plane r of every cell of group g into the map stage (-1 past the end)
  auto stage_map = [&](int64_t g) {
    if (!act || r >= N) return;
    const int64_t cell = g * CPB + c;
    int* ms = mst + c * MP + r * N * N;
    if (g < n_groups && cell < b.n_cells) {
      const int* src = b.map + cell * NB + r * N * N;
#pragma unroll
      for (int e = 0; e < N * N; ++e) cp_async_elem<4>(ms + e, src + e);
    } else {
#pragma unroll
      for (int e = 0; e < N * N; ++e) ms[e] = -1;
    }
  };
  // modes of group g (zeros for -1 entries) and cell sizes, from the staged map entries
  auto stage_x = [&](int64_t g) {
    if (!act) return;
    if (r < N) {
      const int* ms = mst + c * MP + r * N * N;
      T* xs = xst + cb + r * PZ;
#pragma unroll
      for (int yy = 0; yy < N; ++yy)
#pragma unroll
        for (int xx = 0; xx < N; ++xx) {
          const int m = ms[xx + N * yy];
          cp_async_zfill<sizeof(T)>(xs + Q * yy + xx, x + (m >= 0 ? m : 0), m >= 0);
        }
    }
    const int64_t cell = g * CPB + c;
    if (g < n_groups && cell < b.n_cells)
      for (int a = r; a < 3; a += Q) cp_async_elem<8>(hst + c * 4 + a, b.h + cell * 3 + a);  // Q = 2: two per lane
  };

  int64_t g = blockIdx.x;
  stage_map(g);
  cp_async_commit();
  cp_async_wait<0>();
  __syncwarp();
  stage_x(g);
  stage_map(g + G);
  cp_async_commit();
  for (; g < n_groups; g += G) {
    const int64_t cell = g * CPB + c;
    cp_async_wait<0>();
    __syncwarp();
    if (act && r == 0) {
      const bool ok = cell < b.n_cells;
      const double h0 = ok ? hst[c * 4 + 0] : 1.0, h1 = ok ? hst[c * 4 + 1] : 1.0, h2 = ok ? hst[c * 4 + 2] : 1.0;
      const double detJ = h0 * h1 * h2 * 0.125;
      scl[c * 4 + 0] = detJ * (2.0 / h0) * (2.0 / h0);
      scl[c * 4 + 1] = detJ * (2.0 / h1) * (2.0 / h1);
      scl[c * 4 + 2] = detJ * (2.0 / h2) * (2.0 / h2);
      scl[c * 4 + 3] = detJ;
    }
    // 1. plane (z-mode r): x interpolation of the N mode rows, y interpolation of the Q columns
    if (act && r < N) {
      T a[N][Q];
      {
        const T* xs = xst + cb + r * PZ;
#pragma unroll
        for (int yy = 0; yy < N; ++yy) {
          T md[N];
#pragma unroll
          for (int xx = 0; xx < N; ++xx) md[xx] = xs[Q * yy + xx];
          eo_interp(eo, md, a[yy]);
        }
      }
      T* wa = bufA + cb + r * PZ;
#pragma unroll
      for (int xx = 0; xx < Q; ++xx) {
        T col[N], o[Q];
#pragma unroll
        for (int yy = 0; yy < N; ++yy) col[yy] = a[yy][xx];
        eo_interp(eo, col, o);
#pragma unroll
        for (int yy = 0; yy < Q; ++yy) wa[Q * yy + xx] = o[yy];
      }
    }
    // the lanes are past their reads of the stages and of hst: refill them for the next groups
    __syncwarp();
    stage_x(g + G);
    stage_map(g + 2 * G);
    cp_async_commit();
    // 2. slab (y-point r): z interpolation, u, x- and z-fluxes with their transposed derivatives
    //    and the mass term
    {
      T u[Q][Q], R[Q][Q];  // [z][x]
      if (act) {
        const T* wa = bufA + cb + Q * r;
#pragma unroll
        for (int xx = 0; xx < Q; ++xx) {
          T col[N], o[Q];
#pragma unroll
          for (int zz = 0; zz < N; ++zz) col[zz] = wa[PZ * zz + xx];
          eo_interp(eo, col, o);
#pragma unroll
          for (int zz = 0; zz < Q; ++zz) u[zz][xx] = o[zz];
        }
        const double* sc = scl + c * 4;
        const T wr = tab.W[r];
        const T cx = kappa * T(sc[0]) * wr, cz = kappa * T(sc[2]) * wr, cm = mass * T(sc[3]) * wr;
#pragma unroll
        for (int zz = 0; zz < Q; ++zz) {
          T d[Q], t[Q];
          eo_deriv<Q>(eo.DS, eo.DD, u[zz], d);
#pragma unroll
          for (int xx = 0; xx < Q; ++xx) d[xx] *= cx * tab.W[xx] * tab.W[zz];
          eo_deriv<Q>(eo.TS, eo.TD, d, t);
#pragma unroll
          for (int xx = 0; xx < Q; ++xx) R[zz][xx] = cm * tab.W[xx] * tab.W[zz] * u[zz][xx] + t[xx];
        }
#pragma unroll
        for (int xx = 0; xx < Q; ++xx) {
          T col[Q], d[Q], t[Q];
#pragma unroll
          for (int zz = 0; zz < Q; ++zz) col[zz] = u[zz][xx];
          eo_deriv<Q>(eo.DS, eo.DD, col, d);
#pragma unroll
          for (int zz = 0; zz < Q; ++zz) d[zz] *= cz * tab.W[xx] * tab.W[zz];
          eo_deriv<Q>(eo.TS, eo.TD, d, t);
#pragma unroll
          for (int zz = 0; zz < Q; ++zz) R[zz][xx] += t[zz];
        }
      }
      __syncwarp();  // every lane is past its reads of buffer A
      if (act) {
        T* wa = bufA + cb + Q * r;
        T* wb = bufB + cb + Q * r;
#pragma unroll
        for (int zz = 0; zz < Q; ++zz)
#pragma unroll
          for (int xx = 0; xx < Q; ++xx) {
            wa[PZ * zz + xx] = u[zz][xx];
            wb[PZ * zz + xx] = R[zz][xx];
          }
      }
    }
    __syncwarp();
    // 3. plane (z-point r): y-flux and its transposed derivative, then transposed y and x
    //    interpolation
    {
      T M[N][N];
      if (act) {
        T u[Q][Q], R[Q][Q];  // [y][x]
        const T* wa = bufA + cb + r * PZ;
        const T* wb = bufB + cb + r * PZ;
#pragma unroll
        for (int yy = 0; yy < Q; ++yy)
#pragma unroll
          for (int xx = 0; xx < Q; ++xx) {
            u[yy][xx] = wa[Q * yy + xx];
            R[yy][xx] = wb[Q * yy + xx];
          }
        const T cy = kappa * T(scl[c * 4 + 1]) * tab.W[r];
        T P[N][Q];
#pragma unroll
        for (int xx = 0; xx < Q; ++xx) {
          T col[Q], d[Q], t[Q];
#pragma unroll
          for (int yy = 0; yy < Q; ++yy) col[yy] = u[yy][xx];
          eo_deriv<Q>(eo.DS, eo.DD, col, d);
#pragma unroll
          for (int yy = 0; yy < Q; ++yy) d[yy] *= cy * tab.W[xx] * tab.W[yy];
          eo_deriv<Q>(eo.TS, eo.TD, d, t);
#pragma unroll
          for (int yy = 0; yy < Q; ++yy) col[yy] = R[yy][xx] + t[yy];
          T o[N];
          eo_interp_t(eo, col, o);
#pragma unroll
          for (int yy = 0; yy < N; ++yy) P[yy][xx] = o[yy];
        }
#pragma unroll
        for (int yy = 0; yy < N; ++yy) eo_interp_t(eo, P[yy], M[yy]);
      }
      __syncwarp();  // every lane is past its reads of buffers A and B
      if (act) {
        T* wa = bufA + cb + r * PZ;
#pragma unroll
        for (int yy = 0; yy < N; ++yy)
#pragma unroll
          for (int xx = 0; xx < N; ++xx) wa[Q * yy + xx] = M[yy][xx];
      }
    }
    __syncwarp();
    // 4. slab (y-mode r): transposed z interpolation and the scatter
    if (act && r < N) {
      T m[N][N];  // [z][x]
      const T* wa = bufA + cb + Q * r;
#pragma unroll
      for (int xx = 0; xx < N; ++xx) {
        T col[Q], o[N];
#pragma unroll
        for (int zz = 0; zz < Q; ++zz) col[zz] = wa[PZ * zz + xx];
        eo_interp_t(eo, col, o);
#pragma unroll
        for (int zz = 0; zz < N; ++zz) m[zz][xx] = o[zz];
      }
      if (cell < b.n_cells) {
        const int* mp = b.map + cell * NB + N * r;
#pragma unroll
        for (int zz = 0; zz < N; ++zz)
#pragma unroll
          for (int xx = 0; xx < N; ++xx) {
            const int dof = __ldg(mp + N * N * zz + xx);
            if (dof >= 0) atomicAdd(y + dof, m[zz][xx]);
          }
      }
    }
  }
  cp_async_wait<0>();
}

}  // namespace grico
