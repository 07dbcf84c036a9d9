// Persistent, software-pipelined 3-D tensor-cell apply with bank-conflict-free line
// assignment (operator apply of cell_apply_3d, same contraction schedule and results up to
// rounding).
//
// A block of NT = Q*Q*CPB threads walks groups of CPB cells (group g, g + gridDim.x, ...).
// While it computes group g, cp.async copies of x[map[e]] for the next group land in the
// other shared stage and the map entries of the group after that are in flight into
// registers, so the gather's two dependent global round trips overlap a whole group's
// contractions.  The kernel serves plain maps only (every entry a dof or -1, no coefficients,
// no tail expansions): the gather is branch-free (a zero-filling copy for -1 entries) and the
// map entries are staged beside the modes, so the scatter reads them from shared memory.
// Batches with hanging-node tails, coefficients or pointwise mass use cell_apply_3d.
//
// Every contraction step gives each thread one whole line of a cell's Q^3 point box (x-, y- or
// z-line), as in cell_apply_3d.  Which line a thread takes is not tied to its own cell: for each
// of the three line shapes the host computes a lane -> (cell, line) table so that the 16 lanes
// of every half warp (8-byte elements; 32 lanes for 4-byte elements) touch 16 different
// shared-memory bank pairs, with the per-cell buffer pitch chosen by the same search.  With
// the plain (cell-own) assignment every other shared-memory access of a 5^3 cell replays once.
// With a constant coefficient the pointwise flux scaling is folded into the x and y derivative
// steps.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <cmath>
#include <vector>

#include "cell_kernels.cuh"

namespace grico {

// Asynchronous global -> shared copies of one element (cp.async, sm_80+): the copy runs while
// the issuing thread goes on; cp.async.wait_group makes the thread's own copies complete.
template <int BYTES>
__device__ __forceinline__ void cp_async_elem(void* smem_dst, const void* gsrc) {
  const unsigned dst = static_cast<unsigned>(__cvta_generic_to_shared(smem_dst));
  asm volatile("cp.async.ca.shared.global [%0], [%1], %2;\n" ::"r"(dst), "l"(gsrc), "n"(BYTES) : "memory");
}
// Same with a source size of BYTES or 0: with 0 the destination is filled with zeros and the
// source is not read.
template <int BYTES>
__device__ __forceinline__ void cp_async_zfill(void* smem_dst, const void* gsrc, bool read) {
  const unsigned dst = static_cast<unsigned>(__cvta_generic_to_shared(smem_dst));
  const unsigned src_bytes = read ? unsigned(BYTES) : 0u;
  asm volatile("cp.async.ca.shared.global [%0], [%1], %2, %3;\n" ::"r"(dst), "l"(gsrc), "n"(BYTES), "r"(src_bytes)
               : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int PENDING>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(PENDING) : "memory");
}

// Returns v through an opaque register move: the compiler keeps the value in a register (or
// spills it) rather than recomputing it from its operands.
__device__ __forceinline__ int keep_reg(int v) {
  asm volatile("mov.b32 %0, %0;" : "+r"(v));
  return v;
}
__device__ __forceinline__ double keep_reg(double v) {
  asm volatile("mov.b64 %0, %0;" : "+d"(v));
  return v;
}
__device__ __forceinline__ float keep_reg(float v) {
  asm volatile("mov.b32 %0, %0;" : "+f"(v));
  return v;
}

// Line shapes of a Q^3 box stored x fastest (element (ix, iy, iz) at ix + Q iy + Q^2 iz):
// z-lines are indexed by (a, b) = (x, y), y-lines by (x, z), x-lines by (y, z).
enum LineShape { kLineX = 0, kLineY = 1, kLineZ = 2 };

// Lane -> line table of one kernel shape: v[shape][lane] = cell | a << 7 | b << 11; bp = element
// pitch of a per-cell work buffer, sp = pitch between staged cells, pz = pitch between the
// z-planes of a cell's point box in the work buffer (Q*Q, or padded).
template <int NT>
struct LaneLines {
  int bp, sp, pz;
  uint16_t v[3][NT];
};

namespace lanes_detail {

inline int line_offset(int shape, int a, int b, int Q, int pz) {
  return shape == kLineZ ? a + Q * b : shape == kLineY ? a + pz * b : Q * a + pz * b;
}

// Shared-memory wavefronts of one access step: lanes grouped in windows of W, each window
// costs the largest number of distinct addresses that share one bank residue.
inline int window_cost(const std::vector<long>& addr, const std::vector<char>& active, int W) {
  int total = 0;
  const int n = int(addr.size());
  for (int w0 = 0; w0 < n; w0 += W) {
    std::vector<std::vector<long>> by(W);
    for (int l = w0; l < std::min(n, w0 + W); ++l)
      if (active[l]) {
        auto& v = by[size_t(addr[l] % W)];
        if (std::find(v.begin(), v.end(), addr[l]) == v.end()) v.push_back(addr[l]);
      }
    size_t worst = 0;
    for (auto& v : by) worst = std::max(worst, v.size());
    total += int(worst);
  }
  return total;
}

// Greedy assignment of all CPB*Q*Q lines of one shape to lanes: each window takes lines of
// distinct residues, the residue with most lines left first.  Returns the assignment (line
// ids c*Q*Q + a + Q*b) and its cost.
inline int assign_shape(int shape, int Q, int pz, int CPB, int pitch, int W, std::vector<int>& out) {
  const int T = Q * Q, NT = T * CPB;
  std::vector<std::vector<int>> pool(W);
  for (int c = CPB - 1; c >= 0; --c)
    for (int t = T - 1; t >= 0; --t) {
      const long a = long(c) * pitch + line_offset(shape, t % Q, t / Q, Q, pz);
      pool[size_t(a % W)].push_back(c * T + t);
    }
  out.assign(size_t(NT), 0);
  int cost = 0;
  for (int w0 = 0; w0 < NT; w0 += W) {
    std::vector<char> used(size_t(W), 0);
    std::vector<int> count(size_t(W), 0);
    for (int l = w0; l < std::min(NT, w0 + W); ++l) {
      int best = -1;
      for (int pass = 0; pass < 2 && best < 0; ++pass)
        for (int r = 0; r < W; ++r)
          if (!pool[size_t(r)].empty() && (pass == 1 || !used[size_t(r)]) &&
              (best < 0 || pool[size_t(r)].size() > pool[size_t(best)].size()))
            best = r;
      out[size_t(l)] = pool[size_t(best)].back();
      pool[size_t(best)].pop_back();
      used[size_t(best)] = 1;
      ++count[size_t(best)];
    }
    cost += *std::max_element(count.begin(), count.end());
  }
  return cost;
}

}  // namespace lanes_detail

// Builds the lane tables for (N, Q, CPB) and element size `elem` (4 or 8 bytes) for the fewest
// wavefronts (W = 128 / elem lanes per window): the stage pitch sp in [N^3, N^3 + W) and, with
// three work buffers per cell (cell pitch 3 bp), the buffer pitch bp in [Q^3, Q^3 + 2W) at the
// plain plane pitch pz = Q^2; with one work buffer per cell (`single`), also the plane pitch pz in
// [Q^2, Q^2 + W), bp in [pz Q, pz Q + 2W).  The padded plane pitch spreads the cells' lines over
// all banks where the plain box cannot: e.g. FP32 q = 4 / 5 / 8 need 12 / 13 / 24 wavefronts for
// the three line shapes instead of 15 / 15 / 40.  The search takes 15-230 ms per shape on the
// host, once per process.  v: [3][Q*Q*CPB].
inline void build_lane_lines(int N, int Q, int CPB, int elem, bool single, int* bp_out, int* sp_out, int* pz_out,
                             uint16_t* v) {
  using namespace lanes_detail;
  const int W = 128 / elem, T = Q * Q, NT = Q * Q * CPB;
  int best_cost = -1;
  std::vector<std::vector<int>> tmp(3), keep(3);
  const int pz_end = single ? Q * Q + W : Q * Q + 1;
  for (int pz = Q * Q; pz < pz_end; ++pz)
    for (int bp = pz * Q; bp < pz * Q + 2 * W; ++bp) {
      int cost = 0;
      for (int s = 0; s < 3; ++s) cost += assign_shape(s, Q, pz, CPB, single ? bp : 3 * bp, W, tmp[size_t(s)]);
      if (best_cost < 0 || cost < best_cost) {
        best_cost = cost;
        *bp_out = bp;
        *pz_out = pz;
        keep = tmp;
      }
    }
  // stage pitch: step 1 reads N staged modes along each active z-line
  const std::vector<int>& zl = keep[2];
  int best_sp = N * N * N, sp_cost = -1;
  std::vector<long> addr(size_t(NT), 0);
  std::vector<char> act(size_t(NT), 0);
  for (int sp = N * N * N; sp < N * N * N + W; ++sp) {
    for (int l = 0; l < NT; ++l) {
      const int id = zl[size_t(l)];
      const int c = id / T, a = (id % T) % Q, b = (id % T) / Q;
      addr[size_t(l)] = static_cast<long>(c) * sp + a + N * b;
      act[size_t(l)] = static_cast<char>(a < N && b < N);
    }
    const int cost = window_cost(addr, act, W);
    if (sp_cost < 0 || cost < sp_cost) {
      sp_cost = cost;
      best_sp = sp;
    }
  }
  *sp_out = best_sp;
  for (int s = 0; s < 3; ++s)
    for (int l = 0; l < NT; ++l) {
      const int id = keep[size_t(s)][size_t(l)];
      const int c = id / T, a = (id % T) % Q, b = (id % T) / Q;
      v[s * NT + l] = static_cast<uint16_t>(c | (a << 7) | (b << 11));
    }
}

template <int NT>
LaneLines<NT> make_lane_lines(int N, int Q, int CPB, int elem, bool single) {
  LaneLines<NT> L{};
  build_lane_lines(N, Q, CPB, elem, single, &L.bp, &L.sp, &L.pz, &L.v[0][0]);
  return L;
}

// Shared-memory bytes of cell_apply_3d_pipe: two stages of cell sizes (4 doubles per cell), the
// per-cell flux scales (4 doubles), nbuf work buffers of bp elements per cell (3, or 1 for the
// even-odd kernel, whose fluxes live in registers), two stages of sp staged modes per cell and
// two stages of sp staged map entries (int32) per cell.
inline size_t pipe_smem_bytes(int CPB, int bp, int sp, int elem, int nbuf) {
  return size_t(2) * CPB * 4 * 8 + size_t(CPB) * 4 * 8 + size_t(2) * CPB * sp * 4 +
         size_t(nbuf) * CPB * bp * elem + size_t(2) * CPB * sp * elem;
}

// Even-odd form of the 1-D contractions.  Gauss points are mirrored (xi_{Q-1-q} = -xi_q), the
// integrated Legendre modes k >= 2 have parity (-1)^k, the two vertex modes map onto each other
// (psi_0(-x) = psi_1(x)), and the collocation derivative is centro-antisymmetric
// (D[Q-1-q][Q-1-l] = -D[q][l]).  So a line splits into its symmetric and antisymmetric halves:
// modes into the even set {psi_0 + psi_1 (as (psi_0+psi_1)/2 with coefficient c0 + c1),
// psi_2, psi_4, ...} and the odd set {(psi_1-psi_0)/2 with coefficient c1 - c0, psi_3, ...};
// points into sums and differences of mirrored pairs.  Each half is a contraction over half the
// points, so an N x Q contraction costs about N*Q/2 FMAs plus Q adds, and its dependent chains
// are half as long.  (Kopriva's even-odd decomposition; the reference contracts directly,
// integration.jl:995-1136.)
template <int N, int Q, typename T>
struct TablesEO {
  static constexpr int QH = (Q + 1) / 2;   // points of the left half, centre included
  static constexpr int QL = Q / 2;         // mirrored pairs
  static constexpr int NE = 1 + (N - 1) / 2;  // even modes: vertex sum, psi_2, psi_4, ...
  static constexpr int NO = 1 + (N - 2) / 2;  // odd modes: vertex difference, psi_3, ...
  T BE[NE * QH];  // BE[e*QH+q]: even mode e at point q (vertex sum: (psi_0 + psi_1) / 2)
  T BO[NO * QL];  // BO[o*QL+q]: odd mode o at point q (vertex difference: (psi_1 - psi_0) / 2)
  T DS[QL * QH];  // derivative rows q < QL on pair sums: (D[q][l] + D[q][Q-1-l]) / 2, centre D[q][c]
  T DD[QH * QL];  // derivative rows q < QH on pair differences: (D[q][l] - D[q][Q-1-l]) / 2
  T TS[QL * QH];  // the same for the transposed derivative D^T
  T TD[QH * QL];
};

// Even-odd tables from the plain ones; false when the tables lack the symmetry (then the plain
// contractions run).
template <int N, int Q, typename T>
bool make_eo_tables(const double* B, const double* D, TablesEO<N, Q, T>& t) {
  using E = TablesEO<N, Q, T>;
  constexpr int QH = E::QH, QL = E::QL;
  double scale = 0.0;
  for (int i = 0; i < N * Q; ++i) scale = std::max(scale, std::abs(B[i]));
  for (int i = 0; i < Q * Q; ++i) scale = std::max(scale, std::abs(D[i]));
  const double tol = 1e-13 * std::max(scale, 1.0);
  for (int q = 0; q < Q; ++q) {
    if (N < 2 || std::abs(B[0 * Q + Q - 1 - q] - B[1 * Q + q]) > tol) return false;
    for (int k = 2; k < N; ++k)
      if (std::abs(B[k * Q + Q - 1 - q] - ((k & 1) ? -1.0 : 1.0) * B[k * Q + q]) > tol) return false;
    for (int l = 0; l < Q; ++l)
      if (std::abs(D[(Q - 1 - q) * Q + Q - 1 - l] + D[q * Q + l]) > tol) return false;
  }
  for (int q = 0; q < QH; ++q) {
    t.BE[q] = T(0.5 * (B[0 * Q + q] + B[1 * Q + q]));
    for (int k = 2; k < N; k += 2) t.BE[(k / 2) * QH + q] = T(B[k * Q + q]);
  }
  for (int q = 0; q < QL; ++q) {
    t.BO[q] = T(0.5 * (B[1 * Q + q] - B[0 * Q + q]));
    for (int k = 3; k < N; k += 2) t.BO[((k - 1) / 2) * QL + q] = T(B[k * Q + q]);
  }
  auto split = [&](auto at, T* S, T* Dd) {
    for (int q = 0; q < QL; ++q)
      for (int l = 0; l < QH; ++l)
        S[q * QH + l] = T(l < QL ? 0.5 * (at(q, l) + at(q, Q - 1 - l)) : at(q, l));
    for (int q = 0; q < QH; ++q)
      for (int l = 0; l < QL; ++l) Dd[q * QL + l] = T(0.5 * (at(q, l) - at(q, Q - 1 - l)));
  };
  split([&](int q, int l) { return D[q * Q + l]; }, t.DS, t.DD);
  split([&](int q, int l) { return D[l * Q + q]; }, t.TS, t.TD);
  return true;
}

// out[q] = sum_k psi_k(xi_q) in[k]
template <int N, int Q, typename T>
__device__ __forceinline__ void eo_interp(const TablesEO<N, Q, T>& t, const T (&in)[N], T (&out)[Q]) {
  using E = TablesEO<N, Q, T>;
  constexpr int QH = E::QH, QL = E::QL, NE = E::NE, NO = E::NO;
  T ev[NE], od[NO];
  ev[0] = in[0] + in[1];
  od[0] = in[1] - in[0];
#pragma unroll
  for (int k = 2; k < N; ++k) {  // even k: ev[k/2]; odd k: od[(k-1)/2] (both in range for any k < N)
    if (k & 1) od[(k - 1) / 2] = in[k];
    else ev[k / 2] = in[k];
  }
  T e[QH];
#pragma unroll
  for (int q = 0; q < QH; ++q) {
    T v = T(0);
#pragma unroll
    for (int i = 0; i < NE; ++i) v += t.BE[i * QH + q] * ev[i];
    e[q] = v;
  }
#pragma unroll
  for (int q = 0; q < QL; ++q) {
    T v = T(0);
#pragma unroll
    for (int i = 0; i < NO; ++i) v += t.BO[i * QL + q] * od[i];
    out[q] = e[q] + v;
    out[Q - 1 - q] = e[q] - v;
  }
  if constexpr ((Q & 1) != 0) out[QL] = e[QL];
}

// out[k] = sum_q psi_k(xi_q) in[q]
template <int N, int Q, typename T>
__device__ __forceinline__ void eo_interp_t(const TablesEO<N, Q, T>& t, const T (&in)[Q], T (&out)[N]) {
  using E = TablesEO<N, Q, T>;
  constexpr int QH = E::QH, QL = E::QL, NE = E::NE, NO = E::NO;
  T sm[QH], df[QL > 0 ? QL : 1];
#pragma unroll
  for (int q = 0; q < QL; ++q) {
    sm[q] = in[q] + in[Q - 1 - q];
    df[q] = in[q] - in[Q - 1 - q];
  }
  if constexpr ((Q & 1) != 0) sm[QL] = in[QL];
  T ev[NE], od[NO];
#pragma unroll
  for (int i = 0; i < NE; ++i) {
    T v = T(0);
#pragma unroll
    for (int q = 0; q < QH; ++q) v += t.BE[i * QH + q] * sm[q];
    ev[i] = v;
  }
#pragma unroll
  for (int i = 0; i < NO; ++i) {
    T v = T(0);
#pragma unroll
    for (int q = 0; q < QL; ++q) v += t.BO[i * QL + q] * df[q];
    od[i] = v;
  }
  out[0] = ev[0] - od[0];
  out[1] = ev[0] + od[0];
#pragma unroll
  for (int k = 2; k < N; ++k) {
    if (k & 1) out[k] = od[(k - 1) / 2];
    else out[k] = ev[k / 2];
  }
}

// out[q] = sum_l M[q][l] in[l] for the centro-antisymmetric M whose split tables are S, Dd
// (M = D with t.DS, t.DD; M = D^T with t.TS, t.TD)
template <int Q, typename T>
__device__ __forceinline__ void eo_deriv(const T* S, const T* Dd, const T (&in)[Q], T (&out)[Q]) {
  constexpr int QH = (Q + 1) / 2, QL = Q / 2;
  T sm[QH], df[QL > 0 ? QL : 1];
#pragma unroll
  for (int l = 0; l < QL; ++l) {
    sm[l] = in[l] + in[Q - 1 - l];
    df[l] = in[l] - in[Q - 1 - l];
  }
  if constexpr ((Q & 1) != 0) sm[QL] = in[QL];
  T b[QH];
#pragma unroll
  for (int q = 0; q < QH; ++q) {
    T v = T(0);
#pragma unroll
    for (int l = 0; l < QL; ++l) v += Dd[q * QL + l] * df[l];
    b[q] = v;
  }
#pragma unroll
  for (int q = 0; q < QL; ++q) {
    T a = T(0);
#pragma unroll
    for (int l = 0; l < QH; ++l) a += S[q * QH + l] * sm[l];
    out[q] = b[q] + a;
    out[Q - 1 - q] = b[q] - a;
  }
  if constexpr ((Q & 1) != 0) out[QL] = b[QL];
}

// Minimum resident blocks per SM asked of the compiler, from a register target per thread:
// 128 for boxes of 5^3 points and more, 100 below.  Measured on the 5^3 FP64 apply (125
// threads, real 64^3 map): 116 registers, 4 blocks per SM, 0.340 ms; 96 registers (capped),
// 5 blocks, 0.369 ms; an 80-register cap 0.410 ms; 64 registers spill heavily (0.81 ms).
constexpr int pipe_min_blocks(int threads, int q) {
  return (65536 / ((q >= 5 ? 128 : 100) * ((threads + 31) / 32 * 32))) > 0
             ? 65536 / ((q >= 5 ? 128 : 100) * ((threads + 31) / 32 * 32))
             : 1;
}

// EO: the contractions in even-odd form (tables `eo`), constant coefficients only (the launch
// sends batches with tabulated coefficients to EO = false); otherwise directly on `tab`.
template <int N, int Q, int CPB, typename T, bool EO>
__global__ void __launch_bounds__(Q* Q* CPB, pipe_min_blocks(Q* Q* CPB, Q))
    cell_apply_3d_pipe(BatchView b, const Tables1D<N, Q, T> tab, const TablesEO<N, Q, T> eo,
                       const LaneLines<Q * Q * CPB> lanes, const T* __restrict__ x, T* __restrict__ y,
                       int64_t n_vec, T mass, T kappa) {
  constexpr int Q2 = Q * Q;
  constexpr int Q3 = Q * Q * Q;
  constexpr int NB = N * N * N;
  const int BP = lanes.bp, SP = lanes.sp;
  // work buffers per cell and the z-plane pitch of a cell's point box in them: the even-odd
  // kernel keeps one buffer per cell (its fluxes live in registers) at the searched pitch
  constexpr int CM = EO ? 1 : 3;
  const int PZ = EO ? lanes.pz : Q2;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double* hst = reinterpret_cast<double*>(smem_raw);   // [2][CPB][4] staged cell sizes
  double* scl = hst + 2 * CPB * 4;                      // [CPB][4] detJ sx^2, detJ sy^2, detJ sz^2, detJ
  T* work = reinterpret_cast<T*>(scl + CPB * 4);        // [CPB][CM][BP]
  T* stage = work + CM * CPB * BP;                      // [2][CPB][SP]
  int* smap = reinterpret_cast<int*>(stage + 2 * CPB * SP);  // [2][CPB][SP] staged map entries
  const int tid = threadIdx.x;
  x += blockIdx.y * n_vec;
  y += blockIdx.y * n_vec;
  const int64_t n_groups = (int64_t(b.n_cells) + CPB - 1) / CPB;
  const int64_t G = gridDim.x;
  const bool fuse = b.kappa_pts == nullptr;

  // This thread's lines: cell and in-cell position per shape.  The table sits in the
  // parameter bank and is indexed per lane; every derived value goes through keep_reg so that
  // the compiler holds it in a register instead of re-reading the bank (a divergent constant
  // load) inside the group loop.
  int lc[3], la[3], lb[3];
#pragma unroll
  for (int s = 0; s < 3; ++s) {
    const int v = lanes.v[s][tid];
    lc[s] = v & 127;
    la[s] = (v >> 7) & 15;
    lb[s] = (v >> 11) & 15;
  }
  const int baseX = keep_reg(CM * lc[kLineX] * BP + Q * la[kLineX] + PZ * lb[kLineX]);  // x-line (y, z)
  const int baseY = keep_reg(CM * lc[kLineY] * BP + la[kLineY] + PZ * lb[kLineY]);      // y-line (x, z)
  const int baseZ = keep_reg(CM * lc[kLineZ] * BP + la[kLineZ] + Q * lb[kLineZ]);       // z-line (x, y)
  const int stZ = keep_reg(lc[kLineZ] * SP + la[kLineZ] + N * lb[kLineZ]);
  const int cX = keep_reg(lc[kLineX]), cY = keep_reg(lc[kLineY]), cZ = keep_reg(lc[kLineZ]);
  const int pZ = keep_reg(la[kLineZ] + Q * lb[kLineZ]);   // z-line's point offset in the cell box
  const bool zmodes = keep_reg(int(la[kLineZ] < N && lb[kLineZ] < N)) != 0;  // z-line through modes
  const bool ymodes = keep_reg(int(la[kLineY] < N)) != 0;
  const T wX = keep_reg(tab.W[la[kLineX]] * tab.W[lb[kLineX]]);
  const T wY = keep_reg(tab.W[la[kLineY]] * tab.W[lb[kLineY]]);
  const T wZ = keep_reg(tab.W[la[kLineZ]] * tab.W[lb[kLineZ]]);

  // cp.async issue layout: thread (c, ta, tb) = its own cell's z-line
  const int ic = tid / Q2, ita = (tid % Q2) % Q, itb = (tid % Q2) / Q;
  const bool igather = ita < N && itb < N;
  int mv[N];
  auto load_map = [&](int64_t g) {
    const int64_t cell = g * CPB + ic;
    const bool ok = igather && g < n_groups && cell < b.n_cells;
#pragma unroll
    for (int k = 0; k < N; ++k) mv[k] = ok ? __ldg(b.map + cell * NB + ita + N * (itb + N * k)) : -1;
  };
  // group g into stage s: modes (zeros for -1 entries and for cells past the end, whose map
  // entries load_map set to -1), map entries and cell sizes
  auto issue = [&](int64_t g, int s) {
    const int64_t cell = g * CPB + ic;
    if (g < n_groups) {
      T* st = stage + (s * CPB + ic) * SP;
      int* sm = smap + (s * CPB + ic) * SP;
      if (igather) {
#pragma unroll
        for (int k = 0; k < N; ++k) {
          const int e = ita + N * (itb + N * k);
          cp_async_zfill<sizeof(T)>(st + e, x + (mv[k] >= 0 ? mv[k] : 0), mv[k] >= 0);
          sm[e] = mv[k];
        }
      }
      if (cell < b.n_cells && tid % Q2 < 3)
        cp_async_elem<8>(hst + (s * CPB + ic) * 4 + tid % Q2, b.h + cell * 3 + tid % Q2);
    }
    cp_async_commit();  // every thread commits one group per issue, possibly empty
  };

  int64_t g = blockIdx.x;
  load_map(g);
  issue(g, 0);
  load_map(g + G);
  T line[Q], out[Q];
  // EO kernels serve constant coefficients only: the x- and y-fluxes stay in registers from
  // the step that forms them (3, 4) to the step that reads them back (7, 6), on the same line
  // of the same thread, instead of a round trip through shared memory
  T fx[EO ? Q : 1], fy[EO ? Q : 1];
  for (int s = 0; g < n_groups; g += G, s ^= 1) {
    cp_async_wait<0>();
    // Staged modes, map entries and sizes of group g visible; every thread is past the previous
    // group, including its step 9, which read the staged map entries of stage s ^ 1.
    __syncthreads();
    if (tid % Q2 == 0) {
      const double* hc = hst + (s * CPB + ic) * 4;
      const bool ok = g * CPB + ic < b.n_cells;
      const double h0 = ok ? hc[0] : 1.0, h1 = ok ? hc[1] : 1.0, h2 = ok ? hc[2] : 1.0;
      const double detJ = h0 * h1 * h2 * 0.125;
      scl[ic * 4 + 0] = detJ * (2.0 / h0) * (2.0 / h0);
      scl[ic * 4 + 1] = detJ * (2.0 / h1) * (2.0 / h1);
      scl[ic * 4 + 2] = detJ * (2.0 / h2) * (2.0 / h2);
      scl[ic * 4 + 3] = detJ;
    }
    const T* st = stage + s * CPB * SP;
    // 1. z interpolation on z-lines through mode positions, from the staged modes
    if (zmodes) {
      T in[N];
#pragma unroll
      for (int k = 0; k < N; ++k) in[k] = st[stZ + N * N * k];
      if constexpr (EO) {
        eo_interp(eo, in, out);
#pragma unroll
        for (int q = 0; q < Q; ++q) work[baseZ + PZ * q] = out[q];
      } else {
#pragma unroll
        for (int q = 0; q < Q; ++q) {
          T v = T(0);
#pragma unroll
          for (int k = 0; k < N; ++k) v += tab.B[k * Q + q] * in[k];
          work[baseZ + PZ * q] = v;
        }
      }
    }
    // copies of the next group (stage s ^ 1 is free: every thread is past the previous group)
    issue(g + G, s ^ 1);
    __syncthreads();
    // 2. y interpolation on y-lines with x < N
    if (ymodes) {
      if constexpr (EO) {
        T in[N];
#pragma unroll
        for (int j = 0; j < N; ++j) in[j] = work[baseY + Q * j];
        eo_interp(eo, in, out);
      } else {
#pragma unroll
        for (int j = 0; j < N; ++j) line[j] = work[baseY + Q * j];
#pragma unroll
        for (int q = 0; q < Q; ++q) {
          T v = T(0);
#pragma unroll
          for (int j = 0; j < N; ++j) v += tab.B[j * Q + q] * line[j];
          out[q] = v;
        }
      }
#pragma unroll
      for (int q = 0; q < Q; ++q) work[baseY + Q * q] = out[q];
    }
    __syncthreads();
    // 3. x interpolation and x derivative on x-lines; flux scaling folded in
    {
      const T cx = fuse ? wX * kappa * T(scl[cX * 4 + 0]) : T(1);
      if constexpr (EO) {
        T in[N];
#pragma unroll
        for (int i = 0; i < N; ++i) in[i] = work[baseX + i];
        eo_interp(eo, in, out);
        eo_deriv<Q>(eo.DS, eo.DD, out, fx);
#pragma unroll
        for (int q = 0; q < Q; ++q) {
          work[baseX + q] = out[q];
          fx[q] *= cx * tab.W[q];
        }
      } else {
#pragma unroll
        for (int i = 0; i < N; ++i) line[i] = work[baseX + i];
#pragma unroll
        for (int q = 0; q < Q; ++q) {
          T v = T(0);
#pragma unroll
          for (int i = 0; i < N; ++i) v += tab.B[i * Q + q] * line[i];
          out[q] = v;
        }
#pragma unroll
        for (int q = 0; q < Q; ++q) {
          T v = T(0);
#pragma unroll
          for (int l = 0; l < Q; ++l) v += tab.D[q * Q + l] * out[l];
          work[baseX + q] = out[q];
          work[baseX + 2 * BP + q] = fuse ? v * (cx * tab.W[q]) : v;
        }
      }
    }
    __syncthreads();
    // 4. y derivative on y-lines
    {
      const T cy = fuse ? wY * kappa * T(scl[cY * 4 + 1]) : T(1);
#pragma unroll
      for (int l = 0; l < Q; ++l) line[l] = work[baseY + Q * l];
      if constexpr (EO) {
        eo_deriv<Q>(eo.DS, eo.DD, line, fy);
#pragma unroll
        for (int q = 0; q < Q; ++q) fy[q] *= cy * tab.W[q];
      } else {
#pragma unroll
        for (int q = 0; q < Q; ++q) {
          T v = T(0);
#pragma unroll
          for (int l = 0; l < Q; ++l) v += tab.D[q * Q + l] * line[l];
          work[baseY + BP + Q * q] = fuse ? v * (cy * tab.W[q]) : v;
        }
      }
    }
    __syncthreads();
    // 5. z derivative, pointwise flux and transposed z derivative on z-lines
    {
      const double* sc = scl + cZ * 4;
      const T wz = wZ * T(sc[3]);            // W_a W_b detJ
      const T kz = wZ * kappa * T(sc[2]);    // W_a W_b kappa detJ sz^2
      T u[Q], dz[Q];
#pragma unroll
      for (int l = 0; l < Q; ++l) u[l] = work[baseZ + PZ * l];
      if constexpr (EO) {
        eo_deriv<Q>(eo.DS, eo.DD, u, dz);
      } else {
#pragma unroll
        for (int q = 0; q < Q; ++q) {
          T v = T(0);
#pragma unroll
          for (int l = 0; l < Q; ++l) v += tab.D[q * Q + l] * u[l];
          dz[q] = v;
        }
      }
#pragma unroll
      for (int q = 0; q < Q; ++q) {
        const T w = wz * tab.W[q];
        if (EO || fuse) {
          dz[q] *= kz * tab.W[q];
        } else {
          const int64_t cell = g * CPB + cZ;
          const int p = pZ + Q2 * q;
          const T k = cell < b.n_cells ? T(b.kappa_pts[cell * Q3 + p]) : T(0);
          const T wk = wZ * tab.W[q] * kappa * k;
          work[baseZ + 2 * BP + Q2 * q] *= wk * T(sc[0]);
          work[baseZ + BP + Q2 * q] *= wk * T(sc[1]);
          dz[q] *= wk * T(sc[2]);
        }
        u[q] *= w * mass;
      }
      if constexpr (EO) {
        eo_deriv<Q>(eo.TS, eo.TD, dz, out);
#pragma unroll
        for (int l = 0; l < Q; ++l) work[baseZ + PZ * l] = u[l] + out[l];
      } else {
#pragma unroll
        for (int l = 0; l < Q; ++l) {
          T v = u[l];
#pragma unroll
          for (int q = 0; q < Q; ++q) v += tab.D[q * Q + l] * dz[q];
          work[baseZ + PZ * l] = v;
        }
      }
    }
    __syncthreads();
    // 6. transposed y derivative on y-lines
    {
      if constexpr (EO) {
        eo_deriv<Q>(eo.TS, eo.TD, fy, out);
#pragma unroll
        for (int l = 0; l < Q; ++l) work[baseY + Q * l] += out[l];
      } else {
#pragma unroll
        for (int q = 0; q < Q; ++q) line[q] = work[baseY + BP + Q * q];
#pragma unroll
        for (int l = 0; l < Q; ++l) {
          T v = work[baseY + Q * l];
#pragma unroll
          for (int q = 0; q < Q; ++q) v += tab.D[q * Q + l] * line[q];
          work[baseY + Q * l] = v;
        }
      }
    }
    __syncthreads();
    // 7. transposed x derivative and transposed x interpolation on x-lines
    {
#pragma unroll
      for (int l = 0; l < Q; ++l) out[l] = work[baseX + l];
      if constexpr (EO) {
        T t[Q], m[N];
        eo_deriv<Q>(eo.TS, eo.TD, fx, t);
#pragma unroll
        for (int l = 0; l < Q; ++l) out[l] += t[l];
        eo_interp_t(eo, out, m);
#pragma unroll
        for (int i = 0; i < N; ++i) work[baseX + i] = m[i];
      } else {
#pragma unroll
        for (int q = 0; q < Q; ++q) line[q] = work[baseX + 2 * BP + q];
#pragma unroll
        for (int l = 0; l < Q; ++l) {
          T v = out[l];
#pragma unroll
          for (int q = 0; q < Q; ++q) v += tab.D[q * Q + l] * line[q];
          out[l] = v;
        }
#pragma unroll
        for (int i = 0; i < N; ++i) {
          T v = T(0);
#pragma unroll
          for (int q = 0; q < Q; ++q) v += tab.B[i * Q + q] * out[q];
          work[baseX + i] = v;
        }
      }
    }
    __syncthreads();
    // 8. transposed y interpolation on y-lines with x < N
    if (ymodes) {
#pragma unroll
      for (int q = 0; q < Q; ++q) line[q] = work[baseY + Q * q];
      if constexpr (EO) {
        T m[N];
        eo_interp_t(eo, line, m);
#pragma unroll
        for (int j = 0; j < N; ++j) work[baseY + Q * j] = m[j];
      } else {
#pragma unroll
        for (int j = 0; j < N; ++j) {
          T v = T(0);
#pragma unroll
          for (int q = 0; q < Q; ++q) v += tab.B[j * Q + q] * line[q];
          work[baseY + Q * j] = v;
        }
      }
    }
    __syncthreads();
    // map entries of the group after next, consumed by the next iteration's issue (loaded here
    // to keep them out of the registers of steps 1-8)
    load_map(g + 2 * G);
    // 9. transposed z interpolation on z-lines through mode positions and scatter through the
    // staged map entries (the next group writes the work buffers only after its first barrier)
    if (zmodes) {
      const int* sm = smap + s * CPB * SP + stZ;
#pragma unroll
      for (int q = 0; q < Q; ++q) line[q] = work[baseZ + PZ * q];
      if constexpr (EO) {
        T m[N];
        eo_interp_t(eo, line, m);
#pragma unroll
        for (int k = 0; k < N; ++k) {
          const int dof = sm[N * N * k];
          if (dof >= 0) atomicAdd(y + dof, m[k]);
        }
      } else {
        // kept rolled: unrolled, the compiler hoists every map load and output at once and
        // spills (5^3 FP64: 0.37 ms rolled vs 0.50 ms unrolled)
#pragma unroll 1
        for (int k = 0; k < N; ++k) {
          T v = T(0);
#pragma unroll
          for (int q = 0; q < Q; ++q) v += tab.B[k * Q + q] * line[q];
          const int dof = sm[N * N * k];
          if (dof >= 0) atomicAdd(y + dof, v);
        }
      }
    }
  }
  cp_async_wait<0>();
}

}  // namespace grico
