// Device plan of the matrix-free runtime: the B200 counterpart of the runtime half of
// Grico.jl's AssemblyPlan (plans.jl:131-145) plus its reduced operator map
// (assembly.jl:19-27).  C ABI in include/grico_b200.h.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <type_traits>
#include <vector>

#include "cell_kernels.cuh"
#include "cell_pipe.cuh"
#include "cell_plane.cuh"
#include "cell_dense_tc.cuh"
#include "grico_host.h"
#include "grico_plan_internal.h"
#include "vector_kernels.cuh"

namespace grico {

DevBuf::~DevBuf() {
  if (ptr) cudaFree(ptr);
}

bool cuda_ok(cudaError_t e, const char* what) {
  if (e == cudaSuccess) return true;
  set_error(std::string(what) + ": " + cudaGetErrorString(e));
  return false;
}

// Lagrange collocation derivative on Gauss points via barycentric weights:
// D[p*q+l] = L_l'(xi_p).
std::vector<double> collocation_derivative(const std::vector<double>& xi) {
  const int q = int(xi.size());
  std::vector<double> lam(q, 1.0), D(q * q, 0.0);
  for (int j = 0; j < q; ++j)
    for (int k = 0; k < q; ++k)
      if (k != j) lam[j] /= (xi[j] - xi[k]);
  for (int p = 0; p < q; ++p) {
    double diag = 0.0;
    for (int l = 0; l < q; ++l) {
      if (l == p) continue;
      double v = (lam[l] / lam[p]) / (xi[p] - xi[l]);
      D[p * q + l] = v;
      diag -= v;
    }
    D[p * q + p] = diag;
  }
  return D;
}

namespace {

inline int32_t item_count(const GricoCellBatchDesc& b) { return b.n_cells; }
inline int32_t item_count(const GricoPointBatchDesc& b) { return b.n_items; }

// number of box modes prod(n_a) for per-axis mode counts n_a = degree_a + 1
int64_t box_count(int dim, const int* n) {
  int64_t nb = 1;
  for (int a = 0; a < dim; ++a) nb *= n[a];
  return nb;
}

// Compose the cell term map with the reduced map P: every local entry becomes a sparse
// combination of reduced dofs (the composition x_loc = T P x_red used by reduced applies).
template <typename Desc>
void compose_reduced(const Desc& bd, int64_t nb, const GricoPlanDesc& d,
                     std::vector<int32_t>& map, std::vector<double>& coef, bool& need_coef,
                     std::vector<int64_t>& toff, std::vector<int32_t>& tidx, std::vector<double>& tcoef) {
  const int64_t ne = int64_t(item_count(bd)) * nb;
  map.assign(ne, -1);
  coef.assign(ne, 1.0);
  need_coef = false;
  toff.assign(1, 0);
  tidx.clear();
  tcoef.clear();
  std::vector<std::pair<int64_t, double>> acc;
  std::map<std::vector<std::pair<int64_t, double>>, int32_t> known;  // expansion (term order kept) -> tail
  auto add = [&](int64_t r, double c) {
    for (auto& t : acc)
      if (t.first == r) { t.second += c; return; }
    acc.emplace_back(r, c);
  };
  auto add_full = [&](int64_t g, double c) {
    for (int64_t t = d.red_offsets[g]; t < d.red_offsets[g + 1]; ++t) add(d.red_index[t], c * d.red_coef[t]);
  };
  for (int64_t e = 0; e < ne; ++e) {
    int32_t v = bd.map_index[e];
    if (v == -1) continue;
    acc.clear();
    if (v >= 0) {
      add_full(v, bd.map_coef ? bd.map_coef[e] : 1.0);
    } else {
      int64_t k = -(int64_t(v) + 2);
      for (int64_t t = bd.tail_offsets[k]; t < bd.tail_offsets[k + 1]; ++t) add_full(bd.tail_index[t], bd.tail_coef[t]);
    }
    acc.erase(std::remove_if(acc.begin(), acc.end(), [](auto& t) { return t.second == 0.0; }), acc.end());
    if (acc.empty()) continue;
    if (acc.size() == 1) {
      map[e] = int32_t(acc[0].first);
      coef[e] = acc[0].second;
      if (acc[0].second != 1.0) need_coef = true;
    } else {
      // entries with the same expansion (cells sharing a hanging dof) share one tail
      auto found = known.find(acc);
      if (found != known.end()) {
        map[e] = -found->second - 2;
        continue;
      }
      const int32_t id = int32_t(toff.size() - 1);
      known.emplace(acc, id);
      map[e] = -id - 2;
      for (auto& t : acc) {
        tidx.push_back(int32_t(t.first));
        tcoef.push_back(t.second);
      }
      toff.push_back(int64_t(tidx.size()));
    }
  }
}

void fill_view(BatchView& v, const DevBatch& b, bool reduced) {
  v.n_cells = b.n_cells;
  const DevMap& m = reduced ? b.red : b.full;
  v.map = m.map.get<int32_t>();
  v.coef = m.coef.get<double>();
  v.tail_off = m.toff.get<int64_t>();
  v.tail_idx = m.tidx.get<int32_t>();
  v.tail_coef = m.tcoef.get<double>();
  v.h = b.h.get<double>();
  v.kappa_pts = b.kappa.get<double>();
  v.B = b.B.get<double>();
  v.D = b.D.get<double>();
  v.W = b.W.get<double>();
  v.G = b.G.get<double>();
  v.skip = reduced ? b.skip.get<uint8_t>() : nullptr;
  v.mass_pts = b.mass_pts.get<double>();
}

template <int N, int Q, typename T>
Tables1D<N, Q, T> make_tables(const DevBatch& b) {
  Tables1D<N, Q, T> t;
  for (int i = 0; i < N * Q; ++i) t.B[i] = T(b.hB[i]);
  for (int i = 0; i < Q * Q; ++i) t.D[i] = T(b.hD[i]);
  for (int i = 0; i < Q; ++i) t.W[i] = T(b.hW[i]);
  return t;
}

// Default 3-D kernel variant by points per axis.  A sweep of all variants on uniform
// 16-million-dof grids (B200, one apply, degrees 1..7 with q = p + 1) found the pipelined kernel
// fastest at every q (p = 4: 0.367 vs 0.495 ms for the one-block-per-group kernel; p = 3: 0.374
// vs 0.710 ms; p = 7: 0.500 vs 0.843 ms).  Later sweeps (4-million-dof grids, q = p + 1 and
// p + 2, ms per apply) compared its even-odd form (fluxes in registers, one work buffer per cell
// at a searched plane pitch) with the direct one: even-odd wins at every shape, by 10-25 % at
// p = 1..4 and 1.3-1.9x at p = 6..8 in FP64 (p = 4, q = 5: 0.088 vs 0.102 ms; FP32 0.062 vs
// 0.073), and in FP32 it also beats the one-block-per-group kernel at q = 2.  Group sizes: half
// size (3) except default size (4) for FP64 q = 7 and FP32 q = 6, 7, 9.
int default_tile_3d(int q, bool fp32) {
  // thread-per-plane kernel (variant 9), measured on uniform grids (B200, ms per apply): p = 1,
  // 275k dofs: FP64 0.0374 -> 0.0318, FP32 0.0322 -> 0.0250; p = 2, 2.1M dofs: FP64 0.0807 ->
  // 0.0705, FP32 0.0635 -> 0.0566.  At q >= 4 its register and shared-memory footprint leaves too
  // few warps per SM (p = 4 FP64: 0.311 vs 0.423 ms) and the pipelined kernel stays the default.
  if (q <= 3) return 9;
  if (q <= 5) return 3;
  if (fp32) return q == 8 ? 3 : 4;
  return q == 7 ? 4 : 3;
}

int sm_count() {
  static const int n = [] {
    int dev = 0, v = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev);
    return v > 0 ? v : 1;
  }();
  return n;
}

// Resident blocks per SM of a persistent kernel (0 when it cannot launch, e.g. too much shared
// memory); raises the kernel's dynamic shared-memory limit first when it needs more than 48 KB.
int persistent_blocks_per_sm(const void* kern, int threads, size_t smem) {
  if (smem > 48 * 1024 &&
      cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  int n = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, kern, threads, smem) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return n;
}

// FP32 apply of a uniform batch on the tensor cores (cell_dense_tc.cuh): persistent CTAs, one
// per SM (192 KB of shared memory each), gridDim.y = right-hand sides
bool launch_dense(const DevBatch& bt, const BatchView& v, const float* x, float* y, int64_t nvec, int nrhs,
                  cudaStream_t st) {
  int* err = nullptr;
  if (tc_error_flag(&err) != GRICO_OK) return false;
  static const bool attr = cudaFuncSetAttribute(dense::cell_apply_dense_tc, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                int(dense::kSmem)) == cudaSuccess;
  if (!attr) return false;
  const int64_t tiles = (int64_t(v.n_cells) + dense::kM - 1) / dense::kM;
  const dim3 grid(unsigned(std::min<int64_t>(tiles, sm_count())), unsigned(nrhs));
  dense::cell_apply_dense_tc<<<grid, dense::kThreads, dense::kSmem, st>>>(
      v.map, v.n_cells, bt.n[0] * bt.n[1] * bt.n[2], bt.dense.get<__nv_bfloat16>(), x, y, nvec, err);
  return true;
}

template <typename T>
bool launch_fused(int dim, const DevBatch& bt, const BatchView& v, const T* x, T* y, int64_t nvec, T mass, T kappa,
                  int mode, const double* src, int nrhs, cudaStream_t st) {
  if (v.n_cells == 0) return true;
  const int N = bt.n[0], Q = bt.q[0];
  // deterministic applies store local results: the one-block-per-group kernel (scatter_entry)
  const int var = v.local_out ? 1 : bt.tile[sizeof(T) == 4 ? 1 : 0];
  // variant 10, FP32: uniform batch with a plain map on the tensor cores
  if constexpr (std::is_same<T, float>::value) {
    if (dim == 3 && var == kDenseVariant && mode == 0 && bt.dense_ok && v.coef == nullptr && v.tail_off == nullptr &&
        v.mass_pts == nullptr && v.kappa_pts == nullptr && launch_dense(bt, v, x, y, nvec, nrhs, st))
      return true;
  }
#define GRICO_L3_CPB(NN, QQ, CPB_)                                                                             \
  {                                                                                                            \
    constexpr int CPB = CPB_;                                                                                  \
    const size_t smem = size_t(3) * CPB * ((QQ * QQ * QQ) | 1) * sizeof(T);                                    \
    auto kern = cell_apply_3d<NN, QQ, CPB, T>;                                                                \
    if (smem > 48 * 1024) cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));   \
    dim3 block(QQ * QQ, CPB), grid((v.n_cells + CPB - 1) / CPB, nrhs);                                         \
    kern<<<grid, block, smem, st>>>(v, make_tables<NN, QQ, T>(bt), x, y, nvec, mass, kappa, mode, src);       \
    return true;                                                                                               \
  }
#define GRICO_L3_PIPE_EO(NN, QQ, CPB_, EO_)                                                                   \
  {                                                                                                            \
    constexpr int CPB = CPB_;                                                                                  \
    constexpr int NT = QQ * QQ * CPB;                                                                          \
    static const LaneLines<NT> lanes = make_lane_lines<NT>(NN, QQ, CPB, int(sizeof(T)), EO_);                 \
    static const size_t smem = pipe_smem_bytes(CPB, lanes.bp, lanes.sp, int(sizeof(T)), EO_ ? 1 : 3);         \
    auto kern = cell_apply_3d_pipe<NN, QQ, CPB, T, EO_>;                                                      \
    static const int per_sm = persistent_blocks_per_sm(reinterpret_cast<const void*>(kern), NT, smem);        \
    if (per_sm > 0) {                                                                                          \
      const int64_t groups = (int64_t(v.n_cells) + CPB - 1) / CPB;                                             \
      dim3 grid(unsigned(std::min<int64_t>(groups, int64_t(per_sm) * sm_count())), nrhs);                      \
      kern<<<grid, NT, smem, st>>>(v, make_tables<NN, QQ, T>(bt), eo, lanes, x, y, nvec, mass, kappa);         \
      return true;                                                                                             \
    }                                                                                                          \
  }
// variants 3-5: even-odd contractions (constant coefficients, tables with the symmetry), 6-8:
// direct ones
#define GRICO_L3_PIPE(NN, QQ, CPB_, WANT_EO)                                                                   \
  if (mode == 0 && v.coef == nullptr && v.tail_off == nullptr && v.mass_pts == nullptr) {                      \
    TablesEO<NN, QQ, T> eo{};                                                                                  \
    if (WANT_EO && v.kappa_pts == nullptr && make_eo_tables<NN, QQ, T>(bt.hB.data(), bt.hD.data(), eo))       \
      GRICO_L3_PIPE_EO(NN, QQ, CPB_, true)                                                                     \
    GRICO_L3_PIPE_EO(NN, QQ, CPB_, false)                                                                      \
  }
// variant 9: one warp per 32 / q cells, thread per plane (q <= 6; plain maps, constant coefficients)
#define GRICO_L3_PLANE(NN, QQ)                                                                                 \
  if constexpr (QQ <= 6) {                                                                                     \
    if (mode == 0 && v.coef == nullptr && v.tail_off == nullptr && v.mass_pts == nullptr &&                    \
        v.kappa_pts == nullptr) {                                                                              \
      TablesEO<NN, QQ, T> eo{};                                                                                \
      if (make_eo_tables<NN, QQ, T>(bt.hB.data(), bt.hD.data(), eo)) {                                         \
        constexpr int CPB = PlaneShape<QQ>::CPB;                                                               \
        static const PlaneLayout lay = make_plane_layout(NN, QQ, int(sizeof(T)));                              \
        static const size_t smem = plane_smem_bytes(CPB, lay, int(sizeof(T)));                                 \
        auto kern = cell_apply_3d_plane<NN, QQ, T>;                                                            \
        static const int per_sm = persistent_blocks_per_sm(reinterpret_cast<const void*>(kern), 32, smem);    \
        if (per_sm > 0) {                                                                                      \
          const int64_t groups = (int64_t(v.n_cells) + CPB - 1) / CPB;                                         \
          dim3 grid(unsigned(std::min<int64_t>(groups, int64_t(per_sm) * sm_count())), nrhs);                  \
          kern<<<grid, 32, smem, st>>>(v, make_tables<NN, QQ, T>(bt), eo, lay, x, y, nvec, mass, kappa);       \
          return true;                                                                                         \
        }                                                                                                      \
      }                                                                                                        \
    }                                                                                                          \
  }
#define GRICO_L3(NN, QQ)                                                                                       \
  if (N == NN && Q == QQ) {                                                                                    \
    constexpr int C1 = (256 / (QQ * QQ)) > 0 ? (256 / (QQ * QQ)) : 1;                                          \
    constexpr int C0 = C1 / 2 > 0 ? C1 / 2 : 1;                                                                \
    constexpr int C2 = (2 * C1 * QQ * QQ <= 1024) ? 2 * C1 : C1;                                               \
    if (var == 9) GRICO_L3_PLANE(NN, QQ)                                                                       \
    if (var == 3 || var == 6 || var == 9) GRICO_L3_PIPE(NN, QQ, C0, var != 6)                                  \
    if (var == 4 || var == 7) GRICO_L3_PIPE(NN, QQ, C1, var == 4)                                              \
    if (var == 5 || var == 8) GRICO_L3_PIPE(NN, QQ, C2, var == 5)                                              \
    if (var % 3 == 0) GRICO_L3_CPB(NN, QQ, C0)                                                                 \
    if (var % 3 == 2) GRICO_L3_CPB(NN, QQ, C2)                                                                 \
    GRICO_L3_CPB(NN, QQ, C1)                                                                                   \
  }
#define GRICO_L2(NN, QQ)                                                                                     \
  if (N == NN && Q == QQ) {                                                                                  \
    constexpr int CPB = (128 / QQ) > 0 ? (128 / QQ) : 1;                                                     \
    dim3 block(QQ, CPB), grid((v.n_cells + CPB - 1) / CPB, nrhs);                                            \
    cell_apply_2d<NN, QQ, CPB, T><<<grid, block, 0, st>>>(v, x, y, nvec, mass, kappa, mode, src);            \
    return true;                                                                                             \
  }
  if (dim == 3) {
    GRICO_L3(2, 2) GRICO_L3(3, 3) GRICO_L3(4, 4) GRICO_L3(5, 5) GRICO_L3(6, 6) GRICO_L3(7, 7) GRICO_L3(8, 8)
    GRICO_L3(9, 9) GRICO_L3(2, 3) GRICO_L3(3, 4) GRICO_L3(4, 5) GRICO_L3(5, 6)
  } else if (dim == 2) {
    GRICO_L2(2, 2) GRICO_L2(3, 3) GRICO_L2(4, 4) GRICO_L2(5, 5) GRICO_L2(6, 6) GRICO_L2(7, 7) GRICO_L2(8, 8)
    GRICO_L2(9, 9) GRICO_L2(2, 3) GRICO_L2(3, 4) GRICO_L2(4, 5) GRICO_L2(5, 6)
  }
#undef GRICO_L3
#undef GRICO_L3_PIPE
#undef GRICO_L3_PIPE_EO
#undef GRICO_L3_PLANE
#undef GRICO_L3_CPB
#undef GRICO_L2
  return false;
}

// Tail buffers of one batch map (DevMap::n_tail): only when the longest expansion has at least
// kTailBufferMin terms.  Several entries may share a tail (the cell kernel adds their results
// into its slot).
bool setup_tail_buffer(DevMap& m, const int32_t* map, int64_t ne, const int64_t* off, int64_t n_tail) {
  m.n_tail = 0;
  if (n_tail <= 0) return true;
  int64_t longest = 0;
  for (int64_t k = 0; k < n_tail; ++k) longest = std::max(longest, off[k + 1] - off[k]);
  if (longest < kTailBufferMin) return true;
  for (int64_t e = 0; e < ne; ++e)
    if (map[e] <= -2 && -(int64_t(map[e]) + 2) >= n_tail) return true;
  if (!m.tx.alloc(sizeof(double) * size_t(n_tail) * kTailRhs) || !m.ty.alloc(sizeof(double) * size_t(n_tail) * kTailRhs))
    return false;
  std::vector<int32_t> sk;
  std::vector<int64_t> st;
  for (int64_t k = 0; k < n_tail; ++k)
    for (int64_t t = off[k]; t < off[k + 1]; t += kTailSeg) {
      sk.push_back(int32_t(k));
      st.push_back(t);
    }
  if (!m.seg_k.upload(sk) || !m.seg_t.upload(st)) return false;
  m.n_seg = int64_t(sk.size());
  m.n_tail = n_tail;
  return true;
}

// One numbering of the buffered tails of every cell batch of a layout (GricoPlan::TailAll),
// from the batches' device maps; segments of kTailSeg terms as in setup_tail_buffer.
bool build_tail_all(GricoPlan* P, int layout) {
  auto& A = P->tails[layout];
  A.base.assign(P->batches.size(), -1);
  std::vector<int64_t> toff{0};
  std::vector<int32_t> tidx;
  std::vector<double> tcoef;
  int64_t n_tail = 0;
  for (size_t bi = 0; bi < P->batches.size(); ++bi) {
    const DevMap& m = layout ? P->batches[bi].red : P->batches[bi].full;
    if (m.n_tail <= 0) continue;
    std::vector<int64_t> off(static_cast<size_t>(m.n_tail) + 1);
    if (!cuda_ok(cudaMemcpy(off.data(), m.toff.ptr, sizeof(int64_t) * off.size(), cudaMemcpyDeviceToHost), "tails"))
      return false;
    const int64_t nt = off.back();
    std::vector<int32_t> idx(static_cast<size_t>(nt));
    std::vector<double> co(static_cast<size_t>(nt));
    if (nt > 0 && (!cuda_ok(cudaMemcpy(idx.data(), m.tidx.ptr, sizeof(int32_t) * nt, cudaMemcpyDeviceToHost), "tails") ||
                   !cuda_ok(cudaMemcpy(co.data(), m.tcoef.ptr, sizeof(double) * nt, cudaMemcpyDeviceToHost), "tails")))
      return false;
    A.base[bi] = n_tail;
    const int64_t t0 = int64_t(tidx.size());
    for (int64_t k = 0; k < m.n_tail; ++k) toff.push_back(t0 + off[size_t(k) + 1]);
    tidx.insert(tidx.end(), idx.begin(), idx.end());
    tcoef.insert(tcoef.end(), co.begin(), co.end());
    n_tail += m.n_tail;
  }
  A.n_tail = n_tail;
  if (n_tail == 0) return true;
  std::vector<int32_t> sk;
  std::vector<int64_t> st;
  for (int64_t k = 0; k < n_tail; ++k)
    for (int64_t t = toff[size_t(k)]; t < toff[size_t(k) + 1]; t += kTailSeg) {
      sk.push_back(int32_t(k));
      st.push_back(t);
    }
  A.n_seg = int64_t(sk.size());
  return A.toff.upload(toff) && A.tidx.upload(tidx) && A.tcoef.upload(tcoef) && A.seg_k.upload(sk) &&
         A.seg_t.upload(st) && A.tx.alloc(sizeof(double) * size_t(n_tail) * kTailRhs) &&
         A.ty.alloc(sizeof(double) * size_t(n_tail) * kTailRhs);
}

template <typename T>
void launch_batch_cells(const GricoPlan& P, const DevBatch& b, BatchView& v, const T* x, T* y, int64_t nvec, int mode,
                        const double* src, int nrhs, cudaStream_t st);

// One cell batch.  Operator applies of a map with buffered tails run in three launches: the
// tail sums (one warp per expansion), the cell kernel (tails read from and written to the
// buffers), the tail scatter; long expansions no longer serialise one thread of the cell kernel.
template <typename T>
void launch_batch(const GricoPlan& P, const DevBatch& b, bool reduced, const T* x, T* y, int64_t nvec, int mode,
                  const double* src, int nrhs, cudaStream_t st, void* local_out = nullptr, int64_t local_stride = 0,
                  T* merged_tx = nullptr, T* merged_ty = nullptr, int64_t merged_stride = 0) {
  BatchView v;
  fill_view(v, b, reduced);
  v.local_out = local_out;
  v.local_stride = local_stride;
  if (merged_tx) {
    // the tails were summed by the apply's merged pass and are spread by it afterwards
    v.tail_x = merged_tx;
    v.tail_y = merged_ty;
    v.n_tail = merged_stride;
    launch_batch_cells<T>(P, b, v, x, y, nvec, mode, src, nrhs, st);
    return;
  }
  const DevMap& m = reduced ? b.red : b.full;
  const bool buffered = mode == 0 && x && m.n_tail > 0 && nrhs <= kTailRhs && !local_out;
  // several right-hand sides: segments with the columns on the lanes (kTailLaneRhs or more),
  // else one warp per tail with the lanes over its terms
  const bool lanes_rhs = nrhs >= kTailLaneRhs;
  const dim3 tg(int(std::min<int64_t>(((lanes_rhs ? m.n_seg : m.n_tail) * 32 + 255) / 256, 148 * 16)),
                lanes_rhs ? 1u : unsigned(nrhs));
  if (buffered) {
    if (lanes_rhs) {
      cudaMemsetAsync(m.tx.ptr, 0, sizeof(T) * size_t(m.n_tail) * nrhs, st);
      tail_gather_seg<T><<<tg, 256, 0, st>>>(m.seg_k.get<int32_t>(), m.seg_t.get<int64_t>(), m.n_seg,
                                             m.toff.get<int64_t>(), m.tidx.get<int32_t>(), m.tcoef.get<double>(),
                                             m.n_tail, x, nvec, m.tx.get<T>(), m.ty.get<T>(), nrhs);
    } else
      tail_gather<T><<<tg, 256, 0, st>>>(m.toff.get<int64_t>(), m.tidx.get<int32_t>(), m.tcoef.get<double>(),
                                         m.n_tail, x, nvec, m.tx.get<T>(), m.ty.get<T>());
    v.tail_x = m.tx.ptr;
    v.tail_y = m.ty.ptr;
    v.n_tail = m.n_tail;
  }
  launch_batch_cells<T>(P, b, v, x, y, nvec, mode, src, nrhs, st);
  if (buffered && lanes_rhs)
    tail_scatter_seg<T><<<tg, 256, 0, st>>>(m.seg_k.get<int32_t>(), m.seg_t.get<int64_t>(), m.n_seg,
                                            m.toff.get<int64_t>(), m.tidx.get<int32_t>(), m.tcoef.get<double>(),
                                            m.n_tail, m.ty.get<T>(), y, nvec, nrhs);
  else if (buffered)
    tail_scatter<T><<<tg, 256, 0, st>>>(m.toff.get<int64_t>(), m.tidx.get<int32_t>(), m.tcoef.get<double>(),
                                        m.n_tail, m.ty.get<T>(), y, nvec);
}

template <typename T>
void launch_batch_cells(const GricoPlan& P, const DevBatch& b, BatchView& v, const T* x, T* y, int64_t nvec, int mode,
                        const double* src, int nrhs, cudaStream_t st) {
  const int dim = P.dim;
  if (mode != 3 && mode != 4 && b.isotropic && b.q[0] >= b.n[0] &&
      launch_fused<T>(dim, b, v, x, y, nvec, T(P.mass), T(P.kappa), mode, src, nrhs, st))
    return;
  int n[3] = {1, 1, 1}, q[3] = {1, 1, 1};
  for (int a = 0; a < dim; ++a) { n[a] = b.n[a]; q[a] = b.q[a]; }
  int nb = n[0] * n[1] * n[2], nq = q[0] * q[1] * q[2];
  size_t smem = sizeof(T) * (nb + (dim + 1) * nq);
  if (smem > 48 * 1024) cudaFuncSetAttribute(cell_apply_generic<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
  dim3 grid(b.n_cells, nrhs);
  cell_apply_generic<T><<<grid, 128, smem, st>>>(v, dim, n[0], n[1], n[2], q[0], q[1], q[2], x, y, nvec, T(P.mass),
                                                T(P.kappa), mode, src);
}

int grid_for(int64_t n) { return int(std::min<int64_t>((n + 255) / 256, 148 * 16)); }

template <typename T, int D, int N, int Q>
void launch_subcells_nq(const GricoPlan& P, const DevPointBatch& pb, const SubcellView& v, const T* x, T* y,
                        int64_t nvec, int mode, const double* src, int nrhs, cudaStream_t st) {
  SubTables<Q, T> tab;
  for (int j = 0; j < Q; ++j) {
    tab.eta[j] = T(pb.hEta[j]);
    tab.W[j] = T(pb.hW[j]);
  }
  for (int j = 0; j < Q * Q; ++j) tab.Dm[j] = T(pb.hDm[j]);
  using S = SubSizes<D, N, Q>;
  const size_t smem = sizeof(T) * size_t(S::NB + kSubWarps * S::WARP);
  auto kernel = subcell_apply<T, D, N, Q>;
  if (smem > 48 * 1024) cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
  dim3 grid(pb.n_items, nrhs);
  kernel<<<grid, kSubThreads, smem, st>>>(v, tab, x, y, nvec, T(P.mass), T(P.kappa), mode, src);
}

// (modes per axis, points per axis) pairs compiled for the subcell kernel
#define GRICO_SUB3(X) X(2, 2) X(2, 3) X(3, 3) X(2, 4) X(3, 4) X(4, 4)
#define GRICO_SUB2(X)                                                                                     \
  X(2, 2) X(2, 3) X(3, 3) X(3, 4) X(4, 4) X(4, 5) X(5, 5) X(5, 6) X(6, 6) X(6, 7) X(7, 7) X(7, 8) X(8, 8)

bool subcell_shape_supported(int dim, int n, int q) {
#define GRICO_SUB_CHECK(NN, QQ) if (n == NN && q == QQ) return true;
  if (dim == 3) { GRICO_SUB3(GRICO_SUB_CHECK) }
  if (dim == 2) { GRICO_SUB2(GRICO_SUB_CHECK) }
#undef GRICO_SUB_CHECK
  return false;
}

template <typename T>
void launch_subcells(const GricoPlan& P, const DevPointBatch& pb, bool reduced, const T* x, T* y, int64_t nvec,
                     int mode, const double* src, int nrhs, cudaStream_t st, void* local_out = nullptr,
                     int64_t local_stride = 0) {
  SubcellView v;
  v.n_items = pb.n_items;
  v.local_out = local_out;
  v.local_stride = local_stride;
  const DevMap& m = reduced ? pb.red : pb.full;
  v.map = m.map.get<int32_t>();
  v.coef = m.coef.get<double>();
  v.tail_off = m.toff.get<int64_t>();
  v.tail_idx = m.tidx.get<int32_t>();
  v.tail_coef = m.tcoef.get<double>();
  v.h = pb.h.get<double>();
  v.sub_off = pb.sub_off.get<int64_t>();
  v.level = pb.sub_level.get<int32_t>();
  v.pos = pb.sub_pos.get<int32_t>();
  v.mask = pb.sub_mask.get<uint64_t>();
  v.ws = pb.sub_w.get<double>();
  v.kpts = pb.kpts.get<double>();
  v.skip = reduced ? pb.skip.get<uint8_t>() : nullptr;
  const int n = pb.n[0], q = pb.q[0];
#define GRICO_SUB_LAUNCH3(NN, QQ) \
  if (n == NN && q == QQ) return launch_subcells_nq<T, 3, NN, QQ>(P, pb, v, x, y, nvec, mode, src, nrhs, st);
#define GRICO_SUB_LAUNCH2(NN, QQ) \
  if (n == NN && q == QQ) return launch_subcells_nq<T, 2, NN, QQ>(P, pb, v, x, y, nvec, mode, src, nrhs, st);
  if (P.dim == 3) { GRICO_SUB3(GRICO_SUB_LAUNCH3) }
  if (P.dim == 2) { GRICO_SUB2(GRICO_SUB_LAUNCH2) }
#undef GRICO_SUB_LAUNCH3
#undef GRICO_SUB_LAUNCH2
}

template <typename T>
void launch_points(const GricoPlan& P, const DevPointBatch& pb, bool reduced, const T* x, T* y, int64_t nvec, int mode,
                   const double* src, int nrhs, cudaStream_t st, void* local_out = nullptr, int64_t local_stride = 0) {
  if (pb.n_items == 0) return;
  if (pb.kind == GRICO_ITEM_SUBCELLS)
    return launch_subcells<T>(P, pb, reduced, x, y, nvec, mode, src, nrhs, st, local_out, local_stride);
  PointView v;
  v.n_items = pb.n_items;
  v.local_out = local_out;
  v.local_stride = local_stride;
  v.kind = pb.kind;
  for (int a = 0; a < 3; ++a) v.n[a] = pb.n[a];
  const DevMap& m = reduced ? pb.red : pb.full;
  v.map = m.map.get<int32_t>();
  v.coef = m.coef.get<double>();
  v.tail_off = m.toff.get<int64_t>();
  v.tail_idx = m.tidx.get<int32_t>();
  v.tail_coef = m.tcoef.get<double>();
  v.h = pb.h.get<double>();
  v.pt_off = pb.pt_off.get<int64_t>();
  v.ref = pb.ref.get<double>();
  v.w = pb.w.get<double>();
  v.nrm = pb.nrm.get<double>();
  v.eta = pb.eta.get<double>();
  v.kpts = pb.kpts.get<double>();
  v.skip = reduced ? pb.skip.get<uint8_t>() : nullptr;
  const int D = P.dim;
  if (pb.kind == GRICO_ITEM_INTERFACE) {
    if (mode == 1) return;  // no load term on interior interfaces
    for (int a = 0; a < 3; ++a) v.np[a] = pb.np[a];
    v.ref_p = pb.ref_p.get<double>();
    v.h_p = pb.h_p.get<double>();
    v.axis = pb.axis.get<int32_t>();
    const int nbi = pb.n[0] * (D > 1 ? pb.n[1] : 1) * (D > 2 ? pb.n[2] : 1) +
                    pb.np[0] * (D > 1 ? pb.np[1] : 1) * (D > 2 ? pb.np[2] : 1);
    const int nmax = std::max(std::max(pb.n[0], std::max(D > 1 ? pb.n[1] : 1, D > 2 ? pb.n[2] : 1)),
                              std::max(pb.np[0], std::max(D > 1 ? pb.np[1] : 1, D > 2 ? pb.np[2] : 1)));
    dim3 grid(pb.n_items, nrhs);
    if (mode == 0 && pb.sf_ok && D >= 2) {
      // one warp per interface, kPointThreads / 32 interfaces per block
      const size_t item_bytes = interface_sf_smem(nbi, nmax, pb.sf_qmax, int(pb.sf_pmax), sizeof(T));
      const int per_block = kPointThreads / 32;
      const size_t sm = item_bytes * per_block;
      const dim3 gsf(unsigned((pb.n_items + per_block - 1) / per_block), unsigned(nrhs));
      auto go_sf = [&](auto kernel) {
        if (sm > 48 * 1024) cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(sm));
        kernel<<<gsf, kPointThreads, sm, st>>>(v, pb.sf_q.get<int32_t>(), pb.sf_x.get<double>(), pb.sf_stride, x, y,
                                              nvec, int64_t(item_bytes / sizeof(T)));
      };
      if (D == 2) go_sf(interface_apply_sf<T, 2, 32>);
      else go_sf(interface_apply_sf<T, 3, 32>);
      return;
    }
    const size_t smem = sizeof(T) * (size_t(nbi) + 4 * size_t(kPointChunk) * D * nmax + 2 * size_t(kPointChunk));
    auto go = [&](auto kernel) {
      if (smem > 48 * 1024) cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
      kernel<<<grid, kPointThreads, smem, st>>>(v, x, y, nvec, mode);
    };
    if (D == 1) go(interface_apply<T, 1>);
    else if (D == 2) go(interface_apply<T, 2>);
    else go(interface_apply<T, 3>);
    return;
  }
  const int nb = pb.n[0] * (D > 1 ? pb.n[1] : 1) * (D > 2 ? pb.n[2] : 1);
  const int nmax = std::max(pb.n[0], std::max(D > 1 ? pb.n[1] : 1, D > 2 ? pb.n[2] : 1));
  const size_t smem = sizeof(T) * (size_t(nb) + 2 * size_t(kPointChunk) * D * nmax + size_t(kPointChunk) * (D + 1));
  dim3 grid(pb.n_items, nrhs);
  auto go = [&](auto kernel) {
    if (smem > 48 * 1024) cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
    kernel<<<grid, kPointThreads, smem, st>>>(v, x, y, nvec, T(P.mass), T(P.kappa), mode, src);
  };
  if (D == 1) go(point_apply<T, 1>);
  else if (D == 2) go(point_apply<T, 2>);
  else go(point_apply<T, 3>);
}

}  // namespace

// Exact local-matrix diagonal contribution of one point item whose reduced map is not a direct
// injection (cell_diagonal!/face and surface diagonals, accumulators.jl:1056-1083, 1163-1187).
void accumulate_point_item_diagonal(const GricoPlanDesc& d, const GricoPointBatchDesc& pb, const int* n, int64_t it,
                                    int64_t pit, int64_t nb, const std::vector<int32_t>& rmap, const std::vector<double>& rcoef,
                                    const std::vector<int64_t>& toff, const std::vector<int32_t>& tidx,
                                    const std::vector<double>& tcoef, std::map<int64_t, double>& out) {
  const int D = d.dim;
  std::vector<double> A(nb * nb, 0.0), phi(nb), gr(3 * nb);
  double v[3][17], dv[3][17];
  for (int64_t p = pb.point_offsets[pit]; p < pb.point_offsets[pit + 1]; ++p) {
    for (int a = 0; a < D; ++a) {
      fe_basis(pb.ref_points[p * D + a], n[a] - 1, v[a], dv[a]);
      const double s = 2.0 / pb.cell_size[pit * D + a];
      for (int i = 0; i < n[a]; ++i) dv[a][i] *= s;
    }
    for (int64_t i = 0; i < nb; ++i) {
      int mi[3] = {int(i % n[0]), int((i / n[0]) % n[1]), int(i / (n[0] * n[1]))};
      double val = 1.0;
      for (int a = 0; a < D; ++a) val *= v[a][mi[a]];
      phi[i] = val;
      for (int a = 0; a < D; ++a) {
        double g = dv[a][mi[a]];
        for (int e = 0; e < D; ++e)
          if (e != a) g *= v[e][mi[e]];
        gr[a * nb + i] = g;
      }
    }
    const double w = pb.weights[p];
    for (int64_t i = 0; i < nb; ++i)
      for (int64_t j = 0; j < nb; ++j) {
        double aij;
        if (pb.kind == GRICO_ITEM_NITSCHE) {
          // test i, trial j: phi_i(-dn phi_j + eta phi_j) + grad phi_i . (-phi_j n)
          double dnj = 0.0, dni = 0.0;
          for (int a = 0; a < D; ++a) {
            dnj += gr[a * nb + j] * pb.normals[p * D + a];
            dni += gr[a * nb + i] * pb.normals[p * D + a];
          }
          aij = phi[i] * (-dnj + pb.eta[pit] * phi[j]) - dni * phi[j];
        } else {
          double g = 0.0;
          for (int a = 0; a < D; ++a) g += gr[a * nb + i] * gr[a * nb + j];
          const double k = d.kappa * (pb.kappa_points ? pb.kappa_points[p] : 1.0);
          aij = d.mass * phi[i] * phi[j] + k * g;
        }
        A[i * nb + j] += w * aij;
      }
  }
  std::map<int64_t, std::vector<std::pair<int64_t, double>>> by_dof;
  for (int64_t i = 0; i < nb; ++i) {
    const int32_t e = rmap[it * nb + i];
    if (e >= 0) by_dof[e].emplace_back(i, rcoef[it * nb + i]);
    else if (e <= -2) {
      const int64_t k = -(int64_t(e) + 2);
      for (int64_t t = toff[k]; t < toff[k + 1]; ++t) by_dof[tidx[t]].emplace_back(i, tcoef[t]);
    }
  }
  for (auto& kv : by_dof) {
    double s = 0.0;
    for (auto& a : kv.second)
      for (auto& b : kv.second) s += a.second * A[a.first * nb + b.first] * b.second;
    out[kv.first] += s;
  }
}

// The same for a two-sided interface item (local matrix of the SIPG form over the minus and plus
// modes, test i trial j: -[phi_i]{dphi_j/dn} - {dphi_i/dn}[phi_j] + sigma [phi_i][phi_j]).
void accumulate_interface_item_diagonal(const GricoPlanDesc& d, const GricoPointBatchDesc& pb, const int* nm,
                                        const int* npl, int64_t it, int64_t nb, const std::vector<int32_t>& rmap,
                                        const std::vector<double>& rcoef, const std::vector<int64_t>& toff,
                                        const std::vector<int32_t>& tidx, const std::vector<double>& tcoef,
                                        std::map<int64_t, double>& out) {
  const int D = d.dim;
  const int ax = pb.face_axis[it];
  const int64_t nbm = box_count(D, nm);
  std::vector<double> A(nb * nb, 0.0), jump(nb), avg(nb);
  double v[3][17], dv[3][17];
  for (int64_t p = pb.point_offsets[it]; p < pb.point_offsets[it + 1]; ++p) {
    for (int side = 0; side < 2; ++side) {
      const int* n = side ? npl : nm;
      const double* ref = side ? pb.ref_points_plus : pb.ref_points;
      const double* h = side ? pb.cell_size_plus : pb.cell_size;
      for (int a = 0; a < D; ++a) {
        fe_basis(ref[p * D + a], n[a] - 1, v[a], dv[a]);
        for (int i = 0; i < n[a]; ++i) dv[a][i] *= 2.0 / h[it * D + a];
      }
      const int64_t cnt = box_count(D, n), off = side ? nbm : 0;
      for (int64_t i = 0; i < cnt; ++i) {
        const int mi[3] = {int(i % n[0]), int((i / n[0]) % n[1]), int(i / (n[0] * n[1]))};
        double val = 1.0, dn = 1.0;
        for (int a = 0; a < D; ++a) {
          val *= v[a][mi[a]];
          dn *= a == ax ? dv[a][mi[a]] : v[a][mi[a]];
        }
        jump[off + i] = side ? -val : val;
        avg[off + i] = 0.5 * dn;
      }
    }
    const double w = pb.weights[p], sigma = pb.eta[it];
    for (int64_t i = 0; i < nb; ++i)
      for (int64_t j = 0; j < nb; ++j)
        A[i * nb + j] += w * (-jump[i] * avg[j] - avg[i] * jump[j] + sigma * jump[i] * jump[j]);
  }
  std::map<int64_t, std::vector<std::pair<int64_t, double>>> by_dof;
  for (int64_t i = 0; i < nb; ++i) {
    const int32_t e = rmap[it * nb + i];
    if (e >= 0) by_dof[e].emplace_back(i, rcoef[it * nb + i]);
    else if (e <= -2) {
      const int64_t k = -(int64_t(e) + 2);
      for (int64_t t = toff[k]; t < toff[k + 1]; ++t) by_dof[tidx[t]].emplace_back(i, tcoef[t]);
    }
  }
  for (auto& kv : by_dof) {
    double s = 0.0;
    for (auto& a : kv.second)
      for (auto& b : kv.second) s += a.second * A[a.first * nb + b.first] * b.second;
    out[kv.first] += s;
  }
}

// The same for a subcell item: its kept subcell points are listed as one point item.
void accumulate_subcell_item_diagonal(const GricoPlanDesc& d, const GricoPointBatchDesc& pb, const int* n, int64_t it,
                                      int64_t nb, const std::vector<int32_t>& rmap, const std::vector<double>& rcoef,
                                      const std::vector<int64_t>& toff, const std::vector<int32_t>& tidx,
                                      const std::vector<double>& tcoef, std::map<int64_t, double>& out) {
  const int D = d.dim;
  const int q = pb.qpoints[0];
  std::vector<double> eta(q), W(q);
  gauss_legendre(q, eta.data(), W.data());
  int qp = 1;
  for (int a = 0; a < D; ++a) qp *= q;
  double det = 1.0;
  for (int a = 0; a < D; ++a) det *= 0.5 * pb.cell_size[it * D + a];
  std::vector<double> ref, w, kp;
  for (int64_t s = pb.subcell_offsets[it]; s < pb.subcell_offsets[it + 1]; ++s) {
    const double half = std::ldexp(1.0, -pb.subcell_level[s]);
    for (int p = 0; p < qp; ++p) {
      if (!((pb.subcell_mask[s] >> p) & 1ull)) continue;
      int rem = p;
      double wt = pb.subcell_weight[s] * det;
      for (int a = 0; a < D; ++a) {
        const int j = rem % q;
        rem /= q;
        const double c = -1.0 + double(2 * pb.subcell_pos[s * D + a] + 1) * half;
        ref.push_back(c + half * eta[j]);
        wt *= W[j];
      }
      w.push_back(wt);
      if (pb.kappa_points) kp.push_back(pb.kappa_points[s * qp + p]);
    }
  }
  GricoPointBatchDesc one = {};
  one.n_items = 1;
  one.kind = GRICO_ITEM_CELL;
  int64_t offs[2] = {0, int64_t(w.size())};
  one.point_offsets = offs;
  one.ref_points = ref.data();
  one.weights = w.data();
  one.cell_size = pb.cell_size + it * D;
  one.kappa_points = pb.kappa_points ? kp.data() : nullptr;
  accumulate_point_item_diagonal(d, one, n, it, 0, nb, rmap, rcoef, toff, tidx, tcoef, out);
}

// Exact reduced-diagonal contribution sum_{i,j} M_ir A_ij M_jr of one cell whose reduced map is
// not a direct injection.  The local matrix A of TestChannels(mass*u, kappa*k(x)*grad u) is
// assembled from the 1-D tables (cell_matrix! semantics, accumulators.jl:968-1001).
void accumulate_hanging_diagonal(const GricoPlanDesc& d, const GricoCellBatchDesc& bd, const DevBatch& b, int64_t c,
                                 int64_t nb, const std::vector<int32_t>& rmap, const std::vector<double>& rcoef,
                                 const std::vector<int64_t>& toff, const std::vector<int32_t>& tidx,
                                 const std::vector<double>& tcoef, const std::vector<double>& B,
                                 const std::vector<double>& G, const std::vector<double>& W, int nmax, int qmax,
                                 std::map<int64_t, double>& out) {
  const int dim = d.dim;
  int n[3] = {1, 1, 1}, q[3] = {1, 1, 1};
  double h[3] = {1, 1, 1}, detJ = 1.0;
  for (int a = 0; a < dim; ++a) {
    n[a] = b.n[a];
    q[a] = b.q[a];
    h[a] = bd.cell_size[c * dim + a];
    detJ *= 0.5 * h[a];
  }
  auto Bv = [&](int a, int i, int p) { return B[a * nmax * qmax + i * q[a] + p]; };
  auto Gv = [&](int a, int i, int p) { return G[a * nmax * qmax + i * q[a] + p] * (2.0 / h[a]); };
  // reduced terms of every local mode
  std::vector<std::vector<std::pair<int64_t, double>>> terms(nb);
  for (int64_t i = 0; i < nb; ++i) {
    int32_t v = rmap[c * nb + i];
    if (v >= 0) terms[i].emplace_back(v, rcoef[c * nb + i]);
    else if (v <= -2) {
      int64_t k = -(int64_t(v) + 2);
      for (int64_t t = toff[k]; t < toff[k + 1]; ++t) terms[i].emplace_back(tidx[t], tcoef[t]);
    }
  }
  auto digit = [&](int64_t i, int a) {
    for (int e = 0; e < a; ++e) i /= n[e];
    return int(i % n[a]);
  };
  std::vector<double> A(nb * nb, 0.0);
  if (!bd.kappa_points) {
    // 1-D mass and stiffness factors: A = detJ [mass prod_a M_a + kappa sum_a s_a^2 K_a prod_{b!=a} M_b]
    std::vector<double> M1(3 * 16 * 16, 0.0), K1(3 * 16 * 16, 0.0);
    for (int a = 0; a < dim; ++a)
      for (int i = 0; i < n[a]; ++i)
        for (int j = 0; j < n[a]; ++j) {
          double m = 0.0, k = 0.0;
          for (int p = 0; p < q[a]; ++p) {
            m += W[a * qmax + p] * Bv(a, i, p) * Bv(a, j, p);
            k += W[a * qmax + p] * Gv(a, i, p) * Gv(a, j, p);
          }
          M1[a * 256 + i * 16 + j] = m;
          K1[a * 256 + i * 16 + j] = k;
        }
    for (int64_t i = 0; i < nb; ++i)
      for (int64_t j = 0; j < nb; ++j) {
        double mp = 1.0, st = 0.0;
        for (int a = 0; a < dim; ++a) mp *= M1[a * 256 + digit(i, a) * 16 + digit(j, a)];
        for (int a = 0; a < dim; ++a) {
          double t = K1[a * 256 + digit(i, a) * 16 + digit(j, a)];
          for (int e = 0; e < dim; ++e)
            if (e != a) t *= M1[e * 256 + digit(i, e) * 16 + digit(j, e)];
          st += t;
        }
        A[i * nb + j] = detJ * (d.mass * mp + d.kappa * st);
      }
  } else {
    const int64_t nq = int64_t(q[0]) * q[1] * q[2];
    for (int64_t p = 0; p < nq; ++p) {
      int pi[3] = {int(p % q[0]), int((p / q[0]) % q[1]), int(p / (int64_t(q[0]) * q[1]))};
      double w = detJ;
      for (int a = 0; a < dim; ++a) w *= W[a * qmax + pi[a]];
      double kap = d.kappa * bd.kappa_points[c * nq + p];
      std::vector<double> phi(nb), gr(3 * nb);
      for (int64_t i = 0; i < nb; ++i) {
        double bv[3] = {1, 1, 1};
        for (int a = 0; a < dim; ++a) bv[a] = Bv(a, digit(i, a), pi[a]);
        phi[i] = bv[0] * bv[1] * bv[2];
        for (int a = 0; a < dim; ++a) {
          double g = Gv(a, digit(i, a), pi[a]);
          for (int e = 0; e < dim; ++e)
            if (e != a) g *= bv[e];
          gr[a * nb + i] = g;
        }
      }
      for (int64_t i = 0; i < nb; ++i)
        for (int64_t j = 0; j < nb; ++j) {
          double g = 0.0;
          for (int a = 0; a < dim; ++a) g += gr[a * nb + i] * gr[a * nb + j];
          A[i * nb + j] += w * (d.mass * phi[i] * phi[j] + kap * g);
        }
    }
  }
  std::map<int64_t, std::vector<std::pair<int64_t, double>>> by_dof;
  for (int64_t i = 0; i < nb; ++i)
    for (auto& t : terms[i]) by_dof[t.first].emplace_back(i, t.second);
  for (auto& kv : by_dof) {
    double s = 0.0;
    for (auto& x : kv.second)
      for (auto& y : kv.second) s += x.second * A[x.first * nb + y.first] * y.second;
    out[kv.first] += s;
  }
}

template <typename T>
int run_apply(GricoPlan* P, bool reduced, const T* x, T* y, int nrhs, cudaStream_t st, bool y_zero) {
  const int64_t n = reduced ? P->n_red : P->n_full;
  if (nrhs < 1) return GRICO_ERR_INVALID;
  // the final check covers this call's launches only, not an error an earlier call left pending
  (void)cudaGetLastError();
  if (!y_zero) cudaMemsetAsync(y, 0, sizeof(T) * n * nrhs, st);
  // the buffered tails of all batches: one gather pass before the cell kernels
  const GricoPlan::TailAll& TA = P->tails[reduced ? 1 : 0];
  const bool merged = TA.n_tail > 0 && nrhs <= kTailRhs;
  const bool lanes_rhs = nrhs >= kTailLaneRhs;
  const dim3 tg(int(std::min<int64_t>(((lanes_rhs ? TA.n_seg : TA.n_tail) * 32 + 255) / 256, 148 * 16)),
                lanes_rhs ? 1u : unsigned(nrhs));
  if (merged) {
    if (lanes_rhs) {
      cudaMemsetAsync(TA.tx.ptr, 0, sizeof(T) * size_t(TA.n_tail) * nrhs, st);
      tail_gather_seg<T><<<tg, 256, 0, st>>>(TA.seg_k.get<int32_t>(), TA.seg_t.get<int64_t>(), TA.n_seg,
                                             TA.toff.get<int64_t>(), TA.tidx.get<int32_t>(), TA.tcoef.get<double>(),
                                             TA.n_tail, x, n, TA.tx.get<T>(), TA.ty.get<T>(), nrhs);
    } else {
      tail_gather<T><<<tg, 256, 0, st>>>(TA.toff.get<int64_t>(), TA.tidx.get<int32_t>(), TA.tcoef.get<double>(),
                                         TA.n_tail, x, n, TA.tx.get<T>(), TA.ty.get<T>());
    }
  }
  // several batches: round-robin over the branch streams (not while timing batches, whose
  // event pairs need one stream)
  const bool fork = P->n_branches > 1 && !P->time_batches;
  if (fork) {
    cudaEventRecord(P->fork_ev, st);
    for (int k = 0; k < P->n_branches; ++k) cudaStreamWaitEvent(P->branch[k], P->fork_ev, 0);
  }
  int launched = 0;
  auto stream_for = [&]() { return fork ? P->branch[launched++ % P->n_branches] : st; };
  for (size_t bi = 0; bi < P->batches.size(); ++bi) {
    GricoPlan::BatchEvent ev{int(bi), nullptr, nullptr};
    if (P->time_batches && cudaEventCreate(&ev.start) == cudaSuccess && cudaEventCreate(&ev.stop) == cudaSuccess)
      cudaEventRecord(ev.start, st);
    if (merged && TA.base[bi] >= 0)
      launch_batch<T>(*P, P->batches[bi], reduced, x, y, n, 0, nullptr, nrhs, stream_for(), nullptr, 0,
                      TA.tx.get<T>() + TA.base[bi], TA.ty.get<T>() + TA.base[bi], TA.n_tail);
    else
      launch_batch<T>(*P, P->batches[bi], reduced, x, y, n, 0, nullptr, nrhs, stream_for());
    if (ev.stop) {
      cudaEventRecord(ev.stop, st);
      P->batch_events.push_back(ev);
    }
  }
  for (size_t pi = 0; pi < P->pbatches.size(); ++pi) {
    GricoPlan::BatchEvent ev{int(P->batches.size() + pi), nullptr, nullptr};
    if (P->time_batches && cudaEventCreate(&ev.start) == cudaSuccess && cudaEventCreate(&ev.stop) == cudaSuccess)
      cudaEventRecord(ev.start, st);
    launch_points<T>(*P, P->pbatches[pi], reduced, x, y, n, 0, nullptr, nrhs, stream_for());
    if (ev.stop) {
      cudaEventRecord(ev.stop, st);
      P->batch_events.push_back(ev);
    }
  }
  if (fork)
    for (int k = 0; k < P->n_branches; ++k) {
      cudaEventRecord(P->join_ev[k], P->branch[k]);
      cudaStreamWaitEvent(st, P->join_ev[k], 0);
    }
  if (merged) {
    if (lanes_rhs)
      tail_scatter_seg<T><<<tg, 256, 0, st>>>(TA.seg_k.get<int32_t>(), TA.seg_t.get<int64_t>(), TA.n_seg,
                                              TA.toff.get<int64_t>(), TA.tidx.get<int32_t>(), TA.tcoef.get<double>(),
                                              TA.n_tail, TA.ty.get<T>(), y, n, nrhs);
    else
      tail_scatter<T><<<tg, 256, 0, st>>>(TA.toff.get<int64_t>(), TA.tidx.get<int32_t>(), TA.tcoef.get<double>(),
                                          TA.n_tail, TA.ty.get<T>(), y, n);
  }
  if (!reduced && (P->n_fixed + P->n_rel) > 0) {
    dim3 grid(grid_for(P->n_fixed + P->n_rel), nrhs);
    constraint_action<T><<<grid, 256, 0, st>>>(P->fixed.get<int64_t>(), P->n_fixed, P->rel_piv.get<int64_t>(),
                                               P->rel_off.get<int64_t>(), P->rel_idx.get<int64_t>(),
                                               P->rel_coef.get<double>(), P->n_rel, x, y, n);
  }
  return cuda_ok(cudaGetLastError(), "apply launch") ? GRICO_OK : GRICO_ERR_CUDA;
}

template int run_apply<double>(GricoPlan*, bool, const double*, double*, int, cudaStream_t, bool);
template int run_apply<float>(GricoPlan*, bool, const float*, float*, int, cudaStream_t, bool);

namespace {

// Gather CSR of the deterministic apply for one layout, from the device maps of every batch: a
// map entry e of a batch whose local results start at `base` adds coef * local[base + e] to its
// dof (a single-term entry) or coef_t * local[base + e] to each term's dof (an expansion).
bool build_det_map(GricoPlan* P, bool reduced) {
  auto& D = P->det[reduced ? 1 : 0];
  if (D.built) return true;
  const int64_t n = reduced ? P->n_red : P->n_full;
  struct Src {
    int64_t base = 0, ne = 0;
    std::vector<int32_t> map, tidx;
    std::vector<double> coef, tcoef;
    std::vector<int64_t> toff;
  };
  std::vector<Src> src;
  int64_t base = 0;
  auto fetch = [&](const DevMap& m, int64_t ne) {
    Src s;
    s.base = base;
    s.ne = ne;
    s.map.resize(size_t(ne));
    bool ok = ne == 0 || cuda_ok(cudaMemcpy(s.map.data(), m.map.ptr, sizeof(int32_t) * ne, cudaMemcpyDeviceToHost), "det map");
    if (ok && m.coef.ptr) {
      s.coef.resize(size_t(ne));
      ok = cuda_ok(cudaMemcpy(s.coef.data(), m.coef.ptr, sizeof(double) * ne, cudaMemcpyDeviceToHost), "det coef");
    }
    if (ok && m.toff.ptr && m.toff.bytes >= 2 * sizeof(int64_t)) {
      s.toff.resize(m.toff.bytes / sizeof(int64_t));
      ok = cuda_ok(cudaMemcpy(s.toff.data(), m.toff.ptr, m.toff.bytes, cudaMemcpyDeviceToHost), "det tails");
      const int64_t nt = s.toff.back();
      s.tidx.resize(size_t(nt));
      s.tcoef.resize(size_t(nt));
      ok = ok && (nt == 0 || (cuda_ok(cudaMemcpy(s.tidx.data(), m.tidx.ptr, sizeof(int32_t) * nt, cudaMemcpyDeviceToHost), "det tails") &&
                              cuda_ok(cudaMemcpy(s.tcoef.data(), m.tcoef.ptr, sizeof(double) * nt, cudaMemcpyDeviceToHost), "det tails")));
    }
    src.push_back(std::move(s));
    base += ne;
    return ok;
  };
  D.cell_base.clear();
  D.point_base.clear();
  for (const auto& b : P->batches) {
    D.cell_base.push_back(base);
    if (!fetch(reduced ? b.red : b.full, int64_t(b.n_cells) * b.n[0] * b.n[1] * b.n[2])) return false;
  }
  for (const auto& pb : P->pbatches) {
    D.point_base.push_back(base);
    int64_t nb = int64_t(pb.n[0]) * pb.n[1] * pb.n[2];
    if (pb.kind == GRICO_ITEM_INTERFACE) nb += int64_t(pb.np[0]) * pb.np[1] * pb.np[2];
    if (!fetch(reduced ? pb.red : pb.full, int64_t(pb.n_items) * nb)) return false;
  }
  // two passes in one traversal order: count the terms of every dof, then place them
  std::vector<int64_t> off(size_t(n) + 1, 0);
  auto visit = [&](auto&& emit) {
    for (const auto& s : src)
      for (int64_t e = 0; e < s.ne; ++e) {
        const int32_t v = s.map[size_t(e)];
        if (v >= 0) {
          emit(v, s.base + e, s.coef.empty() ? 1.0 : s.coef[size_t(e)]);
        } else if (v <= -2) {
          const int64_t k = -(int64_t(v) + 2);
          for (int64_t t = s.toff[size_t(k)]; t < s.toff[size_t(k) + 1]; ++t)
            emit(s.tidx[size_t(t)], s.base + e, s.tcoef[size_t(t)]);
        }
      }
  };
  visit([&](int64_t d, int64_t, double) { ++off[size_t(d) + 1]; });
  for (int64_t d = 0; d < n; ++d) off[size_t(d) + 1] += off[size_t(d)];
  const size_t n_terms = static_cast<size_t>(off[static_cast<size_t>(n)]);
  std::vector<int32_t> pos(n_terms);
  std::vector<double> coef(n_terms);
  std::vector<int64_t> fill(off.begin(), off.end() - 1);
  visit([&](int64_t d, int64_t p, double c) {
    const int64_t k = fill[size_t(d)]++;
    pos[size_t(k)] = int32_t(p);
    coef[size_t(k)] = c;
  });
  if (!D.off.upload(off) || !D.pos.upload(pos) || !D.coef.upload(coef)) return false;
  D.entries = base;
  D.built = true;
  return true;
}

// GRICO_FLAG_DETERMINISTIC: every batch kernel stores its local results (the one-block kernels,
// no atomics), det_gather sums each dof's terms in the map order, then the constraint rows
template <typename T>
int run_apply_det(GricoPlan* P, bool reduced, const T* x, T* y, int nrhs, cudaStream_t st) {
  const int64_t n = reduced ? P->n_red : P->n_full;
  if (nrhs < 1) return GRICO_ERR_INVALID;
  (void)cudaGetLastError();
  if (!build_det_map(P, reduced)) return GRICO_ERR_CUDA;
  auto& D = P->det[reduced ? 1 : 0];
  if (D.entries >= (int64_t(1) << 31)) {
    set_error("deterministic apply: more than 2^31 local entries");
    return GRICO_ERR_INVALID;
  }
  if (!P->det_local.ensure(sizeof(T) * size_t(std::max<int64_t>(D.entries, 1)) * nrhs)) return GRICO_ERR_CUDA;
  T* loc = P->det_local.get<T>();
  for (size_t bi = 0; bi < P->batches.size(); ++bi)
    launch_batch<T>(*P, P->batches[bi], reduced, x, y, n, 0, nullptr, nrhs, st, loc + D.cell_base[bi], D.entries);
  for (size_t pi = 0; pi < P->pbatches.size(); ++pi)
    launch_points<T>(*P, P->pbatches[pi], reduced, x, y, n, 0, nullptr, nrhs, st, loc + D.point_base[pi], D.entries);
  dim3 grid(grid_for(n), nrhs);
  det_gather<T><<<grid, 256, 0, st>>>(D.off.get<int64_t>(), D.pos.get<int32_t>(), D.coef.get<double>(), n, loc,
                                      D.entries, y, n);
  if (!reduced && (P->n_fixed + P->n_rel) > 0) {
    dim3 cg(grid_for(P->n_fixed + P->n_rel), nrhs);
    constraint_action<T><<<cg, 256, 0, st>>>(P->fixed.get<int64_t>(), P->n_fixed, P->rel_piv.get<int64_t>(),
                                             P->rel_off.get<int64_t>(), P->rel_idx.get<int64_t>(),
                                             P->rel_coef.get<double>(), P->n_rel, x, y, n);
  }
  return cuda_ok(cudaGetLastError(), "deterministic apply launch") ? GRICO_OK : GRICO_ERR_CUDA;
}

}  // namespace

int reduced_diag_device(GricoPlan* P, double* diag, cudaStream_t st) {
  cudaMemsetAsync(diag, 0, sizeof(double) * P->n_red, st);
  for (auto& b : P->batches) launch_batch<double>(*P, b, true, nullptr, diag, P->n_red, 3, nullptr, 1, st);
  for (auto& pb : P->pbatches) launch_points<double>(*P, pb, true, nullptr, diag, P->n_red, 3, nullptr, 1, st);
  if (P->n_hang > 0)
    add_sparse<<<grid_for(P->n_hang), 256, 0, st>>>(P->hang_idx.get<int64_t>(), P->hang_val.get<double>(), P->n_hang,
                                                    diag);
  return cuda_ok(cudaGetLastError(), "diagonal launch") ? GRICO_OK : GRICO_ERR_CUDA;
}

}  // namespace grico

using namespace grico;

extern "C" {

// Host-side validation of a plan descriptor; runs before any CUDA call so malformed descriptors
// are rejected with a precise message (the reference validates plans in check_* helpers).
static int validate_plan_desc(const GricoPlanDesc* d) {
  if (d->form != GRICO_FORM_MASS_DIFFUSION) { set_error("unsupported accumulator form"); return GRICO_ERR_UNSUPPORTED_FORM; }
  if (d->dim < 1 || d->dim > 3 || d->n_full < 0 || d->n_reduced < 0 || d->n_batches < 0 || (d->n_batches && !d->batches)) {
    set_error("grico_plan_create: invalid sizes");
    return GRICO_ERR_INVALID;
  }
  if (d->n_full >= (int64_t(1) << 31)) { set_error("grico_plan_create: more than 2^31-1 dofs"); return GRICO_ERR_INVALID; }
  if (!d->red_offsets) { set_error("grico_plan_create: reduced map missing"); return GRICO_ERR_INVALID; }
  for (int bi = 0; bi < d->n_batches; ++bi) {
    const GricoCellBatchDesc& bd = d->batches[bi];
    if (bd.n_cells < 0 || (bd.n_cells > 0 && (!bd.map_index || !bd.cell_size))) {
      set_error("batch " + std::to_string(bi) + ": missing map or cell sizes");
      return GRICO_ERR_INVALID;
    }
    int n[3] = {1, 1, 1};
    for (int a = 0; a < d->dim; ++a) {
      n[a] = bd.degree[a] + 1;
      if (n[a] < 1 || n[a] > 16 || bd.qpoints[a] < 1 || bd.qpoints[a] > 16) {
        set_error("batch " + std::to_string(bi) + ": degree/quadrature out of range");
        return GRICO_ERR_INVALID;
      }
    }
    if (bd.n_tail < 0 || (bd.n_tail > 0 && (!bd.tail_offsets || !bd.tail_index || !bd.tail_coef))) {
      set_error("batch " + std::to_string(bi) + ": invalid multi-term tail");
      return GRICO_ERR_INVALID;
    }
    const int64_t ne = int64_t(bd.n_cells) * box_count(d->dim, n);
    for (int64_t e = 0; e < ne; ++e) {
      const int32_t v = bd.map_index[e];
      if (v >= d->n_full || (v <= -2 && -(int64_t(v) + 2) >= bd.n_tail)) {
        set_error("batch " + std::to_string(bi) + ": map entry " + std::to_string(e) + " = " + std::to_string(v) +
                  " out of range (n_full " + std::to_string(d->n_full) + ", tails " + std::to_string(bd.n_tail) + ")");
        return GRICO_ERR_INVALID;
      }
    }
    for (int64_t k = 0; k < bd.n_tail; ++k)
      for (int64_t t = bd.tail_offsets[k]; t < bd.tail_offsets[k + 1]; ++t)
        if (bd.tail_index[t] < 0 || bd.tail_index[t] >= d->n_full) {
          set_error("batch " + std::to_string(bi) + ": tail index out of range");
          return GRICO_ERR_INVALID;
        }
  }
  if (d->n_point_batches < 0 || (d->n_point_batches && !d->point_batches)) {
    set_error("grico_plan_create: invalid point batches");
    return GRICO_ERR_INVALID;
  }
  for (int bi = 0; bi < d->n_point_batches; ++bi) {
    const GricoPointBatchDesc& pb = d->point_batches[bi];
    const std::string tag = "point batch " + std::to_string(bi);
    if (pb.kind != GRICO_ITEM_CELL && pb.kind != GRICO_ITEM_NITSCHE && pb.kind != GRICO_ITEM_SUBCELLS &&
        pb.kind != GRICO_ITEM_INTERFACE) {
      set_error(tag + ": unknown item kind");
      return GRICO_ERR_UNSUPPORTED_FORM;
    }
    const bool sub = pb.kind == GRICO_ITEM_SUBCELLS;
    if (pb.n_items < 0 || (pb.n_items > 0 && (!pb.map_index || !pb.cell_size ||
                                              (!sub && (!pb.point_offsets || !pb.ref_points || !pb.weights)) ||
                                              (sub && (!pb.subcell_offsets || !pb.subcell_level || !pb.subcell_pos ||
                                                       !pb.subcell_mask || !pb.subcell_weight))))) {
      set_error(tag + ": missing arrays");
      return GRICO_ERR_INVALID;
    }
    if (sub) {
      const int nn = pb.degree[0] + 1, q = pb.qpoints[0];
      int qp = 1;
      for (int a = 0; a < d->dim; ++a) {
        if (pb.degree[a] != pb.degree[0] || pb.qpoints[a] != q) { set_error(tag + ": subcell items need isotropic degree and quadrature"); return GRICO_ERR_UNSUPPORTED_FORM; }
        qp *= q;
      }
      if (qp > 64 || !subcell_shape_supported(d->dim, nn, q)) { set_error(tag + ": subcell kernel not compiled for this degree/quadrature"); return GRICO_ERR_UNSUPPORTED_FORM; }
      if (pb.n_items > 0 && pb.subcell_offsets[0] != 0) { set_error(tag + ": subcell offsets must start at 0"); return GRICO_ERR_INVALID; }
      for (int64_t it = 0; it < pb.n_items; ++it)
        if (pb.subcell_offsets[it + 1] < pb.subcell_offsets[it]) { set_error(tag + ": subcell offsets must not decrease"); return GRICO_ERR_INVALID; }
      const int64_t ns = pb.n_items > 0 ? pb.subcell_offsets[pb.n_items] : 0;
      for (int64_t s2 = 0; s2 < ns; ++s2) {
        const int lev = pb.subcell_level[s2];
        if (lev < 0 || lev > 30) { set_error(tag + ": subcell level out of range"); return GRICO_ERR_INVALID; }
        for (int a = 0; a < d->dim; ++a) {
          const int32_t ps = pb.subcell_pos[s2 * d->dim + a];
          if (ps < 0 || int64_t(ps) >= (int64_t(1) << lev)) { set_error(tag + ": subcell position out of range"); return GRICO_ERR_INVALID; }
        }
      }
    }
    if (pb.kind == GRICO_ITEM_NITSCHE && pb.n_items > 0 && (!pb.normals || !pb.eta)) { set_error(tag + ": Nitsche items need normals and eta"); return GRICO_ERR_INVALID; }
    const bool iface = pb.kind == GRICO_ITEM_INTERFACE;
    if (iface && pb.n_items > 0 && (!pb.eta || !pb.ref_points_plus || !pb.cell_size_plus || !pb.face_axis)) {
      set_error(tag + ": interface items need eta, plus-side points and sizes, and face axes");
      return GRICO_ERR_INVALID;
    }
    int n[3] = {1, 1, 1}, np_[3] = {1, 1, 1};
    for (int a = 0; a < d->dim; ++a) {
      n[a] = pb.degree[a] + 1;
      if (n[a] < 1 || n[a] > 16) { set_error(tag + ": degree out of range"); return GRICO_ERR_INVALID; }
      if (iface) {
        np_[a] = pb.degree_plus[a] + 1;
        if (np_[a] < 1 || np_[a] > 16) { set_error(tag + ": plus-side degree out of range"); return GRICO_ERR_INVALID; }
      }
    }
    const int64_t nb = box_count(d->dim, n) + (iface ? box_count(d->dim, np_) : 0);
    if (nb > int64_t(iface ? kIfaceModes : kMaxModes) * kPointThreads) { set_error(tag + ": too many local modes for point items"); return GRICO_ERR_INVALID; }
    for (int64_t it = 0; iface && it < pb.n_items; ++it)
      if (pb.face_axis[it] < 0 || pb.face_axis[it] >= d->dim) { set_error(tag + ": face axis out of range"); return GRICO_ERR_INVALID; }
    if (!sub && pb.point_offsets && pb.n_items > 0 && pb.point_offsets[0] != 0) { set_error(tag + ": point offsets must start at 0"); return GRICO_ERR_INVALID; }
    for (int64_t it = 0; !sub && it < pb.n_items; ++it)
      if (pb.point_offsets[it + 1] < pb.point_offsets[it]) { set_error(tag + ": point offsets must not decrease"); return GRICO_ERR_INVALID; }
    if (pb.n_tail < 0 || (pb.n_tail > 0 && (!pb.tail_offsets || !pb.tail_index || !pb.tail_coef))) { set_error(tag + ": invalid tail"); return GRICO_ERR_INVALID; }
    for (int64_t e = 0; e < int64_t(pb.n_items) * nb; ++e) {
      const int32_t v = pb.map_index[e];
      if (v >= d->n_full || (v <= -2 && -(int64_t(v) + 2) >= pb.n_tail)) { set_error(tag + ": map entry out of range"); return GRICO_ERR_INVALID; }
    }
    for (int64_t k = 0; k < pb.n_tail; ++k)
      for (int64_t t = pb.tail_offsets[k]; t < pb.tail_offsets[k + 1]; ++t)
        if (pb.tail_index[t] < 0 || pb.tail_index[t] >= d->n_full) { set_error(tag + ": tail index out of range"); return GRICO_ERR_INVALID; }
  }
  for (int64_t i = 0; i < d->n_fixed; ++i)
    if (d->fixed_dofs[i] < 0 || d->fixed_dofs[i] >= d->n_full) { set_error("fixed dof out of range"); return GRICO_ERR_INVALID; }
  for (int64_t r = 0; r < d->n_relations; ++r) {
    if (d->rel_pivot[r] < 0 || d->rel_pivot[r] >= d->n_full) { set_error("relation pivot out of range"); return GRICO_ERR_INVALID; }
    for (int64_t t = d->rel_offsets[r]; t < d->rel_offsets[r + 1]; ++t)
      if (d->rel_index[t] < 0 || d->rel_index[t] >= d->n_full) { set_error("relation index out of range"); return GRICO_ERR_INVALID; }
  }
  for (int64_t i = 0; i < d->n_full; ++i)
    for (int64_t t = d->red_offsets[i]; t < d->red_offsets[i + 1]; ++t)
      if (d->red_index[t] < 0 || d->red_index[t] >= d->n_reduced) { set_error("reduced map index out of range"); return GRICO_ERR_INVALID; }
  return GRICO_OK;
}

int grico_plan_create(const GricoPlanDesc* d, GricoPlan** out) {
  if (!d || !out) { set_error("grico_plan_create: null argument"); return GRICO_ERR_INVALID; }
  if (int rc = validate_plan_desc(d)) return rc;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    set_error("grico_plan_create: no CUDA device (the library has no CPU fallback)");
    return GRICO_ERR_NO_DEVICE;
  }
  if (d->form != GRICO_FORM_MASS_DIFFUSION) { set_error("unsupported accumulator form"); return GRICO_ERR_UNSUPPORTED_FORM; }
  if (d->dim < 1 || d->dim > 3 || d->n_full < 0 || d->n_reduced < 0 || d->n_batches < 0) {
    set_error("grico_plan_create: invalid sizes");
    return GRICO_ERR_INVALID;
  }
  if (d->n_full >= (int64_t(1) << 31)) { set_error("grico_plan_create: more than 2^31-1 dofs"); return GRICO_ERR_INVALID; }
  std::unique_ptr<GricoPlan> P(new GricoPlan());
  P->dim = d->dim;
  P->mass = d->mass;
  P->kappa = d->kappa;
  P->n_full = d->n_full;
  P->n_red = d->n_reduced;
  if (!cuda_ok(cudaStreamCreateWithFlags(&P->stream, cudaStreamNonBlocking), "stream")) return GRICO_ERR_CUDA;
  for (int bi = 0; bi < d->n_batches; ++bi) {
    const GricoCellBatchDesc& bd = d->batches[bi];
    DevBatch b;
    b.n_cells = bd.n_cells;
    int nmax = 1, qmax = 1;
    for (int a = 0; a < d->dim; ++a) {
      b.n[a] = bd.degree[a] + 1;
      b.q[a] = bd.qpoints[a];
      if (b.q[a] < 1 || b.n[a] < 1 || b.n[a] > 16 || b.q[a] > 16) { set_error("batch degree/quadrature out of range"); return GRICO_ERR_INVALID; }
      nmax = std::max(nmax, b.n[a]);
      qmax = std::max(qmax, b.q[a]);
    }
    b.isotropic = true;
    for (int a = 1; a < d->dim; ++a) b.isotropic &= (b.n[a] == b.n[0] && b.q[a] == b.q[0]);
    if (d->dim == 3) {
      b.tile[0] = default_tile_3d(b.q[0], false);
      b.tile[1] = default_tile_3d(b.q[0], true);
    }
    const int64_t nb = box_count(d->dim, b.n);
    const int64_t ne = int64_t(bd.n_cells) * nb;
    for (int64_t e = 0; e < ne; ++e) {
      int32_t v = bd.map_index[e];
      if (v >= d->n_full || (v <= -2 && -(int64_t(v) + 2) >= bd.n_tail)) {
        set_error("batch map index out of range");
        return GRICO_ERR_INVALID;
      }
    }
    // 1-D tables per axis: B, G [dim][nmax*qmax], W [dim][qmax], D of axis 0
    std::vector<double> B(d->dim * nmax * qmax, 0.0), G(d->dim * nmax * qmax, 0.0), W(d->dim * qmax, 0.0);
    std::vector<double> Dm;
    for (int a = 0; a < d->dim; ++a) {
      std::vector<double> pts(b.q[a]), wts(b.q[a]);
      gauss_legendre(b.q[a], pts.data(), wts.data());
      std::vector<double> v(b.n[a] + 1), g(b.n[a] + 1);
      for (int p = 0; p < b.q[a]; ++p) {
        fe_basis(pts[p], b.n[a] - 1, v.data(), g.data());
        for (int i = 0; i < b.n[a]; ++i) {
          B[a * nmax * qmax + i * b.q[a] + p] = v[i];
          G[a * nmax * qmax + i * b.q[a] + p] = g[i];
        }
        W[a * qmax + p] = wts[p];
      }
      if (a == 0) Dm = collocation_derivative(pts);
    }
    b.hB.assign(B.begin(), B.begin() + b.n[0] * b.q[0]);
    b.hD = Dm;
    b.hW.assign(W.begin(), W.begin() + b.q[0]);
    bool ok = b.B.upload(B) && b.G.upload(G) && b.W.upload(W) && b.D.upload(Dm);
    ok = ok && b.h.upload(bd.cell_size, size_t(bd.n_cells) * d->dim);
    // uniform batch: the element matrix of the sum-factorised kernel, once, for the FP32
    // tensor-core apply (K_e = det J [mass M (x) M (x) M + kappa sum_a (2 / h_a)^2 (1-D
    // stiffness on axis a, mass on the others)], 1-D mass M = B W B^T, stiffness S = G W G^T)
    b.dense_ok = false;
    if (d->dim == 3 && b.isotropic && b.q[0] >= b.n[0] && nb <= dense::kK && !bd.kappa_points && bd.n_cells > 0) {
      bool uniform = true;
      for (int64_t c = 1; c < bd.n_cells && uniform; ++c)
        for (int a = 0; a < 3; ++a) uniform = uniform && bd.cell_size[c * 3 + a] == bd.cell_size[a];
      if (uniform) {
        const int n = b.n[0], q = b.q[0];
        std::vector<double> M1(size_t(n) * n, 0.0), S1(size_t(n) * n, 0.0);
        for (int i = 0; i < n; ++i)
          for (int j = 0; j < n; ++j)
            for (int p = 0; p < q; ++p) {
              M1[i * n + j] += W[p] * B[i * q + p] * B[j * q + p];
              S1[i * n + j] += W[p] * G[i * q + p] * G[j * q + p];
            }
        const double* h = bd.cell_size;
        const double detJ = h[0] * h[1] * h[2] * 0.125;
        const double s0 = 4.0 / (h[0] * h[0]), s1 = 4.0 / (h[1] * h[1]), s2 = 4.0 / (h[2] * h[2]);
        std::vector<double> Ke(size_t(nb) * nb);
        for (int iz = 0; iz < n; ++iz)
          for (int iy = 0; iy < n; ++iy)
            for (int ix = 0; ix < n; ++ix)
              for (int jz = 0; jz < n; ++jz)
                for (int jy = 0; jy < n; ++jy)
                  for (int jx = 0; jx < n; ++jx) {
                    const double mx = M1[ix * n + jx], my = M1[iy * n + jy], mz = M1[iz * n + jz];
                    const double sx = S1[ix * n + jx], sy = S1[iy * n + jy], sz = S1[iz * n + jz];
                    Ke[size_t(ix + n * (iy + n * iz)) * nb + (jx + n * (jy + n * jz))] =
                        detJ * (P->mass * mx * my * mz + P->kappa * (s0 * sx * my * mz + s1 * mx * sy * mz + s2 * mx * my * sz));
                  }
        std::vector<__nv_bfloat16> wp(2 * size_t(dense::kPiece) / sizeof(__nv_bfloat16));
        dense::pack_element_matrix(Ke.data(), int(nb), wp.data());
        ok = ok && b.dense.upload(wp);
        b.dense_ok = true;  // selectable (grico_plan_set_tiles, the autotuner); not the default
      }
    }
    if (bd.kappa_points) {
      int64_t nq = 1;
      for (int a = 0; a < d->dim; ++a) nq *= b.q[a];
      ok = ok && b.kappa.upload(bd.kappa_points, size_t(bd.n_cells) * nq);
    }
    // full-layout map
    ok = ok && b.full.map.upload(bd.map_index, size_t(ne));
    if (bd.map_coef) ok = ok && b.full.coef.upload(bd.map_coef, size_t(ne));
    if (bd.n_tail > 0) {
      ok = ok && b.full.toff.upload(bd.tail_offsets, size_t(bd.n_tail + 1));
      ok = ok && b.full.tidx.upload(bd.tail_index, size_t(bd.tail_offsets[bd.n_tail]));
      ok = ok && b.full.tcoef.upload(bd.tail_coef, size_t(bd.tail_offsets[bd.n_tail]));
      ok = ok && setup_tail_buffer(b.full, bd.map_index, ne, bd.tail_offsets, bd.n_tail);
    }
    // reduced-layout map
    std::vector<int32_t> rmap, tidx;
    std::vector<double> rcoef, tcoef;
    std::vector<int64_t> toff;
    bool need_coef = false;
    compose_reduced(bd, nb, *d, rmap, rcoef, need_coef, toff, tidx, tcoef);
    ok = ok && b.red.map.upload(rmap);
    if (need_coef) ok = ok && b.red.coef.upload(rcoef);
    if (toff.size() > 1)
      ok = ok && b.red.toff.upload(toff) && b.red.tidx.upload(tidx) && b.red.tcoef.upload(tcoef) &&
           setup_tail_buffer(b.red, rmap.data(), int64_t(rmap.size()), toff.data(), int64_t(toff.size()) - 1);
    b.red_multiterm = toff.size() > 1;
    // Cells whose reduced map couples several local modes to one reduced dof (hanging-node
    // expansions) need off-diagonal local entries for the exact Jacobi diagonal; the reference
    // probes with one reduced apply per dof instead (solve.jl:722-738).  Their contribution is
    // computed here once from the tensor-product local matrix; the device diagonal kernel skips
    // them.
    {
      std::vector<uint8_t> skip(bd.n_cells, 0);
      int64_t hanging = 0;
      std::vector<std::pair<int64_t, double>> ent;
      for (int64_t c = 0; c < bd.n_cells; ++c) {
        ent.clear();
        for (int64_t i = 0; i < nb; ++i) {
          int32_t v = rmap[c * nb + i];
          if (v >= 0) ent.emplace_back(v, 0.0);
          else if (v <= -2) { skip[c] = 1; break; }
        }
        if (!skip[c]) {
          std::sort(ent.begin(), ent.end());
          for (size_t k = 1; k < ent.size(); ++k)
            if (ent[k].first == ent[k - 1].first) { skip[c] = 1; break; }
        }
        if (!skip[c]) continue;
        ++hanging;
        accumulate_hanging_diagonal(*d, bd, b, c, nb, rmap, rcoef, toff, tidx, tcoef, B, G, W, nmax, qmax,
                                    P->hang_diag);
      }
      if (hanging) ok = ok && b.skip.upload(skip);
    }
    if (!ok) return GRICO_ERR_CUDA;
    P->batches.push_back(std::move(b));
  }
  for (int bi = 0; bi < d->n_point_batches; ++bi) {
    const GricoPointBatchDesc& pd = d->point_batches[bi];
    DevPointBatch pb;
    pb.n_items = pd.n_items;
    pb.kind = pd.kind;
    for (int a = 0; a < d->dim; ++a) pb.n[a] = pd.degree[a] + 1;
    const bool iface = pd.kind == GRICO_ITEM_INTERFACE;
    if (iface)
      for (int a = 0; a < d->dim; ++a) pb.np[a] = pd.degree_plus[a] + 1;
    const int64_t nb = box_count(d->dim, pb.n) + (iface ? box_count(d->dim, pb.np) : 0);
    const int64_t ne = int64_t(pd.n_items) * nb;
    bool ok = pb.full.map.upload(pd.map_index, size_t(ne)) && pb.h.upload(pd.cell_size, size_t(pd.n_items) * d->dim);
    if (pd.kind == GRICO_ITEM_SUBCELLS) {
      int qp = 1;
      for (int a = 0; a < d->dim; ++a) {
        pb.q[a] = pd.qpoints[a];
        qp *= pd.qpoints[a];
      }
      pb.n_sub = pd.n_items > 0 ? pd.subcell_offsets[pd.n_items] : 0;
      pb.n_points = pb.n_sub * qp;
      ok = ok && pb.sub_off.upload(pd.subcell_offsets, size_t(pd.n_items + 1)) &&
           pb.sub_level.upload(pd.subcell_level, size_t(pb.n_sub)) &&
           pb.sub_pos.upload(pd.subcell_pos, size_t(pb.n_sub) * d->dim) &&
           pb.sub_mask.upload(pd.subcell_mask, size_t(pb.n_sub)) && pb.sub_w.upload(pd.subcell_weight, size_t(pb.n_sub));
      pb.hEta.resize(pb.q[0]);
      pb.hW.resize(pb.q[0]);
      gauss_legendre(pb.q[0], pb.hEta.data(), pb.hW.data());
      pb.hDm = collocation_derivative(pb.hEta);
    } else {
      pb.n_points = pd.n_items > 0 ? pd.point_offsets[pd.n_items] : 0;
      ok = ok && pb.pt_off.upload(pd.point_offsets, size_t(pd.n_items + 1)) &&
           pb.ref.upload(pd.ref_points, size_t(pb.n_points) * d->dim) && pb.w.upload(pd.weights, size_t(pb.n_points));
    }
    if (pd.map_coef) ok = ok && pb.full.coef.upload(pd.map_coef, size_t(ne));
    if (pd.n_tail > 0)
      ok = ok && pb.full.toff.upload(pd.tail_offsets, size_t(pd.n_tail + 1)) &&
           pb.full.tidx.upload(pd.tail_index, size_t(pd.tail_offsets[pd.n_tail])) &&
           pb.full.tcoef.upload(pd.tail_coef, size_t(pd.tail_offsets[pd.n_tail]));
    if (pd.kind == GRICO_ITEM_NITSCHE)
      ok = ok && pb.nrm.upload(pd.normals, size_t(pb.n_points) * d->dim) && pb.eta.upload(pd.eta, size_t(pd.n_items));
    if (iface)
      ok = ok && pb.eta.upload(pd.eta, size_t(pd.n_items)) &&
           pb.ref_p.upload(pd.ref_points_plus, size_t(pb.n_points) * d->dim) &&
           pb.h_p.upload(pd.cell_size_plus, size_t(pd.n_items) * d->dim) && pb.axis.upload(pd.face_axis, size_t(pd.n_items));
    if (iface && d->dim >= 2 && pd.n_items > 0) {
      // the sum-factorised kernel applies when every item's points are a tensor grid over the
      // tangential axes t1 < t2 (t1 fastest) with one normal coordinate per side
      const int D = d->dim;
      int64_t pmax = 1;
      for (int64_t it = 0; it < pd.n_items; ++it)
        pmax = std::max<int64_t>(pmax, pd.point_offsets[it + 1] - pd.point_offsets[it]);
      const int stride = 2 * int(pmax + 2);
      std::vector<int32_t> qv(2 * size_t(pd.n_items));
      std::vector<double> xv(size_t(pd.n_items) * stride, 0.0);
      bool sf = true;
      int qmax = 1;
      for (int64_t it = 0; it < pd.n_items && sf; ++it) {
        const int ax = pd.face_axis[it];
        const int t1 = ax == 0 ? 1 : 0, t2 = D == 3 ? (ax == 2 ? 1 : 2) : -1;
        const int64_t p0 = pd.point_offsets[it], cnt = pd.point_offsets[it + 1] - p0;
        if (cnt < 1 || ax < 0 || ax >= D) {
          sf = false;
          break;
        }
        int64_t q1 = cnt;
        if (D == 3) {
          q1 = 1;
          while (q1 < cnt && pd.ref_points[(p0 + q1) * D + t2] == pd.ref_points[p0 * D + t2]) ++q1;
        }
        if (cnt % q1) {
          sf = false;
          break;
        }
        const int64_t q2 = cnt / q1;
        for (int side = 0; side < 2 && sf; ++side) {
          const double* R = side ? pd.ref_points_plus : pd.ref_points;
          double* c = xv.data() + it * stride + side * (q1 + q2 + 1);
          for (int64_t p = 0; p < cnt && sf; ++p) {
            const int64_t p1 = p % q1, p2 = p / q1;
            const double* r = R + (p0 + p) * D;
            if (p2 == 0) c[p1] = r[t1];
            if (p1 == 0) c[q1 + p2] = D == 3 ? r[t2] : 0.0;
            if (p == 0) c[q1 + q2] = r[ax];
            sf = r[t1] == c[p1] && (D < 3 || r[t2] == c[q1 + p2]) && r[ax] == c[q1 + q2];
          }
        }
        qv[2 * it] = int32_t(q1);
        qv[2 * it + 1] = int32_t(q2);
        qmax = std::max<int>(qmax, int(std::max(q1, q2)));
      }
      if (sf) {
        ok = ok && pb.sf_q.upload(qv) && pb.sf_x.upload(xv);
        pb.sf_ok = true;
        pb.sf_stride = stride;
        pb.sf_qmax = qmax;
        pb.sf_pmax = pmax;
      }
    }
    if (pd.kappa_points) ok = ok && pb.kpts.upload(pd.kappa_points, size_t(pb.n_points));
    std::vector<int32_t> rmap, tidx;
    std::vector<double> rcoef, tcoef;
    std::vector<int64_t> toff;
    bool need_coef = false;
    compose_reduced(pd, nb, *d, rmap, rcoef, need_coef, toff, tidx, tcoef);
    ok = ok && pb.red.map.upload(rmap);
    if (need_coef) ok = ok && pb.red.coef.upload(rcoef);
    if (toff.size() > 1) ok = ok && pb.red.toff.upload(toff) && pb.red.tidx.upload(tidx) && pb.red.tcoef.upload(tcoef);
    std::vector<uint8_t> skip(pd.n_items, 0);
    int64_t hanging = 0;
    std::vector<int64_t> seen;
    for (int64_t it = 0; it < pd.n_items; ++it) {
      seen.clear();
      for (int64_t i = 0; i < nb; ++i) {
        const int32_t v = rmap[it * nb + i];
        if (v >= 0) seen.push_back(v);
        else if (v <= -2) { skip[it] = 1; break; }
      }
      if (!skip[it]) {
        std::sort(seen.begin(), seen.end());
        if (std::adjacent_find(seen.begin(), seen.end()) != seen.end()) skip[it] = 1;
      }
      if (!skip[it]) continue;
      ++hanging;
      if (pd.kind == GRICO_ITEM_SUBCELLS)
        accumulate_subcell_item_diagonal(*d, pd, pb.n, it, nb, rmap, rcoef, toff, tidx, tcoef, P->hang_diag);
      else if (iface)
        accumulate_interface_item_diagonal(*d, pd, pb.n, pb.np, it, nb, rmap, rcoef, toff, tidx, tcoef, P->hang_diag);
      else
        accumulate_point_item_diagonal(*d, pd, pb.n, it, it, nb, rmap, rcoef, toff, tidx, tcoef, P->hang_diag);
    }
    if (hanging) ok = ok && pb.skip.upload(skip);
    if (!ok) return GRICO_ERR_CUDA;
    P->pbatches.push_back(std::move(pb));
  }
  if (!P->hang_diag.empty()) {
    std::vector<int64_t> hi;
    std::vector<double> hv;
    for (auto& kv : P->hang_diag) { hi.push_back(kv.first); hv.push_back(kv.second); }
    if (!P->hang_idx.upload(hi) || !P->hang_val.upload(hv)) return GRICO_ERR_CUDA;
    P->n_hang = int64_t(hi.size());
  }
  bool ok = true;
  P->n_fixed = d->n_fixed;
  if (d->n_fixed) ok = ok && P->fixed.upload(d->fixed_dofs, size_t(d->n_fixed)) && P->fixed_vals.upload(d->fixed_values, size_t(d->n_fixed));
  P->n_rel = d->n_relations;
  if (d->n_relations) {
    ok = ok && P->rel_piv.upload(d->rel_pivot, size_t(d->n_relations)) &&
         P->rel_off.upload(d->rel_offsets, size_t(d->n_relations + 1)) &&
         P->rel_idx.upload(d->rel_index, size_t(d->rel_offsets[d->n_relations])) &&
         P->rel_coef.upload(d->rel_coef, size_t(d->rel_offsets[d->n_relations]));
    if (d->rel_rhs) {
      ok = ok && P->rel_rhs.upload(d->rel_rhs, size_t(d->n_relations));
    } else {
      ok = ok && P->rel_rhs.upload(std::vector<double>(size_t(d->n_relations), 0.0));
    }
  }
  ok = ok && P->red_off.upload(d->red_offsets, size_t(d->n_full + 1));
  if (d->red_offsets[d->n_full] > 0)
    ok = ok && P->red_idx.upload(d->red_index, size_t(d->red_offsets[d->n_full])) &&
         P->red_coef.upload(d->red_coef, size_t(d->red_offsets[d->n_full]));
  P->has_shift = false;
  if (d->red_shift)
    for (int64_t i = 0; i < d->n_full; ++i)
      if (d->red_shift[i] != 0.0) { P->has_shift = true; break; }
  if (P->has_shift) ok = ok && P->shift.upload(d->red_shift, size_t(d->n_full));
  ok = ok && P->partial.alloc(sizeof(double) * (kRedBlocks + 8)) && P->scalars.alloc(sizeof(double) * 16);
  if (!ok) return GRICO_ERR_CUDA;
  if (!cuda_ok(cudaStreamSynchronize(P->stream), "plan upload")) return GRICO_ERR_CUDA;
  if (!build_tail_all(P.get(), 0) || !build_tail_all(P.get(), 1)) return GRICO_ERR_CUDA;
  const int n_launch = int(P->batches.size() + P->pbatches.size());
  if (n_launch > 1) {
    const int nbr = std::min(n_launch, int(GricoPlan::kBranches));
    bool made = cudaEventCreateWithFlags(&P->fork_ev, cudaEventDisableTiming) == cudaSuccess;
    int k = 0;
    for (; made && k < nbr; ++k) {
      if (cudaStreamCreateWithFlags(&P->branch[k], cudaStreamNonBlocking) != cudaSuccess) { made = false; break; }
      if (cudaEventCreateWithFlags(&P->join_ev[k], cudaEventDisableTiming) != cudaSuccess) {
        cudaStreamDestroy(P->branch[k]);
        made = false;
        break;
      }
    }
    P->n_branches = k;  // streams and events made so far (destroyed with the plan)
    if (!made) {
      set_error("plan: branch streams");
      grico_plan_destroy(P.release());
      return GRICO_ERR_CUDA;
    }
  }
  *out = P.release();
  return GRICO_OK;
}

int grico_plan_destroy(GricoPlan* P) {
  if (!P) return GRICO_OK;
  cudaStreamSynchronize(P->stream);
  for (auto& ev : P->batch_events) {
    cudaEventDestroy(ev.start);
    cudaEventDestroy(ev.stop);
  }
  for (auto& sl : P->stage)
    if (sl.done) {
      cudaEventSynchronize(sl.done);
      cudaEventDestroy(sl.done);
    }
  if (P->cg_exec) cudaGraphExecDestroy(P->cg_exec);
  for (int k = 0; k < P->n_branches; ++k) {
    cudaStreamSynchronize(P->branch[k]);
    cudaStreamDestroy(P->branch[k]);
    cudaEventDestroy(P->join_ev[k]);
  }
  if (P->fork_ev) cudaEventDestroy(P->fork_ev);
  cudaStream_t st = P->stream;
  delete P;
  cudaStreamDestroy(st);
  return GRICO_OK;
}

int grico_plan_sizes(const GricoPlan* P, int64_t* n_full, int64_t* n_reduced) {
  if (!P) return GRICO_ERR_INVALID;
  if (n_full) *n_full = P->n_full;
  if (n_reduced) *n_reduced = P->n_red;
  return GRICO_OK;
}

static int apply_common(GricoPlan* P, bool reduced, const void* x, void* y, int nrhs, int precision, int flags,
                        void* stream) {
  if (!P || !x || !y || nrhs < 1) { set_error("apply: invalid argument"); return GRICO_ERR_INVALID; }
  if (x == y) { set_error("result and coefficient vector must not alias"); return GRICO_ERR_INVALID; }
  if (precision != GRICO_PREC_FP64 && precision != GRICO_PREC_FP32) { set_error("apply: unknown precision"); return GRICO_ERR_INVALID; }
  cudaStream_t st = stream ? static_cast<cudaStream_t>(stream) : P->stream;
  const int64_t n = reduced ? P->n_red : P->n_full;
  const size_t es = precision == GRICO_PREC_FP64 ? sizeof(double) : sizeof(float);
  const size_t bytes = es * size_t(n) * nrhs;
  const void* dx = x;
  void* dy = y;
  const bool async = (flags & GRICO_FLAG_HOST_POINTERS) && (flags & GRICO_FLAG_ASYNC);
  GricoPlan::Stage* slot = nullptr;
  if (async) {
    slot = &P->stage[P->stage_next];
    P->stage_next ^= 1;
    if (!slot->done && !cuda_ok(cudaEventCreateWithFlags(&slot->done, cudaEventDisableTiming), "stage event"))
      return GRICO_ERR_CUDA;
    // the slot's previous call (on any stream) must have copied its result out first
    if (slot->used && !cuda_ok(cudaStreamWaitEvent(st, slot->done, 0), "stage wait")) return GRICO_ERR_CUDA;
    if (bytes > slot->x.bytes || bytes > slot->y.bytes) {
      if (slot->used) cudaEventSynchronize(slot->done);
      if (!slot->x.ensure(bytes) || !slot->y.ensure(bytes)) return GRICO_ERR_CUDA;
    }
    if (!cuda_ok(cudaMemcpyAsync(slot->x.ptr, x, bytes, cudaMemcpyHostToDevice, st), "copy in")) return GRICO_ERR_CUDA;
    dx = slot->x.ptr;
    dy = slot->y.ptr;
  } else if (flags & GRICO_FLAG_HOST_POINTERS) {
    if (!P->host_x.ensure(bytes) || !P->host_y.ensure(bytes)) return GRICO_ERR_CUDA;
    if (!cuda_ok(cudaMemcpyAsync(P->host_x.ptr, x, bytes, cudaMemcpyHostToDevice, st), "copy in")) return GRICO_ERR_CUDA;
    dx = P->host_x.ptr;
    dy = P->host_y.ptr;
  }
  P->time_batches = (flags & GRICO_FLAG_TIME_BATCHES) != 0;
  int rc;
  if (flags & GRICO_FLAG_DETERMINISTIC)
    rc = precision == GRICO_PREC_FP64
             ? run_apply_det<double>(P, reduced, static_cast<const double*>(dx), static_cast<double*>(dy), nrhs, st)
             : run_apply_det<float>(P, reduced, static_cast<const float*>(dx), static_cast<float*>(dy), nrhs, st);
  else
    rc = precision == GRICO_PREC_FP64
             ? run_apply<double>(P, reduced, static_cast<const double*>(dx), static_cast<double*>(dy), nrhs, st)
             : run_apply<float>(P, reduced, static_cast<const float*>(dx), static_cast<float*>(dy), nrhs, st);
  P->time_batches = false;
  if (rc != GRICO_OK) return rc;
  if (flags & GRICO_FLAG_HOST_POINTERS) {
    if (!cuda_ok(cudaMemcpyAsync(y, dy, bytes, cudaMemcpyDeviceToHost, st), "copy out")) return GRICO_ERR_CUDA;
    if (async) {
      slot->used = true;
      return cuda_ok(cudaEventRecord(slot->done, st), "stage event") ? GRICO_OK : GRICO_ERR_CUDA;
    }
    if (!cuda_ok(cudaStreamSynchronize(st), "apply")) return GRICO_ERR_CUDA;
  }
  return GRICO_OK;
}

int grico_plan_set_mass_points(GricoPlan* P, const double* const* mass_points, int flags) {
  if (!P) { set_error("grico_plan_set_mass_points: invalid argument"); return GRICO_ERR_INVALID; }
  if (mass_points && !P->pbatches.empty()) {
    set_error("grico_plan_set_mass_points: plans with point-quadrature items are not supported");
    return GRICO_ERR_UNSUPPORTED_FORM;
  }
  const cudaMemcpyKind kind = (flags & GRICO_FLAG_HOST_POINTERS) ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice;
  ++P->epoch;  // kernel arguments baked into a kept solver graph change
  for (size_t bi = 0; bi < P->batches.size(); ++bi) {
    DevBatch& b = P->batches[bi];
    if (!mass_points || !mass_points[bi]) {
      b.mass_pts.alloc(0);
      continue;
    }
    const size_t n = size_t(b.n_cells) * size_t(b.q[0]) * size_t(P->dim > 1 ? b.q[1] : 1) *
                     size_t(P->dim > 2 ? b.q[2] : 1);
    if (!b.mass_pts.ensure(sizeof(double) * n)) return GRICO_ERR_CUDA;
    if (n && !cuda_ok(cudaMemcpyAsync(b.mass_pts.ptr, mass_points[bi], sizeof(double) * n, kind, P->stream),
                      "mass points"))
      return GRICO_ERR_CUDA;
  }
  return cuda_ok(cudaStreamSynchronize(P->stream), "mass points") ? GRICO_OK : GRICO_ERR_CUDA;
}

int grico_eval_points(GricoPlan* P, const double* u, int reduced, double* const* values, int flags) {
  if (!P || !u || !values) { set_error("grico_eval_points: invalid argument"); return GRICO_ERR_INVALID; }
  cudaStream_t st = P->stream;
  const int64_t n = reduced ? P->n_red : P->n_full;
  const bool host = (flags & GRICO_FLAG_HOST_POINTERS) != 0;
  const double* du = u;
  DevBuf ub, vb;
  if (host) {
    if (!ub.alloc(sizeof(double) * std::max<int64_t>(n, 1))) return GRICO_ERR_CUDA;
    cudaMemcpyAsync(ub.ptr, u, sizeof(double) * n, cudaMemcpyHostToDevice, st);
    du = ub.get<double>();
  }
  for (size_t bi = 0; bi < P->batches.size(); ++bi) {
    if (!values[bi]) continue;
    const DevBatch& b = P->batches[bi];
    int nn[3] = {1, 1, 1}, q[3] = {1, 1, 1};
    for (int a = 0; a < P->dim; ++a) { nn[a] = b.n[a]; q[a] = b.q[a]; }
    const size_t nq = size_t(q[0]) * q[1] * q[2], count = size_t(b.n_cells) * nq;
    double* out = values[bi];
    if (host) {
      if (!vb.ensure(sizeof(double) * std::max<size_t>(count, 1))) return GRICO_ERR_CUDA;
      out = vb.get<double>();
    }
    if (b.n_cells > 0) {
      BatchView v;
      fill_view(v, b, reduced != 0);
      const size_t smem = sizeof(double) * (size_t(nn[0]) * nn[1] * nn[2] + (P->dim + 1) * nq);
      if (smem > 48 * 1024)
        cudaFuncSetAttribute(cell_apply_generic<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
      cell_apply_generic<double><<<dim3(b.n_cells, 1), 128, smem, st>>>(v, P->dim, nn[0], nn[1], nn[2], q[0], q[1],
                                                                        q[2], du, out, 0, 0.0, 0.0, 4, nullptr);
    }
    if (host && count &&
        !cuda_ok(cudaMemcpyAsync(values[bi], out, sizeof(double) * count, cudaMemcpyDeviceToHost, st), "values"))
      return GRICO_ERR_CUDA;
    if (host && !cuda_ok(cudaStreamSynchronize(st), "eval points")) return GRICO_ERR_CUDA;
  }
  return cuda_ok(cudaStreamSynchronize(st), "eval points") ? GRICO_OK : GRICO_ERR_CUDA;
}

int grico_plan_batch_times(GricoPlan* P, double* ms, int64_t* launches, int n_batches) {
  const size_t nb = P ? P->batches.size() + P->pbatches.size() : 0;
  if (!P || !ms || n_batches < 0 || size_t(n_batches) > nb) {
    set_error("grico_plan_batch_times: invalid argument");
    return GRICO_ERR_INVALID;
  }
  std::vector<double> total(nb, 0.0);
  std::vector<int64_t> count(nb, 0);
  int rc = GRICO_OK;
  for (auto& ev : P->batch_events) {
    float t = 0.0f;
    if (rc == GRICO_OK && cuda_ok(cudaEventSynchronize(ev.stop), "batch timing") &&
        cuda_ok(cudaEventElapsedTime(&t, ev.start, ev.stop), "batch timing")) {
      total[size_t(ev.batch)] += t;
      count[size_t(ev.batch)] += 1;
    } else {
      rc = GRICO_ERR_CUDA;
    }
    cudaEventDestroy(ev.start);
    cudaEventDestroy(ev.stop);
  }
  P->batch_events.clear();
  for (int i = 0; i < n_batches; ++i) {
    ms[i] = count[size_t(i)] ? total[size_t(i)] / double(count[size_t(i)]) : 0.0;
    if (launches) launches[i] = count[size_t(i)];
  }
  return rc;
}

int grico_apply(GricoPlan* P, const void* x, void* y, int nrhs, int precision, int flags, void* stream) {
  return apply_common(P, false, x, y, nrhs, precision, flags, stream);
}

int grico_reduced_apply(GricoPlan* P, const void* x, void* y, int nrhs, int precision, int flags, void* stream) {
  return apply_common(P, true, x, y, nrhs, precision, flags, stream);
}

}  // extern "C"

namespace {

// The load vector sum_cells P_c^T (w f) on the full layout into `full` (zeroed first), from the
// per-batch source values at the quadrature points (host arrays with GRICO_FLAG_HOST_POINTERS).
int assemble_load(GricoPlan* P, const double* const* source_points, int flags, double* full, cudaStream_t st) {
  DevBuf src;
  cudaMemsetAsync(full, 0, sizeof(double) * P->n_full, st);
  for (size_t bi = 0; bi < P->batches.size(); ++bi) {
    const DevBatch& b = P->batches[bi];
    const double* sp = nullptr;
    if (source_points && source_points[bi]) {
      int64_t nq = 1;
      for (int a = 0; a < P->dim; ++a) nq *= b.q[a];
      if (flags & GRICO_FLAG_HOST_POINTERS) {
        if (!src.alloc(sizeof(double) * nq * b.n_cells)) return GRICO_ERR_CUDA;
        cudaMemcpyAsync(src.ptr, source_points[bi], sizeof(double) * nq * b.n_cells, cudaMemcpyHostToDevice, st);
        sp = src.get<double>();
      } else {
        sp = source_points[bi];
      }
    }
    launch_batch<double>(*P, b, false, nullptr, full, P->n_full, 1, sp, 1, st);
    if (flags & GRICO_FLAG_HOST_POINTERS) cudaStreamSynchronize(st);
  }
  for (size_t bi = 0; bi < P->pbatches.size(); ++bi) {
    const DevPointBatch& pb = P->pbatches[bi];
    const size_t slot = P->batches.size() + bi;
    const double* sp = nullptr;
    if (source_points && source_points[slot] && pb.n_points > 0) {
      if (flags & GRICO_FLAG_HOST_POINTERS) {
        if (!src.alloc(sizeof(double) * pb.n_points)) return GRICO_ERR_CUDA;
        cudaMemcpyAsync(src.ptr, source_points[slot], sizeof(double) * pb.n_points, cudaMemcpyHostToDevice, st);
        sp = src.get<double>();
      } else {
        sp = source_points[slot];
      }
    }
    launch_points<double>(*P, pb, false, nullptr, full, P->n_full, 1, sp, 1, st);
    if (flags & GRICO_FLAG_HOST_POINTERS) cudaStreamSynchronize(st);
  }
  return cuda_ok(cudaGetLastError(), "load assembly") ? GRICO_OK : GRICO_ERR_CUDA;
}

}  // namespace

extern "C" {

// rhs! (assembly.jl:488-507): the load vector on the full layout with the rows of fixed dofs and
// Dirichlet relation pivots replaced by their constraint right-hand sides (_write_constraint_rhs!,
// assembly.jl:1876-1891).
int grico_rhs(GricoPlan* P, const double* const* source_points, double* b_full, int flags) {
  if (!P || !b_full) { set_error("grico_rhs: invalid argument"); return GRICO_ERR_INVALID; }
  (void)cudaGetLastError();
  cudaStream_t st = P->stream;
  DevBuf tmp;
  double* out = b_full;
  if (flags & GRICO_FLAG_HOST_POINTERS) {
    if (!tmp.alloc(sizeof(double) * std::max<int64_t>(P->n_full, 1))) return GRICO_ERR_CUDA;
    out = tmp.get<double>();
  }
  if (int rc = assemble_load(P, source_points, flags, out, st)) return rc;
  if (P->n_fixed + P->n_rel > 0)
    constraint_rhs<<<grid_for(P->n_fixed + P->n_rel), 256, 0, st>>>(
        P->fixed.get<int64_t>(), P->fixed_vals.get<double>(), P->n_fixed, P->rel_piv.get<int64_t>(),
        P->rel_rhs.get<double>(), P->n_rel, out);
  if (flags & GRICO_FLAG_HOST_POINTERS)
    cudaMemcpyAsync(b_full, out, sizeof(double) * P->n_full, cudaMemcpyDeviceToHost, st);
  return cuda_ok(cudaStreamSynchronize(st), "rhs") ? GRICO_OK : GRICO_ERR_CUDA;
}

int grico_reduced_rhs(GricoPlan* P, const double* const* source_points, double* b_reduced, int flags) {
  if (!P || !b_reduced) return GRICO_ERR_INVALID;
  (void)cudaGetLastError();
  cudaStream_t st = P->stream;
  DevBuf full, bred;
  if (!full.alloc(sizeof(double) * std::max<int64_t>(P->n_full, 1))) return GRICO_ERR_CUDA;
  if (int rc = assemble_load(P, source_points, flags, full.get<double>(), st)) return rc;
  if (P->has_shift) {
    DevBuf as;
    if (!as.alloc(sizeof(double) * P->n_full)) return GRICO_ERR_CUDA;
    cudaMemsetAsync(as.ptr, 0, sizeof(double) * P->n_full, st);
    for (auto& b : P->batches)
      launch_batch<double>(*P, b, false, P->shift.get<double>(), as.get<double>(), P->n_full, 0, nullptr, 1, st);
    for (auto& pb : P->pbatches)
      launch_points<double>(*P, pb, false, P->shift.get<double>(), as.get<double>(), P->n_full, 0, nullptr, 1, st);
    axpby_kernel<double><<<grid_for(P->n_full), 256, 0, st>>>(-1.0, as.get<double>(), 1.0, full.get<double>(), P->n_full);
    cudaStreamSynchronize(st);
  }
  double* out = b_reduced;
  if (flags & GRICO_FLAG_HOST_POINTERS) {
    if (!bred.alloc(sizeof(double) * std::max<int64_t>(P->n_red, 1))) return GRICO_ERR_CUDA;
    out = bred.get<double>();
  }
  cudaMemsetAsync(out, 0, sizeof(double) * P->n_red, st);
  project_reduced<<<grid_for(P->n_full), 256, 0, st>>>(P->red_off.get<int64_t>(), P->red_idx.get<int64_t>(),
                                                        P->red_coef.get<double>(), full.get<double>(), out, P->n_full);
  if (flags & GRICO_FLAG_HOST_POINTERS)
    cudaMemcpyAsync(b_reduced, out, sizeof(double) * P->n_red, cudaMemcpyDeviceToHost, st);
  return cuda_ok(cudaStreamSynchronize(st), "reduced rhs") ? GRICO_OK : GRICO_ERR_CUDA;
}

int grico_reduced_diagonal(GricoPlan* P, double* diag, int flags) {
  if (!P || !diag) return GRICO_ERR_INVALID;
  cudaStream_t st = P->stream;
  DevBuf tmp;
  double* out = diag;
  if (flags & GRICO_FLAG_HOST_POINTERS) {
    if (!tmp.alloc(sizeof(double) * std::max<int64_t>(P->n_red, 1))) return GRICO_ERR_CUDA;
    out = tmp.get<double>();
  }
  int rc = reduced_diag_device(P, out, st);
  if (rc) return rc;
  if (flags & GRICO_FLAG_HOST_POINTERS) cudaMemcpyAsync(diag, out, sizeof(double) * P->n_red, cudaMemcpyDeviceToHost, st);
  return cuda_ok(cudaStreamSynchronize(st), "diagonal") ? GRICO_OK : GRICO_ERR_CUDA;
}

int grico_expand_reduced(GricoPlan* P, const double* u_red, double* u_full, int flags) {
  if (!P || !u_red || !u_full) return GRICO_ERR_INVALID;
  cudaStream_t st = P->stream;
  DevBuf a, b;
  const double* in = u_red;
  double* out = u_full;
  if (flags & GRICO_FLAG_HOST_POINTERS) {
    if (!a.alloc(sizeof(double) * std::max<int64_t>(P->n_red, 1)) || !b.alloc(sizeof(double) * std::max<int64_t>(P->n_full, 1)))
      return GRICO_ERR_CUDA;
    cudaMemcpyAsync(a.ptr, u_red, sizeof(double) * P->n_red, cudaMemcpyHostToDevice, st);
    in = a.get<double>();
    out = b.get<double>();
  }
  expand_reduced<<<grid_for(P->n_full), 256, 0, st>>>(P->red_off.get<int64_t>(), P->red_idx.get<int64_t>(),
                                                       P->red_coef.get<double>(),
                                                       P->has_shift ? P->shift.get<double>() : nullptr, in, out,
                                                       P->n_full);
  if (flags & GRICO_FLAG_HOST_POINTERS) cudaMemcpyAsync(u_full, out, sizeof(double) * P->n_full, cudaMemcpyDeviceToHost, st);
  return cuda_ok(cudaStreamSynchronize(st), "expand") ? GRICO_OK : GRICO_ERR_CUDA;
}

}  // extern "C"

// ---------------------------------------------------------------------------------------------
// Allocation-free variant of the reduced right-hand side.
//
// Some callers cannot call cudaMalloc: code that runs while a CUDA stream is being captured into
// a graph, host callbacks, and services whose GPU memory is budgeted up front (a memory pool or
// a fixed partition) all need an entry point that touches no allocator.  grico_reduced_rhs()
// allocates two full-layout temporaries per call; grico_reduced_rhs_static() keeps them in the
// file-scope array below instead.  Every GPU that loads the library holds this array
// (2 * GRICO_STATIC_RHS_MAX_DOFS doubles = 16 MiB) until the process exits.
#define GRICO_STATIC_RHS_MAX_DOFS (1 << 20)
static __device__ __align__(256) double g_rhs_scratch[2 * GRICO_STATIC_RHS_MAX_DOFS];

namespace {

// Device address of g_rhs_scratch per device.  In host code the symbol is only a host-side
// stand-in; the address a kernel may use comes from cudaGetSymbolAddress with the device
// current.  Resolved on the first call on each device.
std::mutex g_rhs_scratch_mutex;
double* g_rhs_scratch_ptr[64] = {nullptr};

int static_rhs_scratch(double** out) {
  int dev = 0;
  if (!cuda_ok(cudaGetDevice(&dev), "cudaGetDevice")) return GRICO_ERR_CUDA;
  if (dev < 0 || dev >= 64) { set_error("device index out of range"); return GRICO_ERR_INVALID; }
  std::lock_guard<std::mutex> lock(g_rhs_scratch_mutex);
  if (!g_rhs_scratch_ptr[dev]) {
    void* p = nullptr;
    if (!cuda_ok(cudaGetSymbolAddress(&p, g_rhs_scratch), "cudaGetSymbolAddress")) return GRICO_ERR_CUDA;
    g_rhs_scratch_ptr[dev] = static_cast<double*>(p);
  }
  *out = g_rhs_scratch_ptr[dev];
  return GRICO_OK;
}

}  // namespace

extern "C" int grico_reduced_rhs_static(GricoPlan* P, const double* const* source_points, double* b_reduced,
                                        void* stream) {
  if (!P || !b_reduced) { set_error("grico_reduced_rhs_static: invalid argument"); return GRICO_ERR_INVALID; }
  if (P->n_full > GRICO_STATIC_RHS_MAX_DOFS) {
    set_error("grico_reduced_rhs_static: the plan has " + std::to_string(P->n_full) +
              " full-layout dofs; the static scratch holds at most " + std::to_string(GRICO_STATIC_RHS_MAX_DOFS));
    return GRICO_ERR_INVALID;
  }
  // a launch error left pending by an earlier, unrelated call would otherwise be reported below
  (void)cudaGetLastError();
  double* scratch = nullptr;
  if (int rc = static_rhs_scratch(&scratch)) return rc;
  cudaStream_t st = stream ? static_cast<cudaStream_t>(stream) : P->stream;
  double* full = scratch;
  double* shifted = scratch + GRICO_STATIC_RHS_MAX_DOFS;
  // the scratch keeps the previous call's contents: clear the accumulation targets
  cudaMemsetAsync(full, 0, sizeof(double) * P->n_full, st);
  for (size_t bi = 0; bi < P->batches.size(); ++bi)
    launch_batch<double>(*P, P->batches[bi], false, nullptr, full, P->n_full, 1,
                         source_points ? source_points[bi] : nullptr, 1, st);
  for (size_t bi = 0; bi < P->pbatches.size(); ++bi)
    launch_points<double>(*P, P->pbatches[bi], false, nullptr, full, P->n_full, 1,
                          source_points ? source_points[P->batches.size() + bi] : nullptr, 1, st);
  if (P->has_shift) {
    cudaMemsetAsync(shifted, 0, sizeof(double) * P->n_full, st);
    for (auto& b : P->batches)
      launch_batch<double>(*P, b, false, P->shift.get<double>(), shifted, P->n_full, 0, nullptr, 1, st);
    for (auto& pb : P->pbatches)
      launch_points<double>(*P, pb, false, P->shift.get<double>(), shifted, P->n_full, 0, nullptr, 1, st);
    axpby_kernel<double><<<grid_for(P->n_full), 256, 0, st>>>(-1.0, shifted, 1.0, full, P->n_full);
  }
  cudaMemsetAsync(b_reduced, 0, sizeof(double) * P->n_red, st);
  project_reduced<<<grid_for(P->n_full), 256, 0, st>>>(P->red_off.get<int64_t>(), P->red_idx.get<int64_t>(),
                                                        P->red_coef.get<double>(), full, b_reduced, P->n_full);
  return cuda_ok(cudaGetLastError(), "grico_reduced_rhs_static") ? GRICO_OK : GRICO_ERR_CUDA;
}

namespace {

template <typename T>
int autotune_typed(GricoPlan* P, int nrhs, int reps, int* chosen) {
  cudaStream_t st = P->stream;
  const int64_t n = P->n_red;
  DevBuf xb, yb;
  if (!xb.alloc(sizeof(T) * std::max<int64_t>(n, 1) * nrhs) || !yb.alloc(sizeof(T) * std::max<int64_t>(n, 1) * nrhs))
    return GRICO_ERR_CUDA;
  fill_kernel<T><<<grid_for(n * nrhs), 256, 0, st>>>(xb.get<T>(), n * nrhs, T(1));
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  const int slot = sizeof(T) == 4 ? 1 : 0;
  for (size_t bi = 0; bi < P->batches.size(); ++bi) {
    DevBatch& b = P->batches[bi];
    int best = 1;
    if (P->dim == 3 && b.isotropic && b.q[0] >= b.n[0] && b.n_cells > 0) {
      float best_ms = 1e30f;
      for (int var = 0; var < kTileVariants; ++var) {
        b.tile[slot] = var;
        launch_batch<T>(*P, b, true, xb.get<T>(), yb.get<T>(), n, 0, nullptr, nrhs, st);  // warm-up
        cudaEventRecord(e0, st);
        for (int r = 0; r < reps; ++r) launch_batch<T>(*P, b, true, xb.get<T>(), yb.get<T>(), n, 0, nullptr, nrhs, st);
        cudaEventRecord(e1, st);
        cudaEventSynchronize(e1);
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, e0, e1);
        if (ms < best_ms) { best_ms = ms; best = var; }
      }
    }
    b.tile[slot] = best;
    if (chosen) chosen[bi] = best;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return cuda_ok(cudaStreamSynchronize(st), "autotune") ? GRICO_OK : GRICO_ERR_CUDA;
}

}  // namespace

extern "C" int grico_plan_autotune(GricoPlan* P, int nrhs, int precision, int reps, int* chosen) {
  if (!P || nrhs < 1 || reps < 1 || (precision != GRICO_PREC_FP64 && precision != GRICO_PREC_FP32)) {
    set_error("grico_plan_autotune: invalid argument");
    return GRICO_ERR_INVALID;
  }
  ++P->epoch;
  return precision == GRICO_PREC_FP64 ? autotune_typed<double>(P, nrhs, reps, chosen)
                                      : autotune_typed<float>(P, nrhs, reps, chosen);
}

extern "C" int grico_plan_set_tiles(GricoPlan* P, int precision, const int* tiles, int n_batches) {
  if (!P || !tiles || (precision != GRICO_PREC_FP64 && precision != GRICO_PREC_FP32) ||
      n_batches != int(P->batches.size())) {
    set_error("grico_plan_set_tiles: invalid argument (tiles must hold one entry per cell batch)");
    return GRICO_ERR_INVALID;
  }
  for (int i = 0; i < n_batches; ++i)
    if (tiles[i] < 0 || tiles[i] >= kTileVariants) {
      set_error("grico_plan_set_tiles: tile variant out of range");
      return GRICO_ERR_INVALID;
    }
  const int slot = precision == GRICO_PREC_FP32 ? 1 : 0;
  for (int i = 0; i < n_batches; ++i) P->batches[size_t(i)].tile[slot] = tiles[i];
  ++P->epoch;  // kernels baked into a kept solver graph change
  return GRICO_OK;
}
