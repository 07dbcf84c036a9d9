// Internal layout of a device plan (HBM-resident data of one AssemblyPlan).
//
// Per cell batch (cells with one kernel signature):
//   map      int32 [n_cells * n_box]   local box mode -> dof (>=0), inactive (-1), tail (<= -2)
//   coef     f64   [n_cells * n_box]   only when some coefficient differs from 1
//   tail     CSR of multi-term (hanging-node) expansions
//   h        f64   [n_cells * dim]     cell sizes (affine axis-aligned geometry)
//   kappa    f64   [n_cells * q^dim]   optional pointwise coefficient
//   B,G,W,D  1-D tables: basis values, reference derivatives, Gauss weights, collocation
//            derivative matrix
// Two maps per batch: full layout (apply!) and reduced layout (composition with P).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <map>
#include <vector>

#include "../../include/grico_b200.h"

namespace grico {

bool cuda_ok(cudaError_t e, const char* what);

struct DevBuf {
  void* ptr = nullptr;
  size_t bytes = 0;
  DevBuf() = default;
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  DevBuf(DevBuf&& o) noexcept : ptr(o.ptr), bytes(o.bytes) { o.ptr = nullptr; o.bytes = 0; }
  DevBuf& operator=(DevBuf&& o) noexcept {
    if (this != &o) {
      if (ptr) cudaFree(ptr);
      ptr = o.ptr;
      bytes = o.bytes;
      o.ptr = nullptr;
      o.bytes = 0;
    }
    return *this;
  }
  ~DevBuf();
  template <typename T>
  T* get() const { return static_cast<T*>(ptr); }
  bool alloc(size_t n) {
    if (ptr) { cudaFree(ptr); ptr = nullptr; }
    bytes = n;
    if (n == 0) return true;
    return cuda_ok(cudaMalloc(&ptr, n), "cudaMalloc");
  }
  bool ensure(size_t n) { return n <= bytes && ptr ? true : alloc(n); }
  template <typename T>
  bool upload(const T* src, size_t count) {
    if (!alloc(sizeof(T) * count)) return false;
    if (count == 0) return true;
    return cuda_ok(cudaMemcpy(ptr, src, sizeof(T) * count, cudaMemcpyHostToDevice), "upload");
  }
  template <typename T>
  bool upload(const std::vector<T>& v) { return upload(v.data(), v.size()); }
};

constexpr int kTileVariants = 11;

struct DevMap {
  DevBuf map, coef, toff, tidx, tcoef;
  // buffered tails (operator apply with long hanging-node expansions): the number of tails
  // (0: the cell kernels walk the expansions themselves) and their per-right-hand-side sums
  int64_t n_tail = 0;
  DevBuf tx, ty;
  // the tails cut into segments of at most kTailSeg terms: tail index and first term
  int64_t n_seg = 0;
  DevBuf seg_k, seg_t;
};
// tile variant of the FP32 tensor-core apply of uniform batches
constexpr int kDenseVariant = 10;
// error flag of the tensor-core kernels on the current device (a bounded wait that gave up);
// defined with the convolutions in csrc/grico_cnn.cu
int tc_error_flag(int** out);
// right-hand sides the tail buffers hold; more fall back to the unbuffered walk
constexpr int kTailRhs = 32;
// right-hand sides from which the tail kernels put the columns on the lanes of a warp
constexpr int kTailLaneRhs = 8;
// buffer the tails of a map whose longest expansion has at least this many terms
constexpr int64_t kTailBufferMin = 8;

struct DevBatch {
  int32_t n_cells = 0;
  int n[3] = {1, 1, 1};
  int q[3] = {1, 1, 1};
  bool isotropic = true;
  bool red_multiterm = false;
  DevMap full, red;
  DevBuf h, kappa, B, G, W, D;
  DevBuf skip;  // uint8 per cell: hanging cells whose diagonal is added from the host
  DevBuf mass_pts;  // optional pointwise mass [n_cells * nq] added to the form's mass (grico_plan_set_mass_points)
  std::vector<double> hB, hD, hW;  // axis-0 tables on the host (kernel parameters)
  // uniform batch (3-D, one cell size, constant coefficients, degree <= 4): the element matrix
  // as BF16 hi/lo pieces for the FP32 tensor-core apply (csrc/cell_dense_tc.cuh)
  bool dense_ok = false;
  DevBuf dense;
  int tile[2] = {1, 1};  // 3-D tensor-kernel variant per precision (0: FP64, 1: FP32): cells per block
                         // half (0), default (1) or double (2) the default, one block per cell group;
                         // 3..5 the same sizes in the persistent cp.async-pipelined apply kernel
                         // with even-odd contractions, 6..8 that kernel with direct contractions;
                         // chosen by grico_plan_autotune or set by grico_plan_set_tiles
};

struct DevPointBatch {
  int32_t n_items = 0;
  int kind = 1;
  int n[3] = {1, 1, 1};
  int64_t n_points = 0;  // points (kind 3: subcells x prod(q), the size of source/kappa arrays)
  DevMap full, red;
  DevBuf h, pt_off, ref, w, nrm, eta, kpts, skip;
  // GRICO_ITEM_SUBCELLS
  int q[3] = {1, 1, 1};
  int64_t n_sub = 0;
  DevBuf sub_off, sub_level, sub_pos, sub_mask, sub_w;
  std::vector<double> hEta, hW, hDm;  // Gauss points, weights, collocation derivative (q[0])
  // GRICO_ITEM_INTERFACE: plus-side modes per axis, reference points, cell sizes, normal axis
  int np[3] = {1, 1, 1};
  DevBuf ref_p, h_p, axis;
  // sum-factorised interfaces (interface_apply_sf): every item's points form a tangential tensor
  // grid; (q1, q2) per item and the 1-D coordinates [side][t1 | t2 | normal] with a fixed stride
  bool sf_ok = false;
  int sf_stride = 0, sf_qmax = 1;
  int64_t sf_pmax = 1;
  DevBuf sf_q, sf_x;
};

}  // namespace grico

struct GricoPlan {
  int dim = 0;
  double mass = 0, kappa = 1;
  int64_t n_full = 0, n_red = 0;
  cudaStream_t stream = nullptr;
  std::vector<grico::DevBatch> batches;
  std::vector<grico::DevPointBatch> pbatches;
  int64_t n_fixed = 0, n_rel = 0;
  grico::DevBuf fixed, fixed_vals, rel_piv, rel_off, rel_idx, rel_coef, rel_rhs;
  grico::DevBuf red_off, red_idx, red_coef, shift;
  bool has_shift = false;
  std::map<int64_t, double> hang_diag;  // exact diagonal contributions of hanging cells
  grico::DevBuf hang_idx, hang_val;
  int64_t n_hang = 0;
  grico::DevBuf partial, scalars;
  grico::DevBuf host_x, host_y;
  // GRICO_FLAG_ASYNC staging ring: device copies of x and y per slot, and the event that marks
  // the end of the slot's last copy out
  struct Stage { grico::DevBuf x, y; cudaEvent_t done = nullptr; bool used = false; };
  Stage stage[2];
  int stage_next = 0;
  // GRICO_FLAG_DETERMINISTIC: per layout (0 full, 1 reduced) the gather CSR of the stored local
  // results (row = dof; its terms in batch, entry, expansion-term order) and the first entry of
  // every cell and point batch; built on the first deterministic apply of that layout
  struct DetMap {
    bool built = false;
    int64_t entries = 0;
    std::vector<int64_t> cell_base, point_base;
    grico::DevBuf off, pos, coef;
  };
  DetMap det[2];
  grico::DevBuf det_local;
  // The buffered tails of every cell batch of one layout (0 full, 1 reduced) in one numbering,
  // so that an apply sums and spreads all of them in one launch each: batch b's tails are
  // base[b] .. base[b] + its n_tail; buffers [rhs][n_tail] (kTailRhs columns)
  struct TailAll {
    int64_t n_tail = 0, n_seg = 0;
    std::vector<int64_t> base;  // per cell batch; -1: not buffered
    grico::DevBuf toff, tidx, tcoef, seg_k, seg_t, tx, ty;
  };
  TailAll tails[2];
  // GRICO_FLAG_TIME_BATCHES: event pairs around cell-batch launches, (batch, start, stop)
  struct BatchEvent { int batch; cudaEvent_t start, stop; };
  bool time_batches = false;
  std::vector<BatchEvent> batch_events;
  std::vector<double> batch_ms;
  std::vector<int64_t> batch_launches;
  // CG iteration graph kept across solves; replayed while its key (multigrid identity,
  // preconditioner, solution buffer, plan epoch) matches.  The epoch changes whenever kernel
  // choices or per-point data baked into launches change.
  cudaGraphExec_t cg_exec = nullptr;
  uint64_t cg_key_mg = 0, cg_key_epoch = 0;
  int cg_key_pc = -1;
  const void* cg_key_x = nullptr;
  uint64_t epoch = 1;
  // The cell and point batches of one apply run concurrently on these streams, forked from and
  // joined back to the launching stream (the scatter is atomic, so their order is free); made
  // when the plan has more than one batch; eight, so that each batch of an hp mesh (up to
  // eight degrees) with its tail passes forms its own chain
  // work buffers of the lockstep solver (grico_cg_solve_multi), kept across calls and grown on
  // demand; calls on one plan share them, as they share its tail buffers and streams
  static constexpr int kSolverWs = 20;
  grico::DevBuf solver_ws[kSolverWs];
  static constexpr int kBranches = 8;
  int n_branches = 0;
  cudaStream_t branch[kBranches] = {};
  cudaEvent_t fork_ev = nullptr, join_ev[kBranches] = {};
  // Krylov workspaces (allocated on first solve)
  grico::DevBuf w_r, w_z, w_p, w_q, w_x, w_b, w_dinv;
};

namespace grico {
// y_zero: y already holds zeros (the caller cleared it in its last pass over it), so the apply
// skips zeroing it
template <typename T>
int run_apply(GricoPlan* P, bool reduced, const T* x, T* y, int nrhs, cudaStream_t st, bool y_zero = false);
int reduced_diag_device(GricoPlan* P, double* diag, cudaStream_t st);
int grid_blocks(int64_t n);
}  // namespace grico
