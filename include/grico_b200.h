/*
 * grico_b200.h — C ABI of the B200 matrix-free runtime for Grico.jl's hot path.
 *
 * Every entry point is plain C: pointers, sizes and POD structs, no C++ or torch types.
 * Indices are 0-based (the reference is 1-based; the binding subtracts 1).  Return codes
 * are GRICO_OK (0) or a negative GRICO_ERR_*; grico_last_error() gives a thread-local
 * message.  No exception crosses the boundary.
 *
 * Reference interfaces each group replaces (paths inside schmaeke/Grico.jl):
 *   host space compile   src/space.jl:300-326, src/continuity.jl:153-1227,
 *                        src/topology.jl:232-300, 1502-1545 (Morton order, faces)
 *   plan create/destroy  compile(problem)            src/plans.jl:170-231
 *   apply                apply!(result, plan, x, ws) src/assembly.jl:540-564
 *   reduced apply        _reduced_apply!             src/assembly.jl:905-915
 *   rhs                  rhs!, _reduced_rhs!         src/assembly.jl:456-507, 917-933
 *   diagonal             _reduced_diagonal!          src/assembly.jl:662-675
 *   cg solve             _cg_solve                   src/solve.jl:376-431
 *   fgmres solve         _fgmres_solve               src/solve.jl:433-589
 *   multigrid            _vcycle!, transfers         src/multigrid.jl:858-1087
 */
#ifndef GRICO_B200_H
#define GRICO_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes (reference raises ArgumentError for every one of these) ---- */
#define GRICO_OK 0
#define GRICO_ERR_INVALID -1          /* bad argument, size mismatch, aliasing          */
#define GRICO_ERR_UNSUPPORTED_FORM -2 /* accumulator form the GPU plan does not know   */
#define GRICO_ERR_NOT_CONVERGED -3    /* Krylov did not reach tolerance in maxiter      */
#define GRICO_ERR_NONFINITE -4        /* NaN/Inf in input, diagonal or residual         */
#define GRICO_ERR_BREAKDOWN -5        /* non-positive CG direction (solve.jl:414-416)   */
#define GRICO_ERR_CUDA -6             /* CUDA runtime error                             */
#define GRICO_ERR_NO_DEVICE -7        /* no CUDA device (the library never falls back)  */
#define GRICO_ERR_TIMEOUT -8          /* bounded device wait gave up                    */

#define GRICO_BASIS_FULL 0  /* FullTensorBasis  basis.jl:60-95  */
#define GRICO_BASIS_TRUNK 1 /* TrunkBasis       basis.jl:97-126 */
#define GRICO_CONTINUITY_CG 0
#define GRICO_CONTINUITY_DG 1

/* Closed set of cell forms.  TestChannels(a0, a_grad) means ∫ a0 v + a_grad·∇v
 * (accumulators.jl:148-160).  GRICO_FORM_MASS_DIFFUSION: a0 = mass*u, a_grad = kappa*k(x)*∇u
 * with k(x) = 1 or tabulated per quadrature point.  Anything else is rejected with
 * GRICO_ERR_UNSUPPORTED_FORM. */
#define GRICO_FORM_MASS_DIFFUSION 1

#define GRICO_PREC_FP64 0 /* vectors double, arithmetic double                      */
#define GRICO_PREC_FP32 1 /* vectors float, arithmetic float (mixed-precision path) */

#define GRICO_FLAG_HOST_POINTERS 1 /* vector arguments are host memory: copy in/out */
#define GRICO_FLAG_NO_GRAPH 2      /* Krylov solves: launch each iteration op by op, no CUDA graph */
#define GRICO_FLAG_MIXED 4         /* grico_cg_solve_multi: FP64 refinement around FP32 inner CG */
#define GRICO_FLAG_TIME_BATCHES 8  /* grico_apply / grico_reduced_apply: record CUDA events around
                                      every cell-batch kernel launch (grico_plan_batch_times)   */
#define GRICO_FLAG_ASYNC 16        /* grico_apply / grico_reduced_apply with host pointers: enqueue
                                      the copy in, the kernels and the copy out on `stream` and
                                      return; the caller synchronises the stream before reading y
                                      or changing x.  Two calls may be in flight per plan (two
                                      staging slots; a third waits for the first on the device) */
#define GRICO_FLAG_DETERMINISTIC 32 /* grico_apply / grico_reduced_apply: no atomic scatter; every
                                      cell and point kernel stores its local results and one pass
                                      sums each dof's terms in a fixed (batch, entry, term) order,
                                      so results are bitwise reproducible run to run, as the
                                      reference's sum is thread-count independent.  Slower; the
                                      first call per layout builds the gather table (allocates) */

/* ================================================================================
 * Host space compile (native replacement of the Julia-side HpSpace construction)
 * ================================================================================ */
typedef struct GricoSpace GricoSpace;

/* Build an hp space from active leaves given as (levels, logical coords) per axis,
 * leaf-major [nleaves*dim].  Leaves are reordered into the reference's Morton order.
 * Replaces HpSpace(domain, SpaceOptions(...)) — space.jl:300-326, continuity.jl:153-1227. */
int grico_space_build(int dim, const int64_t* root_counts, int64_t nleaves, const int32_t* leaf_levels,
                      const int64_t* leaf_coords, const int32_t* leaf_degrees, int basis, int continuity,
                      int quadrature_extra, GricoSpace** out);
int grico_space_destroy(GricoSpace* space);
/* Sizes: scalar dofs, total terms, total box modes (sum over leaves of prod(p+1)),
 * boundary faces, interfaces (topology.jl:1502-1545). */
int grico_space_sizes(const GricoSpace* space, int64_t* ndofs, int64_t* nterms, int64_t* nboxes,
                      int64_t* nboundary, int64_t* ninterfaces);
/* Copy out: Morton order (position -> input leaf), per-leaf box offsets [nleaves+1], term CSR
 * over box modes ([nboxes+1], [nterms], [nterms]; inactive/zero modes have empty ranges),
 * quadrature shape [nleaves*dim], boundary faces (leaf position, axis, side 0=LOWER/1=UPPER)
 * and interfaces (minus position, plus position, axis).  Any output may be NULL. */
int grico_space_export(const GricoSpace* space, int64_t* morton_order, int64_t* leaf_box_offset,
                       int64_t* term_offsets, int64_t* term_index, double* term_coef, int32_t* qshape,
                       int64_t* bnd_leaf, int32_t* bnd_axis, int32_t* bnd_side, int64_t* if_minus,
                       int64_t* if_plus, int32_t* if_axis);
/* Reduced-space multigrid prolongation from a coarse space to the next finer space on the same
 * grid (p-coarsened leaf or one h-split), replacing _compile_multigrid_transfer
 * (multigrid.jl:614-848).  The coarse reduced map is CSR (full dof -> reduced dofs); the fine
 * reduced map is an index per full dof (-1 when constrained).  Result: CSR over fine reduced
 * rows, columns sorted (coarse reduced dofs). */
typedef struct GricoTransfer GricoTransfer;
int grico_transfer_build(const GricoSpace* coarse_space, const GricoSpace* fine_space,
                         const int64_t* coarse_red_offsets, const int64_t* coarse_red_index,
                         const double* coarse_red_coef, int64_t n_coarse_reduced,
                         const int64_t* fine_reduced_index, int64_t n_fine_reduced, GricoTransfer** out);
int grico_transfer_export(const GricoTransfer* transfer, int64_t* nnz, int64_t* row_offsets,
                          int64_t* col_index, double* values);
int grico_transfer_destroy(GricoTransfer* transfer);
/* 1-D numerics of the product: Gauss-Legendre rule (quadrature.jl:342-410) and the
 * integrated-Legendre finite-element basis (polynomials.jl:238-247, 403-434). */
int grico_gauss_legendre(int count, double* points, double* weights);
int grico_fe_basis(double x, int degree, double* values, double* derivatives);

/* ================================================================================
 * Device plan (the drop-in for AssemblyPlan's matrix-free runtime)
 * ================================================================================ */

/* One batch of cells sharing a kernel signature (plans.jl:307-332): same per-axis degree and
 * tensor quadrature.  Local modes are addressed by their box index (axis 1 fastest,
 * basis.jl:150-180); trunk-basis cells mark missing box modes inactive. */
typedef struct GricoCellBatchDesc {
  int32_t n_cells;
  int32_t degree[3];          /* per axis; unused axes 0                                  */
  int32_t qpoints[3];         /* Gauss points per axis (q >= p+1 required)                 */
  const int32_t* map_index;   /* [n_cells*n_box]: >=0 global dof, -1 inactive, <=-2 tail k=-(v+2) */
  const double* map_coef;     /* [n_cells*n_box] or NULL (all 1.0)                          */
  int64_t n_tail;             /* multi-term entries (hanging-node expansions)               */
  const int64_t* tail_offsets;/* [n_tail+1]                                                 */
  const int32_t* tail_index;  /* global dofs                                                */
  const double* tail_coef;
  const double* cell_size;    /* [n_cells*dim] physical cell sizes h_a                      */
  const double* kappa_points; /* NULL or [n_cells*prod(q)] pointwise gradient coefficient    */
} GricoCellBatchDesc;

/* Point-quadrature items (one cell's modes at an arbitrary list of reference points):
 * non-tensor cells such as finite-cell cut cells (accumulators.jl:1022-1054), boundary faces
 * and embedded surfaces (accumulators.jl:1133-1161, 1202-1214).  All items of a batch share the
 * cell degree.  GRICO_ITEM_CELL uses the plan's mass/kappa form; GRICO_ITEM_NITSCHE is the
 * symmetric Nitsche form TestChannels(-du/dn + eta*u, -u*n)
 * (examples/annular_nitsche_fcm/driver.jl:52-62) with eta per item. */
#define GRICO_ITEM_CELL 1
#define GRICO_ITEM_NITSCHE 2
/* Finite-cell cut cells as octree subcells (regions.jl:477-510): each subcell carries the
 * cell's tensor rule of qpoints[a] Gauss points per axis mapped onto the subcell
 * [-1 + 2 pos 2^-level, -1 + 2 (pos + 1) 2^-level] per axis, a keep mask over those
 * prod(qpoints) <= 64 points (bit p, axis 1 fastest) and a weight factor (2^(-dim level) times
 * the measure factor of FiniteCellExtension).  Uses the plan's mass/kappa form; the point
 * arrays of the descriptor (point_offsets, ref_points, weights, normals, eta) are unused and
 * kappa_points / rhs source values are given per subcell point [n_subcells * prod(qpoints)]. */
#define GRICO_ITEM_SUBCELLS 3
/* Two-sided interface items (interface_apply!, accumulators.jl:1576-1616) with the symmetric
 * interior-penalty form -{du/dn}[v] - {dv/dn}[u] + sigma [u][v] of
 * benchmark/sine_poisson_sipg.jl:54-95: [w] = w(minus) - w(plus), {w} = average, n the unit
 * normal e_axis from the minus to the plus cell, sigma = eta[item].  map_index holds the minus
 * cell's box modes followed by the plus cell's (prod(degree+1) + prod(degree_plus+1) entries per
 * item); ref_points / cell_size are the minus side's, ref_points_plus / cell_size_plus the plus
 * side's, both on the shared tangential patch rule with physical `weights`.  No load term. */
#define GRICO_ITEM_INTERFACE 4

typedef struct GricoPointBatchDesc {
  int32_t n_items;
  int32_t kind;               /* GRICO_ITEM_*                                               */
  int32_t degree[3];
  const int32_t* map_index;   /* [n_items*n_box], same encoding as GricoCellBatchDesc       */
  const double* map_coef;
  int64_t n_tail;
  const int64_t* tail_offsets;
  const int32_t* tail_index;
  const double* tail_coef;
  const double* cell_size;    /* [n_items*dim]                                              */
  const int64_t* point_offsets; /* [n_items+1]                                              */
  const double* ref_points;   /* [n_points*dim] reference coordinates in [-1,1]^dim         */
  const double* weights;      /* [n_points] physical weights                                */
  const double* normals;      /* [n_points*dim] unit normals (GRICO_ITEM_NITSCHE)           */
  const double* eta;          /* [n_items] penalty (GRICO_ITEM_NITSCHE)                     */
  const double* kappa_points; /* [n_points] or NULL (GRICO_ITEM_CELL)                       */
  /* GRICO_ITEM_SUBCELLS only */
  int32_t qpoints[3];
  const int64_t* subcell_offsets; /* [n_items+1]                                            */
  const int32_t* subcell_level;   /* [n_subcells]                                           */
  const int32_t* subcell_pos;     /* [n_subcells*dim]                                       */
  const uint64_t* subcell_mask;   /* [n_subcells]                                           */
  const double* subcell_weight;   /* [n_subcells]                                           */
  /* GRICO_ITEM_INTERFACE only */
  int32_t degree_plus[3];
  const double* ref_points_plus;  /* [n_points*dim]                                         */
  const double* cell_size_plus;   /* [n_items*dim]                                          */
  const int32_t* face_axis;       /* [n_items] 0-based normal axis                          */
} GricoPointBatchDesc;

typedef struct GricoPlanDesc {
  int32_t dim;                /* 1..3 (sum-factorized kernels for 2 and 3)                  */
  int32_t form;               /* GRICO_FORM_*                                               */
  double mass;                /* a0 = mass*u                                                */
  double kappa;               /* a_grad = kappa*k(x)*grad u                                 */
  int64_t n_full;             /* full field-layout dofs                                     */
  int32_t n_batches;
  const GricoCellBatchDesc* batches;
  /* constraint rows of the full layout (plans.jl:38-56, assembly.jl:1893-1920) */
  int64_t n_fixed;
  const int64_t* fixed_dofs;
  const double* fixed_values;
  int64_t n_relations;        /* Dirichlet affine rows: x[p] - sum c x[j] = rhs             */
  const int64_t* rel_pivot;
  const int64_t* rel_offsets; /* [n_relations+1]                                            */
  const int64_t* rel_index;
  const double* rel_coef;
  const double* rel_rhs;
  /* reduced map u_full = shift + P u_red (assembly.jl:19-27): CSR rows per full dof */
  int64_t n_reduced;
  const int64_t* red_offsets; /* [n_full+1]                                                 */
  const int64_t* red_index;
  const double* red_coef;
  const double* red_shift;    /* [n_full] or NULL                                           */
  int32_t n_point_batches;    /* point-quadrature items (cut cells, faces, surfaces)        */
  const GricoPointBatchDesc* point_batches;
} GricoPlanDesc;

typedef struct GricoPlan GricoPlan;

/* Copies every descriptor array to the device; the caller may free them afterwards.  The plan
 * owns its workspaces and one CUDA stream.  Calls on one plan are serialised. */
int grico_plan_create(const GricoPlanDesc* desc, GricoPlan** out);
/* Per-batch tile autotuner (no reference counterpart): times the variants of the 3-D
 * tensor-cell kernel on this plan's batches for `nrhs` right-hand sides in `precision`, keeps
 * the fastest per batch for later applies of that precision, and writes the choice per cell
 * batch to `chosen` (may be NULL).  Variants: 0, 1, 2 = half, default, double cells per block
 * with one block per cell group; 3, 4, 5 = the same sizes in the persistent kernel that
 * prefetches the next cell group's gather with asynchronous copies, with the 1-D contractions in
 * even-odd form; 6, 7, 8 = that kernel with direct contractions; 9 = one warp per 32 / q cells
 * with one thread per cell plane (q <= 6, plain maps, constant coefficients; the default at
 * q <= 3); 10 = FP32 only, uniform batches (one cell size, constant coefficients, plain maps,
 * degree <= 4): one element matrix on the tensor cores (tcgen05, BF16 hi/lo pieces of x and of
 * the matrix, FP32 accumulation; measured slower than 3..9 on B200, so never the default; other
 * batches treat 10 as 1;
 * a bounded wait that gave up is reported by grico_tc_status).  Batches without a 3-D
 * isotropic tensor kernel report 1.  Allocates scratch; call before any stream capture. */
int grico_plan_autotune(GricoPlan* plan, int nrhs, int precision, int reps, int* chosen);
/* Sets the kernel variant of every cell batch for `precision` (tiles[n_batches], values as
 * reported by grico_plan_autotune), e.g. to replay a stored tuning without timing again.
 * No reference counterpart. */
int grico_plan_set_tiles(GricoPlan* plan, int precision, const int* tiles, int n_batches);
/* Pointwise mass coefficients c(x_q) added to the form's mass at the quadrature points of every
 * cell batch: mass_points[b] = [n_cells*prod(q)] for batch b (points axis 1 fastest, as the
 * load arrays), NULL entry or NULL array = none.  This is how a Newton tangent
 * (tangent_apply!, assembly.jl:1050-1083) with a state-dependent reaction term (e.g.
 * lambda exp(u), examples/nonlinear_bratu/driver.jl) runs through the ordinary apply, reduced
 * apply and diagonal kernels.  Plans with point-quadrature items are refused.  Arrays are
 * copied (device pointers, or host with GRICO_FLAG_HOST_POINTERS). */
int grico_plan_set_mass_points(GricoPlan* plan, const double* const* mass_points, int flags);
/* u at the quadrature points of every cell batch: values[b] = [n_cells*prod(q)] (NULL entries are
 * skipped), u on the full layout (reduced = 0) or the reduced one (reduced = 1).  The state
 * evaluation of residual!/tangent_apply! (assembly.jl:997-1083). */
int grico_eval_points(GricoPlan* plan, const double* u, int reduced, double* const* values, int flags);
/* Average device time of each batch's kernel launch over the applies called with
 * GRICO_FLAG_TIME_BATCHES since the last query (CUDA events recorded on the apply's stream
 * around each launch).  Batches are numbered cell batches first, then point batches; the first
 * n_batches are reported: ms[i] average milliseconds per launch, launches[i] (may be NULL)
 * launches timed.  Synchronises with those events and resets the record.  No reference
 * counterpart (measurement support). */
int grico_plan_batch_times(GricoPlan* plan, double* ms, int64_t* launches, int n_batches);
int grico_plan_destroy(GricoPlan* plan);
/* n_full, n_reduced */
int grico_plan_sizes(const GricoPlan* plan, int64_t* n_full, int64_t* n_reduced);

/* y = A x on the full layout with constraint rows written explicitly (assembly.jl:540-564).
 * x, y: [nrhs][n_full] device (or host with GRICO_FLAG_HOST_POINTERS) arrays of the precision's
 * element type; x and y must not alias.  stream: cudaStream_t or NULL for the plan stream. */
int grico_apply(GricoPlan* plan, const void* x, void* y, int nrhs, int precision, int flags, void* stream);
/* y_red = P^T A P x_red (assembly.jl:905-915). */
int grico_reduced_apply(GricoPlan* plan, const void* x, void* y, int nrhs, int precision, int flags,
                        void* stream);
/* Full-layout right-hand side (rhs!, assembly.jl:488-507): the load vector from the source
 * values tabulated at the quadrature points (same layout as grico_reduced_rhs), with the rows of
 * fixed dofs set to their values and the rows of Dirichlet relation pivots to the relations'
 * right-hand sides (_write_constraint_rhs!, assembly.jl:1876-1891).  b_full: [n_full]. */
int grico_rhs(GricoPlan* plan, const double* const* source_points, double* b_full, int flags);
/* Reduced right-hand side P^T (b_phys - A shift) from the load tabulated at the quadrature
 * points of every batch: source[b] = [n_cells*prod(q)] for cell batch b, then one array of
 * [n_points] per point batch (cells: f; Nitsche items: boundary data g giving
 * TestChannels(eta*g, -g*n)); NULL => 0 — assembly.jl:917-933. */
int grico_reduced_rhs(GricoPlan* plan, const double* const* source_points, double* b_reduced, int flags);
/* Allocation-free variant of grico_reduced_rhs for callers that cannot allocate GPU memory
 * (host callbacks, services with a fixed GPU memory budget).  No counterpart in the reference.  Its two full-layout temporaries
 * live in a static 16 MiB device array that every GPU loading the library holds until exit, so
 * plans with more than 1,048,576 full-layout dofs are rejected with GRICO_ERR_INVALID.
 * source_points[b] and b_reduced are DEVICE pointers; the work is enqueued on `stream`
 * (NULL = the plan's stream) and the call does not synchronise.  The first call on a device
 * resolves the array's device address (cudaGetSymbolAddress).  All calls share the array: calls whose GPU work overlaps in time (other
 * streams, other threads) race on it. */
int grico_reduced_rhs_static(GricoPlan* plan, const double* const* source_points, double* b_reduced,
                             void* stream);
/* Jacobi diagonal of the reduced operator (assembly.jl:662-675 where the reduced map is direct;
 * exact local-matrix diagonal otherwise, replacing the probe fallback solve.jl:722-738). */
int grico_reduced_diagonal(GricoPlan* plan, double* diag, int flags);
/* Reconstruct the full vector u = shift + P u_red (assembly.jl:965-970). */
int grico_expand_reduced(GricoPlan* plan, const double* u_red, double* u_full, int flags);

/* ---- sharded reduced solves (no reference counterpart: the reference runs in one process) ----
 * A rank holds the plan of its cells with a local reduced numbering: the dofs it owns first,
 * the ghost dofs it shares with other ranks after them.  All pointers are device pointers; the
 * work is enqueued on `stream` (NULL = default stream) and nothing synchronises. */
/* buf[0 .. n_slots) = 0, then buf[slot[i]] = y[local[i]] for i < n: the halo contribution of
 * this rank, summed over ranks by the caller's collective */
int grico_halo_pack(const double* y, const int32_t* local, const int32_t* slot, int64_t n, double* buf,
                    int64_t n_slots, void* stream);
/* y[local[i]] = buf[slot[i]] for i < n */
int grico_halo_unpack(double* y, const int32_t* local, const int32_t* slot, int64_t n, const double* buf,
                      void* stream);
/* *out = sum_{i<n} x_i y_i (deterministic two-stage sum); partial: scratch of 592 doubles */
int grico_vec_dot(int64_t n, const double* x, const double* y, double* out, double* partial, void* stream);
/* y = a x + b y (y is not read when b == 0) */
int grico_vec_axpby(int64_t n, double a, const double* x, double b, double* y, void* stream);
/* dinv = 1 / d; synchronises `stream` and returns GRICO_ERR_NONFINITE if an entry of d is zero
 * or not finite (solve.jl:740-748) */
int grico_vec_invert(int64_t n, const double* d, double* dinv, void* stream);
/* CG steps on device scalars s = scalars[0..3] = (r.z, p.Ap, r.r, r.z new) (solve.jl:376-431):
 * update_xr: x += (s0/s1) p, r -= (s0/s1) q on n entries (nothing when s1 <= 0), s2 = sum of
 *            r*r over the first n_sum entries;
 * precondition: z = dinv .* r (dinv NULL: z = r), s3 = sum of r*z over the first n_sum entries;
 * direction: p = z + (s3/s0) p, then s0 = s3. */
int grico_cg_update_xr(int64_t n, int64_t n_sum, double* x, double* r, const double* p, const double* q,
                       double* scalars, double* partial, void* stream);
int grico_cg_precondition(int64_t n, int64_t n_sum, const double* dinv, const double* r, double* z, double* scalars,
                          double* partial, void* stream);
int grico_cg_direction(int64_t n, double* p, const double* z, double* scalars, void* stream);

/* ---- Krylov solvers on the reduced system ---- */
#define GRICO_PRECOND_IDENTITY 0
#define GRICO_PRECOND_JACOBI 1
#define GRICO_PRECOND_MULTIGRID 2

typedef struct GricoSolveOptions {
  double relative_tolerance;  /* stop when ||r|| <= max(atol, rtol*||b||) (solve.jl:407-421) */
  double absolute_tolerance;
  int32_t maxiter;
  int32_t preconditioner;     /* GRICO_PRECOND_*                                            */
  int32_t restart;            /* FGMRES restart (solve.jl:94-99)                            */
  int32_t use_initial;        /* x holds the initial solution                               */
} GricoSolveOptions;

typedef struct GricoSolveReport {
  int32_t iterations;
  int32_t status;
  double initial_residual;
  double final_residual;
  double seconds;             /* device time of the solve                                  */
} GricoSolveReport;

typedef struct GricoMultigrid GricoMultigrid;

int grico_cg_solve(GricoPlan* plan, GricoMultigrid* mg, const double* b, double* x,
                   const GricoSolveOptions* opts, GricoSolveReport* report, int flags);
/* nrhs systems A x_s = b_s (B, X: [nrhs][n_reduced]) solved by lockstep CG, one operator apply
 * for all systems per iteration, identity or Jacobi preconditioning, each with the reference's
 * stopping rule; with GRICO_FLAG_MIXED the CG runs in FP32 inside FP64 iterative refinement
 * (FP64 residuals and updates).  reports: [nrhs] or NULL.  No reference counterpart for the
 * batching.  Its work vectors (about 4 + 5 per system of n_reduced values, FP32 and FP64) stay
 * on the plan for the next call until grico_plan_destroy, so repeated solves allocate nothing;
 * concurrent calls on one plan share them. */
int grico_cg_solve_multi(GricoPlan* plan, const double* B, double* X, int nrhs, const GricoSolveOptions* opts,
                         GricoSolveReport* reports, int flags);

int grico_fgmres_solve(GricoPlan* plan, GricoMultigrid* mg, const double* b, double* x,
                       const GricoSolveOptions* opts, GricoSolveReport* report, int flags);

/* ---- hp geometric multigrid (multigrid.jl:66-96, 309-345, 858-1087) ---- */
typedef struct GricoTransferDesc {
  /* prolongation coarse -> fine on reduced vectors as CSR over fine rows; restriction is its
   * transpose (multigrid.jl:614-636, 1060-1087) */
  int64_t n_fine, n_coarse;
  const int64_t* row_offsets; /* [n_fine+1] */
  const int64_t* col_index;
  const double* values;
} GricoTransferDesc;

#define GRICO_SMOOTHER_JACOBI 0     /* damped Jacobi, reference default (multigrid.jl:943-956) */
#define GRICO_SMOOTHER_CHEBYSHEV 1  /* Chebyshev-Jacobi (no reference counterpart)            */
#define GRICO_SMOOTHER_GMRES 2      /* fixed-step right-Jacobi GMRES (multigrid.jl:963-1056), for
                                       non-SPD operators; not for CG (multigrid.jl:253-255)      */

typedef struct GricoMGOptions {
  int32_t smoother;
  int32_t pre_steps, post_steps;
  double jacobi_omega;          /* 0.8 default (multigrid.jl:70)                            */
  int32_t chebyshev_degree;
  double chebyshev_lower;       /* fraction of lambda_max for the lower bound               */
  int32_t precision;            /* GRICO_PREC_FP64 or GRICO_PREC_FP32 for level applies     */
  int32_t smoother_restart;     /* GMRES smoother Krylov columns, >= max(pre, post) (8)     */
} GricoMGOptions;

/* levels[0] is the coarsest; transfers[i] maps level i -> i+1.  coarse_matrix is the dense
 * reduced operator of level 0 (row-major n0 x n0), factorised by Cholesky on create. */
int grico_mg_create(GricoPlan* const* levels, int nlevels, const GricoTransferDesc* transfers,
                    const double* coarse_matrix, const GricoMGOptions* opts, GricoMultigrid** out);
int grico_mg_destroy(GricoMultigrid* mg);
/* z = V-cycle(r) on the finest level (multigrid.jl:858-889) */
int grico_mg_vcycle(GricoMultigrid* mg, const double* r, double* z, int flags);
/* Chebyshev eigenvalue estimate lambda_max(D^-1 A) of one level (0 if unused, -1 on error). */
double grico_mg_lambda_max(GricoMultigrid* mg, int level);

const char* grico_last_error(void);

/* ---- learned smoother sweep inside the V-cycle (no reference counterpart) ----
 * On `level` (a smoothed level whose free dofs sit on an nx x ny x nz grid, e.g. the degree-1
 * level of a uniform mesh), the sweep computes r = b - A x, feeds (D^-1 r / sigma, log a) to
 * the network (3x3x3 convolutions, ReLU between layers, BF16 activations, FP32 weights),
 * scatters sigma * omega * output onto x and keeps the new iterate only if its D^-1-weighted
 * residual norm is smaller.  It replaces the last pre-smoothing step on that level. */
typedef struct GricoLearnedDesc {
  int32_t level;
  int32_t nx, ny, nz;
  const int64_t* grid_index;            /* [nz*ny*nx] (x fastest): reduced dof or -1        */
  const float* grid_log_coefficient;    /* [nz*ny*nx] second input channel                 */
  int32_t n_layers;
  const int32_t* channels;              /* [n_layers+1], channels[0] = 2, last = 1          */
  const float* const* weights;          /* per layer [co][ci][27]                          */
  const float* const* biases;           /* per layer [co]                                  */
  double omega;                         /* correction scale                               */
} GricoLearnedDesc;
/* NULL desc removes the sweep.  Host arrays are copied. */
int grico_mg_set_learned(GricoMultigrid* mg, const GricoLearnedDesc* desc);
/* learned sweeps run and kept since grico_mg_set_learned */
int grico_mg_learned_stats(GricoMultigrid* mg, int64_t* sweeps, int64_t* accepted);

/* ---- learned smoother: network primitives (device pointers, asynchronous on `stream`) ----
 * No reference counterpart: the learned smoother is an addition of this library.  Tensors are
 * [batch][channel][z][y][x]; convolutions are 3x3x3, stride 1, zero padding; weights
 * [out][in][27] FP32; activations FP32 or BF16 (x_bf16 / y_bf16), FP32 arithmetic. */
int grico_conv3d_forward(const void* x, int x_bf16, const float* w, const float* bias, void* y, int y_bf16, int B,
                         int Ci, int Co, int Z, int Y, int X, int relu, void* stream);
/* The convolution on the tensor cores (tcgen05.mma, BF16 operands, FP32 accumulation in tensor
 * memory) with channels-last activations: x BF16 [batch][z][y][x][Ci], Ci = 16, 32, 48 or 64;
 * weights packed once by grico_conv3d_pack_weights_tc; y BF16 channels-last [batch][z][y][x][Co]
 * (y_layout 0, Co a multiple of 8) or FP32 [batch][Co][z][y][x] (y_layout 1); Co up to 128; x,
 * wp and a channels-last y 16-byte aligned.  Other shapes are rejected with GRICO_ERR_INVALID. */
int64_t grico_conv_tc_weight_bytes(int Ci, int Co); /* -1: shape not served */
int grico_conv3d_pack_weights_tc(const float* w, int Ci, int Co, void* wp, void* stream);
int grico_conv3d_forward_tc(const void* x, const void* wp, const float* bias, void* y, int y_layout, int B, int Ci,
                            int Co, int Z, int Y, int X, int relu, void* stream);
/* Synchronises `stream`; GRICO_ERR_TIMEOUT (and the flag cleared) if a bounded wait of a
 * tensor-core kernel (the convolutions, the FP32 apply of uniform batches) gave up on the current
 * device since the last call, else GRICO_OK.  grico_conv_tc_status is the same call. */
int grico_tc_status(void* stream);
int grico_conv_tc_status(void* stream);
/* gx = transposed convolution of gy; wt: scratch of Co*Ci*27 floats */
int grico_conv3d_backward_data(const float* gy, const float* w, float* wt, float* gx, int B, int Ci, int Co, int Z,
                               int Y, int X, void* stream);
/* gw = d loss / d w, gb = d loss / d bias (NULL: skipped); overwrites, does not accumulate */
int grico_conv3d_backward_weight(const float* x, const float* gy, float* gw, float* gb, int B, int Ci, int Co, int Z,
                                 int Y, int X, void* stream);
int grico_relu_backward(const float* y, float* g, int64_t n, void* stream);
/* masked mean squared error sum(m (p - t)^2) / count into *loss (device double) and its
 * gradient g; partial: scratch of 592 doubles */
int grico_mse_grad(const float* p, const float* t, const float* mask, float* g, int64_t n, double count,
                   double* partial, double* loss, void* stream);
int grico_adam_step(float* w, const float* g, float* m, float* v, int64_t n, float lr, float beta1, float beta2,
                    int step, float eps, void* stream);
/* grid <-> reduced vector: idx[g] is the reduced dof of grid point g, or -1 (FP32) */
int grico_grid_gather(const int64_t* idx, int64_t n_grid, const float* src, float scale, float* dst, void* stream);
int grico_grid_scatter_add(const int64_t* idx, int64_t n_grid, const float* src, float scale, float* dst,
                           void* stream);
/* out = w (r - ar) and *sum = sum w (r - ar)^2 (device double); partial: scratch of 592 doubles */
int grico_weighted_residual(const float* r, const float* ar, const float* w, float* out, int64_t n, double* partial,
                            double* sum, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* GRICO_B200_H */
