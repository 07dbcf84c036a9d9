// Reduced-space Krylov solvers on the device: preconditioned CG (solve.jl:376-431) with the
// reference's unpreconditioned stopping rule ||r||^2 <= max(atol, rtol*||b||)^2, Jacobi
// (solve.jl:713-774) or multigrid (multigrid.jl:858-865) preconditioning.
#include <cuda_runtime.h>

#include <chrono>
#include <cmath>
#include <string>

#include "grico_host.h"
#include "grico_mg_internal.h"
#include "grico_plan_internal.h"
#include "vector_kernels.cuh"

namespace grico {

int grid_blocks(int64_t n) { return int(std::min<int64_t>((n + 255) / 256, kRedBlocks)); }

constexpr int GRICO_NOT_DONE = 1;

namespace {

struct Scalars {
  // device scalar slots
  enum { RZ = 0, PAP = 1, RR = 2, RZ_NEW = 3, BB = 4 };
};

double read_scalar(GricoPlan* P, int slot, cudaStream_t st) {
  double v = 0.0;
  cudaMemcpyAsync(&v, P->scalars.get<double>() + slot, sizeof(double), cudaMemcpyDeviceToHost, st);
  cudaStreamSynchronize(st);
  return v;
}

void dot_into(GricoPlan* P, const double* a, const double* b, int64_t n, int slot, cudaStream_t st) {
  dot_partial<double><<<kRedBlocks, kRedThreads, 0, st>>>(a, b, n, P->partial.get<double>());
  reduce_final<<<1, kRedThreads, 0, st>>>(P->partial.get<double>(), kRedBlocks, P->scalars.get<double>() + slot);
}

}  // namespace

double read_scalar_pub(GricoPlan* P, int slot, cudaStream_t st) { return read_scalar(P, slot, st); }

// z = M r for the chosen preconditioner; returns status.
int apply_preconditioner(GricoPlan* P, GricoMultigrid* mg, int kind, const double* r, double* z, cudaStream_t st,
                         int slot_rz) {
  const int64_t n = P->n_red;
  if (kind == GRICO_PRECOND_MULTIGRID) {
    int rc = mg_vcycle_device(mg, r, z, st);
    if (rc) return rc;
    if (slot_rz >= 0) dot_into(P, r, z, n, slot_rz, st);
    return GRICO_OK;
  }
  const double* dinv = kind == GRICO_PRECOND_JACOBI ? P->w_dinv.get<double>() : nullptr;
  jacobi_dot<<<kRedBlocks, kRedThreads, 0, st>>>(r, dinv, z, n, P->partial.get<double>());
  if (slot_rz >= 0)
    reduce_final<<<1, kRedThreads, 0, st>>>(P->partial.get<double>(), kRedBlocks, P->scalars.get<double>() + slot_rz);
  return GRICO_OK;
}

int prepare_jacobi(GricoPlan* P, cudaStream_t st) {
  const int64_t n = P->n_red;
  DevBuf d;
  if (!d.alloc(sizeof(double) * std::max<int64_t>(n, 1)) || !P->w_dinv.ensure(sizeof(double) * std::max<int64_t>(n, 1)))
    return GRICO_ERR_CUDA;
  int rc = grico_reduced_diagonal(P, d.get<double>(), 0);
  if (rc) return rc;
  DevBuf flag;
  if (!flag.alloc(sizeof(int))) return GRICO_ERR_CUDA;
  cudaMemsetAsync(flag.ptr, 0, sizeof(int), st);
  invert_diagonal<<<grid_blocks(n), 256, 0, st>>>(d.get<double>(), P->w_dinv.get<double>(), n, flag.get<int>());
  int bad = 0;
  cudaMemcpyAsync(&bad, flag.ptr, sizeof(int), cudaMemcpyDeviceToHost, st);
  cudaStreamSynchronize(st);
  if (bad) {
    set_error("Jacobi preconditioner found a zero or non-finite diagonal entry");
    return GRICO_ERR_NONFINITE;
  }
  return GRICO_OK;
}

}  // namespace grico

using namespace grico;

namespace {

// An empty reduced system (every dof fixed) is solved before the first iteration: ||b|| = 0
// meets the stopping rule of solve.jl:407-421 at once.
int empty_system(GricoSolveReport* report) {
  if (report) *report = GricoSolveReport{};
  return GRICO_OK;
}

}  // namespace

extern "C" int grico_cg_solve(GricoPlan* P, GricoMultigrid* mg, const double* b, double* x,
                              const GricoSolveOptions* opts, GricoSolveReport* report, int flags) {
  if (!P || !b || !x || !opts) { set_error("cg: invalid argument"); return GRICO_ERR_INVALID; }
  if (opts->preconditioner == GRICO_PRECOND_MULTIGRID && !mg) { set_error("cg: multigrid preconditioner missing"); return GRICO_ERR_INVALID; }
  if (opts->preconditioner == GRICO_PRECOND_MULTIGRID && mg_smoother(mg) == GRICO_SMOOTHER_GMRES) {
    // multigrid.jl:253-255: the GMRES smoother makes the V-cycle nonlinear and nonsymmetric
    set_error("cg: the GMRES multigrid smoother needs FGMRES");
    return GRICO_ERR_INVALID;
  }
  if (opts->maxiter < 1) { set_error("maxiter must be positive"); return GRICO_ERR_INVALID; }
  if (!(opts->relative_tolerance >= 0) || !(opts->absolute_tolerance >= 0)) { set_error("tolerances must be non-negative"); return GRICO_ERR_INVALID; }
  if (P->n_red == 0) return empty_system(report);
  cudaStream_t st = P->stream;
  const int64_t n = P->n_red;
  const size_t bytes = sizeof(double) * std::max<int64_t>(n, 1);
  if (!P->w_r.ensure(bytes) || !P->w_z.ensure(bytes) || !P->w_p.ensure(bytes) || !P->w_q.ensure(bytes) ||
      !P->w_x.ensure(bytes) || !P->w_b.ensure(bytes))
    return GRICO_ERR_CUDA;
  double *r = P->w_r.get<double>(), *z = P->w_z.get<double>(), *p = P->w_p.get<double>(), *q = P->w_q.get<double>();
  double* xd = x;
  const double* bd = b;
  if (flags & GRICO_FLAG_HOST_POINTERS) {
    cudaMemcpyAsync(P->w_b.ptr, b, sizeof(double) * n, cudaMemcpyHostToDevice, st);
    bd = P->w_b.get<double>();
    xd = P->w_x.get<double>();
    if (opts->use_initial) cudaMemcpyAsync(xd, x, sizeof(double) * n, cudaMemcpyHostToDevice, st);
  }
  if (opts->preconditioner == GRICO_PRECOND_JACOBI) {
    int rc = prepare_jacobi(P, st);
    if (rc) return rc;
  }
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  cudaEventRecord(e0, st);
  GricoSolveReport rep{};
  int status = GRICO_OK;
  // r = b - A x
  cudaMemcpyAsync(r, bd, sizeof(double) * n, cudaMemcpyDeviceToDevice, st);
  if (opts->use_initial) {
    run_apply<double>(P, true, xd, q, 1, st);
    axpby_kernel<double><<<grid_blocks(n), 256, 0, st>>>(-1.0, q, 1.0, r, n);
  } else {
    cudaMemsetAsync(xd, 0, sizeof(double) * n, st);
  }
  int rc = apply_preconditioner(P, mg, opts->preconditioner, r, z, st, Scalars::RZ);
  if (rc) return rc;
  cudaMemcpyAsync(p, z, sizeof(double) * n, cudaMemcpyDeviceToDevice, st);
  dot_into(P, bd, bd, n, Scalars::BB, st);
  dot_into(P, r, r, n, Scalars::RR, st);
  const double bnorm = std::sqrt(read_scalar(P, Scalars::BB, st));
  const double tol = std::max(opts->absolute_tolerance, opts->relative_tolerance * bnorm);
  double rr = read_scalar(P, Scalars::RR, st);
  rep.initial_residual = std::sqrt(rr);
  int it = 0;
  bool converged = rr <= tol * tol;
  // One iteration as a fixed sequence of stream operations: operator apply, p.Ap, x/r update
  // with ||r||^2, preconditioner with r.z, new direction.  It is replayed as one CUDA graph
  // (the multigrid V-cycle alone is hundreds of small launches); after each replay the host
  // reads p.Ap and ||r||^2 with a single copy.
  auto iteration = [&](cudaStream_t s) -> int {
    run_apply<double>(P, true, p, q, 1, s);
    dot_into(P, p, q, n, Scalars::PAP, s);
    cg_update_xr<<<kRedBlocks, kRedThreads, 0, s>>>(xd, r, p, q, P->scalars.get<double>(), n, P->partial.get<double>());
    reduce_final<<<1, kRedThreads, 0, s>>>(P->partial.get<double>(), kRedBlocks, P->scalars.get<double>() + Scalars::RR);
    int prc = apply_preconditioner(P, mg, opts->preconditioner, r, z, s, Scalars::RZ_NEW);
    if (prc) return prc;
    cg_direction<<<kRedBlocks, kRedThreads, 0, s>>>(p, z, P->scalars.get<double>() + Scalars::RZ_NEW,
                                                    P->scalars.get<double>() + Scalars::RZ, n);
    cudaMemcpyAsync(P->scalars.get<double>() + Scalars::RZ, P->scalars.get<double>() + Scalars::RZ_NEW, sizeof(double),
                    cudaMemcpyDeviceToDevice, s);
    return GRICO_OK;
  };
  // The graph is kept on the plan and replayed by later solves with the same multigrid cycle,
  // preconditioner, solution buffer and plan epochs (every other buffer it touches belongs to the
  // plan or the multigrid object; an epoch changes with the kernels or arguments of a plan).
  cudaGraphExec_t exec = nullptr;
  if (!converged && !(flags & GRICO_FLAG_NO_GRAPH)) {
    const bool use_mg = opts->preconditioner == GRICO_PRECOND_MULTIGRID;
    const uint64_t mg_key = use_mg ? mg_identity(mg) : 0;
    const uint64_t epoch = P->epoch + (use_mg ? mg_epoch(mg) : 0);
    if (P->cg_exec && P->cg_key_mg == mg_key && P->cg_key_pc == opts->preconditioner && P->cg_key_x == xd &&
        P->cg_key_epoch == epoch) {
      exec = P->cg_exec;
    } else {
      if (P->cg_exec) cudaGraphExecDestroy(P->cg_exec);
      P->cg_exec = nullptr;
      cudaGraph_t graph = nullptr;
      if (cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal) == cudaSuccess) {
        const int crc = iteration(st);
        const cudaError_t ec = cudaStreamEndCapture(st, &graph);
        if (crc == GRICO_OK && ec == cudaSuccess && graph &&
            cudaGraphInstantiate(&exec, graph, 0) != cudaSuccess)
          exec = nullptr;
        if (graph) cudaGraphDestroy(graph);
      }
      (void)cudaGetLastError();  // a failed capture falls back to direct launches
      if (exec) {
        P->cg_exec = exec;
        P->cg_key_mg = mg_key;
        P->cg_key_pc = opts->preconditioner;
        P->cg_key_x = xd;
        P->cg_key_epoch = epoch;
      }
    }
  }
  double hs[2] = {0.0, 0.0};  // p.Ap, ||r||^2 (adjacent scalar slots)
  while (!converged && it < opts->maxiter) {
    ++it;
    if (exec) {
      if (cudaGraphLaunch(exec, st) != cudaSuccess) { status = GRICO_ERR_CUDA; set_error("CG graph launch failed"); break; }
    } else {
      rc = iteration(st);
      if (rc) { status = rc; break; }
    }
    cudaMemcpyAsync(hs, P->scalars.get<double>() + Scalars::PAP, 2 * sizeof(double), cudaMemcpyDeviceToHost, st);
    cudaStreamSynchronize(st);
    const double pap = hs[0];
    if (!(pap > 0.0)) {
      status = std::isfinite(pap) ? GRICO_ERR_BREAKDOWN : GRICO_ERR_NONFINITE;
      set_error("CG encountered a non-positive operator direction");
      break;
    }
    rr = hs[1];
    if (!std::isfinite(rr)) { status = GRICO_ERR_NONFINITE; set_error("CG residual is not finite"); break; }
    if (rr <= tol * tol) { converged = true; break; }
  }
  cudaEventRecord(e1, st);
  cudaEventSynchronize(e1);
  float ms = 0;
  cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (status == GRICO_OK && !converged) {
    status = GRICO_ERR_NOT_CONVERGED;
    set_error("CG did not converge in maxiter iterations");
  }
  rep.iterations = it;
  rep.status = status;
  rep.final_residual = std::sqrt(rr);
  rep.seconds = ms * 1e-3;
  if (flags & GRICO_FLAG_HOST_POINTERS) cudaMemcpyAsync(x, xd, sizeof(double) * n, cudaMemcpyDeviceToHost, st);
  if (!cuda_ok(cudaStreamSynchronize(st), "cg")) return GRICO_ERR_CUDA;
  if (report) *report = rep;
  return status;
}

// Right-preconditioned flexible GMRES(restart) with modified Gram-Schmidt and Givens rotations
// (solve.jl:433-614).  Krylov and preconditioned bases live on the device; the small
// Hessenberg least-squares problem is solved on the host.
extern "C" int grico_fgmres_solve(GricoPlan* P, GricoMultigrid* mg, const double* b, double* x,
                                  const GricoSolveOptions* opts, GricoSolveReport* report, int flags) {
  if (!P || !b || !x || !opts) { set_error("fgmres: invalid argument"); return GRICO_ERR_INVALID; }
  if (opts->restart < 1) { set_error("restart must be positive"); return GRICO_ERR_INVALID; }
  if (opts->maxiter < 1) { set_error("maxiter must be positive"); return GRICO_ERR_INVALID; }
  if (opts->preconditioner == GRICO_PRECOND_MULTIGRID && !mg) { set_error("fgmres: multigrid preconditioner missing"); return GRICO_ERR_INVALID; }
  if (P->n_red == 0) return empty_system(report);
  cudaStream_t st = P->stream;
  const int64_t n = P->n_red;
  const int m = int(std::min<int64_t>(opts->restart, std::max<int64_t>(n, 1)));
  const size_t bytes = sizeof(double) * std::max<int64_t>(n, 1);
  DevBuf Vb, Zb;
  if (!Vb.alloc(bytes * (m + 1)) || !Zb.alloc(bytes * m) || !P->w_r.ensure(bytes) || !P->w_q.ensure(bytes) ||
      !P->w_x.ensure(bytes) || !P->w_b.ensure(bytes))
    return GRICO_ERR_CUDA;
  double* V = Vb.get<double>();
  double* Z = Zb.get<double>();
  double *r = P->w_r.get<double>(), *w = P->w_q.get<double>();
  double* xd = x;
  const double* bd = b;
  if (flags & GRICO_FLAG_HOST_POINTERS) {
    cudaMemcpyAsync(P->w_b.ptr, b, sizeof(double) * n, cudaMemcpyHostToDevice, st);
    bd = P->w_b.get<double>();
    xd = P->w_x.get<double>();
    if (opts->use_initial) cudaMemcpyAsync(xd, x, sizeof(double) * n, cudaMemcpyHostToDevice, st);
  }
  if (!opts->use_initial) cudaMemsetAsync(xd, 0, sizeof(double) * n, st);
  if (opts->preconditioner == GRICO_PRECOND_JACOBI) {
    int rc = prepare_jacobi(P, st);
    if (rc) return rc;
  }
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  cudaEventRecord(e0, st);
  auto residual = [&]() {
    cudaMemcpyAsync(r, bd, sizeof(double) * n, cudaMemcpyDeviceToDevice, st);
    run_apply<double>(P, true, xd, w, 1, st);
    axpby_kernel<double><<<grid_blocks(n), 256, 0, st>>>(-1.0, w, 1.0, r, n);
  };
  auto norm = [&](const double* v) {
    dot_into(P, v, v, n, 8, st);
    return std::sqrt(read_scalar(P, 8, st));
  };
  if (opts->use_initial) residual(); else cudaMemcpyAsync(r, bd, sizeof(double) * n, cudaMemcpyDeviceToDevice, st);
  const double bnorm = norm(bd);
  const double tol = std::max(opts->absolute_tolerance, opts->relative_tolerance * bnorm);
  double rnorm = norm(r);
  GricoSolveReport rep{};
  rep.initial_residual = rnorm;
  int status = GRICO_NOT_DONE;
  int total = 0;
  std::vector<double> H((m + 1) * m), g(m + 1), cs(m), sn(m), y(m);
  auto Hc = [&](int i, int j) -> double& { return H[i * m + j]; };
  auto finish = [&](int count) -> int {
    for (int row = count - 1; row >= 0; --row) {
      double v = g[row];
      for (int c = row + 1; c < count; ++c) v -= Hc(row, c) * y[c];
      double dgl = Hc(row, row);
      if (!std::isfinite(dgl) || dgl == 0.0) { set_error("FGMRES encountered a singular Krylov least-squares problem"); return GRICO_ERR_BREAKDOWN; }
      y[row] = v / dgl;
    }
    for (int c = 0; c < count; ++c)
      if (y[c] != 0.0) axpby_kernel<double><<<grid_blocks(n), 256, 0, st>>>(y[c], Z + c * n, 1.0, xd, n);
    residual();
    return GRICO_OK;
  };
  if (rnorm <= tol) status = GRICO_OK;
  while (status == GRICO_NOT_DONE && total < opts->maxiter) {
    rnorm = norm(r);
    if (!std::isfinite(rnorm)) { status = GRICO_ERR_NONFINITE; set_error("FGMRES residual is not finite"); break; }
    if (rnorm <= tol) { status = GRICO_OK; break; }
    std::fill(H.begin(), H.end(), 0.0);
    std::fill(g.begin(), g.end(), 0.0);
    axpby_kernel<double><<<grid_blocks(n), 256, 0, st>>>(1.0 / rnorm, r, 0.0, V, n);
    g[0] = rnorm;
    const int inner_limit = std::min(m, opts->maxiter - total);
    int inner = 0;
    bool updated = false;
    for (int j = 0; j < inner_limit; ++j) {
      ++total;
      inner = j + 1;
      int rc = apply_preconditioner(P, mg, opts->preconditioner, V + j * n, Z + j * n, st, -1);
      if (rc) { status = rc; break; }
      run_apply<double>(P, true, Z + j * n, w, 1, st);
      for (int i = 0; i <= j; ++i) {
        dot_into(P, w, V + i * n, n, 9 + (i % 4), st);
        axpy_dev<<<grid_blocks(n), 256, 0, st>>>(w, V + i * n, P->scalars.get<double>() + 9 + (i % 4), -1.0, n);
        Hc(i, j) = read_scalar(P, 9 + (i % 4), st);
      }
      double next = norm(w);
      Hc(j + 1, j) = next;
      if (next > 0.0) axpby_kernel<double><<<grid_blocks(n), 256, 0, st>>>(1.0 / next, w, 0.0, V + (j + 1) * n, n);
      for (int i = 0; i < j; ++i) {
        double a = Hc(i, j), bb = Hc(i + 1, j);
        Hc(i, j) = cs[i] * a + sn[i] * bb;
        Hc(i + 1, j) = -sn[i] * a + cs[i] * bb;
      }
      double scale = std::hypot(Hc(j, j), Hc(j + 1, j));
      double c = 1.0, s = 0.0;
      if (scale != 0.0) { c = Hc(j, j) / scale; s = Hc(j + 1, j) / scale; }
      cs[j] = c;
      sn[j] = s;
      double a = Hc(j, j), bb = Hc(j + 1, j);
      Hc(j, j) = c * a + s * bb;
      Hc(j + 1, j) = -s * a + c * bb;
      double g0 = g[j], g1 = g[j + 1];
      g[j] = c * g0 + s * g1;
      g[j + 1] = -s * g0 + c * g1;
      if (std::fabs(g[j + 1]) <= tol || next == 0.0) {
        rc = finish(j + 1);
        if (rc) { status = rc; break; }
        if (norm(r) <= tol) status = GRICO_OK;
        updated = true;
        break;
      }
    }
    if (status != GRICO_NOT_DONE) break;
    if (inner == 0) { status = GRICO_ERR_BREAKDOWN; set_error("FGMRES failed to build a Krylov update"); break; }
    if (!updated) {
      int rc = finish(inner);
      if (rc) { status = rc; break; }
    }
    if (norm(r) <= tol) status = GRICO_OK;
  }
  if (status == GRICO_NOT_DONE) { status = GRICO_ERR_NOT_CONVERGED; set_error("FGMRES did not converge in maxiter iterations"); }
  cudaEventRecord(e1, st);
  cudaEventSynchronize(e1);
  float ms = 0;
  cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  rep.iterations = total;
  rep.status = status;
  rep.final_residual = norm(r);
  rep.seconds = ms * 1e-3;
  if (flags & GRICO_FLAG_HOST_POINTERS) cudaMemcpyAsync(x, xd, sizeof(double) * n, cudaMemcpyDeviceToHost, st);
  if (!cuda_ok(cudaStreamSynchronize(st), "fgmres")) return GRICO_ERR_CUDA;
  if (report) *report = rep;
  return status;
}
