// af_imex.cu -- one IMEX-DG time step on the device: the stage drivers and the pressure
// fixed-point loop of the reference's EulerSolver::run (Atmospheric_Flow.cc:1110-1251),
// with device-resident Krylov solvers around the EULEROperator applies of this library.
//
//   update_density      (Atmospheric_Flow.cc:430-537)   M rho = rhs_rho           CG
//   pressure_fixed_point (:544-673)  tmp_1 = A^{-1} rhs_u (CG, tol 1e-12 |rhs_u|),
//                                     rhs_p -= C tmp_1, (D - C A^{-1} B) p = rhs_p  GMRES
//   update_velocity     (:680-781)   A u = rhs_u - B p  (stage 3: explicit rhs)    CG
//   update_pressure     (:788-871)   D p = rhs_p                                   CG
//   fixed point         (:1135-1153) <= 100 iterations, |p - p_old|_inf/(|p|_inf+1e-10) < 1e-10
//
// Solver settings follow the reference: SolverControl(max_its, eps*|rhs|) for every outer
// solve, GMRES with deal.II's defaults (left preconditioning, restart after 28 directions,
// convergence on the preconditioned residual estimate) and the Jacobi preconditioner built
// from the Schur operator's diagonal (the diagonal of D, euler_operator.h:2607-2611).  The
// mass-type systems use CG with Jacobi instead of the reference's geometric multigrid: the
// systems and tolerances are the same, so the solutions agree to the solver tolerance.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <functional>
#include <string>
#include <vector>

#include "../../include/af_gpu.h"
#include "af_handle.h"

namespace af {
void set_last_error(const char* msg);
}
using namespace af;

struct af_imex {
  af_operator* op = nullptr;
  af_imex_options opt{};
  long ns = 0;
  double* mem = nullptr;
  // state and stage vectors
  double *rho0, *rho2, *rho3, *rhoc, *u0, *u2, *u3, *uc, *ufix, *p0, *p2, *p3, *pfix, *pfix_old;
  double *rhs_rho, *rhs_u, *rhs_p, *tmp1, *tmpu, *tmpp;
  // CG workspace and inverse diagonals
  double *cg_r, *cg_z, *cg_p, *cg_Ap, *invd_u, *invd_M, *invd_D;
  // GMRES workspace
  double *V, *gw, *d_h, *scal;
  double* part;
  KrylovState* kst;
  af_schur_solver* schur = nullptr;  // FGMRES + Jacobi/multigrid (schur_preconditioner >= 0)
  af_imex_stats stats{};
  // tangent / adjoint: the recorded fixed-point trajectories of stages 1 and 2 (pres_fixed and
  // u_fixed entering each iteration, and the final iterate), the linearisation point kind
  // (1: stage 1, 2: a whole step) and a workspace, allocated on first use
  int record = 0;  // bit s-1: record the fixed point of stage s
  int rec_iters[2] = {0, 0};
  std::vector<double*> rec_p[2], rec_u[2];
  int lin = 0;
  double* adj_mem = nullptr;
};

static int ierr(int code, const std::string& msg) {
  set_last_error(msg.c_str());
  return code;
}

#define IM_CU(call)                                                                                        \
  do {                                                                                                     \
    cudaError_t e_ = (call);                                                                               \
    if (e_ != cudaSuccess) return ierr(AF_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_));       \
  } while (0)
#define IM_AF(call)                      \
  do {                                   \
    int r_ = (call);                     \
    if (r_ != AF_OK) return r_;          \
  } while (0)

using Apply = std::function<int(const double*, double*)>;

// trajectory buffers of the tangent / adjoint, one pair per fixed-point iterate of stage k+1
static int ensure_rec(af_imex* h, int k, int i) {
  while ((int)h->rec_p[k].size() <= i) {
    double *p = nullptr, *u = nullptr;
    IM_CU(cudaMalloc(&p, h->ns * 8));
    if (cudaMalloc(&u, 2 * h->ns * 8) != cudaSuccess) {
      cudaFree(p);
      return ierr(AF_CUDA, "fixed-point trajectory: device allocation failed");
    }
    h->rec_p[k].push_back(p);
    h->rec_u[k].push_back(u);
  }
  return AF_OK;
}

// CG with Jacobi, x the initial guess, tolerance eps*|b| (deal.II SolverControl + SolverCG)
static int cg_solve(af_imex* h, const Apply& A, const double* invd, double* x, const double* b, long n, double eps,
                    int* its) {
  cudaStream_t st = h->op->stream;
  IM_AF(A(x, h->cg_Ap));
  IM_CU(dot(b, nullptr, n, h->part, h->scal, st));
  IM_CU(cg_set_abs_tol(h->kst, h->scal, eps, st));
  IM_CU(cg_start(h->kst, b, h->cg_Ap, invd, h->cg_r, h->cg_z, h->cg_p, n, h->part, 0.0, 0, st));
  h->op->launches += 6;
  KrylovState hs{};
  const int maxit = h->opt.max_iterations;
  for (int it = 0;; it += 8) {
    IM_CU(cudaMemcpyAsync(&hs, h->kst, sizeof(hs), cudaMemcpyDeviceToHost, st));
    IM_AF(sync_checked(h->op, st));
    if (hs.done || it >= maxit) break;
    for (int k = 0; k < 8; ++k) {
      IM_AF(A(h->cg_p, h->cg_Ap));
      IM_CU(cg_after_apply(h->kst, x, h->cg_r, h->cg_z, h->cg_p, h->cg_Ap, invd, n, h->part, maxit, st));
      h->op->launches += 5;
    }
  }
  if (its) *its = hs.its;
  h->stats.cg_iterations += hs.its;
  if (hs.status == 2 || hs.status == 3) return ierr(AF_NAN, "CG breakdown or NaN");
  if (!hs.done || hs.status == 1) return ierr(AF_NO_CONVERGENCE, "CG: no convergence within max_iterations");
  return AF_OK;
}

// GMRES with left Jacobi preconditioning (deal.II SolverGMRES defaults), |P^{-1} r| <= tol
static int gmres_solve(af_imex* h, const Apply& A, const double* invd, double* x, const double* b, long n, double tol,
                       int* its_out) {
  cudaStream_t st = h->op->stream;
  const int m = h->opt.gmres_restart;
  const long ld = krylov_stride(n);  // basis vectors start on 16-byte boundaries
  int total = 0;
  std::vector<double> H((m + 1) * m), cs(m), sn(m), g(m + 1), hh(2 * (m + 1));
  auto Hs = [&](int i, int j) -> double& { return H[i * m + j]; };
  double res = 0.0;
  bool converged = false;
  while (true) {
    IM_AF(A(x, h->gw));
    IM_CU(sub(b, h->gw, h->gw, n, st));
    IM_CU(dmul(invd, h->gw, h->gw, n, st));
    IM_CU(dot(h->gw, nullptr, n, h->part, h->scal, st));
    double beta2 = 0.0;
    IM_CU(cudaMemcpyAsync(&beta2, h->scal, sizeof(double), cudaMemcpyDeviceToHost, st));
    IM_AF(sync_checked(h->op, st));
    h->op->launches += 4;
    const double beta = std::sqrt(beta2);
    res = beta;
    if (!std::isfinite(beta)) return ierr(AF_NAN, "GMRES: NaN residual");
    if (beta <= tol) { converged = true; break; }
    if (total >= h->opt.max_iterations) break;
    IM_CU(scale(1.0 / beta, h->gw, h->V, n, st));
    std::fill(g.begin(), g.end(), 0.0);
    g[0] = beta;
    int jend = -1;
    for (int j = 0; j < m; ++j) {
      double* w = h->V + (long)(j + 1) * ld;
      IM_AF(A(h->V + (long)j * ld, w));
      IM_CU(dmul(invd, w, w, n, st));
      // classical Gram-Schmidt, twice
      IM_CU(mdot(h->V, ld, j + 1, w, n, h->part, h->d_h, st));
      IM_CU(maxpy(h->V, ld, j + 1, h->d_h, w, n, st));
      IM_CU(mdot(h->V, ld, j + 1, w, n, h->part, h->d_h + (m + 1), st));
      IM_CU(maxpy(h->V, ld, j + 1, h->d_h + (m + 1), w, n, st));
      IM_CU(dot(w, nullptr, n, h->part, h->scal, st));
      IM_CU(cudaMemcpyAsync(hh.data(), h->d_h, sizeof(double) * 2 * (m + 1), cudaMemcpyDeviceToHost, st));
      double hn2 = 0.0;
      IM_CU(cudaMemcpyAsync(&hn2, h->scal, sizeof(double), cudaMemcpyDeviceToHost, st));
      IM_AF(sync_checked(h->op, st));
      h->op->launches += 10;
      for (int i = 0; i <= j; ++i) Hs(i, j) = hh[i] + hh[(m + 1) + i];
      const double hn = std::sqrt(hn2);
      Hs(j + 1, j) = hn;
      if (hn > 0.0) IM_CU(scale(1.0 / hn, w, w, n, st));
      for (int i = 0; i < j; ++i) {  // previous rotations
        const double t = cs[i] * Hs(i, j) + sn[i] * Hs(i + 1, j);
        Hs(i + 1, j) = -sn[i] * Hs(i, j) + cs[i] * Hs(i + 1, j);
        Hs(i, j) = t;
      }
      const double a = Hs(j, j), c = Hs(j + 1, j);
      const double r = std::hypot(a, c);
      cs[j] = r > 0 ? a / r : 1.0;
      sn[j] = r > 0 ? c / r : 0.0;
      Hs(j, j) = r;
      Hs(j + 1, j) = 0.0;
      g[j + 1] = -sn[j] * g[j];
      g[j] = cs[j] * g[j];
      res = std::fabs(g[j + 1]);
      ++total;
      jend = j;
      if (!std::isfinite(res)) return ierr(AF_NAN, "GMRES: NaN in the Arnoldi process");
      if (res <= tol || total >= h->opt.max_iterations || hn == 0.0) break;
    }
    // x += V y with H y = g (upper triangular)
    const int k = jend + 1;
    std::vector<double> y(k);
    for (int i = k - 1; i >= 0; --i) {
      double s = g[i];
      for (int l = i + 1; l < k; ++l) s -= Hs(i, l) * y[l];
      y[i] = s / Hs(i, i);
    }
    IM_CU(mcombine(h->V, ld, k, y.data(), x, n, st));
    h->op->launches += 1;
    if (res <= tol) { converged = true; break; }
    if (total >= h->opt.max_iterations) break;
  }
  if (its_out) *its_out = total;
  h->stats.gmres_iterations += total;
  if (!converged) return ierr(AF_NO_CONVERGENCE, "GMRES: no convergence within max_iterations");
  return AF_OK;
}

static double l2norm(af_imex* h, const double* x, long n) {
  double v = 0.0;
  dot(x, nullptr, n, h->part, h->scal, h->op->stream);
  cudaMemcpyAsync(&v, h->scal, sizeof(double), cudaMemcpyDeviceToHost, h->op->stream);
  cudaStreamSynchronize(h->op->stream);
  return std::sqrt(v);
}

// Mass-type system of the current NS_stage: exact cell-wise inverse or CG + Jacobi to eps
static int mass_solve(af_imex* h, const double* invd, double* x, const double* b, long n, double eps) {
  af_operator* o = h->op;
  if (h->opt.mass_solver == 1) return af_vmult_inverse(o, x, b);
  Apply M = [o](const double* in, double* out) { return af_vmult(o, out, in); };
  return cg_solve(h, M, invd, x, b, n, eps, nullptr);
}

// ------------------------------------------------------------------ stage drivers
static int update_density(af_imex* h, int stage) {
  af_operator* o = h->op;
  const long ns = h->ns;
  IM_AF(af_set_HYPERBOLIC_stage(o, stage));
  IM_AF(af_set_NS_stage(o, stage == 3 ? 4 : 1));
  double* x;
  if (stage == 1) {
    const double* src[] = {h->rho0, h->u0};
    IM_AF(af_vmult_rhs_rho_update(o, h->rhs_rho, src, 2));
    x = h->rho2;
    IM_CU(cudaMemcpyAsync(x, h->rho0, ns * 8, cudaMemcpyDeviceToDevice, o->stream));
  } else if (stage == 2) {
    const double* src[] = {h->rho0, h->u0, h->rho2, h->u2};
    IM_AF(af_vmult_rhs_rho_update(o, h->rhs_rho, src, 4));
    x = h->rho3;
    IM_CU(cudaMemcpyAsync(x, h->rho2, ns * 8, cudaMemcpyDeviceToDevice, o->stream));
  } else {
    const double* src[] = {h->rho0, h->u0, h->rho2, h->u2, h->rho3, h->u3};
    IM_AF(af_vmult_rhs_rho_update(o, h->rhs_rho, src, 6));
    x = h->rhoc;
    IM_CU(cudaMemcpyAsync(x, h->rho3, ns * 8, cudaMemcpyDeviceToDevice, o->stream));
  }
  return mass_solve(h, h->invd_M, x, h->rhs_rho, ns, h->opt.eps);
}

static int pressure_fixed_point(af_imex* h, int stage, int iter) {
  af_operator* o = h->op;
  const long ns = h->ns;
  IM_AF(af_set_pres_fixed(o, h->pfix_old));
  IM_AF(af_set_u_fixed(o, h->ufix));
  // rhs_u and tmp_1 = A^{-1} rhs_u depend only on the stage's explicit fields and on A (the
  // stage's rho_for_fixed), not on pres_fixed or u_fixed: the reference forms them at every
  // fixed-point iteration (Atmospheric_Flow.cc:558-571), here at the first iteration of a stage
  // only (the same values; update_velocity leaves rhs_u as it is)
  if (stage == 1) {
    const double* sp[] = {h->rho0, h->u0, h->p0, h->rho2, h->ufix};
    IM_AF(af_vmult_rhs_pressure(o, h->rhs_p, sp, 5));
    const double* su[] = {h->rho0, h->u0, h->p0, h->rho2};
    if (iter == 0) IM_AF(af_vmult_rhs_velocity_fixed(o, h->rhs_u, su, 4));
  } else {
    const double* sp[] = {h->rho0, h->u0, h->p0, h->rho2, h->u2, h->p2, h->rho3, h->ufix};
    IM_AF(af_vmult_rhs_pressure(o, h->rhs_p, sp, 8));
    const double* su[] = {h->rho0, h->u0, h->p0, h->rho2, h->u2, h->p2, h->rho3};
    if (iter == 0) IM_AF(af_vmult_rhs_velocity_fixed(o, h->rhs_u, su, 7));
  }
  // tmp_1 = A^{-1} rhs_u, CG to 1e-12 |rhs_u| (Atmospheric_Flow.cc:571, 642); tmp_1 persists
  IM_AF(af_set_NS_stage(o, 3));
  if (iter == 0) IM_AF(mass_solve(h, h->invd_u, h->tmp1, h->rhs_u, 2 * ns, 1e-12));
  IM_AF(af_vmult_enthalpy(o, h->tmpp, h->tmp1));
  IM_CU(axpby(-1.0, h->tmpp, 1.0, h->rhs_p, ns, o->stream));
  o->launches += 1;
  // (D - C A^{-1} B) p = rhs_p by GMRES + Jacobi(diag D), x0 = pres_fixed_old
  IM_AF(af_set_NS_stage(o, 2));
  IM_CU(cudaMemcpyAsync(h->pfix, h->pfix_old, ns * 8, cudaMemcpyDeviceToDevice, o->stream));
  if (h->schur) {
    // FGMRES to eps |rhs_p| on the true residual; the preconditioner is rebuilt at the first
    // fixed-point iteration of each stage (rho_for_fixed changes there; pres_fixed changes
    // every iteration but only enters the preconditioner, which may lag)
    if (iter == 0) IM_AF(af_schur_solver_setup(h->schur, 0));
    af_schur_stats st{};
    const int r = af_schur_solve(h->schur, h->pfix, h->rhs_p, h->opt.eps, h->opt.max_iterations, &st);
    h->stats.gmres_iterations += st.iterations;
    return r;
  }
  Apply S = [o](const double* in, double* out) { return af_vmult(o, out, in); };
  const double tol = h->opt.eps * l2norm(h, h->rhs_p, ns);
  return gmres_solve(h, S, h->invd_D, h->pfix, h->rhs_p, ns, tol, nullptr);
}

static int update_velocity(af_imex* h, int stage) {
  af_operator* o = h->op;
  const long ns = h->ns;
  double *x, *b;
  if (stage < 3) {
    // b = rhs_u - B p, in tmpu (rhs_u is kept for the next fixed-point iteration)
    IM_AF(af_set_NS_stage(o, 3));
    IM_AF(af_vmult_pressure(o, h->tmpu, h->pfix));
    IM_CU(axpby(1.0, h->rhs_u, -1.0, h->tmpu, 2 * ns, o->stream));
    o->launches += 1;
    x = h->ufix;
    b = h->tmpu;
  } else {
    IM_AF(af_set_NS_stage(o, 5));
    const double* su[] = {h->rho0, h->u0, h->p0, h->rho2, h->u2, h->p2, h->rho3, h->u3, h->p3};
    IM_AF(af_vmult_rhs_velocity_fixed(o, h->rhs_u, su, 9));
    x = h->uc;
    b = h->rhs_u;
    IM_CU(cudaMemcpyAsync(x, h->u3, 2 * ns * 8, cudaMemcpyDeviceToDevice, o->stream));
  }
  return mass_solve(h, h->invd_u, x, b, 2 * ns, h->opt.eps);
}

static int update_pressure(af_imex* h) {
  af_operator* o = h->op;
  const long ns = h->ns;
  IM_AF(af_set_NS_stage(o, 6));
  const double* sp[] = {h->rho0, h->u0, h->p0, h->rho2, h->u2, h->p2, h->rho3, h->u3, h->p3, h->rhoc, h->uc};
  IM_AF(af_vmult_rhs_pressure(o, h->rhs_p, sp, 11));
  IM_CU(cudaMemcpyAsync(h->p0, h->p3, ns * 8, cudaMemcpyDeviceToDevice, o->stream));  // pres_old = pres_tmp_3
  return mass_solve(h, h->invd_D, h->p0, h->rhs_p, ns, h->opt.eps);
}

static int set_rho_for_fixed(af_imex* h, const double* rho) {
  af_operator* o = h->op;
  IM_AF(af_set_rho_for_fixed(o, rho));
  IM_AF(af_set_NS_stage(o, 3));
  return af_compute_diagonal(o, h->invd_u);
}

static int fixed_point(af_imex* h, int stage, double* p_out, double* u_out) {
  af_operator* o = h->op;
  const long ns = h->ns;
  int iters = 0;
  double err = 0.0;
  for (int iter = 0; iter < h->opt.fixed_point_max_iterations; ++iter) {
    if (h->record & (1 << (stage - 1))) {  // the iteration's inputs: pres_fixed and u_fixed
      const int k = stage - 1;
      IM_AF(ensure_rec(h, k, iter));
      IM_CU(cudaMemcpyAsync(h->rec_p[k][iter], h->pfix_old, ns * 8, cudaMemcpyDeviceToDevice, o->stream));
      IM_CU(cudaMemcpyAsync(h->rec_u[k][iter], h->ufix, 2 * ns * 8, cudaMemcpyDeviceToDevice, o->stream));
    }
    IM_AF(pressure_fixed_point(h, stage, iter));
    IM_AF(update_velocity(h, stage));
    ++iters;
    IM_CU(maxabs2(h->pfix, h->pfix_old, ns, h->part, h->scal, o->stream));
    double mm[2];
    IM_CU(cudaMemcpyAsync(mm, h->scal, sizeof(mm), cudaMemcpyDeviceToHost, o->stream));
    IM_AF(sync_checked(o, o->stream));
    o->launches += 2;
    err = mm[1] / (mm[0] + 1e-10);
    if (err < h->opt.fixed_point_tol) break;
    IM_CU(cudaMemcpyAsync(h->pfix_old, h->pfix, ns * 8, cudaMemcpyDeviceToDevice, o->stream));
  }
  h->stats.fixed_point_iterations[stage - 1] = iters;
  h->stats.last_fixed_point_error = err;
  if (h->record & (1 << (stage - 1))) {  // the final iterate
    const int k = stage - 1;
    IM_AF(ensure_rec(h, k, iters));
    IM_CU(cudaMemcpyAsync(h->rec_p[k][iters], h->pfix, ns * 8, cudaMemcpyDeviceToDevice, o->stream));
    IM_CU(cudaMemcpyAsync(h->rec_u[k][iters], h->ufix, 2 * ns * 8, cudaMemcpyDeviceToDevice, o->stream));
    h->rec_iters[k] = iters;
  }
  IM_CU(cudaMemcpyAsync(p_out, h->pfix, ns * 8, cudaMemcpyDeviceToDevice, o->stream));
  IM_CU(cudaMemcpyAsync(u_out, h->ufix, 2 * ns * 8, cudaMemcpyDeviceToDevice, o->stream));
  return AF_OK;
}

static int one_step(af_imex* h) {
  af_operator* o = h->op;
  const long ns = h->ns;
  // stage 1 (Atmospheric_Flow.cc:1116-1156)
  IM_AF(update_density(h, 1));
  IM_AF(set_rho_for_fixed(h, h->rho2));
  IM_CU(cudaMemcpyAsync(h->pfix_old, h->p0, ns * 8, cudaMemcpyDeviceToDevice, o->stream));
  IM_CU(cudaMemcpyAsync(h->ufix, h->u0, 2 * ns * 8, cudaMemcpyDeviceToDevice, o->stream));
  IM_AF(af_set_HYPERBOLIC_stage(o, 1));
  IM_AF(fixed_point(h, 1, h->p2, h->u2));
  // stage 2 (:1158-1197)
  IM_AF(update_density(h, 2));
  IM_AF(set_rho_for_fixed(h, h->rho3));
  IM_CU(cudaMemcpyAsync(h->pfix_old, h->p2, ns * 8, cudaMemcpyDeviceToDevice, o->stream));
  IM_CU(cudaMemcpyAsync(h->ufix, h->u2, 2 * ns * 8, cudaMemcpyDeviceToDevice, o->stream));
  IM_AF(af_set_HYPERBOLIC_stage(o, 2));
  IM_AF(fixed_point(h, 2, h->p3, h->u3));
  // stage 3 (:1200-1222)
  IM_AF(update_density(h, 3));
  IM_AF(set_rho_for_fixed(h, h->rhoc));
  IM_AF(af_set_HYPERBOLIC_stage(o, 3));
  IM_AF(update_velocity(h, 3));
  IM_AF(update_pressure(h));
  IM_CU(cudaMemcpyAsync(h->rho0, h->rhoc, ns * 8, cudaMemcpyDeviceToDevice, o->stream));
  IM_CU(cudaMemcpyAsync(h->u0, h->uc, 2 * ns * 8, cudaMemcpyDeviceToDevice, o->stream));
  return AF_OK;
}

// ------------------------------------------------------------------ tangent-linear and adjoint
// One IMEX step as a map (rho0, u0, p0) -> (rho_c, u_c, p_new), and stage 1 alone as
// (rho0, u0, p0) -> (rho2, u2, p2).  The tangent-linear and the adjoint differentiate the step
// as the forward ran it: the recorded fixed-point iterations of stages 1 and 2, each linear
// solve taken as exact (Schur solves to a given tolerance with the stepper's FGMRES and
// preconditioner; the cell-wise A, M, D inverses are exact).
//
// Fixed-point stage s (1 or 2), explicit fields E (rho_j, u_j, p_j of the earlier stages):
//   rho_{s+1} = M^{-1} R_rho(E);  with P_0 = p_s, U_0 = u_s the last explicit p, u and A = A(rho_{s+1}):
//   rhs_p, rhs_u = R(E, rho_{s+1}, U_i)                    (fused rhs triple of stage s)
//   t        = A^{-1} rhs_u;  b = rhs_p - C(t; P_i)
//   P_{i+1}  : S(P_i; P_{i+1}) = b,   S(p_f; p) = D p - C(A^{-1} B p; p_f)
//   U_{i+1}  = A^{-1} (rhs_u - B P_{i+1}).
// A is linear in rho and C in p_f, so their coefficient tangents are the operators with the
// perturbation as the coefficient; linearising the Schur solve:
//   J_S(P_{i+1}) dP = db - J_C(w) A^{-1} A(drho) w + C(w; dP_i),   w = A^{-1} B P_{i+1}.
// Stage 3 (explicit fields E of stages 1..3):  rho_c = M^{-1} R_rho(E),  u_c = A(rho_c)^{-1} R_u(E),
//   p_new = D^{-1} R_p(E, rho_c, u_c).

constexpr int kAdjVectors = 64;  // velocity-sized work vectors of the tangent / adjoint
constexpr int kSaved = 3;        // the first three hold the linearisation's input state

static int ensure_adj(af_imex* h) {
  if (h->adj_mem) return AF_OK;
  IM_CU(cudaMalloc(&h->adj_mem, sizeof(double) * 2 * h->ns * kAdjVectors));
  return AF_OK;
}
static double* saved(af_imex* h, int k) { return h->adj_mem + (size_t)k * 2 * h->ns; }

namespace {
struct Ctx {
  af_imex* h;
  af_operator* o;
  long ns;
  cudaStream_t st;
  int next = kSaved;
  // a velocity-sized work vector; past the pool's end it hands out the last one and the
  // caller's ws_ok() check fails before any of them is used
  double* take() {
    const int k = next < kAdjVectors ? next : kAdjVectors - 1;
    ++next;
    return h->adj_mem + (size_t)k * 2 * ns;
  }
  bool ws_ok() const { return next <= kAdjVectors; }
};
}  // namespace


static int ctx_init(af_imex* h, Ctx& c, int need_lin) {
  if (!h->schur) return ierr(AF_UNSUPPORTED, "tangent/adjoint: needs schur_preconditioner >= 0");
  if (h->lin < need_lin) return ierr(AF_BAD_ARG, "tangent/adjoint: run the recorded forward first");
  IM_AF(ensure_adj(h));
  c.h = h;
  c.o = h->op;
  c.ns = h->ns;
  c.st = h->op->stream;
  return AF_OK;
}
static CParams stage_cparams(const af_operator* o, int stage) {
  CParams cp;
  cp.cdt = (stage == 1 ? o->a22t : o->a33t) * o->dt;  // the B/C coefficient (euler_operator.h:1428)
  cp.g1 = 1.0 / (1.4 - 1.0);
  cp.gg = 1.4 / (1.4 - 1.0);
  return cp;
}
// the operator in the state of a stage: HYPERBOLIC_stage, rho_for_fixed, preconditioner
static int stage_setup(Ctx& c, int stage, const double* rho_fixed) {
  IM_AF(af_set_HYPERBOLIC_stage(c.o, stage));
  IM_AF(af_set_rho_for_fixed(c.o, rho_fixed));
  if (stage < 3) IM_AF(af_schur_solver_setup(c.h->schur, 0));
  return AF_OK;
}
// x = A^{-1} b (NS 3), M^{-1} b (NS 1) or D^{-1} b (NS 6), exact cell-wise inverses
static int ad_inv(Ctx& c, int ns_stage, double* x, const double* b) {
  IM_AF(af_set_NS_stage(c.o, ns_stage));
  return af_vmult_inverse(c.o, x, b);
}
// dst = A(rho) x  (rho-weighted velocity mass with an arbitrary weight)
static int ad_A(Ctx& c, const double* rho, const double* x, double* dst) {
  IM_CU(c.o->ops->mass(c.o->mesh, 2, x, rho, 1.0, dst, c.o->ncell, c.st));
  c.o->launches += 1;
  return AF_OK;
}
// dst = C(w; pf)  (vmult_enthalpy with an arbitrary pres_fixed)
static int ad_C(Ctx& c, int stage, const double* w, const double* pf, double* dst) {
  IM_CU(c.o->ops->op_C(c.o->mesh, w, pf, nullptr, stage_cparams(c.o, stage), dst, c.o->ncell, c.st));
  c.o->launches += 1;
  return AF_OK;
}
static int ad_axpby(Ctx& c, double a, const double* x, double b, double* y, long n) {
  IM_CU(axpby(a, x, b, y, n, c.st));
  c.o->launches += 1;
  return AF_OK;
}
static int ad_copy(Ctx& c, double* dst, const double* src, long n) {
  IM_CU(cudaMemcpyAsync(dst, src, n * 8, cudaMemcpyDeviceToDevice, c.st));
  return AF_OK;
}
static int ad_zero(Ctx& c, double* x, long n) {
  IM_CU(cudaMemsetAsync(x, 0, n * 8, c.st));
  return AF_OK;
}
static long comp_len(long ns, int k) { return (k % 3 == 1) ? 2 * ns : ns; }  // rho, u, p pattern

static void lin_fields(af_imex* h, const double** E) {
  E[0] = saved(h, 0); E[1] = saved(h, 1); E[2] = saved(h, 2);
  E[3] = h->rho2; E[4] = h->u2; E[5] = h->p2;
  E[6] = h->rho3; E[7] = h->u3; E[8] = h->p3;
}
static double* rho_next(af_imex* h, int s) { return s == 1 ? h->rho2 : h->rho3; }

// tangent of fixed-point stage s: dE (3 s explicit-field tangents) -> (drho_{s+1}, dU_I, dP_I)
static int fp_tangent(Ctx& c, int s, const double* const* dE, double* drho_out, double* du_out, double* dp_out,
                      double tol, int maxit) {
  af_imex* h = c.h;
  af_operator* o = c.o;
  const long ns = c.ns;
  const int k = s - 1, n = 3 * s + 2;
  const double* E[9];
  lin_fields(h, E);
  double* rn = rho_next(h, s);
  IM_AF(stage_setup(c, s, rn));
  const int mark = c.next;
  double *zs = c.take(), *zv = c.take(), *rhs_u = c.take(), *t = c.take(), *drr = c.take(), *drhs_u = c.take();
  double *drhs_p = c.take(), *tmpA = c.take(), *dt = c.take(), *jc = c.take(), *cc = c.take(), *db = c.take();
  double *Bp = c.take(), *w = c.take(), *aw = c.take(), *z = c.take(), *jz = c.take(), *cw = c.take();
  double *dP = c.take(), *dU = c.take(), *dPf = c.take(), *dUf = c.take(), *drho = c.take(), *bdp = c.take();
  if (!c.ws_ok()) return ierr(AF_BAD_ARG, "tangent: work vectors exhausted");
  IM_AF(ad_zero(c, zs, ns));
  IM_AF(ad_zero(c, zv, 2 * ns));
  const double* su[8];
  for (int j = 0; j < 3 * s; ++j) su[j] = E[j];
  su[3 * s] = rn;
  IM_AF(af_vmult_rhs_velocity_fixed(o, rhs_u, su, 3 * s + 1));
  IM_AF(ad_inv(c, 3, t, rhs_u));
  const double* src[11];
  const double* dsrc[11];
  for (int j = 0; j < 3 * s; ++j) { src[j] = E[j]; dsrc[j] = dE[j]; }
  src[3 * s] = rn;
  src[3 * s + 1] = h->rec_u[k][0];
  dsrc[3 * s] = zs;
  dsrc[3 * s + 1] = zv;
  IM_AF(af_vmult_rhs_fused_tangent(o, src, n, dsrc, drr, drhs_u, drhs_p));  // the density rhs
  IM_AF(ad_inv(c, 1, drho, drr));
  IM_AF(ad_copy(c, dPf, dE[3 * s - 1], ns));      // P_0 = p_s
  IM_AF(ad_copy(c, dUf, dE[3 * s - 2], 2 * ns));  // U_0 = u_s
  dsrc[3 * s] = drho;
  dsrc[3 * s + 1] = dUf;
  for (int i = 0; i < h->rec_iters[k]; ++i) {
    const double *Pi = h->rec_p[k][i], *Ui = h->rec_u[k][i], *Pn = h->rec_p[k][i + 1], *Un = h->rec_u[k][i + 1];
    src[3 * s + 1] = Ui;
    IM_AF(af_vmult_rhs_fused_tangent(o, src, n, dsrc, drr, drhs_u, drhs_p));
    // dt = A^{-1} (drhs_u - A(drho) t)
    IM_AF(ad_A(c, drho, t, tmpA));
    IM_AF(ad_axpby(c, 1.0, drhs_u, -1.0, tmpA, 2 * ns));
    IM_AF(ad_inv(c, 3, dt, tmpA));
    // db = drhs_p - J_C(t; P_i) dt - C(t; dP_i)
    IM_AF(af_set_pres_fixed(o, Pi));
    IM_AF(af_vmult_enthalpy_tangent(o, jc, t, dt));
    IM_AF(ad_C(c, s, t, dPf, cc));
    IM_AF(ad_copy(c, db, drhs_p, ns));
    IM_AF(ad_axpby(c, -1.0, jc, 1.0, db, ns));
    IM_AF(ad_axpby(c, -1.0, cc, 1.0, db, ns));
    // right-hand side of J_S(P_{i+1}) dP: db - J_C(w) A^{-1} A(drho) w + C(w; dP_i)
    IM_AF(af_vmult_pressure(o, Bp, Pn));
    IM_AF(ad_inv(c, 3, w, Bp));
    IM_AF(ad_A(c, drho, w, aw));
    IM_AF(ad_inv(c, 3, z, aw));
    IM_AF(af_vmult_enthalpy_tangent(o, jz, w, z));
    IM_AF(ad_C(c, s, w, dPf, cw));
    IM_AF(ad_axpby(c, -1.0, jz, 1.0, db, ns));
    IM_AF(ad_axpby(c, 1.0, cw, 1.0, db, ns));
    IM_AF(ad_zero(c, dP, ns));
    af_schur_stats sst{};
    IM_AF(af_schur_solve_tangent(h->schur, Pn, dP, db, tol, maxit, &sst));
    // dU = A^{-1} (drhs_u - B dP - A(drho) U_{i+1})
    IM_AF(af_vmult_pressure(o, bdp, dP));
    IM_AF(ad_A(c, drho, Un, tmpA));
    IM_AF(ad_axpby(c, 1.0, drhs_u, -1.0, tmpA, 2 * ns));
    IM_AF(ad_axpby(c, -1.0, bdp, 1.0, tmpA, 2 * ns));
    IM_AF(ad_inv(c, 3, dU, tmpA));
    IM_AF(ad_copy(c, dPf, dP, ns));
    IM_AF(ad_copy(c, dUf, dU, 2 * ns));
  }
  IM_AF(ad_copy(c, drho_out, drho, ns));
  IM_AF(ad_copy(c, du_out, dUf, 2 * ns));
  IM_AF(ad_copy(c, dp_out, dPf, ns));
  c.next = mark;
  return AF_OK;
}

// adjoint of fixed-point stage s: (rho_{s+1}, U_I, P_I) cotangents -> Ebar (3 s, accumulated)
static int fp_backward(Ctx& c, int s, const double* rho_bar, const double* u_bar, const double* p_bar,
                       double* const* Ebar, double tol, int maxit) {
  af_imex* h = c.h;
  af_operator* o = c.o;
  const long ns = c.ns;
  const int k = s - 1, n = 3 * s + 2;
  const double* E[9];
  lin_fields(h, E);
  double* rn = rho_next(h, s);
  IM_AF(stage_setup(c, s, rn));
  const int mark = c.next;
  double *zs = c.take(), *zv = c.take(), *rhs_u = c.take(), *t = c.take(), *R2 = c.take(), *Pb = c.take();
  double *Ub = c.take(), *rub = c.take(), *rpb = c.take(), *Pfb = c.take(), *s1 = c.take(), *tmp = c.take();
  double *x = c.take(), *Bp = c.take(), *w = c.take(), *jt = c.take(), *z = c.take(), *ts = c.take();
  double *dtb = c.take(), *rrb = c.take();
  double* xb[11];
  for (int j = 0; j < n; ++j) xb[j] = c.take();
  if (!c.ws_ok()) return ierr(AF_BAD_ARG, "adjoint: work vectors exhausted");
  IM_AF(ad_zero(c, zs, ns));
  IM_AF(ad_zero(c, zv, 2 * ns));
  IM_AF(ad_copy(c, R2, rho_bar, ns));
  IM_AF(ad_copy(c, Pb, p_bar, ns));
  IM_AF(ad_copy(c, Ub, u_bar, 2 * ns));
  const double* su[8];
  for (int j = 0; j < 3 * s; ++j) su[j] = E[j];
  su[3 * s] = rn;
  IM_AF(af_vmult_rhs_velocity_fixed(o, rhs_u, su, 3 * s + 1));
  IM_AF(ad_inv(c, 3, t, rhs_u));
  const double* src[11];
  for (int j = 0; j < 3 * s; ++j) src[j] = E[j];
  src[3 * s] = rn;
  for (int i = h->rec_iters[k] - 1; i >= 0; --i) {
    const double *Pi = h->rec_p[k][i], *Ui = h->rec_u[k][i], *Pn = h->rec_p[k][i + 1], *Un = h->rec_u[k][i + 1];
    IM_AF(af_set_pres_fixed(o, Pi));
    IM_AF(ad_zero(c, rpb, ns));
    IM_AF(ad_zero(c, Pfb, ns));
    // U_{i+1} = A^{-1} (rhs_u - B P_{i+1}):  s1 = A^{-1} Ub
    IM_AF(ad_inv(c, 3, s1, Ub));
    IM_AF(ad_copy(c, rub, s1, 2 * ns));
    IM_AF(af_vmult_pressure_transpose(o, tmp, s1));
    IM_AF(ad_axpby(c, -1.0, tmp, 1.0, Pb, ns));
    IM_AF(af_vmult_velocity_mass_rho_transpose(o, ts, Un, s1));
    IM_AF(ad_axpby(c, -1.0, ts, 1.0, R2, ns));
    // P_{i+1}: x = J_S(P_{i+1})^{-T} Pb is the cotangent of db
    IM_AF(ad_zero(c, x, ns));
    af_schur_stats sst{};
    IM_AF(af_schur_solve_transpose(h->schur, Pn, x, Pb, tol, maxit, &sst));
    IM_AF(af_vmult_pressure(o, Bp, Pn));
    IM_AF(ad_inv(c, 3, w, Bp));
    IM_AF(af_vmult_enthalpy_pf_transpose(o, ts, w, x));  // + C(w; dP_i)
    IM_AF(ad_axpby(c, 1.0, ts, 1.0, Pfb, ns));
    IM_AF(af_vmult_enthalpy_transpose(o, jt, w, x));     // - J_C(w) A^{-1} A(drho) w
    IM_AF(ad_inv(c, 3, z, jt));
    IM_AF(af_vmult_velocity_mass_rho_transpose(o, ts, w, z));
    IM_AF(ad_axpby(c, -1.0, ts, 1.0, R2, ns));
    // db = drhs_p - J_C(t) dt - C(t; dP_i)
    IM_AF(ad_axpby(c, 1.0, x, 1.0, rpb, ns));
    IM_AF(af_vmult_enthalpy_transpose(o, dtb, t, x));
    IM_AF(af_vmult_enthalpy_pf_transpose(o, ts, t, x));
    IM_AF(ad_axpby(c, -1.0, ts, 1.0, Pfb, ns));
    // dt = A^{-1} (drhs_u - A(drho) t), with the cotangent -J_C(t)^T x
    IM_AF(ad_inv(c, 3, s1, dtb));
    IM_AF(ad_axpby(c, -1.0, s1, 1.0, rub, 2 * ns));
    IM_AF(af_vmult_velocity_mass_rho_transpose(o, ts, t, s1));
    IM_AF(ad_axpby(c, 1.0, ts, 1.0, R2, ns));
    // the rhs triple at (E, rho_{s+1}, U_i)
    src[3 * s + 1] = Ui;
    IM_AF(af_vmult_rhs_fused_backward(o, src, n, zs, rub, rpb, xb));
    for (int j = 0; j < 3 * s; ++j) IM_AF(ad_axpby(c, 1.0, xb[j], 1.0, Ebar[j], comp_len(ns, j)));
    IM_AF(ad_axpby(c, 1.0, xb[3 * s], 1.0, R2, ns));
    // the iteration's inputs P_i, U_i: their cotangents go to the previous iterate
    IM_AF(ad_copy(c, Pb, Pfb, ns));
    IM_AF(ad_copy(c, Ub, xb[3 * s + 1], 2 * ns));
  }
  IM_AF(ad_axpby(c, 1.0, Pb, 1.0, Ebar[3 * s - 1], ns));      // P_0 = p_s
  IM_AF(ad_axpby(c, 1.0, Ub, 1.0, Ebar[3 * s - 2], 2 * ns));  // U_0 = u_s
  // rho_{s+1} = M^{-1} R_rho(E)
  IM_AF(ad_inv(c, 1, rrb, R2));
  src[3 * s + 1] = h->rec_u[k][0];
  IM_AF(af_vmult_rhs_fused_backward(o, src, n, rrb, zv, zs, xb));
  for (int j = 0; j < 3 * s; ++j) IM_AF(ad_axpby(c, 1.0, xb[j], 1.0, Ebar[j], comp_len(ns, j)));
  c.next = mark;
  return AF_OK;
}

// stage 3: dE (9 explicit-field tangents) -> (drho_c, du_c, dp_new)
static int s3_tangent(Ctx& c, const double* const* dE, double* drc, double* duc, double* dpn) {
  af_imex* h = c.h;
  af_operator* o = c.o;
  const long ns = c.ns;
  const double* E[9];
  lin_fields(h, E);
  IM_AF(stage_setup(c, 3, h->rhoc));
  const int mark = c.next;
  double *zs = c.take(), *zv = c.take(), *drr = c.take(), *dru = c.take(), *drp = c.take(), *tmpA = c.take();
  if (!c.ws_ok()) return ierr(AF_BAD_ARG, "tangent: work vectors exhausted");
  IM_AF(ad_zero(c, zs, ns));
  IM_AF(ad_zero(c, zv, 2 * ns));
  const double* src[11];
  const double* dsrc[11];
  for (int j = 0; j < 9; ++j) { src[j] = E[j]; dsrc[j] = dE[j]; }
  src[9] = h->rhoc;
  src[10] = h->uc;
  dsrc[9] = zs;
  dsrc[10] = zv;
  IM_AF(af_vmult_rhs_fused_tangent(o, src, 11, dsrc, drr, dru, drp));  // density and velocity rhs
  IM_AF(ad_inv(c, 1, drc, drr));
  IM_AF(ad_A(c, drc, h->uc, tmpA));  // du_c = A^{-1} (dR_u - A(drho_c) u_c)
  IM_AF(ad_axpby(c, 1.0, dru, -1.0, tmpA, 2 * ns));
  IM_AF(ad_inv(c, 3, duc, tmpA));
  dsrc[9] = drc;
  dsrc[10] = duc;
  IM_AF(af_vmult_rhs_fused_tangent(o, src, 11, dsrc, drr, dru, drp));  // the pressure rhs
  IM_AF(ad_inv(c, 6, dpn, drp));
  c.next = mark;
  return AF_OK;
}

// adjoint of stage 3: (rho_c, u_c, p_new) cotangents -> Ebar (9, accumulated)
static int s3_backward(Ctx& c, const double* rc_bar, const double* uc_bar, const double* pn_bar, double* const* Ebar) {
  af_imex* h = c.h;
  af_operator* o = c.o;
  const long ns = c.ns;
  const double* E[9];
  lin_fields(h, E);
  IM_AF(stage_setup(c, 3, h->rhoc));
  const int mark = c.next;
  double *zs = c.take(), *zv = c.take(), *rpb = c.take(), *Rc = c.take(), *Uc = c.take(), *s1 = c.take();
  double *rub = c.take(), *ts = c.take(), *rrb = c.take();
  double* xb[11];
  for (int j = 0; j < 11; ++j) xb[j] = c.take();
  if (!c.ws_ok()) return ierr(AF_BAD_ARG, "adjoint: work vectors exhausted");
  IM_AF(ad_zero(c, zs, ns));
  IM_AF(ad_zero(c, zv, 2 * ns));
  const double* src[11];
  for (int j = 0; j < 9; ++j) src[j] = E[j];
  src[9] = h->rhoc;
  src[10] = h->uc;
  IM_AF(ad_inv(c, 6, rpb, pn_bar));  // p_new = D^{-1} R_p (D symmetric)
  IM_AF(af_vmult_rhs_fused_backward(o, src, 11, zs, zv, rpb, xb));
  for (int j = 0; j < 9; ++j) IM_AF(ad_axpby(c, 1.0, xb[j], 1.0, Ebar[j], comp_len(ns, j)));
  IM_AF(ad_copy(c, Rc, rc_bar, ns));
  IM_AF(ad_axpby(c, 1.0, xb[9], 1.0, Rc, ns));
  IM_AF(ad_copy(c, Uc, uc_bar, 2 * ns));
  IM_AF(ad_axpby(c, 1.0, xb[10], 1.0, Uc, 2 * ns));
  IM_AF(ad_inv(c, 3, s1, Uc));  // u_c = A(rho_c)^{-1} R_u
  IM_AF(ad_copy(c, rub, s1, 2 * ns));
  IM_AF(af_vmult_velocity_mass_rho_transpose(o, ts, h->uc, s1));
  IM_AF(ad_axpby(c, -1.0, ts, 1.0, Rc, ns));
  IM_AF(ad_inv(c, 1, rrb, Rc));  // rho_c = M^{-1} R_rho
  IM_AF(af_vmult_rhs_fused_backward(o, src, 11, rrb, rub, zs, xb));
  for (int j = 0; j < 9; ++j) IM_AF(ad_axpby(c, 1.0, xb[j], 1.0, Ebar[j], comp_len(ns, j)));
  c.next = mark;
  return AF_OK;
}

static int step_tangent(af_imex* h, const double* const* dx, double* const* dy, double tol, int maxit) {
  Ctx c;
  IM_AF(ctx_init(h, c, 2));
  const double* dE[9] = {dx[0], dx[1], dx[2]};
  double* t[6];
  for (int j = 0; j < 6; ++j) t[j] = c.take();
  IM_AF(fp_tangent(c, 1, dE, t[0], t[1], t[2], tol, maxit));
  dE[3] = t[0]; dE[4] = t[1]; dE[5] = t[2];
  IM_AF(fp_tangent(c, 2, dE, t[3], t[4], t[5], tol, maxit));
  dE[6] = t[3]; dE[7] = t[4]; dE[8] = t[5];
  IM_AF(s3_tangent(c, dE, dy[0], dy[1], dy[2]));
  IM_AF(sync_checked(c.o, c.st));
  return AF_OK;
}

static int step_backward(af_imex* h, const double* const* ybar, double* const* xbar, double tol, int maxit) {
  Ctx c;
  IM_AF(ctx_init(h, c, 2));
  double* Eb[9];
  for (int j = 0; j < 9; ++j) {
    Eb[j] = c.take();
    IM_AF(ad_zero(c, Eb[j], comp_len(c.ns, j)));
  }
  IM_AF(s3_backward(c, ybar[0], ybar[1], ybar[2], Eb));
  IM_AF(fp_backward(c, 2, Eb[6], Eb[7], Eb[8], Eb, tol, maxit));
  IM_AF(fp_backward(c, 1, Eb[3], Eb[4], Eb[5], Eb, tol, maxit));
  for (int j = 0; j < 3; ++j) IM_AF(ad_copy(c, xbar[j], Eb[j], comp_len(c.ns, j)));
  IM_AF(sync_checked(c.o, c.st));
  return AF_OK;
}

static int s1_tangent(af_imex* h, const double* const* dx, double* const* dy, double tol, int maxit) {
  Ctx c;
  IM_AF(ctx_init(h, c, 1));
  IM_AF(fp_tangent(c, 1, dx, dy[0], dy[1], dy[2], tol, maxit));
  IM_AF(sync_checked(c.o, c.st));
  return AF_OK;
}

static int s1_backward(af_imex* h, const double* const* ybar, double* const* xbar, double tol, int maxit) {
  Ctx c;
  IM_AF(ctx_init(h, c, 1));
  for (int j = 0; j < 3; ++j) IM_AF(ad_zero(c, xbar[j], comp_len(c.ns, j)));
  IM_AF(fp_backward(c, 1, ybar[0], ybar[1], ybar[2], xbar, tol, maxit));
  IM_AF(sync_checked(c.o, c.st));
  return AF_OK;
}

// the recorded forward: stage 1 (stages = 1) or a whole step (stages = 3) from (rho0, u0, p0)
static int recorded_forward(af_imex* h, const double* rho0, const double* u0, const double* p0, int stages) {
  af_operator* o = h->op;
  const long ns = h->ns;
  h->lin = 0;
  IM_AF(ensure_adj(h));
  // the linearisation's input state (rho0, u0, p0 may alias the saved copies)
  if (rho0 != saved(h, 0)) IM_CU(cudaMemcpyAsync(saved(h, 0), rho0, ns * 8, cudaMemcpyDeviceToDevice, o->stream));
  if (u0 != saved(h, 1)) IM_CU(cudaMemcpyAsync(saved(h, 1), u0, 2 * ns * 8, cudaMemcpyDeviceToDevice, o->stream));
  if (p0 != saved(h, 2)) IM_CU(cudaMemcpyAsync(saved(h, 2), p0, ns * 8, cudaMemcpyDeviceToDevice, o->stream));
  IM_CU(cudaMemcpyAsync(h->rho0, saved(h, 0), ns * 8, cudaMemcpyDeviceToDevice, o->stream));
  IM_CU(cudaMemcpyAsync(h->u0, saved(h, 1), 2 * ns * 8, cudaMemcpyDeviceToDevice, o->stream));
  IM_CU(cudaMemcpyAsync(h->p0, saved(h, 2), ns * 8, cudaMemcpyDeviceToDevice, o->stream));
  h->stats = af_imex_stats{};
  int r = AF_OK;
  if (stages == 1) {  // stage 1 of one_step
    h->record = 1;
    r = update_density(h, 1);
    if (r == AF_OK) r = set_rho_for_fixed(h, h->rho2);
    if (r == AF_OK && cudaMemcpyAsync(h->pfix_old, h->p0, ns * 8, cudaMemcpyDeviceToDevice, o->stream) != cudaSuccess)
      r = ierr(AF_CUDA, "copy failed");
    if (r == AF_OK && cudaMemcpyAsync(h->ufix, h->u0, 2 * ns * 8, cudaMemcpyDeviceToDevice, o->stream) != cudaSuccess)
      r = ierr(AF_CUDA, "copy failed");
    if (r == AF_OK) r = af_set_HYPERBOLIC_stage(o, 1);
    if (r == AF_OK) r = fixed_point(h, 1, h->p2, h->u2);
  } else {
    h->record = 3;
    r = one_step(h);
  }
  h->record = 0;
  IM_AF(r);
  h->lin = stages == 1 ? 1 : 2;
  return AF_OK;
}
extern "C" {

int af_imex_default_options(af_imex_options* opt) {
  if (!opt) return ierr(AF_BAD_ARG, "null options");
  opt->eps = 1e-8;                    // parameter-file.prm:28
  opt->max_iterations = 30000;        // parameter-file.prm:27
  opt->fixed_point_tol = 1e-10;       // Atmospheric_Flow.cc:1149
  opt->fixed_point_max_iterations = 100;  // :1135
  opt->gmres_restart = 28;            // deal.II SolverGMRES default (30 temporary vectors)
  opt->mass_solver = 1;
  opt->schur_inner = 1;
  opt->schur_preconditioner = -1;
  opt->schur_poly_degree = 0;
  return AF_OK;
}

int af_imex_create(const af_mesh_desc* mesh, int degree, double Ma, double Fr, double dt, const af_imex_options* opt,
                   af_imex** out) {
  if (!out) return ierr(AF_BAD_ARG, "null output");
  *out = nullptr;
  af_imex_options o{};
  af_imex_default_options(&o);
  if (opt) o = *opt;
  if (!(o.eps > 0) || o.max_iterations < 1 || o.gmres_restart < 1 || o.gmres_restart > 60 ||
      o.fixed_point_max_iterations < 1 || o.mass_solver < 0 || o.mass_solver > 1 || o.schur_inner < 0 ||
      o.schur_inner > 1 || o.schur_preconditioner < -1 || o.schur_preconditioner > AF_SCHUR_CHEB_FP32 ||
      o.schur_poly_degree < 0)
    return ierr(AF_BAD_ARG, "af_imex_create: bad options");
  auto* h = new af_imex();
  h->opt = o;
  int r = af_create(mesh, degree, 2 * degree + 1, Ma, Fr, dt, &h->op);
  if (r != AF_OK) { delete h; return r; }
  const long ns = h->op->n_scalar();
  h->ns = ns;
  const int m = o.gmres_restart;
  // scalar vectors: rho0 rho2 rho3 rhoc p0 p2 p3 pfix pfix_old rhs_rho rhs_p tmpp invd_M invd_D gw = 15
  // velocity vectors (2 ns): u0 u2 u3 uc ufix rhs_u tmp1 tmpu cg_r cg_z cg_p cg_Ap invd_u = 13
  r = AF_OK;
  const long total = 15 * (ns + 1) + 13 * 2 * ns + (long)(m + 1) * krylov_stride(ns) + 2 * (m + 1) + 8 +
                     4 * kMaxPartials + 16;
  if (cudaMalloc(&h->mem, total * sizeof(double)) != cudaSuccess) {
    af_destroy(h->op);
    delete h;
    return ierr(AF_CUDA, "af_imex_create: device allocation failed");
  }
  if (cudaMemsetAsync(h->mem, 0, total * sizeof(double), h->op->stream) != cudaSuccess) {
    af_imex_destroy(h);
    return ierr(AF_CUDA, "af_imex_create: memset failed");
  }
  double* c = h->mem;
  auto take = [&](long n) { double* p = c; c += (n + 1) & ~1L; return p; };
  h->rho0 = take(ns); h->rho2 = take(ns); h->rho3 = take(ns); h->rhoc = take(ns);
  h->p0 = take(ns); h->p2 = take(ns); h->p3 = take(ns); h->pfix = take(ns); h->pfix_old = take(ns);
  h->rhs_rho = take(ns); h->rhs_p = take(ns); h->tmpp = take(ns); h->invd_M = take(ns); h->invd_D = take(ns);
  h->gw = take(ns);
  h->u0 = take(2 * ns); h->u2 = take(2 * ns); h->u3 = take(2 * ns); h->uc = take(2 * ns); h->ufix = take(2 * ns);
  h->rhs_u = take(2 * ns); h->tmp1 = take(2 * ns); h->tmpu = take(2 * ns);
  h->cg_r = take(2 * ns); h->cg_z = take(2 * ns); h->cg_p = take(2 * ns); h->cg_Ap = take(2 * ns);
  h->invd_u = take(2 * ns);
  h->V = take((long)(m + 1) * krylov_stride(ns));
  h->d_h = take(2 * (m + 1));
  h->scal = take(8);
  h->part = take(4 * kMaxPartials);
  h->kst = reinterpret_cast<KrylovState*>(take(16));
  r = af_set_schur_mode(h->op, o.schur_inner, 1e-12, 10000);
  // fixed inverse diagonals of M and D (compute_diagonal, NS 1 and NS 2/6)
  if (r == AF_OK) r = af_set_NS_stage(h->op, 1);
  if (r == AF_OK) r = af_compute_diagonal(h->op, h->invd_M);
  if (r == AF_OK) { af_set_NS_stage(h->op, 6); r = af_compute_diagonal(h->op, h->invd_D); }
  if (r == AF_OK && o.schur_preconditioner >= 0) {
    af_schur_options so{};
    af_schur_default_options(&so);
    so.preconditioner = o.schur_preconditioner;
    so.restart = o.gmres_restart;
    // degree 20 measured best over the periodic hill steps at 512x256 (dt 0.5 s) and 1024x256
    // (dt 0.25 s), eps 1e-8 and 1e-10, degrees 8..24: 2.4 % less time in sum than degree 12,
    // 4 % and 8 % at 512x256, within 2 % either way at 1024x256
    so.poly_degree = o.schur_poly_degree > 0 ? o.schur_poly_degree : 20;
    r = af_schur_solver_create(h->op, &so, &h->schur);
  }
  if (r == AF_OK) r = af_synchronize(h->op);
  if (r != AF_OK) { af_imex_destroy(h); return r; }
  *out = h;
  return AF_OK;
}

int af_imex_destroy(af_imex* h) {
  if (!h) return AF_OK;
  if (h->op) af_synchronize(h->op);
  af_schur_solver_destroy(h->schur);
  cudaFree(h->mem);
  cudaFree(h->adj_mem);
  for (int k = 0; k < 2; ++k) {
    for (double* p : h->rec_p[k]) cudaFree(p);
    for (double* u : h->rec_u[k]) cudaFree(u);
  }
  af_destroy(h->op);
  delete h;
  return AF_OK;
}

af_operator* af_imex_operator(af_imex* h) { return h ? h->op : nullptr; }

int af_imex_set_state(af_imex* h, const double* rho, const double* u, const double* p) {
  if (!h || !rho || !u || !p) return ierr(AF_BAD_ARG, "null argument");
  cudaStream_t st = h->op->stream;
  h->lin = 0;  // the recorded linearisation point is gone
  IM_CU(cudaMemcpyAsync(h->rho0, rho, h->ns * 8, cudaMemcpyDeviceToDevice, st));
  IM_CU(cudaMemcpyAsync(h->u0, u, 2 * h->ns * 8, cudaMemcpyDeviceToDevice, st));
  IM_CU(cudaMemcpyAsync(h->p0, p, h->ns * 8, cudaMemcpyDeviceToDevice, st));
  IM_AF(sync_checked(h->op, st));
  return AF_OK;
}

int af_imex_get_state(const af_imex* h, double* rho, double* u, double* p) {
  if (!h || !rho || !u || !p) return ierr(AF_BAD_ARG, "null argument");
  cudaStream_t st = h->op->stream;
  IM_CU(cudaMemcpyAsync(rho, h->rho0, h->ns * 8, cudaMemcpyDeviceToDevice, st));
  IM_CU(cudaMemcpyAsync(u, h->u0, 2 * h->ns * 8, cudaMemcpyDeviceToDevice, st));
  IM_CU(cudaMemcpyAsync(p, h->p0, h->ns * 8, cudaMemcpyDeviceToDevice, st));
  IM_AF(sync_checked(h->op, st));
  return AF_OK;
}

int af_imex_step(af_imex* h, int nsteps) {
  if (!h || nsteps < 0) return ierr(AF_BAD_ARG, "bad argument");
  IM_CU(cudaSetDevice(h->op->device));
  h->lin = 0;  // the recorded linearisation point is gone
  for (int s = 0; s < nsteps; ++s) {
    h->stats = af_imex_stats{};
    IM_AF(one_step(h));
  }
  return af_synchronize(h->op);
}

int af_imex_stage1_forward(af_imex* h, const double* rho0, const double* u0, const double* p0, double* rho2, double* u2,
                           double* p2) {
  if (!h || !rho0 || !u0 || !p0 || !rho2 || !u2 || !p2) return ierr(AF_BAD_ARG, "null argument");
  if (!h->schur) return ierr(AF_UNSUPPORTED, "af_imex_stage1_forward: needs schur_preconditioner >= 0");
  IM_CU(cudaSetDevice(h->op->device));
  IM_AF(recorded_forward(h, rho0, u0, p0, 1));
  cudaStream_t st = h->op->stream;
  IM_CU(cudaMemcpyAsync(rho2, h->rho2, h->ns * 8, cudaMemcpyDeviceToDevice, st));
  IM_CU(cudaMemcpyAsync(u2, h->u2, 2 * h->ns * 8, cudaMemcpyDeviceToDevice, st));
  IM_CU(cudaMemcpyAsync(p2, h->p2, h->ns * 8, cudaMemcpyDeviceToDevice, st));
  IM_AF(sync_checked(h->op, st));
  return AF_OK;
}

int af_imex_stage1_tangent(af_imex* h, const double* drho0, const double* du0, const double* dp0, double* drho2,
                           double* du2, double* dp2, double rel_tol) {
  if (!h || !drho0 || !du0 || !dp0 || !drho2 || !du2 || !dp2) return ierr(AF_BAD_ARG, "null argument");
  if (!(rel_tol > 0.0)) return ierr(AF_BAD_ARG, "af_imex_stage1_tangent: invalid tolerance");
  IM_CU(cudaSetDevice(h->op->device));
  const double* dx[3] = {drho0, du0, dp0};
  double* dy[3] = {drho2, du2, dp2};
  return s1_tangent(h, dx, dy, rel_tol, h->opt.max_iterations);
}

int af_imex_stage1_backward(af_imex* h, const double* rho2bar, const double* u2bar, const double* p2bar,
                            double* rho0bar, double* u0bar, double* p0bar, double rel_tol) {
  if (!h || !rho2bar || !u2bar || !p2bar || !rho0bar || !u0bar || !p0bar) return ierr(AF_BAD_ARG, "null argument");
  if (!(rel_tol > 0.0)) return ierr(AF_BAD_ARG, "af_imex_stage1_backward: invalid tolerance");
  IM_CU(cudaSetDevice(h->op->device));
  const double* yb[3] = {rho2bar, u2bar, p2bar};
  double* xb[3] = {rho0bar, u0bar, p0bar};
  return s1_backward(h, yb, xb, rel_tol, h->opt.max_iterations);
}

int af_imex_step_forward(af_imex* h, const double* rho0, const double* u0, const double* p0, double* rho1, double* u1,
                         double* p1) {
  if (!h || !rho0 || !u0 || !p0 || !rho1 || !u1 || !p1) return ierr(AF_BAD_ARG, "null argument");
  if (!h->schur) return ierr(AF_UNSUPPORTED, "af_imex_step_forward: needs schur_preconditioner >= 0");
  IM_CU(cudaSetDevice(h->op->device));
  IM_AF(recorded_forward(h, rho0, u0, p0, 3));
  IM_AF(af_imex_get_state(h, rho1, u1, p1));
  return AF_OK;
}

int af_imex_step_tangent(af_imex* h, const double* drho0, const double* du0, const double* dp0, double* drho1,
                         double* du1, double* dp1, double rel_tol) {
  if (!h || !drho0 || !du0 || !dp0 || !drho1 || !du1 || !dp1) return ierr(AF_BAD_ARG, "null argument");
  if (!(rel_tol > 0.0)) return ierr(AF_BAD_ARG, "af_imex_step_tangent: invalid tolerance");
  IM_CU(cudaSetDevice(h->op->device));
  const double* dx[3] = {drho0, du0, dp0};
  double* dy[3] = {drho1, du1, dp1};
  return step_tangent(h, dx, dy, rel_tol, h->opt.max_iterations);
}

int af_imex_step_backward(af_imex* h, const double* rho1bar, const double* u1bar, const double* p1bar,
                          double* rho0bar, double* u0bar, double* p0bar, double rel_tol) {
  if (!h || !rho1bar || !u1bar || !p1bar || !rho0bar || !u0bar || !p0bar) return ierr(AF_BAD_ARG, "null argument");
  if (!(rel_tol > 0.0)) return ierr(AF_BAD_ARG, "af_imex_step_backward: invalid tolerance");
  IM_CU(cudaSetDevice(h->op->device));
  const double* yb[3] = {rho1bar, u1bar, p1bar};
  double* xb[3] = {rho0bar, u0bar, p0bar};
  return step_backward(h, yb, xb, rel_tol, h->opt.max_iterations);
}

int af_imex_gradient(af_imex* h, const double* rho0, const double* u0, const double* p0, int nsteps,
                     int checkpoint_every, const double* rhobar, const double* ubar, const double* pbar,
                     double* rho0bar, double* u0bar, double* p0bar, double rel_tol) {
  if (!h || !rho0 || !u0 || !p0 || !rhobar || !ubar || !pbar || !rho0bar || !u0bar || !p0bar)
    return ierr(AF_BAD_ARG, "null argument");
  if (nsteps < 1 || checkpoint_every < 1 || !(rel_tol > 0.0)) return ierr(AF_BAD_ARG, "af_imex_gradient: bad argument");
  if (!h->schur) return ierr(AF_UNSUPPORTED, "af_imex_gradient: needs schur_preconditioner >= 0");
  IM_CU(cudaSetDevice(h->op->device));
  af_operator* o = h->op;
  cudaStream_t st = o->stream;
  // one state: rho, u (2), p, each part starting on a 16-byte boundary
  const long ns = h->ns, sp = krylov_stride(ns), S = 4 * sp;
  const int K = checkpoint_every, nck = (nsteps + K - 1) / K;
  double* mem = nullptr;
  // checkpoints, the states of one segment, and the running cotangent (+ a copy)
  IM_CU(cudaMalloc(&mem, sizeof(double) * S * ((size_t)nck + K + 2)));
  double* ck = mem;
  double* seg = ck + (size_t)S * nck;
  double* bar = seg + (size_t)S * K;
  double* bar2 = bar + S;
  auto R = [](double* b) { return b; };
  auto U = [sp](double* b) { return b + sp; };
  auto Pp = [sp](double* b) { return b + 3 * sp; };
  int r = AF_OK;
  auto copy = [&](double* d, const double* s_, long n) {
    if (r == AF_OK && cudaMemcpyAsync(d, s_, n * 8, cudaMemcpyDeviceToDevice, st) != cudaSuccess)
      r = ierr(AF_CUDA, "af_imex_gradient: copy failed");
  };
  auto save_state = [&](double* b) {
    if (r == AF_OK) r = af_imex_get_state(h, R(b), U(b), Pp(b));
  };
  // forward sweep, one checkpoint every K steps
  r = af_imex_set_state(h, rho0, u0, p0);
  for (int n = 0; n < nsteps && r == AF_OK; ++n) {
    if (n % K == 0) save_state(ck + (size_t)S * (n / K));
    if (r == AF_OK) r = one_step(h);
  }
  copy(R(bar), rhobar, ns);
  copy(U(bar), ubar, 2 * ns);
  copy(Pp(bar), pbar, ns);
  // reverse sweep: recompute each segment's states from its checkpoint, then adjoint steps
  for (int c = nck - 1; c >= 0 && r == AF_OK; --c) {
    const int beg = c * K, end = std::min(nsteps, beg + K);
    double* x = ck + (size_t)S * c;
    r = af_imex_set_state(h, R(x), U(x), Pp(x));
    for (int n = beg; n < end && r == AF_OK; ++n) {
      save_state(seg + (size_t)S * (n - beg));
      if (r == AF_OK && n + 1 < end) r = one_step(h);
    }
    for (int n = end - 1; n >= beg && r == AF_OK; --n) {
      double* xs = seg + (size_t)S * (n - beg);
      r = recorded_forward(h, R(xs), U(xs), Pp(xs), 3);
      if (r != AF_OK) break;
      const double* yb[3] = {R(bar), U(bar), Pp(bar)};
      double* xb[3] = {R(bar2), U(bar2), Pp(bar2)};
      r = step_backward(h, yb, xb, rel_tol, h->opt.max_iterations);
      std::swap(bar, bar2);
    }
  }
  copy(rho0bar, R(bar), ns);
  copy(u0bar, U(bar), 2 * ns);
  copy(p0bar, Pp(bar), ns);
  if (r == AF_OK) r = sync_checked(o, st);
  else cudaStreamSynchronize(st);
  cudaFree(mem);
  return r;
}

int af_imex_last_stats(const af_imex* h, af_imex_stats* out) {
  if (!h || !out) return ierr(AF_BAD_ARG, "null argument");
  *out = h->stats;
  return AF_OK;
}

}  // extern "C"
