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
    IM_CU(cudaStreamSynchronize(st));
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
    IM_CU(cudaStreamSynchronize(st));
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
      double* w = h->V + (long)(j + 1) * n;
      IM_AF(A(h->V + (long)j * n, w));
      IM_CU(dmul(invd, w, w, n, st));
      // classical Gram-Schmidt, twice
      IM_CU(mdot(h->V, n, j + 1, w, n, h->part, h->d_h, st));
      IM_CU(maxpy(h->V, n, j + 1, h->d_h, w, n, st));
      IM_CU(mdot(h->V, n, j + 1, w, n, h->part, h->d_h + (m + 1), st));
      IM_CU(maxpy(h->V, n, j + 1, h->d_h + (m + 1), w, n, st));
      IM_CU(dot(w, nullptr, n, h->part, h->scal, st));
      IM_CU(cudaMemcpyAsync(hh.data(), h->d_h, sizeof(double) * 2 * (m + 1), cudaMemcpyDeviceToHost, st));
      double hn2 = 0.0;
      IM_CU(cudaMemcpyAsync(&hn2, h->scal, sizeof(double), cudaMemcpyDeviceToHost, st));
      IM_CU(cudaStreamSynchronize(st));
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
    IM_CU(mcombine(h->V, n, k, y.data(), x, n, st));
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
  if (stage == 1) {
    const double* sp[] = {h->rho0, h->u0, h->p0, h->rho2, h->ufix};
    IM_AF(af_vmult_rhs_pressure(o, h->rhs_p, sp, 5));
    const double* su[] = {h->rho0, h->u0, h->p0, h->rho2};
    IM_AF(af_vmult_rhs_velocity_fixed(o, h->rhs_u, su, 4));
  } else {
    const double* sp[] = {h->rho0, h->u0, h->p0, h->rho2, h->u2, h->p2, h->rho3, h->ufix};
    IM_AF(af_vmult_rhs_pressure(o, h->rhs_p, sp, 8));
    const double* su[] = {h->rho0, h->u0, h->p0, h->rho2, h->u2, h->p2, h->rho3};
    IM_AF(af_vmult_rhs_velocity_fixed(o, h->rhs_u, su, 7));
  }
  // tmp_1 = A^{-1} rhs_u, CG to 1e-12 |rhs_u| (Atmospheric_Flow.cc:571, 642); tmp_1 persists
  IM_AF(af_set_NS_stage(o, 3));
  IM_AF(mass_solve(h, h->invd_u, h->tmp1, h->rhs_u, 2 * ns, 1e-12));
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
  double* x;
  if (stage < 3) {
    IM_AF(af_set_NS_stage(o, 3));
    IM_AF(af_vmult_pressure(o, h->tmpu, h->pfix));
    IM_CU(axpby(-1.0, h->tmpu, 1.0, h->rhs_u, 2 * ns, o->stream));
    o->launches += 1;
    x = h->ufix;
  } else {
    IM_AF(af_set_NS_stage(o, 5));
    const double* su[] = {h->rho0, h->u0, h->p0, h->rho2, h->u2, h->p2, h->rho3, h->u3, h->p3};
    IM_AF(af_vmult_rhs_velocity_fixed(o, h->rhs_u, su, 9));
    x = h->uc;
    IM_CU(cudaMemcpyAsync(x, h->u3, 2 * ns * 8, cudaMemcpyDeviceToDevice, o->stream));
  }
  return mass_solve(h, h->invd_u, x, h->rhs_u, 2 * ns, h->opt.eps);
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
    IM_AF(pressure_fixed_point(h, stage, iter));
    IM_AF(update_velocity(h, stage));
    ++iters;
    IM_CU(maxabs2(h->pfix, h->pfix_old, ns, h->part, h->scal, o->stream));
    double mm[2];
    IM_CU(cudaMemcpyAsync(mm, h->scal, sizeof(mm), cudaMemcpyDeviceToHost, o->stream));
    IM_CU(cudaStreamSynchronize(o->stream));
    o->launches += 2;
    err = mm[1] / (mm[0] + 1e-10);
    if (err < h->opt.fixed_point_tol) break;
    IM_CU(cudaMemcpyAsync(h->pfix_old, h->pfix, ns * 8, cudaMemcpyDeviceToDevice, o->stream));
  }
  h->stats.fixed_point_iterations[stage - 1] = iters;
  h->stats.last_fixed_point_error = err;
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
  const long total = 15 * ns + 13 * 2 * ns + (long)(m + 1) * ns + 2 * (m + 1) + 8 + 4 * kMaxPartials + 16;
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
  h->V = take((long)(m + 1) * ns);
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
    // inside the time loop each solve starts from the previous iterate: a lower degree than
    // the stand-alone default measured best (512x256 and 1024x256, degrees 4..16; 10 and 12
    // tie at 512x256, 12 is 6 % faster at 1024x256)
    so.poly_degree = o.schur_poly_degree > 0 ? o.schur_poly_degree : 12;
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
  af_destroy(h->op);
  delete h;
  return AF_OK;
}

af_operator* af_imex_operator(af_imex* h) { return h ? h->op : nullptr; }

int af_imex_set_state(af_imex* h, const double* rho, const double* u, const double* p) {
  if (!h || !rho || !u || !p) return ierr(AF_BAD_ARG, "null argument");
  cudaStream_t st = h->op->stream;
  IM_CU(cudaMemcpyAsync(h->rho0, rho, h->ns * 8, cudaMemcpyDeviceToDevice, st));
  IM_CU(cudaMemcpyAsync(h->u0, u, 2 * h->ns * 8, cudaMemcpyDeviceToDevice, st));
  IM_CU(cudaMemcpyAsync(h->p0, p, h->ns * 8, cudaMemcpyDeviceToDevice, st));
  IM_CU(cudaStreamSynchronize(st));
  return AF_OK;
}

int af_imex_get_state(const af_imex* h, double* rho, double* u, double* p) {
  if (!h || !rho || !u || !p) return ierr(AF_BAD_ARG, "null argument");
  cudaStream_t st = h->op->stream;
  IM_CU(cudaMemcpyAsync(rho, h->rho0, h->ns * 8, cudaMemcpyDeviceToDevice, st));
  IM_CU(cudaMemcpyAsync(u, h->u0, 2 * h->ns * 8, cudaMemcpyDeviceToDevice, st));
  IM_CU(cudaMemcpyAsync(p, h->p0, h->ns * 8, cudaMemcpyDeviceToDevice, st));
  IM_CU(cudaStreamSynchronize(st));
  return AF_OK;
}

int af_imex_step(af_imex* h, int nsteps) {
  if (!h || nsteps < 0) return ierr(AF_BAD_ARG, "bad argument");
  IM_CU(cudaSetDevice(h->op->device));
  for (int s = 0; s < nsteps; ++s) {
    h->stats = af_imex_stats{};
    IM_AF(one_step(h));
  }
  return af_synchronize(h->op);
}

int af_imex_last_stats(const af_imex* h, af_imex_stats* out) {
  if (!h || !out) return ierr(AF_BAD_ARG, "null argument");
  *out = h->stats;
  return AF_OK;
}

}  // extern "C"
