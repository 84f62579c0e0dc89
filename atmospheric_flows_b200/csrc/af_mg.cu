// af_mg.cu -- the Schur-complement pressure solver: flexible GMRES in FP64 around the
// operator's NS_stage-2 apply D p - C A^{-1} B p (euler_operator.h:2374-2408), preconditioned
// by Jacobi on diag(D) (what the reference uses, Atmospheric_Flow.cc:657-672 with the
// diagonal of euler_operator.h:2607-2611), by a geometric h-multigrid V-cycle whose levels run
// in FP64 or FP32, or by its single-level case, a Chebyshev polynomial in D^{-1} S0 over the
// whole spectrum (FP64 or FP32).
//
// Multigrid (the role of the reference's MGLevelObject / MGTransferMatrixFree /
// PreconditionChebyshev / coarse-solver stack, Atmospheric_Flow.cc:455-522, rebuilt for the
// Schur system, where the reference has no multigrid):
//   levels      the operator's mesh and its 2:1 coarsenings in both directions (coarse
//               vertices = every other fine vertex), same degree on every level;
//   operator    S0 p = D p - C0 A^{-1} B p, C0 = C without the wave-speed term
//               0.5 lambda(w) [p_fixed]/(gamma-1) (a jump of the fixed coefficient, small,
//               and the only nonlinear part); A^{-1} exact per cell (packed inverse);
//               coefficients rho_for_fixed and pres_fixed injected level to level;
//   smoother    Chebyshev of degree k on D^{-1} S0 with D^{-1} = (gamma-1) M^{-1} exact per
//               cell, interval [1.2 lmax / range, 1.2 lmax], lmax from power iteration;
//   transfer    prolongation = embedding of the coarse polynomial in the four children,
//               restriction = its transpose;
//   coarse      Chebyshev of higher degree on [0.9, 1.2 lmax] on the first level whose lmax
//               is at most coarse_lmax (levels are trimmed there after the eigenvalue
//               estimate): the acoustic Courant number has dropped and D dominates S0.
// The FP32 variant keeps FP64 in the outer Krylov residual and orthogonalisation; the
// V-cycle only has to be a good approximate inverse.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <utility>
#include <vector>

#include "../../include/af_gpu.h"
#include "af_handle.h"

namespace af {
void set_last_error(const char* msg);
}
using namespace af;

namespace {

int merr(int code, const std::string& msg) {
  set_last_error(msg.c_str());
  return code;
}

#define MG_CU(call)                                                                                    \
  do {                                                                                                 \
    cudaError_t e_ = (call);                                                                           \
    if (e_ != cudaSuccess) return merr(AF_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_));    \
  } while (0)
#define MG_AF(call)             \
  do {                          \
    int r_ = (call);            \
    if (r_ != AF_OK) return r_; \
  } while (0)

constexpr double kG1 = 1.0 / (1.4 - 1.0);  // 1/(gamma-1)
constexpr double kGG = 1.4 / (1.4 - 1.0);  // gamma/(gamma-1)
constexpr int kThreads = 256;

unsigned nblocks(long n) { return (unsigned)((n + kThreads - 1) / kThreads); }

// ------------------------------------------------------------------ small vector kernels
template <class A, class B>
__global__ void k_convert(const A* __restrict__ x, B* __restrict__ y, long n) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) y[i] = (B)x[i];
}

__global__ void k_coarsen_vtx(const double2* __restrict__ vf, double2* __restrict__ vc, int nxc, int nzc) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (nxc + 1) * (nzc + 1)) return;
  const int ic = i % (nxc + 1), jc = i / (nxc + 1);
  vc[i] = vf[(2 * jc) * (2 * nxc + 1) + 2 * ic];
}

// deterministic start vector of the power iteration
template <class R>
__global__ void k_hash_fill(R* __restrict__ x, long n) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  unsigned h = (unsigned)i * 2654435761u + 0x9e3779b9u;
  h ^= h >> 16;
  h *= 0x85ebca6bu;
  h ^= h >> 13;
  x[i] = (R)((double)h / 4294967296.0 + 0.25);
}

// partial[b] = sum over the block's share of x^2 (accumulated in FP64)
template <class R>
__global__ void k_norm2_partial(const R* __restrict__ x, long n, double* __restrict__ partial) {
  __shared__ double red[kThreads / 32];
  double s = 0.0;
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    const double v = (double)x[i];
    s = fma(v, v, s);
  }
  for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x < 32) {
    s = threadIdx.x < kThreads / 32 ? red[threadIdx.x] : 0.0;
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if (threadIdx.x == 0) partial[blockIdx.x] = s;
  }
}

__global__ void k_sum_partials(const double* __restrict__ partial, int nb, double* __restrict__ out) {
  __shared__ double red[kThreads / 32];
  double s = 0.0;
  for (int i = threadIdx.x; i < nb; i += blockDim.x) s += partial[i];
  for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x < 32) {
    s = threadIdx.x < kThreads / 32 ? red[threadIdx.x] : 0.0;
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if (threadIdx.x == 0) out[0] = s;
  }
}

// y = x / sqrt(nrm2[0])  (x and y may alias)
template <class R>
__global__ void k_normalize(const R* x, R* y, long n, const double* __restrict__ nrm2) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) y[i] = (R)((double)x[i] / sqrt(nrm2[0]));
}

// y = a x
template <class R>
__global__ void k_scale_to(const R* __restrict__ x, R a, R* __restrict__ y, long n) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) y[i] = a * x[i];
}

constexpr int kNormBlocks = 592;  // 4 x 148 SMs

template <class R>
cudaError_t norm2(const R* x, long n, double* partial, double* out, cudaStream_t st) {
  k_norm2_partial<R><<<kNormBlocks, kThreads, 0, st>>>(x, n, partial);
  k_sum_partials<<<1, kThreads, 0, st>>>(partial, kNormBlocks, out);
  return cudaGetLastError();
}

// ------------------------------------------------------------------ levels
struct Level {
  int nx = 0, nz = 0, ncell = 0;
  long ns = 0;
  MeshDev mesh{};
  double2* vtx = nullptr;      // owned on coarse levels
  double* rho = nullptr;       // rho_for_fixed (owned on coarse levels)
  double* pf = nullptr;        // pres_fixed (owned on coarse levels)
  void* pfR = nullptr;         // pres_fixed in the level precision
  // cell-wise inverses of A (rho-weighted vector mass) and M: packed inverse matrices on FP64
  // levels; Gauss-point inverse weights (change of basis, no stored matrices) on FP32 levels
  void* LA = nullptr;
  void* LM = nullptr;
  void *x = nullptr, *b = nullptr, *r = nullptr, *d = nullptr, *u = nullptr, *w = nullptr;
  // the Gauss-point smoother (af_gauss.cuh): face traces of d and w, p_fixed at the Gauss
  // points and its traces
  float *gdtr = nullptr, *gwtr = nullptr, *gpg = nullptr, *gptr = nullptr;
  double lmax = 0.0;
};

}  // namespace

struct af_schur_solver {
  af_operator* op = nullptr;
  af_schur_options opt{};
  std::vector<Level> lv;
  int nact = 0;                 // levels in use (the coarsest has lmax <= coarse_lmax)
  bool fp32 = false;
  bool rq = false;              // FP32 levels with the reduced quadrature (P+1 Gauss points)
  bool gauss = false;           // the single-level FP32 Chebyshev in the Gauss-point basis
  bool setup_done = false, eig_done = false;
  double cB = 0, cdt = 0;       // B and C coefficients of the last setup
  double* part = nullptr;       // reductions
  double* scal = nullptr;
  double* invd = nullptr;       // Jacobi: inverse diagonal of D
  // FGMRES workspace
  double *V = nullptr, *Z = nullptr, *gw = nullptr, *dh = nullptr;
  std::vector<void*> owned;
  af_schur_stats stats{};
};

namespace {

int alloc(af_schur_solver* s, void** p, size_t bytes) {
  MG_CU(cudaMalloc(p, bytes));
  s->owned.push_back(*p);
  return AF_OK;
}

template <class R>
struct Prec;
// FP32 levels (kFused): B runs with the cell-wise A^{-1} in its epilogue and the residual
// update with the Chebyshev step in its epilogue (two launches per smoothing step instead of
// four), and both inverses are applied by the change of basis to the Gauss points: exact for
// M on bilinear cells, the (P+1)-point approximation of A (a preconditioner may differ from
// the operator), with no stored matrices and no factorisation.  FP64 levels keep the exact
// packed inverses and separate launches: a fused FP64 kernel holding the CTA's packed
// inverses in shared memory measured slower (504 vs 417 us for B + A^{-1}, 704 vs 518 us for
// the residual and Chebyshev step, 1024x256, p = 4).
template <>
struct Prec<double> {
  static constexpr bool kFused = false;
  static cudaError_t B(const DegreeOps* k, const MeshDev& m, const double* p, double c, double* u, int nc,
                       cudaStream_t st) {
    return k->op_B(m, p, c, u, nc, st);
  }
  static cudaError_t res(const DegreeOps* k, const MeshDev& m, const double* w, const double* pf, const double* p,
                         double cdt, double* r, int nc, cudaStream_t st, bool /*rq: FP32 levels only*/) {
    CParams q{cdt, kG1, kGG};
    return k->mg_res_d(m, w, pf, p, q, r, nc, st);
  }
  static cudaError_t solve(const DegreeOps* k, const double* L, int ncomp, const double* b, double s, double* x,
                           int nc, int* status, cudaStream_t st) {
    return k->mass_solve(L, ncomp, b, s, x, nc, status, st);
  }
  static cudaError_t cheb(const DegreeOps* k, const double* L, const double* r, double a, double s, double* d,
                          double* x, int first, int nc, int* status, cudaStream_t st) {
    return k->cheb_d(L, r, a, s, d, x, first, nc, status, st);
  }
  static cudaError_t prolong(const DegreeOps* k, const double* xc, double* xf, int nxc, int nzc, cudaStream_t st) {
    return k->prolong_d(xc, xf, nxc, nzc, st);
  }
  static cudaError_t restr(const DegreeOps* k, const double* rf, double* rc, int nxc, int nzc, cudaStream_t st) {
    return k->restrict_d(rf, rc, nxc, nzc, st);
  }
};
template <>
struct Prec<float> {
  static constexpr bool kFused = true;
  static cudaError_t res(const DegreeOps* k, const MeshDev& m, const float* w, const float* pf, const float* p,
                         double cdt, float* r, int nc, cudaStream_t st, bool rq) {
    CParamsT<float> q{(float)cdt, (float)kG1, (float)kGG};
    return rq ? k->mg_res_fr(m, w, pf, p, q, r, nc, st) : k->mg_res_f(m, w, pf, p, q, r, nc, st);
  }
  static cudaError_t solve(const DegreeOps* k, const float* W, int ncomp, const float* b, double s, float* x, int nc,
                           int* /*status: no bounded waits in the change-of-basis kernels*/, cudaStream_t st) {
    return k->cob_solve_f(W, ncomp, b, (float)s, x, nc, st);
  }
  static cudaError_t cheb(const DegreeOps* k, const float* W, const float* r, double a, double s, float* d, float* x,
                          int first, int nc, int* /*status*/, cudaStream_t st) {
    return k->cob_cheb_f(W, r, (float)a, (float)s, d, x, first, nc, st);
  }
  static cudaError_t b_inv(const DegreeOps* k, const MeshDev& m, const float* p, double c, const float* LA, float* w,
                           int nc, cudaStream_t st, bool rq) {
    return (rq ? k->b_inv_fr : k->b_inv_f)(m, p, (float)c, LA, 1.0f, w, nc, st);
  }
  static cudaError_t res_cheb(const DegreeOps* k, const MeshDev& m, const float* w, const float* pf, const float* din,
                              double cdt, const float* LM, double a, double s, float* r, float* dout, float* x, int nc,
                              cudaStream_t st, bool rq) {
    CParamsT<float> q{(float)cdt, (float)kG1, (float)kGG};
    return (rq ? k->res_cheb_fr : k->res_cheb_f)(m, w, pf, din, q, LM, (float)a, (float)s, r, dout, x, 0, nc, st);
  }
  // the same step on z = D^{-1} r:  z += g M^{-1} C0 w - din;  dout = a din + s z;  x += dout
  static cudaError_t res_chebz(const DegreeOps* k, const MeshDev& m, const float* w, const float* pf,
                               const float* din, double cdt, const float* LM, double g, double a, double s, float* z,
                               float* dout, float* x, int nc, cudaStream_t st, bool rq) {
    CParamsT<float> q{(float)cdt, (float)kG1, (float)kGG};
    return k->res_chebz_f(m, w, pf, din, q, LM, (float)g, (float)a, (float)s, z, dout, x, 0, rq ? 1 : 0, nc, st);
  }
  static cudaError_t prolong(const DegreeOps* k, const float* xc, float* xf, int nxc, int nzc, cudaStream_t st) {
    return k->prolong_f(xc, xf, nxc, nzc, st);
  }
  static cudaError_t restr(const DegreeOps* k, const float* rf, float* rc, int nxc, int nzc, cudaStream_t st) {
    return k->restrict_f(rf, rc, nxc, nzc, st);
  }
};

// r += C0 A^{-1} B v - D v   (= -S0 v when r starts at zero)
template <class R>
int residual_update(af_schur_solver* s, Level& L, const R* v, R* r) {
  af_operator* o = s->op;
  const DegreeOps* k = o->ops;
  if constexpr (Prec<R>::kFused) {  // w = A^{-1} B v in one launch
    MG_CU(Prec<R>::b_inv(k, L.mesh, v, s->cB, (const R*)L.LA, (R*)L.w, L.ncell, o->stream, s->rq));
    o->launches += 1;
  } else {
    MG_CU(Prec<R>::B(k, L.mesh, v, s->cB, (R*)L.u, L.ncell, o->stream));
    MG_CU(Prec<R>::solve(k, (const R*)L.LA, 2, (const R*)L.u, 1.0, (R*)L.w, L.ncell, L.mesh.status, o->stream));
    o->launches += 2;
  }
  MG_CU(Prec<R>::res(k, L.mesh, (const R*)L.w, (const R*)L.pfR, v, s->cdt, r, L.ncell, o->stream, s->rq));
  o->launches += 1;
  return AF_OK;
}

// Chebyshev iteration on D^{-1} S0 over [lo, hi], `degree` applications of D^{-1}:
// x = x0 + d0 + ... (x0 = 0 when zero_init), L.r holds the residual b - S0 x afterwards when
// final_residual (Saad, Iterative Methods for Sparse Linear Systems, 2nd ed., Alg. 12.1).
template <class R>
int chebyshev(af_schur_solver* s, Level& L, int degree, double lo, double hi, bool zero_init, bool final_residual) {
  af_operator* o = s->op;
  const DegreeOps* k = o->ops;
  R* x = (R*)L.x;
  R* r = (R*)L.r;
  R* d = (R*)L.d;
  R* dn = (R*)L.u;  // the next d: the fused step reads d's face nodes from other CTAs
  const R* b = (const R*)L.b;
  const double theta = 0.5 * (hi + lo), delta = 0.5 * (hi - lo), sigma = theta / delta;
  const double ginv = 1.0 / kG1;  // D^{-1} = (gamma-1) M^{-1}
  if constexpr (Prec<R>::kFused) {
    if (zero_init && !final_residual) {
      // FP32 levels, no residual wanted afterwards: carry z = D^{-1} r instead of r.  The
      // cell inverse of D is exact for the level's D, so z' = z + D^{-1} C0 w - d: the step
      // kernel needs no D term (ResChebZPhys).  Same iteration as below up to rounding.
      R* z = r;
      // d = x = D^{-1} b / theta;  z = D^{-1} b = theta d
      MG_CU(Prec<R>::cheb(k, (const R*)L.LM, b, 0.0, ginv / theta, d, x, 1, L.ncell, L.mesh.status, o->stream));
      k_scale_to<R><<<nblocks(L.ns), kThreads, 0, o->stream>>>(d, (R)theta, z, L.ns);
      MG_CU(cudaGetLastError());
      o->launches += 2;
      double rho_old = 1.0 / sigma;
      for (int it = 1; it < degree; ++it) {
        const double rho = 1.0 / (2.0 * sigma - rho_old);
        const double a = rho * rho_old, sc = 2.0 * rho / delta;
        // w = A^{-1} B d;  z += D^{-1} C0 w - d;  dn = a d + sc z;  x += dn  (two launches)
        MG_CU(Prec<R>::b_inv(k, L.mesh, d, s->cB, (const R*)L.LA, (R*)L.w, L.ncell, o->stream, s->rq));
        MG_CU(Prec<R>::res_chebz(k, L.mesh, (const R*)L.w, (const R*)L.pfR, d, s->cdt, (const R*)L.LM, ginv, a, sc, z,
                                 dn, x, L.ncell, o->stream, s->rq));
        o->launches += 2;
        std::swap(d, dn);
        rho_old = rho;
      }
      return AF_OK;
    }
  }
  MG_CU(cudaMemcpyAsync(r, b, sizeof(R) * L.ns, cudaMemcpyDeviceToDevice, o->stream));
  if (!zero_init) MG_AF(residual_update<R>(s, L, x, r));
  MG_CU(Prec<R>::cheb(k, (const R*)L.LM, r, 0.0, ginv / theta, d, x, zero_init ? 1 : 0, L.ncell, L.mesh.status, o->stream));
  o->launches += 1;
  double rho_old = 1.0 / sigma;
  for (int it = 1; it < degree; ++it) {
    const double rho = 1.0 / (2.0 * sigma - rho_old);
    const double a = rho * rho_old, sc = ginv * 2.0 * rho / delta;
    if constexpr (Prec<R>::kFused) {
      // w = A^{-1} B d;  r += C0 w - D d;  dn = a d + sc M^{-1} r;  x += dn  (two launches)
      MG_CU(Prec<R>::b_inv(k, L.mesh, d, s->cB, (const R*)L.LA, (R*)L.w, L.ncell, o->stream, s->rq));
      MG_CU(Prec<R>::res_cheb(k, L.mesh, (const R*)L.w, (const R*)L.pfR, d, s->cdt, (const R*)L.LM, a, sc, r, dn, x,
                              L.ncell, o->stream, s->rq));
      o->launches += 2;
      std::swap(d, dn);
    } else {
      MG_AF(residual_update<R>(s, L, d, r));
      MG_CU(Prec<R>::cheb(k, (const R*)L.LM, r, a, sc, d, x, 0, L.ncell, L.mesh.status, o->stream));
      o->launches += 1;
    }
    rho_old = rho;
  }
  if (final_residual) MG_AF(residual_update<R>(s, L, d, r));
  return AF_OK;
}

template <class R>
int vcycle_level(af_schur_solver* s, int l) {
  af_operator* o = s->op;
  Level& L = s->lv[l];
  const af_schur_options& opt = s->opt;
  const double hi = 1.2 * L.lmax;
  if (l + 1 == s->nact) {
    const double lo = std::fmin(0.9, hi / opt.smoothing_range);
    return chebyshev<R>(s, L, opt.coarse_degree, lo, hi, true, false);
  }
  const double lo = hi / opt.smoothing_range;
  Level& C = s->lv[l + 1];
  MG_AF(chebyshev<R>(s, L, opt.smoother_degree, lo, hi, true, true));
  MG_CU(Prec<R>::restr(o->ops, (const R*)L.r, (R*)C.b, C.nx, C.nz, o->stream));
  o->launches += 1;
  MG_AF(vcycle_level<R>(s, l + 1));
  MG_CU(Prec<R>::prolong(o->ops, (const R*)C.x, (R*)L.x, C.nx, C.nz, o->stream));
  o->launches += 1;
  return chebyshev<R>(s, L, opt.smoother_degree, lo, hi, false, false);
}

// lmax of D^{-1} S0 on one level by power iteration (one host read at the end)
template <class R>
int estimate_lmax(af_schur_solver* s, Level& L) {
  af_operator* o = s->op;
  const DegreeOps* k = o->ops;
  R* v = (R*)L.x;
  R* r = (R*)L.r;
  k_hash_fill<R><<<nblocks(L.ns), kThreads, 0, o->stream>>>(v, L.ns);
  MG_CU(norm2<R>(v, L.ns, s->part, s->scal, o->stream));
  k_normalize<R><<<nblocks(L.ns), kThreads, 0, o->stream>>>(v, v, L.ns, s->scal);
  for (int it = 0; it < s->opt.eig_iterations; ++it) {
    MG_CU(cudaMemsetAsync(r, 0, sizeof(R) * L.ns, o->stream));
    MG_AF(residual_update<R>(s, L, v, r));  // r = -S0 v
    MG_CU(Prec<R>::solve(k, (const R*)L.LM, 1, r, -1.0 / kG1, v, L.ncell, L.mesh.status, o->stream));  // v = D^{-1} S0 v
    MG_CU(norm2<R>(v, L.ns, s->part, s->scal, o->stream));
    k_normalize<R><<<nblocks(L.ns), kThreads, 0, o->stream>>>(v, v, L.ns, s->scal);
    o->launches += 7;
  }
  double n2 = 0.0;
  MG_CU(cudaMemcpyAsync(&n2, s->scal, sizeof(double), cudaMemcpyDeviceToHost, o->stream));
  MG_AF(sync_checked(o, o->stream));
  if (!std::isfinite(n2) || n2 <= 0.0) return merr(AF_NAN, "multigrid: eigenvalue estimate failed");
  L.lmax = std::sqrt(n2);
  return AF_OK;
}

template <class R>
int setup_levels(af_schur_solver* s, bool estimate) {
  af_operator* o = s->op;
  const DegreeOps* k = o->ops;
  const double coeff = o->hs == 1 ? o->a22t : o->a33t;  // euler_operator.h:1428, 1526
  s->cB = coeff * o->dt / (o->Ma * o->Ma);
  s->cdt = coeff * o->dt;
  for (int l = 0; l < s->nact; ++l) {
    Level& L = s->lv[l];
    if (l == 0) {
      L.rho = o->d_rho_fixed;
      L.pf = o->d_pres_fixed;
    } else {
      const Level& F = s->lv[l - 1];
      MG_CU(k->inject(F.rho, L.rho, L.nx, L.nz, o->stream));
      MG_CU(k->inject(F.pf, L.pf, L.nx, L.nz, o->stream));
      o->launches += 2;
    }
    k_convert<double, R><<<nblocks(L.ns), kThreads, 0, o->stream>>>(L.pf, (R*)L.pfR, L.ns);
    if (s->gauss) MG_CU(k->gs_values(L.pf, L.gpg, L.gptr, L.ncell, o->stream));
    if (sizeof(R) == sizeof(float)) {  // Gauss-point inverse weights of A
      MG_CU(k->cob_weights_f(L.mesh, L.rho, (float*)L.LA, L.ncell, o->stream));
    } else if (l == 0) {  // the operator's own inverse of A (built once per rho_for_fixed)
      const double* La = nullptr;
      MG_AF(mass_inverse_A(o, &La));
      const long nf = (long)L.ncell * k->factor_len;
      MG_CU(cudaMemcpyAsync(L.LA, La, sizeof(double) * nf, cudaMemcpyDeviceToDevice, o->stream));
    } else {
      MG_CU(k->mass_factor(L.mesh, L.rho, (double*)L.LA, L.ncell, o->stream));
    }
    MG_CU(cudaGetLastError());
    o->launches += 3;
  }
  if (estimate) {  // top-down; the first level with lmax <= coarse_lmax becomes the coarsest
    for (int l = 0; l < s->nact; ++l) {
      MG_AF(estimate_lmax<R>(s, s->lv[l]));
      if (s->lv[l].lmax <= s->opt.coarse_lmax) {
        s->nact = l + 1;
        break;
      }
    }
  }
  return AF_OK;
}

template <class R>
int build_mass_inverses(af_schur_solver* s) {
  af_operator* o = s->op;
  const DegreeOps* k = o->ops;
  for (auto& L : s->lv) {
    if (sizeof(R) == sizeof(double))
      MG_CU(k->mass_factor(L.mesh, nullptr, (double*)L.LM, L.ncell, o->stream));
    else
      MG_CU(k->cob_weights_f(L.mesh, nullptr, (float*)L.LM, L.ncell, o->stream));
    o->launches += 1;
  }
  return AF_OK;
}

// z = the single-level FP32 Chebyshev polynomial in the Gauss-point basis applied to v (FP64 in
// and out): the iteration of chebyshev() on z = D^{-1} r (zero start, no final residual), with
// the basis changed at entry and exit (af_gauss.cuh)
int apply_gauss(af_schur_solver* s, double* z, const double* v) {
  af_operator* o = s->op;
  const DegreeOps* k = o->ops;
  Level& L = s->lv[0];
  const double hi = 1.2 * L.lmax, lo = std::fmin(0.9, hi / s->opt.smoothing_range);
  const double theta = 0.5 * (hi + lo), delta = 0.5 * (hi - lo), sigma = theta / delta;
  const double ginv = 1.0 / kG1;  // D^{-1} = (gamma-1) M^{-1}
  float* zg = (float*)L.r;
  float* d = (float*)L.d;
  float* x = (float*)L.x;
  const float* WM = (const float*)L.LM;
  // d = x = D^{-1} v / theta;  z = D^{-1} v = theta d
  MG_CU(k->gs_entry(v, WM, (float)(ginv / theta), (float)theta, zg, d, x, L.gdtr, L.ncell, o->stream));
  o->launches += 1;
  double rho_old = 1.0 / sigma;
  for (int it = 1; it < s->opt.coarse_degree; ++it) {
    const double rho = 1.0 / (2.0 * sigma - rho_old);
    const double a = rho * rho_old, sc = 2.0 * rho / delta;
    // w = A^{-1} B d;  z += D^{-1} C0 w - d;  d = a d + sc z;  x += d  (two launches)
    MG_CU(k->gs_binv(L.mesh, d, L.gdtr, (float)s->cB, (const float*)L.LA, 1.0f, (float*)L.w, L.gwtr, L.ncell,
                     o->stream));
    MG_CU(k->gs_zstep(L.mesh, (const float*)L.w, L.gwtr, L.gpg, L.gptr, (float)s->cdt, (float)kGG, WM, (float)ginv,
                      (float)a, (float)sc, zg, d, x, L.gdtr, L.ncell, o->stream));
    o->launches += 2;
    rho_old = rho;
  }
  MG_CU(k->gs_exit(x, z, L.ncell, o->stream));
  o->launches += 1;
  return AF_OK;
}

// z = V-cycle(v): FP64 in and out, level precision inside
template <class R>
int apply_vcycle(af_schur_solver* s, double* z, const double* v) {
  af_operator* o = s->op;
  Level& L = s->lv[0];
  if (sizeof(R) == sizeof(double)) {
    MG_CU(cudaMemcpyAsync(L.b, v, sizeof(double) * L.ns, cudaMemcpyDeviceToDevice, o->stream));
  } else {
    k_convert<double, R><<<nblocks(L.ns), kThreads, 0, o->stream>>>(v, (R*)L.b, L.ns);
  }
  MG_AF(vcycle_level<R>(s, 0));
  k_convert<R, double><<<nblocks(L.ns), kThreads, 0, o->stream>>>((const R*)L.x, z, L.ns);
  MG_CU(cudaGetLastError());
  o->launches += 2;
  return AF_OK;
}

int precondition(af_schur_solver* s, double* z, const double* v) {
  af_operator* o = s->op;
  if (s->opt.preconditioner == AF_SCHUR_JACOBI) {
    MG_CU(dmul(s->invd, v, z, o->n_scalar(), o->stream));
    o->launches += 1;
    return AF_OK;
  }
  if (s->gauss) return apply_gauss(s, z, v);
  return s->fp32 ? apply_vcycle<float>(s, z, v) : apply_vcycle<double>(s, z, v);
}

}  // namespace

extern "C" {

int af_schur_default_options(af_schur_options* opt) {
  if (!opt) return merr(AF_BAD_ARG, "null options");
  opt->preconditioner = AF_SCHUR_CHEB_FP32;
  opt->smoother_degree = 5;
  opt->smoothing_range = 15.0;
  opt->coarse_degree = 10;
  opt->coarse_lmax = 25.0;
  opt->poly_degree = 16;
  opt->max_levels = 0;
  opt->min_coarse_cells = 16;
  opt->eig_iterations = 20;
  opt->restart = 30;
  opt->reduced_quadrature = 2;
  return AF_OK;
}

int af_schur_solver_create(af_operator* op, const af_schur_options* opt, af_schur_solver** out) {
  if (!op || !out) return merr(AF_BAD_ARG, "null argument");
  *out = nullptr;
  af_schur_options o{};
  if (opt) o = *opt;
  else af_schur_default_options(&o);
  if (o.preconditioner < AF_SCHUR_JACOBI || o.preconditioner > AF_SCHUR_CHEB_FP32)
    return merr(AF_BAD_ARG, "af_schur_solver_create: unknown preconditioner");
  if (o.smoother_degree < 1 || o.coarse_degree < 1 || o.smoothing_range <= 1.0 || o.eig_iterations < 1 ||
      o.restart < 1 || o.restart > 64 || !(o.coarse_lmax >= 0.0) || o.poly_degree < 1 || o.reduced_quadrature < 0 ||
      o.reduced_quadrature > 2)
    return merr(AF_BAD_ARG, "af_schur_solver_create: invalid options");
  if (o.preconditioner == AF_SCHUR_CHEB_FP64 || o.preconditioner == AF_SCHUR_CHEB_FP32) {
    // single level: the "coarse solve" on the operator's own mesh is the polynomial
    o.max_levels = 1;
    o.coarse_degree = o.poly_degree;
  }
  MG_CU(cudaSetDevice(op->device));
  auto* s = new af_schur_solver();
  s->op = op;
  s->opt = o;
  s->fp32 = o.preconditioner == AF_SCHUR_MG_FP32 || o.preconditioner == AF_SCHUR_CHEB_FP32;
  s->rq = s->fp32 && o.reduced_quadrature != 0;
  s->gauss = o.preconditioner == AF_SCHUR_CHEB_FP32 && o.reduced_quadrature == 2;
  const size_t rs = s->fp32 ? sizeof(float) : sizeof(double);
  const long ns0 = op->n_scalar();
  auto cleanup = [&](int code) {
    af_schur_solver_destroy(s);
    return code;
  };
  int r = AF_OK;
  // reductions and FGMRES workspace
  if ((r = alloc(s, (void**)&s->part, sizeof(double) * 4 * kMaxPartials)) != AF_OK) return cleanup(r);
  if ((r = alloc(s, (void**)&s->scal, sizeof(double) * 8)) != AF_OK) return cleanup(r);
  if ((r = alloc(s, (void**)&s->dh, sizeof(double) * 2 * (o.restart + 1))) != AF_OK) return cleanup(r);
  const long ld0 = krylov_stride(ns0);
  if ((r = alloc(s, (void**)&s->V, sizeof(double) * ld0 * (o.restart + 1))) != AF_OK) return cleanup(r);
  if ((r = alloc(s, (void**)&s->Z, sizeof(double) * ld0 * o.restart)) != AF_OK) return cleanup(r);
  if ((r = alloc(s, (void**)&s->gw, sizeof(double) * ns0)) != AF_OK) return cleanup(r);
  if (o.preconditioner == AF_SCHUR_JACOBI) {
    if ((r = alloc(s, (void**)&s->invd, sizeof(double) * ns0)) != AF_OK) return cleanup(r);
    *out = s;
    return AF_OK;
  }
  // level hierarchy
  int nx = op->mesh.nx, nz = op->mesh.nz;
  const int nd = op->nd;
  while (true) {
    Level L;
    L.nx = nx;
    L.nz = nz;
    L.ncell = nx * nz;
    L.ns = (long)L.ncell * nd;
    L.mesh = op->mesh;
    L.mesh.nx = nx;
    L.mesh.nz = nz;
    s->lv.push_back(L);
    const bool more = (o.max_levels <= 0 || (int)s->lv.size() < o.max_levels) && nx % 2 == 0 && nz % 2 == 0 &&
                      nx >= 4 && nz >= 2 && L.ncell > o.min_coarse_cells;
    if (!more) break;
    nx /= 2;
    nz /= 2;
  }
  for (size_t l = 0; l < s->lv.size(); ++l) {
    Level& L = s->lv[l];
    // packed inverses (FP64) or Gauss-point weights (FP32, one value per node)
    const size_t nf = s->fp32 ? (size_t)L.ns : (size_t)L.ncell * op->ops->factor_len;
    if (l > 0) {
      const Level& F = s->lv[l - 1];
      if ((r = alloc(s, (void**)&L.vtx, sizeof(double2) * (L.nx + 1) * (L.nz + 1))) != AF_OK) return cleanup(r);
      k_coarsen_vtx<<<nblocks((L.nx + 1) * (L.nz + 1)), kThreads, 0, op->stream>>>(F.mesh.vtx, L.vtx, L.nx, L.nz);
      L.mesh.vtx = L.vtx;
      if ((r = alloc(s, (void**)&L.rho, sizeof(double) * L.ns)) != AF_OK) return cleanup(r);
      if ((r = alloc(s, (void**)&L.pf, sizeof(double) * L.ns)) != AF_OK) return cleanup(r);
    }
    if ((r = alloc(s, &L.pfR, rs * L.ns)) != AF_OK) return cleanup(r);
    if ((r = alloc(s, &L.LA, rs * nf)) != AF_OK) return cleanup(r);
    if ((r = alloc(s, &L.LM, rs * nf)) != AF_OK) return cleanup(r);
    for (void** p : {&L.x, &L.b, &L.r, &L.d})
      if ((r = alloc(s, p, rs * L.ns)) != AF_OK) return cleanup(r);
    for (void** p : {&L.u, &L.w})
      if ((r = alloc(s, p, rs * 2 * L.ns)) != AF_OK) return cleanup(r);
    if (s->gauss) {
      const size_t nt = sizeof(float) * 4 * (size_t)L.ncell * (op->P + 1);
      if ((r = alloc(s, (void**)&L.gdtr, nt)) != AF_OK) return cleanup(r);
      if ((r = alloc(s, (void**)&L.gwtr, 2 * nt)) != AF_OK) return cleanup(r);
      if ((r = alloc(s, (void**)&L.gptr, nt)) != AF_OK) return cleanup(r);
      if ((r = alloc(s, (void**)&L.gpg, sizeof(float) * L.ns)) != AF_OK) return cleanup(r);
    }
  }
  s->nact = (int)s->lv.size();
  r = s->fp32 ? build_mass_inverses<float>(s) : build_mass_inverses<double>(s);
  if (r != AF_OK) return cleanup(r);
  *out = s;
  return AF_OK;
}

int af_schur_solver_destroy(af_schur_solver* s) {
  if (!s) return AF_OK;
  cudaSetDevice(s->op->device);
  cudaStreamSynchronize(s->op->stream);
  for (void* p : s->owned) cudaFree(p);
  delete s;
  return AF_OK;
}

int af_schur_solver_setup(af_schur_solver* s, int estimate_eigenvalues) {
  if (!s) return merr(AF_BAD_ARG, "null solver");
  af_operator* o = s->op;
  if (!o->rho_fixed_set || !o->pres_fixed_set)
    return merr(AF_BAD_ARG, "af_schur_solver_setup: set rho_for_fixed and pres_fixed on the operator first");
  MG_CU(cudaSetDevice(o->device));
  if (s->opt.preconditioner == AF_SCHUR_JACOBI) {
    MG_AF(af_set_NS_stage(o, 2));
    MG_AF(af_compute_diagonal(o, s->invd));
    s->setup_done = true;
    return AF_OK;
  }
  const bool est = estimate_eigenvalues || !s->eig_done;
  MG_AF(s->fp32 ? setup_levels<float>(s, est) : setup_levels<double>(s, est));
  if (est) s->eig_done = true;
  s->setup_done = true;
  return AF_OK;
}

int af_schur_solver_levels(const af_schur_solver* s, int* n_levels, double* lmax) {
  if (!s || !n_levels) return merr(AF_BAD_ARG, "null argument");
  *n_levels = s->nact;
  if (lmax)
    for (int l = 0; l < s->nact; ++l) lmax[l] = s->lv[l].lmax;
  return AF_OK;
}

int af_schur_solver_precondition(af_schur_solver* s, double* dst, const double* src) {
  if (!s || !dst || !src) return merr(AF_BAD_ARG, "null argument");
  if (!s->setup_done) return merr(AF_BAD_ARG, "af_schur_solver_setup first");
  MG_CU(cudaSetDevice(s->op->device));
  return precondition(s, dst, src);
}

}  // extern "C"

namespace {

// Flexible GMRES (right preconditioning, the preconditioned directions kept), classical
// Gram-Schmidt applied twice, Givens rotations; converged when the true residual
// |b - A x| <= rel_tol |b| (the Arnoldi estimate is checked first, the true residual is
// recomputed at every restart).  A is the Schur operator or its transpose.
template <class Apply>
int fgmres(af_schur_solver* s, const Apply& A, double* x, const double* b, double rel_tol, int max_iterations,
           af_schur_stats* stats) {
  af_operator* o = s->op;
  cudaStream_t st = o->stream;
  const long n = o->n_scalar();
  const long ld = krylov_stride(n);  // basis vectors start on 16-byte boundaries
  const int m = s->opt.restart;
  cudaEvent_t e0, e1;
  MG_CU(cudaEventCreate(&e0));
  MG_CU(cudaEventCreate(&e1));
  MG_CU(cudaEventRecord(e0, st));
  std::vector<double> H((m + 1) * m), cs(m), sn(m), g(m + 1), hh(2 * (m + 1));
  auto Hs = [&](int i, int j) -> double& { return H[i * m + j]; };
  auto read_scalar = [&](double* v) -> int {
    MG_CU(cudaMemcpyAsync(v, s->scal, sizeof(double), cudaMemcpyDeviceToHost, st));
    MG_AF(sync_checked(o, st));
    return AF_OK;
  };
  double bb = 0.0;
  MG_CU(dot(b, nullptr, n, s->part, s->scal, st));
  MG_AF(read_scalar(&bb));
  const double tol = rel_tol * std::sqrt(bb);
  int total = 0;
  double res = 0.0, res0 = -1.0;
  bool converged = false;
  while (true) {
    MG_AF(A(s->gw, x));
    MG_CU(sub(b, s->gw, s->gw, n, st));
    MG_CU(dot(s->gw, nullptr, n, s->part, s->scal, st));
    double beta2 = 0.0;
    MG_AF(read_scalar(&beta2));
    o->launches += 2;
    const double beta = std::sqrt(beta2);
    res = beta;
    if (res0 < 0.0) res0 = beta;
    if (!std::isfinite(beta)) return merr(AF_NAN, "Schur FGMRES: NaN residual");
    if (beta <= tol) { converged = true; break; }
    if (total >= max_iterations) break;
    MG_CU(scale(1.0 / beta, s->gw, s->V, n, st));
    std::fill(g.begin(), g.end(), 0.0);
    g[0] = beta;
    int jend = -1;
    for (int j = 0; j < m; ++j) {
      double* zj = s->Z + (long)j * ld;
      double* w = s->V + (long)(j + 1) * ld;
      MG_AF(precondition(s, zj, s->V + (long)j * ld));
      MG_AF(A(w, zj));
      MG_CU(mdot(s->V, ld, j + 1, w, n, s->part, s->dh, st));
      MG_CU(maxpy(s->V, ld, j + 1, s->dh, w, n, st));
      MG_CU(mdot(s->V, ld, j + 1, w, n, s->part, s->dh + (m + 1), st));
      MG_CU(maxpy(s->V, ld, j + 1, s->dh + (m + 1), w, n, st));
      MG_CU(dot(w, nullptr, n, s->part, s->scal, st));
      MG_CU(cudaMemcpyAsync(hh.data(), s->dh, sizeof(double) * 2 * (m + 1), cudaMemcpyDeviceToHost, st));
      double hn2 = 0.0;
      MG_AF(read_scalar(&hn2));
      o->launches += 5;
      for (int i = 0; i <= j; ++i) Hs(i, j) = hh[i] + hh[(m + 1) + i];
      const double hn = std::sqrt(hn2);
      Hs(j + 1, j) = hn;
      if (hn > 0.0) MG_CU(scale(1.0 / hn, w, w, n, st));
      for (int i = 0; i < j; ++i) {
        const double t = cs[i] * Hs(i, j) + sn[i] * Hs(i + 1, j);
        Hs(i + 1, j) = -sn[i] * Hs(i, j) + cs[i] * Hs(i + 1, j);
        Hs(i, j) = t;
      }
      const double a = Hs(j, j), c = Hs(j + 1, j);
      const double rr = std::hypot(a, c);
      cs[j] = rr > 0 ? a / rr : 1.0;
      sn[j] = rr > 0 ? c / rr : 0.0;
      Hs(j, j) = rr;
      Hs(j + 1, j) = 0.0;
      g[j + 1] = -sn[j] * g[j];
      g[j] = cs[j] * g[j];
      res = std::fabs(g[j + 1]);
      ++total;
      jend = j;
      if (!std::isfinite(res)) return merr(AF_NAN, "Schur FGMRES: NaN in the Arnoldi process");
      if (res <= tol || total >= max_iterations || hn == 0.0) break;
    }
    const int kk = jend + 1;
    std::vector<double> y(kk);
    for (int i = kk - 1; i >= 0; --i) {
      double sum = g[i];
      for (int l = i + 1; l < kk; ++l) sum -= Hs(i, l) * y[l];
      y[i] = sum / Hs(i, i);
    }
    MG_CU(mcombine(s->Z, ld, kk, y.data(), x, n, st));
    o->launches += 1;
  }
  MG_CU(cudaEventRecord(e1, st));
  MG_CU(cudaEventSynchronize(e1));
  float ms = 0.f;
  cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  s->stats.iterations = total;
  s->stats.initial_residual = res0;
  s->stats.final_residual = res;
  s->stats.seconds = ms * 1e-3;
  if (stats) *stats = s->stats;
  if (!converged) return merr(AF_NO_CONVERGENCE, "Schur FGMRES: no convergence within max_iterations");
  return AF_OK;
}

}  // namespace

extern "C" {

int af_schur_solve(af_schur_solver* s, double* x, const double* b, double rel_tol, int max_iterations,
                   af_schur_stats* stats) {
  if (!s || !x || !b) return merr(AF_BAD_ARG, "null argument");
  if (!s->setup_done) return merr(AF_BAD_ARG, "af_schur_solver_setup first");
  if (!(rel_tol > 0.0) || max_iterations < 1) return merr(AF_BAD_ARG, "af_schur_solve: invalid tolerance or cap");
  af_operator* o = s->op;
  MG_CU(cudaSetDevice(o->device));
  MG_AF(af_set_NS_stage(o, 2));
  auto A = [o](double* out, const double* in) { return af_vmult(o, out, in); };
  return fgmres(s, A, x, b, rel_tol, max_iterations, stats);
}

// Adjoint pressure solve: J_S(p)^T x = b at the linearisation point p, with the solver's
// preconditioner (a preconditioner of S serves its transpose: the flexible method needs no
// exact correspondence).
int af_schur_solve_transpose(af_schur_solver* s, const double* p, double* x, const double* b, double rel_tol,
                             int max_iterations, af_schur_stats* stats) {
  if (!s || !p || !x || !b) return merr(AF_BAD_ARG, "null argument");
  if (!s->setup_done) return merr(AF_BAD_ARG, "af_schur_solver_setup first");
  if (!(rel_tol > 0.0) || max_iterations < 1) return merr(AF_BAD_ARG, "af_schur_solve_transpose: invalid tolerance or cap");
  af_operator* o = s->op;
  MG_CU(cudaSetDevice(o->device));
  auto A = [o, p](double* out, const double* in) { return af_schur_transpose(o, out, p, in); };
  return fgmres(s, A, x, b, rel_tol, max_iterations, stats);
}

// Tangent pressure solve: J_S(p) x = b, the linearised Schur system that the tangent-linear
// of an IMEX stage solves, with the same FGMRES and preconditioner.
int af_schur_solve_tangent(af_schur_solver* s, const double* p, double* x, const double* b, double rel_tol,
                           int max_iterations, af_schur_stats* stats) {
  if (!s || !p || !x || !b) return merr(AF_BAD_ARG, "null argument");
  if (!s->setup_done) return merr(AF_BAD_ARG, "af_schur_solver_setup first");
  if (!(rel_tol > 0.0) || max_iterations < 1) return merr(AF_BAD_ARG, "af_schur_solve_tangent: invalid tolerance or cap");
  af_operator* o = s->op;
  MG_CU(cudaSetDevice(o->device));
  auto A = [o, p](double* out, const double* in) { return af_schur_tangent(o, out, p, in); };
  return fgmres(s, A, x, b, rel_tol, max_iterations, stats);
}

}  // extern "C"
