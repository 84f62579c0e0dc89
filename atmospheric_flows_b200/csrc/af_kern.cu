// af_kern.cu -- per-degree kernel instantiations.  Compiled once per polynomial degree
// with -DAF_P=<p>; each object registers its entry points in the degree table used by
// the C ABI (af_capi.cu).
#include <cstdint>
#include <cstdio>

#include "af_adjoint.cuh"
#include "af_gauss.cuh"
#include "af_internal.h"

#ifndef AF_P
#error "compile with -DAF_P=<degree>"
#endif

namespace af {

static __constant__ Tab<AF_P> c_tab;
static __constant__ TabT<AF_P, float> c_tabf;
static __constant__ TabT<AF_P, float, AF_P + 1> c_tabfr;  // reduced quadrature (preconditioner)
static __constant__ TabT<AF_P, double, AF_P + 1> c_tabr;  // reduced quadrature (exact B)
static __constant__ TransT<AF_P, double> c_tr;
static __constant__ TransT<AF_P, float> c_trf;
static __constant__ CobT<AF_P, double> c_cob;
static __constant__ CobT<AF_P, float> c_cobf;

template <>
__device__ __forceinline__ const Tab<AF_P>& tabr<AF_P, double>() {
  return c_tab;
}
template <>
__device__ __forceinline__ const TabT<AF_P, float>& tabr<AF_P, float>() {
  return c_tabf;
}
template <>
__device__ __forceinline__ const TabT<AF_P, float, AF_P + 1>& tabr<AF_P, float, AF_P + 1>() {
  return c_tabfr;
}
template <>
__device__ __forceinline__ const TabT<AF_P, double, AF_P + 1>& tabr<AF_P, double, AF_P + 1>() {
  return c_tabr;
}
template <>
__device__ __forceinline__ const CobT<AF_P, double>& cobr<AF_P, double>() {
  return c_cob;
}
template <>
__device__ __forceinline__ const CobT<AF_P, float>& cobr<AF_P, float>() {
  return c_cobf;
}

namespace {

constexpr int P = AF_P;
// cells per CTA of the reduced-quadrature (P+1 points) B kernel: its CTAs have NQ = P+1
// threads per cell, about half of the full-quadrature kernel's
constexpr int kReducedCB = P == 4 ? 32 : cells_per_block<P>();

cudaError_t upload_tables() {
  static const Tab<P> t = host::make_tab<P>();
  static const TabT<P, float> tf = host::make_tab<P, float>();
  static const TabT<P, float, P + 1> tfr = host::make_tab<P, float, P + 1>();
  static const TabT<P, double, P + 1> tr1 = host::make_tab<P, double, P + 1>();
  static const TransT<P, double> tr = host::make_trans<P, double>();
  static const TransT<P, float> trf = host::make_trans<P, float>();
  static const CobT<P, double> cob = host::make_cob<P, double>();
  static const CobT<P, float> cobf = host::make_cob<P, float>();
  cudaError_t e = cudaMemcpyToSymbol(c_tab, &t, sizeof(t));
  if (e == cudaSuccess) e = cudaMemcpyToSymbol(c_cob, &cob, sizeof(cob));
  if (e == cudaSuccess) e = cudaMemcpyToSymbol(c_cobf, &cobf, sizeof(cobf));
  if (e == cudaSuccess) e = cudaMemcpyToSymbol(c_tabf, &tf, sizeof(tf));
  if (e == cudaSuccess) e = cudaMemcpyToSymbol(c_tabfr, &tfr, sizeof(tfr));
  if (e == cudaSuccess) e = cudaMemcpyToSymbol(c_tabr, &tr1, sizeof(tr1));
  if (e == cudaSuccess) e = cudaMemcpyToSymbol(c_tr, &tr, sizeof(tr));
  if (e == cudaSuccess) e = cudaMemcpyToSymbol(c_trf, &trf, sizeof(trf));
  return e;
}

template <int STAGE, int MASK>
cudaError_t rhs_mask(const MeshDev& mesh, const RhsSources& s, const RhsParams& prm, double* o_rho, double* o_u,
                     double* o_p, int ncell, cudaStream_t st) {
  using Ph = RhsPhys<STAGE, MASK>;
  ArgPtrs<PhysInfo<Ph>::NARR_TOTAL, Ph::NOUT_ARR> a{};
  int k = 0;
  for (int j = 0; j < STAGE; ++j) {
    a.in[k++] = s.rho[j];
    a.in[k++] = s.u[j];
    if (Ph::VEL || Ph::PRES) a.in[k++] = s.p[j];
    if (Ph::quirk_group(j)) a.in[k++] = s.u[0];
  }
  if (Ph::HAS_I) {
    a.in[k++] = s.rho_c;
    if (Ph::PRES) a.in[k++] = s.u_fix;
  }
  int o = 0;
  if (Ph::RHO) a.out[o++] = o_rho;
  if (Ph::VEL) a.out[o++] = o_u;
  if (Ph::PRES) a.out[o++] = o_p;
  for (int i = 0; i < k; ++i)
    if (!a.in[i]) return cudaErrorInvalidValue;
  for (int i = 0; i < o; ++i)
    if (!a.out[i]) return cudaErrorInvalidValue;
  return launch_cellop<P, Ph>(mesh, a, prm, ncell, st);
}

template <int STAGE>
cudaError_t rhs_stage(const MeshDev& mesh, int mask, const RhsSources& s, const RhsParams& prm, double* o_rho,
                      double* o_u, double* o_p, int ncell, cudaStream_t st) {
  switch (mask) {
    case 1: return rhs_mask<STAGE, 1>(mesh, s, prm, o_rho, o_u, o_p, ncell, st);
    case 2: return rhs_mask<STAGE, 2>(mesh, s, prm, o_rho, o_u, o_p, ncell, st);
    case 4: return rhs_mask<STAGE, 4>(mesh, s, prm, o_rho, o_u, o_p, ncell, st);
    case 6: return rhs_mask<STAGE, 6>(mesh, s, prm, o_rho, o_u, o_p, ncell, st);
    case 7: return rhs_mask<STAGE, 7>(mesh, s, prm, o_rho, o_u, o_p, ncell, st);
    default: return cudaErrorInvalidValue;
  }
}

cudaError_t rhs(const MeshDev& mesh, int stage, int mask, const RhsSources& s, const RhsParams& prm, double* o_rho,
                double* o_u, double* o_p, int ncell, cudaStream_t st) {
  switch (stage) {
    case 1: return rhs_stage<1>(mesh, mask, s, prm, o_rho, o_u, o_p, ncell, st);
    case 2: return rhs_stage<2>(mesh, mask, s, prm, o_rho, o_u, o_p, ncell, st);
    case 3: return rhs_stage<3>(mesh, mask, s, prm, o_rho, o_u, o_p, ncell, st);
    default: return cudaErrorInvalidValue;
  }
}

cudaError_t mass(const MeshDev& mesh, int ncomp, const double* src, const double* weight, double scale, double* dst,
                 int ncell, cudaStream_t st) {
  MassParams prm{scale};
  if (weight) {
    if (ncomp == 2) {
      ArgPtrs<2, 1> a{{src, weight}, {dst}};
      return launch_cellop<P, MassPhys<2, true>>(mesh, a, prm, ncell, st);
    }
    ArgPtrs<2, 1> a{{src, weight}, {dst}};
    return launch_cellop<P, MassPhys<1, true>>(mesh, a, prm, ncell, st);
  }
  if (ncomp == 2) {
    ArgPtrs<1, 1> a{{src}, {dst}};
    return launch_cellop<P, MassPhys<2, false>>(mesh, a, prm, ncell, st);
  }
  ArgPtrs<1, 1> a{{src}, {dst}};
  return launch_cellop<P, MassPhys<1, false>>(mesh, a, prm, ncell, st);
}

cudaError_t op_B(const MeshDev& mesh, const double* p, double c, double* u, int ncell, cudaStream_t st) {
  ArgPtrs<1, 1> a{{p}, {u}};
  return launch_cellop<P, BPhysExactReduced, kReducedCB>(mesh, a, BParams{c}, ncell, st);
}

cudaError_t op_C(const MeshDev& mesh, const double* w, const double* pf, const double* p, const CParams& prm,
                 double* dst, int ncell, cudaStream_t st) {
  if (p) {
    ArgPtrs<3, 1> a{{p, w, pf}, {dst}};
    return launch_cellop<P, CPhys<true, -1>>(mesh, a, prm, ncell, st);
  }
  ArgPtrs<2, 1> a{{w, pf}, {dst}};
  return launch_cellop<P, CPhys<false, 1>>(mesh, a, prm, ncell, st);
}

// Diagonal of the (weighted) mass matrix, inverted:
//   diag_i = sum_q l_i(x_q)^2 l_j(z_q)^2 w(q) JxW(q)   (what the reference's unit-vector
//   probing in assemble_diagonal_cell_term_* computes, euler_operator.h:2458-2586)
__global__ void k_inv_diag(const MeshDev mesh, const double* __restrict__ weight, const double scale,
                           double* __restrict__ dst, const int ncomp, const int ncell) {
  using T = Tab<P>;
  constexpr int P1 = T::P1, NQ = T::NQ, ND = P1 * P1;
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= ncell) return;
  const Tab<P>& tb = c_tab;
  const int i = c % mesh.nx, j = c / mesh.nx, W = mesh.nx + 1;
  const double2 v0 = mesh.vtx[j * W + i], v1 = mesh.vtx[j * W + i + 1];
  const double2 v2 = mesh.vtx[(j + 1) * W + i], v3 = mesh.vtx[(j + 1) * W + i + 1];
  const double Ax = v1.x - v0.x, Az = v1.y - v0.y, Cx = v2.x - v0.x, Cz = v2.y - v0.y;
  const double Bx = v3.x - v2.x - v1.x + v0.x, Bz = v3.y - v2.y - v1.y + v0.y;
  double wn[ND];
  if (weight) {
#pragma unroll
    for (int k = 0; k < ND; ++k) wn[k] = weight[(size_t)c * ND + k];
  }
  double dz[P1][NQ];
#pragma unroll
  for (int iz = 0; iz < P1; ++iz)
#pragma unroll
    for (int qx = 0; qx < NQ; ++qx) dz[iz][qx] = 0.0;
  for (int qx = 0; qx < NQ; ++qx) {
    double tx[P1];
    if (weight) {
#pragma unroll
      for (int iz = 0; iz < P1; ++iz) {
        double s = 0.0;
#pragma unroll
        for (int ix = 0; ix < P1; ++ix) s = fma(tb.S[qx][ix], wn[iz * P1 + ix], s);
        tx[iz] = s;
      }
    }
    const double xi = tb.x[qx];
    const double J01 = fma(Bx, xi, Cx), J11 = fma(Bz, xi, Cz);
#pragma unroll
    for (int qz = 0; qz < NQ; ++qz) {
      const double eta = tb.x[qz];
      const double J00 = fma(Bx, eta, Ax), J10 = fma(Bz, eta, Az);
      double f = (J00 * J11 - J01 * J10) * tb.w[qx] * tb.w[qz];
      if (weight) {
        double wv = 0.0;
#pragma unroll
        for (int iz = 0; iz < P1; ++iz) wv = fma(tb.S[qz][iz], tx[iz], wv);
        f *= wv;
      } else {
        f *= scale;
      }
#pragma unroll
      for (int iz = 0; iz < P1; ++iz) dz[iz][qx] = fma(tb.S[qz][iz] * tb.S[qz][iz], f, dz[iz][qx]);
    }
  }
#pragma unroll
  for (int iz = 0; iz < P1; ++iz)
#pragma unroll
    for (int ix = 0; ix < P1; ++ix) {
      double s = 0.0;
#pragma unroll
      for (int qx = 0; qx < NQ; ++qx) s = fma(tb.S[qx][ix] * tb.S[qx][ix], dz[iz][qx], s);
      const double inv = 1.0 / s;
      for (int d = 0; d < ncomp; ++d) dst[((size_t)c * ncomp + d) * ND + iz * P1 + ix] = inv;
    }
}

cudaError_t inv_diag(const MeshDev& mesh, int ncomp, const double* weight, double scale, double* dst, int ncell,
                     cudaStream_t st) {
  const int bs = 128;
  k_inv_diag<<<(ncell + bs - 1) / bs, bs, 0, st>>>(mesh, weight, scale, dst, ncomp, ncell);
  return cudaGetLastError();
}

// ---------------------------------------------------------------- exact cell inverse
// Cell mass matrix  M_K[I][J] = sum_q w(q) JxW(q) phi_I(q) phi_J(q)  (w = 1 or a density),
// its Cholesky factor and its inverse, one warp per cell:
//   F(q) = w(q) JxW(q) at the Gauss points (lanes over points);
//   T(qz)[ix][jx] = sum_qx S[qx][ix] S[qx][jx] F(qz, qx),
//   M[I][J] = sum_qz S[qz][iz] S[qz][jz] T(qz)[ix][jx]   (lanes over entries, packed lower);
//   Cholesky M = L L^T in place (lanes over rows, one column at a time);
//   X = L^{-1}: lane j solves L x = e_j for its column in registers;  M^{-1} = X^T X.
// The packed lower triangle of the inverse (row-major) is stored cell-major,
// Minv[c * NPK + k], so that one warp of the apply kernel reads a cell's inverse as one
// contiguous block.
constexpr int kND = (P + 1) * (P + 1);
constexpr int kNPK = kND * (kND + 1) / 2;
constexpr int kFactorWarps = P <= 4 ? 4 : (P == 5 ? 2 : 1);  // static shared memory <= 48 KB

__global__ void __launch_bounds__(32 * kFactorWarps)
    k_mass_factor(const MeshDev mesh, const double* __restrict__ weight, double* __restrict__ Lg, const int ncell) {
  using T = Tab<P>;
  constexpr int P1 = T::P1, NQ = T::NQ, ND = kND, NPK = kNPK;
  constexpr int NT = NQ * P1 * (P1 + 1) / 2;  // T(qz)[ix >= jx]
  __shared__ double sA[kFactorWarps][NPK];
  __shared__ double sX[kFactorWarps][NPK];
  __shared__ double sF[kFactorWarps][NQ * NQ];
  __shared__ double sT[kFactorWarps][NT];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int c = blockIdx.x * kFactorWarps + warp;
  if (c >= ncell) return;  // whole warps; no block-wide barrier below
  const Tab<P>& tb = c_tab;
  double* A = sA[warp];
  double* X = sX[warp];
  double* F = sF[warp];
  double* Tm = sT[warp];
  const int i = c % mesh.nx, j = c / mesh.nx, W = mesh.nx + 1;
  const double2 v0 = mesh.vtx[j * W + i], v1 = mesh.vtx[j * W + i + 1];
  const double2 v2 = mesh.vtx[(j + 1) * W + i], v3 = mesh.vtx[(j + 1) * W + i + 1];
  const double Ax = v1.x - v0.x, Az = v1.y - v0.y, Cx = v2.x - v0.x, Cz = v2.y - v0.y;
  const double Bx = v3.x - v2.x - v1.x + v0.x, Bz = v3.y - v2.y - v1.y + v0.y;
  // F(q) = w(q) JxW(q)
  for (int q = lane; q < NQ * NQ; q += 32) {
    const int qx = q % NQ, qz = q / NQ;
    const double xi = tb.x[qx], eta = tb.x[qz];
    const double J00 = fma(Bx, eta, Ax), J10 = fma(Bz, eta, Az), J01 = fma(Bx, xi, Cx), J11 = fma(Bz, xi, Cz);
    double f = (J00 * J11 - J01 * J10) * tb.w[qx] * tb.w[qz];
    if (weight) {
      const double* wc = weight + (size_t)c * ND;
      double wv = 0.0;
#pragma unroll
      for (int iz = 0; iz < P1; ++iz) {
        double t = 0.0;
#pragma unroll
        for (int ix = 0; ix < P1; ++ix) t = fma(tb.S[qx][ix], wc[iz * P1 + ix], t);
        wv = fma(tb.S[qz][iz], t, wv);
      }
      f *= wv;
    }
    F[q] = f;
  }
  __syncwarp();
  // T(qz)[ix][jx], ix >= jx
  for (int e = lane; e < NT; e += 32) {
    const int qz = e / (P1 * (P1 + 1) / 2);
    int r = e % (P1 * (P1 + 1) / 2), ix = 0;
    while (r > ix) { r -= ix + 1; ++ix; }
    const int jx = r;
    double s = 0.0;
#pragma unroll
    for (int qx = 0; qx < NQ; ++qx) s = fma(tb.S[qx][ix] * tb.S[qx][jx], F[qz * NQ + qx], s);
    Tm[e] = s;
  }
  __syncwarp();
  // M[I][J], I >= J (packed row-major)
  for (int e = lane; e < NPK; e += 32) {
    int I = 0, r = e;
    while (r > I) { r -= I + 1; ++I; }
    const int J = r;
    const int iz = I / P1, ix = I % P1, jz = J / P1, jx = J % P1;
    const int a = ix >= jx ? ix : jx, b = ix >= jx ? jx : ix;
    const int tix = a * (a + 1) / 2 + b;
    double s = 0.0;
#pragma unroll
    for (int qz = 0; qz < NQ; ++qz)
      s = fma(tb.S[qz][iz] * tb.S[qz][jz], Tm[qz * (P1 * (P1 + 1) / 2) + tix], s);
    A[e] = s;
  }
  __syncwarp();
  // Cholesky, one column at a time: L_kk = sqrt(A_kk); L_ik = A_ik / L_kk; A_ij -= L_ik L_jk
  for (int k = 0; k < ND; ++k) {
    const double lkk = sqrt(A[k * (k + 1) / 2 + k]);
    const double inv = 1.0 / lkk;
    for (int r = k + 1 + lane; r < ND; r += 32) A[r * (r + 1) / 2 + k] *= inv;
    __syncwarp();
    if (lane == 0) A[k * (k + 1) / 2 + k] = lkk;
    for (int r = k + 1 + lane; r < ND; r += 32) {
      const double lrk = A[r * (r + 1) / 2 + k];
      for (int q = k + 1; q <= r; ++q) A[r * (r + 1) / 2 + q] -= lrk * A[q * (q + 1) / 2 + k];
    }
    __syncwarp();
  }
  // X = L^{-1}: lane jc solves L x = e_jc (x_i = 0 for i < jc) in registers and stores the
  // column into the packed lower X; then M^{-1}[I][J] = sum_{k >= I} X[k][I] X[k][J]
  for (int jc = lane; jc < ND; jc += 32) {
    double x[ND];
#pragma unroll
    for (int ii = 0; ii < ND; ++ii) {
      double s = (ii == jc) ? 1.0 : 0.0;
#pragma unroll
      for (int kk = 0; kk < ii; ++kk) s = fma(-A[ii * (ii + 1) / 2 + kk], x[kk], s);
      x[ii] = ii >= jc ? s / A[ii * (ii + 1) / 2 + ii] : 0.0;
      if (ii >= jc) X[ii * (ii + 1) / 2 + jc] = x[ii];
    }
  }
  __syncwarp();
  double* out = Lg + (size_t)c * NPK;
  for (int e = lane; e < NPK; e += 32) {
    int I = 0, r = e;
    while (r > I) { r -= I + 1; ++I; }
    const int J = r;
    double s = 0.0;
    for (int k = I; k < ND; ++k) s = fma(X[k * (k + 1) / 2 + I], X[k * (k + 1) / 2 + J], s);
    out[e] = s;
  }
}

// x = scale * M_K^{-1} b per cell and component: one warp per cell stages the cell's packed
// symmetric inverse (contiguous, coalesced) and its right-hand sides in shared memory by
// asynchronous copies, then lane i forms row i.  One load round trip per cell, so small
// grids are not latency-bound.
// MODE 1 is the Chebyshev update of the multigrid smoother: with y = M_K^{-1} b,
// d = alpha d + scale y (d not read when alpha == 0), then x = d (first step) or x += d.
constexpr int kSolveWarps = 4;
template <class R, int MODE>
__global__ void __launch_bounds__(32 * kSolveWarps)
    k_mass_solve(const R* __restrict__ Minv, const R* __restrict__ b, R* __restrict__ x, R* __restrict__ dv,
                 const R scale, const R alpha, const int first, const int ncomp, const int ncell, int* status) {
  constexpr int ND = kND, NPK = kNPK;
  __shared__ alignas(16) R sM[kSolveWarps * NPK];
  __shared__ alignas(16) R sb[kSolveWarps * 2 * ND];
  __shared__ alignas(8) unsigned long long s_bar;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int c0 = blockIdx.x * kSolveWarps, c = c0 + warp;
  // A full block's inverses and right-hand sides are contiguous: one bulk copy (TMA) each when
  // the chunks are 16-byte multiples, else per-element asynchronous copies per warp.
  const size_t mbytes = sizeof(R) * (size_t)kSolveWarps * NPK, bbytes = sizeof(R) * (size_t)kSolveWarps * ncomp * ND;
  const bool bulk = c0 + kSolveWarps <= ncell && mbytes % 16 == 0 && bbytes % 16 == 0 &&
                    (reinterpret_cast<uintptr_t>(Minv + (size_t)c0 * NPK) & 15) == 0 &&
                    (reinterpret_cast<uintptr_t>(b + (size_t)c0 * ncomp * ND) & 15) == 0;
  if (bulk) {
    const unsigned bar = (unsigned)__cvta_generic_to_shared(&s_bar);
    if (threadIdx.x == 0) {
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(bar) : "memory");
      asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
      asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(bar), "r"((unsigned)(mbytes + bbytes))
                   : "memory");
      asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(
                       (unsigned)__cvta_generic_to_shared(sM)),
                   "l"(Minv + (size_t)c0 * NPK), "r"((unsigned)mbytes), "r"(bar)
                   : "memory");
      asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(
                       (unsigned)__cvta_generic_to_shared(sb)),
                   "l"(b + (size_t)c0 * ncomp * ND), "r"((unsigned)bbytes), "r"(bar)
                   : "memory");
    }
    __syncthreads();  // barrier initialised before anyone waits on it
    const bool ok = mbar_wait(bar, 0);
    if (!ok) report_status(status, kStatusStageTimeout);
    if (__syncthreads_or(!ok)) {  // never expected; every thread leaves together
      if (threadIdx.x == 0) mbar_wait(bar, 0);  // (bounded) for the copies still in flight
      return;
    }
  } else {
    if (c >= ncell) return;  // whole warps only; no block-wide barrier on this path
    const R* mp = Minv + (size_t)c * NPK;
    for (int k = lane; k < NPK; k += 32) cp_async_el(&sM[warp * NPK + k], mp + k);
    const R* bp = b + (size_t)c * ncomp * ND;
    for (int k = lane; k < ncomp * ND; k += 32) cp_async_el(&sb[warp * ncomp * ND + k], bp + k);
    cp_async_wait_all();
    __syncwarp();
  }
  const R* M = sM + warp * NPK;
  const R* bb = sb + warp * ncomp * ND;
  for (int i = lane; i < ND; i += 32) {
    const int ri = i * (i + 1) / 2;
    R y0 = R(0), y1 = R(0);  // both components share each matrix load
#pragma unroll
    for (int j = 0; j < ND; ++j) {
      const R m = M[j <= i ? ri + j : j * (j + 1) / 2 + i];
      y0 = fmaR(m, bb[j], y0);
      if (ncomp == 2) y1 = fmaR(m, bb[ND + j], y1);
    }
    for (int d = 0; d < ncomp; ++d) {
      const R y = d == 0 ? y0 : y1;
      const size_t o = ((size_t)c * ncomp + d) * ND + i;
      if constexpr (MODE == 0) {
        x[o] = scale * y;
      } else {
        const R nd = (alpha != R(0) ? alpha * dv[o] : R(0)) + scale * y;
        dv[o] = nd;
        x[o] = first ? nd : x[o] + nd;
      }
    }
  }
}

template <class R, int MODE>
cudaError_t launch_mass_solve(const R* L, int ncomp, const R* b, R scale, R* x, R* d, R alpha, int first, int ncell,
                              int* status, cudaStream_t st) {
  if (ncomp < 1 || ncomp > 2) return cudaErrorInvalidValue;
  k_mass_solve<R, MODE><<<(ncell + kSolveWarps - 1) / kSolveWarps, 32 * kSolveWarps, 0, st>>>(L, b, x, d, scale, alpha,
                                                                                             first, ncomp, ncell, status);
  return cudaGetLastError();
}

// Degrees <= 4 ((P+1)^2 <= 32 rows): the same cell matrix and its inverse with lane i owning
// row i in registers, which removes the shared-memory traffic and index decoding of the
// kernel above (instruction-bound: about 11.5 k warp instructions per cell at p = 4):
//   rows: M[i][j] = sum_qz S[qz][iz] S[qz][jz] T(qz)[ix][jx], T as above (full, not packed),
//   as sum_qz S[qz][jz] U[qz][jx] with U[qz][jx] = S[qz][iz] T(qz)[ix][jx] formed first;
//   the inverse by the symmetric sweep operator (M is symmetric positive definite, no
//   pivoting): sweeping pivot k maps a_kk -> -1/a_kk, a_rk = a_kr -> a_rk/a_kk and, for
//   r, j != k, a_rj -> a_rj - (a_rk/a_kk) a_kj; it keeps the matrix symmetric, and sweeping
//   every pivot leaves -M^{-1}.  By symmetry the pivot row is the column k of the lanes'
//   registers: each lane stores its a_rk (one shared-memory store for the warp) and reads
//   the row back as broadcasts, every row but k updates itself, and row k takes the new
//   column k (the a_rk/a_kk of the other lanes) through shared memory.  (Gauss-Jordan with
//   the pivot lane scaling its row alone, 24 multiplies with one lane active per pivot, and
//   the row broadcast by warp shuffles took 1.19 ms per launch at 131072 cells; with the row
//   broadcast through shared memory 1.0 ms.)  The lower triangle is staged in shared memory
//   and stored coalesced.
constexpr int kGJWarps = 4;
template <int ND_ = kND>
__global__ void __launch_bounds__(32 * kGJWarps)
    k_mass_inverse_rows(const MeshDev mesh, const double* __restrict__ weight, double* __restrict__ Lg,
                        const int ncell) {
  static_assert(ND_ <= 32, "one row per lane");
  using T = Tab<P>;
  constexpr int P1 = T::P1, NQ = T::NQ, ND = ND_, NPK = ND * (ND + 1) / 2;
  __shared__ double sS[NQ * P1];
  __shared__ double sF[kGJWarps][NQ * NQ];
  __shared__ double sT[kGJWarps][NQ * P1 * P1];
  __shared__ double sO[kGJWarps][NPK];
  constexpr int NDE = (ND + 1) / 2 * 2;  // a row padded to whole double2
  // per warp: the pivot row (column k) and the new column k, one slot per lane
  __shared__ __align__(16) double sR[kGJWarps][32];
  __shared__ __align__(16) double sG[kGJWarps][32];
  const Tab<P>& tb = c_tab;
  for (int k = threadIdx.x; k < NQ * P1; k += blockDim.x) sS[k] = tb.S[k / P1][k % P1];
  __syncthreads();  // the only block-wide barrier; warps past the last cell leave after it
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int c = blockIdx.x * kGJWarps + warp;
  if (c >= ncell) return;
  double* F = sF[warp];
  double* Tm = sT[warp];
  double* O = sO[warp];
  const int i = c % mesh.nx, j = c / mesh.nx, W = mesh.nx + 1;
  const double2 v0 = mesh.vtx[j * W + i], v1 = mesh.vtx[j * W + i + 1];
  const double2 v2 = mesh.vtx[(j + 1) * W + i], v3 = mesh.vtx[(j + 1) * W + i + 1];
  const double Ax = v1.x - v0.x, Az = v1.y - v0.y, Cx = v2.x - v0.x, Cz = v2.y - v0.y;
  const double Bx = v3.x - v2.x - v1.x + v0.x, Bz = v3.y - v2.y - v1.y + v0.y;
  // F(q) = w(q) JxW(q)
  for (int q = lane; q < NQ * NQ; q += 32) {
    const int qx = q % NQ, qz = q / NQ;
    const double xi = tb.x[qx], eta = tb.x[qz];
    const double J00 = fma(Bx, eta, Ax), J10 = fma(Bz, eta, Az), J01 = fma(Bx, xi, Cx), J11 = fma(Bz, xi, Cz);
    double f = (J00 * J11 - J01 * J10) * tb.w[qx] * tb.w[qz];
    if (weight) {
      const double* wc = weight + (size_t)c * ND;
      double wv = 0.0;
#pragma unroll
      for (int iz = 0; iz < P1; ++iz) {
        double t = 0.0;
#pragma unroll
        for (int ix = 0; ix < P1; ++ix) t = fma(sS[qx * P1 + ix], wc[iz * P1 + ix], t);
        wv = fma(sS[qz * P1 + iz], t, wv);
      }
      f *= wv;
    }
    F[q] = f;
  }
  __syncwarp();
  // T(qz)[ix][jx]
  for (int e = lane; e < NQ * P1 * P1; e += 32) {
    const int qz = e / (P1 * P1), ix = (e / P1) % P1, jx = e % P1;
    double s = 0.0;
#pragma unroll
    for (int qx = 0; qx < NQ; ++qx) s = fma(sS[qx * P1 + ix] * sS[qx * P1 + jx], F[qz * NQ + qx], s);
    Tm[e] = s;
  }
  __syncwarp();
  // row r = lane of the cell matrix (lanes >= ND duplicate the last row and store nothing)
  const int r = lane < ND ? lane : ND - 1, rz = r / P1, rx = r % P1;
  // U[qz][jx] = S[qz][rz] T(qz)[rx][jx], then a[jz P1 + jx] = sum_qz S[qz][jz] U[qz][jx]
  // (qz outermost: one U row live at a time)
  double a[NDE];
#pragma unroll
  for (int jj = 0; jj < NDE; ++jj) a[jj] = 0.0;
#pragma unroll
  for (int qz = 0; qz < NQ; ++qz) {
    const double sz = sS[qz * P1 + rz];
    double u[P1];
#pragma unroll
    for (int jx = 0; jx < P1; ++jx) u[jx] = sz * Tm[qz * P1 * P1 + rx * P1 + jx];
#pragma unroll
    for (int jj = 0; jj < ND; ++jj) a[jj] = fma(tb.S[qz][jj / P1], u[jj % P1], a[jj]);
  }
  // sweep every pivot; rows r = lane (lanes >= ND repeat the last row and are not stored)
#pragma unroll
  for (int k = 0; k < ND; ++k) {
    // (the previous pivot's barriers order its reads of R and G before these writes)
    double* R = sR[warp];
    double* G = sG[warp];
    R[lane] = a[k];  // a_rk = a_kr: the pivot row, one element per lane
    __syncwarp();
    const double id = 1.0 / R[k];
    const double g = a[k] * id;  // the new a_rk
    if (lane != k) {
#pragma unroll
      for (int jj = 0; jj < NDE / 2; ++jj) {
        const double2 v = reinterpret_cast<const double2*>(R)[jj];
        if (2 * jj != k) a[2 * jj] = fma(-g, v.x, a[2 * jj]);
        if (2 * jj + 1 != k && 2 * jj + 1 < ND) a[2 * jj + 1] = fma(-g, v.y, a[2 * jj + 1]);
      }
      a[k] = g;
    }
    G[lane] = g;
    __syncwarp();
    if (lane == k) {  // row k = the new column k
#pragma unroll
      for (int jj = 0; jj < NDE / 2; ++jj) {
        const double2 v = reinterpret_cast<const double2*>(G)[jj];
        a[2 * jj] = v.x;
        a[2 * jj + 1] = v.y;
      }
      a[k] = -id;
      if (NDE > ND) a[NDE - 1] = 0.0;
    }
  }
#pragma unroll
  for (int jj = 0; jj < ND; ++jj) a[jj] = -a[jj];  // the sweeps leave -M^{-1}
  // lower triangle of row r, packed row-major, then coalesced
#pragma unroll
  for (int jj = 0; jj < ND; ++jj)
    if (lane < ND && jj <= lane) O[lane * (lane + 1) / 2 + jj] = a[jj];
  __syncwarp();
  double* out = Lg + (size_t)c * NPK;
  for (int e = lane; e < NPK; e += 32) out[e] = O[e];
}

cudaError_t mass_factor(const MeshDev& mesh, const double* weight, double* L, int ncell, cudaStream_t st) {
  if constexpr (kND <= 32) {
    k_mass_inverse_rows<<<(ncell + kGJWarps - 1) / kGJWarps, 32 * kGJWarps, 0, st>>>(mesh, weight, L, ncell);
  } else {
    k_mass_factor<<<(ncell + kFactorWarps - 1) / kFactorWarps, 32 * kFactorWarps, 0, st>>>(mesh, weight, L, ncell);
  }
  return cudaGetLastError();
}

cudaError_t mass_solve(const double* L, int ncomp, const double* b, double scale, double* x, int ncell, int* status,
                       cudaStream_t st) {
  return launch_mass_solve<double, 0>(L, ncomp, b, scale, x, nullptr, 0.0, 0, ncell, status, st);
}

// ------------------------------------------------------------------ multigrid kernels
// r += C0 w - D p: CPhys with SIGN +1 gives +C0 w; the D term enters with -g1
template <class R>
cudaError_t mg_res(const MeshDev& mesh, const R* w, const R* pf, const R* p, const CParamsT<R>& prm, R* r, int ncell,
                   cudaStream_t st) {
  ArgPtrs<3, 1, R> a{{p, w, pf}, {r}};
  CParamsT<R> q = prm;
  q.g1 = -prm.g1;
  return launch_cellop<P, CPhys<true, 1, R, false, true>>(mesh, a, q, ncell, st);
}

template <class R>
cudaError_t cheb(const R* L, const R* r, R alpha, R s, R* d, R* x, int first, int ncell, int* status,
                 cudaStream_t st) {
  return launch_mass_solve<R, 1>(L, 1, r, s, x, d, alpha, first, ncell, status, st);
}

template <class R>
__device__ __forceinline__ const TransT<P, R>& trans();
template <>
__device__ __forceinline__ const TransT<P, double>& trans<double>() {
  return c_tr;
}
template <>
__device__ __forceinline__ const TransT<P, float>& trans<float>() {
  return c_trf;
}

// One thread per fine node: xf[k] += sum_j Pz[kz][jz] Px[kx][jx] xc[j] over the parent cell.
template <class R>
__global__ void k_prolong(const R* __restrict__ xc, R* __restrict__ xf, const int nxc, const int nzc) {
  constexpr int P1 = P + 1, ND = P1 * P1;
  __shared__ R sP[2][P1][P1];
  for (int k = threadIdx.x; k < 2 * P1 * P1; k += blockDim.x) (&sP[0][0][0])[k] = (&trans<R>().Pm[0][0][0])[k];
  __syncthreads();
  const long idx = (long)blockIdx.x * blockDim.x + threadIdx.x;
  const long total = 4L * nxc * nzc * ND;
  if (idx >= total) return;
  const int cf = (int)(idx / ND), k = (int)(idx % ND);
  const int nxf = 2 * nxc, i_f = cf % nxf, j_f = cf / nxf;
  const int ox = i_f & 1, oz = j_f & 1, cc = (j_f >> 1) * nxc + (i_f >> 1);
  const int kx = k % P1, kz = k / P1;
  const R* x = xc + (size_t)cc * ND;
  R s = 0;
#pragma unroll
  for (int jz = 0; jz < P1; ++jz) {
    R t = 0;
#pragma unroll
    for (int jx = 0; jx < P1; ++jx) t = fmaR(sP[ox][kx][jx], x[jz * P1 + jx], t);
    s = fmaR(sP[oz][kz][jz], t, s);
  }
  xf[idx] += s;
}

// One thread per coarse node: rc[k] = sum over children and child nodes of P^T rf.
template <class R>
__global__ void k_restrict(const R* __restrict__ rf, R* __restrict__ rc, const int nxc, const int nzc) {
  constexpr int P1 = P + 1, ND = P1 * P1;
  __shared__ R sP[2][P1][P1];
  for (int k = threadIdx.x; k < 2 * P1 * P1; k += blockDim.x) (&sP[0][0][0])[k] = (&trans<R>().Pm[0][0][0])[k];
  __syncthreads();
  const long idx = (long)blockIdx.x * blockDim.x + threadIdx.x;
  const long total = (long)nxc * nzc * ND;
  if (idx >= total) return;
  const int cc = (int)(idx / ND), k = (int)(idx % ND);
  const int ic = cc % nxc, jc = cc / nxc, nxf = 2 * nxc;
  const int kx = k % P1, kz = k / P1;
  R s = 0;
#pragma unroll
  for (int oz = 0; oz < 2; ++oz)
#pragma unroll
    for (int ox = 0; ox < 2; ++ox) {
      const R* r = rf + (size_t)((2 * jc + oz) * nxf + 2 * ic + ox) * ND;
#pragma unroll
      for (int iz = 0; iz < P1; ++iz) {
        R t = 0;
#pragma unroll
        for (int ix = 0; ix < P1; ++ix) t = fmaR(sP[ox][ix][kx], r[iz * P1 + ix], t);
        s = fmaR(sP[oz][iz][kz], t, s);
      }
    }
  rc[idx] = s;
}

// One thread per coarse node: value of the child polynomial containing the node.
__global__ void k_inject(const double* __restrict__ ff, double* __restrict__ fc, const int nxc, const int nzc) {
  constexpr int P1 = P + 1, ND = P1 * P1;
  const long idx = (long)blockIdx.x * blockDim.x + threadIdx.x;
  const long total = (long)nxc * nzc * ND;
  if (idx >= total) return;
  const TransT<P, double>& tr = c_tr;
  const int cc = (int)(idx / ND), k = (int)(idx % ND);
  const int ic = cc % nxc, jc = cc / nxc, nxf = 2 * nxc;
  const int kx = k % P1, kz = k / P1;
  const int ox = tr.ch[kx], oz = tr.ch[kz];
  const double* f = ff + (size_t)((2 * jc + oz) * nxf + 2 * ic + ox) * ND;
  double s = 0.0;
  for (int jz = 0; jz < P1; ++jz) {
    double t = 0.0;
    for (int jx = 0; jx < P1; ++jx) t = fma(tr.E[kx][jx], f[jz * P1 + jx], t);
    s = fma(tr.E[kz][jz], t, s);
  }
  fc[idx] = s;
}

// ------------------------------------------------------------------ adjoint
constexpr int kAdjCells = P <= 2 ? 16 : 8;
cudaError_t rhs_adjoint1(const MeshDev& mesh, const double* const* in, const double* const* ybar,
                         double* const* xbar, const RhsParams& prm, int ncell, cudaStream_t st) {
  ArgPtrs<8, 5> a{{in[0], in[1], in[2], in[3], in[4], ybar[0], ybar[1], ybar[2]},
                  {xbar[0], xbar[1], xbar[2], xbar[3], xbar[4]}};
  return launch_cellop<P, RhsAdj1Phys, kAdjCells, 2>(mesh, a, prm, ncell, st);
}

cudaError_t rhs_tangent1(const MeshDev& mesh, const double* const* in, const double* const* din, double* const* dy,
                         const RhsParams& prm, int ncell, cudaStream_t st) {
  ArgPtrs<10, 3> a{{in[0], in[1], in[2], in[3], in[4], din[0], din[1], din[2], din[3], din[4]}, {dy[0], dy[1], dy[2]}};
  return launch_cellop<P, RhsTlm1Phys, kAdjCells, 2>(mesh, a, prm, ncell, st);
}

// ---- automatic tangents and adjoints of the fused rhs triple of any stage (dual numbers).
// Vectors in the fused order: rho_j, u_j, p_j for each explicit stage j, then rho_c, u_fixed.
template <int STAGE>
cudaError_t rhs_tangent_s(const MeshDev& mesh, const double* const* in, const double* const* din, double* const* dy,
                          const RhsParams& prm, int ncell, cudaStream_t st) {
  using Ph = RhsTanPhys<STAGE>;
  using B = RhsPhys<STAGE, 7>;
  ArgPtrs<PhysInfo<Ph>::NARR_TOTAL, 3> a{};
  int k = 0;
  for (int j = 0; j < STAGE; ++j) {
    for (int c = 0; c < 3; ++c) a.in[k++] = in[3 * j + c];
    for (int c = 0; c < 3; ++c) a.in[k++] = din[3 * j + c];
    if (B::quirk_group(j)) {  // u_old of the stage-2 kinetic jump
      a.in[k++] = in[1];
      a.in[k++] = din[1];
    }
  }
  a.in[k++] = in[3 * STAGE];
  a.in[k++] = in[3 * STAGE + 1];
  a.in[k++] = din[3 * STAGE];
  a.in[k++] = din[3 * STAGE + 1];
  a.out[0] = dy[0];
  a.out[1] = dy[1];
  a.out[2] = dy[2];
  for (int i = 0; i < k; ++i)
    if (!a.in[i]) return cudaErrorInvalidValue;
  return launch_cellop<P, Ph, kAdjCells, 2>(mesh, a, prm, ncell, st);
}

template <int STAGE, int G>
cudaError_t rhs_adj_group(const MeshDev& mesh, const double* const* in, const double* const* ybar, double* const* xbar,
                          double* scratch, const RhsParams& prm, int ncell, cudaStream_t st) {
  using Ph = RhsAdjGPhys<STAGE, G>;
  ArgPtrs<Ph::NB + 3, Ph::NB> a{};
  const int base = 3 * G;  // the group's first vector in the fused order (implicit group: 3 STAGE)
  for (int i = 0; i < Ph::NBC; ++i) {
    a.in[i] = in[base + i];
    a.out[i] = xbar[base + i];
  }
  a.in[Ph::NBC] = ybar[0];
  a.in[Ph::NBC + 1] = ybar[1];
  a.in[Ph::NBC + 2] = ybar[2];
  if constexpr (Ph::Q) {  // u_old: its cotangent goes to scratch, added to u_0's by the caller
    a.in[Ph::NBC + 3] = in[1];
    a.out[Ph::NBC] = scratch;
  }
  return launch_cellop<P, Ph, kAdjCells, 2>(mesh, a, prm, ncell, st);
}

__global__ void k_add(const double* __restrict__ x, double* __restrict__ y, const long n) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) y[i] += x[i];
}

// host-side compile-time loop (sfor is device-only)
template <class F, int... I>
void host_for_impl(F& f, std::integer_sequence<int, I...>) {
  (f(std::integral_constant<int, I>{}), ...);
}
template <int N, class F>
void host_for(F&& f) {
  host_for_impl(f, std::make_integer_sequence<int, N>{});
}

template <int STAGE>
cudaError_t rhs_adjoint_s(const MeshDev& mesh, const double* const* in, const double* const* ybar, double* const* xbar,
                          double* scratch, const RhsParams& prm, int ncell, cudaStream_t st) {
  cudaError_t e = cudaSuccess;
  host_for<STAGE + 1>([&](auto gc) {
    constexpr int G = decltype(gc)::value;
    if (e == cudaSuccess) e = rhs_adj_group<STAGE, G>(mesh, in, ybar, xbar, scratch, prm, ncell, st);
  });
  if (e != cudaSuccess) return e;
  if constexpr (RhsPhys<STAGE, 7>::quirk_group(1)) {
    const long n = 2L * ncell * kND;
    k_add<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(scratch, xbar[1], n);
    e = cudaGetLastError();
  }
  return e;
}

cudaError_t rhs_tangent(const MeshDev& mesh, int stage, const double* const* in, const double* const* din,
                        double* const* dy, const RhsParams& prm, int ncell, cudaStream_t st) {
  switch (stage) {
    case 1: return rhs_tangent_s<1>(mesh, in, din, dy, prm, ncell, st);
    case 2: return rhs_tangent_s<2>(mesh, in, din, dy, prm, ncell, st);
    case 3: return rhs_tangent_s<3>(mesh, in, din, dy, prm, ncell, st);
    default: return cudaErrorInvalidValue;
  }
}
cudaError_t rhs_adjoint(const MeshDev& mesh, int stage, const double* const* in, const double* const* ybar,
                        double* const* xbar, double* scratch, const RhsParams& prm, int ncell, cudaStream_t st) {
  switch (stage) {
    case 1: return rhs_adjoint_s<1>(mesh, in, ybar, xbar, scratch, prm, ncell, st);
    case 2: return rhs_adjoint_s<2>(mesh, in, ybar, xbar, scratch, prm, ncell, st);
    case 3: return rhs_adjoint_s<3>(mesh, in, ybar, xbar, scratch, prm, ncell, st);
    default: return cudaErrorInvalidValue;
  }
}

cudaError_t op_BT(const MeshDev& mesh, const double* ubar, double c, double* pbar, int ncell, cudaStream_t st) {
  ArgPtrs<1, 1> a{{ubar}, {pbar}};
  return launch_cellop<P, BTPhys>(mesh, a, BParams{c}, ncell, st);
}
cudaError_t op_C_tangent(const MeshDev& mesh, const double* w, const double* dw, const double* pf,
                         const CParams& prm, double* dst, int ncell, cudaStream_t st) {
  ArgPtrs<3, 1> a{{w, dw, pf}, {dst}};
  return launch_cellop<P, CTlmPhys>(mesh, a, prm, ncell, st);
}
cudaError_t op_CT(const MeshDev& mesh, const double* w, const double* pf, const double* pbar, const CParams& prm,
                  double* wbar, int ncell, cudaStream_t st) {
  ArgPtrs<3, 1> a{{w, pf, pbar}, {wbar}};
  return launch_cellop<P, CTPhys>(mesh, a, prm, ncell, st);
}

// ------------------------------------------------------------------ change-of-basis inverses
// Gauss-point inverse weights of a cell's mass matrix: W[c][qz (P+1) + qx] = 1 / (rho JxW) at
// the (P+1)-point Gauss points (rho = 1 when null), for the sum-factorised inverse
// M_K^{-1} = Vi diag(W) Vi^T of CobT (exact for the plain mass matrix on bilinear cells).
template <class R>
__global__ void k_cob_weights(const MeshDev mesh, const double* __restrict__ rho, R* __restrict__ W, const int ncell) {
  constexpr int P1 = P + 1, ND = P1 * P1;
  const long e = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= (long)ncell * ND) return;
  const int c = (int)(e / ND), q = (int)(e % ND), qx = q % P1, qz = q / P1;
  const CobT<P, double>& cb = c_cob;
  const int i = c % mesh.nx, j = c / mesh.nx, Wd = mesh.nx + 1;
  const double2 v0 = mesh.vtx[j * Wd + i], v1 = mesh.vtx[j * Wd + i + 1];
  const double2 v2 = mesh.vtx[(j + 1) * Wd + i], v3 = mesh.vtx[(j + 1) * Wd + i + 1];
  const double Ax = v1.x - v0.x, Az = v1.y - v0.y, Cx = v2.x - v0.x, Cz = v2.y - v0.y;
  const double Bx = v3.x - v2.x - v1.x + v0.x, Bz = v3.y - v2.y - v1.y + v0.y;
  const double xi = cb.g[qx], eta = cb.g[qz];
  const double J00 = fma(Bx, eta, Ax), J10 = fma(Bz, eta, Az), J01 = fma(Bx, xi, Cx), J11 = fma(Bz, xi, Cz);
  double f = (J00 * J11 - J01 * J10) * cb.w[qx] * cb.w[qz];
  if (rho) {
    const double* rc = rho + (size_t)c * ND;
    double rv = 0.0;
#pragma unroll
    for (int iz = 0; iz < P1; ++iz) {
      double t = 0.0;
#pragma unroll
      for (int ix = 0; ix < P1; ++ix) t = fma(cb.V[qx][ix], rc[iz * P1 + ix], t);
      rv = fma(cb.V[qz][iz], t, rv);
    }
    f *= rv;
  }
  W[e] = (R)(1.0 / f);
}

// x = scale M_K^{-1} b per cell and component by the change of basis (MODE 0), or the
// Chebyshev update d = alpha d + scale M_K^{-1} b, x = d (first) or x += d (MODE 1, ncomp 1).
// Tasks are (component, cell, line) over three passes in shared memory.
constexpr int kCobCells = 32;
template <class R, int MODE>
__global__ void __launch_bounds__(128)
    k_cob_solve(const R* __restrict__ W, const R* __restrict__ b, R* __restrict__ x, R* __restrict__ dv,
                const R scale, const R alpha, const int first, const int ncomp, const int ncell) {
  constexpr int P1 = P + 1, ND = P1 * P1;
  __shared__ R sy[kCobCells * 2 * ND];
  __shared__ R sw[kCobCells * ND];
  const CobT<P, R>& cb = cobr<P, R>();
  const int c0 = blockIdx.x * kCobCells, ncb = min(kCobCells, ncell - c0);
  for (int e = threadIdx.x; e < ncb * ncomp * ND; e += blockDim.x) sy[e] = b[(size_t)c0 * ncomp * ND + e];
  for (int e = threadIdx.x; e < ncb * ND; e += blockDim.x) sw[e] = W[(size_t)c0 * ND + e];
  __syncthreads();
  const int nt = ncomp * ncb * P1;  // tasks (cell, component, line); sy is [cell][comp][node]
  for (int e = threadIdx.x; e < nt; e += blockDim.x) {  // along x, in place per row
    R* row = sy + (e / P1) * ND + (e % P1) * P1;
    R y[P1];
#pragma unroll
    for (int ix = 0; ix < P1; ++ix) y[ix] = row[ix];
#pragma unroll
    for (int qx = 0; qx < P1; ++qx) {
      R t = R(0);
#pragma unroll
      for (int ix = 0; ix < P1; ++ix) t = fmaR(cb.Vi[ix][qx], y[ix], t);
      row[qx] = t;
    }
  }
  __syncthreads();
  for (int e = threadIdx.x; e < nt; e += blockDim.x) {  // along z per column, weights, back
    const int cc = e / (ncomp * P1), qx = e % P1;
    R* col = sy + (e / P1) * ND + qx;
    R u[P1], t[P1];
#pragma unroll
    for (int iz = 0; iz < P1; ++iz) u[iz] = col[iz * P1];
#pragma unroll
    for (int qz = 0; qz < P1; ++qz) {
      R a = R(0);
#pragma unroll
      for (int iz = 0; iz < P1; ++iz) a = fmaR(cb.Vi[iz][qz], u[iz], a);
      t[qz] = a * sw[cc * ND + qz * P1 + qx];
    }
#pragma unroll
    for (int iz = 0; iz < P1; ++iz) {
      R a = R(0);
#pragma unroll
      for (int qz = 0; qz < P1; ++qz) a = fmaR(cb.Vi[iz][qz], t[qz], a);
      col[iz * P1] = a;
    }
  }
  __syncthreads();
  for (int e = threadIdx.x; e < nt; e += blockDim.x) {  // along x, then the store or update
    const R* row = sy + (e / P1) * ND + (e % P1) * P1;
    R v[P1];
#pragma unroll
    for (int qx = 0; qx < P1; ++qx) v[qx] = row[qx];
#pragma unroll
    for (int ix = 0; ix < P1; ++ix) {
      R y = R(0);
#pragma unroll
      for (int qx = 0; qx < P1; ++qx) y = fmaR(cb.Vi[ix][qx], v[qx], y);
      const size_t g = (size_t)c0 * ncomp * ND + (size_t)(e / P1) * ND + (e % P1) * P1 + ix;
      if constexpr (MODE == 0) {
        x[g] = scale * y;
      } else {
        const R nd = (alpha != R(0) ? alpha * dv[g] : R(0)) + scale * y;
        dv[g] = nd;
        x[g] = first ? nd : x[g] + nd;
      }
    }
  }
}

template <class R>
cudaError_t cob_weights(const MeshDev& mesh, const double* rho, R* W, int ncell, cudaStream_t st) {
  const long n = (long)ncell * kND;
  k_cob_weights<R><<<(unsigned)((n + 255) / 256), 256, 0, st>>>(mesh, rho, W, ncell);
  return cudaGetLastError();
}
template <class R>
cudaError_t cob_solve(const R* W, int ncomp, const R* b, R scale, R* x, int ncell, cudaStream_t st) {
  if (ncomp < 1 || ncomp > 2) return cudaErrorInvalidValue;
  k_cob_solve<R, 0><<<(ncell + kCobCells - 1) / kCobCells, 128, 0, st>>>(W, b, x, nullptr, scale, R(0), 0, ncomp,
                                                                         ncell);
  return cudaGetLastError();
}
template <class R>
cudaError_t cob_cheb(const R* W, const R* r, R alpha, R s, R* d, R* x, int first, int ncell, cudaStream_t st) {
  k_cob_solve<R, 1><<<(ncell + kCobCells - 1) / kCobCells, 128, 0, st>>>(W, r, x, d, s, alpha, first, 1, ncell);
  return cudaGetLastError();
}

// ------------------------------------------------------------------ fused epilogues
// Launch shapes of the two FP32 smoother kernels at p = 4 (1024x256, us per launch):
// cells per CTA / CTAs per SM  16/2: B+A^-1 190.6, residual+Chebyshev 258.2;  32/2: 176.4,
// 237.7;  32/3: 172.5, 240.5;  8/8: 215.1, 314.7;  64/1: 209.1, 372.2.
constexpr int kFusedCB = P == 4 ? 32 : cells_per_block<P>();
constexpr int kBInvMinB = P == 4 ? 3 : min_blocks_per_sm<P>();
constexpr int kResChebMinB = min_blocks_per_sm<P>();
template <class R>
cudaError_t b_inv(const MeshDev& mesh, const R* p, R c, const R* WA, R scale, R* w, int ncell, cudaStream_t st) {
  ArgPtrs<1, 1, R> a{{p}, {w}};
  BInvParams<R> q;
  q.c = c;
  q.inv = WA;
  q.scale = scale;
  return launch_cellop<P, BInvPhys<R>, kFusedCB, kBInvMinB>(mesh, a, q, ncell, st);
}

template <class R>
cudaError_t res_cheb(const MeshDev& mesh, const R* w, const R* pf, const R* din, const CParamsT<R>& prm, const R* WM,
                     R alpha, R s, R* r, R* dout, R* x, int first, int ncell, cudaStream_t st) {
  if (din == dout) return cudaErrorInvalidValue;
  ArgPtrs<3, 1, R> a{{din, w, pf}, {r}};
  ResChebParams<R> q;
  static_cast<CParamsT<R>&>(q) = prm;
  q.g1 = -prm.g1;
  q.inv = WM;
  q.alpha = alpha;
  q.s = s;
  q.r = r;
  q.din = din;
  q.dout = dout;
  q.x = x;
  q.first = first;
  return launch_cellop<P, ResChebPhys<R>, kFusedCB, kResChebMinB>(mesh, a, q, ncell, st);
}

// reduced-quadrature (P+1 Gauss points) counterparts of mg_res, b_inv and res_cheb in FP32
cudaError_t mg_res_fr(const MeshDev& mesh, const float* w, const float* pf, const float* p, const CParamsT<float>& prm,
                      float* r, int ncell, cudaStream_t st) {
  ArgPtrs<3, 1, float> a{{p, w, pf}, {r}};
  CParamsT<float> q = prm;
  q.g1 = -prm.g1;
  return launch_cellop<P, CResRPhys<float>, kFusedCB, kResChebMinB>(mesh, a, q, ncell, st);
}
cudaError_t b_inv_fr(const MeshDev& mesh, const float* p, float c, const float* WA, float scale, float* w, int ncell,
                     cudaStream_t st) {
  ArgPtrs<1, 1, float> a{{p}, {w}};
  BInvParams<float> q;
  q.c = c;
  q.inv = WA;
  q.scale = scale;
  return launch_cellop<P, BInvRPhys<float>, kFusedCB, (P == 4 ? 4 : kBInvMinB)>(mesh, a, q, ncell, st);  // 92 vs 95 us
}
cudaError_t res_cheb_fr(const MeshDev& mesh, const float* w, const float* pf, const float* din,
                        const CParamsT<float>& prm, const float* WM, float alpha, float s, float* r, float* dout,
                        float* x, int first, int ncell, cudaStream_t st) {
  if (din == dout) return cudaErrorInvalidValue;
  ArgPtrs<3, 1, float> a{{din, w, pf}, {r}};
  ResChebParams<float> q;
  static_cast<CParamsT<float>&>(q) = prm;
  q.g1 = -prm.g1;
  q.inv = WM;
  q.alpha = alpha;
  q.s = s;
  q.r = r;
  q.din = din;
  q.dout = dout;
  q.x = x;
  q.first = first;
  return launch_cellop<P, ResChebRPhys<float>, kFusedCB, kResChebMinB>(mesh, a, q, ncell, st);
}

// the smoother step on the preconditioned residual z (ResChebZPhys): the kernel evaluates C0 w
// alone; full (2P+1) or reduced (P+1) Gauss points per direction
template <class Phys>
cudaError_t res_chebz_launch(const MeshDev& mesh, const float* w, const float* pf, const float* din,
                             const CParamsT<float>& prm, const float* WM, float g, float alpha, float s, float* z,
                             float* dout, float* x, int first, int ncell, cudaStream_t st) {
  if (din == dout) return cudaErrorInvalidValue;
  ArgPtrs<2, 1, float> a{{w, pf}, {z}};
  ResChebZParams<float> q;
  static_cast<CParamsT<float>&>(q) = prm;
  q.inv = WM;
  q.g = g;
  q.alpha = alpha;
  q.s = s;
  q.r = z;
  q.din = din;
  q.dout = dout;
  q.x = x;
  q.first = first;
  return launch_cellop<P, Phys, kFusedCB, kResChebMinB>(mesh, a, q, ncell, st);
}
cudaError_t res_chebz_f(const MeshDev& mesh, const float* w, const float* pf, const float* din,
                        const CParamsT<float>& prm, const float* WM, float g, float alpha, float s, float* z,
                        float* dout, float* x, int first, int reduced, int ncell, cudaStream_t st) {
  return reduced ? res_chebz_launch<ResChebZRPhys<float>>(mesh, w, pf, din, prm, WM, g, alpha, s, z, dout, x, first,
                                                          ncell, st)
                 : res_chebz_launch<ResChebZPhys<float>>(mesh, w, pf, din, prm, WM, g, alpha, s, z, dout, x, first,
                                                         ncell, st);
}

// ------------------------------------------------------------------ Gauss-point smoother
template <class K, class... A>
cudaError_t launch_gs(K kernel, int ncell, cudaStream_t st, bool pdl, A... args) {
  using S = GsShape<P>;
  const int nblk = (ncell + S::CB - 1) / S::CB;
  if (ncell <= 0) return cudaSuccess;
  cudaLaunchConfig_t cfg{};
  cfg.gridDim = dim3((unsigned)nblk);
  cfg.blockDim = dim3((unsigned)S::NT);
  cfg.stream = st;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = at;
  cfg.numAttrs = (kPDL && pdl) ? 1 : 0;
  return cudaLaunchKernelEx(&cfg, kernel, args...);
}
cudaError_t gs_entry(const double* v, const float* WM, float sc, float theta, float* z, float* d, float* x,
                     float* dtr, int ncell, cudaStream_t st) {
  return launch_gs(k_gs_entry<P>, ncell, st, true, v, WM, sc, theta, z, d, x, dtr, ncell);
}
cudaError_t gs_binv(const MeshDev& mesh, const float* d, const float* dtr, float c, const float* WA, float scale,
                    float* w, float* wtr, int ncell, cudaStream_t st) {
  if (mesh.cell0 != 0) return cudaErrorInvalidValue;
  return launch_gs(k_gs_binv<P>, ncell, st, true, mesh, d, dtr, c, WA, scale, w, wtr, ncell);
}
cudaError_t gs_zstep(const MeshDev& mesh, const float* w, const float* wtr, const float* pg, const float* ptr,
                     float cdt, float gg, const float* WM, float g, float alpha, float s, float* z, float* d,
                     float* x, float* dtr, int ncell, cudaStream_t st) {
  if (mesh.cell0 != 0) return cudaErrorInvalidValue;
  return launch_gs(k_gs_zstep<P>, ncell, st, true, mesh, w, wtr, pg, ptr, cdt, gg, WM, g, alpha, s, z, d, x, 0, dtr,
                   ncell);
}
cudaError_t gs_exit(const float* x, double* out, int ncell, cudaStream_t st) {
  return launch_gs(k_gs_exit<P>, ncell, st, true, x, out, ncell);
}
cudaError_t gs_values(const double* p, float* pg, float* ptr, int ncell, cudaStream_t st) {
  return launch_gs(k_gs_values<P>, ncell, st, false, p, pg, ptr, ncell);
}

cudaError_t op_A_rho_T(const MeshDev& mesh, const double* x, const double* y, double* rhobar, int ncell,
                       cudaStream_t st) {
  ArgPtrs<2, 1> a{{x, y}, {rhobar}};
  return launch_cellop<P, MassRhoTPhys>(mesh, a, MassParams{1.0}, ncell, st);
}
cudaError_t op_C_pf_T(const MeshDev& mesh, const double* w, const double* pbar, const CParams& prm, double* pfbar,
                      int ncell, cudaStream_t st) {
  ArgPtrs<2, 1> a{{w, pbar}, {pfbar}};
  return launch_cellop<P, CPfTPhys>(mesh, a, prm, ncell, st);
}

constexpr int kTransferThreads = 256;

template <class R>
cudaError_t prolong(const R* xc, R* xf, int nxc, int nzc, cudaStream_t st) {
  const long n = 4L * nxc * nzc * kND;
  k_prolong<R><<<(unsigned)((n + kTransferThreads - 1) / kTransferThreads), kTransferThreads, 0, st>>>(xc, xf, nxc, nzc);
  return cudaGetLastError();
}
template <class R>
cudaError_t restrict_(const R* rf, R* rc, int nxc, int nzc, cudaStream_t st) {
  const long n = (long)nxc * nzc * kND;
  k_restrict<R><<<(unsigned)((n + kTransferThreads - 1) / kTransferThreads), kTransferThreads, 0, st>>>(rf, rc, nxc, nzc);
  return cudaGetLastError();
}
cudaError_t inject(const double* ff, double* fc, int nxc, int nzc, cudaStream_t st) {
  const long n = (long)nxc * nzc * kND;
  k_inject<<<(unsigned)((n + kTransferThreads - 1) / kTransferThreads), kTransferThreads, 0, st>>>(ff, fc, nxc, nzc);
  return cudaGetLastError();
}

const DegreeOps kOps = {upload_tables,     rhs,
                        mass,              op_B,
                        op_C,              inv_diag,
                        mass_factor,       mass_solve,
                        cells_per_block<P>(), kNPK,
                        mg_res<double>,    mg_res<float>,
                        cheb<double>,
                        prolong<double>,   prolong<float>,
                        restrict_<double>, restrict_<float>,
                        inject,            rhs_adjoint1,
                        rhs_tangent1,      op_BT,
                        op_C_tangent,      op_CT,
                        cob_weights<float>, cob_weights<double>,
                        cob_solve<float>,  cob_solve<double>,
                        cob_cheb<float>,   b_inv<float>,
                        res_cheb<float>,   mg_res_fr,
                        b_inv_fr,          res_cheb_fr,
                        op_A_rho_T,        op_C_pf_T,
                        rhs_tangent,       rhs_adjoint,
                        res_chebz_f,       gs_entry,
                        gs_binv,           gs_zstep,
                        gs_exit,           gs_values};

}  // namespace

void register_degree(int p, const DegreeOps* ops);

namespace {
struct Registrar {
  Registrar() { register_degree(P, &kOps); }
} registrar;
}  // namespace

}  // namespace af
