// af_blas.h -- BLAS-1 / Krylov helpers (see af_blas.cu).
#pragma once

#include <cuda_runtime.h>

namespace af {

constexpr int kMaxPartials = 1184;  // 8 x 148 SMs

// Leading dimension of a stored Krylov basis of length-n FP64 vectors: n rounded up to even,
// so that every basis vector starts on a 16-byte boundary (the operator entry points and the
// cell kernel's bulk copies need that) when n is odd, e.g. 1 x 3 cells at degree 4.
constexpr long krylov_stride(long n) { return (n + 1) & ~1L; }

// Device-resident Krylov scalars.  status: 0 ok, 1 iteration cap, 2 breakdown, 3 NaN/Inf.
struct KrylovState {
  double rr, rz, rr0, tol2, pAp, alpha, beta;
  int its, done, status, pad;
};

int reduce_blocks(long n);
// out (device) = x.y (y == null: x.x); partial needs reduce_blocks(n) doubles
cudaError_t dot(const double* x, const double* y, long n, double* partial, double* out, cudaStream_t st);
// y = a x + b y
cudaError_t axpby(double a, const double* x, double b, double* y, long n, cudaStream_t st);

// Preconditioned CG in pieces (x is the initial guess; Ax = A x, or null when x == 0):
//   cg_start(...)                     r = b - Ax, z = invd r, p = z, tolerance, done flag
//   loop: Ap = A p ; cg_after_apply   alpha, x/r/z update, beta, p = z + beta p
// part needs 2 * kMaxPartials doubles.  tol2 is preset in the state unless rel_to_initial,
// in which case tol = rel_tol * |r0|.
cudaError_t cg_start(KrylovState* s, const double* b, const double* Ax, const double* invd, double* r, double* z,
                     double* p, long n, double* part, double rel_tol, int rel_to_initial, cudaStream_t st);
cudaError_t cg_after_apply(KrylovState* s, double* x, double* r, double* z, double* p, const double* Ap,
                           const double* invd, long n, double* part, int maxit, cudaStream_t st);

// GMRES / fixed-point helpers
// out[j] = V_j . w, j < k, V_j = V + j*ldv  (partial needs k * reduce_blocks(n) <= 4*kMaxPartials doubles)
cudaError_t mdot(const double* V, long ldv, int k, const double* w, long n, double* partial, double* out,
                 cudaStream_t st);
cudaError_t maxpy(const double* V, long ldv, int k, const double* h, double* w, long n, cudaStream_t st);  // w -= V h
cudaError_t mcombine(const double* V, long ldv, int k, const double* y_host, double* x, long n,
                     cudaStream_t st);  // x += V y
cudaError_t scale(double a, const double* x, double* y, long n, cudaStream_t st);   // y = a x
cudaError_t dmul(const double* d, const double* x, double* z, long n, cudaStream_t st);  // z = d .* x
cudaError_t sub(const double* x, const double* y, double* z, long n, cudaStream_t st);   // z = x - y
// out[0] = max|x|, out[1] = max|x - y| (0 when y is null); partial needs 2*kMaxPartials doubles
cudaError_t maxabs2(const double* x, const double* y, long n, double* partial, double* out, cudaStream_t st);
// state->tol2 = eps^2 * bb[0]  (bb a device scalar, e.g. |b|^2 from dot)
cudaError_t cg_set_abs_tol(KrylovState* s, const double* bb, double eps, cudaStream_t st);

}  // namespace af
