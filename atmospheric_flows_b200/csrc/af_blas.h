// af_blas.h -- BLAS-1 / Krylov helpers (see af_blas.cu).
#pragma once

#include <cuda_runtime.h>

namespace af {

constexpr int kMaxPartials = 1184;  // 8 x 148 SMs

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

}  // namespace af
