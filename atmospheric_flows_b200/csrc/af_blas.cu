// af_blas.cu -- BLAS-1 and Krylov helper kernels (FP64), device-resident scalars.
//
// Reductions are deterministic: a fixed grid (a function of n only) produces per-block
// partial sums in a fixed order, and one block adds the partials in a fixed order.
// Krylov scalars live in a device KrylovState so iterations can be queued without host
// round trips; every update kernel returns early once state->done is set, which lets the
// host enqueue a batch of iterations and test convergence once per batch.
#include <cuda_runtime.h>

#include "af_blas.h"

namespace af {

constexpr int RB = 256;  // threads per reduction block

__device__ __forceinline__ double block_sum(double v, double* sh) {
  const int t = threadIdx.x;
  sh[t] = v;
  __syncthreads();
#pragma unroll
  for (int s = RB / 2; s > 0; s >>= 1) {
    if (t < s) sh[t] += sh[t + s];
    __syncthreads();
  }
  return sh[0];
}

int reduce_blocks(long n) {
  long b = (n + RB * 4 - 1) / (RB * 4);
  if (b > kMaxPartials) b = kMaxPartials;
  if (b < 1) b = 1;
  return (int)b;
}

// partial[b] = sum over the block's grid-stride range of x*y (y == null: x*x)
__global__ void k_dot_partial(const double* __restrict__ x, const double* __restrict__ y, long n,
                              double* __restrict__ partial) {
  __shared__ double sh[RB];
  double s = 0.0;
  const long stride = (long)gridDim.x * RB;
  for (long i = (long)blockIdx.x * RB + threadIdx.x; i < n; i += stride) s = fma(x[i], y ? y[i] : x[i], s);
  const double b = block_sum(s, sh);
  if (threadIdx.x == 0) partial[blockIdx.x] = b;
}

// out = sum(partial[0..nb)) ; optional: also writes sqrt into out_sqrt
__global__ void k_sum_partials(const double* __restrict__ partial, int nb, double* out) {
  __shared__ double sh[RB];
  double s = 0.0;
  for (int i = threadIdx.x; i < nb; i += RB) s += partial[i];
  const double b = block_sum(s, sh);
  if (threadIdx.x == 0) *out = b;
}

cudaError_t dot(const double* x, const double* y, long n, double* partial, double* out, cudaStream_t st) {
  const int nb = reduce_blocks(n);
  k_dot_partial<<<nb, RB, 0, st>>>(x, y, n, partial);
  k_sum_partials<<<1, RB, 0, st>>>(partial, nb, out);
  return cudaGetLastError();
}

__global__ void k_axpby(double a, const double* __restrict__ x, double b, double* __restrict__ y, long n) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) y[i] = fma(a, x[i], b * y[i]);
}

cudaError_t axpby(double a, const double* x, double b, double* y, long n, cudaStream_t st) {
  const int bs = 256;
  k_axpby<<<(unsigned)((n + bs - 1) / bs), bs, 0, st>>>(a, x, b, y, n);
  return cudaGetLastError();
}

// ------------------------------------------------------------------ CG pieces
// state layout: see KrylovState in af_blas.h

// r = b - Ax (or r = b when x == 0), z = invd * r, p = z; partials of r.r and r.z
__global__ void k_cg_init(const double* __restrict__ b, const double* __restrict__ Ax, const double* __restrict__ invd,
                          double* __restrict__ r, double* __restrict__ z, double* __restrict__ p, long n,
                          double* __restrict__ part_rr, double* __restrict__ part_rz) {
  __shared__ double sh[RB];
  double rr = 0.0, rz = 0.0;
  const long stride = (long)gridDim.x * RB;
  for (long i = (long)blockIdx.x * RB + threadIdx.x; i < n; i += stride) {
    const double ri = Ax ? b[i] - Ax[i] : b[i];
    const double zi = invd ? invd[i] * ri : ri;
    r[i] = ri;
    z[i] = zi;
    p[i] = zi;
    rr = fma(ri, ri, rr);
    rz = fma(ri, zi, rz);
  }
  double v = block_sum(rr, sh);
  if (threadIdx.x == 0) part_rr[blockIdx.x] = v;
  __syncthreads();
  v = block_sum(rz, sh);
  if (threadIdx.x == 0) part_rz[blockIdx.x] = v;
}

// finalise: rr, rz from partials; tol2 = (rel * sqrt(bb))^2 given bb = rr at start when
// rel_to_initial, else tol2 preset; done if rr <= tol2
__global__ void k_cg_start(KrylovState* s, const double* __restrict__ part_rr, const double* __restrict__ part_rz,
                           int nb, double rel_tol, int rel_to_initial) {
  __shared__ double sh[RB];
  double a = 0.0, c = 0.0;
  for (int i = threadIdx.x; i < nb; i += RB) { a += part_rr[i]; c += part_rz[i]; }
  const double rr = block_sum(a, sh);
  __syncthreads();
  const double rz = block_sum(c, sh);
  if (threadIdx.x == 0) {
    s->rr = rr;
    s->rz = rz;
    s->rr0 = rr;
    if (rel_to_initial) s->tol2 = rel_tol * rel_tol * rr;
    s->its = 0;
    s->done = (rr <= s->tol2) ? 1 : 0;
    s->status = 0;
  }
}

__global__ void k_pAp_partial(const KrylovState* s, const double* __restrict__ p, const double* __restrict__ Ap,
                              long n, double* __restrict__ part) {
  if (s->done) return;
  __shared__ double sh[RB];
  double v = 0.0;
  const long stride = (long)gridDim.x * RB;
  for (long i = (long)blockIdx.x * RB + threadIdx.x; i < n; i += stride) v = fma(p[i], Ap[i], v);
  v = block_sum(v, sh);
  if (threadIdx.x == 0) part[blockIdx.x] = v;
}

__global__ void k_cg_alpha(KrylovState* s, const double* __restrict__ part, int nb) {
  if (s->done) return;
  __shared__ double sh[RB];
  double a = 0.0;
  for (int i = threadIdx.x; i < nb; i += RB) a += part[i];
  const double pAp = block_sum(a, sh);
  if (threadIdx.x == 0) {
    s->pAp = pAp;
    s->alpha = s->rz / pAp;
    if (!(pAp > 0.0) || !isfinite(s->alpha)) { s->status = 2; s->done = 1; }
  }
}

// x += alpha p, r -= alpha Ap, z = invd r ; partials of r.r and r.z
__global__ void k_cg_update(const KrylovState* s, double* __restrict__ x, double* __restrict__ r,
                            double* __restrict__ z, const double* __restrict__ p, const double* __restrict__ Ap,
                            const double* __restrict__ invd, long n, double* __restrict__ part_rr,
                            double* __restrict__ part_rz) {
  if (s->done) return;
  __shared__ double sh[RB];
  const double alpha = s->alpha;
  double rr = 0.0, rz = 0.0;
  const long stride = (long)gridDim.x * RB;
  for (long i = (long)blockIdx.x * RB + threadIdx.x; i < n; i += stride) {
    x[i] = fma(alpha, p[i], x[i]);
    const double ri = fma(-alpha, Ap[i], r[i]);
    r[i] = ri;
    const double zi = invd ? invd[i] * ri : ri;
    z[i] = zi;
    rr = fma(ri, ri, rr);
    rz = fma(ri, zi, rz);
  }
  double v = block_sum(rr, sh);
  if (threadIdx.x == 0) part_rr[blockIdx.x] = v;
  __syncthreads();
  v = block_sum(rz, sh);
  if (threadIdx.x == 0) part_rz[blockIdx.x] = v;
}

__global__ void k_cg_beta(KrylovState* s, const double* __restrict__ part_rr, const double* __restrict__ part_rz,
                          int nb, int maxit) {
  if (s->done) return;
  __shared__ double sh[RB];
  double a = 0.0, c = 0.0;
  for (int i = threadIdx.x; i < nb; i += RB) { a += part_rr[i]; c += part_rz[i]; }
  const double rr = block_sum(a, sh);
  __syncthreads();
  const double rz = block_sum(c, sh);
  if (threadIdx.x == 0) {
    s->its += 1;
    s->rr = rr;
    s->beta = rz / s->rz;
    s->rz = rz;
    if (!isfinite(rr)) { s->status = 3; s->done = 1; }
    else if (rr <= s->tol2) s->done = 1;
    else if (s->its >= maxit) { s->status = 1; s->done = 1; }
  }
}

__global__ void k_cg_dir(const KrylovState* s, double* __restrict__ p, const double* __restrict__ z, long n) {
  if (s->done) return;
  const double beta = s->beta;
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) p[i] = fma(beta, p[i], z[i]);
}

cudaError_t cg_start(KrylovState* s, const double* b, const double* Ax, const double* invd, double* r, double* z,
                     double* p, long n, double* part, double rel_tol, int rel_to_initial, cudaStream_t st) {
  const int nb = reduce_blocks(n);
  k_cg_init<<<nb, RB, 0, st>>>(b, Ax, invd, r, z, p, n, part, part + kMaxPartials);
  k_cg_start<<<1, RB, 0, st>>>(s, part, part + kMaxPartials, nb, rel_tol, rel_to_initial);
  return cudaGetLastError();
}

cudaError_t cg_after_apply(KrylovState* s, double* x, double* r, double* z, double* p, const double* Ap,
                           const double* invd, long n, double* part, int maxit, cudaStream_t st) {
  const int nb = reduce_blocks(n);
  k_pAp_partial<<<nb, RB, 0, st>>>(s, p, Ap, n, part);
  k_cg_alpha<<<1, RB, 0, st>>>(s, part, nb);
  k_cg_update<<<nb, RB, 0, st>>>(s, x, r, z, p, Ap, invd, n, part, part + kMaxPartials);
  k_cg_beta<<<1, RB, 0, st>>>(s, part, part + kMaxPartials, nb, maxit);
  k_cg_dir<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(s, p, z, n);
  return cudaGetLastError();
}

}  // namespace af

// ---------------------------------------------------------------- FP64 peak probe
// 8 independent FMA chains per thread, enough warps to fill every SM: the measured
// DFMA throughput is the denominator of the FP64 roofline reported by bench.py.
namespace af {
__global__ void k_dfma_peak(double* out, int iters, double a, double b) {
  double x0 = threadIdx.x * 1e-7, x1 = x0 + 1e-9, x2 = x0 + 2e-9, x3 = x0 + 3e-9;
  double x4 = x0 + 4e-9, x5 = x0 + 5e-9, x6 = x0 + 6e-9, x7 = x0 + 7e-9;
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int k = 0; k < 16; ++k) {
      x0 = fma(x0, a, b); x1 = fma(x1, a, b); x2 = fma(x2, a, b); x3 = fma(x3, a, b);
      x4 = fma(x4, a, b); x5 = fma(x5, a, b); x6 = fma(x6, a, b); x7 = fma(x7, a, b);
    }
  }
  const double s = x0 + x1 + x2 + x3 + x4 + x5 + x6 + x7;
  if (s == 12345.678) out[0] = s;  // keeps the chains alive
}
}  // namespace af

extern "C" int af_measure_fp64_peak(double* tflops) {
  if (!tflops) return 1;
  int dev = 0, nsm = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
    return 2;
  double* d = nullptr;
  if (cudaMalloc(&d, sizeof(double)) != cudaSuccess) return 2;
  const int blocks = nsm * 8, threads = 256, iters = 2048;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  af::k_dfma_peak<<<blocks, threads>>>(d, 64, 0.999999, 1e-9);  // warm-up
  float best = 1e30f;
  for (int r = 0; r < 5; ++r) {
    cudaEventRecord(e0);
    af::k_dfma_peak<<<blocks, threads>>>(d, iters, 0.999999, 1e-9);
    cudaEventRecord(e1);
    cudaEventSynchronize(e1);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    if (ms < best) best = ms;
  }
  const double flops = 2.0 * 8 * 16 * (double)iters * blocks * threads;
  *tflops = flops / (best * 1e-3) / 1e12;
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(d);
  return cudaGetLastError() == cudaSuccess ? 0 : 2;
}

// ------------------------------------------------------------------ GMRES / IMEX pieces
namespace af {

// out[j] = V_j . w for j < k (V_j = V + j*ldv); partials per (j, block), fixed order
__global__ void k_mdot_partial(const double* __restrict__ V, long ldv, const double* __restrict__ w, long n,
                               double* __restrict__ partial, int nb) {
  __shared__ double sh[RB];
  const int j = blockIdx.y;
  const double* v = V + (long)j * ldv;
  double s = 0.0;
  const long stride = (long)gridDim.x * RB;
  for (long i = (long)blockIdx.x * RB + threadIdx.x; i < n; i += stride) s = fma(v[i], w[i], s);
  const double b = block_sum(s, sh);
  if (threadIdx.x == 0) partial[(long)j * nb + blockIdx.x] = b;
}

__global__ void k_mdot_final(const double* __restrict__ partial, int nb, double* __restrict__ out) {
  __shared__ double sh[RB];
  const int j = blockIdx.x;
  double s = 0.0;
  for (int i = threadIdx.x; i < nb; i += RB) s += partial[(long)j * nb + i];
  const double b = block_sum(s, sh);
  if (threadIdx.x == 0) out[j] = b;
}

cudaError_t mdot(const double* V, long ldv, int k, const double* w, long n, double* partial, double* out,
                 cudaStream_t st) {
  int nb = reduce_blocks(n);
  if (nb * k > 4 * kMaxPartials) nb = (4 * kMaxPartials) / k;
  if (nb < 1) nb = 1;
  k_mdot_partial<<<dim3(nb, k), RB, 0, st>>>(V, ldv, w, n, partial, nb);
  k_mdot_final<<<k, RB, 0, st>>>(partial, nb, out);
  return cudaGetLastError();
}

// w -= sum_{j<k} h[j] V_j  (h on the device)
__global__ void k_maxpy(const double* __restrict__ V, long ldv, int k, const double* __restrict__ h,
                        double* __restrict__ w, long n) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double s = 0.0;
  for (int j = 0; j < k; ++j) s = fma(h[j], V[(long)j * ldv + i], s);
  w[i] -= s;
}

cudaError_t maxpy(const double* V, long ldv, int k, const double* h, double* w, long n, cudaStream_t st) {
  k_maxpy<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(V, ldv, k, h, w, n);
  return cudaGetLastError();
}

// x += sum_{j<k} y[j] V_j  (y passed by value, k <= 64)
struct SmallVec { double v[64]; };
__global__ void k_mcombine(const double* __restrict__ V, long ldv, int k, const SmallVec y, double* __restrict__ x,
                           long n) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double s = 0.0;
  for (int j = 0; j < k; ++j) s = fma(y.v[j], V[(long)j * ldv + i], s);
  x[i] += s;
}

cudaError_t mcombine(const double* V, long ldv, int k, const double* y_host, double* x, long n, cudaStream_t st) {
  if (k > 64) return cudaErrorInvalidValue;
  SmallVec y{};
  for (int j = 0; j < k; ++j) y.v[j] = y_host[j];
  k_mcombine<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(V, ldv, k, y, x, n);
  return cudaGetLastError();
}

// y = a*x (+ y if add)   and   z = d .* x
__global__ void k_scale(double a, const double* __restrict__ x, double* __restrict__ y, long n) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) y[i] = a * x[i];
}
cudaError_t scale(double a, const double* x, double* y, long n, cudaStream_t st) {
  k_scale<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(a, x, y, n);
  return cudaGetLastError();
}
__global__ void k_dmul(const double* __restrict__ d, const double* __restrict__ x, double* __restrict__ z, long n) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) z[i] = d[i] * x[i];
}
cudaError_t dmul(const double* d, const double* x, double* z, long n, cudaStream_t st) {
  k_dmul<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(d, x, z, n);
  return cudaGetLastError();
}
// z = x - y
__global__ void k_sub(const double* __restrict__ x, const double* __restrict__ y, double* __restrict__ z, long n) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) z[i] = x[i] - y[i];
}
cudaError_t sub(const double* x, const double* y, double* z, long n, cudaStream_t st) {
  k_sub<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(x, y, z, n);
  return cudaGetLastError();
}

// out[0] = max |x| ; out[1] = max |x - y| (y may be null -> only out[0])
__device__ __forceinline__ double block_max(double v, double* sh) {
  const int t = threadIdx.x;
  sh[t] = v;
  __syncthreads();
#pragma unroll
  for (int s = RB / 2; s > 0; s >>= 1) {
    if (t < s) sh[t] = fmax(sh[t], sh[t + s]);
    __syncthreads();
  }
  return sh[0];
}
__global__ void k_maxabs2_partial(const double* __restrict__ x, const double* __restrict__ y, long n,
                                  double* __restrict__ partial) {
  __shared__ double sh[RB];
  double a = 0.0, b = 0.0;
  const long stride = (long)gridDim.x * RB;
  for (long i = (long)blockIdx.x * RB + threadIdx.x; i < n; i += stride) {
    a = fmax(a, fabs(x[i]));
    if (y) b = fmax(b, fabs(x[i] - y[i]));
  }
  double v = block_max(a, sh);
  if (threadIdx.x == 0) partial[blockIdx.x] = v;
  __syncthreads();
  v = block_max(b, sh);
  if (threadIdx.x == 0) partial[kMaxPartials + blockIdx.x] = v;
}
__global__ void k_maxabs2_final(const double* __restrict__ partial, int nb, double* out) {
  __shared__ double sh[RB];
  double a = 0.0, b = 0.0;
  for (int i = threadIdx.x; i < nb; i += RB) { a = fmax(a, partial[i]); b = fmax(b, partial[kMaxPartials + i]); }
  const double ma = block_max(a, sh);
  __syncthreads();
  const double mb = block_max(b, sh);
  if (threadIdx.x == 0) { out[0] = ma; out[1] = mb; }
}
cudaError_t maxabs2(const double* x, const double* y, long n, double* partial, double* out, cudaStream_t st) {
  const int nb = reduce_blocks(n);
  k_maxabs2_partial<<<nb, RB, 0, st>>>(x, y, n, partial);
  k_maxabs2_final<<<1, RB, 0, st>>>(partial, nb, out);
  return cudaGetLastError();
}

__global__ void k_cg_set_tol(KrylovState* s, const double* bb, double eps) { s->tol2 = eps * eps * bb[0]; }
cudaError_t cg_set_abs_tol(KrylovState* s, const double* bb, double eps, cudaStream_t st) {
  k_cg_set_tol<<<1, 1, 0, st>>>(s, bb, eps);
  return cudaGetLastError();
}

}  // namespace af
