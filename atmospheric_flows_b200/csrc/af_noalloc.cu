// af_noalloc.cu -- the Schur complement apply D p - C A^{-1} B p without device allocation.
//
// Some callers cannot call cudaMalloc: code that lives inside a framework whose caching
// allocator owns the device memory (a private cudaMalloc bypasses the pool, can fail once
// the pool has claimed the memory, and fragments it), and long time-stepping loops that
// budget device memory up front and must not allocate per step (cudaMalloc can fail in the
// middle of a run and may synchronize the device).  af_schur_apply_noalloc serves them: it
// needs no handle (af_create allocates), takes every input and output from the caller, and
// keeps its scratch (B p, A^{-1} B p, the inner-CG vectors, the inverse diagonal of A, the
// reduction partials and the solver state) in one file-scope __device__ array.
//
// Properties of that array: it exists once per GPU that loads the library and stays
// allocated until the process exits; it bounds the problem size (kNoAllocMaxScalar
// pressure DoFs); every call uses the same array, so calls that overlap on the GPU race
// with each other (enqueue them on one stream, or synchronize in between); it keeps the
// previous call's contents, so this file clears what must start at zero (the CG iterate)
// and overwrites everything else before reading it.
//
// The call returns once its work is done on the stream: the inner CG reads its state back every
// 8 iterations, and a last read of the kernels' status word (a bounded wait that gave up:
// AF_TIMEOUT) waits for C.
//
// Set-up: the first call on a device (with that device current) looks up the array's
// device address with cudaGetSymbolAddress and uploads the degree's basis tables; make
// that first call before any other work that must not be interrupted by set-up.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <mutex>

#include "../../include/af_gpu.h"
#include "af_blas.h"
#include "af_internal.h"

namespace af {
void set_last_error(const char* msg);
}

using namespace af;

namespace {

constexpr long kNoAllocMaxScalar = 65536;  // cells * (degree+1)^2
constexpr long kScratchDoubles = 14 * kNoAllocMaxScalar + 4 * kMaxPartials + 16;
constexpr int kMaxDevices = 64;

static __device__ __align__(256) double g_schur_scratch[kScratchDoubles];

std::mutex g_mu;
double* g_scratch_ptr[kMaxDevices] = {nullptr};
bool g_tables_ready[kMaxDevices][8] = {{false}};

constexpr const char* kTimeoutMessage =
    "af_schur_apply_noalloc: a kernel gave up a bounded wait for its staged inputs; dst is not valid";

int err(int code, const char* msg) {
  set_last_error(msg);
  return code;
}

}  // namespace

extern "C" int af_schur_apply_noalloc(int nx, int nz, int periodic_x, const double* vertices, int degree, double Mach,
                                      double dt, int hyperbolic_stage, const double* rho_for_fixed,
                                      const double* pres_fixed, const double* src, double* dst, void* stream,
                                      int* inner_iterations) {
  if (!vertices || !rho_for_fixed || !pres_fixed || !src || !dst)
    return err(AF_BAD_ARG, "af_schur_apply_noalloc: null pointer argument");
  if (nx < 1 || nz < 1 || hyperbolic_stage < 1 || hyperbolic_stage > 2 || !(Mach > 0) || !(dt > 0))
    return err(AF_BAD_ARG, "af_schur_apply_noalloc: bad mesh size, stage (1 or 2), Mach or dt");
  const DegreeOps* ops = degree_ops(degree);
  if (!ops) return err(AF_UNSUPPORTED, "af_schur_apply_noalloc: degree not compiled in");
  const long n = (long)nx * nz * (degree + 1) * (degree + 1);
  if (n > kNoAllocMaxScalar) {
    char buf[200];
    std::snprintf(buf, sizeof(buf),
                  "af_schur_apply_noalloc: %ld pressure DoFs exceed the static scratch limit of %ld "
                  "(cells*(degree+1)^2); use af_vmult with a handle",
                  n, kNoAllocMaxScalar);
    return err(AF_BAD_ARG, buf);
  }
  for (const void* p : {(const void*)vertices, (const void*)rho_for_fixed, (const void*)pres_fixed, (const void*)src,
                        (const void*)dst})
    if (reinterpret_cast<uintptr_t>(p) & 15u) return err(AF_BAD_ARG, "af_schur_apply_noalloc: pointers must be 16-byte aligned");
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices)
    return err(AF_NO_DEVICE, "af_schur_apply_noalloc: no current CUDA device");
  double* scratch = nullptr;
  {
    std::lock_guard<std::mutex> lock(g_mu);
    if (!g_scratch_ptr[dev]) {  // set-up once per device, with that device current
      double* ptr = nullptr;
      cudaError_t e = cudaGetSymbolAddress((void**)&ptr, g_schur_scratch);
      if (e != cudaSuccess) return err(AF_CUDA, cudaGetErrorString(e));
      g_scratch_ptr[dev] = ptr;
    }
    if (!g_tables_ready[dev][degree]) {
      if (ops->upload_tables() != cudaSuccess) return err(AF_CUDA, "af_schur_apply_noalloc: table upload failed");
      g_tables_ready[dev][degree] = true;
    }
    scratch = g_scratch_ptr[dev];
  }
  cudaStream_t st = (cudaStream_t)stream;
  const long nu = 2 * n;  // velocity-space length
  double* t1 = scratch;            // B p
  double* t2 = scratch + nu;       // A^{-1} B p (CG iterate)
  double* rv = scratch + 2 * nu;   // inner CG residual, preconditioned residual, direction, A p
  double* zv = scratch + 3 * nu;
  double* pv = scratch + 4 * nu;
  double* Ap = scratch + 5 * nu;
  double* invd = scratch + 6 * nu;  // inverse diagonal of A
  double* part = scratch + 7 * nu;  // reduction partials (4 * kMaxPartials)
  KrylovState* kst = reinterpret_cast<KrylovState*>(part + 4 * kMaxPartials);
  // the kernels' status word (a bounded wait that gave up), after the solver state in the
  // 16 reserved doubles
  static_assert(sizeof(KrylovState) <= 14 * sizeof(double), "solver state overlaps the status word");
  int* status = reinterpret_cast<int*>(part + 4 * kMaxPartials + 14);
  int h_status = 0;

  MeshDev mesh{};
  mesh.vtx = reinterpret_cast<const double2*>(vertices);
  mesh.nx = nx;
  mesh.nz = nz;
  mesh.periodic_x = periodic_x ? 1 : 0;
  mesh.status = status;
  const int ncell = nx * nz;
  // euler_operator.h:1428, 1526 and the tableau at :233-240
  const double gamma = 2.0 - std::sqrt(2.0);
  const double coeff = hyperbolic_stage == 1 ? 0.5 * gamma : 1.0 - std::sqrt(2.0) / 2.0;
  const int maxit = 10000;
  cudaError_t e;
  if ((e = cudaMemsetAsync(status, 0, sizeof(int), st)) != cudaSuccess ||
      (e = ops->inv_diag(mesh, 2, rho_for_fixed, 1.0, invd, ncell, st)) != cudaSuccess ||
      (e = ops->op_B(mesh, src, coeff * dt / (Mach * Mach), t1, ncell, st)) != cudaSuccess ||
      (e = cudaMemsetAsync(t2, 0, nu * sizeof(double), st)) != cudaSuccess ||
      (e = cg_start(kst, t1, nullptr, invd, rv, zv, pv, nu, part, 1e-12, 1, st)) != cudaSuccess)
    return err(AF_CUDA, cudaGetErrorString(e));
  KrylovState hs{};
  for (int it = 0; it < maxit; it += 8) {
    for (int k = 0; k < 8 && it + k < maxit; ++k) {
      if ((e = ops->mass(mesh, 2, pv, rho_for_fixed, 1.0, Ap, ncell, st)) != cudaSuccess ||
          (e = cg_after_apply(kst, t2, rv, zv, pv, Ap, invd, nu, part, maxit, st)) != cudaSuccess)
        return err(AF_CUDA, cudaGetErrorString(e));
    }
    if ((e = cudaMemcpyAsync(&hs, kst, sizeof(hs), cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
        (e = cudaMemcpyAsync(&h_status, status, sizeof(int), cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
        (e = cudaStreamSynchronize(st)) != cudaSuccess)
      return err(AF_CUDA, cudaGetErrorString(e));
    if (h_status != 0) return err(AF_TIMEOUT, kTimeoutMessage);
    if (hs.done) break;
  }
  if (inner_iterations) *inner_iterations = hs.its;
  if (hs.status == 2 || hs.status == 3) return err(AF_NAN, "af_schur_apply_noalloc: inner CG breakdown");
  if (!hs.done || hs.status == 1) return err(AF_NO_CONVERGENCE, "af_schur_apply_noalloc: inner CG did not converge");
  CParams cp;
  cp.cdt = coeff * dt;
  cp.g1 = 1.0 / (1.4 - 1.0);
  cp.gg = 1.4 / (1.4 - 1.0);
  if ((e = ops->op_C(mesh, t2, pres_fixed, src, cp, dst, ncell, st)) != cudaSuccess ||
      (e = cudaMemcpyAsync(&h_status, status, sizeof(int), cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
      (e = cudaStreamSynchronize(st)) != cudaSuccess)
    return err(AF_CUDA, cudaGetErrorString(e));
  if (h_status != 0) return err(AF_TIMEOUT, kTimeoutMessage);
  return AF_OK;
}
