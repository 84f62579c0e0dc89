// af_capi.cu -- the C ABI (include/af_gpu.h): handle, EULEROperator semantics, dispatch
// to the per-degree kernels, and the Schur complement orchestration.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/af_gpu.h"
#include "af_blas.h"
#include "af_handle.h"
#include "af_internal.h"

namespace af {

static const DegreeOps* g_ops[8] = {nullptr};

void register_degree(int p, const DegreeOps* ops) {
  if (p >= 0 && p < 8) g_ops[p] = ops;
}

const DegreeOps* degree_ops(int P) { return (P >= 1 && P <= 6) ? g_ops[P] : nullptr; }

}  // namespace af

using namespace af;

static thread_local std::string g_last_error;

static int fail(int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  std::vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_last_error = buf;
  return code;
}

#define AF_CU(call)                                                                                   \
  do {                                                                                                \
    cudaError_t e_ = (call);                                                                          \
    if (e_ != cudaSuccess) return fail(AF_CUDA, "%s: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__, __LINE__); \
  } while (0)

// A code that an earlier kernel of the handle left in its status word is reported by the next
// call (kernels run asynchronously: the call that queued them has returned by then).
#define AF_PENDING(o)                              \
  do {                                             \
    const int r_ = af::take_kernel_status(o);     \
    if (r_ != AF_OK) return r_;                   \
  } while (0)

namespace af {
int take_kernel_status(af_operator* o) {
  if (!o || !o->h_status) return AF_OK;
  volatile int* w = o->h_status;
  const int v = *w;
  if (v == 0) return AF_OK;
  *w = 0;
  return fail(AF_TIMEOUT,
              "a kernel gave up a bounded wait for its staged inputs (code %d) and did not write its outputs; "
              "the results of the calls queued since the last check are invalid",
              v);
}

int sync_checked(af_operator* o, cudaStream_t st) {
  const cudaError_t e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return fail(AF_CUDA, "cudaStreamSynchronize: %s", cudaGetErrorString(e));
  return take_kernel_status(o);
}
}  // namespace af

static void set_tableau(af_operator* o) {
  o->gamma = 2.0 - std::sqrt(2.0);
  o->a21 = o->gamma; o->a22 = 0.0; o->a31 = 0.5; o->a32 = 0.5; o->a33 = 0.0;
  o->a21t = 0.5 * o->gamma; o->a22t = 0.5 * o->gamma;
  o->a31t = std::sqrt(2.0) / 4.0; o->a32t = std::sqrt(2.0) / 4.0; o->a33t = 1.0 - std::sqrt(2.0) / 2.0;
  o->b1 = o->a31t; o->b2 = o->a32t; o->b3 = o->a33t;
}

static bool aligned16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; }

static RhsParams rhs_params(const af_operator* o, int stage) {
  RhsParams r{};
  r.dt = o->dt;
  r.Ma2 = o->Ma * o->Ma;
  r.invMa2 = 1.0 / r.Ma2;
  r.invFr2 = 1.0 / (o->Fr * o->Fr);
  r.Ma2Fr2 = r.Ma2 / (o->Fr * o->Fr);
  r.a2 = o->mesh.radial_a * o->mesh.radial_a;
  r.g1 = 1.0 / (1.4 - 1.0);
  r.gg = 1.4 / (1.4 - 1.0);
  r.radial = o->mesh.gravity == 1;
  r.sponge = (o->sp_rate > 0 || o->sp_rate_lat > 0) ? 1 : 0;
  r.sp_z0 = o->sp_z0; r.sp_z1 = o->sp_z1; r.sp_rate = o->sp_rate;
  r.sp_x0 = o->sp_x0; r.sp_x1 = o->sp_x1; r.sp_width = o->sp_width; r.sp_rate_lat = o->sp_rate_lat;
  r.sp_u = o->sp_u;
  if (stage == 1) {
    r.ca[0] = o->a21; r.ct[0] = o->a21t;
    r.cg[0] = o->a21t; r.cgI = o->a22t;
  } else if (stage == 2) {
    r.ca[0] = o->a31; r.ct[0] = o->a31t; r.ca[1] = o->a32; r.ct[1] = o->a32t;
    r.cg[0] = o->a31t; r.cg[1] = o->a32t; r.cgI = o->a33t;
  } else {
    r.ca[0] = r.ct[0] = r.cg[0] = o->b1;
    r.ca[1] = r.ct[1] = r.cg[1] = o->b2;
    r.ca[2] = r.ct[2] = r.cg[2] = o->b3;
    r.cgI = 0.0;
  }
  return r;
}

extern "C" {

const char* af_error_string(int s) {
  switch (s) {
    case AF_OK: return "ok";
    case AF_BAD_ARG: return "bad argument";
    case AF_CUDA: return "CUDA error";
    case AF_NO_CONVERGENCE: return "no convergence";
    case AF_NAN: return "NaN or Inf";
    case AF_UNSUPPORTED: return "unsupported degree";
    case AF_NO_DEVICE: return "no CUDA device";
    case AF_TIMEOUT: return "a kernel gave up a bounded wait";
    default: return "unknown status";
  }
}

const char* af_last_error_message(void) { return g_last_error.c_str(); }

int af_create(const af_mesh_desc* m, int degree, int nq, double Ma, double Fr, double dt, af_operator** out) {
  if (!m || !out || !m->vertices) return fail(AF_BAD_ARG, "af_create: null argument");
  *out = nullptr;
  if (m->nx < 1 || m->nz < 1) return fail(AF_BAD_ARG, "af_create: mesh needs nx, nz >= 1");
  if ((long)m->nx * m->nz > (1L << 30)) return fail(AF_BAD_ARG, "af_create: mesh too large");
  if (m->gravity != 0 && m->gravity != 1) return fail(AF_BAD_ARG, "af_create: gravity must be 0 or 1");
  if (nq != 2 * degree + 1) return fail(AF_BAD_ARG, "af_create: n_q_points_1d must be 2*degree+1");
  const DegreeOps* ops = degree_ops(degree);
  if (!ops) return fail(AF_UNSUPPORTED, "af_create: degree %d not compiled in", degree);
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return fail(AF_NO_DEVICE, "af_create: no CUDA device");
  }
  auto* o = new af_operator();
  o->ops = ops;
  o->P = degree;
  o->NQ = nq;
  o->nd = (degree + 1) * (degree + 1);
  o->ncell = m->nx * m->nz;
  o->Ma = Ma; o->Fr = Fr; o->dt = dt;
  set_tableau(o);
  auto cleanup = [&](int code) { af_destroy(o); return code; };
  if (cudaGetDevice(&o->device) != cudaSuccess) return cleanup(fail(AF_CUDA, "cudaGetDevice failed"));
  if (cudaStreamCreateWithFlags(&o->own_stream, cudaStreamNonBlocking) != cudaSuccess)
    return cleanup(fail(AF_CUDA, "stream creation failed"));
  o->stream = o->own_stream;
  if (ops->upload_tables() != cudaSuccess) return cleanup(fail(AF_CUDA, "table upload failed"));
  const size_t nv = (size_t)(m->nx + 1) * (m->nz + 1);
  const long ns = o->n_scalar();
  if (cudaMalloc(&o->d_vtx, nv * sizeof(double2)) != cudaSuccess ||
      cudaMalloc(&o->d_rho_fixed, ns * sizeof(double)) != cudaSuccess ||
      cudaMalloc(&o->d_pres_fixed, ns * sizeof(double)) != cudaSuccess ||
      cudaMalloc(&o->d_u_fixed, 2 * ns * sizeof(double)) != cudaSuccess ||
      cudaMalloc(&o->d_invdA, 2 * ns * sizeof(double)) != cudaSuccess ||
      cudaMalloc(&o->d_ws, 6 * 2 * ns * sizeof(double)) != cudaSuccess ||  // t1, t2, r, z, p, Ap
      cudaMalloc(&o->d_part, 4 * kMaxPartials * sizeof(double)) != cudaSuccess ||
      cudaMalloc(&o->d_kst, sizeof(KrylovState)) != cudaSuccess)
    return cleanup(fail(AF_CUDA, "device allocation failed"));
  if (cudaMemcpy(o->d_vtx, m->vertices, nv * sizeof(double2), cudaMemcpyHostToDevice) != cudaSuccess)
    return cleanup(fail(AF_CUDA, "vertex upload failed"));
  int* d_status = nullptr;
  if (cudaHostAlloc((void**)&o->h_status, sizeof(int), cudaHostAllocMapped | cudaHostAllocPortable) != cudaSuccess)
    return cleanup(fail(AF_CUDA, "status word allocation failed"));
  *o->h_status = 0;
  if (cudaHostGetDevicePointer((void**)&d_status, o->h_status, 0) != cudaSuccess)
    return cleanup(fail(AF_CUDA, "status word mapping failed"));
  o->mesh.status = d_status;
  o->mesh.vtx = o->d_vtx;
  o->mesh.nx = m->nx;
  o->mesh.nz = m->nz;
  o->mesh.periodic_x = m->periodic_x ? 1 : 0;
  o->mesh.gravity = m->gravity;
  o->mesh.radial_a = m->radial_a;
  *out = o;
  return AF_OK;
}

int af_destroy(af_operator* o) {
  if (!o) return AF_OK;
  cudaSetDevice(o->device);
  if (o->stream) cudaStreamSynchronize(o->stream);
  cudaFree(o->d_vtx);
  cudaFree(o->d_rho_fixed);
  cudaFree(o->d_pres_fixed);
  cudaFree(o->d_u_fixed);
  cudaFree(o->d_invdA);
  cudaFree(o->d_ws);
  cudaFree(o->d_part);
  cudaFree(o->d_kst);
  cudaFree(o->d_stage);
  cudaFree(o->d_Wm);
  cudaFree(o->d_La);
  if (o->h_status) cudaFreeHost(o->h_status);
  if (o->own_stream) cudaStreamDestroy(o->own_stream);
  if (o->copy_in) cudaStreamDestroy(o->copy_in);
  if (o->copy_out) cudaStreamDestroy(o->copy_out);
  if (o->ev_start) cudaEventDestroy(o->ev_start);
  for (int k = 0; k < af_operator::kHostChunks; ++k) {
    if (o->ev_in[k]) cudaEventDestroy(o->ev_in[k]);
    if (o->ev_done[k]) cudaEventDestroy(o->ev_done[k]);
  }
  delete o;
  return AF_OK;
}

int af_set_stream(af_operator* o, void* s) {
  if (!o) return fail(AF_BAD_ARG, "null handle");
  o->stream = s ? (cudaStream_t)s : o->own_stream;
  return AF_OK;
}

int af_synchronize(af_operator* o) {
  if (!o) return fail(AF_BAD_ARG, "null handle");
  return sync_checked(o, o->stream);
}

int af_set_sponge(af_operator* o, double z_start, double z_top, double rate_top, double x_left, double x_right,
                  double width_lateral, double rate_lateral, double u_ref) {
  if (!o) return fail(AF_BAD_ARG, "null handle");
  if (!(rate_top >= 0) || !(rate_lateral >= 0) || (rate_top > 0 && !(z_top > z_start)) ||
      (rate_lateral > 0 && (!(width_lateral > 0) || !(x_right > x_left))))
    return fail(AF_BAD_ARG, "af_set_sponge: need rates >= 0, z_top > z_start and width > 0, x_right > x_left "
                            "for the layers that are on");
  o->sp_z0 = z_start; o->sp_z1 = z_top; o->sp_rate = rate_top;
  o->sp_x0 = x_left; o->sp_x1 = x_right; o->sp_width = width_lateral; o->sp_rate_lat = rate_lateral;
  o->sp_u = u_ref;
  return AF_OK;
}

int af_set_stage_wait_test(af_operator* o, int polls) {
  if (!o || polls < 0) return fail(AF_BAD_ARG, "af_set_stage_wait_test: bad handle or negative poll count");
  o->mesh.test_wait_polls = polls;
  return AF_OK;
}

int af_set_dt(af_operator* o, double v) {
  if (!o || !(v > 0)) return fail(AF_BAD_ARG, "af_set_dt: bad handle or dt");
  o->dt = v;
  return AF_OK;
}
int af_set_Mach(af_operator* o, double v) {
  if (!o || !(v > 0)) return fail(AF_BAD_ARG, "af_set_Mach: bad handle or Mach");
  o->Ma = v;
  return AF_OK;
}
int af_set_Froude(af_operator* o, double v) {
  if (!o || !(v > 0)) return fail(AF_BAD_ARG, "af_set_Froude: bad handle or Froude");
  o->Fr = v;
  return AF_OK;
}
int af_set_HYPERBOLIC_stage(af_operator* o, int s) {  // AssertIndexRange(stage, 4), stage > 0
  if (!o || s < 1 || s > 3) return fail(AF_BAD_ARG, "HYPERBOLIC_stage must be 1..3");
  o->hs = s;
  return AF_OK;
}
int af_set_NS_stage(af_operator* o, int s) {  // AssertIndexRange(stage, 7), stage > 0
  if (!o || s < 1 || s > 6) return fail(AF_BAD_ARG, "NS_stage must be 1..6");
  o->ns = s;
  return AF_OK;
}

static int copy_fixed(af_operator* o, double* dst, const double* src, long n) {
  if (!o || !src) return fail(AF_BAD_ARG, "null argument");
  AF_CU(cudaSetDevice(o->device));
  AF_PENDING(o);
  AF_CU(cudaMemcpyAsync(dst, src, n * sizeof(double), cudaMemcpyDeviceToDevice, o->stream));
  return AF_OK;
}
int af_set_rho_for_fixed(af_operator* o, const double* v) {
  int r = copy_fixed(o, o ? o->d_rho_fixed : nullptr, v, o ? o->n_scalar() : 0);
  if (r == AF_OK) { o->rho_fixed_set = true; o->invdA_valid = false; o->La_valid = false; }
  return r;
}
int af_set_pres_fixed(af_operator* o, const double* v) {
  int r = copy_fixed(o, o ? o->d_pres_fixed : nullptr, v, o ? o->n_scalar() : 0);
  if (r == AF_OK) o->pres_fixed_set = true;
  return r;
}
int af_set_u_fixed(af_operator* o, const double* v) {
  return copy_fixed(o, o ? o->d_u_fixed : nullptr, v, o ? 2 * o->n_scalar() : 0);
}

// cells [cbeg, cend) (cend < 0: the whole mesh); cbeg must be a multiple of the degree's
// cells per CTA
static int run_rhs(af_operator* o, int mask, const RhsSources& s, double* d_rho, double* d_u, double* d_p,
                   int cbeg = 0, int cend = -1) {
  const double* ptrs[] = {s.rho[0], s.rho[1], s.rho[2], s.u[0], s.u[1], s.u[2], s.p[0], s.p[1], s.p[2], s.rho_c, s.u_fix,
                          d_rho, d_u, d_p};
  for (const double* p : ptrs)
    if (p && !aligned16(p)) return fail(AF_BAD_ARG, "device pointers must be 16-byte aligned");
  AF_CU(cudaSetDevice(o->device));
  AF_PENDING(o);
  const RhsParams prm = rhs_params(o, o->hs);
  MeshDev m = o->mesh;
  m.cell0 = cbeg;
  cudaError_t e = o->ops->rhs(m, o->hs, mask, s, prm, d_rho, d_u, d_p, cend < 0 ? o->ncell : cend, o->stream);
  if (e == cudaErrorInvalidValue) return fail(AF_BAD_ARG, "rhs: missing source or output for stage %d", o->hs);
  AF_CU(e);
  o->launches += 1;
  return AF_OK;
}

int af_vmult_rhs_rho_update(af_operator* o, double* dst, const double* const* src, int n) {
  if (!o || !dst || !src) return fail(AF_BAD_ARG, "null argument");
  if (n != 2 * o->hs) return fail(AF_BAD_ARG, "vmult_rhs_rho_update: stage %d expects %d sources, got %d", o->hs, 2 * o->hs, n);
  RhsSources s{};
  for (int j = 0; j < o->hs; ++j) { s.rho[j] = src[2 * j]; s.u[j] = src[2 * j + 1]; }
  return run_rhs(o, 1, s, dst, nullptr, nullptr);
}

int af_vmult_rhs_velocity_fixed(af_operator* o, double* dst, const double* const* src, int n) {
  if (!o || !dst || !src) return fail(AF_BAD_ARG, "null argument");
  const int need = o->hs == 1 ? 4 : (o->hs == 2 ? 7 : 9);
  if (n != need) return fail(AF_BAD_ARG, "vmult_rhs_velocity_fixed: stage %d expects %d sources, got %d", o->hs, need, n);
  RhsSources s{};
  for (int j = 0; j < o->hs; ++j) { s.rho[j] = src[3 * j]; s.u[j] = src[3 * j + 1]; s.p[j] = src[3 * j + 2]; }
  if (o->hs < 3) s.rho_c = src[3 * o->hs];
  return run_rhs(o, 2, s, nullptr, dst, nullptr);
}

static int pressure_sources(const af_operator* o, const double* const* src, int n, RhsSources& s) {
  const int need = 3 * o->hs + 2;
  if (n != need) return fail(AF_BAD_ARG, "vmult_rhs_pressure: stage %d expects %d sources, got %d", o->hs, need, n);
  s = RhsSources{};
  for (int j = 0; j < o->hs; ++j) { s.rho[j] = src[3 * j]; s.u[j] = src[3 * j + 1]; s.p[j] = src[3 * j + 2]; }
  s.rho_c = src[3 * o->hs];
  s.u_fix = src[3 * o->hs + 1];
  return AF_OK;
}

int af_vmult_rhs_pressure(af_operator* o, double* dst, const double* const* src, int n) {
  if (!o || !dst || !src) return fail(AF_BAD_ARG, "null argument");
  RhsSources s;
  int r = pressure_sources(o, src, n, s);
  if (r != AF_OK) return r;
  return run_rhs(o, 4, s, nullptr, nullptr, dst);
}

// the fused rhs over cells [cbeg, cend) (see run_rhs)
static int rhs_fused_range(af_operator* o, double* d_rho, double* d_u, double* d_p, const double* const* src, int n,
                           int cbeg, int cend) {
  if (!o || !src) return fail(AF_BAD_ARG, "null argument");
  const int mask = (d_rho ? 1 : 0) | (d_u ? 2 : 0) | (d_p ? 4 : 0);
  if (mask == 0) return fail(AF_BAD_ARG, "af_vmult_rhs_fused: no output requested");
  if (mask == 5 || mask == 3) {
    // rho+p or rho+u without the third: run as two launches
    RhsSources s;
    int r = pressure_sources(o, src, n, s);
    if (r != AF_OK) return r;
    r = run_rhs(o, 1, s, d_rho, nullptr, nullptr, cbeg, cend);
    if (r != AF_OK) return r;
    return run_rhs(o, mask & 6, s, nullptr, d_u, d_p, cbeg, cend);
  }
  RhsSources s;
  int r = pressure_sources(o, src, n, s);
  if (r != AF_OK) return r;
  if (mask == 2 && o->hs == 3) s.rho_c = nullptr;
  return run_rhs(o, mask, s, d_rho, d_u, d_p, cbeg, cend);
}

int af_vmult_rhs_fused(af_operator* o, double* d_rho, double* d_u, double* d_p, const double* const* src, int n) {
  return rhs_fused_range(o, d_rho, d_u, d_p, src, n, 0, -1);
}

// Stage 1: the hand-written adjoint / tangent kernels (RhsAdj1Phys, RhsTlm1Phys); stages 2 and
// 3: the dual-number kernels (RhsAdjGPhys per group, RhsTanPhys), which differentiate the
// forward physics itself.
int af_vmult_rhs_fused_backward(af_operator* o, const double* const* src, int n, const double* ybar_rho,
                                const double* ybar_u, const double* ybar_p, double* const* xbar) {
  if (!o || !src || !xbar || !ybar_rho || !ybar_u || !ybar_p) return fail(AF_BAD_ARG, "null argument");
  const int need = 3 * o->hs + 2;
  if (n != need) return fail(AF_BAD_ARG, "af_vmult_rhs_fused_backward: stage %d expects %d sources", o->hs, need);
  for (int k = 0; k < n; ++k)
    if (!src[k] || !xbar[k] || !aligned16(src[k]) || !aligned16(xbar[k]))
      return fail(AF_BAD_ARG, "af_vmult_rhs_fused_backward: null or unaligned vector");
  AF_CU(cudaSetDevice(o->device));
  AF_PENDING(o);
  if (o->hs == 1 && (o->sp_rate > 0 || o->sp_rate_lat > 0))
    return fail(AF_UNSUPPORTED, "af_vmult_rhs_fused_backward: the stage-1 adjoint kernel has no sponge term");
  const double* yb[3] = {ybar_rho, ybar_u, ybar_p};
  if (o->hs == 1) {
    AF_CU(o->ops->rhs_adjoint1(o->mesh, src, yb, xbar, rhs_params(o, 1), o->ncell, o->stream));
    o->launches += 1;
  } else {
    AF_CU(o->ops->rhs_adjoint(o->mesh, o->hs, src, yb, xbar, o->d_ws, rhs_params(o, o->hs), o->ncell, o->stream));
    o->launches += o->hs + 2;
  }
  return AF_OK;
}

int af_vmult_rhs_fused_tangent(af_operator* o, const double* const* src, int n, const double* const* dsrc,
                               double* d_rho, double* d_u, double* d_p) {
  if (!o || !src || !dsrc || !d_rho || !d_u || !d_p) return fail(AF_BAD_ARG, "null argument");
  const int need = 3 * o->hs + 2;
  if (n != need) return fail(AF_BAD_ARG, "af_vmult_rhs_fused_tangent: stage %d expects %d sources", o->hs, need);
  for (int k = 0; k < n; ++k)
    if (!src[k] || !dsrc[k] || !aligned16(src[k]) || !aligned16(dsrc[k]))
      return fail(AF_BAD_ARG, "af_vmult_rhs_fused_tangent: null or unaligned vector");
  AF_CU(cudaSetDevice(o->device));
  AF_PENDING(o);
  if (o->hs == 1 && (o->sp_rate > 0 || o->sp_rate_lat > 0))
    return fail(AF_UNSUPPORTED, "af_vmult_rhs_fused_tangent: the stage-1 tangent kernel has no sponge term");
  double* dy[3] = {d_rho, d_u, d_p};
  if (o->hs == 1)
    AF_CU(o->ops->rhs_tangent1(o->mesh, src, dsrc, dy, rhs_params(o, 1), o->ncell, o->stream));
  else
    AF_CU(o->ops->rhs_tangent(o->mesh, o->hs, src, dsrc, dy, rhs_params(o, o->hs), o->ncell, o->stream));
  o->launches += 1;
  return AF_OK;
}

int af_vmult_rhs_fused_host(af_operator* o, double* h_rho, double* h_u, double* h_p, const double* const* h_src, int n) {
  if (!o || !h_src) return fail(AF_BAD_ARG, "null argument");
  const int need = 3 * o->hs + 2;
  if (n != need) return fail(AF_BAD_ARG, "af_vmult_rhs_fused_host: stage %d expects %d sources", o->hs, need);
  const long ns = o->n_scalar();
  // lengths in the pressure-list order: rho, u, p per explicit stage, then rho_c, u_fix
  std::vector<long> len(n);
  for (int j = 0; j < o->hs; ++j) { len[3 * j] = ns; len[3 * j + 1] = 2 * ns; len[3 * j + 2] = ns; }
  len[3 * o->hs] = ns;
  len[3 * o->hs + 1] = 2 * ns;
  auto up2 = [](long v) { return (v + 1) & ~1L; };  // keep every staged vector 16-byte aligned
  size_t total = up2(ns) + 2 * ns + up2(ns);         // outputs: rho, u (2), p
  for (long l : len) total += up2(l);
  AF_CU(cudaSetDevice(o->device));
  AF_PENDING(o);
  if (o->stage_len < total) {
    cudaFree(o->d_stage);
    o->d_stage = nullptr;
    AF_CU(cudaMalloc(&o->d_stage, total * sizeof(double)));
    o->stage_len = total;
  }
  // Rows of cells go through in chunks so that the copies overlap the kernel: the sources of
  // chunk k+1 travel (copy_in) while chunk k is computed (the operator's stream) and chunk
  // k-1's results return (copy_out).  A chunk's kernel also reads the row of cells above it
  // (face neighbours), so it starts once the next chunk's sources are in.  Chunk boundaries
  // are multiples of the kernel's cells per CTA; otherwise the call runs as one chunk.
  const int nx = o->mesh.nx, nz = o->mesh.nz, cpb = o->ops->cells_per_block;
  int rpc = (nz + af_operator::kHostChunks - 1) / af_operator::kHostChunks;  // rows per chunk
  if (((long)rpc * nx) % cpb != 0) rpc = nz;
  const int K = (nz + rpc - 1) / rpc;
  if (!o->copy_in) AF_CU(cudaStreamCreateWithFlags(&o->copy_in, cudaStreamNonBlocking));
  if (!o->copy_out) AF_CU(cudaStreamCreateWithFlags(&o->copy_out, cudaStreamNonBlocking));
  if (!o->ev_start) {
    AF_CU(cudaEventCreateWithFlags(&o->ev_start, cudaEventDisableTiming));
    for (int k = 0; k < af_operator::kHostChunks; ++k) {
      AF_CU(cudaEventCreateWithFlags(&o->ev_in[k], cudaEventDisableTiming));
      AF_CU(cudaEventCreateWithFlags(&o->ev_done[k], cudaEventDisableTiming));
    }
  }
  std::vector<double*> d_src(n);
  double* cur = o->d_stage;
  for (int k = 0; k < n; ++k) {
    if (!h_src[k]) return fail(AF_BAD_ARG, "af_vmult_rhs_fused_host: null source %d", k);
    d_src[k] = cur;
    cur += up2(len[k]);
  }
  double* d_rho = h_rho ? cur : nullptr;
  double* d_u = h_u ? cur + up2(ns) : nullptr;
  double* d_p = h_p ? cur + up2(ns) + 2 * ns : nullptr;
  const long nd = o->nd;
  // the staging buffer is reused: copies start after earlier work on the operator's stream
  AF_CU(cudaEventRecord(o->ev_start, o->stream));
  AF_CU(cudaStreamWaitEvent(o->copy_in, o->ev_start, 0));
  AF_CU(cudaStreamWaitEvent(o->copy_out, o->ev_start, 0));
  for (int c = 0; c < K; ++c) {
    const long c0 = (long)c * rpc * nx, c1 = std::min<long>((long)(c + 1) * rpc, nz) * nx;
    for (int k = 0; k < n; ++k) {
      const long comps = len[k] / ns, off = c0 * comps * nd, cnt = (c1 - c0) * comps * nd;
      AF_CU(cudaMemcpyAsync(d_src[k] + off, h_src[k] + off, cnt * sizeof(double), cudaMemcpyHostToDevice,
                            o->copy_in));
    }
    AF_CU(cudaEventRecord(o->ev_in[c], o->copy_in));
  }
  std::vector<const double*> d_srcc(d_src.begin(), d_src.end());
  for (int c = 0; c < K; ++c) {
    const long c0 = (long)c * rpc * nx, c1 = std::min<long>((long)(c + 1) * rpc, nz) * nx;
    AF_CU(cudaStreamWaitEvent(o->stream, o->ev_in[std::min(c + 1, K - 1)], 0));
    const int r = rhs_fused_range(o, d_rho, d_u, d_p, d_srcc.data(), n, (int)c0, (int)c1);
    if (r != AF_OK) {  // nothing may still read or write the caller's host buffers
      cudaStreamSynchronize(o->copy_in);
      cudaStreamSynchronize(o->stream);
      cudaStreamSynchronize(o->copy_out);
      return r;
    }
    AF_CU(cudaEventRecord(o->ev_done[c], o->stream));
    AF_CU(cudaStreamWaitEvent(o->copy_out, o->ev_done[c], 0));
    const long cnt = (c1 - c0) * nd;
    if (h_rho)
      AF_CU(cudaMemcpyAsync(h_rho + c0 * nd, d_rho + c0 * nd, cnt * sizeof(double), cudaMemcpyDeviceToHost,
                            o->copy_out));
    if (h_u)
      AF_CU(cudaMemcpyAsync(h_u + 2 * c0 * nd, d_u + 2 * c0 * nd, 2 * cnt * sizeof(double), cudaMemcpyDeviceToHost,
                            o->copy_out));
    if (h_p)
      AF_CU(cudaMemcpyAsync(h_p + c0 * nd, d_p + c0 * nd, cnt * sizeof(double), cudaMemcpyDeviceToHost, o->copy_out));
  }
  AF_CU(cudaStreamSynchronize(o->copy_out));
  return sync_checked(o, o->stream);
}

static double coeff_BC(const af_operator* o) { return o->hs == 1 ? o->a22t : o->a33t; }  // :1428, 1526

int af_vmult_pressure(af_operator* o, double* dst, const double* src) {
  if (!o || !dst || !src) return fail(AF_BAD_ARG, "null argument");
  if (!aligned16(dst) || !aligned16(src)) return fail(AF_BAD_ARG, "device pointers must be 16-byte aligned");
  AF_CU(cudaSetDevice(o->device));
  AF_PENDING(o);
  AF_CU(o->ops->op_B(o->mesh, src, coeff_BC(o) * o->dt / (o->Ma * o->Ma), dst, o->ncell, o->stream));
  o->launches += 1;
  return AF_OK;
}

static CParams c_params(const af_operator* o) {
  CParams c;
  c.cdt = coeff_BC(o) * o->dt;
  c.g1 = 1.0 / (1.4 - 1.0);
  c.gg = 1.4 / (1.4 - 1.0);
  return c;
}

int af_vmult_enthalpy(af_operator* o, double* dst, const double* src) {
  if (!o || !dst || !src) return fail(AF_BAD_ARG, "null argument");
  if (!o->pres_fixed_set) return fail(AF_BAD_ARG, "vmult_enthalpy: set_pres_fixed first");
  if (!aligned16(dst) || !aligned16(src)) return fail(AF_BAD_ARG, "device pointers must be 16-byte aligned");
  AF_CU(cudaSetDevice(o->device));
  AF_PENDING(o);
  AF_CU(o->ops->op_C(o->mesh, src, o->d_pres_fixed, nullptr, c_params(o), dst, o->ncell, o->stream));
  o->launches += 1;
  return AF_OK;
}

static int ensure_invdA(af_operator* o) {
  if (o->invdA_valid) return AF_OK;
  if (!o->rho_fixed_set) return fail(AF_BAD_ARG, "set_rho_for_fixed first");
  AF_CU(o->ops->inv_diag(o->mesh, 2, o->d_rho_fixed, 1.0, o->d_invdA, o->ncell, o->stream));
  o->launches += 1;
  o->invdA_valid = true;
  return AF_OK;
}

// x = A^{-1} b by CG + Jacobi, tol = rel_tol |b| (x starts at 0), as SolverCG in apply_add
static int solve_A(af_operator* o, double* x, const double* b) {
  const long n = 2 * o->n_scalar();
  int r = ensure_invdA(o);
  if (r != AF_OK) return r;
  double* ws = o->d_ws + 2 * n;  // r, z, p, Ap
  double *rv = ws, *zv = ws + n, *pv = ws + 2 * n, *Ap = ws + 3 * n;
  AF_CU(cudaMemsetAsync(x, 0, n * sizeof(double), o->stream));
  // tol2 preset relative to |b| = |r0|
  AF_CU(cg_start(o->d_kst, b, nullptr, o->d_invdA, rv, zv, pv, n, o->d_part, o->schur_tol, 1, o->stream));
  o->launches += 3;
  const int chunk = 8;
  KrylovState hs{};
  for (int it = 0; it < o->schur_maxit; it += chunk) {
    for (int k = 0; k < chunk && it + k < o->schur_maxit; ++k) {
      AF_CU(o->ops->mass(o->mesh, 2, pv, o->d_rho_fixed, 1.0, Ap, o->ncell, o->stream));
      AF_CU(cg_after_apply(o->d_kst, x, rv, zv, pv, Ap, o->d_invdA, n, o->d_part, o->schur_maxit, o->stream));
      o->launches += 6;
    }
    AF_CU(cudaMemcpyAsync(&hs, o->d_kst, sizeof(hs), cudaMemcpyDeviceToHost, o->stream));
    const int rs = sync_checked(o, o->stream);
    if (rs != AF_OK) return rs;
    if (hs.done) break;
  }
  o->last_inner_its = hs.its;
  if (hs.status == 3 || hs.status == 2) return fail(AF_NAN, "inner CG breakdown (status %d)", hs.status);
  if (!hs.done || hs.status == 1) return fail(AF_NO_CONVERGENCE, "inner CG: no convergence in %d iterations", hs.its);
  return AF_OK;
}

// Packed inverses of the cell mass matrices (built on first use)
// packed exact inverses of A (rho_for_fixed); M uses the change of basis instead
static int ensure_factor(af_operator* o) {
  if (o->La_valid) return AF_OK;
  if (!o->rho_fixed_set) return fail(AF_BAD_ARG, "set_rho_for_fixed first");
  if (!o->d_La) AF_CU(cudaMalloc(&o->d_La, sizeof(double) * (size_t)o->ncell * o->ops->factor_len));
  AF_CU(o->ops->mass_factor(o->mesh, o->d_rho_fixed, o->d_La, o->ncell, o->stream));
  o->launches += 1;
  o->La_valid = true;
  return AF_OK;
}

// Gauss-point weights of M for its inverse by the change of basis (exact on bilinear cells:
// M_K = (V x V)^T diag(JxW) (V x V) with V the nodal basis at the P+1 Gauss points)
static int ensure_mass_weights(af_operator* o) {
  if (o->Wm_valid) return AF_OK;
  if (!o->d_Wm) AF_CU(cudaMalloc(&o->d_Wm, sizeof(double) * (size_t)o->n_scalar()));
  AF_CU(o->ops->cob_weights_d(o->mesh, nullptr, o->d_Wm, o->ncell, o->stream));
  o->launches += 1;
  o->Wm_valid = true;
  return AF_OK;
}

int af_vmult_inverse(af_operator* o, double* dst, const double* src) {
  if (!o || !dst || !src) return fail(AF_BAD_ARG, "null argument");
  const int ns = o->ns;
  if (ns == 2) return fail(AF_BAD_ARG, "af_vmult_inverse: NS_stage 2 (Schur complement) has no cell-wise inverse");
  AF_CU(cudaSetDevice(o->device));
  AF_PENDING(o);
  if (ns == 3 || ns == 5) {  // A: packed exact inverses (rho-weighted, rebuilt per rho_for_fixed)
    const int r = ensure_factor(o);
    if (r != AF_OK) return r;
    AF_CU(o->ops->mass_solve(o->d_La, 2, src, 1.0, dst, o->ncell, o->mesh.status, o->stream));
  } else {  // M (NS 1/4) and D = M/(gamma-1) (NS 6): change of basis, no stored matrices
    const int r = ensure_mass_weights(o);
    if (r != AF_OK) return r;
    AF_CU(o->ops->cob_solve_d(o->d_Wm, 1, src, ns == 6 ? (1.4 - 1.0) : 1.0, dst, o->ncell, o->stream));
  }
  o->launches += 1;
  return AF_OK;
}

int af_vmult(af_operator* o, double* dst, const double* src) {
  if (!o || !dst || !src) return fail(AF_BAD_ARG, "null argument");
  if (!aligned16(dst) || !aligned16(src)) return fail(AF_BAD_ARG, "device pointers must be 16-byte aligned");
  AF_CU(cudaSetDevice(o->device));
  AF_PENDING(o);
  const int ns = o->ns;
  if (ns == 1 || ns == 4) {
    AF_CU(o->ops->mass(o->mesh, 1, src, nullptr, 1.0, dst, o->ncell, o->stream));
    o->launches += 1;
    return AF_OK;
  }
  if (ns == 6) {
    AF_CU(o->ops->mass(o->mesh, 1, src, nullptr, 1.0 / (1.4 - 1.0), dst, o->ncell, o->stream));
    o->launches += 1;
    return AF_OK;
  }
  if (ns == 3 || ns == 5) {
    if (!o->rho_fixed_set) return fail(AF_BAD_ARG, "set_rho_for_fixed first");
    AF_CU(o->ops->mass(o->mesh, 2, src, o->d_rho_fixed, 1.0, dst, o->ncell, o->stream));
    o->launches += 1;
    return AF_OK;
  }
  // NS 2: Schur complement D p - C A^{-1} B p  (euler_operator.h:2374-2408)
  if (!o->rho_fixed_set || !o->pres_fixed_set) return fail(AF_BAD_ARG, "Schur apply needs rho_for_fixed and pres_fixed");
  const long n = 2 * o->n_scalar();
  double* t1 = o->d_ws;
  double* t2 = o->d_ws + n;
  // B and the cell-wise A^{-1} stay two launches in FP64: a fused kernel holding the CTA's
  // inverses in shared memory measured slower (504 vs 417 us at 1024x256, p = 4)
  AF_CU(o->ops->op_B(o->mesh, src, coeff_BC(o) * o->dt / (o->Ma * o->Ma), t1, o->ncell, o->stream));
  o->launches += 1;
  int r;
  if (o->schur_mode == 1) {  // exact cell-wise A^{-1}
    r = ensure_factor(o);
    if (r != AF_OK) return r;
    AF_CU(o->ops->mass_solve(o->d_La, 2, t1, 1.0, t2, o->ncell, o->mesh.status, o->stream));
    o->launches += 1;
    o->last_inner_its = 0;
  } else {
    r = solve_A(o, t2, t1);
    if (r != AF_OK) return r;
  }
  AF_CU(o->ops->op_C(o->mesh, t2, o->d_pres_fixed, src, c_params(o), dst, o->ncell, o->stream));
  o->launches += 1;
  return AF_OK;
}

int af_compute_diagonal(af_operator* o, double* inv_diag) {
  if (!o || !inv_diag) return fail(AF_BAD_ARG, "null argument");
  AF_CU(cudaSetDevice(o->device));
  AF_PENDING(o);
  const int ns = o->ns;
  if (ns == 1 || ns == 4) AF_CU(o->ops->inv_diag(o->mesh, 1, nullptr, 1.0, inv_diag, o->ncell, o->stream));
  else if (ns == 2 || ns == 6) AF_CU(o->ops->inv_diag(o->mesh, 1, nullptr, 1.0 / (1.4 - 1.0), inv_diag, o->ncell, o->stream));
  else {
    if (!o->rho_fixed_set) return fail(AF_BAD_ARG, "set_rho_for_fixed first");
    AF_CU(o->ops->inv_diag(o->mesh, 2, o->d_rho_fixed, 1.0, inv_diag, o->ncell, o->stream));
  }
  o->launches += 1;
  return AF_OK;
}

int af_set_schur_mode(af_operator* o, int mode, double rel_tol, int max_iter) {
  if (!o || mode < 0 || mode > 1 || !(rel_tol > 0) || max_iter < 1)
    return fail(AF_BAD_ARG, "af_set_schur_mode: bad argument");
  o->schur_mode = mode;
  o->schur_tol = rel_tol;
  o->schur_maxit = max_iter;
  return AF_OK;
}

int af_last_inner_iterations(const af_operator* o, int* its) {
  if (!o || !its) return fail(AF_BAD_ARG, "null argument");
  *its = o->last_inner_its;
  return AF_OK;
}

int af_n_dofs(const af_operator* o, int space, long long* n) {
  if (!o || !n || space < 0 || space > 2) return fail(AF_BAD_ARG, "af_n_dofs: bad argument");
  *n = (long long)o->n_scalar() * (space == 0 ? 2 : 1);
  return AF_OK;
}

int af_launch_count(const af_operator* o, long long* n) {
  if (!o || !n) return fail(AF_BAD_ARG, "null argument");
  *n = o->launches;
  return AF_OK;
}


// ------------------------------------------------------------- tangents and transposes
// of the implicit operators (no counterpart in the reference): the pieces of an adjoint
// pressure solve.  A^{-1} is always the exact cell-wise inverse here.

int af_vmult_pressure_transpose(af_operator* o, double* pbar, const double* ubar) {
  if (!o || !pbar || !ubar) return fail(AF_BAD_ARG, "null argument");
  if (!aligned16(pbar) || !aligned16(ubar)) return fail(AF_BAD_ARG, "device pointers must be 16-byte aligned");
  AF_CU(cudaSetDevice(o->device));
  AF_PENDING(o);
  AF_CU(o->ops->op_BT(o->mesh, ubar, coeff_BC(o) * o->dt / (o->Ma * o->Ma), pbar, o->ncell, o->stream));
  o->launches += 1;
  return AF_OK;
}

int af_vmult_enthalpy_tangent(af_operator* o, double* dst, const double* w, const double* dw) {
  if (!o || !dst || !w || !dw) return fail(AF_BAD_ARG, "null argument");
  if (!o->pres_fixed_set) return fail(AF_BAD_ARG, "set_pres_fixed first");
  if (!aligned16(dst) || !aligned16(w) || !aligned16(dw)) return fail(AF_BAD_ARG, "device pointers must be 16-byte aligned");
  AF_CU(cudaSetDevice(o->device));
  AF_PENDING(o);
  AF_CU(o->ops->op_C_tangent(o->mesh, w, dw, o->d_pres_fixed, c_params(o), dst, o->ncell, o->stream));
  o->launches += 1;
  return AF_OK;
}

int af_vmult_enthalpy_transpose(af_operator* o, double* wbar, const double* w, const double* pbar) {
  if (!o || !wbar || !w || !pbar) return fail(AF_BAD_ARG, "null argument");
  if (!o->pres_fixed_set) return fail(AF_BAD_ARG, "set_pres_fixed first");
  if (!aligned16(wbar) || !aligned16(w) || !aligned16(pbar)) return fail(AF_BAD_ARG, "device pointers must be 16-byte aligned");
  AF_CU(cudaSetDevice(o->device));
  AF_PENDING(o);
  AF_CU(o->ops->op_CT(o->mesh, w, o->d_pres_fixed, pbar, c_params(o), wbar, o->ncell, o->stream));
  o->launches += 1;
  return AF_OK;
}

int af_vmult_velocity_mass_rho_transpose(af_operator* o, double* rhobar, const double* x, const double* y) {
  if (!o || !rhobar || !x || !y) return fail(AF_BAD_ARG, "null argument");
  if (!aligned16(rhobar) || !aligned16(x) || !aligned16(y)) return fail(AF_BAD_ARG, "device pointers must be 16-byte aligned");
  AF_CU(cudaSetDevice(o->device));
  AF_PENDING(o);
  AF_CU(o->ops->op_A_rho_T(o->mesh, x, y, rhobar, o->ncell, o->stream));
  o->launches += 1;
  return AF_OK;
}

int af_vmult_enthalpy_pf_transpose(af_operator* o, double* pfbar, const double* w, const double* pbar) {
  if (!o || !pfbar || !w || !pbar) return fail(AF_BAD_ARG, "null argument");
  if (!aligned16(pfbar) || !aligned16(w) || !aligned16(pbar)) return fail(AF_BAD_ARG, "device pointers must be 16-byte aligned");
  AF_CU(cudaSetDevice(o->device));
  AF_PENDING(o);
  AF_CU(o->ops->op_C_pf_T(o->mesh, w, pbar, c_params(o), pfbar, o->ncell, o->stream));
  o->launches += 1;
  return AF_OK;
}

// w = A^{-1} B p into the workspace (2 ns), exact inverse
static int schur_w(af_operator* o, const double* p, double* w, double* t) {
  AF_CU(o->ops->op_B(o->mesh, p, coeff_BC(o) * o->dt / (o->Ma * o->Ma), t, o->ncell, o->stream));
  int r = ensure_factor(o);
  if (r != AF_OK) return r;
  AF_CU(o->ops->mass_solve(o->d_La, 2, t, 1.0, w, o->ncell, o->mesh.status, o->stream));
  o->launches += 2;
  return AF_OK;
}

int af_schur_tangent(af_operator* o, double* dst, const double* p, const double* dp) {
  if (!o || !dst || !p || !dp) return fail(AF_BAD_ARG, "null argument");
  if (!o->rho_fixed_set || !o->pres_fixed_set) return fail(AF_BAD_ARG, "set rho_for_fixed and pres_fixed first");
  if (!aligned16(dst) || !aligned16(p) || !aligned16(dp)) return fail(AF_BAD_ARG, "device pointers must be 16-byte aligned");
  AF_CU(cudaSetDevice(o->device));
  AF_PENDING(o);
  const long n = o->n_scalar();
  double *w = o->d_ws, *z = o->d_ws + 2 * n, *t = o->d_ws + 4 * n, *c = o->d_ws + 6 * n;
  int r = schur_w(o, p, w, t);
  if (r == AF_OK) r = schur_w(o, dp, z, t);
  if (r != AF_OK) return r;
  AF_CU(o->ops->op_C_tangent(o->mesh, w, z, o->d_pres_fixed, c_params(o), c, o->ncell, o->stream));
  AF_CU(o->ops->mass(o->mesh, 1, dp, nullptr, 1.0 / (1.4 - 1.0), dst, o->ncell, o->stream));  // D dp
  AF_CU(axpby(-1.0, c, 1.0, dst, n, o->stream));
  o->launches += 3;
  return AF_OK;
}

int af_schur_transpose(af_operator* o, double* dst, const double* p, const double* pbar) {
  if (!o || !dst || !p || !pbar) return fail(AF_BAD_ARG, "null argument");
  if (!o->rho_fixed_set || !o->pres_fixed_set) return fail(AF_BAD_ARG, "set rho_for_fixed and pres_fixed first");
  if (!aligned16(dst) || !aligned16(p) || !aligned16(pbar)) return fail(AF_BAD_ARG, "device pointers must be 16-byte aligned");
  AF_CU(cudaSetDevice(o->device));
  AF_PENDING(o);
  const long n = o->n_scalar();
  double *w = o->d_ws, *t = o->d_ws + 2 * n, *t2 = o->d_ws + 4 * n, *q = o->d_ws + 6 * n;
  int r = schur_w(o, p, w, t);
  if (r != AF_OK) return r;
  AF_CU(o->ops->op_CT(o->mesh, w, o->d_pres_fixed, pbar, c_params(o), t, o->ncell, o->stream));  // J_C^T pbar
  AF_CU(o->ops->mass_solve(o->d_La, 2, t, 1.0, t2, o->ncell, o->mesh.status, o->stream));                        // A^{-1} (A = A^T)
  AF_CU(o->ops->op_BT(o->mesh, t2, coeff_BC(o) * o->dt / (o->Ma * o->Ma), q, o->ncell, o->stream));
  AF_CU(o->ops->mass(o->mesh, 1, pbar, nullptr, 1.0 / (1.4 - 1.0), dst, o->ncell, o->stream));    // D = D^T
  AF_CU(axpby(-1.0, q, 1.0, dst, n, o->stream));
  o->launches += 5;
  return AF_OK;
}

}  // extern "C"

namespace af {
// Lets other translation units of the library report through af_last_error_message().
void set_last_error(const char* msg) { g_last_error = msg; }
}  // namespace af

namespace af {
// The operator's packed cell inverses of A (rho_for_fixed), built if needed; used by the FP64
// pressure solver's finest level instead of factorising the same matrices again.
int mass_inverse_A(af_operator* o, const double** out) {
  const int r = ensure_factor(o);
  if (r != AF_OK) return r;
  *out = o->d_La;
  return AF_OK;
}
}  // namespace af
