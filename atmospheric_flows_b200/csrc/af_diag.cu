// af_diag.cu -- diagnostics of the reference's time loop on the device.
//
//   get_max_velocity / get_min_density / get_max_density / compute_max_celerity
//   (Atmospheric_Flow.cc:991-1087): the reference evaluates them with QGaussLobatto(p+1),
//   whose points are the DG support points, so they are reductions over nodal values:
//     max |u|,  min rho,  max |rho|,  max sqrt(gamma p / rho);
//   GridTools::minimal_cell_diameter (the CFL numbers, :1224-1235): min over cells of the
//   longer diagonal of the mapped cell;
//   integrate_difference(..., QGauss(p+1), L2_norm) of analyze_results (:925-985): the L2
//   norm of a field over the mesh, sum over cells and Gauss points of |v|^2 JxW.
#include <cuda_runtime.h>

#include <cmath>
#include <string>
#include <vector>

#include "../../include/af_gpu.h"
#include "af_handle.h"

namespace af {
void set_last_error(const char* msg);
}
using namespace af;

namespace {

int derr(int code, const std::string& msg) {
  set_last_error(msg.c_str());
  return code;
}
#define DG_CU(call)                                                                                   \
  do {                                                                                                \
    cudaError_t e_ = (call);                                                                          \
    if (e_ != cudaSuccess) return derr(AF_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_));   \
  } while (0)

constexpr int kThreads = 256;
constexpr int kBlocks = 592;  // 4 x 148 SMs; 5 partials per block fit the handle's partial array
constexpr int kNV = 5;        // max|u|, -min rho, max|rho|, max celerity, -min diameter

__device__ __forceinline__ void block_max(double (&v)[kNV], double* red) {
  for (int k = 0; k < kNV; ++k)
    for (int o = 16; o > 0; o >>= 1) v[k] = fmax(v[k], __shfl_down_sync(0xffffffffu, v[k], o));
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  if (l == 0)
    for (int k = 0; k < kNV; ++k) red[k * (kThreads / 32) + w] = v[k];
  __syncthreads();
  if (w == 0) {
    for (int k = 0; k < kNV; ++k) {
      v[k] = l < kThreads / 32 ? red[k * (kThreads / 32) + l] : -INFINITY;
      for (int o = 16; o > 0; o >>= 1) v[k] = fmax(v[k], __shfl_down_sync(0xffffffffu, v[k], o));
    }
  }
}

// all five quantities as maxima (minima negated); partial[k * gridDim.x + block]
__global__ void k_diag_partial(const double* __restrict__ rho_c, const double* __restrict__ rho_s,
                               const double* __restrict__ u, const double* __restrict__ p, const double2* __restrict__ vtx,
                               const int nx, const int ncell, const int nd, double* __restrict__ partial) {
  __shared__ double red[kNV * (kThreads / 32)];
  double v[kNV] = {-INFINITY, -INFINITY, -INFINITY, -INFINITY, -INFINITY};
  const long n = (long)ncell * nd;
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    const long c = i / nd, k = i % nd;
    const double ux = u[c * 2 * nd + k], uz = u[c * 2 * nd + nd + k];
    v[0] = fmax(v[0], sqrt(ux * ux + uz * uz));
    v[1] = fmax(v[1], -rho_s[i]);
    v[2] = fmax(v[2], fabs(rho_s[i]));
    v[3] = fmax(v[3], sqrt(1.4 * p[i] / rho_c[i]));
  }
  const int W = nx + 1;
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < ncell; c += gridDim.x * blockDim.x) {
    const int i = c % nx, j = c / nx;
    const double2 a = vtx[j * W + i], b = vtx[j * W + i + 1], d = vtx[(j + 1) * W + i], e = vtx[(j + 1) * W + i + 1];
    const double d1 = hypot(e.x - a.x, e.y - a.y), d2 = hypot(d.x - b.x, d.y - b.y);
    v[4] = fmax(v[4], -fmax(d1, d2));
  }
  block_max(v, red);
  if (threadIdx.x == 0)
    for (int k = 0; k < kNV; ++k) partial[k * gridDim.x + blockIdx.x] = v[k];
}

__global__ void k_diag_final(const double* __restrict__ partial, int nb, double* __restrict__ out) {
  __shared__ double red[kNV * (kThreads / 32)];
  double v[kNV] = {-INFINITY, -INFINITY, -INFINITY, -INFINITY, -INFINITY};
  for (int b = threadIdx.x; b < nb; b += blockDim.x)
    for (int k = 0; k < kNV; ++k) v[k] = fmax(v[k], partial[k * nb + b]);
  block_max(v, red);
  if (threadIdx.x == 0)
    for (int k = 0; k < kNV; ++k) out[k] = v[k];
}

// 1D tables of the L2 norm: Lagrange basis of the Gauss-Lobatto nodes at QGauss(p+1)
struct L2Tab {
  double B[7][7];  // B[q][i] = l_i(x_q)
  double x[7], w[7];
  int P1;
};

// one thread per cell: sum_q |v(x_q)|^2 JxW(q), ncomp components per cell; partial per block
__global__ void k_l2_partial(const double* __restrict__ v, const double2* __restrict__ vtx, const int nx,
                             const int ncell, const int ncomp, const L2Tab tb, double* __restrict__ partial) {
  __shared__ double red[kThreads / 32];
  const int P1 = tb.P1, ND = P1 * P1;
  double s = 0.0;
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < ncell; c += gridDim.x * blockDim.x) {
    const int i = c % nx, j = c / nx, W = nx + 1;
    const double2 v0 = vtx[j * W + i], v1 = vtx[j * W + i + 1];
    const double2 v2 = vtx[(j + 1) * W + i], v3 = vtx[(j + 1) * W + i + 1];
    const double Ax = v1.x - v0.x, Az = v1.y - v0.y, Cx = v2.x - v0.x, Cz = v2.y - v0.y;
    const double Bx = v3.x - v2.x - v1.x + v0.x, Bz = v3.y - v2.y - v1.y + v0.y;
    for (int d = 0; d < ncomp; ++d) {
      const double* f = v + ((size_t)c * ncomp + d) * ND;
      for (int qz = 0; qz < P1; ++qz) {
        double row[7];
        for (int ix = 0; ix < P1; ++ix) {  // contract along z first
          double t = 0.0;
          for (int iz = 0; iz < P1; ++iz) t = fma(tb.B[qz][iz], f[iz * P1 + ix], t);
          row[ix] = t;
        }
        const double eta = tb.x[qz];
        for (int qx = 0; qx < P1; ++qx) {
          double val = 0.0;
          for (int ix = 0; ix < P1; ++ix) val = fma(tb.B[qx][ix], row[ix], val);
          const double xi = tb.x[qx];
          const double J00 = Ax + Bx * eta, J10 = Az + Bz * eta, J01 = Cx + Bx * xi, J11 = Cz + Bz * xi;
          s += val * val * (J00 * J11 - J01 * J10) * tb.w[qx] * tb.w[qz];
        }
      }
    }
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

__global__ void k_sum(const double* __restrict__ partial, int nb, double* __restrict__ out) {
  __shared__ double red[kThreads / 32];
  double s = 0.0;
  for (int b = threadIdx.x; b < nb; b += blockDim.x) s += partial[b];
  for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x < 32) {
    s = threadIdx.x < kThreads / 32 ? red[threadIdx.x] : 0.0;
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if (threadIdx.x == 0) out[0] = s;
  }
}

}  // namespace

extern "C" {

int af_compute_diagnostics(af_operator* o, const double* rho, const double* rho_stage, const double* u,
                           const double* p, af_diagnostics* out) {
  if (!o || !rho || !u || !p || !out) return derr(AF_BAD_ARG, "af_compute_diagnostics: null argument");
  DG_CU(cudaSetDevice(o->device));
  double* part = o->d_part;  // 4 * kMaxPartials doubles >= 5 * kBlocks
  static_assert(kNV * kBlocks <= 4 * kMaxPartials - 8, "partials exceed the handle's reduction scratch");
  double* res = part + 4 * kMaxPartials - 8;
  k_diag_partial<<<kBlocks, kThreads, 0, o->stream>>>(rho, rho_stage ? rho_stage : rho, u, p, o->mesh.vtx, o->mesh.nx,
                                                      o->ncell, o->nd, part);
  k_diag_final<<<1, kThreads, 0, o->stream>>>(part, kBlocks, res);
  DG_CU(cudaGetLastError());
  double h[kNV];
  DG_CU(cudaMemcpyAsync(h, res, sizeof(h), cudaMemcpyDeviceToHost, o->stream));
  {
    const int r_ = sync_checked(o, o->stream);
    if (r_ != AF_OK) return r_;
  }
  o->launches += 2;
  out->max_velocity = h[0];
  out->min_density = -h[1];
  out->max_density = h[2];
  out->max_celerity = h[3];  // compute_max_celerity's value (the reference prints it times 1/Ma)
  out->min_cell_diameter = -h[4];
  // Courant numbers as Atmospheric_Flow.cc:1227-1235 (degree_u * sqrt(dim) / min diameter)
  const double f = o->dt * o->P * std::sqrt(2.0) / out->min_cell_diameter;
  out->cfl_c = out->max_celerity / o->Ma * f;
  out->cfl_u = out->max_velocity * f;
  return AF_OK;
}

int af_l2_norm(af_operator* o, int ncomp, const double* v, double* norm) {
  if (!o || !v || !norm || ncomp < 1 || ncomp > 2) return derr(AF_BAD_ARG, "af_l2_norm: bad argument");
  DG_CU(cudaSetDevice(o->device));
  L2Tab tb{};
  const int P1 = o->P + 1;
  tb.P1 = P1;
  const std::vector<long double> nd = host::gll(o->P);
  std::vector<long double> x, w;
  host::gauss(P1, x, w);
  for (int q = 0; q < P1; ++q) {
    tb.x[q] = (double)x[q];
    tb.w[q] = (double)w[q];
    for (int i = 0; i < P1; ++i) tb.B[q][i] = (double)host::lag(nd, i, x[q]);
  }
  double* part = o->d_part;
  double* res = part + 4 * kMaxPartials - 8;
  k_l2_partial<<<kBlocks, kThreads, 0, o->stream>>>(v, o->mesh.vtx, o->mesh.nx, o->ncell, ncomp, tb, part);
  k_sum<<<1, kThreads, 0, o->stream>>>(part, kBlocks, res);
  DG_CU(cudaGetLastError());
  double h = 0.0;
  DG_CU(cudaMemcpyAsync(&h, res, sizeof(double), cudaMemcpyDeviceToHost, o->stream));
  {
    const int r_ = sync_checked(o, o->stream);
    if (r_ != AF_OK) return r_;
  }
  o->launches += 2;
  *norm = std::sqrt(h);
  return AF_OK;
}

}  // extern "C"
