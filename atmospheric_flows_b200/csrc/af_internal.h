// af_internal.h -- host-side declarations shared by the C ABI and the per-degree kernel
// translation units (af_kern.cu is compiled once per polynomial degree 1..6).
#pragma once

#include <cuda_runtime.h>

#include "af_cellop.cuh"
#include "af_physics.cuh"

namespace af {

// Sources of an explicit right-hand side in the reference's positional order of
// vmult_rhs_pressure (the superset list, Atmospheric_Flow.cc:555-556, 562-564, 796-799):
//   stage 1: rho0 u0 p0 rho2 u_fixed
//   stage 2: rho0 u0 p0 rho2 u2 p2 rho3 u_fixed
//   stage 3: rho0 u0 p0 rho2 u2 p2 rho3 u3 p3 rho_curr u_curr
// Unused slots may be null.
struct RhsSources {
  const double* rho[3];
  const double* u[3];
  const double* p[3];
  const double* rho_c;  // rho_tmp_2 / rho_tmp_3 / rho_curr
  const double* u_fix;  // u_fixed / u_curr
};

struct DegreeOps {
  cudaError_t (*upload_tables)();
  cudaError_t (*rhs)(const MeshDev&, int stage, int mask, const RhsSources&, const RhsParams&, double* out_rho,
                     double* out_u, double* out_p, int ncell, cudaStream_t);
  // dst = scale * M src (ncomp 1 or 2), or M_rho src with a density weight
  cudaError_t (*mass)(const MeshDev&, int ncomp, const double* src, const double* weight, double scale, double* dst,
                      int ncell, cudaStream_t);
  cudaError_t (*op_B)(const MeshDev&, const double* p, double c, double* u, int ncell, cudaStream_t);
  // dst = C w (sign +1), or dst = D p - C w when p != null
  cudaError_t (*op_C)(const MeshDev&, const double* w, const double* pf, const double* p, const CParams&, double* dst,
                      int ncell, cudaStream_t);
  // inverse of the diagonal of scale*M (weight null) or of M_rho (ncomp copies)
  cudaError_t (*inv_diag)(const MeshDev&, int ncomp, const double* weight, double scale, double* dst, int ncell,
                          cudaStream_t);
  // packed inverses (lower triangle) of the cell mass matrices (weight null: plain mass),
  // stored interleaved L[k * ncell + c], factor_len() doubles per cell
  cudaError_t (*mass_factor)(const MeshDev&, const double* weight, double* L, int ncell, cudaStream_t);
  // x = scale * M^{-1} b (block diagonal, exact), ncomp components per cell
  cudaError_t (*mass_solve)(const double* L, int ncomp, const double* b, double scale, double* x, int ncell,
                            int* status, cudaStream_t);
  int cells_per_block;
  int factor_len;  // (p+1)^2 ((p+1)^2 + 1) / 2

  // ---- h-multigrid level kernels, in FP64 (_d) and FP32 (_f) ----
  // r += C0 w - D p: the residual update of the linearised Schur complement (C0 = C
  // without the wave-speed term); prm.g1 carries +1/(gamma-1)
  cudaError_t (*mg_res_d)(const MeshDev&, const double* w, const double* pf, const double* p, const CParams&,
                          double* r, int ncell, cudaStream_t);
  cudaError_t (*mg_res_f)(const MeshDev&, const float* w, const float* pf, const float* p, const CParamsT<float>&,
                          float* r, int ncell, cudaStream_t);
  // Chebyshev update with the packed cell-wise inverse D^{-1} = s M^{-1} (FP64 levels):
  //   d = alpha d + s M^{-1} r  (alpha == 0: d not read);  x = d (first) or x += d
  cudaError_t (*cheb_d)(const double* L, const double* r, double alpha, double s, double* d, double* x, int first,
                        int ncell, int* status, cudaStream_t);
  // xf += P xc (coarse nx_c x nz_c cells, fine 2nx_c x 2nz_c); rc = P^T rf
  cudaError_t (*prolong_d)(const double* xc, double* xf, int nxc, int nzc, cudaStream_t);
  cudaError_t (*prolong_f)(const float* xc, float* xf, int nxc, int nzc, cudaStream_t);
  cudaError_t (*restrict_d)(const double* rf, double* rc, int nxc, int nzc, cudaStream_t);
  cudaError_t (*restrict_f)(const float* rf, float* rc, int nxc, int nzc, cudaStream_t);
  // coarse nodal values of a fine coefficient field (injection from the child cell)
  cudaError_t (*inject)(const double* ff, double* fc, int nxc, int nzc, cudaStream_t);

  // adjoint of the fused stage-1 rhs triple: in = rho0 u0 p0 rho2 u_fixed, ybar = cotangents of
  // the rho, u, p outputs, xbar = cotangents of the five inputs (overwritten)
  cudaError_t (*rhs_adjoint1)(const MeshDev&, const double* const* in, const double* const* ybar, double* const* xbar,
                              const RhsParams&, int ncell, cudaStream_t);
  // its tangent-linear: dy (rho, u, p) = J(in) din
  cudaError_t (*rhs_tangent1)(const MeshDev&, const double* const* in, const double* const* din, double* const* dy,
                              const RhsParams&, int ncell, cudaStream_t);
  // implicit operators: pbar = B^T ubar;  dst = J_C(w) dw;  wbar = J_C(w)^T pbar
  cudaError_t (*op_BT)(const MeshDev&, const double* ubar, double c, double* pbar, int ncell, cudaStream_t);
  cudaError_t (*op_C_tangent)(const MeshDev&, const double* w, const double* dw, const double* pf, const CParams&,
                              double* dst, int ncell, cudaStream_t);
  cudaError_t (*op_CT)(const MeshDev&, const double* w, const double* pf, const double* pbar, const CParams&,
                       double* wbar, int ncell, cudaStream_t);

  // ---- cell-wise inverses by the change of basis to the Gauss points (no stored matrices):
  // W = 1 / (rho JxW) at the (P+1)^2 Gauss points, rho = 1 when null.  Exact for the plain
  // mass matrix on bilinear cells (FP64: the operator's M and D inverses); the FP32 levels
  // of the pressure preconditioner also use it for A
  cudaError_t (*cob_weights_f)(const MeshDev&, const double* rho, float* W, int ncell, cudaStream_t);
  cudaError_t (*cob_weights_d)(const MeshDev&, const double* rho, double* W, int ncell, cudaStream_t);
  // x = scale M_W^{-1} b (ncomp 1 or 2)
  cudaError_t (*cob_solve_f)(const float* W, int ncomp, const float* b, float scale, float* x, int ncell,
                             cudaStream_t);
  cudaError_t (*cob_solve_d)(const double* W, int ncomp, const double* b, double scale, double* x, int ncell,
                             cudaStream_t);
  // d = alpha d + s M_W^{-1} r;  x = d (first) or x += d
  cudaError_t (*cob_cheb_f)(const float* W, const float* r, float alpha, float s, float* d, float* x, int first,
                            int ncell, cudaStream_t);
  // w = scale A_W^{-1} (B p) with B's coefficient c: one launch for B and the cell-wise solve
  cudaError_t (*b_inv_f)(const MeshDev&, const float* p, float c, const float* WA, float scale, float* w, int ncell,
                         cudaStream_t);
  // the smoother step:  r += C0 w - D din;  dout = alpha din + s M_W^{-1} r;  x = dout (first)
  // or x += dout.  prm.g1 carries +1/(gamma-1) as for mg_res; din and dout are distinct arrays.
  cudaError_t (*res_cheb_f)(const MeshDev&, const float* w, const float* pf, const float* din,
                            const CParamsT<float>&, const float* WM, float alpha, float s, float* r, float* dout,
                            float* x, int first, int ncell, cudaStream_t);
  // the same three FP32 level operators with P+1 Gauss points per direction (exact for B and
  // D on bilinear cells, approximate for C0 and A): the reduced-quadrature preconditioner
  cudaError_t (*mg_res_fr)(const MeshDev&, const float* w, const float* pf, const float* p,
                           const CParamsT<float>&, float* r, int ncell, cudaStream_t);
  cudaError_t (*b_inv_fr)(const MeshDev&, const float* p, float c, const float* WA, float scale, float* w,
                          int ncell, cudaStream_t);
  cudaError_t (*res_cheb_fr)(const MeshDev&, const float* w, const float* pf, const float* din,
                             const CParamsT<float>&, const float* WM, float alpha, float s, float* r, float* dout,
                             float* x, int first, int ncell, cudaStream_t);
  // coefficient derivatives of the implicit operators, transposed:
  //   rhobar = (d/drho [A(rho) x])^T y;   pfbar = (d/dp_f [C(w; p_f)])^T pbar
  cudaError_t (*op_A_rho_T)(const MeshDev&, const double* x, const double* y, double* rhobar, int ncell,
                            cudaStream_t);
  cudaError_t (*op_C_pf_T)(const MeshDev&, const double* w, const double* pbar, const CParams&, double* pfbar,
                           int ncell, cudaStream_t);
  // tangent and adjoint of the fused rhs triple of any stage (dual-number evaluation of the
  // same physics); vectors in the fused order rho_j, u_j, p_j (explicit stages), rho_c,
  // u_fixed; dy / ybar = rho, u, p; scratch: one velocity-sized vector (stage 2)
  cudaError_t (*rhs_tangent)(const MeshDev&, int stage, const double* const* in, const double* const* din,
                             double* const* dy, const RhsParams&, int ncell, cudaStream_t);
  cudaError_t (*rhs_adjoint)(const MeshDev&, int stage, const double* const* in, const double* const* ybar,
                             double* const* xbar, double* scratch, const RhsParams&, int ncell, cudaStream_t);
  // the smoother step on the preconditioned residual z = D^{-1} r, D^{-1} = g M_W^{-1}:
  //   z += g M_W^{-1} C0 w - din;  dout = alpha din + s z;  x = dout (first) or x += dout.
  // prm.g1 is unused (no D term in the kernel); reduced != 0 selects P+1 Gauss points.
  cudaError_t (*res_chebz_f)(const MeshDev&, const float* w, const float* pf, const float* din,
                             const CParamsT<float>&, const float* WM, float g, float alpha, float s, float* z,
                             float* dout, float* x, int first, int reduced, int ncell, cudaStream_t);
  // ---- the same smoother in the Gauss-point basis (af_gauss.cuh): vectors hold values at the
  // (P+1)^2 Gauss points, face traces tr[face][comp][cell][P+1] go with them
  //   entry: d = x = sc WM (Vi x Vi)^T v (v FP64 nodal), z = theta d, dtr = traces of d
  cudaError_t (*gs_entry)(const double* v, const float* WM, float sc, float theta, float* z, float* d, float* x,
                          float* dtr, int ncell, cudaStream_t);
  //   w = scale diag(WA) B_g d (two components) and its traces
  cudaError_t (*gs_binv)(const MeshDev&, const float* d, const float* dtr, float c, const float* WA, float scale,
                         float* w, float* wtr, int ncell, cudaStream_t);
  //   z += g WM C0_g(w; pg) - d;  d = alpha d + s z (in place);  x += d;  dtr = traces of d
  cudaError_t (*gs_zstep)(const MeshDev&, const float* w, const float* wtr, const float* pg, const float* ptr,
                          float cdt, float gg, const float* WM, float g, float alpha, float s, float* z, float* d,
                          float* x, float* dtr, int ncell, cudaStream_t);
  //   out = (Vi x Vi) x (FP64 nodal)
  cudaError_t (*gs_exit)(const float* x, double* out, int ncell, cudaStream_t);
  //   a coefficient at the Gauss points and its traces: pg = (V x V) p
  cudaError_t (*gs_values)(const double* p, float* pg, float* ptr, int ncell, cudaStream_t);
};

const DegreeOps* degree_ops(int P);  // null if the degree was not compiled

}  // namespace af
