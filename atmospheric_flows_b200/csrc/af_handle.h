// af_handle.h -- the operator handle behind the C ABI (shared by af_capi.cu and af_imex.cu).
#pragma once

#include <cuda_runtime.h>

#include "af_blas.h"
#include "af_internal.h"

using af::MeshDev;
using af::KrylovState;
using af::DegreeOps;

struct af_operator {
  int device = 0;
  cudaStream_t own_stream = nullptr, stream = nullptr;
  int P = 0, NQ = 0, ncell = 0, nd = 0;
  MeshDev mesh{};
  double2* d_vtx = nullptr;
  double Ma = 1, Fr = 1, dt = 1;
  // Rayleigh damping of the momentum (af_set_sponge; off when both rates are 0)
  double sp_z0 = 0, sp_z1 = 1, sp_rate = 0, sp_x0 = 0, sp_x1 = 1, sp_width = 1, sp_rate_lat = 0, sp_u = 0;
  int hs = 1, ns = 1;
  // IMEX-ARK tableau, euler_operator.h:233-240
  double gamma, a21, a22, a31, a32, a33, a21t, a22t, a31t, a32t, a33t, b1, b2, b3;
  double* d_rho_fixed = nullptr;
  double* d_pres_fixed = nullptr;
  double* d_u_fixed = nullptr;
  bool rho_fixed_set = false, pres_fixed_set = false;
  // workspace: 6 velocity-space vectors (Schur t1, t2; inner CG r, z, p, Ap), reduction
  // partials, Krylov state
  double* d_ws = nullptr;
  double* d_part = nullptr;
  KrylovState* d_kst = nullptr;
  double* d_invdA = nullptr;  // inverse diagonal of A for the current rho_for_fixed
  bool invdA_valid = false;
  int schur_mode = 0;
  double schur_tol = 1e-12;
  int schur_maxit = 10000;
  int last_inner_its = 0;
  long long launches = 0;
  const DegreeOps* ops = nullptr;
  // exact cell-wise inverses: Gauss-point weights of M (fixed mesh; change of basis) and the
  // packed inverses of A (rho_for_fixed)
  double* d_Wm = nullptr;
  double* d_La = nullptr;
  bool Wm_valid = false, La_valid = false;
  // host-buffer entry points: device staging, and the copy streams and events of the
  // row-chunk pipeline (sources in / results out overlapping the kernel)
  static constexpr int kHostChunks = 16;
  double* d_stage = nullptr;
  size_t stage_len = 0;
  cudaStream_t copy_in = nullptr, copy_out = nullptr;
  cudaEvent_t ev_start = nullptr, ev_in[kHostChunks] = {}, ev_done[kHostChunks] = {};
  // status word of the handle's kernels (mapped pinned host memory; mesh.status is its device
  // address): a kernel that gives up a bounded wait leaves a code there
  int* h_status = nullptr;

  long n_scalar() const { return (long)ncell * nd; }
};

namespace af {
int mass_inverse_A(af_operator* o, const double** out);
// AF_TIMEOUT (with a message) when a kernel of the handle left a code in its status word since
// the last report, which also clears the word; AF_OK otherwise.  Reads host memory, no sync.
int take_kernel_status(af_operator* o);
// cudaStreamSynchronize(st), then take_kernel_status(o)
int sync_checked(af_operator* o, cudaStream_t st);
}
