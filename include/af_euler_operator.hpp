// af_euler_operator.hpp -- C++ mirror of the reference's EULEROperator (euler_operator.h:24-211)
// and of the pieces of EulerSolver (Atmospheric_Flow.cc) it is driven by, over the C ABI of
// libaf_gpu.so (af_gpu.h).  Header only.
//
// Method names and argument meaning follow the reference: set_dt / set_Mach / set_Froude /
// set_HYPERBOLIC_stage / set_NS_stage / set_rho_for_fixed / set_pres_fixed / set_u_fixed,
// vmult_rhs_rho_update / vmult_rhs_velocity_fixed / vmult_rhs_pressure with the positional
// source lists, vmult (the NS_stage operator), vmult_pressure (B), vmult_enthalpy (C),
// compute_diagonal.  Vectors are DEVICE pointers in deal.II's DoF layout (the library's
// conventions); sizes come from n_dofs().  Failures throw af::Error (the reference throws
// deal.II exceptions, SolverControl::NoConvergence among them).
#pragma once

#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "af_gpu.h"

namespace af {

struct Error : std::runtime_error {
  int status;
  Error(int s, const std::string& where)
      : std::runtime_error(where + ": " + af_error_string(s) + ": " + af_last_error_message()), status(s) {}
};

inline void check(int status, const char* where) {
  if (status != AF_OK) throw Error(status, where);
}

class EulerOperator {
 public:
  // mesh.vertices: HOST array of (nz+1)(nx+1) (x, z) pairs; QGauss(2 degree + 1)
  EulerOperator(const af_mesh_desc& mesh, int degree, double Ma, double Fr, double dt) {
    check(af_create(&mesh, degree, 2 * degree + 1, Ma, Fr, dt, &h_), "af_create");
  }
  ~EulerOperator() {
    if (h_) af_destroy(h_);
  }
  EulerOperator(const EulerOperator&) = delete;
  EulerOperator& operator=(const EulerOperator&) = delete;
  EulerOperator(EulerOperator&& o) noexcept : h_(std::exchange(o.h_, nullptr)) {}

  af_operator* handle() const { return h_; }
  // 0 velocity (2 components per node), 1 pressure, 2 density
  long long n_dofs(int space) const {
    long long n = 0;
    check(af_n_dofs(h_, space, &n), "af_n_dofs");
    return n;
  }
  void set_stream(void* stream) { check(af_set_stream(h_, stream), "af_set_stream"); }
  void synchronize() { check(af_synchronize(h_), "af_synchronize"); }

  // setters, euler_operator.h:243-339 (the fixed fields are deep-copied)
  void set_dt(double v) { check(af_set_dt(h_, v), "set_dt"); }
  void set_Mach(double v) { check(af_set_Mach(h_, v), "set_Mach"); }
  void set_Froude(double v) { check(af_set_Froude(h_, v), "set_Froude"); }
  // Rayleigh damping layers of the 2D hill case (no counterpart in the reference)
  void set_sponge(double z_start, double z_top, double rate_top, double x_left, double x_right, double width_lateral,
                  double rate_lateral, double u_ref) {
    check(af_set_sponge(h_, z_start, z_top, rate_top, x_left, x_right, width_lateral, rate_lateral, u_ref),
          "set_sponge");
  }
  void set_HYPERBOLIC_stage(int s) { check(af_set_HYPERBOLIC_stage(h_, s), "set_HYPERBOLIC_stage"); }
  void set_NS_stage(int s) { check(af_set_NS_stage(h_, s), "set_NS_stage"); }
  void set_rho_for_fixed(const double* v) { check(af_set_rho_for_fixed(h_, v), "set_rho_for_fixed"); }
  void set_pres_fixed(const double* v) { check(af_set_pres_fixed(h_, v), "set_pres_fixed"); }
  void set_u_fixed(const double* v) { check(af_set_u_fixed(h_, v), "set_u_fixed"); }

  // explicit right-hand sides with the reference's positional source lists
  void vmult_rhs_rho_update(double* dst, const std::vector<const double*>& src) {
    check(af_vmult_rhs_rho_update(h_, dst, src.data(), (int)src.size()), "vmult_rhs_rho_update");
  }
  void vmult_rhs_velocity_fixed(double* dst, const std::vector<const double*>& src) {
    check(af_vmult_rhs_velocity_fixed(h_, dst, src.data(), (int)src.size()), "vmult_rhs_velocity_fixed");
  }
  void vmult_rhs_pressure(double* dst, const std::vector<const double*>& src) {
    check(af_vmult_rhs_pressure(h_, dst, src.data(), (int)src.size()), "vmult_rhs_pressure");
  }

  // implicit operators
  void vmult(double* dst, const double* src) const { check(af_vmult(h_, dst, src), "vmult"); }
  void vmult_pressure(double* dst, const double* src) const { check(af_vmult_pressure(h_, dst, src), "vmult_pressure"); }
  void vmult_enthalpy(double* dst, const double* src) const { check(af_vmult_enthalpy(h_, dst, src), "vmult_enthalpy"); }
  // compute_diagonal + get_matrix_diagonal_inverse
  void compute_diagonal(double* inverse_diagonal) const {
    check(af_compute_diagonal(h_, inverse_diagonal), "compute_diagonal");
  }
  // exact block inverse of the mass-type operator of the current NS_stage
  void vmult_inverse(double* dst, const double* src) const { check(af_vmult_inverse(h_, dst, src), "vmult_inverse"); }

 private:
  af_operator* h_ = nullptr;
};

// The pressure system of pressure_fixed_point (Atmospheric_Flow.cc:657-672) with the library's
// FGMRES and preconditioners.
class SchurSolver {
 public:
  SchurSolver(EulerOperator& op, int preconditioner) {
    af_schur_options o;
    check(af_schur_default_options(&o), "af_schur_default_options");
    o.preconditioner = preconditioner;
    check(af_schur_solver_create(op.handle(), &o, &s_), "af_schur_solver_create");
  }
  ~SchurSolver() {
    if (s_) af_schur_solver_destroy(s_);
  }
  SchurSolver(const SchurSolver&) = delete;
  SchurSolver& operator=(const SchurSolver&) = delete;
  void setup(bool estimate_eigenvalues = false) { check(af_schur_solver_setup(s_, estimate_eigenvalues), "setup"); }
  af_schur_stats solve(double* x, const double* b, double rel_tol, int max_iterations) {
    af_schur_stats st{};
    check(af_schur_solve(s_, x, b, rel_tol, max_iterations, &st), "af_schur_solve");
    return st;
  }

 private:
  af_schur_solver* s_ = nullptr;
};

// EulerSolver::run's time loop (Atmospheric_Flow.cc:1100-1257) on the device.
class IMEXStepper {
 public:
  IMEXStepper(const af_mesh_desc& mesh, int degree, double Ma, double Fr, double dt,
              const af_imex_options* opt = nullptr) {
    check(af_imex_create(&mesh, degree, Ma, Fr, dt, opt, &h_), "af_imex_create");
  }
  ~IMEXStepper() {
    if (h_) af_imex_destroy(h_);
  }
  IMEXStepper(const IMEXStepper&) = delete;
  IMEXStepper& operator=(const IMEXStepper&) = delete;
  void set_state(const double* rho, const double* u, const double* p) {
    check(af_imex_set_state(h_, rho, u, p), "af_imex_set_state");
  }
  void get_state(double* rho, double* u, double* p) const { check(af_imex_get_state(h_, rho, u, p), "af_imex_get_state"); }
  void step(int n) { check(af_imex_step(h_, n), "af_imex_step"); }
  af_imex_stats stats() const {
    af_imex_stats s{};
    check(af_imex_last_stats(h_, &s), "af_imex_last_stats");
    return s;
  }

  // The forward / backward pair of one step, the role a torch.autograd.Function plays in a
  // Python code (no counterpart in the reference): forward records the linearisation point,
  // tangent and backward apply J and J^T there (Schur solves to rel_tol).
  void step_forward(const double* rho0, const double* u0, const double* p0, double* rho1, double* u1, double* p1) {
    check(af_imex_step_forward(h_, rho0, u0, p0, rho1, u1, p1), "af_imex_step_forward");
  }
  void step_tangent(const double* drho0, const double* du0, const double* dp0, double* drho1, double* du1,
                    double* dp1, double rel_tol = 1e-12) {
    check(af_imex_step_tangent(h_, drho0, du0, dp0, drho1, du1, dp1, rel_tol), "af_imex_step_tangent");
  }
  void step_backward(const double* rho1bar, const double* u1bar, const double* p1bar, double* rho0bar,
                     double* u0bar, double* p0bar, double rel_tol = 1e-12) {
    check(af_imex_step_backward(h_, rho1bar, u1bar, p1bar, rho0bar, u0bar, p0bar, rel_tol), "af_imex_step_backward");
  }
  // cotangent of a functional of the state after nsteps, pulled back to (rho0, u0, p0) with
  // one checkpoint every checkpoint_every steps
  void gradient(const double* rho0, const double* u0, const double* p0, int nsteps, int checkpoint_every,
                const double* rhobar, const double* ubar, const double* pbar, double* rho0bar, double* u0bar,
                double* p0bar, double rel_tol = 1e-12) {
    check(af_imex_gradient(h_, rho0, u0, p0, nsteps, checkpoint_every, rhobar, ubar, pbar, rho0bar, u0bar, p0bar,
                           rel_tol),
          "af_imex_gradient");
  }

 private:
  af_imex* h_ = nullptr;
};

}  // namespace af
