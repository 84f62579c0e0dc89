// C++ caller of libaf_gpu.so through include/af_euler_operator.hpp, in the shape of the
// reference's stage drivers: density rhs -> mass solve, pressure/velocity rhs, Schur solve,
// a time step and its forward / tangent / backward pair; checked against the C ABI called
// directly, by a dot-product test and for error reporting.
// Built and run by tests/test_gpu_cpp_shim.py.  Prints "OK" on success.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <vector>

#include "af_euler_operator.hpp"

#define REQUIRE(c)                                                   \
  do {                                                               \
    if (!(c)) {                                                      \
      std::printf("FAILED %s at line %d\n", #c, __LINE__);          \
      return 1;                                                      \
    }                                                                \
  } while (0)

static double* upload(const std::vector<double>& h) {
  double* d = nullptr;
  if (cudaMalloc(&d, h.size() * sizeof(double)) != cudaSuccess) return nullptr;
  cudaMemcpy(d, h.data(), h.size() * sizeof(double), cudaMemcpyHostToDevice);
  return d;
}
static std::vector<double> download(const double* d, size_t n) {
  std::vector<double> h(n);
  cudaMemcpy(h.data(), d, n * sizeof(double), cudaMemcpyDeviceToHost);
  return h;
}

int main() {
  const int nx = 16, nz = 8, P = 3, ND = (P + 1) * (P + 1);
  // terrain-following mesh over a bell-shaped hill, z from h(x) to 16 km
  std::vector<double> vtx((nx + 1) * (nz + 1) * 2);
  for (int j = 0; j <= nz; ++j)
    for (int i = 0; i <= nx; ++i) {
      const double x = -20000.0 + 40000.0 * i / nx, s = 16000.0 * j / nz;
      const double h = 400.0 / (1.0 + (x / 1000.0) * (x / 1000.0));
      vtx[(j * (nx + 1) + i) * 2] = x;
      vtx[(j * (nx + 1) + i) * 2 + 1] = h + s * (1.0 - h / 16000.0);
    }
  af_mesh_desc mesh{nx, nz, 1, vtx.data(), 0, 0.0};
  const double Ma = std::sqrt(1.0 / (287.0 * 300.0)), Fr = 1.0 / std::sqrt(9.81), dt = 2.0;
  af::EulerOperator op(mesh, P, Ma, Fr, dt);
  const long n = (long)op.n_dofs(1);
  REQUIRE(n == (long)nx * nz * ND && op.n_dofs(0) == 2 * n);
  // smooth states: density and pressure decaying with the cell row, a uniform wind
  std::vector<double> rho(n), u(2 * n), p(n);
  for (long k = 0; k < n; ++k) {
    const long c = k / ND, row = c / nx;
    rho[k] = 1.16 * std::exp(-0.05 * row) * (1.0 + 0.001 * std::sin(0.3 * k));
    p[k] = std::exp(-0.06 * row) * (1.0 + 0.001 * std::cos(0.2 * k));
  }
  for (long c = 0; c < n / ND; ++c)
    for (int q = 0; q < ND; ++q) {
      u[c * 2 * ND + q] = 10.0 + 0.1 * std::sin(0.1 * (c * ND + q));
      u[c * 2 * ND + ND + q] = 0.05 * std::cos(0.1 * (c * ND + q));
    }
  double *d_rho = upload(rho), *d_u = upload(u), *d_p = upload(p);
  REQUIRE(d_rho && d_u && d_p);
  double *r_rho = upload(std::vector<double>(n)), *r_u = upload(std::vector<double>(2 * n)),
         *r_p = upload(std::vector<double>(n));
  double *f_rho = upload(std::vector<double>(n)), *f_u = upload(std::vector<double>(2 * n)),
         *f_p = upload(std::vector<double>(n));

  // stage-1 right-hand sides, the reference's positional lists (Atmospheric_Flow.cc:439-449, 555-568)
  op.set_HYPERBOLIC_stage(1);
  op.vmult_rhs_rho_update(r_rho, {d_rho, d_u});
  op.vmult_rhs_velocity_fixed(r_u, {d_rho, d_u, d_p, d_rho});
  op.vmult_rhs_pressure(r_p, {d_rho, d_u, d_p, d_rho, d_u});
  const double* src[] = {d_rho, d_u, d_p, d_rho, d_u};
  af::check(af_vmult_rhs_fused(op.handle(), f_rho, f_u, f_p, src, 5), "af_vmult_rhs_fused");
  op.synchronize();
  auto rel = [](const std::vector<double>& a, const std::vector<double>& b) {
    double num = 0, den = 0;
    for (size_t k = 0; k < a.size(); ++k) {
      num += (a[k] - b[k]) * (a[k] - b[k]);
      den += b[k] * b[k];
    }
    return std::sqrt(num / den);
  };
  REQUIRE(rel(download(r_rho, n), download(f_rho, n)) < 1e-13);
  REQUIRE(rel(download(r_u, 2 * n), download(f_u, 2 * n)) < 1e-13);
  REQUIRE(rel(download(r_p, n), download(f_p, n)) < 1e-13);

  // update_density: M rho_2 = rhs (exact cell inverse), then M rho_2 reproduces the rhs
  op.set_NS_stage(1);
  op.vmult_inverse(f_rho, r_rho);
  op.vmult(r_p, f_rho);
  op.synchronize();
  REQUIRE(rel(download(r_p, n), download(r_rho, n)) < 1e-12);

  // the pressure system and its solver
  op.set_rho_for_fixed(d_rho);
  op.set_pres_fixed(d_p);
  op.set_NS_stage(2);
  op.vmult(r_p, d_p);  // b = S p
  af::SchurSolver solver(op, AF_SCHUR_CHEB_FP32);
  solver.setup();
  cudaMemset(f_p, 0, n * sizeof(double));
  const af_schur_stats st = solver.solve(f_p, r_p, 1e-10, 1000);
  REQUIRE(st.iterations > 0 && st.final_residual <= 1e-10 * 1.000001 * std::sqrt([&] {
            auto b = download(r_p, n);
            double s = 0;
            for (double v : b) s += v * v;
            return s;
          }()));
  REQUIRE(rel(download(f_p, n), p) < 1e-7);

  // errors are reported as exceptions carrying the status
  bool thrown = false;
  try {
    op.set_NS_stage(9);
  } catch (const af::Error& e) {
    thrown = e.status == AF_BAD_ARG;
  }
  REQUIRE(thrown);

  // one IMEX step of the time loop
  af_imex_options io;
  af_imex_default_options(&io);
  io.schur_preconditioner = AF_SCHUR_CHEB_FP32;
  af::IMEXStepper stepper(mesh, P, Ma, Fr, dt, &io);
  stepper.set_state(d_rho, d_u, d_p);
  stepper.step(1);
  stepper.get_state(f_rho, f_u, f_p);
  const auto s = stepper.stats();
  REQUIRE(s.fixed_point_iterations[0] >= 1 && s.gmres_iterations > 0);
  for (double v : download(f_p, n)) REQUIRE(std::isfinite(v) && v > 0.0);

  // the step's forward / tangent / backward pair: <J dx, ybar> = <dx, J^T ybar>
  {
    std::vector<double> hx(n), hu(2 * n);
    for (long k = 0; k < n; ++k) hx[k] = std::sin(0.7 * k);
    for (long k = 0; k < 2 * n; ++k) hu[k] = std::cos(0.3 * k);
    double *dr = upload(hx), *du = upload(hu), *dp = upload(hx), *yr = upload(hx), *yu = upload(hu), *yp = upload(hx);
    double *tr = upload(hx), *tu = upload(hu), *tp = upload(hx), *xr = upload(hx), *xu = upload(hu), *xp = upload(hx);
    stepper.step_forward(d_rho, d_u, d_p, f_rho, f_u, f_p);
    stepper.step_tangent(dr, du, dp, tr, tu, tp, 1e-12);
    stepper.step_backward(yr, yu, yp, xr, xu, xp, 1e-12);
    auto dot = [&](const double* a, const double* b, size_t m, double& scale) {
      auto x = download(a, m), y = download(b, m);
      double s = 0;
      for (size_t k = 0; k < m; ++k) { s += x[k] * y[k]; scale += std::fabs(x[k] * y[k]); }
      return s;
    };
    double s1 = 0, s2 = 0;
    const double lhs = dot(tr, yr, n, s1) + dot(tu, yu, 2 * n, s1) + dot(tp, yp, n, s1);
    const double rhs = dot(xr, dr, n, s2) + dot(xu, du, 2 * n, s2) + dot(xp, dp, n, s2);
    REQUIRE(std::fabs(lhs - rhs) <= 1e-10 * s1);
    for (double* q : {dr, du, dp, yr, yu, yp, tr, tu, tp, xr, xu, xp}) cudaFree(q);
  }
  for (double* q : {d_rho, d_u, d_p, r_rho, r_u, r_p, f_rho, f_u, f_p}) cudaFree(q);
  std::printf("OK\n");
  return 0;
}
