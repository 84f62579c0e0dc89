// af_adjoint.cuh -- adjoint (vector-Jacobian product) of the fused stage-1 explicit
// right-hand side triple, as a policy of the generic cell kernel.
//
// Forward (RhsPhys<1, 7>, euler_operator.h:344-692, 745-1361, 1622-2305 at HYPERBOLIC_stage 1):
//   y_o[i] = sum_q [ f_o(v(q)) phi_i(q) + g_o(v(q)) . grad phi_i(q) ] JxW  +  face terms,
// v = (rho0, u0, p0, rho2, u_fixed) at the point.  Its adjoint for output cotangents ybar:
//   xbar_a[j] = sum_q [ sum_o ybar_o(q) df_o/dv_a + grad ybar_o(q) . dg_o/dv_a ] phi_j(q) JxW
//              + faces,
// i.e. the same cell-centric sum factorisation with the cotangents' values and physical
// gradients at the points (the kernel's gradient fields) and a value-only test.  Faces: the
// fluxes are antisymmetric under a side swap, F(v_N, v_K; -n) = -F(v_K, v_N; n), so the cell
// K receives, from its own face term and from its neighbour's,
//   xbar_K += sum_q (d_1 F(v_K, v_N; n))^T (ybar_K(q) - ybar_N(q)) phi_K JxW,
// where d_1 is the derivative with respect to the own side.  The Rusanov wave speed
// lambda = max(|u+.n|, |u-.n|) is differentiated along the branch the forward pass takes
// (own side when |u+.n| >= |u-.n|).  Boundary faces (velocity wall pressure term) give
// xbar_p += (dF_b/dp)^T ybar_u.
#pragma once

#include "af_physics.cuh"

namespace af {

// One group: rho0, u0 (2), p0, rho2, u_fixed (2), then the cotangents ybar_rho, ybar_u (2),
// ybar_p (gradient fields).  Outputs: xbar of rho0, u0, p0, rho2, u_fixed.
struct RhsAdj1Phys {
  static constexpr int NG = 1;
  static constexpr bool FACES = true, NEED_X = true, ACCUMULATE = false;
  static constexpr bool FOLD = true;  // z-face folding measured faster (1.53 -> 1.43 ms, 0.97 -> 0.90 ms)
  static constexpr int NOUT_ARR = 5, NOUT = 7;
  using Params = RhsParams;
  using real = double;
  static constexpr int out_ncomp(int a) { return (a == 1 || a == 4) ? 2 : 1; }
  static constexpr bool has_val(int) { return true; }
  static constexpr bool has_grad(int) { return false; }
  static constexpr int narr_of(int) { return 8; }
  static constexpr int nf_of(int) { return 11; }
  static constexpr int nfc_of(int) { return 11; }
  static constexpr int nfg_of(int) { return 4; }
  template <int G>
  struct Grp {
    static constexpr int NARR = 8;
    static constexpr bool FACE = true;
    static constexpr int ncomp(int a) { return (a == 1 || a == 4 || a == 6) ? 2 : 1; }
    static constexpr bool face_only(int) { return false; }
  };

  // v: rho, ux, uz, p, rho2, fx, fz, yr, yux, yuz, yp | d/dxi of yr, yux, yuz, yp;  deta: d/deta
  template <int G>
  __device__ __forceinline__ static void point(const Params& prm, const double* v, const double* deta,
                                               const PointGeo& pg, double* val, double (*)[2]) {
    double e0, e1, fac;
    gravity_dir(prm, pg, e0, e1, fac);
    const double rho = v[0], ux = v[1], uz = v[2], p = v[3], r2 = v[4], fx = v[5], fz = v[6];
    const double yr = v[7], yux = v[8], yuz = v[9], yp = v[10];
    // physical gradients of the cotangents: grad = J^{-T} (d/dxi, d/deta)
    const double J00 = pg.J[0], J01 = pg.J[1], J10 = pg.J[2], J11 = pg.J[3];
    const double idet = 1.0 / (J00 * J11 - J01 * J10);
    double Gd[4][2];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const double dx = v[11 + k], de = deta[k];
      Gd[k][0] = (J11 * dx - J10 * de) * idet;
      Gd[k][1] = (J00 * de - J01 * dx) * idet;
    }
    const double* Gr = Gd[0];
    const double Gu[2][2] = {{Gd[1][0], Gd[1][1]}, {Gd[2][0], Gd[2][1]}};  // Gu[d][e] = d_e ybar_u_d
    const double* Gp = Gd[3];
    const double ca = prm.ca[0] * prm.dt, cg = prm.cg[0] * prm.dt, ct = prm.ct[0] * prm.dt, cgI = prm.cgI * prm.dt;
    const double u[2] = {ux, uz}, e[2] = {e0, e1};
    const double uu = ux * ux + uz * uz, ue = ux * e0 + uz * e1;
    const double Gru = Gr[0] * ux + Gr[1] * uz, Gpu = Gp[0] * ux + Gp[1] * uz;
    const double s = 0.5 * ca * prm.Ma2 * uu * rho + ct * prm.gg * p;
    // rho0
    double xr = yr + ca * Gru;                                             // density :378-380
    xr += yux * (ux - cg * prm.invFr2 * fac * e0) + yuz * (uz - cg * prm.invFr2 * fac * e1);  // :1686-1691
    double uGu = 0.0;
#pragma unroll
    for (int dd = 0; dd < 2; ++dd)
#pragma unroll
      for (int ee = 0; ee < 2; ++ee) uGu += Gu[dd][ee] * u[dd] * u[ee];
    xr += ca * uGu;
    xr += yp * (0.5 * prm.Ma2 * uu - cg * prm.Ma2Fr2 * ue * fac) + Gpu * (0.5 * ca * prm.Ma2 * uu);  // :806-813
    val[0] += xr;
    // u0
    const double yu[2] = {yux, yuz};
#pragma unroll
    for (int k = 0; k < 2; ++k) {
      double xu = ca * rho * Gr[k] + yu[k] * rho;
      xu += ca * rho * (Gu[k][0] * ux + Gu[k][1] * uz + Gu[0][k] * ux + Gu[1][k] * uz);
      xu += yp * (prm.Ma2 * rho * u[k] - cg * prm.Ma2Fr2 * rho * e[k] * fac) + Gp[k] * s + Gpu * ca * prm.Ma2 * rho * u[k];
      val[1 + k] += xu;
    }
    // p0
    val[3] += ct * prm.invMa2 * (Gu[0][0] + Gu[1][1]) + yp * prm.g1 + Gpu * ct * prm.gg;
    // rho2 (implicit gravity terms) and u_fixed (kinetic energy and gravity of the implicit group)
    const double ff = fx * fx + fz * fz, fe = fx * e0 + fz * e1;
    val[4] += -(yux * e0 + yuz * e1) * cgI * prm.invFr2 * fac - yp * (0.5 * prm.Ma2 * ff + cgI * prm.Ma2Fr2 * fe * fac);
    val[5] += -yp * (r2 * prm.Ma2 * fx + cgI * prm.Ma2Fr2 * r2 * e0 * fac);
    val[6] += -yp * (r2 * prm.Ma2 * fz + cgI * prm.Ma2Fr2 * r2 * e1 * fac);
  }

  template <int G>
  __device__ __forceinline__ static void face(const Params& prm, const double* vp, const double* vm,
                                              const double* n, double* flux) {
    const double rp = vp[0], ap = vp[1], bp = vp[2], pp = vp[3];
    const double rm = vm[0], am = vm[1], bm = vm[2], pm = vm[3];
    const double dyr = vp[7] - vm[7], dyu[2] = {vp[8] - vm[8], vp[9] - vm[9]}, dyp = vp[10] - vm[10];
    const double unp = ap * n[0] + bp * n[1], unm = am * n[0] + bm * n[1];
    const bool own = fabs(unp) >= fabs(unm);
    const double lam = own ? fabs(unp) : fabs(unm);
    const double sg = own ? (unp > 0.0 ? 1.0 : (unp < 0.0 ? -1.0 : 0.0)) : 0.0;
    const double dl[2] = {sg * n[0], sg * n[1]};  // d lambda / d u+
    const double ca = prm.ca[0] * prm.dt, ct = prm.ct[0] * prm.dt;
    const double up[2] = {ap, bp}, um[2] = {am, bm};
    const double uup = ap * ap + bp * bp, uum = am * am + bm * bm;
    const double jk = rp * 0.5 * uup - rm * 0.5 * uum, je = prm.g1 * (pp - pm);
    // density flux Rr = -ca (1/2 (rp unp + rm unm) + 1/2 lam (rp - rm))          :519-526
    double xr = -ca * (0.5 * unp + 0.5 * lam) * dyr;
    double xu[2], xp = 0.0;
#pragma unroll
    for (int k = 0; k < 2; ++k) xu[k] = -ca * (0.5 * rp * n[k] + 0.5 * (rp - rm) * dl[k]) * dyr;
    // velocity flux Ru_d = -[ca/2 (rp up_d unp + rm um_d unm) + pa n_d + ca/2 lam (rp up_d - rm um_d)]  :1938-1950
#pragma unroll
    for (int d = 0; d < 2; ++d) {
      xr += -ca * (0.5 * up[d] * unp + 0.5 * lam * up[d]) * dyu[d];
#pragma unroll
      for (int k = 0; k < 2; ++k) {
        const double dk = d == k ? 1.0 : 0.0;
        xu[k] += -ca * (0.5 * rp * (dk * unp + up[d] * n[k]) + 0.5 * lam * rp * dk +
                        0.5 * (rp * up[d] - rm * um[d]) * dl[k]) * dyu[d];
      }
      xp += -ct * prm.invMa2 * 0.5 * n[d] * dyu[d];
    }
    // pressure flux Rp = -[ca Ma^2 (kin + lam/2 jk) + ct (ent + lam/2 je)]  (stage 1)  :1057-1079
    xr += -prm.Ma2 * ca * (0.25 * uup * unp + 0.25 * lam * uup) * dyp;
#pragma unroll
    for (int k = 0; k < 2; ++k)
      xu[k] += -(ca * prm.Ma2 * (0.5 * rp * up[k] * unp + 0.25 * uup * rp * n[k] + 0.5 * lam * rp * up[k] +
                                 0.5 * jk * dl[k]) +
                 ct * (0.5 * prm.gg * pp * n[k] + 0.5 * je * dl[k])) * dyp;
    xp += -ct * (0.5 * prm.gg * unp + 0.5 * lam * prm.g1) * dyp;
    flux[0] = xr;
    flux[1] = xu[0];
    flux[2] = xu[1];
    flux[3] = xp;
    flux[4] = flux[5] = flux[6] = 0.0;
  }

  template <int G>
  __device__ __forceinline__ static void boundary(const Params& prm, const double* vp, const double* n,
                                                  double* flux) {
    // wall pressure term of the velocity equation, p_D = p:  Ru = -ct/Ma^2 p n   :2189-2305
    const double ct = prm.ct[0] * prm.dt;
    flux[3] = -ct * prm.invMa2 * (vp[8] * n[0] + vp[9] * n[1]);
  }
};

// Tangent-linear (Jacobian-vector product) of the same operator: the forward's structure
// (values only, tested with phi and grad phi) on the pairs (v, dv); the wave speed is
// differentiated along the forward's branch as in the adjoint, so that
// <ybar, J dv> = <J^T ybar, dv> holds to rounding (the dot-product test).
// One group: rho0, u0 (2), p0, rho2, u_fixed (2), then d of each.  Outputs: rho, u, p.
struct RhsTlm1Phys {
  static constexpr int NG = 1;
  static constexpr bool FACES = true, NEED_X = true, ACCUMULATE = false;
  static constexpr bool FOLD = true;  // z-face folding measured faster (1.53 -> 1.43 ms, 0.97 -> 0.90 ms)
  static constexpr int NOUT_ARR = 3, NOUT = 4;
  using Params = RhsParams;
  using real = double;
  static constexpr int out_ncomp(int a) { return a == 1 ? 2 : 1; }
  static constexpr bool has_val(int) { return true; }
  static constexpr bool has_grad(int) { return true; }
  static constexpr int narr_of(int) { return 10; }
  static constexpr int nf_of(int) { return 14; }
  static constexpr int nfc_of(int) { return 14; }
  template <int G>
  struct Grp {
    static constexpr int NARR = 10;
    static constexpr bool FACE = true;
    static constexpr int ncomp(int a) { return (a == 1 || a == 4 || a == 6 || a == 9) ? 2 : 1; }
    static constexpr bool face_only(int) { return false; }
  };

  // v: rho ux uz p rho2 fx fz | drho dux duz dp drho2 dfx dfz
  template <int G>
  __device__ __forceinline__ static void point(const Params& prm, const double* v, const PointGeo& pg, double* val,
                                               double (*gr)[2]) {
    double e0, e1, fac;
    gravity_dir(prm, pg, e0, e1, fac);
    const double rho = v[0], u[2] = {v[1], v[2]}, p = v[3], r2 = v[4], f[2] = {v[5], v[6]};
    const double dr = v[7], du[2] = {v[8], v[9]}, dp = v[10], dr2 = v[11], df[2] = {v[12], v[13]};
    const double e[2] = {e0, e1};
    const double ca = prm.ca[0] * prm.dt, cg = prm.cg[0] * prm.dt, ct = prm.ct[0] * prm.dt, cgI = prm.cgI * prm.dt;
    const double uu = u[0] * u[0] + u[1] * u[1], udu = u[0] * du[0] + u[1] * du[1];
    const double ue = u[0] * e0 + u[1] * e1, due = du[0] * e0 + du[1] * e1;
    // density
    val[0] += dr;
#pragma unroll
    for (int k = 0; k < 2; ++k) gr[0][k] += ca * (dr * u[k] + rho * du[k]);
    // velocity
#pragma unroll
    for (int d = 0; d < 2; ++d) {
      val[1 + d] += dr * u[d] + rho * du[d] - cg * prm.invFr2 * fac * e[d] * dr - cgI * prm.invFr2 * fac * e[d] * dr2;
#pragma unroll
      for (int k = 0; k < 2; ++k)
        gr[1 + d][k] += ca * (dr * u[d] * u[k] + rho * du[d] * u[k] + rho * u[d] * du[k]) +
                        (d == k ? ct * prm.invMa2 * dp : 0.0);
    }
    // pressure
    const double s = 0.5 * ca * prm.Ma2 * uu * rho + ct * prm.gg * p;
    const double ds = 0.5 * ca * prm.Ma2 * (2.0 * udu * rho + uu * dr) + ct * prm.gg * dp;
    const double ff = f[0] * f[0] + f[1] * f[1], fdf = f[0] * df[0] + f[1] * df[1];
    const double fe = f[0] * e0 + f[1] * e1, dfe = df[0] * e0 + df[1] * e1;
    val[3] += dp * prm.g1 + 0.5 * prm.Ma2 * (dr * uu + 2.0 * rho * udu) - cg * prm.Ma2Fr2 * fac * (dr * ue + rho * due) -
              0.5 * prm.Ma2 * (dr2 * ff + 2.0 * r2 * fdf) - cgI * prm.Ma2Fr2 * fac * (dr2 * fe + r2 * dfe);
#pragma unroll
    for (int k = 0; k < 2; ++k) gr[3][k] += ds * u[k] + s * du[k];
  }

  template <int G>
  __device__ __forceinline__ static void face(const Params& prm, const double* vp, const double* vm,
                                              const double* n, double* flux) {
    const double rp = vp[0], up[2] = {vp[1], vp[2]}, pp = vp[3];
    const double rm = vm[0], um[2] = {vm[1], vm[2]}, pm = vm[3];
    const double drp = vp[7], dup[2] = {vp[8], vp[9]}, dpp = vp[10];
    const double drm = vm[7], dum[2] = {vm[8], vm[9]}, dpm = vm[10];
    const double unp = up[0] * n[0] + up[1] * n[1], unm = um[0] * n[0] + um[1] * n[1];
    const double dunp = dup[0] * n[0] + dup[1] * n[1], dunm = dum[0] * n[0] + dum[1] * n[1];
    const bool own = fabs(unp) >= fabs(unm);
    const double lam = own ? fabs(unp) : fabs(unm);
    const double sgn = own ? (unp > 0.0 ? 1.0 : (unp < 0.0 ? -1.0 : 0.0)) : (unm > 0.0 ? 1.0 : (unm < 0.0 ? -1.0 : 0.0));
    const double dlam = sgn * (own ? dunp : dunm);
    const double ca = prm.ca[0] * prm.dt, ct = prm.ct[0] * prm.dt;
    // density :519-526
    flux[0] = -ca * (0.5 * (drp * unp + rp * dunp + drm * unm + rm * dunm) + 0.5 * dlam * (rp - rm) +
                     0.5 * lam * (drp - drm));
    // velocity :1938-1950
    const double dpa = ct * prm.invMa2 * 0.5 * (dpp + dpm);
#pragma unroll
    for (int d = 0; d < 2; ++d) {
      const double dqp = drp * up[d] + rp * dup[d], dqm = drm * um[d] + rm * dum[d];  // d(rho u_d)
      const double tp = dqp * unp + rp * up[d] * dunp, tm = dqm * unm + rm * um[d] * dunm;
      flux[1 + d] = -(ca * 0.5 * (tp + tm) + dpa * n[d] + ca * 0.5 * (dlam * (rp * up[d] - rm * um[d]) + lam * (dqp - dqm)));
    }
    // pressure (stage 1) :1057-1079
    const double uup = up[0] * up[0] + up[1] * up[1], uum = um[0] * um[0] + um[1] * um[1];
    const double udp = up[0] * dup[0] + up[1] * dup[1], udm = um[0] * dum[0] + um[1] * dum[1];
    const double dkin = 0.5 * (0.5 * (2.0 * udp * rp * unp + uup * drp * unp + uup * rp * dunp) +
                               0.5 * (2.0 * udm * rm * unm + uum * drm * unm + uum * rm * dunm));
    const double jk = rp * 0.5 * uup - rm * 0.5 * uum;
    const double djk = 0.5 * drp * uup + rp * udp - 0.5 * drm * uum - rm * udm;
    const double dent = 0.5 * prm.gg * (dpp * unp + pp * dunp + dpm * unm + pm * dunm);
    const double je = prm.g1 * (pp - pm), dje = prm.g1 * (dpp - dpm);
    flux[3] = -(ca * prm.Ma2 * (dkin + 0.5 * dlam * jk + 0.5 * lam * djk) + ct * (dent + 0.5 * dlam * je + 0.5 * lam * dje));
  }

  template <int G>
  __device__ __forceinline__ static void boundary(const Params& prm, const double* vp, const double* n,
                                                  double* flux) {
    const double s = prm.ct[0] * prm.dt * prm.invMa2 * vp[10];  // :2189-2305, p_D = p
    flux[1] = -s * n[0];
    flux[2] = -s * n[1];
  }
};

// ------------------------------------------------------------- implicit operators
// B^T (vmult_pressure transposed, euler_operator.h:1512-1617): pbar = B^T ubar.
//   cell:  (B p)_{i,d} = -c int p d_d psi_i  ->  pbar_j = -c int phi_j div(ubar_h)
//   face:  c {p} n.psi  -> own side c/2 n, so  pbar += c/2 (ubar+ - ubar-).n
//   wall:  c p n.psi    ->  pbar += c ubar+.n
struct BTPhys {
  static constexpr int NG = 1;
  static constexpr bool FACES = true, NEED_X = false, ACCUMULATE = false;
  static constexpr int NOUT_ARR = 1, NOUT = 1;
  using Params = BParams;
  using real = double;
  static constexpr int out_ncomp(int) { return 1; }
  static constexpr bool has_val(int) { return true; }
  static constexpr bool has_grad(int) { return false; }
  static constexpr int narr_of(int) { return 1; }
  static constexpr int nf_of(int) { return 2; }
  static constexpr int nfc_of(int) { return 2; }
  static constexpr int nfg_of(int) { return 2; }
  template <int G>
  struct Grp {
    static constexpr int NARR = 1;
    static constexpr bool FACE = true;
    static constexpr int ncomp(int) { return 2; }
    static constexpr bool face_only(int) { return false; }
  };
  template <int G>
  __device__ __forceinline__ static void point(const Params& prm, const double* v, const double* deta,
                                               const PointGeo& pg, double* val, double (*)[2]) {
    const double J00 = pg.J[0], J01 = pg.J[1], J10 = pg.J[2], J11 = pg.J[3];
    const double idet = 1.0 / (J00 * J11 - J01 * J10);
    const double dxux = (J11 * v[2] - J10 * deta[0]) * idet;  // d ubar_x / dx
    const double dzuz = (J00 * deta[1] - J01 * v[3]) * idet;  // d ubar_z / dz
    val[0] += -prm.c * (dxux + dzuz);
  }
  template <int G>
  __device__ __forceinline__ static void face(const Params& prm, const double* vp, const double* vm,
                                              const double* n, double* flux) {
    flux[0] = prm.c * 0.5 * ((vp[0] - vm[0]) * n[0] + (vp[1] - vm[1]) * n[1]);
  }
  template <int G>
  __device__ __forceinline__ static void boundary(const Params& prm, const double* vp, const double* n,
                                                  double* flux) {
    flux[0] = prm.c * (vp[0] * n[0] + vp[1] * n[1]);
  }
};

// Jacobian of C (vmult_enthalpy, euler_operator.h:1413-1507) at w, applied to dw; the
// wave speed lambda(w) is differentiated along the forward's branch.
//   cell:  -cdt gg p_f dw . grad phi
//   face:  cdt (gg/2 (p_f+ dw+.n + p_f- dw-.n) + g1/2 dlambda (p_f+ - p_f-))
// One group: w (2), dw (2), p_f.  Output: a pressure-space field.
struct CTlmPhys {
  static constexpr int NG = 1;
  static constexpr bool FACES = true, NEED_X = false, ACCUMULATE = false;
  static constexpr int NOUT_ARR = 1, NOUT = 1;
  using Params = CParams;
  using real = double;
  static constexpr int out_ncomp(int) { return 1; }
  static constexpr bool has_val(int) { return false; }
  static constexpr bool has_grad(int) { return true; }
  static constexpr int narr_of(int) { return 3; }
  static constexpr int nf_of(int) { return 5; }
  static constexpr int nfc_of(int) { return 5; }
  template <int G>
  struct Grp {
    static constexpr int NARR = 3;
    static constexpr bool FACE = true;
    static constexpr int ncomp(int a) { return a < 2 ? 2 : 1; }
    static constexpr bool face_only(int) { return false; }
  };
  template <int G>
  __device__ __forceinline__ static void point(const Params& prm, const double* v, const PointGeo&, double*,
                                               double (*gr)[2]) {
    const double s = -prm.cdt * prm.gg * v[4];
    gr[0][0] += s * v[2];
    gr[0][1] += s * v[3];
  }
  template <int G>
  __device__ __forceinline__ static void face(const Params& prm, const double* vp, const double* vm,
                                              const double* n, double* flux) {
    const double wnp = vp[0] * n[0] + vp[1] * n[1], wnm = vm[0] * n[0] + vm[1] * n[1];
    const double dwnp = vp[2] * n[0] + vp[3] * n[1], dwnm = vm[2] * n[0] + vm[3] * n[1];
    const bool own = fabs(wnp) >= fabs(wnm);
    const double sg = own ? (wnp > 0.0 ? 1.0 : (wnp < 0.0 ? -1.0 : 0.0)) : (wnm > 0.0 ? 1.0 : (wnm < 0.0 ? -1.0 : 0.0));
    const double dlam = sg * (own ? dwnp : dwnm);
    flux[0] = prm.cdt * (0.5 * prm.gg * (vp[4] * dwnp + vm[4] * dwnm) + 0.5 * dlam * prm.g1 * (vp[4] - vm[4]));
  }
  template <int G>
  __device__ __forceinline__ static void boundary(const Params&, const double*, const double*, double*) {}
};

// Its transpose: wbar = J_C(w)^T pbar.
//   cell:  wbar = -cdt gg p_f grad(pbar_h) (tested with phi)
//   face:  own-side derivative applied to the cotangent jump:
//          wbar+ += cdt (gg/2 p_f+ n + g1/2 (p_f+ - p_f-) dlambda/dw+) (pbar+ - pbar-)
// One group: w (2), p_f, pbar (gradient field).  Output: wbar (2).
struct CTPhys {
  static constexpr int NG = 1;
  static constexpr bool FACES = true, NEED_X = false, ACCUMULATE = false;
  static constexpr int NOUT_ARR = 1, NOUT = 2;
  using Params = CParams;
  using real = double;
  static constexpr int out_ncomp(int) { return 2; }
  static constexpr bool has_val(int) { return true; }
  static constexpr bool has_grad(int) { return false; }
  static constexpr int narr_of(int) { return 3; }
  static constexpr int nf_of(int) { return 4; }
  static constexpr int nfc_of(int) { return 4; }
  static constexpr int nfg_of(int) { return 1; }
  template <int G>
  struct Grp {
    static constexpr int NARR = 3;
    static constexpr bool FACE = true;
    static constexpr int ncomp(int a) { return a == 0 ? 2 : 1; }
    static constexpr bool face_only(int) { return false; }
  };
  template <int G>
  __device__ __forceinline__ static void point(const Params& prm, const double* v, const double* deta,
                                               const PointGeo& pg, double* val, double (*)[2]) {
    const double J00 = pg.J[0], J01 = pg.J[1], J10 = pg.J[2], J11 = pg.J[3];
    const double idet = 1.0 / (J00 * J11 - J01 * J10);
    const double gx = (J11 * v[4] - J10 * deta[0]) * idet, gz = (J00 * deta[0] - J01 * v[4]) * idet;
    const double s = -prm.cdt * prm.gg * v[2];
    val[0] += s * gx;
    val[1] += s * gz;
  }
  template <int G>
  __device__ __forceinline__ static void face(const Params& prm, const double* vp, const double* vm,
                                              const double* n, double* flux) {
    const double wnp = vp[0] * n[0] + vp[1] * n[1], wnm = vm[0] * n[0] + vm[1] * n[1];
    const bool own = fabs(wnp) >= fabs(wnm);
    const double sg = own ? (wnp > 0.0 ? 1.0 : (wnp < 0.0 ? -1.0 : 0.0)) : 0.0;
    const double jump = vp[3] - vm[3];
#pragma unroll
    for (int k = 0; k < 2; ++k)
      flux[k] = prm.cdt * (0.5 * prm.gg * vp[2] * n[k] + 0.5 * prm.g1 * (vp[2] - vm[2]) * sg * n[k]) * jump;
  }
  template <int G>
  __device__ __forceinline__ static void boundary(const Params&, const double*, const double*, double*) {}
};

// Derivatives of the implicit operators with respect to their fixed coefficients, transposed
// (the tangents are the forward operators themselves, since A is linear in rho_for_fixed and C
// is linear in pres_fixed):
//   A(rho) x = int rho x . phi  ->  (d/drho [A(rho) x])^T y :  rhobar_j = int psi_j (x . y)
// One group: x (2), y (2), no faces.  Output: rhobar (1).
struct MassRhoTPhys {
  static constexpr int NG = 1;
  static constexpr bool FACES = false, NEED_X = false, ACCUMULATE = false;
  static constexpr int NOUT_ARR = 1, NOUT = 1;
  using Params = MassParams;
  using real = double;
  static constexpr int out_ncomp(int) { return 1; }
  static constexpr bool has_val(int) { return true; }
  static constexpr bool has_grad(int) { return false; }
  static constexpr int narr_of(int) { return 2; }
  static constexpr int nf_of(int) { return 4; }
  static constexpr int nfc_of(int) { return 4; }
  template <int G>
  struct Grp {
    static constexpr int NARR = 2;
    static constexpr bool FACE = false;
    static constexpr int ncomp(int) { return 2; }
    static constexpr bool face_only(int) { return false; }
  };
  template <int G>
  __device__ __forceinline__ static void point(const Params&, const double* v, const PointGeo&, double* val,
                                               double (*)[2]) {
    val[0] += v[0] * v[2] + v[1] * v[3];
  }
  template <int G>
  __device__ __forceinline__ static void face(const Params&, const double*, const double*, const double*, double*) {}
  template <int G>
  __device__ __forceinline__ static void boundary(const Params&, const double*, const double*, double*) {}
};

//   C(w; p_f) (vmult_enthalpy, euler_operator.h:1413-1507) is linear in p_f for a fixed w:
//   (d/dp_f [C(w; p_f)])^T pbar = pfbar:
//   cell:  pfbar = -cdt gg w . grad(pbar_h) (tested with psi)
//   face:  F = cdt (gg/2 (p_f+ w+.n + p_f- w-.n) + g1/2 lambda(w) (p_f+ - p_f-)) enters the two
//          sides with opposite signs, so  pfbar+ += cdt (gg/2 w+.n + g1/2 lambda) (pbar+ - pbar-)
//   walls: no term (as C).
// One group: w (2), pbar (gradient field).  Output: pfbar (1).
struct CPfTPhys {
  static constexpr int NG = 1;
  static constexpr bool FACES = true, NEED_X = false, ACCUMULATE = false;
  static constexpr int NOUT_ARR = 1, NOUT = 1;
  using Params = CParams;
  using real = double;
  static constexpr int out_ncomp(int) { return 1; }
  static constexpr bool has_val(int) { return true; }
  static constexpr bool has_grad(int) { return false; }
  static constexpr int narr_of(int) { return 2; }
  static constexpr int nf_of(int) { return 3; }
  static constexpr int nfc_of(int) { return 3; }
  static constexpr int nfg_of(int) { return 1; }
  template <int G>
  struct Grp {
    static constexpr int NARR = 2;
    static constexpr bool FACE = true;
    static constexpr int ncomp(int a) { return a == 0 ? 2 : 1; }
    static constexpr bool face_only(int) { return false; }
  };
  template <int G>
  __device__ __forceinline__ static void point(const Params& prm, const double* v, const double* deta,
                                               const PointGeo& pg, double* val, double (*)[2]) {
    const double J00 = pg.J[0], J01 = pg.J[1], J10 = pg.J[2], J11 = pg.J[3];
    const double idet = 1.0 / (J00 * J11 - J01 * J10);
    // v[3]: d/dxi of pbar (the gradient slot after the three cell fields), deta[0]: d/deta
    const double gx = (J11 * v[3] - J10 * deta[0]) * idet, gz = (J00 * deta[0] - J01 * v[3]) * idet;
    val[0] += -prm.cdt * prm.gg * (v[0] * gx + v[1] * gz);
  }
  template <int G>
  __device__ __forceinline__ static void face(const Params& prm, const double* vp, const double* vm,
                                              const double* n, double* flux) {
    const double wnp = vp[0] * n[0] + vp[1] * n[1], wnm = vm[0] * n[0] + vm[1] * n[1];
    const double lam = fmax(fabs(wnp), fabs(wnm));
    flux[0] = prm.cdt * (0.5 * prm.gg * wnp + 0.5 * prm.g1 * lam) * (vp[2] - vm[2]);
  }
  template <int G>
  __device__ __forceinline__ static void boundary(const Params&, const double*, const double*, double*) {}
};

}  // namespace af

namespace af {

// ------------------------------------------------------------- automatic rhs derivatives
// Tangent-linear and adjoint of the fused rhs triple RhsPhys<STAGE, 7> for every stage, from
// its physics evaluated with dual numbers (af_physics.cuh), so that the derivatives follow the
// forward code exactly (quirks included).  The rhs is a sum over the policy's groups of terms
// that depend on that group's fields only, which both policies use.

// Tangent: dy = sum_G J_G dv_G.  Group G's arrays: its cell arrays, their tangents, then the
// face-only arrays (the stage-2 kinetic-jump quirk) and their tangents.
template <int STAGE>
struct RhsTanPhys {
  using Base = RhsPhys<STAGE, 7>;
  static constexpr int NG = Base::NG;
  static constexpr bool FACES = true, NEED_X = true, ACCUMULATE = false;
  static constexpr int NOUT_ARR = Base::NOUT_ARR, NOUT = Base::NOUT;
  using Params = RhsParams;
  using real = double;
  static constexpr int out_ncomp(int a) { return Base::out_ncomp(a); }
  static constexpr bool has_val(int o) { return Base::has_val(o); }
  static constexpr bool has_grad(int o) { return Base::has_grad(o); }
  static constexpr int narr_of(int g) { return 2 * Base::narr_of(g); }
  static constexpr int nf_of(int g) { return 2 * Base::nf_of(g); }
  static constexpr int nfc_of(int g) { return 2 * Base::nfc_of(g); }
  template <int G>
  struct Grp {
    using BG = typename Base::template Grp<G>;
    static constexpr int NB = BG::NARR;
    static constexpr bool Q = Base::quirk_group(G);  // its last base array is face-only
    static constexpr int NBC = Q ? NB - 1 : NB;
    static constexpr int NARR = 2 * NB;
    static constexpr bool FACE = BG::FACE;
    static constexpr int base_of(int a) { return a < NBC ? a : (a < 2 * NBC ? a - NBC : NBC); }
    static constexpr int ncomp(int a) { return BG::ncomp(base_of(a)); }
    static constexpr bool face_only(int a) { return Q && a >= 2 * NBC; }
  };
  template <int G>
  __device__ __forceinline__ static void point(const Params& prm, const double* v, const PointGeo& pg, double* val,
                                               double (*gr)[2]) {
    constexpr int NFC = Base::nfc_of(G), NF = Base::nf_of(G);
    Dual vb[NF], fv[NOUT], fg[NOUT][2];
#pragma unroll
    for (int k = 0; k < NF; ++k) vb[k] = k < NFC ? Dual{v[k], v[NFC + k]} : Dual{0.0, 0.0};
#pragma unroll
    for (int o = 0; o < NOUT; ++o) fv[o] = fg[o][0] = fg[o][1] = Dual{0.0, 0.0};
    Base::template point_t<G, Dual>(prm, vb, pg, fv, fg);
#pragma unroll
    for (int o = 0; o < NOUT; ++o) {
      val[o] += fv[o].d;
      gr[o][0] += fg[o][0].d;
      gr[o][1] += fg[o][1].d;
    }
  }
  template <int G>
  __device__ __forceinline__ static void load_face(const double* w, Dual* out) {
    constexpr int NFC = Base::nfc_of(G), NF = Base::nf_of(G), NFO = NF - NFC;
#pragma unroll
    for (int k = 0; k < NF; ++k)
      out[k] = k < NFC ? Dual{w[k], w[NFC + k]} : Dual{w[2 * NFC + (k - NFC)], w[2 * NFC + NFO + (k - NFC)]};
  }
  template <int G>
  __device__ __forceinline__ static void face(const Params& prm, const double* vp, const double* vm, const double* n,
                                              double* flux) {
    constexpr int NF = Base::nf_of(G);
    Dual a[NF], b[NF], fl[NOUT];
    load_face<G>(vp, a);
    load_face<G>(vm, b);
#pragma unroll
    for (int o = 0; o < NOUT; ++o) fl[o] = Dual{0.0, 0.0};
    Base::template face_t<G, Dual>(prm, a, b, n, fl);
#pragma unroll
    for (int o = 0; o < NOUT; ++o) flux[o] = fl[o].d;
  }
  template <int G>
  __device__ __forceinline__ static void boundary(const Params& prm, const double* vp, const double* n,
                                                  double* flux) {
    constexpr int NF = Base::nf_of(G);
    Dual a[NF], fl[NOUT];
    load_face<G>(vp, a);
#pragma unroll
    for (int o = 0; o < NOUT; ++o) fl[o] = Dual{0.0, 0.0};
    Base::template boundary_t<G, Dual>(prm, a, n, fl);
#pragma unroll
    for (int o = 0; o < NOUT; ++o) flux[o] = fl[o].d;
  }
};

// Adjoint of group GB of RhsPhys<STAGE, 7>: xbar_GB = J_GB^T ybar, one launch per group.
// Arrays: the group's cell arrays, the cotangents ybar_rho, ybar_u (2), ybar_p (gradient
// fields), then the group's face-only array (quirk).  Outputs: xbar of the group's arrays.
//   cell:     xbar_s = sum_o [ybar_o df_o/dv_s + grad(ybar_o) . dg_o/dv_s]   (tested with phi)
//   faces:    xbar_s += sum_o dF_o/dv+_s (ybar_o+ - ybar_o-)   (the flux is antisymmetric under
//             a side swap, so the neighbour's term supplies the minus side)
//   boundary: xbar_s += sum_o dF_o/dv+_s ybar_o+
// Each derivative is one dual evaluation seeded in field s.
template <int STAGE, int GB>
struct RhsAdjGPhys {
  using Base = RhsPhys<STAGE, 7>;
  using BG = typename Base::template Grp<GB>;
  static constexpr int NFb = Base::nf_of(GB), NFCb = Base::nfc_of(GB), NFOb = NFb - NFCb;
  static constexpr int NB = BG::NARR;
  static constexpr bool Q = Base::quirk_group(GB);
  static constexpr int NBC = Q ? NB - 1 : NB;
  static constexpr int NG = 1;
  static constexpr bool FACES = BG::FACE, NEED_X = true, ACCUMULATE = false;
  static constexpr int NOUT_ARR = NB, NOUT = NFb;
  static constexpr int NY = Base::NOUT;  // cotangent components: rho, u (2), p
  using Params = RhsParams;
  using real = double;
  static constexpr int out_ncomp(int a) { return BG::ncomp(a); }
  static constexpr bool has_val(int) { return true; }
  static constexpr bool has_grad(int) { return false; }
  static constexpr int narr_of(int) { return NB + 3; }
  static constexpr int nf_of(int) { return NFb + NY; }
  static constexpr int nfc_of(int) { return NFCb + NY; }
  static constexpr int nfg_of(int) { return NY; }
  template <int G>
  struct Grp {
    static constexpr int NARR = NB + 3;
    static constexpr bool FACE = BG::FACE;
    static constexpr int ncomp(int a) {
      return a < NBC ? BG::ncomp(a) : (a < NBC + 3 ? (a == NBC + 1 ? 2 : 1) : BG::ncomp(NBC));
    }
    static constexpr bool face_only(int a) { return Q && a == NBC + 3; }
  };
  template <int G>
  __device__ __forceinline__ static void point(const Params& prm, const double* v, const double* deta,
                                               const PointGeo& pg, double* val, double (*)[2]) {
    const double J00 = pg.J[0], J01 = pg.J[1], J10 = pg.J[2], J11 = pg.J[3];
    const double idet = 1.0 / (J00 * J11 - J01 * J10);
    double y[NY], gy[NY][2];
#pragma unroll
    for (int o = 0; o < NY; ++o) {
      y[o] = v[NFCb + o];
      const double dx = v[NFCb + NY + o], de = deta[o];  // d/dxi slots follow the cell fields
      gy[o][0] = (J11 * dx - J10 * de) * idet;
      gy[o][1] = (J00 * de - J01 * dx) * idet;
    }
#pragma unroll
    for (int s = 0; s < NFCb; ++s) {
      Dual vb[NFb], fv[NY], fg[NY][2];
#pragma unroll
      for (int k = 0; k < NFb; ++k) vb[k] = Dual{k < NFCb ? v[k] : 0.0, k == s ? 1.0 : 0.0};
#pragma unroll
      for (int o = 0; o < NY; ++o) fv[o] = fg[o][0] = fg[o][1] = Dual{0.0, 0.0};
      Base::template point_t<GB, Dual>(prm, vb, pg, fv, fg);
      double acc = 0.0;
#pragma unroll
      for (int o = 0; o < NY; ++o) acc += y[o] * fv[o].d + gy[o][0] * fg[o][0].d + gy[o][1] * fg[o][1].d;
      val[s] += acc;
    }
  }
  __device__ __forceinline__ static double field(const double* w, int k) {
    return k < NFCb ? w[k] : w[NFCb + NY + (k - NFCb)];
  }
  template <int G>
  __device__ __forceinline__ static void face(const Params& prm, const double* vp, const double* vm, const double* n,
                                              double* flux) {
    double dy[NY];
#pragma unroll
    for (int o = 0; o < NY; ++o) dy[o] = vp[NFCb + o] - vm[NFCb + o];
#pragma unroll
    for (int s = 0; s < NFb; ++s) {
      Dual a[NFb], b[NFb], fl[NY];
#pragma unroll
      for (int k = 0; k < NFb; ++k) {
        a[k] = Dual{field(vp, k), k == s ? 1.0 : 0.0};
        b[k] = Dual{field(vm, k), 0.0};
      }
#pragma unroll
      for (int o = 0; o < NY; ++o) fl[o] = Dual{0.0, 0.0};
      Base::template face_t<GB, Dual>(prm, a, b, n, fl);
      double acc = 0.0;
#pragma unroll
      for (int o = 0; o < NY; ++o) acc += fl[o].d * dy[o];
      flux[s] = acc;
    }
  }
  template <int G>
  __device__ __forceinline__ static void boundary(const Params& prm, const double* vp, const double* n,
                                                  double* flux) {
#pragma unroll
    for (int s = 0; s < NFb; ++s) {
      Dual a[NFb], fl[NY];
#pragma unroll
      for (int k = 0; k < NFb; ++k) a[k] = Dual{field(vp, k), k == s ? 1.0 : 0.0};
#pragma unroll
      for (int o = 0; o < NY; ++o) fl[o] = Dual{0.0, 0.0};
      Base::template boundary_t<GB, Dual>(prm, a, n, fl);
      double acc = 0.0;
#pragma unroll
      for (int o = 0; o < NY; ++o) acc += fl[o].d * vp[NFCb + o];
      flux[s] = acc;
    }
  }
};

}  // namespace af
