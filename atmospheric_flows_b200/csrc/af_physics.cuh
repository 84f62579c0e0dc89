// af_physics.cuh -- pointwise integrands and numerical fluxes of the reference's operators,
// as policies for the generic kernel in af_cellop.cuh.
//
// Each policy restates, per group of input fields, one family of EULEROperator integrals
// (file:line in the reference's euler_operator.h):
//   RhsPhys<STAGE, MASK>  assemble_rhs_{cell,face,boundary}_term_{rho_update,pressure,
//                         velocity_fixed} for HYPERBOLIC_stage = STAGE, fused over the
//                         equations selected by MASK (1 density, 2 velocity, 4 pressure):
//                         :344-692, :745-1361, :1622-2305
//   BPhys                 assemble_{cell,face,boundary}_term_pressure (matrix B) :1512-1617
//   CPhys<WITH_D, SIGN>   assemble_{cell,face}_term_enthalpy (matrix C) :1413-1507, with
//                         the internal-energy mass D (:1386-1408) fused for the Schur
//                         complement output D p - C w (:2374-2408)
//   MassPhys<NC, W>       assemble_cell_term_{rho_update,internal_energy,velocity_fixed}
//                         (:715-740, :1386-1408, :2330-2357)
//
// Conventions of the cell-centric kernel: the calling cell is always the "+" side, n its
// outward unit normal, and the returned flux is the integrand tested against the cell's
// own basis functions on that face (already carrying the reference's phi_p sign).
// Integrands are algebraically equal to the reference's (e.g. rho*(p/((g-1) rho)) is
// formed as p/(g-1)); the oracle keeps the literal forms and parity is checked at 1e-12.
#pragma once

#include "af_cellop.cuh"

namespace af {

struct RhsParams {
  double dt, Ma2, invMa2, invFr2, Ma2Fr2, a2;
  double g1, gg;          // 1/(gamma-1), gamma/(gamma-1)
  double ca[3], ct[3];    // explicit weights a_j and a~_j of the stage's explicit terms
  double cg[3], cgI;      // gravity weights of the explicit terms and of the implicit one
  int radial;             // 0: e_z, |g| const; 1: e_r = X/|X|, factor a^2/|X|^2
  // Rayleigh damping of the momentum towards (sp_u, 0) (the 2D hill case's upper sponge and
  // lateral relaxation zones; no counterpart in the reference): rate tau(x, z) of sponge_rate
  int sponge;
  double sp_z0, sp_z1, sp_rate, sp_x0, sp_x1, sp_width, sp_rate_lat, sp_u;
  // the point functions read the physical position for radial gravity and for the sponge
  __device__ bool needs_position() const { return radial != 0 || sponge != 0; }
};

// tau(x, z) = rate sin^2(pi/2 (z - z0)/(z1 - z0)) above z0, plus rate_lat cos^2(pi/2 d/width)
// within width of the nearer lateral boundary (d its distance); 1/s in the non-dimensional units
__device__ __forceinline__ double sponge_rate(const RhsParams& prm, const PointGeo& pg) {
  const double half_pi = 1.5707963267948966;
  double tau = 0.0;
  if (pg.X[1] > prm.sp_z0) {
    const double s = sin(half_pi * (pg.X[1] - prm.sp_z0) / (prm.sp_z1 - prm.sp_z0));
    tau += prm.sp_rate * s * s;
  }
  const double d = fmin(pg.X[0] - prm.sp_x0, prm.sp_x1 - pg.X[0]);
  if (d < prm.sp_width) {
    const double c = cos(half_pi * d / prm.sp_width);
    tau += prm.sp_rate_lat * c * c;
  }
  return tau;
}

__device__ __forceinline__ void gravity_dir(const RhsParams& prm, const PointGeo& pg, double& e0, double& e1,
                                            double& fac) {
  if (prm.radial) {
    const double r2 = pg.X[0] * pg.X[0] + pg.X[1] * pg.X[1];
    const double ir = 1.0 / sqrt(r2);
    e0 = pg.X[0] * ir;
    e1 = pg.X[1] * ir;
    fac = prm.a2 / r2;
  } else {
    e0 = 0.0;
    e1 = 1.0;
    fac = 1.0;
  }
}

// Forward-mode dual number (value, one directional derivative) for the automatic tangents and
// adjoints of the rhs policies: the rhs physics below is written once for a scalar type T and
// evaluated with T = double (the operator) or T = Dual (its derivatives).  |x| and max(a, b)
// follow the branch of the value (at max(a, b) the first argument when a >= b), which is the
// frozen-branch derivative of the Rusanov wave speed.
struct Dual {
  double v, d;
};
__device__ __forceinline__ Dual operator+(Dual a, Dual b) { return {a.v + b.v, a.d + b.d}; }
__device__ __forceinline__ Dual operator-(Dual a, Dual b) { return {a.v - b.v, a.d - b.d}; }
__device__ __forceinline__ Dual operator-(Dual a) { return {-a.v, -a.d}; }
__device__ __forceinline__ Dual operator*(Dual a, Dual b) { return {a.v * b.v, fma(a.v, b.d, a.d * b.v)}; }
__device__ __forceinline__ Dual operator+(Dual a, double b) { return {a.v + b, a.d}; }
__device__ __forceinline__ Dual operator+(double a, Dual b) { return {a + b.v, b.d}; }
__device__ __forceinline__ Dual operator-(Dual a, double b) { return {a.v - b, a.d}; }
__device__ __forceinline__ Dual operator-(double a, Dual b) { return {a - b.v, -b.d}; }
__device__ __forceinline__ Dual operator*(Dual a, double b) { return {a.v * b, a.d * b}; }
__device__ __forceinline__ Dual operator*(double a, Dual b) { return {a * b.v, a * b.d}; }
__device__ __forceinline__ Dual& operator+=(Dual& a, Dual b) { a.v += b.v; a.d += b.d; return a; }
__device__ __forceinline__ Dual& operator-=(Dual& a, Dual b) { a.v -= b.v; a.d -= b.d; return a; }
__device__ __forceinline__ double aabs(double x) { return fabs(x); }
__device__ __forceinline__ double amax(double a, double b) { return fmax(a, b); }
__device__ __forceinline__ Dual aabs(Dual x) { return x.v > 0.0 ? x : (x.v < 0.0 ? -x : Dual{0.0, 0.0}); }
__device__ __forceinline__ Dual amax(Dual a, Dual b) { return a.v >= b.v ? a : b; }

template <int STAGE, int MASK>
struct RhsPhys {
  static constexpr bool RHO = (MASK & 1) != 0, VEL = (MASK & 2) != 0, PRES = (MASK & 4) != 0;
  static constexpr bool HAS_I = STAGE < 3 ? (VEL || PRES) : PRES;
  static constexpr int NG = STAGE + (HAS_I ? 1 : 0);
  static constexpr bool FACES = true, NEED_X = true, ACCUMULATE = false;
  static constexpr bool FOLD = true;  // z-face folding (Layout::FOLD_Z) measured faster here
  static constexpr int NOUT_ARR = (RHO ? 1 : 0) + (VEL ? 1 : 0) + (PRES ? 1 : 0);
  static constexpr int NOUT = (RHO ? 1 : 0) + (VEL ? 2 : 0) + (PRES ? 1 : 0);
  static constexpr int O_RHO = 0, O_U = RHO ? 1 : 0, O_P = (RHO ? 1 : 0) + (VEL ? 2 : 0);
  using Params = RhsParams;
  using real = double;

  static constexpr int out_ncomp(int a) {
    // output arrays in the order rho, u, p (present ones only)
    return (VEL && a == (RHO ? 1 : 0)) ? 2 : 1;
  }
  static constexpr bool has_val(int) { return true; }
  static constexpr bool has_grad(int) { return true; }

  static constexpr bool quirk_group(int g) { return STAGE == 2 && PRES && g == 1; }
  static constexpr int narr_of(int g) {
    if (g < STAGE) return 2 + ((VEL || PRES) ? 1 : 0) + (quirk_group(g) ? 1 : 0);
    return STAGE < 3 ? (1 + (PRES ? 1 : 0)) : 2;
  }
  static constexpr int nf_of(int g) {
    if (g < STAGE) return 3 + ((VEL || PRES) ? 1 : 0) + (quirk_group(g) ? 2 : 0);
    return STAGE < 3 ? (1 + (PRES ? 2 : 0)) : 3;
  }
  static constexpr int nfc_of(int g) { return nf_of(g) - (quirk_group(g) ? 2 : 0); }

  template <int G>
  struct Grp {
    static constexpr bool EXPL = G < STAGE;
    static constexpr int NARR = narr_of(G);
    static constexpr bool FACE = EXPL;
    // explicit: rho_j, u_j, [p_j], [u_0 face-only];  implicit: rho_c, [u_fixed]
    static constexpr int ncomp(int a) { return a == 1 ? 2 : (EXPL && a == 3 ? 2 : 1); }
    static constexpr bool face_only(int a) { return EXPL && a == 3; }
  };

  // The hill's vertical gravity (e_z, |g| constant) and the reference's radial one are two
  // compiled paths (a uniform branch): on the vertical path the terms with e_x = 0 and the
  // factor 1 are left out, which gives bit for bit the same values with fewer operations.
  template <int G, class T>
  __device__ __forceinline__ static void point_t(const Params& prm, const T* v, const PointGeo& pg, T* val,
                                                 T (*gr)[2]) {
    if (prm.radial) point_g<G, T, true>(prm, v, pg, val, gr);
    else point_g<G, T, false>(prm, v, pg, val, gr);
  }

  template <int G, class T, bool RADIAL>
  __device__ __forceinline__ static void point_g(const Params& prm, const T* v, const PointGeo& pg, T* val,
                                                 T (*gr)[2]) {
    double e0 = 0.0, e1 = 1.0, fac = 1.0;
    if constexpr (RADIAL) gravity_dir(prm, pg, e0, e1, fac);
    if constexpr (G < STAGE) {
      const T rho = v[0], ux = v[1], uz = v[2];
      const double ca = prm.ca[G] * prm.dt, cg = prm.cg[G] * prm.dt;
      if constexpr (RHO) {  // euler_operator.h:378-380 (and stage 2/3 analogues)
        if (G == 0) val[O_RHO] += rho;
        gr[O_RHO][0] += ca * rho * ux;
        gr[O_RHO][1] += ca * rho * uz;
      }
      if constexpr (VEL || PRES) {
        const T p = v[3];
        const double ct = prm.ct[G] * prm.dt;
        if constexpr (VEL) {  // :1686-1691
          if (G == 0) { val[O_U] += rho * ux; val[O_U + 1] += rho * uz; }
          if constexpr (RADIAL) {
            const T gfac = cg * prm.invFr2 * rho * fac;
            val[O_U] -= gfac * e0;
            val[O_U + 1] -= gfac * e1;
          } else {
            val[O_U + 1] -= cg * prm.invFr2 * rho;
          }
          if (prm.sponge) {  // -dt a_j tau rho_j (u_j - u_ref)
            const T ct_ = ca * sponge_rate(prm, pg) * rho;
            val[O_U] -= ct_ * (ux - prm.sp_u);
            val[O_U + 1] -= ct_ * uz;
          }
          const T cr = ca * rho, pt = ct * prm.invMa2 * p;
          gr[O_U][0] += cr * ux * ux + pt;
          gr[O_U][1] += cr * ux * uz;
          gr[O_U + 1][0] += cr * uz * ux;
          gr[O_U + 1][1] += cr * uz * uz + pt;
        }
        if constexpr (PRES) {  // :806-813: rho E = p/(g-1) + Ma^2 rho |u|^2 / 2
          const T uu = ux * ux + uz * uz;
          if (G == 0) val[O_P] += p * prm.g1 + 0.5 * prm.Ma2 * rho * uu;
          if constexpr (RADIAL) val[O_P] -= cg * prm.Ma2Fr2 * rho * (ux * e0 + uz * e1) * fac;
          else val[O_P] -= cg * prm.Ma2Fr2 * rho * uz;
          const T s = 0.5 * ca * prm.Ma2 * uu * rho + ct * prm.gg * p;
          gr[O_P][0] += s * ux;
          gr[O_P][1] += s * uz;
        }
      }
    } else {
      const T rc = v[0];
      const double cgI = prm.cgI * prm.dt;
      if constexpr (VEL && STAGE < 3) {
        if constexpr (RADIAL) {
          const T gfac = cgI * prm.invFr2 * rc * fac;
          val[O_U] -= gfac * e0;
          val[O_U + 1] -= gfac * e1;
        } else {
          val[O_U + 1] -= cgI * prm.invFr2 * rc;
        }
      }
      if constexpr (PRES) {
        const T fx = v[1], fz = v[2];
        val[O_P] -= 0.5 * rc * prm.Ma2 * (fx * fx + fz * fz);
        if (STAGE < 3) {
          if constexpr (RADIAL) val[O_P] -= cgI * prm.Ma2Fr2 * rc * (fx * e0 + fz * e1) * fac;
          else val[O_P] -= cgI * prm.Ma2Fr2 * rc * fz;
        }
      }
    }
  }

  // The integrand of point_t mapped to the reference cell (see MappedOf in af_cellop.cuh):
  // every flux of the explicit group is a multiple of the velocity u_j plus pressure times the
  // identity, so its mapped form shares the contravariant velocity (U1, U2) = adj(J) w u_j:
  //   rho:       ca rho (U1, U2)
  //   rho u_x:   ca rho u_x (U1, U2) + pt (A0, -A2)      rho u_z: ca rho u_z (U1, U2) + pt (-A1, A3)
  //   pressure:  s (U1, U2)
  // (ca = a_j dt, pt = a~_j dt p_j / Ma^2, s as in point_t); values are multiplied by |J| w.
  static constexpr bool MAPPED = true;
  template <int G>
  __device__ __forceinline__ static void point_mapped(const Params& prm, const double* v, const PointGeo& pg,
                                                      const double (&A)[4], double dw, double* fv, double* fx,
                                                      double* fe) {
    if (prm.radial) point_mapped_g<G, true>(prm, v, pg, A, dw, fv, fx, fe);
    else point_mapped_g<G, false>(prm, v, pg, A, dw, fv, fx, fe);
  }
  template <int G, bool RADIAL>
  __device__ __forceinline__ static void point_mapped_g(const Params& prm, const double* v, const PointGeo& pg,
                                                        const double (&A)[4], double dw, double* fv, double* fx,
                                                        double* fe) {
    double e0 = 0.0, e1 = 1.0, fac = 1.0;
    if constexpr (RADIAL) gravity_dir(prm, pg, e0, e1, fac);
    if constexpr (G < STAGE) {
      const double rho = v[0], ux = v[1], uz = v[2];
      const double ca = prm.ca[G] * prm.dt, cg = prm.cg[G] * prm.dt;
      const double U1 = A[0] * ux - A[1] * uz, U2 = A[3] * uz - A[2] * ux;
      const double cr = ca * rho;
      if constexpr (RHO) {
        if (G == 0) fv[O_RHO] += rho * dw;
        fx[O_RHO] += cr * U1;
        fe[O_RHO] += cr * U2;
      }
      if constexpr (VEL || PRES) {
        const double p = v[3];
        const double ct = prm.ct[G] * prm.dt;
        if constexpr (VEL) {
          const double rdw = rho * dw;
          if (G == 0) { fv[O_U] += rdw * ux; fv[O_U + 1] += rdw * uz; }
          if constexpr (RADIAL) {
            const double gfac = cg * prm.invFr2 * rdw * fac;
            fv[O_U] -= gfac * e0;
            fv[O_U + 1] -= gfac * e1;
          } else {
            fv[O_U + 1] -= cg * prm.invFr2 * rdw;
          }
          if (prm.sponge) {  // -dt a_j tau rho_j (u_j - u_ref)
            const double ct_ = ca * sponge_rate(prm, pg) * rdw;
            fv[O_U] -= ct_ * (ux - prm.sp_u);
            fv[O_U + 1] -= ct_ * uz;
          }
          const double pt = ct * prm.invMa2 * p;
          const double cx = cr * ux, cz = cr * uz;
          fx[O_U] += cx * U1 + pt * A[0];
          fe[O_U] += cx * U2 - pt * A[2];
          fx[O_U + 1] += cz * U1 - pt * A[1];
          fe[O_U + 1] += cz * U2 + pt * A[3];
        }
        if constexpr (PRES) {
          const double uu = ux * ux + uz * uz;
          double val = G == 0 ? p * prm.g1 + 0.5 * prm.Ma2 * rho * uu : 0.0;
          if constexpr (RADIAL) val -= cg * prm.Ma2Fr2 * rho * (ux * e0 + uz * e1) * fac;
          else val -= cg * prm.Ma2Fr2 * rho * uz;
          fv[O_P] += val * dw;
          const double s = 0.5 * ca * prm.Ma2 * uu * rho + ct * prm.gg * p;
          fx[O_P] += s * U1;
          fe[O_P] += s * U2;
        }
      }
    } else {
      const double rc = v[0];
      const double cgI = prm.cgI * prm.dt;
      if constexpr (VEL && STAGE < 3) {
        if constexpr (RADIAL) {
          const double gfac = cgI * prm.invFr2 * rc * fac * dw;
          fv[O_U] -= gfac * e0;
          fv[O_U + 1] -= gfac * e1;
        } else {
          fv[O_U + 1] -= cgI * prm.invFr2 * rc * dw;
        }
      }
      if constexpr (PRES) {
        const double fxv = v[1], fzv = v[2];
        double val = 0.5 * rc * prm.Ma2 * (fxv * fxv + fzv * fzv);
        if (STAGE < 3) {
          if constexpr (RADIAL) val += cgI * prm.Ma2Fr2 * rc * (fxv * e0 + fzv * e1) * fac;
          else val += cgI * prm.Ma2Fr2 * rc * fzv;
        }
        fv[O_P] -= val * dw;
      }
    }
  }

  template <int G, class T>
  __device__ __forceinline__ static void face_t(const Params& prm, const T* vp, const T* vm, const double* n,
                                                T* flux) {
    if constexpr (G < STAGE) {
      const T rp = vp[0], upx = vp[1], upz = vp[2];
      const T rm = vm[0], umx = vm[1], umz = vm[2];
      const T unp = upx * n[0] + upz * n[1], unm = umx * n[0] + umz * n[1];
      const T lam = amax(aabs(unp), aabs(unm));
      const double ca = prm.ca[G] * prm.dt;
      if constexpr (RHO) {  // :519-526
        const T F = ca * (0.5 * (rp * unp + rm * unm) + 0.5 * lam * (rp - rm));
        flux[O_RHO] = -F;
      }
      if constexpr (VEL || PRES) {
        const T pp = vp[3], pm = vm[3];
        const double ct = prm.ct[G] * prm.dt;
        if constexpr (VEL) {  // :1938-1950
          const T pa = ct * prm.invMa2 * 0.5 * (pp + pm);
          const T Fx = ca * 0.5 * (rp * upx * unp + rm * umx * unm) + pa * n[0] + ca * 0.5 * lam * (rp * upx - rm * umx);
          const T Fz = ca * 0.5 * (rp * upz * unp + rm * umz * unm) + pa * n[1] + ca * 0.5 * lam * (rp * upz - rm * umz);
          flux[O_U] = -Fx;
          flux[O_U + 1] = -Fz;
        }
        if constexpr (PRES) {  // :1057-1079 (stage 1), :1141-1194 (2), :1275-1355 (3)
          const T uup = upx * upx + upz * upz, uum = umx * umx + umz * umz;
          const T kin = 0.5 * (0.5 * uup * rp * unp + 0.5 * uum * rm * unm);
          const T ent = 0.5 * prm.gg * (pp * unp + pm * unm);
          T F;
          if constexpr (STAGE < 3) {
            T jk;
            if constexpr (quirk_group(G)) {  // :1182-1183 uses u_tmp_2 . u_old
              jk = rp * 0.5 * (upx * vp[4] + upz * vp[5]) - rm * 0.5 * (umx * vm[4] + umz * vm[5]);
            } else {
              jk = rp * 0.5 * uup - rm * 0.5 * uum;
            }
            const T je = prm.g1 * (pp - pm);
            F = ca * prm.Ma2 * (kin + 0.5 * lam * jk) + ct * (ent + 0.5 * lam * je);
          } else {
            const T jE = prm.g1 * (pp - pm) + 0.5 * prm.Ma2 * (rp * uup - rm * uum);
            F = ca * prm.Ma2 * kin + ca * ent + ca * 0.5 * lam * jE;
          }
          flux[O_P] = -F;
        }
      }
    }
  }

  template <int G, class T>
  __device__ __forceinline__ static void boundary_t(const Params& prm, const T* vp, const double* n, T* flux) {
    if constexpr (G < STAGE && VEL) {  // :2189-2305, p_D = p
      const T pp = vp[3];
      const T s = prm.ct[G] * prm.dt * prm.invMa2 * (0.5 * (pp + pp));
      flux[O_U] = -s * n[0];
      flux[O_U + 1] = -s * n[1];
    }
  }
  template <int G>
  __device__ __forceinline__ static void point(const Params& prm, const double* v, const PointGeo& pg,
                                               double* val, double (*gr)[2]) {
    point_t<G, double>(prm, v, pg, val, gr);
  }
  template <int G>
  __device__ __forceinline__ static void face(const Params& prm, const double* vp, const double* vm,
                                              const double* n, double* flux) {
    face_t<G, double>(prm, vp, vm, n, flux);
  }
  template <int G>
  __device__ __forceinline__ static void boundary(const Params& prm, const double* vp, const double* n,
                                                  double* flux) {
    boundary_t<G, double>(prm, vp, n, flux);
  }
};

// ---------------------------------------------------------------- B: p -> u
// R is the working precision: double for the operator itself, float for the multigrid
// preconditioner's level operators.
template <class R>
struct BParamsT {
  R c;  // coeff * dt / Ma^2, coeff = a~22 (stage 1) or a~33
};
using BParams = BParamsT<double>;

template <class R = double>
struct BPhysT {
  static constexpr int NG = 1;
  static constexpr bool FACES = true, NEED_X = false, ACCUMULATE = false;
  static constexpr int NOUT_ARR = 1, NOUT = 2;
  using Params = BParamsT<R>;
  using real = R;
  static constexpr int out_ncomp(int) { return 2; }
  static constexpr bool has_val(int) { return false; }
  static constexpr bool has_grad(int) { return true; }
  static constexpr int narr_of(int) { return 1; }
  static constexpr int nf_of(int) { return 1; }
  static constexpr int nfc_of(int) { return 1; }
  template <int G>
  struct Grp {
    static constexpr int NARR = 1;
    static constexpr bool FACE = true;
    static constexpr int ncomp(int) { return 1; }
    static constexpr bool face_only(int) { return false; }
  };
  template <int G>
  __device__ __forceinline__ static void point(const Params& prm, const R* v, const PointGeo&, R*, R (*gr)[2]) {
    const R s = -prm.c * v[0];  // submit_divergence (:1536)
    gr[0][0] += s;
    gr[1][1] += s;
  }
  template <int G>
  __device__ __forceinline__ static void face(const Params& prm, const R* vp, const R* vm, const R* n, R* flux) {
    const R a = prm.c * R(0.5) * (vp[0] + vm[0]);  // :1574-1577
    flux[0] = a * n[0];
    flux[1] = a * n[1];
  }
  template <int G>
  __device__ __forceinline__ static void boundary(const Params& prm, const R* vp, const R* n, R* flux) {
    const R a = prm.c * R(0.5) * (vp[0] + vp[0]);  // :1611-1613
    flux[0] = a * n[0];
    flux[1] = a * n[1];
  }
};
using BPhys = BPhysT<double>;

// B of the operator with P+1 Gauss points per direction: the same bilinear form exactly (on a
// bilinear cell p, the adjugate of the Jacobian and the test gradient give degree <= 2P per
// direction, the face terms degree 2P), so it equals the 2P+1-point result up to rounding,
// at a little over half of the work.
struct BPhysExactReduced : BPhysT<double> {
  static constexpr bool REDUCED_Q = true;
};

// B followed by the cell-wise A^{-1} in the kernel's epilogue: w = scale A^{-1} B p, with A^{-1}
// by the change of basis to the Gauss points (inv = 1 / (rho JxW) there; cellop epilogue 1).
template <class R>
struct BInvParams : BParamsT<R> {
  const R* inv;  // [cell][(P+1)^2] Gauss-point inverse weights
  R scale;
};
template <class R = double>
struct BInvPhys : BPhysT<R> {
  using Params = BInvParams<R>;
  static constexpr int EPI = 1;
};

// ------------------------------------------- C (u -> p), optionally D p - C w (Schur)
template <class R>
struct CParamsT {
  R cdt;     // coeff * dt
  R g1, gg;  // 1/(gamma-1), gamma/(gamma-1)
};
using CParams = CParamsT<double>;

// LAM = false drops the reference's wave-speed term 0.5 lambda(w) [p_fixed]/(gamma-1):
// the linear part of C, used by the multigrid preconditioner's level operators.
// ACC = true adds the result to dst instead of overwriting it.
template <bool WITH_D, int SIGN, class R = double, bool LAM = true, bool ACC = false>
struct CPhys {
  static constexpr int NG = WITH_D ? 2 : 1;
  static constexpr int GW = WITH_D ? 1 : 0;  // group of (w, p_fixed)
  static constexpr bool FACES = true, NEED_X = false, ACCUMULATE = ACC;
  static constexpr int NOUT_ARR = 1, NOUT = 1;
  using Params = CParamsT<R>;
  using real = R;
  static constexpr int out_ncomp(int) { return 1; }
  static constexpr bool has_val(int) { return WITH_D; }
  static constexpr bool has_grad(int) { return true; }
  static constexpr int narr_of(int g) { return g == GW ? 2 : 1; }
  static constexpr int nf_of(int g) { return g == GW ? 3 : 1; }
  static constexpr int nfc_of(int g) { return nf_of(g); }
  template <int G>
  struct Grp {
    static constexpr int NARR = G == GW ? 2 : 1;
    static constexpr bool FACE = G == GW;
    static constexpr int ncomp(int a) { return (G == GW && a == 0) ? 2 : 1; }
    static constexpr bool face_only(int) { return false; }
  };
  template <int G>
  __device__ __forceinline__ static void point(const Params& prm, const R* v, const PointGeo&, R* val,
                                               R (*gr)[2]) {
    if constexpr (G == GW) {  // :1444
      const R s = R(-SIGN) * prm.cdt * prm.gg * v[2];
      gr[0][0] += s * v[0];
      gr[0][1] += s * v[1];
    } else {                  // :1403
      val[0] += prm.g1 * v[0];
    }
  }
  template <int G>
  __device__ __forceinline__ static void face(const Params& prm, const R* vp, const R* vm, const R* n, R* flux) {
    if constexpr (G == GW) {  // :1494-1502
      const R wnp = vp[0] * n[0] + vp[1] * n[1], wnm = vm[0] * n[0] + vm[1] * n[1];
      R F;
      if constexpr (LAM) {
        const R lam = fmax(fabs(wnp), fabs(wnm));
        F = prm.cdt * (R(0.5) * prm.gg * (vp[2] * wnp + vm[2] * wnm) + R(0.5) * lam * (prm.g1 * (vp[2] - vm[2])));
      } else {
        F = prm.cdt * (R(0.5) * prm.gg * (vp[2] * wnp + vm[2] * wnm));
      }
      flux[0] = R(SIGN) * F;
    }
  }
  template <int G>
  __device__ __forceinline__ static void boundary(const Params&, const R*, const R*, R*) {}
};

// The multigrid smoother's residual update followed by its Chebyshev step in the kernel's
// epilogue (the linearised Schur operator: r += C0 w - D d, then d' = alpha d + s M^{-1} r,
// x += d').  Inputs as CPhys<true, +1>: d (the D term), w, p_fixed; g1 carries -1/(gamma-1).
template <class R>
struct ResChebParams : CParamsT<R> {
  const R* inv;  // [cell][(P+1)^2] Gauss-point inverse weights of M (1 / JxW)
  R alpha, s;
  R* r;
  const R* din;  // the operator's input d (own cells read again for alpha d)
  R* dout;
  R* x;
  int first;
};
template <class R>
struct ResChebPhys : CPhys<true, 1, R, false, true> {
  using Params = ResChebParams<R>;
  static constexpr int EPI = 2;
};

// The same smoother step carried on the preconditioned residual z = D^{-1} r (epilogue 3).
// The cell inverse of D is exact for the D the level operator applies (both are M-type at the
// same Gauss points; the change of basis inverts M exactly on bilinear cells), so
//   z' = D^{-1} (r + C0 w - D d) = z + D^{-1} C0 w - d,
// and the kernel evaluates C0 w alone: no D group, one field group fewer than ResChebPhys.
// Then d' = alpha d + s z' and x = d' (first) or x += d'.  Inputs as CPhys<false, +1>: w,
// p_fixed; r holds z on input and z' on output; D^{-1} = g M^{-1} with M's weights in inv.
template <class R>
struct ResChebZParams : CParamsT<R> {
  const R* inv;  // [cell][(P+1)^2] Gauss-point inverse weights of M (1 / JxW)
  R g;           // D^{-1} = g M^{-1}
  R alpha, s;
  R* r;          // the preconditioned residual z (read, then overwritten by z')
  const R* din;  // the direction d (read for alpha d and for z' = z + ... - d)
  R* dout;
  R* x;
  int first;
};
template <class R>
struct ResChebZPhys : CPhys<false, 1, R, false, true> {
  using Params = ResChebZParams<R>;
  static constexpr int EPI = 3;
};

// Reduced-quadrature variants of the FP32 preconditioner's level operators: P+1 Gauss points
// per direction instead of 2P+1.  On bilinear cells this integrates B (p div v: degree 2P+1
// per direction with the adjugate of the Jacobian) and M, D exactly; C0 (p_fixed w . grad q,
// degree 3P+1) and the rho-weighted A become approximations, which a preconditioner may use.
template <class R>
struct BInvRPhys : BInvPhys<R> {
  static constexpr bool REDUCED_Q = true;
};
template <class R>
struct ResChebRPhys : ResChebPhys<R> {
  static constexpr bool REDUCED_Q = true;
};
template <class R>
struct CResRPhys : CPhys<true, 1, R, false, true> {
  static constexpr bool REDUCED_Q = true;
};
template <class R>
struct ResChebZRPhys : ResChebZPhys<R> {
  static constexpr bool REDUCED_Q = true;
};

// ---------------------------------------------------------------- mass-type operators
struct MassParams {
  double scale;
};

template <int NC, bool WEIGHTED>
struct MassPhys {
  static constexpr int NG = 1;
  static constexpr bool FACES = false, NEED_X = false, ACCUMULATE = false;
  static constexpr int NOUT_ARR = 1, NOUT = NC;
  using Params = MassParams;
  using real = double;
  static constexpr int out_ncomp(int) { return NC; }
  static constexpr bool has_val(int) { return true; }
  static constexpr bool has_grad(int) { return false; }
  static constexpr int narr_of(int) { return WEIGHTED ? 2 : 1; }
  static constexpr int nf_of(int) { return NC + (WEIGHTED ? 1 : 0); }
  static constexpr int nfc_of(int) { return NC + (WEIGHTED ? 1 : 0); }
  template <int G>
  struct Grp {
    static constexpr int NARR = WEIGHTED ? 2 : 1;
    static constexpr bool FACE = false;
    static constexpr int ncomp(int a) { return a == 0 ? NC : 1; }
    static constexpr bool face_only(int) { return false; }
  };
  template <int G>
  __device__ __forceinline__ static void point(const Params& prm, const double* v, const PointGeo&, double* val,
                                               double (*)[2]) {
#pragma unroll
    for (int d = 0; d < NC; ++d) val[d] += (WEIGHTED ? v[NC] : prm.scale) * v[d];
  }
  template <int G>
  __device__ __forceinline__ static void face(const Params&, const double*, const double*, const double*,
                                              double*) {}
  template <int G>
  __device__ __forceinline__ static void boundary(const Params&, const double*, const double*, double*) {}
};

}  // namespace af
