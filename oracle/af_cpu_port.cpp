/*
 * af_cpu_port.cpp -- a tuned CPU implementation of the fused stage-1 explicit right-hand
 * side (density, velocity and pressure rhs of HYPERBOLIC_stage 1), used as the timed CPU
 * baseline.
 *
 * TEST AND MEASUREMENT INFRASTRUCTURE ONLY.  Nothing in the product library links, calls or
 * ships it; bench.py (the cpu_baseline leg and the reference arm) and tests/ load it from the
 * oracle's library.  Its results are checked against the oracle (tests/test_cpu_port.py,
 * 1e-12 relative L2).
 *
 * Why a second CPU code: the oracle (af_oracle.cpp) is a literal restatement written to be
 * read against the reference; it evaluates face traces by dense tensor sums, recomputes the
 * geometry per face point and allocates per cell.  A baseline has to be timed on code written
 * the way a tuned matrix-free CPU operator is (deal.II's MatrixFree::loop, which the reference
 * runs: euler_operator.h:697-712, 1366-1381, 2310-2325):
 *   - cell integrals by sum factorisation, vectorised over batches of kW consecutive cells
 *     (the role of deal.II's VectorizedArray), geometry of the bilinear map per point;
 *   - each interior face evaluated once, from the face's Gauss-Lobatto nodes (a 1D
 *     interpolation per field and side), the flux added to both cells;
 *   - OpenMP over batches of cells, over rows of x-faces and over columns of z-faces (no two
 *     threads write the same cell within a phase), no allocation inside the loops.
 * Physics per point and per face is the reference's stage-1 integrand (euler_operator.h:
 * 344-473, 478-692 density; 745-1007, 1012-1361 pressure; 1622-2305 velocity) in the same
 * algebraic form as the oracle; gravity is e_z with constant magnitude (the 2D hill).
 */
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

extern "C" void orc_tables(int P, int NQ, double* nodes, double* qp, double* qw, double* S, double* D);

namespace {

constexpr int kW = 4;  // cells per SIMD batch

template <int P>
struct Tables {
  static constexpr int P1 = P + 1, NQ = 2 * P + 1;
  double node[P1], x[NQ], w[NQ], S[NQ][P1], D[NQ][P1];
  Tables() { orc_tables(P, NQ, node, x, w, &S[0][0], &D[0][0]); }
};

struct Coef {  // stage-1 weights times dt and the non-dimensional constants
  double ca, ct, cg, cgI, invMa2, invFr2, Ma2, Ma2Fr2, g1, gg;
};

template <int P>
struct Port {
  static constexpr int P1 = P + 1, NQ = 2 * P + 1, ND = P1 * P1, NQ2 = NQ * NQ;
  const Tables<P>& T;
  int nx, nz, periodic;
  const double* vtx;
  Coef k;

  // ---- cell integrals of one batch of kW cells [c0, c0 + kW) (cells past the end clamp to
  //      the last one and are not stored)
  void cells(int c0, int ncell, const double* const* in, double* out_r, double* out_u, double* out_p) const {
    alignas(64) double u[7][ND][kW];        // nodal values: rho, ux, uz, p, rc, fx, fz
    alignas(64) double t[NQ * P1][kW];      // x-pass scratch
    alignas(64) double v[7][NQ2][kW];       // values at the quadrature points
    alignas(64) double fv[4][NQ2][kW], fx[4][NQ2][kW], fe[4][NQ2][kW];
    int cell[kW];
    for (int l = 0; l < kW; ++l) cell[l] = std::min(c0 + l, ncell - 1);
    // gather: per field its cell-local nodes (vectors component-blocked)
    const double* fld[7] = {in[0], in[1], in[1], in[2], in[3], in[4], in[4]};
    const int comp[7] = {0, 0, 1, 0, 0, 0, 1}, ncomp[7] = {1, 2, 2, 1, 1, 2, 2};
    for (int f = 0; f < 7; ++f)
      for (int l = 0; l < kW; ++l) {
        const double* s = fld[f] + ((long)cell[l] * ncomp[f] + comp[f]) * ND;
        for (int i = 0; i < ND; ++i) u[f][i][l] = s[i];
      }
    for (int f = 0; f < 7; ++f) {
      for (int iz = 0; iz < P1; ++iz)
        for (int qx = 0; qx < NQ; ++qx) {
          double a[kW] = {};
          for (int ix = 0; ix < P1; ++ix) {
            const double s = T.S[qx][ix];
#pragma omp simd
            for (int l = 0; l < kW; ++l) a[l] += s * u[f][iz * P1 + ix][l];
          }
#pragma omp simd
          for (int l = 0; l < kW; ++l) t[iz * NQ + qx][l] = a[l];
        }
      for (int qz = 0; qz < NQ; ++qz)
        for (int qx = 0; qx < NQ; ++qx) {
          double a[kW] = {};
          for (int iz = 0; iz < P1; ++iz) {
            const double s = T.S[qz][iz];
#pragma omp simd
            for (int l = 0; l < kW; ++l) a[l] += s * t[iz * NQ + qx][l];
          }
#pragma omp simd
          for (int l = 0; l < kW; ++l) v[f][qz * NQ + qx][l] = a[l];
        }
    }
    // bilinear map per cell: x = v0 + A xi + C eta + B xi eta
    double A[2][kW], B[2][kW], C[2][kW];
    for (int l = 0; l < kW; ++l) {
      const int i = cell[l] % nx, j = cell[l] / nx, Wv = nx + 1;
      const double* a = vtx + 2 * (j * Wv + i);
      const double* b = vtx + 2 * (j * Wv + i + 1);
      const double* c = vtx + 2 * ((j + 1) * Wv + i);
      const double* d = vtx + 2 * ((j + 1) * Wv + i + 1);
      for (int e = 0; e < 2; ++e) {
        A[e][l] = b[e] - a[e];
        C[e][l] = c[e] - a[e];
        B[e][l] = d[e] - c[e] - b[e] + a[e];
      }
    }
    for (int qz = 0; qz < NQ; ++qz)
      for (int qx = 0; qx < NQ; ++qx) {
        const int q = qz * NQ + qx;
        const double xi = T.x[qx], eta = T.x[qz], wq = T.w[qx] * T.w[qz];
#pragma omp simd
        for (int l = 0; l < kW; ++l) {
          const double J00 = A[0][l] + B[0][l] * eta, J01 = C[0][l] + B[0][l] * xi;
          const double J10 = A[1][l] + B[1][l] * eta, J11 = C[1][l] + B[1][l] * xi;
          const double det = J00 * J11 - J01 * J10;
          const double jxw = det * wq;
          // J^{-1} times JxW: [[J11, -J01], [-J10, J00]] * w
          const double i00 = J11 * wq, i01 = -J01 * wq, i10 = -J10 * wq, i11 = J00 * wq;
          const double r = v[0][q][l], ux = v[1][q][l], uz = v[2][q][l], p = v[3][q][l];
          const double rc = v[4][q][l], fxx = v[5][q][l], fzz = v[6][q][l];
          const double uu = ux * ux + uz * uz, ff = fxx * fxx + fzz * fzz;
          // density: rho0 phi + dt a21 rho0 u0 . grad phi
          double g0 = k.ca * r * ux, g1 = k.ca * r * uz;
          fv[0][q][l] = r * jxw;
          fx[0][q][l] = i00 * g0 + i01 * g1;
          fe[0][q][l] = i10 * g0 + i11 * g1;
          // velocity: rho0 u0 - dt/Fr^2 (a~21 rho0 + a~22 rho2) e_z; rho0 u0 u0 a + a~/Ma^2 p0 I
          const double grav = k.invFr2 * (k.cg * r + k.cgI * rc);
          const double cr = k.ca * r, pt = k.ct * k.invMa2 * p;
          fv[1][q][l] = r * ux * jxw;
          fv[2][q][l] = (r * uz - grav) * jxw;
          g0 = cr * ux * ux + pt;
          g1 = cr * ux * uz;
          fx[1][q][l] = i00 * g0 + i01 * g1;
          fe[1][q][l] = i10 * g0 + i11 * g1;
          g0 = cr * uz * ux;
          g1 = cr * uz * uz + pt;
          fx[2][q][l] = i00 * g0 + i01 * g1;
          fe[2][q][l] = i10 * g0 + i11 * g1;
          // pressure form of the energy: rho0 E0 - rho2 Ma^2 |u_fix|^2 / 2 - gravity work;
          // (Ma^2 |u0|^2 rho0 / 2 a + a~ (rho0 e0 + p0)) u0 with rho e = p/(gamma-1)
          const double val = p * k.g1 + 0.5 * k.Ma2 * r * uu - 0.5 * rc * k.Ma2 * ff -
                             k.Ma2Fr2 * (k.cg * r * uz + k.cgI * rc * fzz);
          const double s = 0.5 * k.ca * k.Ma2 * uu * r + k.ct * k.gg * p;
          fv[3][q][l] = val * jxw;
          fx[3][q][l] = i00 * (s * ux) + i01 * (s * uz);
          fe[3][q][l] = i10 * (s * ux) + i11 * (s * uz);
        }
      }
    // integrate: out[iz][ix] = sum_q S(qz,iz) [S(qx,ix) fv + D(qx,ix) fx] + D(qz,iz) S(qx,ix) fe
    double* dsts[4] = {out_r, out_u, out_u, out_p};
    const int oc[4] = {0, 0, 1, 0}, onc[4] = {1, 2, 2, 1};
    for (int o = 0; o < 4; ++o) {
      alignas(64) double a[NQ * P1][kW], b[NQ * P1][kW];
      for (int qz = 0; qz < NQ; ++qz)
        for (int ix = 0; ix < P1; ++ix) {
          double sa[kW] = {}, sb[kW] = {};
          for (int qx = 0; qx < NQ; ++qx) {
            const int q = qz * NQ + qx;
            const double s = T.S[qx][ix], d = T.D[qx][ix];
#pragma omp simd
            for (int l = 0; l < kW; ++l) {
              sa[l] += s * fv[o][q][l] + d * fx[o][q][l];
              sb[l] += s * fe[o][q][l];
            }
          }
#pragma omp simd
          for (int l = 0; l < kW; ++l) {
            a[qz * P1 + ix][l] = sa[l];
            b[qz * P1 + ix][l] = sb[l];
          }
        }
      for (int iz = 0; iz < P1; ++iz)
        for (int ix = 0; ix < P1; ++ix) {
          double r[kW] = {};
          for (int qz = 0; qz < NQ; ++qz) {
            const double s = T.S[qz][iz], d = T.D[qz][iz];
#pragma omp simd
            for (int l = 0; l < kW; ++l) r[l] += s * a[qz * P1 + ix][l] + d * b[qz * P1 + ix][l];
          }
          for (int l = 0; l < kW && c0 + l < ncell; ++l)
            dsts[o][((long)(c0 + l) * onc[o] + oc[o]) * ND + iz * P1 + ix] = r[l];
        }
    }
  }

  // nodes of face f of a cell, along the face parameter: 0 xi=0, 1 xi=1, 2 eta=0, 3 eta=1
  static int fnode(int f, int i) { return f == 0 ? i * P1 : (f == 1 ? i * P1 + P : (f == 2 ? i : P * P1 + i)); }

  // traces of the explicit fields (rho, ux, uz, p) of a cell on face f at the NQ face points
  void trace(const double* const* in, int c, int f, double (*tr)[NQ]) const {
    const double* src[4] = {in[0] + (long)c * ND, in[1] + (long)c * 2 * ND, in[1] + (long)c * 2 * ND + ND,
                            in[2] + (long)c * ND};
    for (int m = 0; m < 4; ++m) {
      double nv[P1];
      for (int i = 0; i < P1; ++i) nv[i] = src[m][fnode(f, i)];
      for (int q = 0; q < NQ; ++q) {
        double s = 0.0;
        for (int i = 0; i < P1; ++i) s += T.S[q][i] * nv[i];
        tr[m][q] = s;
      }
    }
  }

  // adds the face integral of a flux (NQ values per output, already times JxW) to cell c
  void face_add(int c, int f, const double (*F)[NQ], double* out_r, double* out_u, double* out_p, int first_o) const {
    double* dst[4] = {out_r + (long)c * ND, out_u + (long)c * 2 * ND, out_u + (long)c * 2 * ND + ND,
                      out_p + (long)c * ND};
    for (int o = first_o; o < 4; ++o) {
      if (first_o == 1 && o == 3) break;  // boundary faces: velocity only
      for (int i = 0; i < P1; ++i) {
        double s = 0.0;
        for (int q = 0; q < NQ; ++q) s += T.S[q][i] * F[o][q];
        dst[o][fnode(f, i)] += s;
      }
    }
  }

  // outward unit normal and length of face f of cell (i, j), from the face's two vertices
  void normal(int i, int j, int f, double n[2], double& len) const {
    const int Wv = nx + 1;
    const int ia = f == 1 ? i + 1 : i, ja = f == 3 ? j + 1 : j;
    const int ib = f == 0 ? i : i + 1, jb = f == 2 ? j : j + 1;
    const double tx = vtx[2 * (jb * Wv + ib)] - vtx[2 * (ja * Wv + ia)];
    const double tz = vtx[2 * (jb * Wv + ib) + 1] - vtx[2 * (ja * Wv + ia) + 1];
    len = std::sqrt(tx * tx + tz * tz);
    const double sg = (f == 0 || f == 3) ? 1.0 : -1.0;
    n[0] = sg * (-tz / len);
    n[1] = sg * (tx / len);
  }

  // interior face: + side cell cp (face fp, normal n), - side cell cm (face fm)
  void interior(const double* const* in, int ip, int jp, int fp, int cm, int fm, double* out_r, double* out_u,
                double* out_p) const {
    const int cp = jp * nx + ip;
    double tp[4][NQ], tm[4][NQ], F[4][NQ], G[4][NQ];
    trace(in, cp, fp, tp);
    trace(in, cm, fm, tm);
    double n[2], len;
    normal(ip, jp, fp, n, len);
    for (int q = 0; q < NQ; ++q) {
      const double rp = tp[0][q], upx = tp[1][q], upz = tp[2][q], pp = tp[3][q];
      const double rm = tm[0][q], umx = tm[1][q], umz = tm[2][q], pm = tm[3][q];
      const double unp = upx * n[0] + upz * n[1], unm = umx * n[0] + umz * n[1];
      const double lam = std::max(std::fabs(unp), std::fabs(unm));
      const double jxw = len * T.w[q];
      const double Fr = k.ca * (0.5 * (rp * unp + rm * unm) + 0.5 * lam * (rp - rm));
      const double pa = k.ct * k.invMa2 * 0.5 * (pp + pm);
      const double Fx = k.ca * 0.5 * (rp * upx * unp + rm * umx * unm) + pa * n[0] + k.ca * 0.5 * lam * (rp * upx - rm * umx);
      const double Fz = k.ca * 0.5 * (rp * upz * unp + rm * umz * unm) + pa * n[1] + k.ca * 0.5 * lam * (rp * upz - rm * umz);
      const double uup = upx * upx + upz * upz, uum = umx * umx + umz * umz;
      const double kin = 0.5 * (0.5 * uup * rp * unp + 0.5 * uum * rm * unm);
      const double ent = 0.5 * k.gg * (pp * unp + pm * unm);
      const double jk = rp * 0.5 * uup - rm * 0.5 * uum, je = k.g1 * (pp - pm);
      const double Fp = k.ca * k.Ma2 * (kin + 0.5 * lam * jk) + k.ct * (ent + 0.5 * lam * je);
      const double f4[4] = {Fr, Fx, Fz, Fp};
      for (int o = 0; o < 4; ++o) {
        F[o][q] = -f4[o] * jxw;
        G[o][q] = f4[o] * jxw;
      }
    }
    face_add(cp, fp, F, out_r, out_u, out_p, 0);
    face_add(cm, fm, G, out_r, out_u, out_p, 0);
  }

  // wall: the reference's reflective pressure term of the velocity rhs (p_D = p)
  void wall(const double* const* in, int i, int j, int f, double* out_r, double* out_u, double* out_p) const {
    const int c = j * nx + i;
    double t[4][NQ], F[4][NQ];
    trace(in, c, f, t);
    double n[2], len;
    normal(i, j, f, n, len);
    for (int q = 0; q < NQ; ++q) {
      const double s = k.ct * k.invMa2 * (0.5 * (t[3][q] + t[3][q])) * len * T.w[q];
      F[1][q] = -s * n[0];
      F[2][q] = -s * n[1];
    }
    face_add(c, f, F, out_r, out_u, out_p, 1);
  }

  void run(const double* const* in, double* out_r, double* out_u, double* out_p) const {
    const int ncell = nx * nz;
#pragma omp parallel
    {
#pragma omp for schedule(static)
      for (int b = 0; b < (ncell + kW - 1) / kW; ++b) cells(b * kW, ncell, in, out_r, out_u, out_p);
      // x-faces, one row per thread at a time: face between (i-1, j) and (i, j), the periodic
      // face or the lateral walls
#pragma omp for schedule(static)
      for (int j = 0; j < nz; ++j) {
        for (int i = 1; i < nx; ++i) interior(in, i - 1, j, 1, j * nx + i, 0, out_r, out_u, out_p);
        if (periodic) {
          interior(in, nx - 1, j, 1, j * nx, 0, out_r, out_u, out_p);
        } else {
          wall(in, 0, j, 0, out_r, out_u, out_p);
          wall(in, nx - 1, j, 1, out_r, out_u, out_p);
        }
      }
      // z-faces, one column per thread at a time, and the bottom and top walls
#pragma omp for schedule(static)
      for (int i = 0; i < nx; ++i) {
        wall(in, i, 0, 2, out_r, out_u, out_p);
        for (int j = 1; j < nz; ++j) interior(in, i, j - 1, 3, j * nx + i, 2, out_r, out_u, out_p);
        wall(in, i, nz - 1, 3, out_r, out_u, out_p);
      }
    }
  }
};

template <int P>
void run_degree(int nx, int nz, int periodic, const double* vtx, const Coef& k, const double* const* in,
                double* out_r, double* out_u, double* out_p) {
  static const Tables<P> tab;
  Port<P> port{tab, nx, nz, periodic, vtx, k};
  port.run(in, out_r, out_u, out_p);
}

}  // namespace

extern "C" {

/* The fused stage-1 rhs triple on the host: in = {rho0, u0, p0, rho_tmp_2, u_fixed} in the
 * library's DoF layout; gravity e_z (mode 0).  Returns 0, or -1 for an unsupported degree. */
int cpu_rhs_fused_stage1(int degree, int nx, int nz, int periodic_x, const double* vtx, double Ma, double Fr,
                         double dt, const double* const* in, double* out_rho, double* out_u, double* out_p) {
  const double gamma = 2.0 - std::sqrt(2.0);  // euler_operator.h:233-240
  Coef k;
  k.ca = gamma * dt;              // a21
  k.ct = 0.5 * gamma * dt;        // a~21
  k.cg = 0.5 * gamma * dt;        // a~21 (explicit gravity)
  k.cgI = 0.5 * gamma * dt;       // a~22 (implicit gravity)
  k.Ma2 = Ma * Ma;
  k.invMa2 = 1.0 / k.Ma2;
  k.invFr2 = 1.0 / (Fr * Fr);
  k.Ma2Fr2 = k.Ma2 / (Fr * Fr);
  k.g1 = 1.0 / (1.4 - 1.0);
  k.gg = 1.4 / (1.4 - 1.0);
  switch (degree) {
    case 2: run_degree<2>(nx, nz, periodic_x, vtx, k, in, out_rho, out_u, out_p); return 0;
    case 3: run_degree<3>(nx, nz, periodic_x, vtx, k, in, out_rho, out_u, out_p); return 0;
    case 4: run_degree<4>(nx, nz, periodic_x, vtx, k, in, out_rho, out_u, out_p); return 0;
    case 5: run_degree<5>(nx, nz, periodic_x, vtx, k, in, out_rho, out_u, out_p); return 0;
    case 6: run_degree<6>(nx, nz, periodic_x, vtx, k, in, out_rho, out_u, out_p); return 0;
    default: return -1;
  }
}

}  // extern "C"
