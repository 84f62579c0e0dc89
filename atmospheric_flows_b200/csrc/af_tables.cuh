// af_tables.cuh -- 1D basis tables for FE_DGQ(P) on Gauss-Lobatto points with QGauss(2P+1)
// (and QGauss(P+1) for the reduced-quadrature preconditioner operators).
//
// The reference evaluates its fields with deal.II FEEvaluation<dim, p, 2p+1> (template
// arguments at Atmospheric_Flow.cc:151-153, quadrature at :345).  Here the 1D values S and
// derivatives D of the Lagrange basis at the Gauss points are precomputed on the host in
// long double and kept in __constant__ memory, together with their even/odd splits:
//   Se[q][i] = (S[q][i] + S[q][P-i])/2,  So[q][i] = (S[q][i] - S[q][P-i])/2   (i < H)
//   De, Do likewise for D, and Sm[q] = S[q][P/2], Dm[q] = D[q][P/2] (P even).
// Symmetric nodes and points give S[NQ-1-q][i] = S[q][P-i] and D[NQ-1-q][i] = -D[q][P-i],
// so every 1D contraction costs about half of the direct one.
#pragma once

#include <cmath>
#include <utility>
#include <vector>

namespace af {

// NQ_ Gauss points per direction: 2P+1 for the operators (the reference's quadrature), P+1
// for the reduced-quadrature preconditioner operators.  Quadrature points pair as
// (q, NQ-1-q) for q < QH, with a middle point q = QH when NQ is odd.
template <int P, class R = double, int NQ_ = 2 * P + 1>
struct TabT {
  static constexpr int P1 = P + 1;
  static constexpr int NQ = NQ_;
  static constexpr int H = P1 / 2;        // node pairs (i, P-i), i < H
  static constexpr bool MIDN = (P % 2) == 0;  // a middle node exists
  static constexpr int QH = NQ / 2;       // quadrature point pairs
  static constexpr bool QMID = (NQ % 2) == 1;  // a middle quadrature point exists
  static constexpr int QE = QH + (QMID ? 1 : 0);  // rows of the even/odd tables
  R S[NQ][P1], D[NQ][P1];
  R Se[QE][H > 0 ? H : 1], So[QE][H > 0 ? H : 1];
  R De[QE][H > 0 ? H : 1], Do[QE][H > 0 ? H : 1];
  R Sm[QE], Dm[QE];
  R w[NQ], x[NQ];
};
template <int P>
using Tab = TabT<P, double>;


// Level-transfer tables of the h-multigrid (same degree on every level; a coarse cell's
// reference square is split into 2 x 2 children, child o in {0,1} per direction covering
// [o/2, (o+1)/2]):
//   Pm[o][i][j] = l_j((o + x_i)/2)   value of coarse basis j at child-o node i (prolongation;
//                                    its transpose restricts residuals)
//   E[i][j]     = l_j(2 x_i - ch[i]) value of the child-ch[i] basis j at coarse node i
//                                    (injection of coefficient fields; ch[i] = 0 for x_i <= 1/2)
template <int P, class R = double>
struct TransT {
  R Pm[2][P + 1][P + 1];
  R E[P + 1][P + 1];
  int ch[P + 1];
};

// Change of basis between the nodal basis and the (P+1) x (P+1) Gauss points.  With
// V[q][i] = l_i(g_q) (square and invertible), the mass matrix of a bilinear cell is exactly
// (V x V)^T diag(JxW) (V x V) over the P+1 Gauss points -- its integrand l_i l_j det J has
// degree <= 2P+1 per direction, which (P+1)-point Gauss integrates exactly -- so
//   M_K^{-1} = (V x V)^{-1} diag(1 / JxW) (V x V)^{-T},
// applied by sum factorisation with Vi = V^{-1} and no stored matrices.  A density weight
// rho (degree P) makes the integrand degree 3P+1: the same formula with rho(g_q) JxW is then
// the inverse of the (P+1)-point approximation of the weighted mass matrix.
template <int P, class R = double>
struct CobT {
  R Vi[P + 1][P + 1];  // Vi[i][q] = (V^{-1})[i][q]
  R V[P + 1][P + 1];   // V[q][i] = l_i(g_q)
  R g[P + 1], w[P + 1];  // Gauss points and weights on [0, 1]
  // the Lagrange basis L_i of the Gauss points (the collocated basis of the Gauss-point
  // smoother): Dg[q][i] = L_i'(g_q), lo[i] = L_i(0), hi[i] = L_i(1)
  R Dg[P + 1][P + 1];
  R lo[P + 1], hi[P + 1];
};

namespace host {

using LD = long double;

inline void legendre(int n, LD x, LD& Pn, LD& dPn) {
  LD p0 = 1, p1 = x;
  if (n == 0) { Pn = 1; dPn = 0; return; }
  for (int k = 2; k <= n; ++k) {
    LD p2 = ((2 * k - 1) * x * p1 - (k - 1) * p0) / k;
    p0 = p1;
    p1 = p2;
  }
  Pn = p1;
  dPn = n * (x * p1 - p0) / (x * x - 1);
}

// Gauss-Lobatto nodes on [0,1]: endpoints and the roots of P'_p.
inline std::vector<LD> gll(int p) {
  std::vector<LD> x(p + 1);
  const LD pi = 3.14159265358979323846264338327950288L;
  x[0] = 0;
  x[p] = 1;
  for (int k = 1; k < p; ++k) {
    LD t = -cosl(pi * k / p);
    for (int it = 0; it < 60; ++it) {
      LD Pn, dPn;
      legendre(p, t, Pn, dPn);
      LD d2 = (2 * t * dPn - p * (p + 1) * Pn) / (1 - t * t);
      LD dt = dPn / d2;
      t -= dt;
      if (fabsl(dt) < 1e-30L) break;
    }
    x[k] = (t + 1) / 2;
  }
  return x;
}

// Gauss-Legendre points and weights on [0,1], ascending.
inline void gauss(int n, std::vector<LD>& x, std::vector<LD>& w) {
  x.assign(n, 0);
  w.assign(n, 0);
  const LD pi = 3.14159265358979323846264338327950288L;
  for (int k = 0; k < n; ++k) {
    LD t = -cosl(pi * (k + 0.75L) / (n + 0.5L));
    LD Pn = 0, dPn = 1;
    for (int it = 0; it < 60; ++it) {
      legendre(n, t, Pn, dPn);
      LD dt = Pn / dPn;
      t -= dt;
      if (fabsl(dt) < 1e-30L) break;
    }
    legendre(n, t, Pn, dPn);
    x[k] = (t + 1) / 2;
    w[k] = 1 / ((1 - t * t) * dPn * dPn);
  }
}

inline LD lag(const std::vector<LD>& nd, int i, LD s) {
  LD v = 1;
  for (int j = 0; j < (int)nd.size(); ++j)
    if (j != i) v *= (s - nd[j]) / (nd[i] - nd[j]);
  return v;
}

inline LD dlag(const std::vector<LD>& nd, int i, LD s) {
  LD acc = 0;
  for (int k = 0; k < (int)nd.size(); ++k) {
    if (k == i) continue;
    LD t = 1 / (nd[i] - nd[k]);
    for (int j = 0; j < (int)nd.size(); ++j)
      if (j != i && j != k) t *= (s - nd[j]) / (nd[i] - nd[j]);
    acc += t;
  }
  return acc;
}

template <int P, class R = double, int NQ = 2 * P + 1>
inline TabT<P, R, NQ> make_tab() {
  using T = TabT<P, R, NQ>;
  T t{};
  std::vector<LD> nd = gll(P), x, w;
  gauss(T::NQ, x, w);
  LD S[T::NQ][T::P1], D[T::NQ][T::P1];
  for (int q = 0; q < T::NQ; ++q)
    for (int i = 0; i < T::P1; ++i) {
      S[q][i] = lag(nd, i, x[q]);
      D[q][i] = dlag(nd, i, x[q]);
      t.S[q][i] = (R)S[q][i];
      t.D[q][i] = (R)D[q][i];
    }
  for (int q = 0; q < T::QE; ++q) {
    for (int i = 0; i < T::H; ++i) {
      t.Se[q][i] = (R)((S[q][i] + S[q][P - i]) / 2);
      t.So[q][i] = (R)((S[q][i] - S[q][P - i]) / 2);
      t.De[q][i] = (R)((D[q][i] + D[q][P - i]) / 2);
      t.Do[q][i] = (R)((D[q][i] - D[q][P - i]) / 2);
    }
    t.Sm[q] = T::MIDN ? (R)S[q][P / 2] : R(0);
    t.Dm[q] = T::MIDN ? (R)D[q][P / 2] : R(0);
  }
  for (int q = 0; q < T::NQ; ++q) {
    t.w[q] = (R)w[q];
    t.x[q] = (R)x[q];
  }
  return t;
}

template <int P, class R = double>
inline CobT<P, R> make_cob() {
  constexpr int P1 = P + 1;
  CobT<P, R> t{};
  std::vector<LD> nd = gll(P), x, w;
  gauss(P1, x, w);
  LD V[P1][P1], Vi[P1][2 * P1];
  for (int q = 0; q < P1; ++q)
    for (int i = 0; i < P1; ++i) V[q][i] = lag(nd, i, x[q]);
  // Gauss-Jordan with partial pivoting on [V | I]
  for (int r = 0; r < P1; ++r)
    for (int c = 0; c < 2 * P1; ++c) Vi[r][c] = c < P1 ? V[r][c] : (c - P1 == r ? 1 : 0);
  for (int c = 0; c < P1; ++c) {
    int piv = c;
    for (int r = c + 1; r < P1; ++r)
      if (fabsl(Vi[r][c]) > fabsl(Vi[piv][c])) piv = r;
    for (int k = 0; k < 2 * P1; ++k) std::swap(Vi[c][k], Vi[piv][k]);
    const LD d = Vi[c][c];
    for (int k = 0; k < 2 * P1; ++k) Vi[c][k] /= d;
    for (int r = 0; r < P1; ++r)
      if (r != c) {
        const LD f = Vi[r][c];
        for (int k = 0; k < 2 * P1; ++k) Vi[r][k] -= f * Vi[c][k];
      }
  }
  for (int i = 0; i < P1; ++i)
    for (int q = 0; q < P1; ++q) {
      t.Vi[i][q] = (R)Vi[i][P1 + q];
      t.V[q][i] = (R)V[q][i];
    }
  for (int q = 0; q < P1; ++q) {
    t.g[q] = (R)x[q];
    t.w[q] = (R)w[q];
  }
  for (int i = 0; i < P1; ++i) {
    for (int q = 0; q < P1; ++q) t.Dg[q][i] = (R)dlag(x, i, x[q]);
    t.lo[i] = (R)lag(x, i, 0);
    t.hi[i] = (R)lag(x, i, 1);
  }
  return t;
}

template <int P, class R = double>
inline TransT<P, R> make_trans() {
  TransT<P, R> t{};
  std::vector<LD> nd = gll(P);
  for (int o = 0; o < 2; ++o)
    for (int i = 0; i <= P; ++i)
      for (int j = 0; j <= P; ++j) t.Pm[o][i][j] = (R)lag(nd, j, (o + nd[i]) / 2);
  for (int i = 0; i <= P; ++i) {
    const int c = nd[i] <= 0.5L ? 0 : 1;
    t.ch[i] = c;
    for (int j = 0; j <= P; ++j) t.E[i][j] = (R)lag(nd, j, 2 * nd[i] - c);
  }
  return t;
}

}  // namespace host
}  // namespace af
