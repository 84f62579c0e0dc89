// af_tables.cuh -- 1D basis tables for FE_DGQ(P) on Gauss-Lobatto points with QGauss(2P+1).
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
#include <vector>

namespace af {

template <int P, class R = double>
struct TabT {
  static constexpr int P1 = P + 1;
  static constexpr int NQ = 2 * P + 1;
  static constexpr int H = P1 / 2;        // node pairs (i, P-i), i < H
  static constexpr bool MIDN = (P % 2) == 0;  // a middle node exists
  R S[NQ][P1], D[NQ][P1];
  R Se[P + 1][H > 0 ? H : 1], So[P + 1][H > 0 ? H : 1];
  R De[P + 1][H > 0 ? H : 1], Do[P + 1][H > 0 ? H : 1];
  R Sm[P + 1], Dm[P + 1];
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

template <int P, class R = double>
inline TabT<P, R> make_tab() {
  using T = TabT<P, R>;
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
  for (int q = 0; q <= P; ++q) {
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
