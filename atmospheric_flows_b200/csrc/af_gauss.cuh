// af_gauss.cuh -- the FP32 Chebyshev smoother of the Schur preconditioner in the Gauss-point
// basis (reduced quadrature: P+1 Gauss points per direction).
//
// The polynomial preconditioner iterates on D^{-1} S0, S0 = D - C0 A^{-1} B (the linearised
// Schur operator).  With P+1 Gauss points per direction, M, D and (approximately) A are
// V^T diag(.) V in the nodal (Gauss-Lobatto) basis, V[q][i] = l_i(g_q) square and invertible.
// In the basis of the Lagrange polynomials L_i of the Gauss points (coefficients = values at
// the Gauss points, u_g = (V x V) u) the three mass-type matrices are diagonal:
//   w_g  = diag(1 / (rho JxW)) B_g d_g         (w = A^{-1} B d)
//   (D^{-1} C0 w)_g = g diag(1 / JxW) C0_g w_g  (D^{-1} = g M^{-1})
// where B_g, C0_g are B and C0 with the L_i as test functions and the Gauss-point values as
// trial coefficients: (B d)_nodal = (V x V)^T B_g (V x V) d.  So the whole Chebyshev
// recurrence runs in the Gauss basis with element-wise inverses; only its input (the
// residual: z0 = g diag(1/JxW) (V x V)^{-T} r) and its output (x = (V x V)^{-1} x_g) change
// basis, once per preconditioner application.  In exact arithmetic this is the same
// preconditioner as the nodal reduced-quadrature smoother; the FP32 rounding differs.
//
// Per cell, the operators need the values of their inputs at the volume points (the
// coefficients themselves: no contraction) and their traces on the faces; test functions
// enter through Dg[q][i] = L_i'(g_q) (volume gradients) and L_i(0), L_i(1) (faces).  A face
// trace is an extrapolation along the normal line: u(0, g_q) = sum_i L_i(0) u_g[q][i].  Each
// kernel writes the face traces of its output, which the next kernel reads for its own and
// its neighbours' faces (the neighbour's trace on the shared face: 4 (P+1) values per cell
// and field, as many as the nodal kernels gather).
//   trace layout: tr[((f * NC + comp) * ncell + cell) * (P+1) + point], faces 0 (xi = 0),
//   1 (xi = 1), 2 (eta = 0), 3 (eta = 1); the point runs along the face (eta for faces 0, 1,
//   xi for faces 2, 3), so a face and the neighbour's opposite face share point indices.
// CTA: GS_CB cells x (P+1) threads; thread (cell, m) owns the column m (x index) of its cell in
// the volume pass and the row m in the passes along x.
#pragma once

#include "af_cellop.cuh"

namespace af {

template <int P>
constexpr int gs_cells() { return P <= 4 ? 32 : 16; }

// per cell: bilinear map A, B, C (6), four faces (normal x, z, length) (12), neighbours (4);
// an odd stride against bank conflicts
constexpr int kGsGeo = 23;

template <int P>
struct GsShape {
  static constexpr int P1 = P + 1, ND = P1 * P1, CB = gs_cells<P>(), NT = CB * P1;
  static constexpr int NDS = ND | 1;  // per-cell stride of nodal arrays in shared memory
  static constexpr int P1S = P1 | 1;  // per-cell stride of face arrays
};

// the cell map, face normals and lengths and the neighbours of cell c, spread over the
// cell's threads: task 4 the map and neighbours, task f < 4 face f (as the cell kernel)
template <int P>
__device__ __forceinline__ void gs_geometry(const MeshDev& mesh, int c, int m, float* g) {
  constexpr int P1 = P + 1;
  const int i = c % mesh.nx, j = c / mesh.nx, W = mesh.nx + 1;
  for (int task = m; task < 5; task += P1) {
    if (task == 4) {
      const double2 v0 = mesh.vtx[j * W + i], v1 = mesh.vtx[j * W + i + 1];
      const double2 v2 = mesh.vtx[(j + 1) * W + i], v3 = mesh.vtx[(j + 1) * W + i + 1];
      g[0] = (float)(v1.x - v0.x);
      g[1] = (float)(v1.y - v0.y);
      g[2] = (float)(v3.x - v2.x - v1.x + v0.x);
      g[3] = (float)(v3.y - v2.y - v1.y + v0.y);
      g[4] = (float)(v2.x - v0.x);
      g[5] = (float)(v2.y - v0.y);
      int nb[4];
      cell_neighbours(mesh, c, nb);
#pragma unroll
      for (int f = 0; f < 4; ++f) put_index(g[18 + f], nb[f]);
    } else {
      const int f = task;
      const int ia = (f == 1) ? i + 1 : i, ja = (f == 3) ? j + 1 : j;
      const int ib = (f == 0) ? i : i + 1, jb = (f == 2) ? j : j + 1;
      const double2 a = mesh.vtx[ja * W + ia], b = mesh.vtx[jb * W + ib];
      const double tx = b.x - a.x, tz = b.y - a.y, len = sqrt(tx * tx + tz * tz);
      const double il = ((f == 0 || f == 3) ? 1.0 : -1.0) / len;
      g[6 + 3 * f] = (float)(-tz * il);
      g[7 + 3 * f] = (float)(tx * il);
      g[8 + 3 * f] = (float)len;
    }
  }
}

// own and neighbour traces of NC components of a field into s_own / s_nb
// [face][comp][cell][point] (point stride P1S), by asynchronous element copies (the caller
// waits for them before its barrier); a boundary face takes the own trace as the
// neighbour's (B's wall flux uses it so; C0 has no wall flux).  Thread t copies point
// t % (P+1) of cell t / (P+1) for every face and component: consecutive threads read
// consecutive elements.  The neighbours come from the CTA's geometry block (complete).
template <int P, int NC>
__device__ __forceinline__ void gs_load_traces(const float* __restrict__ tr, const float* s_geo, int c0, int ncb,
                                               int ncell, float* s_own, float* s_nb) {
  using S = GsShape<P>;
  const int cc = threadIdx.x / S::P1, p = threadIdx.x % S::P1;
  if (cc >= ncb) return;
  const int c = c0 + cc;
  int nb[4];
#pragma unroll
  for (int f = 0; f < 4; ++f) nb[f] = get_index(s_geo[cc * kGsGeo + 18 + f]);
#pragma unroll
  for (int fc = 0; fc < 4 * NC; ++fc) {
    const int f = fc / NC, comp = fc % NC;
    const int o = (fc * S::CB + cc) * S::P1S + p;
    const float* own = tr + ((size_t)(f * NC + comp) * ncell + c) * S::P1 + p;
    const float* oth = nb[f] >= 0 ? tr + ((size_t)((f ^ 1) * NC + comp) * ncell + nb[f]) * S::P1 + p : own;
    cp_async_el(&s_own[o], own);
    cp_async_el(&s_nb[o], oth);
  }
}

// the face traces of NC components of a cell field staged in shared memory (cell stride NDS,
// component stride CB NDS) into s_t [face][comp][cell][point]: thread (cell, m) extrapolates
// along row m (faces 0, 1) and column m (faces 2, 3)
template <int P, int NC>
__device__ __forceinline__ void gs_traces(const float* s_val, int cl, int m, float* s_t) {
  using S = GsShape<P>;
  const CobT<P, float>& cb = cobr<P, float>();
#pragma unroll
  for (int comp = 0; comp < NC; ++comp) {
    const float* cell = s_val + (comp * S::CB + cl) * S::NDS;
    float t0 = 0.f, t1 = 0.f, t2 = 0.f, t3 = 0.f;
#pragma unroll
    for (int i = 0; i < S::P1; ++i) {
      t0 = fmaf(cb.lo[i], cell[m * S::P1 + i], t0);
      t1 = fmaf(cb.hi[i], cell[m * S::P1 + i], t1);
      t2 = fmaf(cb.lo[i], cell[i * S::P1 + m], t2);
      t3 = fmaf(cb.hi[i], cell[i * S::P1 + m], t3);
    }
    s_t[((0 * NC + comp) * S::CB + cl) * S::P1S + m] = t0;
    s_t[((1 * NC + comp) * S::CB + cl) * S::P1S + m] = t1;
    s_t[((2 * NC + comp) * S::CB + cl) * S::P1S + m] = t2;
    s_t[((3 * NC + comp) * S::CB + cl) * S::P1S + m] = t3;
  }
}

// s_t [face][comp][cell][point] to the trace array, consecutive threads on consecutive elements
template <int P, int NC>
__device__ __forceinline__ void gs_store_traces(const float* s_t, int c0, int ncb, int ncell, float* __restrict__ tr) {
  using S = GsShape<P>;
  const int cc = threadIdx.x / S::P1, p = threadIdx.x % S::P1;
  if (cc >= ncb) return;
#pragma unroll
  for (int fc = 0; fc < 4 * NC; ++fc)
    tr[((size_t)fc * ncell + c0) * S::P1 + threadIdx.x] = s_t[(fc * S::CB + cc) * S::P1S + p];
}

// ---------------------------------------------------------------- w = A^{-1} B d
// d_g, its traces dtr -> w_g = scale diag(WA) B_g d_g (two components) and its traces wtr.
// B with coefficient cB (euler_operator.h:1536, 1574-1577, 1611-1613): volume
// -cB d div(phi), face cB {{d}} phi . n, wall cB d+ phi . n.
template <int P>
__global__ void __launch_bounds__(GsShape<P>::NT)
    k_gs_binv(const MeshDev mesh, const float* __restrict__ d, const float* __restrict__ dtr, const float cB,
              const float* __restrict__ WA, const float scale, float* __restrict__ w, float* __restrict__ wtr,
              const int ncell) {
  using S = GsShape<P>;
  constexpr int P1 = S::P1, ND = S::ND, CB = S::CB, NT = S::NT, NDS = S::NDS, P1S = S::P1S;
  __shared__ float s_geo[CB * kGsGeo];
  __shared__ float s_d[CB * NDS];
  __shared__ float s_wa[CB * NDS];
  __shared__ float s_tpm[2 * 4 * CB * P1S];  // own and neighbour traces of d
  __shared__ float s_fx[2 * CB * NDS];
  __shared__ float s_xf[2 * 2 * CB * P1S];  // x-face fluxes [face 0, 1][comp][cell][point]
  __shared__ float s_out[2 * CB * NDS];
  float* const s_tp = s_tpm;
  float* const s_tm = s_tpm + 4 * CB * P1S;
  // the traces of w take the place of d's traces, which the face terms read before the
  // barrier that ends the volume and face phase: 30 KB instead of 35 KB per CTA, 7 CTAs per SM
  float* const s_wt = s_tpm;
  pdl_allow_next();
  const CobT<P, float>& cb = cobr<P, float>();
  const int tid = threadIdx.x, cl = tid % CB, m = tid / CB;
  const int c0 = blockIdx.x * CB, ncb = min(CB, ncell - c0);
  const bool live = cl < ncb;
  const int c = c0 + (live ? cl : ncb - 1);
  float* g = s_geo + cl * kGsGeo;
  gs_geometry<P>(mesh, c, m, g);
  pdl_wait_previous();
  for (int e = tid; e < ncb * ND; e += NT) {
    const int o = (e / ND) * NDS + e % ND;
    cp_async_el(&s_d[o], d + (size_t)c0 * ND + e);
    cp_async_el(&s_wa[o], WA + (size_t)c0 * ND + e);
  }
  __syncthreads();  // the geometry block (neighbours) complete
  gs_load_traces<P, 1>(dtr, s_geo, c0, ncb, ncell, s_tp, s_tm);
  cp_async_wait_all();
  __syncthreads();
  float acc[2][P1];
#pragma unroll
  for (int o = 0; o < 2; ++o)
#pragma unroll
    for (int i = 0; i < P1; ++i) acc[o][i] = 0.f;
  if (live) {
    // volume points of column qx = m: x-fluxes to shared memory, the z-derivative test in registers
    const int qx = m;
    const float xi = cb.g[qx], wx = cb.w[qx];
    const float J01 = fmaf(g[2], xi, g[4]), J11 = fmaf(g[3], xi, g[5]);
#pragma unroll
    for (int qz = 0; qz < P1; ++qz) {
      const float eta = cb.g[qz];
      const float J00 = fmaf(g[2], eta, g[0]), J10 = fmaf(g[3], eta, g[1]);
      const float sw = -cB * s_d[cl * NDS + qz * P1 + qx] * (wx * cb.w[qz]);
      s_fx[(0 * CB + cl) * NDS + qz * P1 + qx] = J11 * sw;
      s_fx[(1 * CB + cl) * NDS + qz * P1 + qx] = -J01 * sw;
      const float fe0 = -J10 * sw, fe1 = J00 * sw;
#pragma unroll
      for (int iz = 0; iz < P1; ++iz) {
        acc[0][iz] = fmaf(cb.Dg[qz][iz], fe0, acc[0][iz]);
        acc[1][iz] = fmaf(cb.Dg[qz][iz], fe1, acc[1][iz]);
      }
    }
    // z-faces at point qx (test L_iz(0) or L_iz(1) on the column), x-faces at point m
#pragma unroll
    for (int f = 0; f < 4; ++f) {
      const int p = m;
      const float tp = s_tp[(f * CB + cl) * P1S + p], tm = s_tm[(f * CB + cl) * P1S + p];
      const float a = cB * 0.5f * (tp + tm) * (g[8 + 3 * f] * cb.w[p]);
      const float F0 = a * g[6 + 3 * f], F1 = a * g[7 + 3 * f];
      if (f >= 2) {
#pragma unroll
        for (int iz = 0; iz < P1; ++iz) {
          const float e = f == 2 ? cb.lo[iz] : cb.hi[iz];
          acc[0][iz] = fmaf(e, F0, acc[0][iz]);
          acc[1][iz] = fmaf(e, F1, acc[1][iz]);
        }
      } else {
        s_xf[((f * 2 + 0) * CB + cl) * P1S + p] = F0;
        s_xf[((f * 2 + 1) * CB + cl) * P1S + p] = F1;
      }
    }
  }
  __syncthreads();
  if (live) {
    // node (ix = m, iz): the x-derivative test along row iz, the x-face terms, A^{-1}
    const int ix = m;
#pragma unroll
    for (int iz = 0; iz < P1; ++iz) {
#pragma unroll
      for (int o = 0; o < 2; ++o) {
        float v = acc[o][iz];
        const float* fx = s_fx + (o * CB + cl) * NDS + iz * P1;
#pragma unroll
        for (int qx = 0; qx < P1; ++qx) v = fmaf(cb.Dg[qx][ix], fx[qx], v);
        v = fmaf(cb.lo[ix], s_xf[((0 * 2 + o) * CB + cl) * P1S + iz], v);
        v = fmaf(cb.hi[ix], s_xf[((1 * 2 + o) * CB + cl) * P1S + iz], v);
        s_out[(o * CB + cl) * NDS + iz * P1 + ix] = scale * s_wa[cl * NDS + iz * P1 + ix] * v;
      }
    }
  }
  __syncthreads();
  for (int e = tid; e < ncb * 2 * ND; e += NT) {  // [cell][comp][node], coalesced
    const int cc = e / (2 * ND), o = (e / ND) % 2, k = e % ND;
    w[(size_t)c0 * 2 * ND + e] = s_out[(o * CB + cc) * NDS + k];
  }
  if (live) gs_traces<P, 2>(s_out, cl, m, s_wt);
  __syncthreads();
  gs_store_traces<P, 2>(s_wt, c0, ncb, ncell, wtr);
}

// ------------------------------------------------- the Chebyshev step on z = D^{-1} r
// w_g (two components) and p_fixed (pg) with their traces -> y = C0_g w_g, then per node
//   z' = z + g WM y - d,  d' = alpha d + s z',  x = d' (first) or x += d',
// d' in place of d (each CTA reads only its own cells of d), and the traces of d'.
// C0 (euler_operator.h:1444, 1494-1502 without the wave-speed term): volume
// -cdt gg p_f w . grad(q), face cdt gg/2 (p_f+ w+ . n + p_f- w- . n) q, no wall term.
template <int P>
__global__ void __launch_bounds__(GsShape<P>::NT)
    k_gs_zstep(const MeshDev mesh, const float* __restrict__ w, const float* __restrict__ wtr,
               const float* __restrict__ pg, const float* __restrict__ ptr, const float cdt, const float gg,
               const float* __restrict__ WM, const float gfac, const float alpha, const float s,
               float* __restrict__ z, float* __restrict__ d, float* __restrict__ x, const int first,
               float* __restrict__ dtr, const int ncell) {
  using S = GsShape<P>;
  constexpr int P1 = S::P1, ND = S::ND, CB = S::CB, NT = S::NT, NDS = S::NDS, P1S = S::P1S;
  __shared__ float s_geo[CB * kGsGeo];
  __shared__ float s_w[2 * CB * NDS];
  __shared__ float s_p[CB * NDS];
  __shared__ float s_twp[4 * 2 * CB * P1S], s_twm[4 * 2 * CB * P1S];
  __shared__ float s_tpp[4 * CB * P1S], s_tpm[4 * CB * P1S];
  __shared__ float s_fx[CB * NDS];
  __shared__ float s_xf[2 * CB * P1S];
  // C0 w and then d' take the place of w, and the traces of d' that of w's own traces; w and
  // its traces are last read before the barrier that ends the volume and face phase (32 KB
  // instead of 38 KB per CTA: 6 CTAs per SM instead of 5)
  float* const s_out = s_w;
  float* const s_dt = s_twp;
  pdl_allow_next();
  const CobT<P, float>& cb = cobr<P, float>();
  const int tid = threadIdx.x, cl = tid % CB, m = tid / CB;
  const int c0 = blockIdx.x * CB, ncb = min(CB, ncell - c0);
  const bool live = cl < ncb;
  const int c = c0 + (live ? cl : ncb - 1);
  float* g = s_geo + cl * kGsGeo;
  gs_geometry<P>(mesh, c, m, g);
  pdl_wait_previous();
  for (int e = tid; e < ncb * ND; e += NT) {
    const int cc = e / ND, k = e % ND;
    cp_async_el(&s_p[cc * NDS + k], pg + (size_t)c0 * ND + e);
  }
  for (int e = tid; e < ncb * 2 * ND; e += NT) {
    const int cc = e / (2 * ND), o = (e / ND) % 2, k = e % ND;
    cp_async_el(&s_w[(o * CB + cc) * NDS + k], w + (size_t)c0 * 2 * ND + e);
  }
  __syncthreads();  // the geometry block (neighbours) complete
  gs_load_traces<P, 2>(wtr, s_geo, c0, ncb, ncell, s_twp, s_twm);
  gs_load_traces<P, 1>(ptr, s_geo, c0, ncb, ncell, s_tpp, s_tpm);
  // the epilogue's operands of this thread's elements (CB ND = (P+1) NT elements per CTA)
  static_assert(CB * ND == P1 * NT, "P+1 epilogue elements per thread");
  float ez[P1], ed[P1], ex[P1], ew[P1];
#pragma unroll
  for (int k = 0; k < P1; ++k) {
    const int e = tid + k * NT;
    const size_t gi = (size_t)c0 * ND + (e < ncb * ND ? e : 0);
    ez[k] = z[gi];
    ed[k] = d[gi];
    ex[k] = first ? 0.f : x[gi];
    ew[k] = WM[gi];
  }
  cp_async_wait_all();
  __syncthreads();
  float acc[P1];
#pragma unroll
  for (int i = 0; i < P1; ++i) acc[i] = 0.f;
  if (live) {
    const int qx = m;
    const float xi = cb.g[qx], wx = cb.w[qx];
    const float J01 = fmaf(g[2], xi, g[4]), J11 = fmaf(g[3], xi, g[5]);
    const float k0 = -cdt * gg;
#pragma unroll
    for (int qz = 0; qz < P1; ++qz) {
      const float eta = cb.g[qz];
      const float J00 = fmaf(g[2], eta, g[0]), J10 = fmaf(g[3], eta, g[1]);
      const int o = cl * NDS + qz * P1 + qx;
      const float sv = k0 * s_p[o] * (wx * cb.w[qz]);
      const float gr0 = sv * s_w[(0 * CB + cl) * NDS + qz * P1 + qx];
      const float gr1 = sv * s_w[(1 * CB + cl) * NDS + qz * P1 + qx];
      s_fx[o] = J11 * gr0 - J01 * gr1;
      const float fe = J00 * gr1 - J10 * gr0;
#pragma unroll
      for (int iz = 0; iz < P1; ++iz) acc[iz] = fmaf(cb.Dg[qz][iz], fe, acc[iz]);
    }
    const float hg = 0.5f * cdt * gg;
#pragma unroll
    for (int f = 0; f < 4; ++f) {
      const int p = m;
      float F = 0.f;
      if (get_index(g[18 + f]) >= 0) {
        const float nx = g[6 + 3 * f], nz = g[7 + 3 * f];
        const float wnp = s_twp[((f * 2 + 0) * CB + cl) * P1S + p] * nx + s_twp[((f * 2 + 1) * CB + cl) * P1S + p] * nz;
        const float wnm = s_twm[((f * 2 + 0) * CB + cl) * P1S + p] * nx + s_twm[((f * 2 + 1) * CB + cl) * P1S + p] * nz;
        const float pp = s_tpp[(f * CB + cl) * P1S + p], pm = s_tpm[(f * CB + cl) * P1S + p];
        F = hg * (pp * wnp + pm * wnm) * (g[8 + 3 * f] * cb.w[p]);
      }
      if (f >= 2) {
#pragma unroll
        for (int iz = 0; iz < P1; ++iz) acc[iz] = fmaf(f == 2 ? cb.lo[iz] : cb.hi[iz], F, acc[iz]);
      } else {
        s_xf[(f * CB + cl) * P1S + p] = F;
      }
    }
  }
  __syncthreads();
  if (live) {
    const int ix = m;
#pragma unroll
    for (int iz = 0; iz < P1; ++iz) {
      float v = acc[iz];
      const float* fx = s_fx + cl * NDS + iz * P1;
#pragma unroll
      for (int qx = 0; qx < P1; ++qx) v = fmaf(cb.Dg[qx][ix], fx[qx], v);
      v = fmaf(cb.lo[ix], s_xf[(0 * CB + cl) * P1S + iz], v);
      v = fmaf(cb.hi[ix], s_xf[(1 * CB + cl) * P1S + iz], v);
      s_out[cl * NDS + iz * P1 + ix] = v;
    }
  }
  __syncthreads();
  // the update in global order (coalesced; element tid + k NT, k < P+1, of the CTA's chunk,
  // its z, d, x and WM read at kernel start); d' back into s_out for its traces
#pragma unroll
  for (int k = 0; k < P1; ++k) {
    const int e = tid + k * NT;
    if (e < ncb * ND) {
      const int cc = e / ND, kk = e % ND;
      const size_t gi = (size_t)c0 * ND + e;
      const float y = s_out[cc * NDS + kk];
      const float zn = ez[k] + gfac * ew[k] * y - ed[k];
      const float nd = alpha * ed[k] + s * zn;
      z[gi] = zn;
      d[gi] = nd;
      x[gi] = first ? nd : ex[k] + nd;
      s_out[cc * NDS + kk] = nd;
    }
  }
  __syncthreads();
  if (live) gs_traces<P, 1>(s_out, cl, m, s_dt);
  __syncthreads();
  gs_store_traces<P, 1>(s_dt, c0, ncb, ncell, dtr);
}

// ------------------------------------------------------------ basis changes
// The preconditioner's input: v (FP64, a residual: dual, nodal) -> b_g = (Vi x Vi)^T v,
// d = x = sc WM b_g, z = theta d and the traces of d.
template <int P>
__global__ void __launch_bounds__(GsShape<P>::NT)
    k_gs_entry(const double* __restrict__ v, const float* __restrict__ WM, const float sc, const float theta,
               float* __restrict__ z, float* __restrict__ d, float* __restrict__ x, float* __restrict__ dtr,
               const int ncell) {
  using S = GsShape<P>;
  constexpr int P1 = S::P1, ND = S::ND, CB = S::CB, NT = S::NT, NDS = S::NDS;
  __shared__ float s_a[CB * NDS];
  __shared__ float s_t[4 * CB * S::P1S];
  pdl_allow_next();
  pdl_wait_previous();
  const CobT<P, float>& cb = cobr<P, float>();
  const int tid = threadIdx.x, cl = tid % CB, m = tid / CB;
  const int c0 = blockIdx.x * CB, ncb = min(CB, ncell - c0);
  const bool live = cl < ncb;
  for (int e = tid; e < ncb * ND; e += NT) s_a[(e / ND) * NDS + e % ND] = (float)v[(size_t)c0 * ND + e];
  __syncthreads();
  float t[P1];
  if (live) {  // along x on row iz = m: t[qx] = sum_ix Vi[ix][qx] v[iz][ix]
    const float* row = s_a + cl * NDS + m * P1;
    float r[P1];
#pragma unroll
    for (int i = 0; i < P1; ++i) r[i] = row[i];
#pragma unroll
    for (int qx = 0; qx < P1; ++qx) {
      float a = 0.f;
#pragma unroll
      for (int ix = 0; ix < P1; ++ix) a = fmaf(cb.Vi[ix][qx], r[ix], a);
      t[qx] = a;
    }
  }
  __syncthreads();
  if (live) {
#pragma unroll
    for (int qx = 0; qx < P1; ++qx) s_a[cl * NDS + m * P1 + qx] = t[qx];
  }
  __syncthreads();
  if (live) {  // along z on column qx = m, then the weights
    const int qx = m;
    float u[P1];
#pragma unroll
    for (int iz = 0; iz < P1; ++iz) u[iz] = s_a[cl * NDS + iz * P1 + qx];
#pragma unroll
    for (int qz = 0; qz < P1; ++qz) {
      float a = 0.f;
#pragma unroll
      for (int iz = 0; iz < P1; ++iz) a = fmaf(cb.Vi[iz][qz], u[iz], a);
      t[qz] = a;
    }
  }
  __syncthreads();
  if (live) {
#pragma unroll
    for (int qz = 0; qz < P1; ++qz) s_a[cl * NDS + qz * P1 + m] = t[qz];
  }
  __syncthreads();
  for (int e = tid; e < ncb * ND; e += NT) {
    const size_t gi = (size_t)c0 * ND + e;
    const float dv = sc * WM[gi] * s_a[(e / ND) * NDS + e % ND];
    d[gi] = dv;
    x[gi] = dv;
    z[gi] = theta * dv;
    s_a[(e / ND) * NDS + e % ND] = dv;
  }
  __syncthreads();
  if (live) gs_traces<P, 1>(s_a, cl, m, s_t);
  __syncthreads();
  gs_store_traces<P, 1>(s_t, c0, ncb, ncell, dtr);
}

// The preconditioner's output: x = (Vi x Vi) x_g (nodal, FP64).
template <int P>
__global__ void __launch_bounds__(GsShape<P>::NT)
    k_gs_exit(const float* __restrict__ xg, double* __restrict__ out, const int ncell) {
  using S = GsShape<P>;
  constexpr int P1 = S::P1, ND = S::ND, CB = S::CB, NT = S::NT, NDS = S::NDS;
  __shared__ float s_a[CB * NDS];
  pdl_allow_next();
  pdl_wait_previous();
  const CobT<P, float>& cb = cobr<P, float>();
  const int tid = threadIdx.x, cl = tid % CB, m = tid / CB;
  const int c0 = blockIdx.x * CB, ncb = min(CB, ncell - c0);
  const bool live = cl < ncb;
  for (int e = tid; e < ncb * ND; e += NT) s_a[(e / ND) * NDS + e % ND] = xg[(size_t)c0 * ND + e];
  __syncthreads();
  float t[P1];
  if (live) {  // along z on column qx = m: t[iz] = sum_qz Vi[iz][qz] x_g[qz][qx]
    float u[P1];
#pragma unroll
    for (int qz = 0; qz < P1; ++qz) u[qz] = s_a[cl * NDS + qz * P1 + m];
#pragma unroll
    for (int iz = 0; iz < P1; ++iz) {
      float a = 0.f;
#pragma unroll
      for (int qz = 0; qz < P1; ++qz) a = fmaf(cb.Vi[iz][qz], u[qz], a);
      t[iz] = a;
    }
  }
  __syncthreads();
  if (live) {
#pragma unroll
    for (int iz = 0; iz < P1; ++iz) s_a[cl * NDS + iz * P1 + m] = t[iz];
  }
  __syncthreads();
  if (live) {  // along x on row iz = m
    float r[P1];
#pragma unroll
    for (int qx = 0; qx < P1; ++qx) r[qx] = s_a[cl * NDS + m * P1 + qx];
#pragma unroll
    for (int ix = 0; ix < P1; ++ix) {
      float a = 0.f;
#pragma unroll
      for (int qx = 0; qx < P1; ++qx) a = fmaf(cb.Vi[ix][qx], r[qx], a);
      t[ix] = a;
    }
  }
  __syncthreads();
  if (live) {
#pragma unroll
    for (int ix = 0; ix < P1; ++ix) s_a[cl * NDS + m * P1 + ix] = t[ix];
  }
  __syncthreads();
  for (int e = tid; e < ncb * ND; e += NT) out[(size_t)c0 * ND + e] = (double)s_a[(e / ND) * NDS + e % ND];
}

// A coefficient field (FP64, nodal) at the Gauss points, pg = (V x V) p, and its traces.
template <int P>
__global__ void __launch_bounds__(GsShape<P>::NT)
    k_gs_values(const double* __restrict__ p, float* __restrict__ pg, float* __restrict__ ptr, const int ncell) {
  using S = GsShape<P>;
  constexpr int P1 = S::P1, ND = S::ND, CB = S::CB, NT = S::NT, NDS = S::NDS;
  __shared__ double s_a[CB * NDS];
  const CobT<P, double>& cb = cobr<P, double>();
  const int tid = threadIdx.x, cl = tid % CB, m = tid / CB;
  const int c0 = blockIdx.x * CB, ncb = min(CB, ncell - c0);
  const bool live = cl < ncb;
  const int c = c0 + (live ? cl : ncb - 1);
  for (int e = tid; e < ncb * ND; e += NT) s_a[(e / ND) * NDS + e % ND] = p[(size_t)c0 * ND + e];
  __syncthreads();
  double t[P1];
  if (live) {  // along x on row iz = m: t[qx] = sum_ix V[qx][ix] p[iz][ix]
    double r[P1];
#pragma unroll
    for (int i = 0; i < P1; ++i) r[i] = s_a[cl * NDS + m * P1 + i];
#pragma unroll
    for (int qx = 0; qx < P1; ++qx) {
      double a = 0.0;
#pragma unroll
      for (int ix = 0; ix < P1; ++ix) a = fma(cb.V[qx][ix], r[ix], a);
      t[qx] = a;
    }
  }
  __syncthreads();
  if (live) {
#pragma unroll
    for (int qx = 0; qx < P1; ++qx) s_a[cl * NDS + m * P1 + qx] = t[qx];
  }
  __syncthreads();
  if (live) {  // along z on column qx = m
    double u[P1];
#pragma unroll
    for (int iz = 0; iz < P1; ++iz) u[iz] = s_a[cl * NDS + iz * P1 + m];
#pragma unroll
    for (int qz = 0; qz < P1; ++qz) {
      double a = 0.0;
#pragma unroll
      for (int iz = 0; iz < P1; ++iz) a = fma(cb.V[qz][iz], u[iz], a);
      t[qz] = a;
    }
  }
  __syncthreads();
  if (live) {
#pragma unroll
    for (int qz = 0; qz < P1; ++qz) s_a[cl * NDS + qz * P1 + m] = t[qz];
  }
  __syncthreads();
  for (int e = tid; e < ncb * ND; e += NT) pg[(size_t)c0 * ND + e] = (float)s_a[(e / ND) * NDS + e % ND];
  if (live) {
    const double* cell = s_a + cl * NDS;
    double t0 = 0.0, t1 = 0.0, t2 = 0.0, t3 = 0.0;
#pragma unroll
    for (int i = 0; i < P1; ++i) {
      t0 = fma(cb.lo[i], cell[m * P1 + i], t0);
      t1 = fma(cb.hi[i], cell[m * P1 + i], t1);
      t2 = fma(cb.lo[i], cell[i * P1 + m], t2);
      t3 = fma(cb.hi[i], cell[i * P1 + m], t3);
    }
    ptr[((size_t)0 * ncell + c) * P1 + m] = (float)t0;
    ptr[((size_t)1 * ncell + c) * P1 + m] = (float)t1;
    ptr[((size_t)2 * ncell + c) * P1 + m] = (float)t2;
    ptr[((size_t)3 * ncell + c) * P1 + m] = (float)t3;
  }
}

}  // namespace af
