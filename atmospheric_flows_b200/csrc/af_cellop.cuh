// af_cellop.cuh -- generic cell-centric, sum-factorised DG operator kernel for sm_100a.
//
// One CTA owns CB consecutive cells (deal.II active-cell order = DoF order) and NQ
// threads per cell ("members").  Every operator of the reference's EULEROperator is a
// sum over "groups" of input fields of (cell integral) + (face integral) terms, so a
// Phys policy describes, per group, the input arrays, the pointwise integrand and the
// numerical flux; this kernel does the data movement and the tensor-product algebra:
//
//   per group:  global -> smem (coalesced, 16-byte loads, odd-padded per cell)
//               X pass : rows (i, P-i) combined even/odd, contracted along x  -> smem
//               Z pass : member = quadrature column qx; points (qz, NQ-1-qz) in pairs,
//                        integrand, then test-function contraction along z accumulated
//                        in registers (even/odd split, constant-memory coefficients)
//               faces  : member = face quadrature point; own trace and the neighbour's
//                        trace (GLL nodes on the face), numerical flux, weighted and
//                        accumulated per (face, output, point) in smem
//   then:       XT pass: contraction along x of the accumulated rows, plus the face
//                        terms on the face nodes -> smem -> coalesced global stores.
//
// Faces are evaluated from both sides (cell-centric): no atomics, deterministic, and the
// flux seen by the two cells of a face is the exact negation of each other because the
// normals come from the same two vertices.  Boundary faces call Phys::boundary.
#pragma once

#include <cuda_runtime.h>

#include <atomic>
#include <type_traits>
#include <utility>

#include "af_tables.cuh"

namespace af {

struct MeshDev {
  const double2* vtx;  // (nz+1)*(nx+1) vertices, row-major in (j, i)
  int nx, nz, periodic_x, gravity;
  double radial_a;
  int cell0;  // cell kernels: the first cell of the launch (a multiple of its cells per CTA);
              // the launch covers [cell0, ncell).  0 for whole-mesh launches
  // Status word of the caller (host-visible; null: not reported).  A kernel that gives up a
  // bounded wait writes kStatusStageTimeout there and leaves without writing its outputs.
  int* status;
  // Test hook (0 in normal use): when > 0, each CTA of a cell kernel first waits on a barrier
  // phase that never completes and gives up after this many polls, before it issues any copy.
  int test_wait_polls;
};

// Codes a kernel leaves in MeshDev::status.
constexpr int kStatusStageTimeout = 1;

struct PointGeo {
  double X[2];  // physical position (valid when Phys::NEED_X)
  double J[4];  // Jacobian (x_xi, x_eta, z_xi, z_eta) (valid for policies with gradient fields)
};

// Policies may declare "gradient fields": the last nfg_of(G) cell fields of group G, whose
// reference-coordinate derivatives at the quadrature points are passed to their point
// function as well (point<G>(prm, v, deta, pg, val, gr): v holds the group's values, then
// d/dxi of the gradient fields; deta holds their d/deta).  Policies without nfg_of have none.
template <class Phys, class = void>
struct NfgOf {
  static constexpr int get(int) { return 0; }
};
template <class Phys>
struct NfgOf<Phys, std::void_t<decltype(Phys::nfg_of(0))>> {
  static constexpr int get(int g) { return Phys::nfg_of(g); }
};

// Policies may map their integrand to the reference cell themselves (Phys::MAPPED): their
// point_mapped<G>(prm, v, pg, A, dw, fv, fx, fe) adds, per output o, fv[o] = value * |J| w and
// (fx[o], fe[o]) = (A0 g0 - A1 g1, A3 g1 - A2 g0) for the output's flux g, with
// A = (J11, J01, J10, J00) w = adj(J) w.  A policy that knows the structure of its fluxes can
// share products of the Jacobian between outputs (contravariant velocities); the others return
// physical values and fluxes and the kernel maps them.
template <class Phys, class = void>
struct MappedOf {
  static constexpr bool value = false;
};
template <class Phys>
struct MappedOf<Phys, std::void_t<decltype(Phys::MAPPED)>> {
  static constexpr bool value = Phys::MAPPED;
};

// Policies opt in to z-face folding (Layout::FOLD_Z) with Phys::FOLD = true.  Measured at
// 512x256, p = 4: the fused rhs 439 -> 399 us with it, its stage-1 backward 1.53 -> 1.43 ms;
// C (the enthalpy operator) 125 -> 153 us and the FP64 IMEX step 265 -> 275 ms, where the
// z-faces evaluated after the z pass serialise behind it; the FP32 smoother kernels are
// indifferent (mixed step 77.1 vs 77.4 ms).
template <class Phys, class = void>
struct FoldOf {
  static constexpr bool value = false;
};
template <class Phys>
struct FoldOf<Phys, std::void_t<decltype(Phys::FOLD)>> {
  static constexpr bool value = Phys::FOLD;
};

// Whether a policy's point functions read the physical position: Phys::NEED_X, and for
// parameters that say so (needs_position()) only when they do (the vertical gravity of the hill
// needs no position, radial gravity and the sponge do).
template <class Prm, class = void>
struct PositionUse {
  __device__ static bool get(const Prm&) { return true; }
};
template <class Prm>
struct PositionUse<Prm, std::void_t<decltype(std::declval<const Prm&>().needs_position())>> {
  __device__ static bool get(const Prm& p) { return p.needs_position(); }
};

// Policies may declare a cell-local epilogue (Phys::EPI) that replaces the plain store.  Both
// apply a cell-wise inverse mass matrix by the change of basis to the Gauss points (CobT):
//   M_K^{-1} y = Vi (W_K (Vi^T y)),  W_K = prm.inv[cell][q] = 1 / (rho(g_q) JxW(g_q)),
//   1: out = scale * M_K^{-1} y per cell and component;
//   2: the Chebyshev step on a residual increment y:  r += y;  d' = alpha d + s M_K^{-1} r;
//      x = d' (first) or x += d'   (prm.r, prm.din, prm.dout, prm.x).  d' goes to its own
//      array: other CTAs still read d's face nodes when the operator's input is d.
//   3: the Chebyshev step on a preconditioned residual z (prm.r holds z):
//      z' = z + g M_K^{-1} y - d;  d' = alpha d + s z';  x = d' (first) or x += d'.
// The CTA's weights are brought in by a bulk copy issued at kernel start.
template <class Phys, class = void>
struct EpiOf {
  static constexpr int value = 0;
};
template <class Phys>
struct EpiOf<Phys, std::void_t<decltype(Phys::EPI)>> {
  static constexpr int value = Phys::EPI;
};

// Cell indices kept in the real-typed geometry block, stored bit for bit (a float holds
// integers exactly only up to 2^24, fewer than the cells of a large mesh).
__device__ __forceinline__ void put_index(float& s, int v) { s = __int_as_float(v); }
__device__ __forceinline__ void put_index(double& s, int v) { s = __longlong_as_double((long long)v); }
__device__ __forceinline__ int get_index(float s) { return __float_as_int(s); }
__device__ __forceinline__ int get_index(double s) { return (int)__double_as_longlong(s); }

// Face neighbours of cell c (faces 0: xi=0, 1: xi=1, 2: eta=0, 3: eta=1); -1 on a wall.
__device__ __forceinline__ void cell_neighbours(const MeshDev& mesh, int c, int nb[4]) {
  const int i = c % mesh.nx, j = c / mesh.nx;
  nb[0] = i > 0 ? c - 1 : (mesh.periodic_x ? c + mesh.nx - 1 : -1);
  nb[1] = i < mesh.nx - 1 ? c + 1 : (mesh.periodic_x ? c - mesh.nx + 1 : -1);
  nb[2] = j > 0 ? c - mesh.nx : -1;
  nb[3] = j < mesh.nz - 1 ? c + mesh.nx : -1;
}

template <int N, class F, int... I>
__device__ __forceinline__ void sfor_impl(F& f, std::integer_sequence<int, I...>) {
  (f(std::integral_constant<int, I>{}), ...);
}
template <int N, class F>
__device__ __forceinline__ void sfor(F&& f) {
  sfor_impl<N>(f, std::make_integer_sequence<int, N>{});
}

// 1D tables of degree P in precision R; each kernel translation unit defines the
// specialisations it uses (constant memory is per module).
template <int P, class R, int NQ = 2 * P + 1>
__device__ __forceinline__ const TabT<P, R, NQ>& tabr();
template <int P>
__device__ __forceinline__ const Tab<P>& tab() {
  return tabr<P, double>();
}
// change-of-basis tables (cell-wise inverse mass matrices without stored matrices)
template <int P, class R>
__device__ __forceinline__ const CobT<P, R>& cobr();

// Fused multiply-add in the working precision (no silent promotion of float operands).
__device__ __forceinline__ double fmaR(double a, double b, double c) { return __fma_rn(a, b, c); }
__device__ __forceinline__ float fmaR(float a, float b, float c) { return __fmaf_rn(a, b, c); }

// Working precision of a Phys policy: Phys::real.
template <class Phys>
using RealOf = typename Phys::real;

// Asynchronous global -> shared copies (all of a group in flight, one wait).
__device__ __forceinline__ void cp_async_el(double* smem_dst, const double* gsrc) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem_dst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gsrc) : "memory");
}
__device__ __forceinline__ void cp_async_el(float* smem_dst, const float* gsrc) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem_dst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(s), "l"(gsrc) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

constexpr int odd(int n) { return n | 1; }

// Own-cell staging by bulk copies (1) or per-element cp.async (0); see Layout::BULK.
#ifndef AF_BULK_STAGING
#define AF_BULK_STAGING 1
#endif
constexpr bool kBulkStaging = AF_BULK_STAGING != 0;

// Programmatic dependent launch between consecutive cell-operator launches in a stream: every
// CTA allows the next launch at its entry (griddepcontrol.launch_dependents), so the next
// launch's CTAs start on the SMs this one frees and run their prologue while it finishes; they
// wait (griddepcontrol.wait: this grid complete, its writes visible) before they read or write
// anything a kernel can write.  Geometry-first prologue (the geometry before the wait, the
// own-cell copies after it) or wait-first (the copies issued at once, overlapping the
// geometry, as without the dependent launch): AF_PDL_GEO_FIRST 1 always, 0 never, 2 for the
// FP32 kernels only.  Measured at 512x256, p = 4: the fused FP64 rhs 401.0 us without the
// dependent launch, 401.9 geometry-first, 397.5 wait-first; the mixed IMEX step (FP32
// smoothers, about 1000 launches of 45-55 us) 77.8, 75.0 and 75.6 ms.
#ifndef AF_PDL
#define AF_PDL 1
#endif
#ifndef AF_PDL_GEO_FIRST
#define AF_PDL_GEO_FIRST 2
#endif
constexpr bool kPDL = AF_PDL != 0;
template <class R>
constexpr bool pdl_geo_first() {
  return kPDL && (AF_PDL_GEO_FIRST == 1 || (AF_PDL_GEO_FIRST == 2 && sizeof(R) == 4));
}
__device__ __forceinline__ void pdl_allow_next() {
  if constexpr (kPDL) asm volatile("griddepcontrol.launch_dependents;\n" ::: "memory");
}
__device__ __forceinline__ void pdl_wait_previous() {
  if constexpr (kPDL) asm volatile("griddepcontrol.wait;\n" ::: "memory");
}

// Bounded wait on a shared-memory mbarrier phase; false when the bound was reached.
constexpr int kStageWaitPolls = 1 << 20;
__device__ __forceinline__ bool mbar_wait(unsigned bar, unsigned phase, int polls = kStageWaitPolls) {
  for (int it = 0; it < polls; ++it) {
    unsigned ok;
    asm volatile(
        "{\n.reg .pred p;\nmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\nselp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(bar), "r"(phase)
        : "memory");
    if (ok) return true;
  }
  return false;
}

// Records a given-up wait in the caller's status word (mapped host memory or device memory;
// every CTA that gives up writes the same code, so a plain store is enough).
__device__ __forceinline__ void report_status(int* status, int code) {
  if (status) {
    *reinterpret_cast<volatile int*>(status) = code;
    __threadfence_system();
  }
}

// Unroll factor of the z-pass loop over quadrature-point pairs (see the kernel).
#ifndef AF_Z_UNROLL
#define AF_Z_UNROLL 1
#endif
constexpr int kZUnroll = AF_Z_UNROLL;

// Cells per CTA and the CTAs-per-SM hint of __launch_bounds__, per degree.  Measured on
// B200 for the fused stage-1 right-hand side at 512x256 cells, degree 4 (CB, MINB):
// (16,1) 781 us, (16,2) 502 us, (32,1) 529 us, (8,3) 592 us, (8,4) 588 us (z loop not
// unrolled; fully unrolled: 764 / 521 / 567 / 554 / 550 us).  Degree 5: (8,3) 822 us,
// (8,2) 842, (12,2) 863, (16,2) 995 (one CTA per SM: 128 KB of shared memory).  Degree 6:
// (8,2) 1070 us, (4,4) 1153, (6,3) 1406.  Degree 3: (16,3) 244 us, (16,2) 266, (24,2) 273,
// (32,1) 299.
template <int P>
constexpr int cells_per_block() {
  return P <= 1 ? 64 : (P == 2 ? 32 : (P <= 4 ? 16 : 8));
}
template <int P>
constexpr int min_blocks_per_sm() {
  return P == 3 || P == 5 ? 3 : 2;
}

template <int MAXARR, int MAXOUT, class R = double>
struct ArgPtrs {
  const R* in[MAXARR];
  R* out[MAXOUT];
};

// ----------------------------------------------------------------------------------
// compile-time helpers over a Phys policy
// ----------------------------------------------------------------------------------
template <class Phys, int G>
struct GroupInfo {
  static constexpr int NARR = Phys::template Grp<G>::NARR;
  static constexpr int arr_base() {
    int b = 0;
    for (int g = 0; g < G; ++g) b += Phys::narr_of(g);
    return b;
  }
  static constexpr int NF = [] {
    int n = 0;
    for (int a = 0; a < NARR; ++a) n += Phys::template Grp<G>::ncomp(a);
    return n;
  }();
  static constexpr int NF_GRAD = NfgOf<Phys>::get(G);  // the last NF_GRAD cell fields
  static constexpr int NF_CELL = [] {  // fields used by cell integrals (face-only ones last)
    int n = 0;
    for (int a = 0; a < NARR; ++a)
      if (!Phys::template Grp<G>::face_only(a)) n += Phys::template Grp<G>::ncomp(a);
    return n;
  }();
};

template <class Phys, int... G>
constexpr int count_face_groups(std::integer_sequence<int, G...>) {
  return ((Phys::FACES && Phys::template Grp<G>::FACE ? 1 : 0) + ... + 0);
}
template <class Phys, int... G>
constexpr int last_face_group(std::integer_sequence<int, G...>) {
  int r = -1;
  ((r = (Phys::FACES && Phys::template Grp<G>::FACE) ? G : r), ...);
  return r;
}

template <class Phys>
struct PhysInfo {
  static constexpr int NFACEG = count_face_groups<Phys>(std::make_integer_sequence<int, Phys::NG>{});
  static constexpr int FACE_G = last_face_group<Phys>(std::make_integer_sequence<int, Phys::NG>{});
  static constexpr int NFMAX = [] {
    int m = 0;
    for (int g = 0; g < Phys::NG; ++g) m = m > Phys::nf_of(g) ? m : Phys::nf_of(g);
    return m;
  }();
  static constexpr int NARR_TOTAL = [] {
    int n = 0;
    for (int g = 0; g < Phys::NG; ++g) n += Phys::narr_of(g);
    return n;
  }();
  // cell fields (all groups) evaluated together in the merged z pass
  // x-contracted slots: per group its cell fields (S rows), then its gradient fields again
  // (D rows, for d/dxi)
  static constexpr int NFC_TOTAL = [] {
    int n = 0;
    for (int g = 0; g < Phys::NG; ++g) n += Phys::nfc_of(g) + NfgOf<Phys>::get(g);
    return n;
  }();
  static constexpr int eo_offset(int G) {
    int n = 0;
    for (int g = 0; g < G; ++g) n += Phys::nfc_of(g) + NfgOf<Phys>::get(g);
    return n;
  }
  static constexpr int NFG_TOTAL = [] {
    int n = 0;
    for (int g = 0; g < Phys::NG; ++g) n += NfgOf<Phys>::get(g);
    return n;
  }();
  static constexpr int grad_offset(int G) {
    int n = 0;
    for (int g = 0; g < G; ++g) n += NfgOf<Phys>::get(g);
    return n;
  }
};

// Gauss points per direction of a policy: the operator's 2P+1, or P+1 for a policy that
// declares REDUCED_Q (preconditioner operators; exact for B, M and D on bilinear cells).
template <int P, class Phys, class = void>
struct NQOf {
  static constexpr int value = 2 * P + 1;
};
template <int P, class Phys>
struct NQOf<P, Phys, std::void_t<decltype(Phys::REDUCED_Q)>> {
  static constexpr int value = Phys::REDUCED_Q ? P + 1 : 2 * P + 1;
};

template <int P, class Phys, int CB_ = cells_per_block<P>()>
struct Layout {
  using R = RealOf<Phys>;
  using T = TabT<P, R, NQOf<P, Phys>::value>;
  static constexpr int P1 = T::P1, NQ = T::NQ, ND = P1 * P1;
  static constexpr int CB = CB_;
  static constexpr int NT = CB * NQ;
  static constexpr int NDP = odd(ND);
  static constexpr int P1P = odd(P1);
  static constexpr int EOS = odd(P1 * NQ);
  static constexpr int NF = PhysInfo<Phys>::NFMAX;
  static constexpr int NFC = PhysInfo<Phys>::NFC_TOTAL;
  static constexpr int NOUT = Phys::NOUT;
  // region A: x-contracted rows of every cell field, later the z-accumulators
  static constexpr int R_EO = NFC * CB * EOS;
  static constexpr int R_ACC = NOUT * 2 * CB * EOS;
  static constexpr int ALIGN = 16 / (int)sizeof(R);  // region B starts on a 16-byte boundary
  static constexpr int RA = ((R_EO > R_ACC ? R_EO : R_ACC) + ALIGN - 1) / ALIGN * ALIGN;
  // Own-cell staging by bulk asynchronous copies (TMA, one per array and CTA): the
  // shared-memory image of an array equals its global chunk, laid out [cell][comp][node], and
  // chunk sizes are multiples of 16 bytes (CB even).  Without padding an even ND puts the same
  // node of consecutive cells on few banks: at degree 3 (ND 16, every cell on the same bank)
  // bulk staging measured 414 us against 245 us with the padded per-element copies, at degree 5
  // (ND 36 doubles, a 4-way conflict) 748 us against 836 us, and 707 us with the padded slots
  // below; so even ND stages in bulk only at degree 5 in FP64.
  static constexpr bool BULK =
      kBulkStaging && (CB % 2 == 0) && ((ND % 2 == 1) || (P == 5 && sizeof(R) == 8));
  // Padded bulk layout (even ND, i.e. degree 5 in FP64): each cell's chunk of an array arrives
  // by its own bulk copy into a slot 16 bytes longer than the chunk (38 doubles for a scalar
  // field, 74 for a velocity), so that the same node of the CTA's 8 cells lies on 8 different
  // bank pairs instead of 4 (36 doubles = 8 banks apart).  The copies are spread over warp 0.
  static constexpr int PADB = (BULK && ND % 2 == 0) ? ALIGN : 0;
  static constexpr int slot(int nc) { return nc * ND + PADB; }  // one cell of an array
  static constexpr int ISSUE_LANES = PADB ? 32 : 1;             // threads that issue the copies
  // region B: one group's nodal values and neighbour face nodes, later the outputs
  static constexpr int R_IN = NF * CB * (NDP > ND + PADB ? NDP : ND + PADB);
  static constexpr int R_NB = Phys::FACES ? 4 * NF * CB * P1P : 0;
  static constexpr int R_OUT = NOUT * CB * NDP;
  static constexpr int RB = (R_IN + R_NB) > R_OUT ? (R_IN + R_NB) : R_OUT;
  // z-face folding: with one face group whose staged nodes and neighbour face nodes are still in
  // place after the z pass (no later group reuses its buffer), the fluxes of the z-faces are
  // evaluated at the end of the z pass by the thread of quadrature column q and added to its
  // accumulators of node rows 0 and P (the face term of node (iz, ix) on face 2 is
  // delta(iz, 0) sum_q S(q, ix) F(q), the x-transpose pass's contraction of row 0); the
  // x-transpose pass then has no edge rows with extra work
  // (two input buffers: FACE_G + 2 >= NG; one buffer: FACE_G is the last group)
  static constexpr int FACE_G = PhysInfo<Phys>::FACE_G;
  static constexpr bool FOLD_OK = FoldOf<Phys>::value && Phys::FACES && PhysInfo<Phys>::NFACEG == 1;
  static constexpr bool FOLD_2BUF = FOLD_OK && FACE_G + 2 >= Phys::NG;
  static constexpr bool FOLD_1BUF = FOLD_OK && FACE_G == Phys::NG - 1;
  static constexpr int flux_size(bool fold) { return Phys::FACES ? (fold ? 2 : 4) * NOUT * CB * NQ : 0; }

  // per cell: A,B,C,v0 (8) + 4 faces x (nx,nz,len) (12) + 4 nb; an odd stride, so that a warp
  // reading one slot of consecutive cells meets no bank conflicts (4- and 8-byte elements)
  static constexpr int GS = 25;
  static constexpr int R_GEO = CB * GS;
  static constexpr int R_S = NQ * P1 + NQ;
  // bulk staging of several groups: the own-cell chunks of group G+1 are copied into a second
  // input buffer while group G is computed (group 0's at kernel entry); buffers alternate.
  // Only where the second buffer leaves the number of resident CTAs per SM unchanged (228 KB
  // of shared memory per SM, 1 KB reserved per CTA).
  static constexpr int RBA = (RB + ALIGN - 1) / ALIGN * ALIGN;
  static constexpr int R_IN_A = (R_IN + ALIGN - 1) / ALIGN * ALIGN;
  static constexpr int EPI = EpiOf<Phys>::value;
  static constexpr int NE = EPI >= 2 ? 4 : 1;
  static constexpr int total_with(int rin2, int rflux) {
    const int base = RA + RBA + rin2 + rflux + R_GEO + R_S;
    return EPI ? (base + ALIGN - 1) / ALIGN * ALIGN + NE * CB * ND : base;
  }
  static constexpr int ctas_per_sm(int total) { return (228 * 1024) / ((int)sizeof(R) * total + 1024); }
  static constexpr int T_PF = total_with(R_IN_A, flux_size(FOLD_2BUF)), T_NOPF = total_with(0, flux_size(FOLD_1BUF));
  static constexpr bool PREFETCH =
      BULK && Phys::NG > 1 && (int)sizeof(R) * T_PF <= 227 * 1024 && ctas_per_sm(T_PF) >= ctas_per_sm(T_NOPF);
  static constexpr int R_IN2 = PREFETCH ? R_IN_A : 0;
  static constexpr bool FOLD_Z = PREFETCH ? FOLD_2BUF : FOLD_1BUF;
  // the flux accumulators of the x-faces (0, 1) and, unless folded, of the z-faces (2, 3)
  static constexpr int R_FLUX = flux_size(FOLD_Z);
  static constexpr int RB2 = RBA + R_IN2;
  // region E (epilogue policies): the CTA's Gauss-point inverse weights, 16-byte aligned
  static constexpr int OE = (RA + RB2 + R_FLUX + R_GEO + R_S + ALIGN - 1) / ALIGN * ALIGN;
  // (EPI 2 and 3 also prefetch the residual (or z), the previous direction and the iterate of
  // their cells: NE chunks)
  static constexpr int TOTAL = EPI ? OE + NE * CB * ND : RA + RB2 + R_FLUX + R_GEO + R_S;
  // the epilogue's scratch (input rows and half-transformed values) lives in region A
  static_assert(EPI == 0 || RA >= (NOUT + 1) * CB * ND, "region A too small for the epilogue");
  static constexpr size_t BYTES = sizeof(R) * TOTAL;
  static_assert(BYTES <= 227 * 1024, "shared memory of one CTA above the sm_100 limit");
};

// even/odd contraction of a P1-vector r along one direction to NQ values
template <int P, class R, int NQ>
__device__ __forceinline__ void contract_eo(const R* r, R* y) {
  using T = TabT<P, R, NQ>;
  const T& t = tabr<P, R, NQ>();
  R re[T::H > 0 ? T::H : 1], ro[T::H > 0 ? T::H : 1];
#pragma unroll
  for (int i = 0; i < T::H; ++i) {
    re[i] = r[i] + r[P - i];
    ro[i] = r[i] - r[P - i];
  }
  const R rm = T::MIDN ? r[P / 2] : 0.0;
#pragma unroll
  for (int k = 0; k < T::QH; ++k) {
    R e = 0.0, o = 0.0;
#pragma unroll
    for (int i = 0; i < T::H; ++i) {
      e = fmaR(t.Se[k][i], re[i], e);
      o = fmaR(t.So[k][i], ro[i], o);
    }
    if (T::MIDN) e = fmaR(t.Sm[k], rm, e);
    y[k] = e + o;
    y[T::NQ - 1 - k] = e - o;
  }
  if constexpr (T::QMID) {  // the middle point sees the even part only
    R e = 0.0;
#pragma unroll
    for (int i = 0; i < T::H; ++i) e = fmaR(t.Se[T::QH][i], re[i], e);
    if (T::MIDN) e = fmaR(t.Sm[T::QH], rm, e);
    y[T::QH] = e;
  }
}

// derivative counterpart: y[q] = sum_i D[q][i] r[i] with D[NQ-1-q][i] = -D[q][P-i]
template <int P, class R, int NQ>
__device__ __forceinline__ void contract_eo_D(const R* r, R* y) {
  using T = TabT<P, R, NQ>;
  const T& t = tabr<P, R, NQ>();
  R re[T::H > 0 ? T::H : 1], ro[T::H > 0 ? T::H : 1];
#pragma unroll
  for (int i = 0; i < T::H; ++i) {
    re[i] = r[i] + r[P - i];
    ro[i] = r[i] - r[P - i];
  }
  const R rm = T::MIDN ? r[P / 2] : R(0);
#pragma unroll
  for (int k = 0; k < T::QE; ++k) {
    R e = 0.0, o = 0.0;
#pragma unroll
    for (int i = 0; i < T::H; ++i) {
      e = fmaR(t.De[k][i], re[i], e);
      o = fmaR(t.Do[k][i], ro[i], o);
    }
    if (T::MIDN) e = fmaR(t.Dm[k], rm, e);
    y[k] = e + o;
    if (k < T::QH) y[T::NQ - 1 - k] = o - e;
  }
}

// ----------------------------------------------------------------------------------
// the kernel
// ----------------------------------------------------------------------------------
template <int P, class Phys, int CB_ = cells_per_block<P>(), int MINB = min_blocks_per_sm<P>()>
__global__ void __launch_bounds__(Layout<P, Phys, CB_>::NT, MINB)
    k_cellop(const MeshDev mesh, const ArgPtrs<PhysInfo<Phys>::NARR_TOTAL, Phys::NOUT_ARR, RealOf<Phys>> ptr,
             const typename Phys::Params prm, const int ncell) {
  using L = Layout<P, Phys, CB_>;
  using R = RealOf<Phys>;
  using T = typename L::T;
  constexpr int P1 = L::P1, NQ = L::NQ, ND = L::ND, CB = L::CB, NT = L::NT;
  constexpr int H = T::H;
  constexpr bool MIDN = T::MIDN;
  constexpr int QH = T::QH;  // quadrature point pairs (q, NQ-1-q); middle point QH if T::QMID
  constexpr int NOUT = Phys::NOUT;
  constexpr int NFC_ALL = L::NFC;
  const T& tb = tabr<P, R, NQ>();

  extern __shared__ __align__(16) unsigned char smem_raw[];
  R* smem = reinterpret_cast<R*>(smem_raw);
  R* s_eo = smem;             // region A
  R* s_acc = smem;            //   (after the z pass)
  R* s_in0 = smem + L::RA;    // region B
  R* s_nb = s_in0 + L::R_IN;
  R* s_out = s_in0;           //   (after the last group)
  R* s_in2 = smem + L::RA + (L::RB2 - L::R_IN2);  // second input buffer (Layout::PREFETCH)
  R* s_flux = smem + L::RA + L::RB2;
  R* s_geo = s_flux + L::R_FLUX;
  R* s_S = s_geo + L::R_GEO;
  R* s_w = s_S + NQ * P1;

  // bulk-copy completion (Layout::BULK), one barrier per input buffer
  __shared__ alignas(8) unsigned long long s_bar[2];
  const unsigned bar = (unsigned)__cvta_generic_to_shared(&s_bar[0]);
  const unsigned bar2 = (unsigned)__cvta_generic_to_shared(&s_bar[1]);
  pdl_allow_next();
  if (mesh.test_wait_polls > 0) {
    // test hook: the bounded wait gives up on a phase that nobody completes (s_bar is armed
    // with an arrival count of 1 and nobody arrives), then the CTA leaves as after a real
    // staging timeout; no copy has been issued yet
    bool ok = true;
    if (threadIdx.x == 0) {
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(bar) : "memory");
      ok = mbar_wait(bar, 0, mesh.test_wait_polls);
      if (!ok) report_status(mesh.status, kStatusStageTimeout);
    }
    if (__syncthreads_or(!ok)) return;
  }
  const int c0 = mesh.cell0 + blockIdx.x * CB;
  const int ncb = min(CB, ncell - c0);  // valid cells in this block
  // own cells of a group: the contiguous chunk of each array, by one bulk copy per array (TMA)
  // when the layout allows (uniform per CTA), otherwise by coalesced per-element copies
  const bool bulk = L::BULK && ((size_t)ncb * ND * sizeof(R)) % 16 == 0;
  // issued by warp 0 (lane 0 alone without padding): group G's chunks into input buffer G % 2
  // (buffer 0 without prefetch)
  auto issue_group = [&](auto gc) {
    constexpr int G = decltype(gc)::value;
    using Gi = GroupInfo<Phys, G>;
    using Gr = typename Phys::template Grp<G>;
    R* buf = (L::PREFETCH && (G & 1)) ? s_in2 : s_in0;
    const unsigned gbar = (L::PREFETCH && (G & 1)) ? bar2 : bar;
    const int lane = threadIdx.x;
    if (lane == 0) {
      unsigned bytes = 0;
      sfor<Gi::NARR>([&](auto ac) { bytes += (unsigned)(ncb * Gr::ncomp(decltype(ac)::value) * ND * sizeof(R)); });
      asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
      asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(gbar), "r"(bytes) : "memory");
    }
    if constexpr (L::PADB == 0) {
      if (lane == 0) {
        sfor<Gi::NARR>([&](auto ac) {
          constexpr int A = decltype(ac)::value;
          constexpr int NC = Gr::ncomp(A);
          constexpr int fb = [] { int b = 0; for (int a = 0; a < A; ++a) b += Gr::ncomp(a); return b; }();
          const R* src = ptr.in[Gi::arr_base() + A] + (size_t)c0 * NC * ND;
          const unsigned dst = (unsigned)__cvta_generic_to_shared(buf + fb * CB * ND);
          asm volatile(
              "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(
                  dst),
              "l"(src), "r"((unsigned)(ncb * NC * ND * sizeof(R))), "r"(gbar)
              : "memory");
        });
      }
    } else {
      // one copy per (array, cell), spread over the lanes of warp 0; every chunk and slot is a
      // multiple of 16 bytes (ND * 8 = 288 bytes, slots of 304 and 592), so both addresses stay
      // 16-byte aligned
      __syncwarp();
      asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
      sfor<Gi::NARR>([&](auto ac) {
        constexpr int A = decltype(ac)::value;
        constexpr int NC = Gr::ncomp(A);
        constexpr int ab = [] { int b = 0; for (int a = 0; a < A; ++a) b += CB * L::slot(Gr::ncomp(a)); return b; }();
        const R* src = ptr.in[Gi::arr_base() + A] + (size_t)c0 * NC * ND;
        for (int cc = lane; cc < ncb; cc += 32) {
          const unsigned dst = (unsigned)__cvta_generic_to_shared(buf + ab + cc * L::slot(NC));
          asm volatile(
              "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(
                  dst),
              "l"(src + (size_t)cc * NC * ND), "r"((unsigned)(NC * ND * sizeof(R))), "r"(gbar)
              : "memory");
        }
      });
    }
  };
  // neighbours' face nodes of a face group (L2-resident), ordered along the face parameter, by
  // per-element asynchronous copies; one element per thread for each (face, field):
  // CB * P1 <= NT for every degree
  auto gather_neighbours = [&](auto gc) {
    constexpr int G = decltype(gc)::value;
    using Gi = GroupInfo<Phys, G>;
    using Gr = typename Phys::template Grp<G>;
    constexpr int NF = Gi::NF;
    static_assert(CB * P1 <= NT, "neighbour staging assumes one element per thread");
    const int tid = threadIdx.x;
    const int cc = tid / P1, i = tid % P1;
    if (tid < CB * P1) {
      int nbs[4];
      cell_neighbours(mesh, c0 + (cc < ncb ? cc : ncb - 1), nbs);
#pragma unroll
      for (int f = 0; f < 4; ++f) {
        const int nb = nbs[f];
        const bool ok = nb >= 0 && cc < ncb;
        const int kk = f == 0 ? i * P1 + P : (f == 1 ? i * P1 : (f == 2 ? P * P1 + i : i));
        sfor<Gi::NARR>([&](auto ac) {
          constexpr int A = decltype(ac)::value;
          constexpr int NC = Gr::ncomp(A);
          constexpr int fb = [] { int b = 0; for (int a = 0; a < A; ++a) b += Gr::ncomp(a); return b; }();
          const R* base = ptr.in[Gi::arr_base() + A];
#pragma unroll
          for (int d = 0; d < NC; ++d) {
            R* dst = &s_nb[((f * NF + fb + d) * CB + cc) * L::P1P + i];
            if (ok) cp_async_el(dst, base + (size_t)nb * NC * ND + d * ND + kk);
            else *dst = 0.0;
          }
        });
      }
    }
  };
  // shared-memory offset of field fi (group-local) of cell cl_ in the staged nodes of group G
  auto field_offset = [&](auto gc, int fi, int cl_) -> int {
    constexpr int G = decltype(gc)::value;
    using Gi = GroupInfo<Phys, G>;
    using Gr = typename Phys::template Grp<G>;
    if constexpr (!L::BULK) {
      return (fi * CB + cl_) * L::NDP;
    } else {
      int off = 0, fb = 0, ab = 0;
#pragma unroll
      for (int a = 0; a < Gi::NARR; ++a) {
        const int nc = Gr::ncomp(a);
        if (fi >= fb && fi < fb + nc) off = ab + cl_ * L::slot(nc) + (fi - fb) * ND;
        fb += nc;
        ab += CB * L::slot(nc);
      }
      return off;
    }
  };
  // numerical flux of face group G on face f of this thread's cell at face point q, times the
  // face JxW: the own trace from the group's staged nodes, the neighbour's from its gathered
  // face nodes; sq = the basis at point q
  auto face_flux = [&](auto gc, int f, int q, const R* sq, R* fo) {
    constexpr int G = decltype(gc)::value;
    constexpr int NF = GroupInfo<Phys, G>::NF;
    const R* sin = (L::PREFETCH && (G & 1)) ? s_in2 : s_in0;
    const int cl_ = threadIdx.x % CB;
    const R* g = s_geo + cl_ * L::GS;
    const int nb = get_index(g[20 + f]);
    R vp[NF], vm[NF];
#pragma unroll
    for (int fi = 0; fi < NF; ++fi) {
      const R* cell = sin + field_offset(gc, fi, cl_);
      const R* nbv = s_nb + ((f * NF + fi) * CB + cl_) * L::P1P;
      R a = 0.0, b = 0.0;
#pragma unroll
      for (int i = 0; i < P1; ++i) {
        const int kk = f == 0 ? i * P1 : (f == 1 ? i * P1 + P : (f == 2 ? i : P * P1 + i));
        a = fmaR(sq[i], cell[kk], a);
        b = fmaR(sq[i], nbv[i], b);
      }
      vp[fi] = a;
      vm[fi] = b;
    }
    const R n[2] = {g[8 + 3 * f], g[9 + 3 * f]};
    const R jxw = g[10 + 3 * f] * s_w[q];
#pragma unroll
    for (int o = 0; o < NOUT; ++o) fo[o] = 0.0;
    if (nb >= 0) Phys::template face<G>(prm, vp, vm, n, fo);
    else Phys::template boundary<G>(prm, vp, n, fo);
#pragma unroll
    for (int o = 0; o < NOUT; ++o) fo[o] *= jxw;
  };
  // per barrier: the phase a wait expects, and whether copies were issued and not yet waited for
  unsigned ph[2] = {0u, 0u};
  bool pending[2] = {false, false};
  if constexpr (L::BULK) {
    if (threadIdx.x == 0) {
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(bar) : "memory");
      if (L::PREFETCH) asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(bar2) : "memory");
      asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
    }
    pending[0] = bulk;
  }

  bool abort = false;
  // epilogue policies: the CTA's inverse weights (and for EPI 2, 3: r, din, x), each
  // [cell][node] over the CTA's cells, copied from the start of the kernel on
  __shared__ alignas(8) unsigned long long s_bar_e;
  const unsigned bar_e = (unsigned)__cvta_generic_to_shared(&s_bar_e);
  R* s_minv = smem + L::OE;
  bool epi_bulk = false;
  const R* epi_src[4] = {nullptr, nullptr, nullptr, nullptr};
  size_t epi_bytes = 0;
  int epi_ncb = 0;
  if constexpr (L::EPI != 0) {
    const int c0e = mesh.cell0 + blockIdx.x * CB;
    epi_ncb = min(CB, ncell - c0e);
    epi_bytes = sizeof(R) * (size_t)epi_ncb * ND;
    epi_src[0] = prm.inv + (size_t)c0e * ND;
    if constexpr (L::EPI >= 2) {
      epi_src[1] = prm.r + (size_t)c0e * ND;
      epi_src[2] = prm.din + (size_t)c0e * ND;
      epi_src[3] = prm.x + (size_t)c0e * ND;
    }
    epi_bulk = epi_bytes % 16 == 0;
#pragma unroll
    for (int k = 0; k < L::NE; ++k) epi_bulk = epi_bulk && (reinterpret_cast<size_t>(epi_src[k]) & 15) == 0;
    if (epi_bulk && threadIdx.x == 0) {
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(bar_e) : "memory");
      asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
    }
  }
  // the copies that read what earlier kernels wrote: group 0's own-cell chunks (bulk layout)
  // and the epilogue's chunks
  auto issue_inputs = [&]() {
    if constexpr (L::BULK) {
      if (threadIdx.x < L::ISSUE_LANES && bulk) issue_group(std::integral_constant<int, 0>{});
    }
    if constexpr (L::EPI != 0) {
      if (epi_bulk) {
        if (threadIdx.x == 0) {
          asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(bar_e),
                       "r"((unsigned)(epi_bytes * L::NE))
                       : "memory");
#pragma unroll
          for (int k = 0; k < L::NE; ++k)
            asm volatile(
                "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(
                    (unsigned)__cvta_generic_to_shared(s_minv + k * CB * ND)),
                "l"(epi_src[k]), "r"((unsigned)epi_bytes), "r"(bar_e)
                : "memory");
        }
      } else {
#pragma unroll
        for (int k = 0; k < L::NE; ++k)
          for (int e = threadIdx.x; e < epi_ncb * ND; e += L::NT) cp_async_el(&s_minv[k * CB * ND + e], epi_src[k] + e);
      }
    }
  };
  // without the geometry-first prologue the copies start at once and overlap the geometry
  constexpr bool GEO_FIRST = pdl_geo_first<R>();
  if constexpr (!GEO_FIRST) {
    pdl_wait_previous();
    issue_inputs();
  }

  const int tid = threadIdx.x;
  const int m = tid / CB;   // member: row / column / face point
  const int cl = tid % CB;  // cell within the block
  const int c = c0 + (cl < ncb ? cl : ncb - 1);

  // ---- per-cell geometry and neighbours, spread over the cell's threads (task f < 4: face f,
  //      task 4: the bilinear map and the neighbour indices); basis copy for runtime indexing
  for (int k = tid; k < NQ * P1; k += NT) s_S[k] = tb.S[k / P1][k % P1];
  for (int k = tid; k < NQ; k += NT) s_w[k] = tb.w[k];
  for (int task = m; task < 5; task += NQ) {
    const int i = c % mesh.nx, j = c / mesh.nx, W = mesh.nx + 1;
    R* g = s_geo + cl * L::GS;
    if (task == 4) {
      const double2 v0 = mesh.vtx[j * W + i], v1 = mesh.vtx[j * W + i + 1];
      const double2 v2 = mesh.vtx[(j + 1) * W + i], v3 = mesh.vtx[(j + 1) * W + i + 1];
      g[0] = v1.x - v0.x; g[1] = v1.y - v0.y;                        // A = x_xi at eta = 0
      g[2] = v3.x - v2.x - v1.x + v0.x; g[3] = v3.y - v2.y - v1.y + v0.y;  // B (bilinear term)
      g[4] = v2.x - v0.x; g[5] = v2.y - v0.y;                        // C = x_eta at xi = 0
      g[6] = v0.x; g[7] = v0.y;
      int nb[4];
      cell_neighbours(mesh, c, nb);
      put_index(g[20], nb[0]); put_index(g[21], nb[1]); put_index(g[22], nb[2]); put_index(g[23], nb[3]);
    } else {
      // faces: 0 (xi=0, edge v0->v2), 1 (xi=1, v1->v3), 2 (eta=0, v0->v1), 3 (eta=1, v2->v3);
      // a face's normal is formed from its two vertices the same way by both cells
      const int f = task;
      const int ia = (f == 1) ? i + 1 : i, ja = (f == 3) ? j + 1 : j;                       // first vertex
      const int ib = (f == 0) ? i : i + 1, jb = (f == 2) ? j : j + 1;                       // second vertex
      const double2 a = mesh.vtx[ja * W + ia], b = mesh.vtx[jb * W + ib];
      const double tx = b.x - a.x, tz = b.y - a.y, len = sqrt(tx * tx + tz * tz);
      const double sg = (f == 0 || f == 3) ? 1.0 : -1.0;  // outward: (-tz, tx) on faces 0 and 3
      const double il = sg / len;
      g[8 + 3 * f] = -tz * il;
      g[9 + 3 * f] = tx * il;
      g[10 + 3 * f] = len;
    }
  }
  if (Phys::FACES) {
    for (int k = tid; k < L::R_FLUX; k += NT) s_flux[k] = 0.0;
  }
  // geometry-first prologue: everything above read only the mesh vertices and the constant
  // tables, which no kernel writes just before a cell-operator launch; from here on the
  // previous grid's writes are visible
  if constexpr (GEO_FIRST) {
    pdl_wait_previous();
    issue_inputs();
  }

  // ================= per group: stage, x pass (to region A), face terms =================
  sfor<Phys::NG>([&](auto gc) {
    constexpr int G = decltype(gc)::value;
    using Gi = GroupInfo<Phys, G>;
    using Gr = typename Phys::template Grp<G>;
    constexpr int NF = Gi::NF, NFC = Gi::NF_CELL;
    constexpr int EOFF = PhysInfo<Phys>::eo_offset(G);
    constexpr bool GFACE = Phys::FACES && Gr::FACE;

    constexpr int B = (L::PREFETCH && (G & 1)) ? 1 : 0;  // this group's input buffer and barrier
    R* const s_in = B ? s_in2 : s_in0;

    if (abort) return;
    __syncthreads();  // the buffer of group G-1 and the neighbour area free / geometry visible
    if (bulk) {
      // group 0 was issued at kernel entry; with prefetch, group G+1 goes into the other buffer
      // now (group G-1 has finished reading it), otherwise group G is issued here
      if constexpr (L::PREFETCH) {
        if constexpr (G + 1 < Phys::NG) {
          if (tid < L::ISSUE_LANES) issue_group(std::integral_constant<int, G + 1>{});
          pending[B ^ 1] = true;
        }
      } else if constexpr (G > 0) {
        if (tid < L::ISSUE_LANES) issue_group(std::integral_constant<int, G>{});
        pending[0] = true;
      }
    } else {
      sfor<Gi::NARR>([&](auto ac) {
        constexpr int A = decltype(ac)::value;
        constexpr int NC = Gr::ncomp(A);
        constexpr int fb = [] { int b = 0; for (int a = 0; a < A; ++a) b += Gr::ncomp(a); return b; }();
        const R* src = ptr.in[Gi::arr_base() + A] + (size_t)c0 * NC * ND;
        for (int e = tid; e < ncb * NC * ND; e += NT) {
          if constexpr (L::BULK) {
            // [cell][comp][node] in the slots of the bulk layout
            constexpr int ab = [] { int b = 0; for (int a = 0; a < A; ++a) b += CB * L::slot(Gr::ncomp(a)); return b; }();
            cp_async_el(&s_in[ab + (e / (NC * ND)) * L::slot(NC) + e % (NC * ND)], src + e);
          } else {
            const int cc = e / (NC * ND), r = e % (NC * ND);
            cp_async_el(&s_in[((fb + r / ND) * CB + cc) * L::NDP + r % ND], src + e);
          }
        }
      });
    }
    auto foff = [&](int fi, int cl_) -> int { return field_offset(gc, fi, cl_); };
    if constexpr (GFACE) gather_neighbours(gc);
    cp_async_wait_all();
    if (bulk) {
      const bool ok = mbar_wait(B ? bar2 : bar, ph[B]);
      if (ok) {
        ph[B] ^= 1u;
        pending[B] = false;
      }
      if (!ok) report_status(mesh.status, kStatusStageTimeout);
      if (__syncthreads_or(!ok)) {  // every thread leaves together, nothing waits on a barrier
        abort = true;
        return;
      }
    } else {
      __syncthreads();
    }
    // ---- X pass: rows (k, P-k) even/odd, contracted along x, for the cell fields (S) and
    //      again for the gradient fields (D, slots NFC..NFC+NFG-1)
    {
      constexpr int NPR = H + (MIDN ? 1 : 0);
      constexpr int NFG = Gi::NF_GRAD;
      for (int task = m; task < (NFC + NFG) * NPR; task += NQ) {
        const int fi = task / NPR, k = task % NPR;
        const bool dxi = NFG > 0 && fi >= NFC;
        const int src = dxi ? fi - NFG : fi;  // gradient fields are the last NFG cell fields
        const R* cell = s_in + foff(src, cl);
        R* eo = s_eo + ((EOFF + fi) * CB + cl) * L::EOS;
        R r[P1], y[NQ];
        auto contract = [&]() {
          if (NFG > 0 && dxi) contract_eo_D<P, R, NQ>(r, y);
          else contract_eo<P, R, NQ>(r, y);
        };
        if (k < H) {
#pragma unroll
          for (int ix = 0; ix < P1; ++ix) r[ix] = cell[k * P1 + ix] + cell[(P - k) * P1 + ix];
          contract();
#pragma unroll
          for (int q = 0; q < NQ; ++q) eo[k * NQ + q] = y[q];
#pragma unroll
          for (int ix = 0; ix < P1; ++ix) r[ix] = cell[k * P1 + ix] - cell[(P - k) * P1 + ix];
          contract();
#pragma unroll
          for (int q = 0; q < NQ; ++q) eo[(H + k) * NQ + q] = y[q];
        } else {
#pragma unroll
          for (int ix = 0; ix < P1; ++ix) r[ix] = cell[(P / 2) * P1 + ix];
          contract();
#pragma unroll
          for (int q = 0; q < NQ; ++q) eo[(2 * H) * NQ + q] = y[q];
        }
      }
    }
    // ---- faces (same phase: reads region B only): member = face quadrature point; the
    //      z-faces of a folding layout come after the z pass
    if constexpr (GFACE) {
      const int q = m;
      R sq[P1];
#pragma unroll
      for (int i = 0; i < P1; ++i) sq[i] = s_S[q * P1 + i];
#pragma unroll
      for (int f = 0; f < (L::FOLD_Z ? 2 : 4); ++f) {
        R fo[NOUT];
        face_flux(gc, f, q, sq, fo);
#pragma unroll
        for (int o = 0; o < NOUT; ++o) s_flux[((f * NOUT + o) * CB + cl) * NQ + q] += fo[o];
      }
    }
  });
  if (abort) {  // a staging wait gave up: wait (bounded) for this CTA's copies before leaving
    if (tid == 0) {
      if (pending[0]) mbar_wait(bar, ph[0]);
      if (pending[1]) mbar_wait(bar2, ph[1]);
      if (epi_bulk) mbar_wait(bar_e, 0);
    }
    return;
  }
  __syncthreads();

  // ================= merged z pass: member = quadrature column qx =================
  // All groups' fields are evaluated at each point, their integrands summed, and the sum
  // is mapped to reference coordinates and contracted along z once.  The contraction of a
  // point pair (q, NQ-1-q) goes into even/odd accumulators of the node pairs (i, P-i):
  //   S terms:  E_i += Se[q][i] (f1 + f2),  O_i += So[q][i] (f1 - f2),  mid += Sm[q] (f1 + f2)
  //   D terms:  E_i += De[q][i] (g1 - g2),  O_i += Do[q][i] (g1 + g2),  mid += Dm[q] (g1 - g2)
  // (S[NQ-1-q][i] = S[q][P-i], D[NQ-1-q][i] = -D[q][P-i]); node i gets E_i + O_i, node P-i
  // gets E_i - O_i.  A middle point is a pair with f2 = g2 = 0.
  constexpr int HE = H > 0 ? H : 1;
  R aE[NOUT][HE], aO[NOUT][HE], aM[NOUT], bE[NOUT][HE], bO[NOUT][HE], bM[NOUT];
#pragma unroll
  for (int o = 0; o < NOUT; ++o) {
#pragma unroll
    for (int i = 0; i < HE; ++i) aE[o][i] = aO[o][i] = bE[o][i] = bO[o][i] = R(0);
    aM[o] = bM[o] = R(0);
  }
  {
    const int qx = m;
    const R* g = s_geo + cl * L::GS;
    const R xi = tb.x[qx];
    const R wx = s_w[qx];
    const R J01 = fmaR(g[2], xi, g[4]);  // x_eta (x component)
    const R J11 = fmaR(g[3], xi, g[5]);  // x_eta (z component)
    const bool need_x = Phys::NEED_X && PositionUse<typename Phys::Params>::get(prm);
    constexpr int NFG_ALL = PhysInfo<Phys>::NFG_TOTAL;
    // the mapped integrands of one point: fv (tested with phi), fx, fe (with d/dxi, d/deta phi)
    auto integrand = [&](const R* v, const R* deta, const int qz, R* fvo, R* fxo, R* feo) {
      const R eta = tb.x[qz];
      const R J00 = fmaR(g[2], eta, g[0]);
      const R J10 = fmaR(g[3], eta, g[1]);
      const R w = wx * tb.w[qz];
      const R dw = (J00 * J11 - J01 * J10) * w;
      PointGeo pg;
      if (need_x) {
        pg.X[0] = g[6] + g[0] * xi + g[4] * eta + g[2] * xi * eta;
        pg.X[1] = g[7] + g[1] * xi + g[5] * eta + g[3] * xi * eta;
      }
      if constexpr (NFG_ALL > 0) {
        pg.J[0] = J00; pg.J[1] = J01; pg.J[2] = J10; pg.J[3] = J11;
      }
      if constexpr (MappedOf<Phys>::value) {  // the policy maps its own integrand
        const R A[4] = {J11 * w, J01 * w, J10 * w, J00 * w};
#pragma unroll
        for (int o = 0; o < NOUT; ++o) fvo[o] = fxo[o] = feo[o] = R(0);
        sfor<Phys::NG>([&](auto gc) {
          constexpr int G = decltype(gc)::value;
          Phys::template point_mapped<G>(prm, v + PhysInfo<Phys>::eo_offset(G), pg, A, dw, fvo, fxo, feo);
        });
        return;
      }
      R val[NOUT], gr[NOUT][2];
#pragma unroll
      for (int o = 0; o < NOUT; ++o) { val[o] = 0.0; gr[o][0] = gr[o][1] = 0.0; }
      sfor<Phys::NG>([&](auto gc) {
        constexpr int G = decltype(gc)::value;
        if constexpr (NFG_ALL > 0)
          Phys::template point<G>(prm, v + PhysInfo<Phys>::eo_offset(G), deta + PhysInfo<Phys>::grad_offset(G), pg,
                                  val, gr);
        else
          Phys::template point<G>(prm, v + PhysInfo<Phys>::eo_offset(G), pg, val, gr);
      });
      const R a00 = J11 * w, a01 = J01 * w, a10 = J10 * w, a11 = J00 * w;  // adj(J) w
#pragma unroll
      for (int o = 0; o < NOUT; ++o) {
        fvo[o] = val[o] * dw;
        fxo[o] = a00 * gr[o][0] - a01 * gr[o][1];
        feo[o] = a11 * gr[o][1] - a10 * gr[o][0];
      }
    };
#pragma unroll kZUnroll
    for (int k = 0; k < T::QE; ++k) {
      const bool pair = k < QH;
      R v1[NFC_ALL], v2[NFC_ALL];
#pragma unroll
      for (int fi = 0; fi < NFC_ALL; ++fi) {
        const R* eo = s_eo + (fi * CB + cl) * L::EOS + qx;
        R e = 0.0, o = 0.0;
#pragma unroll
        for (int i = 0; i < H; ++i) {
          e = fmaR(tb.Se[k][i], eo[i * NQ], e);
          if (pair) o = fmaR(tb.So[k][i], eo[(H + i) * NQ], o);
        }
        if (MIDN) e = fmaR(tb.Sm[k], eo[(2 * H) * NQ], e);
        v1[fi] = e + o;
        v2[fi] = e - o;
      }
      // d/deta of the gradient fields: their S-row slots contracted with D along z
      R d1[NFG_ALL > 0 ? NFG_ALL : 1], d2[NFG_ALL > 0 ? NFG_ALL : 1];
      if constexpr (NFG_ALL > 0) {
        sfor<Phys::NG>([&](auto gc) {
          constexpr int G = decltype(gc)::value;
          using Gi = GroupInfo<Phys, G>;
          constexpr int NFG = Gi::NF_GRAD;
#pragma unroll
          for (int kk = 0; kk < NFG; ++kk) {
            const int slot = PhysInfo<Phys>::eo_offset(G) + Gi::NF_CELL - NFG + kk;
            const R* eo = s_eo + (slot * CB + cl) * L::EOS + qx;
            R e = 0.0, o = 0.0;
#pragma unroll
            for (int i = 0; i < H; ++i) {
              e = fmaR(tb.De[k][i], eo[i * NQ], e);
              o = fmaR(tb.Do[k][i], eo[(H + i) * NQ], o);  // at the middle point only o remains
            }
            if (MIDN) e = fmaR(tb.Dm[k], eo[(2 * H) * NQ], e);
            d1[PhysInfo<Phys>::grad_offset(G) + kk] = e + o;
            d2[PhysInfo<Phys>::grad_offset(G) + kk] = o - e;
          }
        });
      }
      R fv1[NOUT], fx1[NOUT], fe1[NOUT], fv2[NOUT], fx2[NOUT], fe2[NOUT];
      integrand(v1, d1, k, fv1, fx1, fe1);
      if (pair) {
        integrand(v2, d2, NQ - 1 - k, fv2, fx2, fe2);
      } else {
#pragma unroll
        for (int o = 0; o < NOUT; ++o) fv2[o] = fx2[o] = fe2[o] = R(0);
      }
#pragma unroll
      for (int o = 0; o < NOUT; ++o) {
        const bool hv = Phys::has_val(o), hg = Phys::has_grad(o);
        const R se = hv ? fv1[o] + fv2[o] : R(0), so = hv ? fv1[o] - fv2[o] : R(0);
        const R ge = hg ? fe1[o] - fe2[o] : R(0), go = hg ? fe1[o] + fe2[o] : R(0);
        const R xe = fx1[o] + fx2[o], xo = fx1[o] - fx2[o];
#pragma unroll
        for (int i = 0; i < H; ++i) {
          if (hv) {
            aE[o][i] = fmaR(tb.Se[k][i], se, aE[o][i]);
            aO[o][i] = fmaR(tb.So[k][i], so, aO[o][i]);
          }
          if (hg) {
            aE[o][i] = fmaR(tb.De[k][i], ge, aE[o][i]);
            aO[o][i] = fmaR(tb.Do[k][i], go, aO[o][i]);
            bE[o][i] = fmaR(tb.Se[k][i], xe, bE[o][i]);
            bO[o][i] = fmaR(tb.So[k][i], xo, bO[o][i]);
          }
        }
        if (MIDN) {
          if (hv) aM[o] = fmaR(tb.Sm[k], se, aM[o]);
          if (hg) {
            aM[o] = fmaR(tb.Dm[k], ge, aM[o]);
            bM[o] = fmaR(tb.Sm[k], xe, bM[o]);
          }
        }
      }
    }
  }
  // node values of the accumulators
  R acc_a[NOUT][P1], acc_b[NOUT][P1];
#pragma unroll
  for (int o = 0; o < NOUT; ++o) {
#pragma unroll
    for (int i = 0; i < H; ++i) {
      acc_a[o][i] = aE[o][i] + aO[o][i];
      acc_a[o][P - i] = aE[o][i] - aO[o][i];
      acc_b[o][i] = bE[o][i] + bO[o][i];
      acc_b[o][P - i] = bE[o][i] - bO[o][i];
    }
    if (MIDN) {
      acc_a[o][P / 2] = aM[o];
      acc_b[o][P / 2] = bM[o];
    }
  }
  if constexpr (L::FOLD_Z) {  // z-faces at face point qx = m, into node rows 0 (face 2) and P (3)
    R sq[P1];
#pragma unroll
    for (int i = 0; i < P1; ++i) sq[i] = s_S[m * P1 + i];
#pragma unroll
    for (int f = 2; f < 4; ++f) {
      R fo[NOUT];
      face_flux(std::integral_constant<int, L::FACE_G>{}, f, m, sq, fo);
#pragma unroll
      for (int o = 0; o < NOUT; ++o) acc_a[o][f == 2 ? 0 : P] += fo[o];
    }
  }
  __syncthreads();  // region A: x-contracted rows consumed -> accumulators
  {
    const int qx = m;
#pragma unroll
    for (int o = 0; o < NOUT; ++o) {
      R* A = s_acc + ((o * 2 + 0) * CB + cl) * L::EOS;
      R* B = s_acc + ((o * 2 + 1) * CB + cl) * L::EOS;
#pragma unroll
      for (int iz = 0; iz < P1; ++iz) {
        A[iz * NQ + qx] = acc_a[o][iz];
        B[iz * NQ + qx] = acc_b[o][iz];
      }
    }
  }
  __syncthreads();
  // ---- XT pass: task (output, row iz) -> P1 outputs, plus face terms on face nodes
  for (int task = m; task < NOUT * P1; task += NQ) {
    const int o = task / P1, iz = task % P1;
    const R* A = s_acc + ((o * 2 + 0) * CB + cl) * L::EOS + iz * NQ;
    const R* B = s_acc + ((o * 2 + 1) * CB + cl) * L::EOS + iz * NQ;
    R oE[H > 0 ? H : 1], oO[H > 0 ? H : 1], oM = 0.0;
#pragma unroll
    for (int i = 0; i < H; ++i) oE[i] = oO[i] = 0.0;
#pragma unroll
    for (int k = 0; k < QH; ++k) {
      const R a1 = A[k], a2 = A[NQ - 1 - k], b1 = B[k], b2 = B[NQ - 1 - k];
      const R As = a1 + a2, Ad = a1 - a2, Bs = b1 + b2, Bd = b1 - b2;
#pragma unroll
      for (int i = 0; i < H; ++i) {
        oE[i] = fmaR(tb.Se[k][i], As, oE[i]);
        oE[i] = fmaR(tb.De[k][i], Bd, oE[i]);
        oO[i] = fmaR(tb.So[k][i], Ad, oO[i]);
        oO[i] = fmaR(tb.Do[k][i], Bs, oO[i]);
      }
      if (MIDN) { oM = fmaR(tb.Sm[k], As, oM); oM = fmaR(tb.Dm[k], Bd, oM); }
    }
    if constexpr (T::QMID) {  // the middle point: even part of S, odd part of D
      const R am = A[QH], bm = B[QH];
#pragma unroll
      for (int i = 0; i < H; ++i) {
        oE[i] = fmaR(tb.Se[QH][i], am, oE[i]);
        oO[i] = fmaR(tb.Do[QH][i], bm, oO[i]);
      }
      if (MIDN) oM = fmaR(tb.Sm[QH], am, oM);
    }
    R out[P1];
#pragma unroll
    for (int i = 0; i < H; ++i) {
      out[i] = oE[i] + oO[i];
      out[P - i] = oE[i] - oO[i];
    }
    if (MIDN) out[P / 2] = oM;
    if (Phys::FACES) {
      const R* F0 = s_flux + ((0 * NOUT + o) * CB + cl) * NQ;
      const R* F1 = s_flux + ((1 * NOUT + o) * CB + cl) * NQ;
      R l = 0.0, r = 0.0;
#pragma unroll
      for (int q = 0; q < NQ; ++q) {
        const R s = s_S[q * P1 + iz];
        l = fmaR(s, F0[q], l);
        r = fmaR(s, F1[q], r);
      }
      out[0] += l;
      out[P] += r;
      if (!L::FOLD_Z && (iz == 0 || iz == P)) {
        const R* F = s_flux + (((iz == 0 ? 2 : 3) * NOUT + o) * CB + cl) * NQ;
#pragma unroll
        for (int ix = 0; ix < P1; ++ix) {
          R s = 0.0;
#pragma unroll
          for (int q = 0; q < NQ; ++q) s = fmaR(tb.S[q][ix], F[q], s);
          out[ix] += s;
        }
      }
    }
    R* dst = s_out + (o * CB + cl) * L::NDP + iz * P1;
    if constexpr (L::EPI == 1 || L::EPI == 3) {
      // the epilogue's first change-of-basis pass on the row in registers:
      // u[iz][qx] = sum_ix Vi[ix][qx] out[ix], stored in place of the row
      const CobT<P, R>& cbx = cobr<P, R>();
#pragma unroll
      for (int qx = 0; qx < P1; ++qx) {
        R t = R(0);
#pragma unroll
        for (int ix = 0; ix < P1; ++ix) t = fmaR(cbx.Vi[ix][qx], out[ix], t);
        dst[qx] = t;
      }
    } else {
#pragma unroll
      for (int ix = 0; ix < P1; ++ix) dst[ix] = out[ix];
    }
  }
  __syncthreads();
  if constexpr (L::EPI == 0) {
    // ---- store (coalesced)
    sfor<Phys::NOUT_ARR>([&](auto oc) {
      constexpr int OA = decltype(oc)::value;
      constexpr int NC = Phys::out_ncomp(OA);
      constexpr int ob = [] { int b = 0; for (int a = 0; a < OA; ++a) b += Phys::out_ncomp(a); return b; }();
      R* dst = ptr.out[OA] + (size_t)c0 * NC * ND;
      for (int e = tid; e < ncb * NC * ND; e += NT) {
        const int cc = e / (NC * ND), r = e % (NC * ND);
        const R v = s_out[((ob + r / ND) * CB + cc) * L::NDP + r % ND];
        if (Phys::ACCUMULATE) dst[e] += v;
        else dst[e] = v;
      }
    });
  } else {
    // ---- cell-local epilogue: the inverse weights (copied since kernel start)
    if (epi_bulk) {
      const bool ok = mbar_wait(bar_e, 0);
      if (!ok) report_status(mesh.status, kStatusStageTimeout);
      if (__syncthreads_or(!ok)) {
        if (tid == 0) mbar_wait(bar_e, 0);
        return;
      }
    } else {
      cp_async_wait_all();
      __syncthreads();
    }
    // EPI 2: region A is free after the x-transpose pass: s_y = the updated residual rows,
    // s_u = the values between the passes
    constexpr int NC = L::EPI == 1 ? NOUT : 1;
    R* s_y = smem;
    R* s_u = smem + CB * ND;
    const CobT<P, R>& cb = cobr<P, R>();
    if constexpr (L::EPI == 2) {
      R* r = prm.r + (size_t)c0 * ND;
      const R* s_r = s_minv + CB * ND;  // prefetched residual
      for (int e = tid; e < ncb * ND; e += NT) {
        const int cc = e / ND, k = e % ND;
        const R rn = s_r[e] + s_out[cc * L::NDP + k];
        r[e] = rn;
        s_y[cc * ND + k] = rn;
      }
      __syncthreads();
    }
    // the half-transformed values u of component o of cell cc: EPI 1 and 3 formed them in the
    // x-transpose pass (in place of the output rows), EPI 2 forms them here from the updated
    // residual
    auto ubase = [&](int o, int cc) -> R* {
      if constexpr (L::EPI == 2) return s_u + (o * CB + cc) * ND;
      else return s_out + (o * CB + cc) * L::NDP;
    };
    if constexpr (L::EPI == 2) {
      // pass 1 (along x): u[iz][qx] = sum_ix Vi[ix][qx] y[iz][ix]; task (cell, row)
      for (int e = tid; e < ncb * P1; e += NT) {
        const int cc = e / P1, iz = e % P1;
        R yr[P1];
#pragma unroll
        for (int ix = 0; ix < P1; ++ix) yr[ix] = s_y[cc * ND + iz * P1 + ix];
#pragma unroll
        for (int qx = 0; qx < P1; ++qx) {
          R t = R(0);
#pragma unroll
          for (int ix = 0; ix < P1; ++ix) t = fmaR(cb.Vi[ix][qx], yr[ix], t);
          s_u[cc * ND + iz * P1 + qx] = t;
        }
      }
      __syncthreads();
    }
    // pass 2 (along z, per column qx): to the Gauss points, times the weights, and back
    for (int e = tid; e < NC * ncb * P1; e += NT) {
      const int o = e / (ncb * P1), cc = (e / P1) % ncb, qx = e % P1;
      R* col = ubase(o, cc) + qx;
      R u[P1], t[P1];
#pragma unroll
      for (int iz = 0; iz < P1; ++iz) u[iz] = col[iz * P1];
#pragma unroll
      for (int qz = 0; qz < P1; ++qz) {
        R a = R(0);
#pragma unroll
        for (int iz = 0; iz < P1; ++iz) a = fmaR(cb.Vi[iz][qz], u[iz], a);
        t[qz] = a * s_minv[cc * ND + qz * P1 + qx];
      }
#pragma unroll
      for (int iz = 0; iz < P1; ++iz) {
        R a = R(0);
#pragma unroll
        for (int qz = 0; qz < P1; ++qz) a = fmaR(cb.Vi[iz][qz], t[qz], a);
        col[iz * P1] = a;
      }
    }
    __syncthreads();
    // pass 3 (along x): x[iz][ix] = sum_qx Vi[ix][qx] v[iz][qx], in place of the row
    for (int e = tid; e < NC * ncb * P1; e += NT) {
      const int o = e / (ncb * P1), cc = (e / P1) % ncb, iz = e % P1;
      R* row = ubase(o, cc) + iz * P1;
      R v[P1];
#pragma unroll
      for (int qx = 0; qx < P1; ++qx) v[qx] = row[qx];
#pragma unroll
      for (int ix = 0; ix < P1; ++ix) {
        R y = R(0);
#pragma unroll
        for (int qx = 0; qx < P1; ++qx) y = fmaR(cb.Vi[ix][qx], v[qx], y);
        row[ix] = y;
      }
    }
    __syncthreads();
    // the store or the update, one element per thread in global order (coalesced)
    for (int e = tid; e < NC * ncb * ND; e += NT) {
      if constexpr (L::EPI == 1) {
        // one output array, NOUT components, [cell][comp][node]: e is the offset from the CTA's first
        const int cc = e / (NOUT * ND), o = (e / ND) % NOUT, k = e % ND;
        ptr.out[0][(size_t)c0 * NOUT * ND + e] = prm.scale * ubase(o, cc)[k];
      } else if constexpr (L::EPI == 3) {  // z, din and x come from the prefetched chunks
        const int cc = e / ND, k = e % ND;
        const size_t g = (size_t)c0 * ND + e;
        const R y = ubase(0, cc)[k];
        const R dl = s_minv[2 * CB * ND + e];
        const R zn = s_minv[CB * ND + e] + prm.g * y - dl;
        const R nd = prm.alpha * dl + prm.s * zn;
        prm.r[g] = zn;
        prm.dout[g] = nd;
        prm.x[g] = prm.first ? nd : s_minv[3 * CB * ND + e] + nd;
      } else {  // din and x come from the prefetched chunks
        const int cc = e / ND, k = e % ND;
        const size_t g = (size_t)c0 * ND + e;
        const R y = ubase(0, cc)[k];
        const R nd = (prm.alpha != R(0) ? prm.alpha * s_minv[2 * CB * ND + e] : R(0)) + prm.s * y;
        prm.dout[g] = nd;
        prm.x[g] = prm.first ? nd : s_minv[3 * CB * ND + e] + nd;
      }
    }
  }
}

template <int P, class Phys, int CB_ = cells_per_block<P>(), int MINB = min_blocks_per_sm<P>()>
cudaError_t launch_cellop(const MeshDev& mesh,
                          const ArgPtrs<PhysInfo<Phys>::NARR_TOTAL, Phys::NOUT_ARR, RealOf<Phys>>& ptr,
                          const typename Phys::Params& prm, int ncell, cudaStream_t stream) {
  using L = Layout<P, Phys, CB_>;
  // The shared-memory attribute belongs to the function on the current device: one bit per
  // device (devices 0..63; beyond that it is set on every launch), set by whichever thread gets
  // there first (setting it twice is harmless).
  static std::atomic<unsigned long long> configured{0};
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  const unsigned long long bit = dev < 64 ? 1ull << dev : 0ull;
  if (bit == 0 || (configured.load(std::memory_order_acquire) & bit) == 0) {
    e = cudaFuncSetAttribute(k_cellop<P, Phys, CB_, MINB>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)L::BYTES);
    if (e != cudaSuccess) return e;
    configured.fetch_or(bit, std::memory_order_release);
  }
  if (mesh.cell0 % L::CB != 0 || mesh.cell0 < 0) return cudaErrorInvalidValue;
  if (ncell <= mesh.cell0) return cudaSuccess;
  const int nblk = (ncell - mesh.cell0 + L::CB - 1) / L::CB;
  if constexpr (!kPDL) {
    k_cellop<P, Phys, CB_, MINB><<<nblk, L::NT, L::BYTES, stream>>>(mesh, ptr, prm, ncell);
    return cudaGetLastError();
  } else {
    // may overlap the previous kernel of the stream; the kernel waits for it (griddepcontrol)
    // before it touches anything that kernel can write
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3((unsigned)nblk);
    cfg.blockDim = dim3((unsigned)L::NT);
    cfg.dynamicSmemBytes = L::BYTES;
    cfg.stream = stream;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, k_cellop<P, Phys, CB_, MINB>, mesh, ptr, prm, ncell);
  }
}

}  // namespace af
