/*
 * af_gpu.h -- C ABI of libaf_gpu.so, the B200 (sm_100a) implementation of the reference's
 * matrix-free IMEX-DG operator class EULEROperator (euler_operator.h:24-211).
 *
 * Every function returns an int status (AF_OK on success).  Vectors are FP64 device
 * pointers (16-byte aligned) in deal.II's DoF layout for the 2D structured meshes of this
 * library: cell-major in active-cell order, FE_DGQ(p) Gauss-Lobatto nodes lexicographic
 * (x fastest), velocity component-blocked inside each cell.  Work is queued on the
 * handle's CUDA stream; results are visible after af_synchronize or stream ordering.
 * A handle is not re-entrant (the reference's operator is not either: NS_stage is
 * mutable and apply_add re-initializes the operator, euler_operator.h:91, 2383-2406).
 *
 * Spaces follow the reference's DoFHandler indices (Atmospheric_Flow.cc:334-336):
 *   0 velocity (2 components), 1 pressure, 2 density.
 */
#ifndef AF_GPU_H
#define AF_GPU_H

#ifdef __cplusplus
extern "C" {
#endif

enum {
  AF_OK = 0,
  AF_BAD_ARG = 1,          /* invalid argument, stage or source count            */
  AF_CUDA = 2,             /* CUDA runtime error (see af_last_error_message)      */
  AF_NO_CONVERGENCE = 3,   /* SolverControl::NoConvergence of the reference       */
  AF_NAN = 4,              /* NaN/Inf met in a Krylov recurrence                  */
  AF_UNSUPPORTED = 5,      /* degree not compiled into this library               */
  AF_NO_DEVICE = 6,        /* no CUDA device available                            */
  AF_TIMEOUT = 7           /* a kernel gave up a bounded wait for its staged
                              inputs and left its outputs unwritten (reported by
                              the next call on the handle, or by the call that
                              synchronizes; see af_synchronize)                    */
};

typedef struct af_operator af_operator;

/* Mesh: nx x nz quadrilateral cells, cell (i, j) -> index j*nx + i, vertices
 * vertices[(j*(nx+1) + i)*2 + {0,1}] = (x, z) on the HOST.  Bilinear geometry (deal.II
 * MappingQ1).  Bottom and top are walls; lateral faces are walls or periodic.
 * gravity 0: e_z with |g| = 1/Fr^2 constant; 1: the reference's radial gravity
 * e_r |g| a^2/r^2 (euler_operator.h:790-811) with a = radial_a. */
typedef struct {
  int nx, nz;
  int periodic_x;
  const double* vertices;
  int gravity;
  double radial_a;
} af_mesh_desc;

/* EULEROperator(RunTimeParameters::Data_Storage&) + MatrixFree::reinit
 * (euler_operator.h:229-240, Atmospheric_Flow.cc:325-348).  n_q_points_1d must be
 * 2*degree+1 (QGauss(2*degree_u+1), Atmospheric_Flow.cc:345).  The handle creates its
 * own CUDA stream on the current device. */
int af_create(const af_mesh_desc* mesh, int degree, int n_q_points_1d, double Mach, double Froude, double dt,
              af_operator** out);
int af_destroy(af_operator* op);
/* Use an external stream (cudaStream_t passed as void*); NULL restores the handle's own
 * (non-blocking) stream.  To run on the legacy default stream pass cudaStreamLegacy
 * ((void*)0x1), not NULL. */
int af_set_stream(af_operator* op, void* stream);
int af_synchronize(af_operator* op);

/* Setters: euler_operator.h:243-303 */
int af_set_dt(af_operator* op, double dt);
int af_set_Mach(af_operator* op, double Ma);
int af_set_Froude(af_operator* op, double Fr);
int af_set_HYPERBOLIC_stage(af_operator* op, int stage);  /* 1..3 */
int af_set_NS_stage(af_operator* op, int stage);          /* 1..6 */

/* Deep copies of the fixed-point fields: set_rho_for_fixed / set_pres_fixed /
 * set_u_fixed, euler_operator.h:306-339.  Device pointers. */
int af_set_rho_for_fixed(af_operator* op, const double* rho);
int af_set_pres_fixed(af_operator* op, const double* p);
int af_set_u_fixed(af_operator* op, const double* u);

/* Explicit right-hand sides, src in the reference's positional order:
 *  vmult_rhs_rho_update (euler_operator.h:697-712): {rho0,u0 [,rho2,u2 [,rho3,u3]]}
 *  vmult_rhs_velocity_fixed (:2310-2325): st1 {rho0,u0,p0,rho2}; st2 {rho0,u0,p0,rho2,u2,p2,rho3};
 *                                          st3 {rho0,u0,p0,rho2,u2,p2,rho3,u3,p3}
 *  vmult_rhs_pressure (:1366-1381):        st1 {rho0,u0,p0,rho2,u_fixed};
 *                                          st2 {rho0,u0,p0,rho2,u2,p2,rho3,u_fixed};
 *                                          st3 {rho0,u0,p0,rho2,u2,p2,rho3,u3,p3,rho_curr,u_curr}
 * The stage is the HYPERBOLIC_stage set on the handle.  dst is overwritten. */
int af_vmult_rhs_rho_update(af_operator* op, double* dst, const double* const* src, int n_src);
int af_vmult_rhs_velocity_fixed(af_operator* op, double* dst, const double* const* src, int n_src);
int af_vmult_rhs_pressure(af_operator* op, double* dst, const double* const* src, int n_src);

/* The three right-hand sides of one stage in a single fused launch (no counterpart in the
 * reference, which runs three MatrixFree::loop calls).  src follows the vmult_rhs_pressure
 * list of the stage; any of dst_rho / dst_u / dst_p may be NULL to skip that equation. */
int af_vmult_rhs_fused(af_operator* op, double* dst_rho, double* dst_u, double* dst_p, const double* const* src,
                       int n_src);
/* Same with HOST buffers: copies in, computes, copies out, synchronizes.  This is the
 * call a deal.II host-vector caller makes. */
int af_vmult_rhs_fused_host(af_operator* op, double* dst_rho, double* dst_u, double* dst_p,
                            const double* const* src, int n_src);
/* Backward (vector-Jacobian product) of af_vmult_rhs_fused, the role of a
 * torch.autograd.Function's backward for the forward above (no counterpart in the
 * reference): src as for the forward (3 HYPERBOLIC_stage + 2 vectors), ybar_* = cotangents of
 * its rho, u, p outputs, xbar[n] receives the cotangents of the sources (overwritten).
 * Stage 1: a hand-written adjoint kernel (transposed sum factorisation of the cell terms, the
 * own-side flux Jacobian applied to the cotangent jump on faces, the Rusanov wave-speed branch
 * frozen as taken by the forward pass).  Stages 2 and 3: one dual-number kernel per group of
 * sources, differentiating the forward physics with the same frozen branch. */
int af_vmult_rhs_fused_backward(af_operator* op, const double* const* src, int n, const double* ybar_rho,
                                const double* ybar_u, const double* ybar_p, double* const* xbar);
/* Tangent-linear of the same forward (no counterpart in the reference): dy = J(src) dsrc, with
 * dsrc[n] directions of the sources and the wave-speed branch frozen as in the backward, so
 * that <ybar, tangent(dsrc)> = <backward(ybar), dsrc> to rounding (any stage). */
int af_vmult_rhs_fused_tangent(af_operator* op, const double* const* src, int n, const double* const* dsrc,
                               double* d_rho, double* d_u, double* d_p);

/* MatrixFreeOperators::Base::vmult -> apply_add (euler_operator.h:2362-2417):
 *  NS 1/4: density mass;  NS 3/5: rho_for_fixed-weighted velocity mass (A);
 *  NS 6: internal-energy mass D = M/(gamma-1);
 *  NS 2: Schur complement D p - C A^{-1} B p.  A^{-1} follows af_set_schur_mode. */
int af_vmult(af_operator* op, double* dst, const double* src);
/* B: pressure -> velocity space (vmult_pressure, :2422-2435) */
int af_vmult_pressure(af_operator* op, double* dst, const double* src);
/* C: velocity -> pressure space (vmult_enthalpy, :2440-2453), uses pres_fixed */
int af_vmult_enthalpy(af_operator* op, double* dst, const double* src);
/* Exact inverse of the block-diagonal mass-type operator selected by NS_stage (1/4: M,
 * 6: D = M/(gamma-1), 3/5: A weighted by rho_for_fixed): per-cell inverses (from a Cholesky
 * factorisation, stored as packed symmetric matrices), built
 * on first use and after set_rho_for_fixed.  Replaces the CG + multigrid solves of the
 * reference's update_density / update_velocity / update_pressure (Atmospheric_Flow.cc:
 * 527-535, 775-779, 870) by a direct solve; NS_stage 2 returns AF_BAD_ARG. */
int af_vmult_inverse(af_operator* op, double* dst, const double* src);
/* compute_diagonal + get_matrix_diagonal_inverse (:2591-2626): writes the inverse
 * diagonal of the operator selected by NS_stage into dst (its space). */
int af_compute_diagonal(af_operator* op, double* inv_diag);

/* A^{-1} inside the Schur apply: mode 0 = CG + Jacobi to rel_tol (the reference:
 * SolverControl(10000, 1e-12 |B p|), euler_operator.h:2391-2397; the default, with rel_tol
 * 1e-12 and max_iter 10000); mode 1 = exact cell-wise inverse (A is block diagonal for DG:
 * per-cell inverses), which replaces the nested CG. */
int af_set_schur_mode(af_operator* op, int mode, double rel_tol, int max_iter);
/* iterations of the last inner A^{-1} solve */
int af_last_inner_iterations(const af_operator* op, int* its);

/* Number of DoFs of a space (0 velocity, 1 pressure, 2 density): MatrixFree::initialize_dof_vector */
int af_n_dofs(const af_operator* op, int space, long long* n);
/* Number of kernels this library launched on the handle since creation. */
int af_launch_count(const af_operator* op, long long* n);

/* Rayleigh damping of the momentum towards (u_ref, 0), added to the explicit momentum rhs of
 * every stage with the stage's explicit weights: -dt sum_j a_j tau rho_j (u_j - u_ref), with
 * tau(x, z) = rate_top sin^2(pi/2 (z - z_start)/(z_top - z_start)) above z_start (an upper
 * sponge) plus rate_lateral cos^2(pi/2 d/width_lateral) within width_lateral of the nearer of
 * x_left and x_right (relaxation zones; d the distance).  Rates in 1/s of the non-dimensional
 * units; both 0 (the default) switch it off.  No counterpart in the reference: the damping
 * layers of the 2D hill configuration.  The stage-1 tangent and adjoint kernels have no sponge
 * term (AF_UNSUPPORTED while it is on). */
int af_set_sponge(af_operator* op, double z_start, double z_top, double rate_top, double x_left, double x_right,
                  double width_lateral, double rate_lateral, double u_ref);

/* Failure detection (no counterpart in the reference, whose deal.II loops have no waits):
 * the cell kernels wait for their bulk copies with a bounded number of polls.  A kernel that
 * gives up leaves a code in the handle's status word and returns without writing its
 * outputs; the next call on the handle (any call that queues work, af_synchronize, and every
 * call that synchronizes internally: solves, IMEX steps, host-buffer applies, diagnostics)
 * then returns AF_TIMEOUT once and clears the word.
 * Test hook: polls > 0 makes every cell kernel of this handle first wait on a barrier phase
 * that nothing completes and give up after that many polls, before it issues any copy (the
 * timeout path without copies in flight); 0 restores normal operation. */
int af_set_stage_wait_test(af_operator* op, int polls);

/* ---------------------------------------------------------------- Schur pressure solver
 * Solves the NS_stage-2 system (D - C A^{-1} B) p = b of af_vmult, the linear solve of the
 * reference's pressure_fixed_point (Atmospheric_Flow.cc:544-673: SolverGMRES + Jacobi on the
 * diagonal of D, euler_operator.h:2607-2611), by flexible GMRES in FP64 (right
 * preconditioning; converged when the TRUE residual |b - S x| <= rel_tol |b|).  The
 * preconditioner is Jacobi on diag(D) or a geometric h-multigrid V-cycle (the role of the
 * reference's MGLevelObject / MGTransferMatrixFree / PreconditionChebyshev stack,
 * Atmospheric_Flow.cc:455-522, which the reference applies to the mass-type systems only):
 * 2:1 coarsened meshes of the same degree, the linearised Schur operator (C without its
 * wave-speed term) on every level, Chebyshev smoothing on D^{-1} S with the exact cell-wise
 * D^{-1}, transfer by polynomial embedding and its transpose, a Chebyshev coarse solve.  Its
 * levels run in FP64 (AF_SCHUR_MG_FP64) or FP32 (AF_SCHUR_MG_FP32).  AF_SCHUR_CHEB_FP64 /
 * _FP32 is the single-level case: a Chebyshev polynomial of degree poly_degree in D^{-1} S
 * over its whole spectrum [0.9, 1.2 lmax] (no coarse levels).
 * The solver uses the operator's stream and its rho_for_fixed / pres_fixed / dt / Mach /
 * HYPERBOLIC_stage at af_schur_solver_setup time; af_schur_solve sets NS_stage 2. */
typedef struct af_schur_solver af_schur_solver;
enum { AF_SCHUR_JACOBI = 0, AF_SCHUR_MG_FP64 = 1, AF_SCHUR_MG_FP32 = 2, AF_SCHUR_CHEB_FP64 = 3, AF_SCHUR_CHEB_FP32 = 4 };
typedef struct {
  int preconditioner;       /* AF_SCHUR_* (default AF_SCHUR_CHEB_FP32)                        */
  int smoother_degree;      /* Chebyshev degree of each pre/post smoothing (5)                 */
  double smoothing_range;   /* the smoother targets [lmax/range, lmax] (15)                    */
  int coarse_degree;        /* Chebyshev degree of the coarse solve (10)                       */
  int max_levels;           /* 0: coarsen while nx, nz are even and cells > min_coarse_cells  */
  int min_coarse_cells;     /* 16                                                              */
  int eig_iterations;       /* power iterations of the per-level lmax estimate (20)            */
  int restart;              /* FGMRES directions per cycle, 1..64 (30)                         */
  double coarse_lmax;       /* the first level with lmax <= this is the coarsest (25)          */
  int poly_degree;          /* degree of the AF_SCHUR_CHEB_* polynomial preconditioner (16)    */
  int reduced_quadrature;   /* FP32 levels: B, C0 with P+1 Gauss points per direction instead  */
                            /* of 2P+1 (exact for B and D on bilinear cells, approximate for   */
                            /* C0 and A; the outer FGMRES keeps the exact operator): 1; 2: the */
                            /* same, and AF_SCHUR_CHEB_FP32 iterates in the basis of the       */
                            /* Lagrange polynomials of those Gauss points, where the cell      */
                            /* inverses are diagonal (the same polynomial; multigrid levels    */
                            /* stay nodal); 0: 2P+1 points (2)                                 */
} af_schur_options;
typedef struct {
  int iterations;           /* FGMRES iterations of the last solve                             */
  double initial_residual;  /* |b - S x0|                                                      */
  double final_residual;    /* |b - S x| (Arnoldi estimate when it stopped inside a cycle)     */
  double seconds;           /* device time of the last solve (CUDA events on the stream)       */
} af_schur_stats;
int af_schur_default_options(af_schur_options* opt);
int af_schur_solver_create(af_operator* op, const af_schur_options* opt, af_schur_solver** out);
int af_schur_solver_destroy(af_schur_solver* s);
/* Rebuilds the level coefficients and cell inverses from the operator's current state;
 * the per-level eigenvalue estimate runs on the first setup or when estimate_eigenvalues. */
int af_schur_solver_setup(af_schur_solver* s, int estimate_eigenvalues);
int af_schur_solver_levels(const af_schur_solver* s, int* n_levels, double* lmax);
/* dst = one application of the preconditioner to src (DEVICE pointers, pressure space). */
int af_schur_solver_precondition(af_schur_solver* s, double* dst, const double* src);
/* x (initial guess in, solution out) for S x = b; returns AF_NO_CONVERGENCE at the cap. */
int af_schur_solve(af_schur_solver* s, double* x, const double* b, double rel_tol, int max_iterations,
                   af_schur_stats* stats);
/* Adjoint pressure solve (no counterpart in the reference): J_S(p)^T x = b, J_S(p) the Jacobian
 * of the Schur apply at p (see af_schur_transpose), same FGMRES and preconditioner. */
int af_schur_solve_transpose(af_schur_solver* s, const double* p, double* x, const double* b, double rel_tol,
                             int max_iterations, af_schur_stats* stats);
/* Tangent pressure solve (no counterpart in the reference): J_S(p) x = b, same FGMRES and
 * preconditioner; the tangent-linear counterpart of af_schur_solve_transpose. */
int af_schur_solve_tangent(af_schur_solver* s, const double* p, double* x, const double* b, double rel_tol,
                           int max_iterations, af_schur_stats* stats);

/* ---------------------------------------------------------------- IMEX time stepping
 * One IMEX-DG step of the reference's EulerSolver::run (Atmospheric_Flow.cc:1110-1251):
 * update_density, the pressure fixed point (pressure_fixed_point + update_velocity, at most
 * fixed_point_max_iterations, |p - p_old|_inf / (|p|_inf + 1e-10) < fixed_point_tol) for
 * stages 1 and 2, then update_density, update_velocity and update_pressure for stage 3.
 * Outer solves stop at eps*|rhs| (SolverControl(max_its, eps*rhs.l2_norm())); the Schur
 * system uses GMRES with left Jacobi preconditioning restarted after gmres_restart
 * directions; the inner A^{-1} of pressure_fixed_point stops at 1e-12 |rhs_u|. */
typedef struct af_imex af_imex;
typedef struct {
  double eps;                      /* parameter-file.prm "eps" (default 1e-8)            */
  int max_iterations;              /* parameter-file.prm "max_iterations" (30000)        */
  double fixed_point_tol;          /* 1e-10                                               */
  int fixed_point_max_iterations;  /* 100                                                 */
  int gmres_restart;               /* 28 (deal.II SolverGMRES default)                     */
  int mass_solver;                 /* 0: CG + Jacobi to eps; 1: exact cell-wise inverse (default) */
  int schur_inner;                 /* A^{-1} in the Schur apply: 0 nested CG; 1 exact (default)   */
  int schur_preconditioner;        /* -1: the reference's GMRES + left Jacobi (default);
                                      AF_SCHUR_*: af_schur_solve (FGMRES, true residual <= eps |rhs_p|,
                                      preconditioner rebuilt once per stage) */
  int schur_poly_degree;           /* AF_SCHUR_CHEB_*: polynomial degree (0: 20)                 */
} af_imex_options;
typedef struct {
  int fixed_point_iterations[2];   /* stage 1, stage 2 of the last step                   */
  long long gmres_iterations;      /* summed over the last step                           */
  long long cg_iterations;
  double last_fixed_point_error;
} af_imex_stats;
int af_imex_default_options(af_imex_options* opt);
/* Creates its own operator handle (degree p, QGauss(2p+1)) and all stage vectors. */
int af_imex_create(const af_mesh_desc* mesh, int degree, double Mach, double Froude, double dt,
                   const af_imex_options* opt, af_imex** out);
int af_imex_destroy(af_imex* h);
/* The operator handle used by the stepper (e.g. for af_set_stream). */
af_operator* af_imex_operator(af_imex* h);
/* State (rho, u, p) at the start of the next step; DEVICE pointers, copied. */
int af_imex_set_state(af_imex* h, const double* rho, const double* u, const double* p);
int af_imex_get_state(const af_imex* h, double* rho, double* u, double* p);
int af_imex_step(af_imex* h, int nsteps);
int af_imex_last_stats(const af_imex* h, af_imex_stats* stats);
/* Tangent-linear and adjoint of IMEX stage 1 (no counterpart in the reference): the map
 * (rho0, u0, p0) -> (rho_tmp_2, u_tmp_2, p_tmp_2) of the density update and the pressure fixed
 * point (Atmospheric_Flow.cc:1116-1156).
 *   af_imex_stage1_forward:  runs stage 1 from the given state (it also becomes the handle's
 *                            state) and records the fixed-point trajectory;
 *   af_imex_stage1_tangent:  (drho2, du2, dp2) = J (drho0, du0, dp0);
 *   af_imex_stage1_backward: (rho0bar, u0bar, p0bar) = J^T (rho2bar, u2bar, p2bar);
 * J differentiates the recorded iterations, each Schur solve taken as exact (solved to
 * rel_tol with the handle's FGMRES and preconditioner: af_schur_solve_tangent / _transpose;
 * the cell-wise A and M solves are exact).  Needs schur_preconditioner >= 0; af_imex_step
 * drops the recorded linearisation point.  All vectors are device arrays. */
int af_imex_stage1_forward(af_imex* h, const double* rho0, const double* u0, const double* p0, double* rho2, double* u2,
                           double* p2);
int af_imex_stage1_tangent(af_imex* h, const double* drho0, const double* du0, const double* dp0, double* drho2,
                           double* du2, double* dp2, double rel_tol);
int af_imex_stage1_backward(af_imex* h, const double* rho2bar, const double* u2bar, const double* p2bar,
                            double* rho0bar, double* u0bar, double* p0bar, double rel_tol);
/* The same for one whole IMEX step (stages 1-3, no counterpart in the reference):
 * (rho0, u0, p0) -> (rho1, u1, p1) = the state after af_imex_step(h, 1) from (rho0, u0, p0);
 * the forward records both fixed points and leaves (rho1, u1, p1) as the handle's state. */
int af_imex_step_forward(af_imex* h, const double* rho0, const double* u0, const double* p0, double* rho1, double* u1,
                         double* p1);
int af_imex_step_tangent(af_imex* h, const double* drho0, const double* du0, const double* dp0, double* drho1,
                         double* du1, double* dp1, double rel_tol);
int af_imex_step_backward(af_imex* h, const double* rho1bar, const double* u1bar, const double* p1bar,
                          double* rho0bar, double* u0bar, double* p0bar, double rel_tol);
/* Gradient through nsteps IMEX steps with checkpointed recomputation (no counterpart in the
 * reference): (rho0bar, u0bar, p0bar) = (d state_N / d state_0)^T (rhobar, ubar, pbar), the
 * cotangent of a functional of the final state pulled back to the initial state.  The forward
 * sweep keeps one state every checkpoint_every steps; the reverse sweep recomputes each segment
 * from its checkpoint and runs af_imex_step_backward step by step (device memory:
 * ceil(nsteps / checkpoint_every) + checkpoint_every + 2 states).  The handle's state is
 * overwritten. */
int af_imex_gradient(af_imex* h, const double* rho0, const double* u0, const double* p0, int nsteps,
                     int checkpoint_every, const double* rhobar, const double* ubar, const double* pbar,
                     double* rho0bar, double* u0bar, double* p0bar, double rel_tol);

/* The Schur complement apply D p - C A^{-1} B p of af_vmult (NS_stage 2) for callers that
 * must not allocate device memory (e.g. code inside a framework whose caching allocator owns
 * the device memory, or a time loop that budgets memory up front).  No counterpart in the
 * reference.  It needs no handle: the mesh vertices ((nz+1)*(nx+1)*2 doubles), rho_for_fixed,
 * pres_fixed, src and dst are DEVICE pointers owned by the caller, and all scratch lives in a
 * static device array of the library (about 7.4 MB per GPU, held until exit) that limits the
 * problem to nx*nz*(degree+1)^2 <= 65536 pressure DoFs (larger sizes return AF_BAD_ARG).  The
 * first call on a device sets the array up (cudaGetSymbolAddress, basis tables); calls that
 * overlap on the GPU share the array and race.  stream may be NULL (default stream). */
int af_schur_apply_noalloc(int nx, int nz, int periodic_x, const double* vertices, int degree, double Mach, double dt,
                           int hyperbolic_stage, const double* rho_for_fixed, const double* pres_fixed,
                           const double* src, double* dst, void* stream, int* inner_iterations);

/* ---------------------------------------------------------------- diagnostics
 * The reference's time-loop diagnostics (Atmospheric_Flow.cc:991-1087, 1224-1235), which it
 * evaluates at QGaussLobatto(p+1) = the DG support points: max |u| (get_max_velocity),
 * min / max density (get_min_density / get_max_density, taken from the current stage's
 * density: pass it as rho_stage, or NULL to use rho), max sqrt(gamma p / rho)
 * (compute_max_celerity, from rho and p), the minimal cell diameter (longer diagonal of the
 * mapped cell, GridTools::minimal_cell_diameter) and the Courant numbers
 * CFL_c = dt max_celerity / Ma * degree sqrt(2) / d_min, CFL_u = dt max|u| degree sqrt(2) / d_min.
 * DEVICE vectors; synchronises the operator's stream. */
typedef struct {
  double max_velocity, min_density, max_density, max_celerity, min_cell_diameter, cfl_c, cfl_u;
} af_diagnostics;
int af_compute_diagnostics(af_operator* op, const double* rho, const double* rho_stage, const double* u,
                           const double* p, af_diagnostics* out);
/* L2 norm over the mesh of a DEVICE field with ncomp (1 or 2) components per cell, by
 * QGauss(p+1) as the reference's integrate_difference(..., L2_norm) in analyze_results
 * (Atmospheric_Flow.cc:925-985); the difference to a reference field is the caller's. */
int af_l2_norm(af_operator* op, int ncomp, const double* v, double* norm);

/* ---------------------------------------------------------------- state files and VTU output
 * HOST arrays; no GPU needed.  af_io_write_vtu writes what the reference's output_results
 * (Atmospheric_Flow.cc:886-918) writes in 2D: each cell subdivided into degree x degree
 * quadrilaterals at equispaced reference points (DataOut::build_patches with n_subdivisions =
 * degree), fields rho, u, p interpolated there, ASCII .vtu.  af_io_write_state /
 * af_io_read_state: a binary restart file (mesh, degree, time, step, rho, u, p) with no
 * counterpart in the reference (it has no restart). */
typedef struct {
  int nx, nz, degree, periodic_x, gravity;
  double radial_a, time;
  long long step;
} af_state_header;
int af_io_write_state(const char* path, const af_mesh_desc* mesh, int degree, double time, long long step,
                      const double* rho, const double* u, const double* p);
int af_io_read_state_header(const char* path, af_state_header* header);
/* vertices: (nz+1)(nx+1)2, rho and p: n, u: 2n doubles, n = nx nz (degree+1)^2 */
int af_io_read_state(const char* path, double* vertices, double* rho, double* u, double* p);
int af_io_write_vtu(const char* path, const af_mesh_desc* mesh, int degree, const double* rho, const double* u,
                    const double* p);

/* ---------------------------------------------------------------- tangents and transposes
 * of the implicit operators (no counterpart in the reference; the pieces of an adjoint IMEX
 * stage).  DEVICE vectors; the operator's HYPERBOLIC_stage coefficient, dt, Mach,
 * rho_for_fixed and pres_fixed as in the forward.  C is nonlinear in w through the wave
 * speed lambda(w); its Jacobian differentiates lambda along the branch the forward takes.
 *   af_vmult_pressure_transpose:  pbar = B^T ubar
 *   af_vmult_enthalpy_tangent:    dst = J_C(w) dw
 *   af_vmult_enthalpy_transpose:  wbar = J_C(w)^T pbar
 *   af_schur_tangent:             dst = J_S(p) dp = D dp - J_C(w) A^{-1} B dp,  w = A^{-1} B p
 *   af_schur_transpose:           dst = J_S(p)^T pbar = D pbar - B^T A^{-1} J_C(w)^T pbar
 * (A^{-1}: the exact cell-wise inverse.) */
int af_vmult_pressure_transpose(af_operator* op, double* pbar, const double* ubar);
int af_vmult_enthalpy_tangent(af_operator* op, double* dst, const double* w, const double* dw);
int af_vmult_enthalpy_transpose(af_operator* op, double* wbar, const double* w, const double* pbar);
int af_schur_tangent(af_operator* op, double* dst, const double* p, const double* dp);
int af_schur_transpose(af_operator* op, double* dst, const double* p, const double* pbar);
/* Coefficient derivatives of the implicit operators, transposed (no counterpart in the
 * reference; building blocks of the IMEX-stage adjoint).  A (NS 3/5) is linear in
 * rho_for_fixed and C (vmult_enthalpy) in pres_fixed, so their tangents are the operators
 * applied with the perturbation as the coefficient; the transposes are
 *   af_vmult_velocity_mass_rho_transpose:  rhobar = (d/drho [A(rho) x])^T y = int psi (x . y)
 *   af_vmult_enthalpy_pf_transpose:        pfbar = (d/dp_f [C(w; p_f)])^T pbar
 * (the HYPERBOLIC_stage coefficient of C as in af_vmult_enthalpy). */
int af_vmult_velocity_mass_rho_transpose(af_operator* op, double* rhobar, const double* x, const double* y);
int af_vmult_enthalpy_pf_transpose(af_operator* op, double* pfbar, const double* w, const double* pbar);

/* Measures the FP64 FMA throughput of the current device (TFLOP/s) with a short
 * dependent-chain kernel; the denominator of the FP64 roofline the benchmark reports.
 * No counterpart in the reference. */
int af_measure_fp64_peak(double* tflops);

const char* af_error_string(int status);
const char* af_last_error_message(void);

#ifdef __cplusplus
}
#endif

#endif /* AF_GPU_H */
