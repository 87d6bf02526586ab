/*
 * nodals_b200 -- C ABI of the B200 steady P1+BF3/P0 SIMPLE solver.
 *
 * The reference (JD63021/NodalS, gpu/serial_cuda) exposes no library API:
 * its drop-in surface is the process boundary of nodals_gpu_h8_{fp32,fp64}
 * (argv flags gpu/serial_cuda/h8_main_base.cu:1787-1911, NODALS_GPU_* stdout
 * markers, exit codes 0/35/90 at :2202-2203, --vtu-out files).  This header
 * is the layer underneath the drop-in executable of this package; each entry
 * point names the reference step it replaces.
 *
 * Conventions
 *  - every call returns an int status: NDS_OK (0) or a negative NDS_E_* code;
 *    nds_last_error() gives the message of the calling thread's last failure;
 *  - nothing throws across this boundary and nothing aborts the process;
 *  - the caller owns all host arrays passed in or out; the library owns all
 *    device memory;
 *  - one solver handle per thread; a handle is not internally synchronised;
 *  - the GPU solver entry points fail loudly (NDS_E_CUDA) when no CUDA
 *    device or kernel image is available: there is no CPU fallback.
 */
#ifndef NODALS_B200_H
#define NODALS_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define NDS_OK 0
#define NDS_E_INVALID (-1)      /* bad argument / option (reference: "H8 usage error") */
#define NDS_E_SETUP (-2)        /* mesh or setup failure (reference: std::runtime_error during setup) */
#define NDS_E_CUDA (-3)         /* CUDA runtime failure or no device */
#define NDS_E_BREAKDOWN (-4)    /* Krylov breakdown / non-finite value (reference throws, h8_main_base.cu:570-572) */
#define NDS_E_NOT_CONVERGED (-5)/* pressure solve missed its target within p_max (h8_main_base.cu:2101) */
#define NDS_E_STATE (-6)        /* call out of order */

typedef struct nds_mesh nds_mesh;
typedef struct nds_problem nds_problem;
typedef struct nds_solver nds_solver;

/* NDS_FP64 / NDS_FP32: the reference's two builds (NODALS_GPU_PRECISION_MODE
 * 0 / 1, gpu/serial_cuda/h8_main.cu).  NDS_AMG_FP32 has no reference build:
 * state, momentum, continuity and the Krylov method (including its A*p) stay
 * FP64 while the AMG V-cycle -- levels, transfers, smoothers and an FP32 copy
 * of the fine Schur operator written by the same refresh -- runs in FP32.
 * NDS_MIXED has no reference build either: state, momentum, continuity and
 * the outer residual of an FP64 defect-correction loop around each pressure
 * solve stay FP64; each inner solve (PCG or FGMRES, options p_krylov ...)
 * runs in FP32 on the FP32 operator copy with the FP32 V-cycle, with FP64
 * reductions, FGMRES Gram-Schmidt and Hessenberg least squares.  The
 * pressure solve meets the same FP64 target max(p_atol, p_rtol ||b||). */
enum nds_precision { NDS_FP64 = 0, NDS_FP32 = 1, NDS_AMG_FP32 = 2, NDS_MIXED = 3 };
/* inner Krylov method of NDS_MIXED */
enum nds_krylov { NDS_KRYLOV_PCG = 0, NDS_KRYLOV_FGMRES = 1 };
enum nds_run_mode { NDS_RUN_FIXED10 = 0, NDS_RUN_CONVERGE = 1 };
enum nds_momentum_work { NDS_MOM_FGS1 = 0, NDS_MOM_ALTGS1 = 1, NDS_MOM_SGS1 = 2 };
enum nds_pressure_solver { NDS_P_PCG = 0, NDS_P_RICHARDSON = 1, NDS_P_CHEB = 2 };
enum nds_amg_hierarchy { NDS_AMG_SA = 0, NDS_AMG_CF = 1 };
enum nds_amg_smoother { NDS_SM_CHEB2 = 0, NDS_SM_JACOBI = 1, NDS_SM_L1JACOBI = 2, NDS_SM_MCGS = 3 };
enum nds_spectrum_policy { NDS_SPEC_AUTO = 0, NDS_SPEC_ALWAYS = 1, NDS_SPEC_OFF = 2 };
enum nds_mcgs_order { NDS_MCGS_SYMMETRIC = 0, NDS_MCGS_FORWARD = 1, NDS_MCGS_BACKWARD = 2 };
enum nds_cf_interp { NDS_CF_DIRECT = 0, NDS_CF_EXTI = 1 };

/* All H8 CLI controls (h8_main_base.cu:1749-1850); nds_options_default()
 * fills the binary's own defaults. */
typedef struct nds_options {
  double re, bulk, simple_tol, alpha_u, alpha_p, rau_scale;
  int max_outer, run_mode, momentum_work;
  double mom_omega, mom_rtol, mom_atol, mom_drop;
  int mom_max;
  int pressure_solver;
  double p_rtol, p_atol;
  int p_max;
  double snapshot_tol;
  int fine_csr_refresh_every;
  double p_richardson_omega;
  int p_cheb_degree, p_power_its;
  double p_cheb_low_fraction, p_power_safety;
  int amg_hierarchy, amg_smoother, amg_terminal, amg_spectrum_policy;
  int amg_power_its, amg_cheb_degree;
  double amg_lambda_safety, amg_lambda_low_fraction, amg_jacobi_omega;
  int amg_jacobi_fine_sweeps, amg_jacobi_coarse_sweeps;
  double amg_mcgs_omega;
  int amg_mcgs_fine_sweeps, amg_mcgs_coarse_sweeps, amg_mcgs_order;
  double cf_theta;
  int cf_pmax, cf_interp, cf_aggressive_first;
  char wall[64], inlet[64], outlet[64];
  int precision;   /* enum nds_precision */
  int threads;     /* host threads for setup; 0 = all */
  int device;      /* CUDA device ordinal */
  int verbose;     /* 1: print the reference's NODALS_GPU_* markers to stdout */
  /* laminar SUPG stabilisation of the momentum operator, implicit form with
   * the 64-point collapsed rule (h8_supg_main_cli.inc, h7_momentum_assembly.cuh:100-226) */
  int supg;
  double supg_tau_scale, supg_magic;
  /* pressure solve of NDS_MIXED (no reference counterpart; ignored by the
   * other precisions).  p_max caps the inner iterations of one solve. */
  int p_krylov;          /* enum nds_krylov (default PCG) */
  int p_restart;         /* FGMRES basis vectors per pass, 1..64 (default 30) */
  double p_inner_rtol;   /* relative target of one FP32 inner pass (default 1e-3) */
  int p_refine_max;      /* FP64 defect-correction passes per solve (default 8) */
  int p_guess;           /* earlier corrections spanning a Galerkin initial guess, 0..8 (0: zero guess) */
  int learned;           /* 1: learned stage ahead of the V-cycle (FGMRES only; nds_solver_load_stage) */
  /* 1: pipe centre and radius from the inlet patch instead of the bounding
   * box (bent pipes); 0: the reference's bounding-box rule (g4_host.hpp:37-49) */
  int geom_from_inlet;
  /* products A y of the guess: 0 kept from the solve that made each y
   * (w = b - r, free, from an operator up to p_guess iterations old), 1
   * recomputed with the current FP32 operator copy every solve */
  int p_guess_fresh;
  /* 1: the V-cycle's fine-level operator in FP16 (values scaled by a power of
   * two into FP16 range, FP32 arithmetic); precision mixed only -- the
   * inner Krylov product keeps the FP32 copy, the outer residual FP64 */
  int amg_half;
} nds_options;

/* One SIMPLE outer iteration (h8_main_base.cu:2046-2119). */
typedef struct nds_iter_report {
  int it;
  double rel_cont;          /* ||B u + fixedDiv|| / same at it = 1 */
  double cont_norm;
  int p_its;
  double p_rel;
  int audited;              /* pre-sweep momentum audit performed this iteration */
  double audit_rel[3];
  int all_momentum_met;
  int converged;
  double ms_assembly, ms_momentum, ms_continuity, ms_pressure, ms_update;
  double ms_refresh;        /* the part of the fine Schur refresh (run beside the momentum
                               sweep and continuity) still pending when the pressure stage
                               starts; the first part of ms_pressure */
} nds_iter_report;

typedef struct nds_solve_report {
  int outer_its;
  int converged;
  int pressure_all;         /* every pressure solve met its target */
  int finite_all;
  double final_rel_cont;
  double final_audit_rel[3];
  double avg_pressure_its;
  double loop_ms;           /* device-timed loop */
  double assembly_ms, momentum_ms, continuity_ms, pressure_ms, update_ms;
} nds_solve_report;

/* Host array view of a named setup array (read-only, owned by the problem). */
typedef struct nds_array {
  const void* data;
  int64_t count;
  int dtype;                /* 0 f64, 1 i32, 2 i64, 3 u8, 4 u32 */
} nds_array;

const char* nds_last_error(void);
const char* nds_version(void);
void nds_options_default(nds_options* o);

/* ---- meshes: replace load_foam_tet_mesh (foam_mesh_g2.hpp:55) ---------- */
int nds_mesh_read_polymesh(const char* polymesh_dir, nds_mesh** out);
int nds_mesh_read_msh2(const char* path, nds_mesh** out);
/* binary HXT1 mesh (hybrid_hxt1/hxt1_mesh.hpp:19-103, as written by the
 * reference's turbulence/sst_gpu_v2/tools/msh2_to_hxt1.py): files without
 * hex cells; inlet/outlet from the tet boundary records, every other
 * exterior face wall */
int nds_mesh_read_hxt1(const char* path, nds_mesh** out);
int nds_mesh_from_arrays(int n_points, const double* xyz, int n_cells, const int32_t* tets, int n_bfaces,
                         const int32_t* btri, const int32_t* bpatch, int n_patches, const char* const* patch_names,
                         nds_mesh** out);
int nds_mesh_counts(const nds_mesh* m, int* n_points, int* n_cells, int* n_faces, int* n_internal);
void nds_mesh_destroy(nds_mesh* m);

/* ---- host setup: replaces build_g4_setup (g4_host.hpp:289),
 *      build_h2_fine_csr_host (h2b_fine_csr.cuh:445) and
 *      build_sa_hierarchy / build_cf_hierarchy (g5_sa_host.hpp:1545,
 *      g8_cf_hierarchy_host.hpp:1584) ------------------------------------- */
int nds_problem_create(const nds_mesh* m, const nds_options* o, nds_problem** out);
int nds_problem_array(const nds_problem* p, const char* name, nds_array* out);
int nds_problem_counts(const nds_problem* p, int* nc, int* nv, int* ncolors, int* levels);
void nds_problem_destroy(nds_problem* p);

/* ---- output surface: replaces h12_write_vtu (h12_vtu_output.hpp:26-94),
 *      h8_compute_hp_errors (h8_hp_diagnostics.inc:18-100) and
 *      pressure_drop_fit_g4 (g4_host.hpp:424).  Fields are the solver's
 *      free-DOF vectors (nv velocity values per component, nc pressures). */
typedef struct nds_hp_errors {
  double h_eff, u_l2, u_rel_l2, p_shifted_l2, p_shifted_rel_l2, pressure_shift;
  double dp_fit, dp_exact, dp_rel_err;
} nds_hp_errors;
int nds_write_vtu(const nds_problem* p, const char* path, const double* u0, const double* u1, const double* u2,
                  const double* pr, int converged, int outer_its);
int nds_compute_hp_errors(const nds_problem* p, const double* u0, const double* u1, const double* u2, const double* pr,
                          nds_hp_errors* out);
int nds_cell_average_velocity(const nds_problem* p, const double* u0, const double* u1, const double* u2,
                              double* out_xyz /* 3 * nc */);

/* ---- device solver: replaces upload_all (h8_main_base.cu:761-788), the
 *      setup policies (:1984-2025) and the SIMPLE loop (:2046-2119) ------- */
int nds_solver_create(const nds_problem* p, nds_solver** out);
int nds_solver_reset(nds_solver* s);                         /* u = p = 0, it = 0 */
int nds_simple_step(nds_solver* s, nds_iter_report* rep);
int nds_solve(nds_solver* s, nds_solve_report* rep);         /* the run_mode loop */
int nds_get_fields(nds_solver* s, double* u0, double* u1, double* u2, double* p);
int nds_set_fields(nds_solver* s, const double* u0, const double* u1, const double* u2, const double* p);
/* One SIMPLE iteration whose state goes through host memory (no reference
 * counterpart: the reference keeps the state on the device for the whole
 * loop).  Same result as nds_set_fields(in) + nds_simple_step +
 * nds_get_fields(out); any input or output pointer may be NULL (that field
 * is kept / not read back), and an input may alias an output.  With an FP64
 * state and page-locked outputs (cudaMallocHost / cudaHostRegister) the
 * velocity read-back runs under the pressure solve instead of after it.
 * Returns once every copy into the outputs has finished; after a failure
 * their contents are unspecified. */
int nds_simple_step_io(nds_solver* s, const double* u0_in, const double* u1_in, const double* u2_in,
                       const double* p_in, double* u0_out, double* u1_out, double* u2_out, double* p_out,
                       nds_iter_report* rep);
void nds_solver_destroy(nds_solver* s);

/* ---- kernel timing by category with CUDA events on the solver's stream
 *      (replaces the reference's H0Profiler, h8_main_base.cu:58-99) -------- */
typedef struct nds_profile_entry {
  char name[32];
  long long calls;
  double total_ms;
} nds_profile_entry;
int nds_profile_enable(nds_solver* s, int on);   /* resets the counters */
int nds_profile_read(nds_solver* s, nds_profile_entry* out, int max_entries, int* n_out);
/* number of kernels this library has launched in this process */
unsigned long long nds_launch_count(void);

/* ---- allocation-free continuity residual (no counterpart in the
 *      reference).
 * For callers that must not allocate device memory: code that runs between
 * the steps of its own captured or real-time loop, or under an allocator
 * that forbids cudaMalloc once it has started.  u0..u2 (nv doubles each),
 * r (nc doubles) and norm (1 double) are caller-owned DEVICE pointers on the
 * solver's device; stream is a cudaStream_t (NULL: the legacy default
 * stream).  Enqueues r = -(B u + fixedDiv) and *norm = ||B u + fixedDiv||_2,
 * the quantity nds_simple_step reports as cont_norm, and returns without
 * synchronising.  Needs a solver whose state is FP64 (precision fp64,
 * amg_fp32 or mixed); any mesh size and any device ordinal the solver runs
 * on.  Makes no cudaMalloc/cudaFree or other allocating call: the block
 * partial sums live in a 16 KiB device array of the library (at most 1184
 * blocks, whatever the mesh size), held on every device that loads the
 * library until the process exits.  Each call looks that array's address up
 * (cudaGetSymbolAddress, which allocates nothing) with the solver's device
 * current.  Calls that overlap in time on one device race on the array, and
 * so do calls overlapping an nds_simple_step of the same solver.  Launches
 * are checked with cudaPeekAtLastError, so an error still pending from the
 * caller's own earlier CUDA work is reported as NDS_E_CUDA too (and left
 * pending).  Failures return a status only: nds_last_error() is not
 * updated. */
int nds_continuity_noalloc(nds_solver* s, const double* u0, const double* u1, const double* u2, double* r,
                           double* norm, void* stream);

/* ---- learned pressure stage (no counterpart in the reference) ----------
 * A message-passing network on the face graph of the pressure cells (3
 * layers of width 64, BF16 weights, tcgen05 tensor-core GEMMs with FP32
 * accumulation) that maps a pressure-correction residual v to an
 * approximate correction z.  With options learned = 1 (precision mixed,
 * p_krylov fgmres) it is a flexible-preconditioner stage ahead of the AMG
 * V-cycle: z = N(v) + V(v - A N(v)), or the plain V(v) whenever the stage
 * does not reduce the residual (||v - A N(v)|| >= ||v||).
 * The graph: n nodes, nbr[4 n] face neighbours (-1: boundary face), ew[4 n]
 * edge weights a_ij / sqrt(a_ii a_jj) of the Jacobi-scaled pressure
 * operator, dscale[n] = 1 / sqrt(a_ii); device pointers.  Parameter vector
 * (FP32, NDS_MPNN_NPARAM values): We[64][2], be[64], then for l = 1..3
 * W_l[64][128] (out x in, input [h ; sum_j e_ij h_j]), b_l[64], then
 * wd[64], bd, cs (out = wd . h3 + bd + cs s). */
#define NDS_MPNN_NPARAM 25026
typedef struct nds_mpnn_graph {
  int n;
  const int32_t* nbr;
  const float* ew;
  const float* dscale;
} nds_mpnn_graph;
typedef struct nds_mpnn nds_mpnn;
int nds_mpnn_param_count(void);
/* device state for graphs of up to n_max nodes; training = 1 keeps the
 * activations, gradients and Adam moments */
int nds_mpnn_create(int n_max, int training, int device, nds_mpnn** out);
int nds_mpnn_set_params(nds_mpnn* m, const float* host_params, int count);
int nds_mpnn_get_params(nds_mpnn* m, float* host_params, int count);
/* z = N(v) (device pointers); the graph may hold nseg independent segments
 * (seg_off[0..nseg] host offsets, each normalised on its own; nseg = 0: one) */
int nds_mpnn_forward(nds_mpnn* m, const nds_mpnn_graph* g, int nseg, const int32_t* seg_off, const float* v,
                     float* z);
/* forward, loss and backward for pairs (v, x) of right-hand sides and
 * solutions: loss = mean over segments of sum_i (out_i - t_i)^2 / sum_i t_i^2,
 * t_i = x_i / (dscale_i sigma_s); gradients kept for nds_mpnn_get_grads and
 * nds_mpnn_adam_step */
int nds_mpnn_loss_backward(nds_mpnn* m, const nds_mpnn_graph* g, int nseg, const int32_t* seg_off, const float* v,
                           const float* x, double* loss);
/* gradients from dL/dz (device, n values) of the last nds_mpnn_forward on
 * the same graph (training handle): for losses computed outside, e.g. on the
 * residual b - A z with the solver's operator */
int nds_mpnn_backward(nds_mpnn* m, const nds_mpnn_graph* g, const float* dz);
int nds_mpnn_get_grads(nds_mpnn* m, float* host_grads, int count);
int nds_mpnn_adam_step(nds_mpnn* m, float lr, float beta1, float beta2, float eps, int step);
/* BF16 activations h^layer (n_max x 64, row-major) into a device buffer */
int nds_mpnn_activations(nds_mpnn* m, int layer, void* out_dev);
void nds_mpnn_destroy(nds_mpnn* m);
/* the solver's side of the stage: load its parameters (host array); copy the
 * current graph (face neighbours, edge weights and scaling from the operator
 * of the last refresh) into device arrays of nc (4 nc) entries; copy the
 * last pressure solve's right-hand side and solution as FP32 (device arrays
 * of nc entries) -- the training pairs */
int nds_solver_load_stage(nds_solver* s, const float* host_params, int count);
int nds_solver_stage_graph(nds_solver* s, int32_t* nbr, float* ew, float* dscale);
int nds_solver_pressure_pair(nds_solver* s, float* rhs, float* x);
/* y = A x with the solver's current pressure operator in FP32 (device
 * arrays of nc values; precision mixed) */
int nds_solver_apply_operator(nds_solver* s, const float* x, float* y);
/* counters of the learned stage since the solver was created: applications
 * and fallbacks to the plain V-cycle */
int nds_solver_stage_counts(nds_solver* s, long long* applied, long long* fallbacks);

/* ---- mixed hexahedron/tetrahedron Stokes gate: replaces the reference's
 *      HXT4A executable (gpu/serial_cuda/hybrid_hxt4a/hxt4a_main.cu:405-518,
 *      operators from hybrid_hxt2/hxt2_main.cu and hybrid_hxt3a/hxt3a_main.cu).
 * Reads a binary HXT1 mesh with hex and tet cells (Q1+BF2 hex and P1+BF3
 * tet velocity, P0 pressure, Nitsche-coupled interface), sets the
 * manufactured axial pressure p* (cell centroid z, 0 at cell 0) and runs the
 * SIMPLE loop of the gate: three Jacobi-PCG momentum solves with forcing
 * B^T p* - B^T p, one Jacobi-PCG solve of B diag(rAU) B^T (rAU = rau_scale /
 * penalty-free diag A), p += alpha_p dp, until relCont <= simple_tol.
 * verbose = 1 prints the reference's NODALS_HXT4A_* lines.  Returns NDS_OK
 * when the loop ran to convergence (pass tells whether the gate's
 * accuracy criteria hold), NDS_E_SETUP for a bad mesh or a failed solve,
 * NDS_E_CUDA without a device. */
typedef struct nds_hybrid_report {
  int outer_its, converged, pass;
  int n_hex, n_tet, n_interface, n_velocity;
  double final_rel_cont, pressure_rel_l2, slope, slope_exact, delta, delta_exact, velocity_rel;
  double avg_momentum_cg, avg_pressure_cg;
  double a_norm, b_norm, s_norm;   /* operator audit: ||A a||, ||B b||, ||S p|| on fixed vectors */
  double loop_ms;                  /* wall time of the SIMPLE loop and final predictor */
} nds_hybrid_report;
int nds_hybrid_stokes_gate(const char* hxt1_path, double nu, double gamma, double rau_scale, double alpha_p,
                           double simple_tol, int max_outer, int device, int verbose, nds_hybrid_report* out);
/* Host-only operator audit of the same gate (no device needed): norms[0..2] =
 * ||A a||, ||B b||, ||S p|| for the gate's fixed vectors a_g = sin(0.00113
 * (g+1)), b = (cos(0.00131 (g+1)), sin(0.00091 (g+1) + 0.2), cos(0.00157
 * (g+1) - 0.1)), p_i = sin(0.00107 (i+1)), as the reference prints them in
 * NODALS_HXT4A_OPERATOR_AUDIT (hxt4a_main.cu:429-437). */
int nds_hybrid_operator_audit(const char* hxt1_path, double nu, double gamma, double rau_scale, double norms[3]);

/* ---- mixed-mesh pipe SIMPLE: replaces the reference's HXT4B executable
 *      (gpu/serial_cuda/hybrid_hxt4b/hxt4b_main.cu:211-268).
 * Steady Navier-Stokes in a straight pipe of 10 diameters on a binary HXT1
 * mesh with hex and tet cells: parabolic inlet, no-slip wall (hex faces),
 * natural outlet, nu = bulk D / Re.  Per iteration the lagged central
 * advective convection is assembled into the velocity CSR, the diagonal is
 * relaxed by alpha_u, rAU = rau_scale alpha_u / (penalty-free diagonal +
 * convection diagonal), each velocity component gets the multicolour
 * Gauss-Seidel work momentum_work (0 fgs1, 1 altgs1, 2 sgs1), and
 * B diag(rAU) B^T dp = B u is solved by Jacobi PCG to max(p_atol, p_rtol
 * ||r0||) within p_max iterations, p -= alpha_p dp, until relCont <=
 * simple_tol.  mom_rtol / mom_atol are accepted and unused, as in the
 * reference (fixed-work sweeps).  verbose = 1 prints the reference's
 * NODALS_HXT4B_* lines. */
typedef struct nds_hybrid_flow_options {
  double re, bulk, gamma, alpha_u, alpha_p, rau_scale, simple_tol;
  int max_outer, momentum_work;
  double mom_omega, mom_rtol, mom_atol, p_rtol, p_atol;
  int p_max;
  /* Pressure preconditioner: 0 Jacobi (the HXT4B solver), 1 the classical
   * AMG V-cycle of the reference's turbulent entry (hxt4c::HybridAMG,
   * hybrid_hxt5b/hybrid_amg.cuh:353-533; options and defaults of
   * hxt5b_main.cu:49-86, 195-210).  The hierarchy is built once from the
   * initial rAU; the fine matrix B diag(rAU) B^T is refreshed every
   * iteration, the coarse levels are kept. */
  int pressure_solver;
  int amg_smoother;                 /* enum nds_amg_smoother */
  int amg_spectrum_policy;          /* enum nds_spectrum_policy (auto: power iterations for cheb2 only) */
  int amg_terminal, amg_power_its, amg_cheb_degree;
  int amg_jacobi_fine_sweeps, amg_jacobi_coarse_sweeps;
  int amg_mcgs_fine_sweeps, amg_mcgs_coarse_sweeps, amg_mcgs_order; /* enum nds_mcgs_order */
  int cf_pmax, cf_interp, cf_aggressive_first;                       /* enum nds_cf_interp */
  double cf_theta, amg_lambda_safety, amg_lambda_low_fraction, amg_jacobi_omega, amg_mcgs_omega;
  /* 0: the reference's V-cycle, whose post-smoothing calls pass one work
   * vector as both the result and the Chebyshev product (and on the fine
   * level the right-hand side as the scaled right-hand side), which makes
   * its cheb2 V-cycle nonsymmetric; 1: separate work vectors there, a
   * symmetric V-cycle (same result for jacobi with one sweep and mcgs). */
  int amg_separate_post;
} nds_hybrid_flow_options;
typedef struct nds_hybrid_flow_report {
  int outer_its, converged, pass;
  int n_hex, n_tet, n_velocity;
  double final_rel_cont, avg_pressure_cg;
  double slope, slope_exact, p_in, p_out, drop, drop_exact;   /* pressure against Hagen-Poiseuille */
  double profile_rel_l2, transverse_rel_l2;                   /* vertex velocity against the profile */
  double conv_norm, velocity_norm;
  double loop_ms;
} nds_hybrid_flow_report;
void nds_hybrid_flow_defaults(nds_hybrid_flow_options* o);   /* the reference binary's defaults */
int nds_hybrid_flow(const char* hxt1_path, const nds_hybrid_flow_options* o, int device, int verbose,
                    nds_hybrid_flow_report* out);
/* The same solve, also returning the final fields: u0, u1, u2 hold
 * counts[5] velocity unknowns each (vertices first, then face bubbles) and
 * pressure counts[6] P0 values (hexes first), counts[] being the HXT1
 * header read by nds_hybrid_counts.  Any of the four may be NULL. */
int nds_hybrid_flow_fields(const char* hxt1_path, const nds_hybrid_flow_options* o, int device, int verbose,
                           nds_hybrid_flow_report* out, double* u0, double* u1, double* u2, double* pressure);
/* Host only: the patch and symmetry audit of the mixed-mesh velocity
 * operator that the reference's HXT2 gate prints (hybrid_hxt2/hxt2_main.cu:
 * 296-315), on the operator without boundary conditions (nu-scaled
 * diffusion, with or without the Nitsche interface terms):
 * out[0] max |A 1| (constant patch, with interface); out[1..3] and out[4..6]
 * max |A u| over the interface bubbles for the three affine fields, without
 * and with the interface terms; out[7..10] x.Ax, y.Ay, x.Ay, y.Ax for x, y
 * supported on the interface bubbles (x_g = sin(0.001731 (g+1)), y_g =
 * cos(0.002117 (g+3))); out[11] the number of interface bubble unknowns. */
int nds_hybrid_operator_patch(const char* hxt1_path, double nu, double gamma, double out[12]);
/* Host only: the divergence audit that the reference's HXT3A gate prints
 * (hybrid_hxt3a/hxt3a_main.cu main), with its synthetic rAU_g = 0.8 + 0.2
 * (0.5 + 0.5 sin(0.000731 (g+1))): out[0] nnz of B; out[1] max |B u| over
 * the three constant fields; out[2], out[3] max abs / rel error of B (x,y,z)
 * against 3 V; out[4], out[5] p.Bu and u.B^T p; out[6..9] x.Sx, y.Sy, x.Sy,
 * y.Sx with S = B diag(rAU) B^T; out[10], out[11] min / max norm of the
 * cross-region trace coefficients of each interface triangle pair; out[12],
 * out[13] min / max |S_ht| of those pairs; out[14] the number of pairs;
 * out[15] pairs missing a cross trace or with S_ht = 0. */
int nds_hybrid_divergence_audit(const char* hxt1_path, double out[16]);
/* Host only: the 13 counts of a mixed-mesh HXT1 header (nv nhex ntet
 * nhexface ntetface nvel npressure ninterface nwallhex ninhex nintet
 * nouthex nouttet). */
int nds_hybrid_counts(const char* hxt1_path, uint64_t counts[13]);
/* Host only: the HXT4B VTU (hxt4b_main.cu:203-209, written for --vtu at
 * :265): points, hex then tet connectivity (VTK types 12 and 10), vertex
 * velocity from the first nv entries of u0/u1/u2, the P0 pressure, its
 * volume-weighted vertex average, and region 1 (hex) / 2 (tet). */
int nds_hybrid_write_vtu(const char* hxt1_path, const char* vtu_path, const double* u0, const double* u1,
                         const double* u2, const double* pressure);
/* Host only: the pressure preconditioner's setup for a given rAU (nvel
 * values): the pressure matrix (pin = the first outlet face's cell) and its
 * CF hierarchy, as hxt4c::build_hybrid_fine_host (hybrid_amg.cuh:63) and
 * build_cf_hierarchy_from_csr (hybrid_cf_overload.inc:5) build them.  Named
 * arrays: "pin", "fine.row|col|val|diag|entryRow|diagPos", "amg.levels",
 * "amg.fineLambda", "amg.levelLambda", "amg.P<l>.row|col|val|nCoarse",
 * "amg.A<l>.row|col|val|diag", "amg.terminal_inv". */
typedef struct nds_hybrid_amg nds_hybrid_amg;
int nds_hybrid_amg_create(const char* hxt1_path, const double* rau, const nds_hybrid_flow_options* o,
                          nds_hybrid_amg** out);
int nds_hybrid_amg_array(const nds_hybrid_amg* h, const char* name, nds_array* out);
void nds_hybrid_amg_destroy(nds_hybrid_amg* h);
/* Host only: the mixed-mesh pipe SIMPLE's host setup, as a handle of the same
 * kind (read with nds_hybrid_amg_array, free with nds_hybrid_amg_destroy):
 * "flow.scalars" (pin, R, L, D, nu, nhex, ntet), the velocity CSR
 * "flow.row|col|diagPos", its constant values "flow.base" and penalty-free
 * diagonal "flow.diagRBase", the convection gather lists "flow.srcOff|src",
 * "flow.fixed", the initial state "flow.u0|u1|u2", the colours
 * "flow.colourOff|colourRows" and the divergence "b.row|col|bx|by|bz". */
int nds_hybrid_flow_setup(const char* hxt1_path, const nds_hybrid_flow_options* o, nds_hybrid_amg** out);
/* One application of that preconditioner on the device: the hierarchy is
 * built from rau, the fine matrix refreshed from rau on the device, and
 * z = M^-1 b (np values each) computed by the reference's V-cycle
 * (hxt4c::HybridAMG::apply, hybrid_amg.cuh:519-533). */
int nds_hybrid_amg_vcycle(const char* hxt1_path, const double* rau, const nds_hybrid_flow_options* o, int device,
                          const double* b, double* z);

#ifdef __cplusplus
}
#endif
#endif /* NODALS_B200_H */
