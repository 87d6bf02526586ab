/*
 * TEST INFRASTRUCTURE ONLY -- the CPU oracle of the H8 SIMPLE loop.
 *
 * A plain-C, FP64 restatement of the reference solver's per-iteration
 * algorithm (JD63021/NodalS gpu/serial_cuda/h8_main_base.cu:2046-2119 and
 * the kernels it launches).  Only tests/, __graft_entry__.smoke() and the
 * CPU-baseline leg of bench.py may load it; the product never does.
 *
 * Parity pinning: the setup arrays it consumes are checked bit-exactly
 * (integers) and to round-off (floats) against the reference's own setup
 * builders compiled from the reference tree (oracle/ref_setup_dump.cu); its
 * SIMPLE history is checked against committed fixtures produced by the
 * reference H8 binaries (tests/golden/).
 */
#ifndef NDS_H8_ORACLE_H
#define NDS_H8_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct ora_level {
  int n;
  const int64_t* row;
  const int32_t* col;
  const double* val;
  const double* diag;
} ora_level;

typedef struct ora_xfer {
  int nf, nc;
  const int64_t* row;
  const int32_t* col;
  const double* val;
} ora_xfer;

typedef struct ora_problem {
  int nc, nv, ncolors;
  /* momentum operator */
  const int64_t* mrow;
  const int32_t* mcol;
  const double* K;          /* diffusion values at nu */
  const int32_t* mdpos;     /* absolute diagonal positions */
  const int32_t* color_off; /* ncolors + 1 */
  const int32_t* color_rows;
  const int32_t* inc_off;   /* free velocity dof -> incident (cell<<3 | basis), ascending cell */
  const uint32_t* inc;
  /* cells */
  const int32_t* ref;       /* 8 per cell */
  const uint8_t* row_slot;  /* 64 per cell */
  const double* det;
  const double* invJ;       /* 9 per cell */
  const double* bco;        /* 24 per cell */
  const double* fixed;      /* 3 per fixed slot */
  const double* fixed_div;
  const double* s0;
  const double* s1;
  const double* s2;
  const double* centT;      /* 8*8*8*3 */
  const double* init_rau;
  /* fine Schur CSR topology and refresh map */
  const int32_t* frow;
  const int32_t* fcol;
  const int32_t* fdpos;
  const int32_t* fcontrib_off;
  const uint8_t* fslot;
  /* AMG */
  int nlev;                 /* explicit levels; the last is terminal */
  const ora_level* L;
  const ora_xfer* P;        /* nlev transfers: P[0] fine -> L[0] */
  const double* tinv;       /* terminal dense inverse */
  int power_its;            /* effective AMG power iterations (0: lambdas = 1) */
  /* options (nds_options semantics) */
  double alpha_u, alpha_p, rau_scale, simple_tol, mom_omega;
  int run_mode, momentum_work;
  int pressure_solver;
  double p_rtol, p_atol;
  int p_max;
  double p_richardson_omega;
  int p_cheb_degree, p_power_its;
  double p_cheb_low_fraction, p_power_safety;
  int amg_smoother, amg_cheb_degree;
  double amg_lambda_safety, amg_lambda_low_fraction, amg_jacobi_omega;
  int amg_jacobi_fine_sweeps, amg_jacobi_coarse_sweeps;
  int threads;
  /* laminar SUPG (0: off) */
  int supg;
  double nu, supg_tau_scale, supg_magic;
  const double* h2;         /* per cell */
  const double* supg_rule;  /* 64 x (lambda0..3, weight) */
} ora_problem;

typedef struct ora_report {
  int it;
  double rel_cont, cont_norm;
  int p_its;
  double p_rel;
  int p_ok;
  int audited;
  double audit_rel[3];
  int converged;
  int status;               /* 0 ok, <0 breakdown */
  double ms_total;          /* wall time of the step */
  double ms_pressure;       /* wall time of the pressure solve */
} ora_report;

typedef struct ora_state ora_state;

ora_state* ora_create(const ora_problem* p);
int ora_step(ora_state* s, ora_report* r);
void ora_get(const ora_state* s, double* u0, double* u1, double* u2, double* p);
void ora_set(ora_state* s, const double* u0, const double* u1, const double* u2, const double* p);
double ora_fine_lambda(const ora_state* s);
void ora_destroy(ora_state* s);

#ifdef __cplusplus
}
#endif
#endif
