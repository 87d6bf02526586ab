/*
 * TEST INFRASTRUCTURE ONLY -- CPU oracle of the reference's H8 SIMPLE loop.
 * See h8_oracle.h.  Every function names the reference file:line it restates
 * (paths relative to the reference repository).  All arithmetic is FP64 with
 * contraction disabled (-ffp-contract=off); loops that own their outputs run
 * under OpenMP, sums that the reference accumulates in cell order are
 * gathered in ascending cell order.
 */
#define _POSIX_C_SOURCE 199309L /* clock_gettime */
#include "h8_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

#ifdef _OPENMP
#include <omp.h>
#endif

struct ora_state {
  const ora_problem* P;
  int it;
  double cont0, cont_rel;
  double fine_lambda, p_cheb_lambda;
  double* level_lambda;
  /* momentum */
  double *A, *delta, *diag, *rau, *u[3], *b[3];
  double* supg; /* 64 per cell when SUPG is on */
  /* pressure */
  double *p, *rhs, *fval, *fdiag, *fl1;
  double *x, *r, *z, *pp, *q, *fr, *fcorr, *frhs, *ftmp, *fpong;
  double **lb, **lx, **lr, **ltmp, **lcorr, **lpong, **ll1;
};

static double* dalloc(long n) { return (double*)calloc((size_t)(n > 0 ? n : 1), sizeof(double)); }

/* ------------------------------------------------------------------------
 * momentum assembly: A = K + C(u), Dirichlet convection into conv
 * (gpu/serial_cuda/g4_host.hpp:326-340 host_assemble_central_g4), then the
 * row-L1 relaxation (g5e_fp32_kernels.cuh:78-85), rAU scaling
 * (h8_main_base.cu:1154), B^T p (h8_precomputed_b.cuh:93-114) and the RHS
 * (g5e_fp32_kernels.cuh:97-105).  Gathered per row over the incident cells
 * in ascending cell order, which is the host twin's accumulation order.
 * ---------------------------------------------------------------------- */
static void cell_ur(const ora_problem* P, int c, double* const u[3], double ur[8][3], double q[8][3]) {
  const double* I = P->invJ + 9L * c;
  for (int m = 0; m < 8; ++m) {
    const int g = P->ref[8L * c + m];
    for (int d = 0; d < 3; ++d) q[m][d] = g >= 0 ? u[d][g] : P->fixed[3L * (-g - 1) + d];
    for (int j = 0; j < 3; ++j) {
      double s = 0.0;
      for (int d = 0; d < 3; ++d) s += q[m][d] * I[3 * j + d];
      ur[m][j] = s;
    }
  }
}

/* implicit SUPG block S[a][b] of cell c at the lagged velocity u
 * (g4_host.hpp:324-419, the host twin of h7_momentum_assembly.cuh:100-226):
 * S[a][b] = sum_q tau_q w_q det (adv_q . grad phi_a)(adv_q . grad phi_b - nu lap phi_b [bubbles]) */
static void supg_block(const ora_problem* P, int c, double* const u[3], double out[64]) {
  double coeff[3][8];
  for (int m = 0; m < 8; ++m) {
    const int g = P->ref[8L * c + m];
    for (int d = 0; d < 3; ++d) coeff[d][m] = g >= 0 ? u[d][g] : P->fixed[3L * (-g - 1) + d];
  }
  const double* I = P->invJ + 9L * c;
  double gl[4][3], gd[4][4];
  for (int d = 0; d < 3; ++d) {
    gl[0][d] = -(I[d] + I[3 + d] + I[6 + d]);
    gl[1][d] = I[d];
    gl[2][d] = I[3 + d];
    gl[3][d] = I[6 + d];
  }
  for (int i = 0; i < 4; ++i)
    for (int j = i; j < 4; ++j) {
      double q = 0.0;
      for (int d = 0; d < 3; ++d) q += gl[i][d] * gl[j][d];
      gd[i][j] = gd[j][i] = q;
    }
  for (int k = 0; k < 64; ++k) out[k] = 0.0;
  const double h2 = P->h2[c], diff = 4.0 * P->nu / h2;
  for (int qp = 0; qp < 64; ++qp) {
    const double* lam = P->supg_rule + 5 * qp;
    const double qw = lam[4];
    double phi[8];
    int js[4][3];
    for (int i = 0; i < 4; ++i) {
      int kk = 0;
      for (int j = 0; j < 4; ++j)
        if (j != i) js[i][kk++] = j;
      phi[i] = lam[i];
      phi[4 + i] = 27.0 * lam[js[i][0]] * lam[js[i][1]] * lam[js[i][2]];
    }
    double adv[3] = {0, 0, 0};
    for (int d = 0; d < 3; ++d)
      for (int m = 0; m < 8; ++m) adv[d] += coeff[d][m] * phi[m];
    const double speed2 = adv[0] * adv[0] + adv[1] * adv[1] + adv[2] * adv[2];
    double stream[8], strong[8];
    for (int a = 0; a < 4; ++a) stream[a] = adv[0] * gl[a][0] + adv[1] * gl[a][1] + adv[2] * gl[a][2];
    for (int i = 0; i < 4; ++i) {
      const int* j = js[i];
      double gb[3];
      for (int d = 0; d < 3; ++d)
        gb[d] = 27.0 * (lam[j[1]] * lam[j[2]] * gl[j[0]][d] + lam[j[0]] * lam[j[2]] * gl[j[1]][d] +
                        lam[j[0]] * lam[j[1]] * gl[j[2]][d]);
      stream[4 + i] = adv[0] * gb[0] + adv[1] * gb[1] + adv[2] * gb[2];
      const double lap = 54.0 * (lam[j[2]] * gd[j[0]][j[1]] + lam[j[1]] * gd[j[0]][j[2]] + lam[j[0]] * gd[j[1]][j[2]]);
      strong[4 + i] = -P->nu * lap + stream[4 + i];
    }
    for (int a = 0; a < 4; ++a) strong[a] = stream[a];
    const double den = fmax(4.0 * speed2 / h2 + P->supg_magic * diff * diff, 1.0e-30);
    const double w = P->supg_tau_scale / sqrt(den) * qw * P->det[c];
    for (int a = 0; a < 8; ++a) {
      const double ta = w * stream[a];
      for (int b = 0; b < 8; ++b) out[8 * a + b] += ta * strong[b];
    }
  }
}

static void assemble(ora_state* S) {
  const ora_problem* P = S->P;
  const double fac = 1.0 / P->alpha_u - 1.0;
  if (P->supg) {
#pragma omp parallel for schedule(static)
    for (int c = 0; c < P->nc; ++c) supg_block(P, c, S->u, S->supg + 64L * c);
  }
#pragma omp parallel for schedule(dynamic, 256)
  for (int i = 0; i < P->nv; ++i) {
    const int64_t rb = P->mrow[i], re = P->mrow[i + 1];
    for (int64_t k = rb; k < re; ++k) S->A[k] = P->K[k];
    double conv[3] = {0, 0, 0}, bt[3] = {0, 0, 0};
    for (int z = P->inc_off[i]; z < P->inc_off[i + 1]; ++z) {
      const int c = (int)(P->inc[z] >> 3), a = (int)(P->inc[z] & 7u);
      double ur[8][3], q[8][3];
      cell_ur(P, c, S->u, ur, q);
      for (int b = 0; b < 8; ++b) {
        double v = 0.0;
        for (int m = 0; m < 8; ++m)
          for (int j = 0; j < 3; ++j) v += ur[m][j] * P->centT[((a * 8 + m) * 8 + b) * 3 + j];
        const double C = P->supg ? P->det[c] * v + S->supg[64L * c + 8 * a + b] : P->det[c] * v;
        if (P->ref[8L * c + b] >= 0) {
          S->A[rb + P->row_slot[64L * c + 8 * a + b]] += C;
        } else {
          for (int d = 0; d < 3; ++d) conv[d] -= C * q[b][d];
        }
      }
      for (int d = 0; d < 3; ++d) bt[d] += P->bco[24L * c + 3 * a + d] * S->p[c];
    }
    double m = 0.0;
    for (int64_t k = rb; k < re; ++k) m += fabs(S->A[k]);
    const double de = fac * m;
    const int64_t dp = P->mdpos[i];
    S->A[dp] += de;
    S->delta[i] = de;
    S->diag[i] = S->A[dp];
    S->rau[i] = (1.0 / S->A[dp]) * P->rau_scale;
    const double* sv[3] = {P->s0, P->s1, P->s2};
    for (int d = 0; d < 3; ++d) S->b[d][i] = sv[d][i] + conv[d] + bt[d] + de * S->u[d][i];
  }
}

/* one multicolour GS colour pass, 3 RHS (g5e_fp32_kernels.cuh:106-116) */
static void gs_color(ora_state* S, int color) {
  const ora_problem* P = S->P;
  const double om = P->mom_omega;
#pragma omp parallel for schedule(static)
  for (int q = P->color_off[color]; q < P->color_off[color + 1]; ++q) {
    const int i = P->color_rows[q];
    double s[3] = {0, 0, 0};
    for (int64_t k = P->mrow[i]; k < P->mrow[i + 1]; ++k) {
      const int j = P->mcol[k];
      if (j == i) continue;
      for (int d = 0; d < 3; ++d) s[d] += S->A[k] * S->u[d][j];
    }
    const double iv = 1.0 / S->diag[i];
    for (int d = 0; d < 3; ++d) S->u[d][i] = (1.0 - om) * S->u[d][i] + om * ((S->b[d][i] - s[d]) * iv);
  }
}

/* fixed_momentum_work (h8_main_base.cu:1700-1715) */
static void momentum_work(ora_state* S, int it) {
  const ora_problem* P = S->P;
  if (P->momentum_work == 0) {
    for (int c = 0; c < P->ncolors; ++c) gs_color(S, c);
  } else if (P->momentum_work == 1) {
    if (it & 1)
      for (int c = 0; c < P->ncolors; ++c) gs_color(S, c);
    else
      for (int c = P->ncolors - 1; c >= 0; --c) gs_color(S, c);
  } else {
    for (int c = 0; c < P->ncolors; ++c) gs_color(S, c);
    for (int c = P->ncolors - 1; c >= 0; --c) gs_color(S, c);
  }
}

/* pre-sweep momentum audit (g5e_fp32_kernels.cuh:117-126, h8_main_base.cu:1716-1726) */
static void audit(ora_state* S, double rel[3]) {
  const ora_problem* P = S->P;
  double h[6] = {0, 0, 0, 0, 0, 0};
  for (int i = 0; i < P->nv; ++i) {
    double ax[3] = {0, 0, 0};
    for (int64_t k = P->mrow[i]; k < P->mrow[i + 1]; ++k)
      for (int d = 0; d < 3; ++d) ax[d] += S->A[k] * S->u[d][P->mcol[k]];
    for (int d = 0; d < 3; ++d) {
      h[d] += S->b[d][i] * S->b[d][i];
      const double rr = S->b[d][i] - ax[d];
      h[3 + d] += rr * rr;
    }
  }
  for (int d = 0; d < 3; ++d) {
    double bn = sqrt(h[d] > 0 ? h[d] : 0);
    if (bn == 0.0) bn = 1.0;
    rel[d] = sqrt(h[3 + d] > 0 ? h[3 + d] : 0) / bn;
  }
}

/* continuity r = fixedDiv + B u (h8_precomputed_b.cuh:140-163); returns ||r|| */
static double continuity(ora_state* S) {
  const ora_problem* P = S->P;
  double ss = 0.0;
#pragma omp parallel for schedule(static) reduction(+ : ss)
  for (int c = 0; c < P->nc; ++c) {
    double s = P->fixed_div[c];
    for (int a = 0; a < 8; ++a) {
      const int g = P->ref[8L * c + a];
      if (g < 0) continue;
      const double* B = P->bco + 24L * c + 3 * a;
      s += B[0] * S->u[0][g] + B[1] * S->u[1][g] + B[2] * S->u[2][g];
    }
    S->rhs[c] = -s;
    ss += s * s;
  }
  return sqrt(ss);
}

/* fine Schur refresh, serial row order (h2b_fine_csr.cuh:480-520) */
static void refresh(ora_state* S) {
  const ora_problem* P = S->P;
#pragma omp parallel for schedule(dynamic, 128)
  for (int c = 0; c < P->nc; ++c) {
    const int rb = P->frow[c], re = P->frow[c + 1];
    for (int j = rb; j < re; ++j) S->fval[j] = 0.0;
    int q = P->fcontrib_off[c];
    for (int a = 0; a < 8; ++a) {
      const int g = P->ref[8L * c + a];
      if (g < 0) continue;
      const double rv = S->rau[g];
      const double* A = P->bco + 24L * c + 3 * a;
      for (int k = P->inc_off[g]; k < P->inc_off[g + 1]; ++k, ++q) {
        const uint32_t pk = P->inc[k];
        const double* B = P->bco + 24L * (pk >> 3) + 3 * (pk & 7u);
        const double dot = A[0] * B[0] + A[1] * B[1] + A[2] * B[2];
        S->fval[rb + P->fslot[q]] += rv * dot;
      }
    }
    S->fdiag[c] = S->fval[P->fdpos[c]];
    if (S->fl1) {
      double s = 0;
      for (int j = rb; j < re; ++j) s += fabs(S->fval[j]);
      S->fl1[c] = s;
    }
  }
}

/* ---------------------------------------------------------------- AMG */
static void spmv32(int n, const int32_t* rp, const int32_t* ci, const double* v, const double* x, double* y) {
#pragma omp parallel for schedule(static)
  for (int i = 0; i < n; ++i) {
    double s = 0;
    for (int k = rp[i]; k < rp[i + 1]; ++k) s += v[k] * x[ci[k]];
    y[i] = s;
  }
}
static void spmv64(int n, const int64_t* rp, const int32_t* ci, const double* v, const double* x, double* y) {
#pragma omp parallel for schedule(static)
  for (int i = 0; i < n; ++i) {
    double s = 0;
    for (int64_t k = rp[i]; k < rp[i + 1]; ++k) s += v[k] * x[ci[k]];
    y[i] = s;
  }
}
static void fine_apply(ora_state* S, const double* x, double* y) {
  spmv32(S->P->nc, S->P->frow, S->P->fcol, S->fval, x, y);
}
static double dotp(int n, const double* x, const double* y) {
  double s = 0;
#pragma omp parallel for schedule(static) reduction(+ : s)
  for (int i = 0; i < n; ++i) s += x[i] * y[i];
  return s;
}

static double cheb_root(double hi, double lo, int k, int deg) {
  const double c = .5 * (hi + lo), r = .5 * (hi - lo), pi = 3.141592653589793238462643383279502884;
  return c - r * cos(pi * (2.0 * (double)k + 1.0) / (2.0 * (double)deg));
}

/* smoother on one operator from a zero guess (h8_main_base.cu:429-463) */
typedef struct {
  int n;
  const int64_t* r64;
  const int32_t* r32;
  const int32_t* col;
  const double* val;
  const double* diag;
  const double* l1;
} opview;

static void op_apply(const opview* A, const double* x, double* y) {
  if (A->r32) spmv32(A->n, A->r32, A->col, A->val, x, y);
  else spmv64(A->n, A->r64, A->col, A->val, x, y);
}

static void smooth(ora_state* S, const opview* A, const double* b, double* x, double* tmp, double lambda, int sweeps) {
  const ora_problem* P = S->P;
  const int n = A->n;
  if (P->amg_smoother == 0) { /* cheb2 */
    const double lo = P->amg_lambda_low_fraction * lambda;
    const int deg = P->amg_cheb_degree;
    const double w0 = 1.0 / cheb_root(lambda, lo, 0, deg);
    for (int i = 0; i < n; ++i) x[i] = w0 * b[i] / A->diag[i];
    for (int k = 1; k < deg; ++k) {
      op_apply(A, x, tmp);
      const double w = 1.0 / cheb_root(lambda, lo, k, deg);
      for (int i = 0; i < n; ++i) x[i] += w * (b[i] - tmp[i]) / A->diag[i];
    }
  } else { /* jacobi / l1jacobi */
    const double* den = P->amg_smoother == 2 ? A->l1 : A->diag;
    const double w = P->amg_jacobi_omega;
    for (int i = 0; i < n; ++i) x[i] = w * b[i] / den[i];
    for (int s = 1; s < sweeps; ++s) {
      op_apply(A, x, tmp);
      for (int i = 0; i < n; ++i) x[i] += w * (b[i] - tmp[i]) / den[i];
    }
  }
}

/* c = P^T f (g5e_fp32_kernels.cuh:145), f += P c (:148) */
static void restrict_t(const ora_xfer* X, const double* f, double* c) {
  memset(c, 0, sizeof(double) * (size_t)X->nc);
  for (int i = 0; i < X->nf; ++i)
    for (int64_t k = X->row[i]; k < X->row[i + 1]; ++k) c[X->col[k]] += X->val[k] * f[i];
}
static void prolong_add(const ora_xfer* X, const double* c, double* f) {
#pragma omp parallel for schedule(static)
  for (int i = 0; i < X->nf; ++i) {
    double s = 0;
    for (int64_t k = X->row[i]; k < X->row[i + 1]; ++k) s += X->val[k] * c[X->col[k]];
    f[i] += s;
  }
}

static opview level_view(ora_state* S, int l) {
  const ora_level* L = &S->P->L[l];
  opview v = {L->n, L->row, NULL, L->col, L->val, L->diag, S->ll1[l]};
  return v;
}
static opview fine_view(ora_state* S) {
  opview v = {S->P->nc, NULL, S->P->frow, S->P->fcol, S->fval, S->fdiag, S->fl1};
  return v;
}

/* explicit_vcycle (h8_main_base.cu:544-556) */
static void vcycle(ora_state* S, int l, const double* b, double* x) {
  const ora_problem* P = S->P;
  const int n = P->L[l].n;
  if (l == P->nlev - 1) {
#pragma omp parallel for schedule(static)
    for (int i = 0; i < n; ++i) {
      double s = 0;
      for (int j = 0; j < n; ++j) s += P->tinv[(size_t)i * n + j] * b[j];
      x[i] = s;
    }
    return;
  }
  opview A = level_view(S, l);
  smooth(S, &A, b, x, S->ltmp[l], S->level_lambda[l], P->amg_jacobi_coarse_sweeps);
  op_apply(&A, x, S->ltmp[l]);
  for (int i = 0; i < n; ++i) S->lr[l][i] = b[i] - S->ltmp[l][i];
  restrict_t(&P->P[l + 1], S->lr[l], S->lb[l + 1]);
  vcycle(S, l + 1, S->lb[l + 1], S->lx[l + 1]);
  prolong_add(&P->P[l + 1], S->lx[l + 1], x);
  op_apply(&A, x, S->ltmp[l]);
  double* rb = S->lpong[l];
  for (int i = 0; i < n; ++i) rb[i] = b[i] - S->ltmp[l][i];
  smooth(S, &A, rb, S->lcorr[l], S->ltmp[l], S->level_lambda[l], P->amg_jacobi_coarse_sweeps);
  for (int i = 0; i < n; ++i) x[i] += S->lcorr[l][i];
}

/* G4AMG::apply (h8_main_base.cu:557-564) */
static void amg_apply(ora_state* S, const double* b, double* z) {
  const ora_problem* P = S->P;
  const int n = P->nc;
  opview F = fine_view(S);
  smooth(S, &F, b, z, S->ftmp, S->fine_lambda, P->amg_jacobi_fine_sweeps);
  fine_apply(S, z, S->ftmp);
  for (int i = 0; i < n; ++i) S->fr[i] = b[i] - S->ftmp[i];
  restrict_t(&P->P[0], S->fr, S->lb[0]);
  vcycle(S, 0, S->lb[0], S->lx[0]);
  prolong_add(&P->P[0], S->lx[0], z);
  fine_apply(S, z, S->ftmp);
  for (int i = 0; i < n; ++i) S->frhs[i] = b[i] - S->ftmp[i];
  smooth(S, &F, S->frhs, S->fcorr, S->ftmp, S->fine_lambda, P->amg_jacobi_fine_sweeps);
  for (int i = 0; i < n; ++i) z[i] += S->fcorr[i];
}

/* power iterations on D^-1/2 A D^-1/2 (h8_main_base.cu:873-889) */
static double power_op(const opview* A, int its, double safety, double* v, double* u, double* au, double* w) {
  const int n = A->n;
  for (int i = 0; i < n; ++i) {
    const double g = (double)(i + 1);
    v[i] = sin(0.731 * g) + 0.27 * cos(1.117 * g);
  }
  const double vn = sqrt(dotp(n, v, v));
  for (int i = 0; i < n; ++i) v[i] *= 1.0 / vn;
  double ray = 0.0;
  for (int it = 0; it < its; ++it) {
    for (int i = 0; i < n; ++i) u[i] = v[i] / sqrt(A->diag[i]);
    op_apply(A, u, au);
    for (int i = 0; i < n; ++i) w[i] = au[i] / sqrt(A->diag[i]);
    const double num = dotp(n, v, w), den = dotp(n, v, v);
    ray = num / (den > 1e-300 ? den : 1e-300);
    const double wn = sqrt(dotp(n, w, w));
    if (!(ray > 0.0) || !(wn > 0.0) || !isfinite(ray) || !isfinite(wn)) return -1.0;
    for (int i = 0; i < n; ++i) v[i] = w[i] * (1.0 / wn);
  }
  return safety * ray;
}

/* pressure_precond_power (h8_main_base.cu:613-668) */
static double precond_power(ora_state* S) {
  const ora_problem* P = S->P;
  const int n = P->nc;
  for (int i = 0; i < n; ++i) {
    const double g = (double)(i + 1);
    S->pp[i] = sin(0.731 * g) + 0.27 * cos(1.117 * g);
  }
  const double vn = sqrt(dotp(n, S->pp, S->pp));
  for (int i = 0; i < n; ++i) S->pp[i] *= 1.0 / vn;
  double est = 0.0;
  for (int k = 0; k < P->p_power_its; ++k) {
    fine_apply(S, S->pp, S->q);
    amg_apply(S, S->q, S->z);
    const double zn = sqrt(dotp(n, S->z, S->z)), ray = dotp(n, S->pp, S->z);
    if (!(zn > 0.0) || !isfinite(zn) || !isfinite(ray)) return -1.0;
    const double last = fabs(ray);
    if (last > est) est = last;
    if (zn > est) est = zn;
    for (int i = 0; i < n; ++i) S->pp[i] = S->z[i] * (1.0 / zn);
  }
  return P->p_power_safety * est;
}

/* pressure_pcg / richardson / cheb_poly (h8_main_base.cu:569-611, 670-726) */
static int pressure(ora_state* S, int* its, double* rel) {
  const ora_problem* P = S->P;
  const int n = P->nc;
  memset(S->x, 0, sizeof(double) * (size_t)n);
  memcpy(S->r, S->rhs, sizeof(double) * (size_t)n);
  const double r0 = sqrt(dotp(n, S->r, S->r));
  *its = 0;
  *rel = 1.0;
  if (!isfinite(r0)) return -4;
  if (r0 <= P->p_atol) {
    *rel = 0.0;
    return 1;
  }
  const double target = fmax(P->p_atol, P->p_rtol * r0);
  if (P->pressure_solver == 0) {
    amg_apply(S, S->r, S->z);
    memcpy(S->pp, S->z, sizeof(double) * (size_t)n);
    double rho = dotp(n, S->r, S->z);
    if (!(rho > 0) || !isfinite(rho)) return -4;
    for (int k = 0; k < P->p_max; ++k) {
      fine_apply(S, S->pp, S->q);
      const double pq = dotp(n, S->pp, S->q);
      if (!(pq > 0) || !isfinite(pq)) return -4;
      const double alpha = rho / pq;
      for (int i = 0; i < n; ++i) {
        S->x[i] += alpha * S->pp[i];
        S->r[i] -= alpha * S->q[i];
      }
      const double rn = sqrt(dotp(n, S->r, S->r));
      *its = k + 1;
      *rel = rn / fmax(r0, 1e-300);
      if (rn <= target) return 1;
      amg_apply(S, S->r, S->z);
      const double rhon = dotp(n, S->r, S->z);
      if (!(rhon > 0) || !isfinite(rhon)) return -4;
      const double beta = rhon / rho;
      for (int i = 0; i < n; ++i) S->pp[i] = S->z[i] + beta * S->pp[i];
      rho = rhon;
    }
    return 0;
  }
  const int cheb = P->pressure_solver == 2;
  const double lo = P->p_cheb_low_fraction * S->p_cheb_lambda;
  const double centre = .5 * (S->p_cheb_lambda + lo), radius = .5 * (S->p_cheb_lambda - lo);
  const double pi = 3.141592653589793238462643383279502884;
  for (int k = 0; k < P->p_max; ++k) {
    double omega = P->p_richardson_omega;
    if (cheb) omega = 1.0 / (centre - radius * cos(pi * (2.0 * (double)(k % P->p_cheb_degree) + 1.0) / (2.0 * (double)P->p_cheb_degree)));
    amg_apply(S, S->r, S->z);
    fine_apply(S, S->z, S->q);
    for (int i = 0; i < n; ++i) {
      S->x[i] += omega * S->z[i];
      S->r[i] -= omega * S->q[i];
    }
    const double rn = sqrt(dotp(n, S->r, S->r));
    *its = k + 1;
    *rel = rn / fmax(r0, 1e-300);
    if (!isfinite(*rel)) return -4;
    if (rn <= target) return 1;
  }
  return 0;
}

ora_state* ora_create(const ora_problem* P) {
#ifdef _OPENMP
  if (P->threads > 0) omp_set_num_threads(P->threads);
#endif
  ora_state* S = (ora_state*)calloc(1, sizeof(ora_state));
  S->P = P;
  const int64_t mz = P->mrow[P->nv];
  S->A = dalloc(mz);
  S->delta = dalloc(P->nv);
  S->diag = dalloc(P->nv);
  S->rau = dalloc(P->nv);
  memcpy(S->rau, P->init_rau, sizeof(double) * (size_t)P->nv);
  for (int d = 0; d < 3; ++d) {
    S->u[d] = dalloc(P->nv);
    S->b[d] = dalloc(P->nv);
  }
  const int n = P->nc;
  if (P->supg) S->supg = dalloc(64L * n);
  S->p = dalloc(n);
  S->rhs = dalloc(n);
  S->fval = dalloc(P->frow[n]);
  S->fdiag = dalloc(n);
  S->fl1 = P->amg_smoother == 2 ? dalloc(n) : NULL;
  double** vs[] = {&S->x, &S->r, &S->z, &S->pp, &S->q, &S->fr, &S->fcorr, &S->frhs, &S->ftmp, &S->fpong};
  for (unsigned k = 0; k < sizeof(vs) / sizeof(vs[0]); ++k) *vs[k] = dalloc(n);
  const int nl = P->nlev;
  double*** lv[] = {&S->lb, &S->lx, &S->lr, &S->ltmp, &S->lcorr, &S->lpong, &S->ll1};
  for (unsigned k = 0; k < sizeof(lv) / sizeof(lv[0]); ++k) {
    *lv[k] = (double**)calloc((size_t)nl, sizeof(double*));
    for (int l = 0; l < nl; ++l) (*lv[k])[l] = dalloc(P->L[l].n);
  }
  for (int l = 0; l < nl; ++l)
    for (int i = 0; i < P->L[l].n; ++i) {
      double s = 0;
      for (int64_t k = P->L[l].row[i]; k < P->L[l].row[i + 1]; ++k) s += fabs(P->L[l].val[k]);
      S->ll1[l][i] = s;
    }
  S->level_lambda = dalloc(nl);
  /* setup state: fine CSR at the initial rAU, spectrum (h8_main_base.cu:2014-2025) */
  refresh(S);
  if (P->power_its > 0) {
    opview F = fine_view(S);
    S->fine_lambda = power_op(&F, P->power_its, P->amg_lambda_safety, S->fcorr, S->frhs, S->ftmp, S->fr);
    for (int l = 0; l + 1 < nl; ++l) {
      opview A = level_view(S, l);
      S->level_lambda[l] = power_op(&A, P->power_its, P->amg_lambda_safety, S->lcorr[l], S->lb[l], S->ltmp[l], S->lr[l]);
    }
  } else {
    S->fine_lambda = 1.0;
    for (int l = 0; l < nl; ++l) S->level_lambda[l] = 1.0;
  }
  if (P->pressure_solver == 2) S->p_cheb_lambda = precond_power(S);
  S->cont0 = -1.0;
  S->cont_rel = 1.0;
  return S;
}

double ora_fine_lambda(const ora_state* S) { return S->fine_lambda; }

static double now_ms(void) {
  struct timespec t;
  clock_gettime(CLOCK_MONOTONIC, &t);
  return 1e3 * (double)t.tv_sec + 1e-6 * (double)t.tv_nsec;
}

/* one SIMPLE iteration (h8_main_base.cu:2046-2119) */
int ora_step(ora_state* S, ora_report* R) {
  const ora_problem* P = S->P;
  memset(R, 0, sizeof(*R));
  const double t0 = now_ms();
  const int it = ++S->it;
  R->it = it;
  assemble(S);
  if (P->run_mode == 1 && it > 1 && S->cont_rel <= P->simple_tol) {
    audit(S, R->audit_rel);
    R->audited = 1;
  }
  momentum_work(S, it);
  const double cn = continuity(S);
  if (it == 1) S->cont0 = cn;
  S->cont_rel = cn / fmax(S->cont0, 1e-300);
  R->rel_cont = S->cont_rel;
  R->cont_norm = cn;
  refresh(S);
  const double tp = now_ms();
  const int st = pressure(S, &R->p_its, &R->p_rel);
  R->ms_pressure = now_ms() - tp;
  if (st < 0) {
    R->status = st;
    return st;
  }
  R->p_ok = st;
  if (!st) {
    R->status = -5;
    return -5;
  }
  for (int i = 0; i < P->nc; ++i) S->p[i] += P->alpha_p * S->x[i];
  const int met = R->audited && R->audit_rel[0] <= P->simple_tol && R->audit_rel[1] <= P->simple_tol &&
                  R->audit_rel[2] <= P->simple_tol;
  R->converged = P->run_mode == 1 && isfinite(R->rel_cont) && R->rel_cont <= P->simple_tol && met;
  R->ms_total = now_ms() - t0;
  return 0;
}

void ora_get(const ora_state* S, double* u0, double* u1, double* u2, double* p) {
  const size_t nv = (size_t)S->P->nv;
  if (u0) memcpy(u0, S->u[0], sizeof(double) * nv);
  if (u1) memcpy(u1, S->u[1], sizeof(double) * nv);
  if (u2) memcpy(u2, S->u[2], sizeof(double) * nv);
  if (p) memcpy(p, S->p, sizeof(double) * (size_t)S->P->nc);
}

void ora_set(ora_state* S, const double* u0, const double* u1, const double* u2, const double* p) {
  const size_t nv = (size_t)S->P->nv;
  if (u0) memcpy(S->u[0], u0, sizeof(double) * nv);
  if (u1) memcpy(S->u[1], u1, sizeof(double) * nv);
  if (u2) memcpy(S->u[2], u2, sizeof(double) * nv);
  if (p) memcpy(S->p, p, sizeof(double) * (size_t)S->P->nc);
}

void ora_destroy(ora_state* S) {
  if (!S) return;
  free(S->A); free(S->delta); free(S->diag); free(S->rau); free(S->supg);
  for (int d = 0; d < 3; ++d) { free(S->u[d]); free(S->b[d]); }
  free(S->p); free(S->rhs); free(S->fval); free(S->fdiag); free(S->fl1);
  double* vs[] = {S->x, S->r, S->z, S->pp, S->q, S->fr, S->fcorr, S->frhs, S->ftmp, S->fpong};
  for (unsigned k = 0; k < sizeof(vs) / sizeof(vs[0]); ++k) free(vs[k]);
  double** lv[] = {S->lb, S->lx, S->lr, S->ltmp, S->lcorr, S->lpong, S->ll1};
  for (unsigned k = 0; k < sizeof(lv) / sizeof(lv[0]); ++k) {
    for (int l = 0; l < S->P->nlev; ++l) free(lv[k][l]);
    free(lv[k]);
  }
  free(S->level_lambda);
  free(S);
}
