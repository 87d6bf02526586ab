/* Compiled by tests/test_c_abi.py: drives the C ABI from plain C on a
 * one-hexahedron pipe-like block (5 tets) without touching the GPU, and
 * checks that the device solver refuses to start without a CUDA device. */
#include <stdio.h>
#include <string.h>

#include "nodals_b200.h"

int main(int argc, char** argv) {
  (void)argc;
  nds_options o;
  nds_options_default(&o);
  if (o.precision != NDS_FP64 || o.p_max <= 0) return 10;
  printf("version %s\n", nds_version());
  nds_mesh* m = NULL;
  if (nds_mesh_read_msh2(argv[1], &m) != NDS_OK) {
    printf("mesh error: %s\n", nds_last_error());
    return 11;
  }
  int np, nc, nf, ni;
  if (nds_mesh_counts(m, &np, &nc, &nf, &ni) != NDS_OK) return 12;
  printf("mesh %d %d %d %d\n", np, nc, nf, ni);
  o.max_outer = 10;
  o.amg_terminal = 60;
  nds_problem* p = NULL;
  if (nds_problem_create(m, &o, &p) != NDS_OK) {
    printf("problem error: %s\n", nds_last_error());
    return 13;
  }
  int pc, pv, col, lev;
  if (nds_problem_counts(p, &pc, &pv, &col, &lev) != NDS_OK || pc != nc) return 14;
  nds_array a;
  if (nds_problem_array(p, "color", &a) != NDS_OK || a.count != pv || a.dtype != 1) return 15;
  if (nds_problem_array(p, "no.such.array", &a) != NDS_E_INVALID) return 16;
  printf("problem %d %d %d %d\n", pc, pv, col, lev);
  o.alpha_u = 7.0; /* out of range: rejected like the reference's usage check */
  nds_problem* bad = NULL;
  if (nds_problem_create(m, &o, &bad) != NDS_E_INVALID || bad != NULL) return 17;
  nds_solver* s = NULL;
  const int st = nds_solver_create(p, &s);
  printf("solver_create %d %s\n", st, st ? nds_last_error() : "");
  if (st == NDS_OK) nds_solver_destroy(s);
  nds_problem_destroy(p);
  nds_mesh_destroy(m);
  return 0;
}
