/* heom_oracle CLI -- TEST INFRASTRUCTURE ONLY.
 * Prints the same sections as oracle/ref_driver so the restatement can be
 * diffed against the reference's own code:
 *   heom_oracle <file.key> [--structured | --quad] [--max-steps N] [--single-manifold]
 * --quad propagates and combines in binary128 (ho_2des_q); --quad-mask abc runs one
 * binary128 trajectory and prints each value as a (hi, lo) pair (ho_traj_q_split). */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include "heom_oracle.h"

int main(int argc, char **argv) {
  if (argc < 2) {
    fprintf(stderr, "usage: %s <file.key> [--structured | --quad] [--max-steps N] [--single-manifold]\n", argv[0]);
    return 2;
  }
  int mode = HO_DENSE, max_steps = 0, single = 0, quad = 0;
  const char *mask = NULL; /* --quad-mask abc: one binary128 trajectory as (hi, lo) pairs */
  for (int a = 2; a < argc; a++) {
    if (!strcmp(argv[a], "--structured")) mode = HO_STRUCTURED;
    else if (!strcmp(argv[a], "--max-steps") && a + 1 < argc) max_steps = atoi(argv[++a]);
    else if (!strcmp(argv[a], "--single-manifold")) single = 1;
    else if (!strcmp(argv[a], "--quad")) quad = 1;
    else if (!strcmp(argv[a], "--quad-mask") && a + 1 < argc) mask = argv[++a];
  }
  ho_problem *p = NULL;
  char err[512];
  if (ho_load_key(argv[1], single, &p, err, sizeof err)) {
    fprintf(stderr, "error: %s\n", err);
    return 1;
  }
  int info[10];
  ho_info(p, info);
  int cap = info[7] + 1, ns = info[6], n = 0;
  if (mask) {
    if (strlen(mask) != 3) { fprintf(stderr, "error: --quad-mask wants three digits\n"); return 2; }
    double *hi = calloc(2 * (size_t)cap, sizeof(double)), *lo = calloc(2 * (size_t)cap, sizeof(double));
    if (ho_traj_q_split(p, mask[0] - '0', mask[1] - '0', mask[2] - '0', max_steps, hi, lo, cap, &n)) {
      fprintf(stderr, "error: propagation failed\n");
      return 1;
    }
    printf("#trajq %s %d\n", mask, n);
    for (int j = 0; j < n; j++) printf("%.17e %.17e %.17e %.17e\n", hi[2 * j], lo[2 * j], hi[2 * j + 1], lo[2 * j + 1]);
    free(hi);
    free(lo);
    ho_free(p);
    return 0;
  }
  double *P = calloc(2 * (size_t)cap, sizeof(double));
  double *traj = calloc(2 * (size_t)cap * 3 * ns, sizeof(double));
  if (quad ? ho_2des_q(p, max_steps, P, cap, &n, traj) : ho_2des(p, mode, max_steps, P, cap, &n, traj)) {
    fprintf(stderr, "error: propagation failed\n");
    return 1;
  }
  for (int s = 0; s < ns; s++) {
    printf("#traj %d %d\n", s, n);
    const double *tp = traj + 2 * (size_t)cap * 3 * s;
    for (int j = 0; j < n; j++)
      printf("%.17e %.17e %.17e %.17e %.17e %.17e\n", tp[2 * j], tp[2 * j + 1], tp[2 * (cap + j)],
             tp[2 * (cap + j) + 1], tp[2 * (2 * cap + j)], tp[2 * (2 * cap + j) + 1]);
  }
  printf("#combined %d\n", n);
  for (int j = 0; j < n; j++) printf("%.17e %.17e\n", P[2 * j], P[2 * j + 1]);
  free(P);
  free(traj);
  ho_free(p);
  return 0;
}
