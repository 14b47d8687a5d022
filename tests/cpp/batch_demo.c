/* A C caller of the batch API (plain C11: the header is C-compatible).
 * Builds three uneven forests, solves them in one batched launch from host
 * buffers and prints each problem's status.  Exit code 2 when no CUDA
 * device is present. */
#include <stdio.h>
#include <stdlib.h>

#include "cup2d_poisson.h"

int main(void) {
  const double disk_a[3] = {0.6, 0.5, 0.1};
  const double disk_b[6] = {1.2, 0.4, 0.1, 0.5, 0.6, 0.07};
  cup2d_mesh* mesh[3] = {NULL, NULL, NULL};
  if (cup2d_mesh_disks(4, 2, 4, 2.0, 0, 0, 1, disk_a, 0.15, &mesh[0]) ||
      cup2d_mesh_disks(4, 2, 3, 2.0, 0, 0, 2, disk_b, 0.1, &mesh[1]) ||
      cup2d_mesh_uniform(2, 1, 2, 1, 2.0, 0, 0, &mesh[2])) {
    printf("mesh construction failed\n");
    return 1;
  }
  cup2d_forest forest[3];
  double* b[3];
  double* x[3];
  for (int i = 0; i < 3; ++i) {
    cup2d_mesh_forest(mesh[i], &forest[i]);
    const int64_t n = 64 * forest[i].nblocks;
    b[i] = (double*)malloc(sizeof(double) * (size_t)n);
    x[i] = (double*)calloc((size_t)n, sizeof(double));
    cup2d_rhs_fourier(&forest[i], 100 + (uint64_t)i, 8, b[i]);
  }
  cup2d_solve_opts opts;
  cup2d_default_opts(&opts);
  opts.tol_rel = 1e-8;
  opts.max_iter = 5000;
  opts.precision = CUP2D_PREC_MIXED;
  cup2d_batch* B = NULL;
  int st = cup2d_batch_create(3, forest, &opts, &B);
  int rc = 0;
  if (st == CUP2D_NO_DEVICE) {
    printf("status %d (%s)\n", st, cup2d_status_string(st));
    rc = 2;
  } else if (st != CUP2D_OK) {
    printf("cup2d_batch_create: %s\n", cup2d_status_string(st));
    rc = 1;
  } else {
    cup2d_solve_stats stats[3];
    st = cup2d_batch_solve(B, (const double* const*)b, x, stats);
    for (int i = 0; i < 3 && st == CUP2D_OK; ++i)
      printf("problem %d: status %d, %d iterations\n", i, stats[i].status, stats[i].iterations);
    if (st != CUP2D_OK) {
      printf("cup2d_batch_solve: %s\n", cup2d_status_string(st));
      rc = 1;
    }
    cup2d_batch_destroy(B);
  }
  for (int i = 0; i < 3; ++i) {
    free(b[i]);
    free(x[i]);
    cup2d_mesh_destroy(mesh[i]);
  }
  return rc;
}
