/*
 * ref_cpu_bench.c -- project-written timing harness around the reference's
 * unmodified CPU driver (src/mc_cpu.c:106-308, MT19937 from src/mt19937ar.c).
 * TEST/BENCH INFRASTRUCTURE ONLY: bench.py runs one process of this per host
 * core (the reference's MT19937 state is a process global) for its CPU
 * baseline and its `--impl reference` arm.
 *
 * usage: ref_cpu_bench L ngrids nsweeps mag_output_int beta h seed
 * prints one line to stderr: "<attempts> <wall_seconds>"
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

#include "mc_cpu.h"
#include "grid.h"

static int null_outfunc(int L, int ngrids, int *grid_data, int isweep, float *m,
                        float *lc, char *cv, double dn, double up, char *fn) {
  (void)L; (void)ngrids; (void)grid_data; (void)isweep; (void)m; (void)lc;
  (void)cv; (void)dn; (void)up; (void)fn;
  return 0;
}

int main(int argc, char **argv) {
  if (argc != 8) {
    fprintf(stderr, "usage: ref_cpu_bench L ngrids nsweeps mag_output_int beta h seed\n");
    return 2;
  }
  int L = atoi(argv[1]), ngrids = atoi(argv[2]), nsweeps = atoi(argv[3]);
  int mag = atoi(argv[4]);
  double beta = atof(argv[5]), h = atof(argv[6]);
  unsigned long seed = strtoul(argv[7], NULL, 10);

  int *grids = init_grids_uniform(L, ngrids, -1);
  float *result = (float *)malloc(sizeof(float) * (size_t)(nsweeps / mag + 1));
  init_genrand(seed);
  preComputeProbs_cpu(beta, h);

  mc_grids_t g; g.L = L; g.ngrids = ngrids; g.ising_grids = grids;
  mc_sampler_t s; s.tot_nsweeps = nsweeps; s.mag_output_int = mag; s.grid_output_int = mag;
  mc_function_t c; memset(&c, 0, sizeof c);
  c.itask = 0; c.dn_thr = -0.90; c.up_thr = 0.90; c.ninputs = 1; c.initial_spin = -1;
  c.cv = (char *)"magnetisation"; c.result = result; c.filename = (char *)"/dev/null";

  if (!freopen("/dev/null", "w", stdout)) return 3;
  struct timespec t0, t1;
  clock_gettime(CLOCK_MONOTONIC, &t0);
  mc_driver_cpu(g, beta, h, NULL, s, c, null_outfunc);
  clock_gettime(CLOCK_MONOTONIC, &t1);
  double wall = (double)(t1.tv_sec - t0.tv_sec) + 1e-9 * (double)(t1.tv_nsec - t0.tv_nsec);
  double attempts = (double)L * L * (double)ngrids * (double)nsweeps;
  fprintf(stderr, "%.0f %.6f\n", attempts, wall);
  free(grids);
  free(result);
  return 0;
}
