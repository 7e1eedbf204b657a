/*
 * ref_cpu_bench.c -- project-written timing harness around the reference's
 * unmodified CPU driver (src/mc_cpu.c:106-308, MT19937 from src/mt19937ar.c).
 * TEST/BENCH INFRASTRUCTURE ONLY: bench.py runs one process of this per host
 * core (the reference's MT19937 state is a process global) for its CPU
 * baseline and its `--impl reference` arm.
 *
 * usage: ref_cpu_bench L ngrids nsweeps mag_output_int beta h seed [grid_output_int]
 * prints two lines to stderr:
 *   "<attempts> <wall_seconds>"  attempts actually made (the driver stops
 *                                early once every replica has nucleated)
 *   "T <t0> <isweep> <t> ..."    CLOCK_MONOTONIC seconds at the start and at
 *                                each output callback (every grid_output_int
 *                                sweeps, before that batch is swept), so a
 *                                caller can cut one run into steps
 *   "C <cpu_seconds>"            CPU time the process used in the driver (below
 *                                the wall time when the core was shared)
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

#include "mc_cpu.h"
#include "grid.h"

#define MAX_MARKS 4096
static int n_marks = 0;
static int mark_sweep[MAX_MARKS];
static double mark_time[MAX_MARKS];

static double cpu_s(void) {
  struct timespec t;
  clock_gettime(CLOCK_PROCESS_CPUTIME_ID, &t);
  return (double)t.tv_sec + 1e-9 * (double)t.tv_nsec;
}

static double now_s(void) {
  struct timespec t;
  clock_gettime(CLOCK_MONOTONIC, &t);
  return (double)t.tv_sec + 1e-9 * (double)t.tv_nsec;
}

/* Output callback: writes nothing, records when each batch starts. */
static int mark_outfunc(int L, int ngrids, int *grid_data, int isweep, float *m,
                        float *lc, char *cv, double dn, double up, char *fn) {
  (void)L; (void)ngrids; (void)grid_data; (void)m; (void)lc;
  (void)cv; (void)dn; (void)up; (void)fn;
  if (n_marks < MAX_MARKS) {
    mark_sweep[n_marks] = isweep;
    mark_time[n_marks] = now_s();
    n_marks++;
  }
  return 0;
}

int main(int argc, char **argv) {
  if (argc != 8 && argc != 9) {
    fprintf(stderr,
            "usage: ref_cpu_bench L ngrids nsweeps mag_output_int beta h seed [grid_output_int]\n");
    return 2;
  }
  int L = atoi(argv[1]), ngrids = atoi(argv[2]), nsweeps = atoi(argv[3]);
  int mag = atoi(argv[4]);
  int gint = argc == 9 ? atoi(argv[8]) : mag;
  if (L < 1 || ngrids < 1 || nsweeps < 1 || mag < 1 || gint < 1) return 2;
  const int spc = mag < gint ? mag : gint;  /* sweeps per batch, src/mc_cpu.c:140 */
  double beta = atof(argv[5]), h = atof(argv[6]);
  unsigned long seed = strtoul(argv[7], NULL, 10);

  int *grids = init_grids_uniform(L, ngrids, -1);
  float *result = (float *)malloc(sizeof(float) * (size_t)(nsweeps / mag + 1));
  init_genrand(seed);
  preComputeProbs_cpu(beta, h);

  mc_grids_t g; g.L = L; g.ngrids = ngrids; g.ising_grids = grids;
  mc_sampler_t s; s.tot_nsweeps = nsweeps; s.mag_output_int = mag; s.grid_output_int = gint;
  mc_function_t c; memset(&c, 0, sizeof c);
  c.itask = 0; c.dn_thr = -0.90; c.up_thr = 0.90; c.ninputs = 1; c.initial_spin = -1;
  c.cv = (char *)"magnetisation"; c.result = result; c.filename = (char *)"/dev/null";

  if (!freopen("/dev/null", "w", stdout)) return 3;
  const double c0 = cpu_s();
  const double t0 = now_s();
  mc_driver_cpu(g, beta, h, NULL, s, c, mark_outfunc);
  const double t1 = now_s();
  const double c1 = cpu_s();
  /* The callback runs before each batch (isweep % grid_output_int == 0) and
   * the driver breaks at a check before the callback, so the sweeps made are
   * the last callback's isweep plus one batch, capped at nsweeps. */
  long long done = n_marks ? (long long)mark_sweep[n_marks - 1] + spc : 0;
  if (done > nsweeps) done = nsweeps;
  const double attempts = (double)L * L * (double)ngrids * (double)done;
  fprintf(stderr, "%.0f %.6f\n", attempts, t1 - t0);
  fprintf(stderr, "T %.6f", t0);
  for (int i = 0; i < n_marks; ++i) fprintf(stderr, " %d %.6f", mark_sweep[i], mark_time[i]);
  fprintf(stderr, " %lld %.6f\n", done, t1);
  fprintf(stderr, "C %.6f\n", c1 - c0);
  free(grids);
  free(result);
  return 0;
}
