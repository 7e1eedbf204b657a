/*
 * ref_cpu_harness.c -- project-written glue around the reference's CPU code,
 * which is compiled UNMODIFIED from the reference tree by oracle/Makefile into
 * oracle/_ref/.  TEST INFRASTRUCTURE ONLY (tests/, bench.py cpu_baseline and
 * --impl reference).
 *
 * Two builds link this file:
 *   libref_cpu.so        reference mc_cpu.c + mt19937ar.c + grid.c + bootstrap.c
 *   libref_cpu_replay.so reference mc_cpu.c + grid.c + bootstrap.c, with
 *                        genrand_real3() served from a caller-provided stream
 *                        (REF_REPLAY defined) instead of MT19937.
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "mc_cpu.h"
#include "grid.h"
#include "bootstrap.h"

#include "gasp_oracle.h"

/* ---- capture of the driver's output callback ------------------------- */
static int *cap_grids = NULL;      /* [max_frames][ngrids*L*L] */
static int *cap_isweep = NULL;     /* [max_frames] */
static float *cap_mag = NULL;      /* [max_frames][ngrids] */
static int cap_max = 0, cap_n = 0;

static int capture_outfunc(int L, int ngrids, int *grid_data, int isweep,
                           float *magnetisation, float *lclus_size, char *cv,
                           double dn_thr, double up_thr, char *filename) {
  (void)lclus_size; (void)cv; (void)dn_thr; (void)up_thr; (void)filename;
  if (cap_n < cap_max) {
    size_t n = (size_t)L * L * ngrids;
    if (cap_grids) memcpy(cap_grids + (size_t)cap_n * n, grid_data, n * sizeof(int));
    if (cap_mag) memcpy(cap_mag + (size_t)cap_n * ngrids, magnetisation, ngrids * sizeof(float));
    if (cap_isweep) cap_isweep[cap_n] = isweep;
  }
  cap_n++;
  return 0;
}

/* Runs the reference mc_driver_cpu (src/mc_cpu.c:106-308) on caller grids.
 * Frames passed to the output callback are captured (up to max_frames).
 * Returns the number of callback invocations. */
int ref_driver_cpu(int L, int ngrids, unsigned long seed, double beta, double h,
                   int tot_nsweeps, int mag_output_int, int grid_output_int,
                   int itask, double dn_thr, double up_thr, int ninputs,
                   int *grids_inout, int *fates_inout, float *result,
                   int max_frames, int *frame_grids, int *frame_isweep, float *frame_mag) {
#ifndef REF_REPLAY
  init_genrand(seed);
#else
  (void)seed;
#endif
  preComputeProbs_cpu(beta, h);
  cap_grids = frame_grids; cap_isweep = frame_isweep; cap_mag = frame_mag;
  cap_max = max_frames; cap_n = 0;
  mc_grids_t grids; grids.L = L; grids.ngrids = ngrids; grids.ising_grids = grids_inout;
  mc_sampler_t samples; samples.tot_nsweeps = tot_nsweeps;
  samples.mag_output_int = mag_output_int; samples.grid_output_int = grid_output_int;
  mc_function_t calc; memset(&calc, 0, sizeof calc);
  calc.itask = itask; calc.dn_thr = dn_thr; calc.up_thr = up_thr; calc.ninputs = ninputs;
  calc.initial_spin = -1; calc.cv = (char *)"magnetisation"; calc.result = result;
  calc.filename = (char *)"gridstates.bin";
  mc_driver_cpu(grids, beta, h, fates_inout, samples, calc, capture_outfunc);
  fflush(stdout);
  return cap_n;
}

/* Direct access to single reference routines. */
void ref_precompute_probs_cpu(double beta, double h, double *out20) {
  extern double Pacc[20];
  preComputeProbs_cpu(beta, h);
  memcpy(out20, Pacc, 20 * sizeof(double));
}

void ref_sweep_cpu(int L, int *grids, int igrid, double beta, double h, int nsweeps) {
  preComputeProbs_cpu(beta, h);
  mc_sweep_cpu(L, grids, igrid, beta, h, nsweeps);
}

float ref_magnetisation_cpu(int L, int *grids, int igrid) {
  float m[1];
  /* compute_magnetisation_cpu writes magnetisation[grid_index]; give it a
   * base pointer such that index igrid lands in m[0]. */
  float *base = m - igrid;
  compute_magnetisation_cpu(L, grids, igrid, base);
  return m[0];
}

double ref_bootstrap_errbar(int ngrids, int m, int *fates) {
  return bootstrap_errbar(ngrids, m, fates);
}

int ref_init_grids_from_array(int L, int ngrids, int ninputs, int *array, int *out) {
  int *g = init_grids_from_array(L, ngrids, ninputs, array);
  if (!g) return -1;
  memcpy(out, g, sizeof(int) * (size_t)L * L * ngrids);
  free(g);
  return 0;
}

#ifndef REF_REPLAY
unsigned long ref_genrand_int32(void) { return genrand_int32(); }
double ref_genrand_real3(void) { return genrand_real3(); }
void ref_init_genrand(unsigned long s) { init_genrand(s); }
#endif

/* grid.c's init_grids_from_file calls io.c's read_input_grid, which cannot be
 * compiled here (it shares a file with the HDF5 writer).  This forwards to the
 * restated reader on the same fixed file name (src/io.c:9-11). */
void read_input_grid(int L, int ngrids, int *ising_grids) {
  int rc = orc_read_input_grid("gridinput.bin", L, ngrids, ising_grids);
  if (rc != 0) {
    fprintf(stderr, "Error reading gridinput.bin (%d)\n", rc);
    exit(EXIT_FAILURE);
  }
}

#ifdef REF_REPLAY
/* ---- replayed genrand_real3 ------------------------------------------- */
static const double *rp_buf = NULL;
static long long rp_n = 0, rp_pos = 0;
static int rp_overrun = 0;

void ref_replay_set(const double *buf, long long n) { rp_buf = buf; rp_n = n; rp_pos = 0; rp_overrun = 0; }
long long ref_replay_pos(void) { return rp_pos; }
int ref_replay_overrun(void) { return rp_overrun; }

double genrand_real3(void) {
  if (rp_pos < rp_n) return rp_buf[rp_pos++];
  rp_overrun = 1;
  return 0.5;
}
#endif
