/*
 * gasp_cli.c -- the `gasp` command, a drop-in for the reference CLI
 * (src/ising.cu:34-206): same ten positional arguments, same fixed L=64,
 * thresholds -0.90/+0.90 and time-based seed, same stdout lines, same
 * gridstates.bin output (appended per dump) and gridinput.bin input.
 *
 * Optional environment overrides (all default to the reference behaviour):
 *   GASP_SEED  fixed RNG seed        GASP_L      lattice side
 *   GASP_DN    dn_threshold          GASP_UP     up_threshold
 *   GASP_COMPACT=1  itask 1: stop simulating resolved replicas
 *
 * Errors from the library are reported on stderr and end the process with a
 * non-zero status, as the reference's exit() calls do.  There is no CPU
 * fallback: without a CUDA device the command fails.
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

#include "gasp.h"

static int write_packed(int L, int ngrids, const uint8_t *payload, size_t nbytes, int isweep,
                        const float *mag, void *user) {
  (void)mag;
  return gasp_write_packed_frame((const char *)user, L, ngrids, isweep, payload, nbytes);
}

static void die(int rc, const char *what) {
  fprintf(stderr, "gasp: %s failed: %s (%s)\n", what, gasp_status_string(rc), gasp_last_error());
  exit(EXIT_FAILURE);
}

int main(int argc, char *argv[]) {
  int L = 64;
  double dn_threshold = -0.90, up_threshold = 0.90;
  unsigned long long rngseed = (unsigned long long)(long)time(NULL);

  if (argc != 11) {
    printf("Usage : GPU_2DIsing nsweeps nreplicas mag_output_int grid_output_int threadsPerBlock "
           "gpu_device gpu_method beta h itask \n");
    exit(EXIT_FAILURE);
  }
  const int tot_nsweeps = atoi(argv[1]);
  const int ngrids = atoi(argv[2]);
  const int mag_output_int = atoi(argv[3]);
  const int grid_output_int = atoi(argv[4]);
  const int threadsPerBlock = atoi(argv[5]);
  const int gpu_device = atoi(argv[6]);
  const int gpu_method = atoi(argv[7]);
  const double beta = atof(argv[8]);
  const double h = atof(argv[9]);
  const int itask = (int)atof(argv[10]);

  const char *e;
  if ((e = getenv("GASP_SEED"))) rngseed = strtoull(e, NULL, 10);
  if ((e = getenv("GASP_L"))) L = atoi(e);
  if ((e = getenv("GASP_DN"))) dn_threshold = atof(e);
  if ((e = getenv("GASP_UP"))) up_threshold = atof(e);
  const int compact = (e = getenv("GASP_COMPACT")) ? atoi(e) : 0;

  remove("gridstates.bin");
  if (itask == 0) printf("# isweep    nucleated fraction\n");

  if (ngrids <= 0 || L <= 0) {
    fprintf(stderr, "gasp: nreplicas and L must be positive\n");
    exit(EXIT_FAILURE);
  }
  int *ising_grids = (int *)malloc(sizeof(int) * (size_t)L * L * ngrids);
  int *grid_fate = NULL;
  if (!ising_grids) {
    fprintf(stderr, "Error allocating memory for Ising grids!\n");
    exit(EXIT_FAILURE);
  }
  int rc;
  if (itask == 0) {
    gasp_init_grids_uniform(L, ngrids, -1, ising_grids);
  } else if (itask == 1) {
    rc = gasp_init_grids_from_file("gridinput.bin", L, ngrids, ising_grids);
    if (rc == GASP_ERR_FORMAT) {
      fprintf(stderr, "Error - size of grid in input file does not match L!\n");
      exit(EXIT_FAILURE);
    } else if (rc != GASP_OK) {
      fprintf(stderr, "Error opening %s for input!\n", "gridinput.bin");
      exit(EXIT_FAILURE);
    }
    fprintf(stderr, "Read initial configuration of all grids from gridinput.bin\n");
    grid_fate = (int *)malloc(sizeof(int) * (size_t)ngrids);
    if (!grid_fate) {
      printf("Error allocating memory for grid fates\n");
      exit(EXIT_FAILURE);
    }
    gasp_init_fates(ngrids, grid_fate);
  } else {
    printf("Error - unknown value of itask!");
    exit(EXIT_FAILURE);
  }

  int dev = 0, nsms = 0;
  rc = gasp_init_device(gpu_device, 1, &dev, &nsms);
  if (rc != GASP_OK) die(rc, "device initialisation");

  gasp_grids_t *dgrids = NULL;
  gasp_rng_t *rng = NULL;
  if ((rc = gasp_init_grid(L, ngrids, threadsPerBlock, ising_grids, &dgrids))) die(rc, "grid upload");
  if ((rc = gasp_init_rand(ngrids, threadsPerBlock, rngseed, &rng))) die(rc, "RNG initialisation");

  float result = 0.0f;
  gasp_gpu_grids_t grids = {L, ngrids, ising_grids, dgrids};
  gasp_sampler_t samples = {tot_nsweeps, mag_output_int, grid_output_int};
  gasp_function_t calc;
  memset(&calc, 0, sizeof calc);
  calc.itask = itask;
  calc.dn_thr = dn_threshold;
  calc.up_thr = up_threshold;
  calc.ninputs = 1;
  calc.initial_spin = -1;
  calc.cv = "magnetisation";
  calc.result = itask == 0 ? (float *)malloc(sizeof(float) * (size_t)(tot_nsweeps / (mag_output_int > 0 ? mag_output_int : 1) + 1)) : &result;
  calc.filename = "gridstates.bin";
  gasp_gpu_run_t run = {rng, threadsPerBlock, gpu_method};
  gasp_driver_opts_t opts;
  memset(&opts, 0, sizeof opts);
  opts.verbosity = 1;
  opts.compact = compact;
  opts.packed_out = write_packed;
  opts.packed_user = (void *)"gridstates.bin";
  rc = gasp_mc_driver_gpu_ex(grids, beta, h, grid_fate, samples, calc, run, NULL, &opts);
  if (rc != GASP_OK) die(rc, "simulation");

  gasp_free_rand(rng);
  gasp_free_grid(dgrids);
  if (itask == 0) free(calc.result);
  free(grid_fate);
  free(ising_grids);
  return EXIT_SUCCESS;
}
