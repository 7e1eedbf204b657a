/*
 * gasp.h -- C ABI of gasp-b200, a B200-native (sm_100a) engine for the
 * many-replica 2D Ising Metropolis path of GASP (dquigley533/GPU_2DIsing).
 *
 * Every entry point is extern "C", takes plain pointers and sizes, and returns
 * a status code (GASP_OK == 0) instead of calling exit() as the reference
 * does.  Each declaration names the reference interface it replaces
 * (file:line inside the reference project).  Host grids use the reference's
 * layout: int32 spins (+1/-1), [grid][row][col] (src/grid.c:10).
 *
 * Threading: calls on one handle must not overlap; different handles may be
 * used from different host threads.  All device work of a handle is issued on
 * that handle's CUDA stream (gasp_set_stream).
 */
#ifndef GASP_H
#define GASP_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------------------------------------------------------- status */
enum {
  GASP_OK = 0,
  GASP_ERR_INVALID = 1,     /* bad argument: sizes, method, divisibility      */
  GASP_ERR_CUDA = 2,        /* CUDA runtime error (message via gasp_last_error) */
  GASP_ERR_NO_DEVICE = 3,   /* no CUDA device (reference returns -1, src/gpu_tools.cu:27-29) */
  GASP_ERR_ALLOC = 4,       /* host or device allocation failed               */
  GASP_ERR_IO = 5,          /* file open/read/write failed                    */
  GASP_ERR_FORMAT = 6,      /* file header does not match (src/io.c:25-28)    */
  GASP_ERR_CALLBACK = 7,    /* user output callback returned non-zero         */
  GASP_ERR_UNSUPPORTED = 8, /* e.g. L above 8192 or an unknown cv name          */
  GASP_ERR_TIMEOUT = 9      /* a bounded device-side wait expired             */
};

/* Human-readable text for a status code. */
const char *gasp_status_string(int status);
/* Detail of the last error raised on the calling host thread. */
const char *gasp_last_error(void);
/* Library version string. */
const char *gasp_version(void);

/* --------------------------------------------------------------- device */
/* Replaces gpuInitDevice (include/gpu_tools.h:16, src/gpu_tools.cu:18-99):
 * selects device_index (-1 keeps the current device), reports the device in
 * use and its SM count.  verbose != 0 prints the reference's device summary. */
int gasp_init_device(int device_index, int verbose, int *device_out, int *nsms_out);

/* Replaces select_gpu_method (include/gpu_tools.h:38, src/gpu_tools.cu:205-232):
 * the reference's rule, evaluated against the device's default per-block
 * shared memory (method 2 if it fits, else 0). */
int gasp_select_gpu_method(int L, int ngrids, int threads_per_block, int gpu_device,
                           int *method_out);

/* Replaces preComputeProbs_gpu (include/mc_gpu.h:28, src/mc_gpu.cu:21-37):
 * the 20-slot float acceptance table exp(-beta*2*s*(nsum+h)) computed with the
 * host expf exactly as the reference does; index 5*(s+1)+nsum+4. */
int gasp_acceptance_table(double beta, double h, float table_out[20]);

/* Largest L swept in shared memory on this device; larger lattices (up to
 * L = 8192, the reference's MAXL) are swept in place in HBM, the role of the
 * reference's global-memory method 0. */
int gasp_max_shared_L(int device, int *maxL_out);

/* Makes subsequent device work of this thread's handles go to `stream`
 * (a cudaStream_t; NULL restores the library's own stream). */
int gasp_set_stream(void *stream);

/* ----------------------------------------------------- device grid sets */
/* Opaque device-resident replica set: bit-packed lattices, magnetisation,
 * fates.  Replaces the raw int* d_ising_grids + d_neighbour_list pair of
 * mc_gpu_grids_t (include/mc_gpu.h:12-18). */
typedef struct gasp_grids gasp_grids_t;

/* Replaces gpuInitGrid (include/gpu_tools.h:19, src/gpu_tools.cu:143-159):
 * allocates the device set for ngrids LxL replicas and uploads host_grids
 * (may be NULL: all spins -1).  threads_per_block is accepted for signature
 * parity; the kernels choose their own launch shape. */
int gasp_init_grid(int L, int ngrids, int threads_per_block, const int *host_grids,
                   gasp_grids_t **grids_out);
/* Frees a grid set (replaces the cudaFree calls of src/ising.cu:191-193). */
int gasp_free_grid(gasp_grids_t *grids);
/* Host <-> device copies of all replicas in the reference's int32 layout. */
int gasp_grids_upload(gasp_grids_t *grids, const int *host_grids);
int gasp_grids_download(gasp_grids_t *grids, int *host_grids);
/* Device-side form of init_grids_from_array (src/grid.c:41-71) + upload:
 * `inputs` holds ninputs LxL grids (int32); replica r starts from input
 * r / (ngrids/ninputs).  Only the distinct inputs cross PCIe. */
int gasp_grids_upload_inputs(gasp_grids_t *grids, const int *inputs, int ninputs);
/* Same result as gasp_grids_upload_inputs, allocating no memory: the inputs
 * are staged in one fixed device array of GASP_NOALLOC_MAX_INPUT_INTS int32
 * (1 MiB; 64 inputs at L=64) instead of a buffer sized for the whole set.
 * For callers that cannot allocate: a set filling most of the device, or a
 * shooting loop that must not let cudaMalloc/cudaFree synchronise the device
 * under work on other streams.  No counterpart in the reference.
 * - ninputs * L * L above GASP_NOALLOC_MAX_INPUT_INTS -> GASP_ERR_INVALID
 *   with a message naming the limit; nothing is copied.
 * - Nothing has to start at zero: each call overwrites the staged inputs.
 * - The first call on each device looks up the array's device address and
 *   keeps it for the life of the process; make that first call before any
 *   stream capture.  After cudaDeviceReset the kept address is stale: a
 *   process that resets a device must not call this function again.
 * - Like the other gasp_grids_* calls, it leaves grids->device current.
 * - There is one array per device: calls that overlap in time (two host
 *   threads, or a call while another is still running) race on it.  Calls
 *   that follow one another are safe, as each waits for its copy and pack
 *   on the current stream before returning. */
#define GASP_NOALLOC_MAX_INPUT_INTS (1 << 18)
int gasp_grids_upload_inputs_noalloc(gasp_grids_t *grids, const int *inputs, int ninputs);
/* Replica count / side length of a set. */
int gasp_grids_shape(const gasp_grids_t *grids, int *L_out, int *ngrids_out);

/* Launch tuning of a set (no reference counterpart; results never depend on
 * it, except that variant 6 and GASP_OPT_TAIL_REPLICAS assign the MWC64X
 * stream's draws to attempts differently: same dynamics, other trajectories).  GASP_OPT_SWEEP_VARIANT: 0 the fastest kernel for L (default: for
 * L = 32, 64, 96, 128 the row kernel writing the centre word back on every
 * attempt, no divergent branch), 1 the generic kernel, 2 the row kernel with a
 * store only on acceptance, 5 the generic
 * kernel writing the centre word back on every attempt, 6 one warp per
 * replica (3 <= L <= 512; GASP_ERR_UNSUPPORTED otherwise): the warp applies
 * up to 32 queued attempts of its replica per step, all those that touch no
 * site or neighbour of another, in the order drawn -- on the XORWOW stream
 * the attempts are drawn in the replica's own order, so the result is
 * bit-identical to variant 0; on MWC64X each lane draws from its own
 * substream, the same dynamics as the other variants with a different
 * assignment of draws, ~5x less time per sweep of a single replica, at a
 * quarter of the throughput per SM when many replicas are live; 7 the multispin
 * shared-site sweep (MWC64X stream only, integer thresholds, no active
 * list; GASP_ERR_UNSUPPORTED otherwise): the 32 replicas of a tile share each
 * attempt's site, held as one word per site, neighbour counts by bitwise
 * full adders, per-replica acceptance draws, a ballot flip mask -- replicas
 * of a tile are correlated; about half the throughput of variant 0;
 * 9 variant 0 with each tile staged between HBM and shared memory by one
 * bulk copy (cp.async.bulk, completion on an mbarrier) instead of per-lane
 * loads and stores (L = 32, 64, 96, 128 in replica order, i.e. without an
 * active list; bit-identical to 0, measured slower; each launch reads back
 * a device flag, so a copy that did not complete within its bounded wait
 * returns GASP_ERR_TIMEOUT); 10 variant 0 with one block of attempts per
 * loop iteration (half the loop's code, for kernels that share an SM's
 * instruction cache with other kernels -- the batched groups use it; on the
 * MWC64X stream it differs from 0 only at L = 64).  Values 3, 4 and 8 (retired kernels that
 * were measured slower) and values outside 0..10 return GASP_ERR_INVALID.
 * GASP_OPT_WARPS_PER_CTA: tiles per CTA of the generic kernel (1..8).
 * GASP_OPT_TAIL_REPLICAS: device-side committor shooting (itask 1 with
 * compaction) sweeps with variant 6 once at most this many replicas are
 * undecided (default 4096 on the MWC64X stream, 1024 on XORWOW; 0: never).
 * On the XORWOW stream the trajectories stay bit-identical to the
 * reference's either way. */
enum { GASP_OPT_SWEEP_VARIANT = 1, GASP_OPT_WARPS_PER_CTA = 2, GASP_OPT_TAIL_REPLICAS = 3 };
int gasp_grids_set_option(gasp_grids_t *grids, int option, int value);

/* ------------------------------------------------------------ RNG states */
/* Opaque per-replica XORWOW states (cuRAND device API), replaces curandState*. */
typedef struct gasp_rng gasp_rng_t;

/* Replaces gpuInitRand (include/gpu_tools.h:22, src/gpu_tools.cu:162-174):
 * curand_init(seed, subsequence = replica index, offset 0) per replica, so a
 * replica's stream is independent of the launch shape, exactly as the
 * reference. */
int gasp_init_rand(int ngrids, int threads_per_block, unsigned long long seed,
                   gasp_rng_t **rng_out);

/* RNG kinds.  GASP_RNG_XORWOW is the reference's stream (gpuInitRand);
 * GASP_RNG_MWC64X is the production stream (no reference counterpart): per
 * replica an MWC64X generator, non-overlapping substreams 2^40 draws apart,
 * integer site selection.  Sweeps with an MWC64X state are statistically,
 * not bitwise, equivalent to the reference and about twice as fast. */
enum { GASP_RNG_XORWOW = 0, GASP_RNG_MWC64X = 1 };
int gasp_init_rand_mode(int ngrids, int threads_per_block, unsigned long long seed, int kind,
                        gasp_rng_t **rng_out);
/* Host-only: the MWC64X start states gasp_init_rand_mode uploads, x of
 * replica r at out[r] and carry at out[stride + r] (2*stride words). */
int gasp_mwc64x_seed_states(unsigned long long seed, int ngrids, int stride, uint32_t *out);
/* The integer acceptance thresholds the sweep kernels use for (beta, h) on
 * this set's device: an attempt at class c = 5*(spin up) + (# up neighbours)
 * accepts iff its raw 32-bit draw u <= thr10[c], which is exactly
 * curand_uniform-style "u2 < P" of the reference's float table.
 * *float_compare (optional) is set when some class can never accept and the
 * kernels compare in float instead. */
int gasp_acceptance_thresholds(gasp_grids_t *grids, double beta, double h, uint32_t *thr10,
                               int *float_compare);
/* Host-only: the lane substream multipliers of sweep variant 6: lane j of a
 * replica with MWC64X state X = x*A + c starts at X * mul32[j] mod M
 * (mul32[j] = A^(j*2^35)); inv32[j] = A^-(j*2^35) mod M.  A = 4294883355,
 * M = A*2^32 - 1. */
int gasp_mwc64x_lane_multipliers(uint64_t *mul32, uint64_t *inv32);
/* Copies an RNG set's device states to the host: the XORWOW layout of
 * gasp_init_rand (6 words per replica) or the MWC64X layout of
 * gasp_mwc64x_seed_states (x at [r], carry at [stride + r]), stride = ngrids
 * rounded up to 32.  nwords must cover words * stride. */
int gasp_rng_read_states(const gasp_rng_t *rng, uint32_t *out, long long nwords);
int gasp_free_rand(gasp_rng_t *rng);

/* ------------------------------------------------------------ kernels */
/* Sweep modes. */
enum {
  /* Reference-exact: per-replica cuRAND XORWOW stream, two draws per attempt,
   * site = floor(fl((1-FLT_EPSILON)*L*L) * u1), accept iff u2 < P (float).
   * Bit-identical to mc_sweep_gpu (method 0), mc_sweep_gpu_bitrep (method 1)
   * and mc_sweep_gpu_bitmap32 (method 2) for the same seed. */
  GASP_MODE_EXACT = 0,
  /* CPU-trace: consumes a caller-supplied stream of doubles (row-u, col-u, xi
   * per attempt) with mc_sweep_cpu's arithmetic (src/mc_cpu.c:41-89).
   * Bit-identical to the reference CPU path fed the same stream. */
  GASP_MODE_TRACE_CPU = 1
};

/* One sweep batch: every replica does L*L*nsweeps attempted flips
 * (replaces one launch of the mc_sweep_gpu* kernels, include/mc_gpu.h:35-38,
 * launched from src/mc_gpu.cu:679-706).  gpu_method (0, 1, 2) is accepted for
 * parity; all three map to the exact kernel, which reproduces each of them.
 * mag_out (device or NULL) receives each replica's magnetisation after the
 * batch.  Asynchronous on the handle's stream. */
int gasp_sweep(gasp_grids_t *grids, gasp_rng_t *rng, double beta, double h, int nsweeps,
               int gpu_method);

/* CPU-trace sweep: stream holds, for replica r, 3*L*L*nsweeps doubles starting
 * at stream[r * 3*L*L*nsweeps] (host or device pointer; host is copied). */
int gasp_sweep_trace_cpu(gasp_grids_t *grids, const double *stream, double beta, double h,
                         int nsweeps);

/* Replaces compute_magnetisation_gpu (include/mc_gpu.h:41, src/mc_gpu.cu:437-455):
 * m = (float)(sum of spins) / (float)(L*L) per replica, bit-identical.
 * host_mag receives ngrids floats (synchronous). */
int gasp_magnetisation(gasp_grids_t *grids, float *host_mag);

/* Replaces compute_largest_cluster_gpu (src/mc_gpu.cu:457-526; CPU twin
 * compute_largest_cluster_cpu, src/mc_cpu.c:310-364): size of the largest
 * 4-connected periodic cluster of sites with spin `spin` (+1 or -1; any other
 * value gives 0) per replica, as float.  No user work area: labels live in
 * shared memory up to L=170 and in a library-owned area beyond.
 * host_out receives ngrids floats (synchronous). */
int gasp_largest_cluster(gasp_grids_t *grids, int spin, float *host_out);

/* gridstates.bin frame payload (src/io.c:89-117): ceil(L*L*ngrids/8) bytes,
 * grid-major, row-major, LSB-first, bit 1 iff spin +1.  Packed on the device;
 * host_out receives the bytes (synchronous). */
int gasp_pack_frame(gasp_grids_t *grids, uint8_t *host_out);
size_t gasp_frame_bytes(int L, int ngrids);

/* ----------------------------------------------------------- the driver */
/* Mirrors mc_sampler_t (include/mc_cpu.h:13-17). */
typedef struct {
  int tot_nsweeps;
  int mag_output_int;
  int grid_output_int;
} gasp_sampler_t;

/* Mirrors mc_function_t (include/mc_cpu.h:19-28).  cv: "magnetisation" (also
 * for NULL) or "largest_cluster", the size of the largest cluster of spins
 * -initial_spin, computed at each check (src/mc_gpu.cu:586-605,669-672) and
 * compared with dn_thr/up_thr as a number of sites; other names are rejected
 * with GASP_ERR_UNSUPPORTED (the reference treats them as magnetisation). */
typedef struct {
  int itask;           /* 0 nucleation swarm, 1 committor                  */
  double dn_thr;       /* below: basin A (strict <)                        */
  double up_thr;       /* above: basin B / nucleated (strict >)            */
  int ninputs;         /* committor input blocks (ngrids % ninputs == 0)   */
  int initial_spin;
  const char *cv;
  float *result;       /* itask 0: tot/mag_int floats; itask 1: ninputs    */
  const char *filename;
} gasp_function_t;

/* Mirrors gpu_run_t (include/mc_gpu.h:20-24). */
typedef struct {
  gasp_rng_t *d_state;
  int threadsPerBlock;
  int gpu_method;
} gasp_gpu_run_t;

/* Mirrors mc_gpu_grids_t (include/mc_gpu.h:12-18): ising_grids is the host
 * copy the output callback receives. */
typedef struct {
  int L;
  int ngrids;
  int *ising_grids;
  gasp_grids_t *d_grids;
} gasp_gpu_grids_t;

/* Same signature as GridOutputFunc (include/mc_cpu.h:31).  Non-zero return
 * stops the driver with GASP_ERR_CALLBACK. */
typedef int (*gasp_grid_output_fn)(int L, int ngrids, int *grid_data, int isweep,
                                   float *magnetisation, float *lclus_size, char *cv,
                                   double dn_thr, double up_thr, char *filename);

/* Faster alternative callback: receives the packed gridstates.bin payload of
 * the frame (gasp_frame_bytes bytes) instead of expanded int32 grids. */
typedef int (*gasp_packed_output_fn)(int L, int ngrids, const uint8_t *payload,
                                     size_t nbytes, int isweep,
                                     const float *magnetisation, void *user);

/* Driver options beyond the reference's arguments. */
typedef struct {
  int verbosity;        /* 0 silent; 1 the reference CLI's stdout lines;   
                         * 2 PyGASP's progress line                       */
  int compact;          /* itask 1: stop simulating resolved replicas      */
  gasp_packed_output_fn packed_out; /* if set, used instead of outfunc     */
  void *packed_user;
  double *elapsed_s;    /* if set, receives the driver's wall time          */
  long long *attempts;  /* if set, receives attempted flips simulated       */
  int *first_up;        /* if set (ngrids ints): first check isweep with
                         * cv > up_thr per replica, -1 if never            */
} gasp_driver_opts_t;

/* Replaces mc_driver_gpu (include/mc_gpu.h:47, src/mc_gpu.cu:530-831): the
 * sweep / magnetisation / threshold-check / dump loop with the reference's
 * timing: checks at isweep % mag_output_int == 0 or isweep == tot-1, dumps at
 * isweep % grid_output_int == 0 or isweep == tot-1, sweeps_per_call =
 * min(mag_output_int, grid_output_int); itask 0 fills result with the
 * nucleated fraction (pre-filled with 1.0) and stops when all replicas are
 * above up_thr; itask 1 records absorbing fates (-1 pending, 0 A, 1 B) in
 * grid_fate and writes pB per input block.  outfunc may be NULL. */
int gasp_mc_driver_gpu(gasp_gpu_grids_t grids, double beta, double h, int *grid_fate,
                       gasp_sampler_t samples, gasp_function_t calc, gasp_gpu_run_t gpu_state,
                       gasp_grid_output_fn outfunc);
int gasp_mc_driver_gpu_ex(gasp_gpu_grids_t grids, double beta, double h, int *grid_fate,
                          gasp_sampler_t samples, gasp_function_t calc,
                          gasp_gpu_run_t gpu_state, gasp_grid_output_fn outfunc,
                          const gasp_driver_opts_t *opts);

/* ------------------------------------------ batched groups of uneven L */
/* Several replica groups with their own L, beta and h driven together (no
 * reference counterpart: the reference runs one (L, beta, h) per process). */
typedef struct {
  int L;
  int ngrids;
  double beta;
  double h;
} gasp_group_t;
typedef struct gasp_batch gasp_batch_t;

int gasp_batch_create(const gasp_group_t *groups, int ngroups, unsigned long long seed,
                      int rng_kind, gasp_batch_t **out);
int gasp_batch_free(gasp_batch_t *batch);

enum { GASP_BATCH_PLAIN = 0, GASP_BATCH_GRAPH = 1, GASP_BATCH_MULTI = 2 };
/* Nucleation swarm of every group from all spins -1, re-seeded each call:
 * every check_int sweeps a replica whose magnetisation exceeds up_thr is
 * finished (absorbing).  GASP_BATCH_GRAPH: each interval is one CUDA graph
 * running all groups concurrently, finished replicas compacted out on the
 * device, no host synchronisation until the end.  GASP_BATCH_PLAIN: one launch
 * per group per interval over all its replicas, groups in turn, checks on the
 * host (the comparison path).  GASP_BATCH_MULTI: as GASP_BATCH_GRAPH with
 * the sweeps of all groups in one persistent launch (each CTA runs its
 * group's L-specialised loop; integer thresholds and lattices in shared
 * memory only, else GASP_ERR_UNSUPPORTED); GASP_BATCH_GRAPH uses that layout
 * too when the autotuner found it faster.  All modes give identical counts.
 * counts_out[i*ngroups + g] (tot_nsweeps/check_int rows): finished replicas
 * of group g after interval i.  attempts_out: attempted flips credited to
 * unfinished replicas only (the same workload for both modes). */
int gasp_batch_swarm(gasp_batch_t *batch, int tot_nsweeps, int check_int, double up_thr,
                     int mode, int *counts_out, long long *attempts_out, double *elapsed_out);
/* Autotuner: times the candidate kernels (row kernel with or without the
 * every-attempt store; tiles per CTA of the generic kernel) for each group on
 * an nsweeps run and keeps the fastest; then times the interval graph in both
 * layouts (one kernel per group, or one persistent launch for all groups) on
 * intervals of max(nsweeps, 20) sweeps with all, half and 15 % of every
 * group live, and keeps the faster for GASP_BATCH_GRAPH.  choice_out (2*ngroups ints, may be
 * NULL): (variant, warps per CTA) chosen per group. */
int gasp_batch_autotune(gasp_batch_t *batch, int nsweeps, int *choice_out);
/* The layout the autotuner chose (0: one kernel per group, 1: one persistent
 * launch; -1 for a NULL batch) and its timings of the two (ms over the six
 * timed intervals; -1 when not timed). */
int gasp_batch_layout(const gasp_batch_t *batch, float *ms_per_group_kernels,
                      float *ms_one_launch);

/* ---------------------------------------------- committor surrogate CNN */
/* A small network predicting pB from a spin grid (no reference counterpart):
 * 4 circular 3x3 convolutions (1->32, then 32->32 three times) each with
 * ReLU, global average pool, 32->1 linear, sigmoid; BF16 weights and
 * activations, FP32 accumulation (tcgen05 tensor cores for the
 * convolutions), binomial cross-entropy loss, Adam.  Parameters are a flat
 * FP32 vector of gasp_cnn_param_count() values:
 *   W1[32][9] b1[32] W2[32][9][32] b2[32] W3 b3 W4 b4 Wf[32] bf[1],
 * tap = (dy+1)*3 + (dx+1), W[co][tap][ci].  Spins are int8 +-1, [B][L][L]
 * on the host; L*L must be a multiple of 128. */
typedef struct gasp_cnn gasp_cnn_t;
int gasp_cnn_param_count(void);
int gasp_cnn_create(int L, int max_batch, gasp_cnn_t **out);
int gasp_cnn_free(gasp_cnn_t *cnn);
int gasp_cnn_set_params(gasp_cnn_t *cnn, const float *params);  /* also resets Adam */
int gasp_cnn_get_params(gasp_cnn_t *cnn, float *params);
int gasp_cnn_predict(gasp_cnn_t *cnn, const int8_t *spins, int batch, float *q_out);
/* The same for any number of grids, and (mag_out non-NULL) each grid's
 * magnetisation from the uploaded spins, for out-of-distribution checks
 * before trusting q.  Batches above max_batch run in chunks of max_batch
 * whose uploads overlap the previous chunk's network (the first such call
 * allocates a second input buffer and a copy stream). */
int gasp_cnn_predict_ex(gasp_cnn_t *cnn, const int8_t *spins, int batch, float *q_out,
                        float *mag_out);
/* Prediction path for L = 64: on, the whole network runs as one kernel per
 * band of 8 rows with the activations kept on the chip; off (the default,
 * measured faster so far), layer by layer through HBM as training does.  Same
 * arithmetic either way (BF16 activations, FP32 accumulation); only the order
 * of the pooled FP32 sums differs.  Other L always run layer by layer. */
int gasp_cnn_set_fused(gasp_cnn_t *cnn, int on);
/* Loss (mean over the batch) and its gradient for labels in [0, 1]. */
int gasp_cnn_gradients(gasp_cnn_t *cnn, const int8_t *spins, const float *labels, int batch,
                       float *loss_out, float *grad_out);
/* One Adam step (beta1 0.9, beta2 0.999, eps 1e-8) on the batch. */
int gasp_cnn_train_step(gasp_cnn_t *cnn, const int8_t *spins, const float *labels, int batch,
                        float lr, float *loss_out);

/* ---------------------------------------------------- host-side helpers */
/* Replace init_grids_uniform / init_grids_from_file / init_grids_from_array /
 * init_fates (include/grid.h:5-9, src/grid.c:5-87); caller owns the memory
 * (ngrids*L*L ints, or ngrids ints for fates). */
int gasp_init_grids_uniform(int L, int ngrids, int spin, int *out);
int gasp_init_grids_from_file(const char *path, int L, int ngrids, int *out);
int gasp_init_grids_from_array(int L, int ngrids, int ninputs, const int *array, int *out);
int gasp_init_fates(int ngrids, int *out);

/* Replaces read_input_grid (include/io.h:8, src/io.c:4-65): gridinput.bin
 * (int32 L + ceil(L*L/8) LSB-first bytes) copied into all ngrids grids.
 * GASP_ERR_FORMAT if the file's L differs. */
int gasp_read_input_grid(const char *path, int L, int ngrids, int *out);

/* Replaces write_ising_grids (include/io.h:11, src/io.c:67-130) and has its
 * GridOutputFunc signature: appends one gridstates.bin frame to filename. */
int gasp_write_ising_grids(int L, int ngrids, int *ising_grids, int isweep,
                           float *magnetisation, float *lclus_size, char *cv,
                           double dn_thr, double up_thr, char *filename);
/* Appends a frame from an already packed payload. */
int gasp_write_packed_frame(const char *path, int L, int ngrids, int isweep,
                            const uint8_t *payload, size_t nbytes);
/* Reads frame `iframe` (0-based) of a gridstates.bin file: its header
 * (L, ngrids, isweep) and, when grids_out is not NULL, its spins as int32
 * [ngrids][L][L] (grids_cap ints available).  The frame layout is that of
 * write_ising_grids (src/io.c:89-117): 12-byte header, ceil(L*L*ngrids/8)
 * payload bytes.  GASP_ERR_IO if the file has fewer frames. */
int gasp_read_frame(const char *path, int iframe, int *L_out, int *ngrids_out, int *isweep_out,
                    int *grids_out, long long grids_cap);
/* Writes one grid as gridinput.bin (int32 L, then ceil(L*L/8) bytes
 * LSB-first, bit 1 iff +1): what the viewer's `w` key writes
 * (tools/vis_gridstates.py:109-114) and read_input_grid (src/io.c:4-65)
 * reads.  path NULL: "gridinput.bin". */
int gasp_write_input_grid(const char *path, int L, const int *grid);

/* Replaces create_ising_grids_hdf5 (include/io.h, src/io.c:132-199), the
 * PyGASP side file gridstates.hdf5 / pBgrids.hdf5, written without libhdf5
 * (csrc/gasp_hdf5.c follows the HDF5 file format specification: version 0
 * superblock, version 1 object headers, symbol-table groups): creates or
 * truncates filename with the scalars L, ngrids, tot_nsweeps (int32), h,
 * beta (double) and total_saved_grids = 0.  itask is accepted and unused.
 * GASP_ERR_IO (and the reference's stderr message) if the file cannot be
 * created. */
int gasp_create_ising_grids_hdf5(int L, int ngrids, int tot_nsweeps, double h, double beta,
                                 int itask, const char *filename);
/* Replaces write_ising_grids_hdf5 (src/io.c:201-301) with its GridOutputFunc
 * arguments: appends the group /sweep_<isweep> holding grid_<g> (int32
 * [L][L]) for every replica, each with the string attributes magnetisation
 * and lclus_size ("%g" of the value, "null" when the array is NULL),
 * committor and committor_error ("null"), and adds ngrids to
 * total_saved_grids.  ngrids == 0 writes no group (the reference creates it
 * and deletes it again).  GASP_ERR_IO if the file cannot be opened or
 * already holds /sweep_<isweep>; GASP_ERR_FORMAT if it was not made by
 * gasp_create_ising_grids_hdf5. */
int gasp_write_ising_grids_hdf5(int L, int ngrids, const int *ising_grids, int isweep,
                                const float *magnetisation, const float *lclus_size,
                                const char *cv, double dn_thr, double up_thr,
                                const char *filename);

/* ----------------------------------------------------------- checkpoints */
/* Checkpoint / resume of a run's state (no reference counterpart; the
 * reference can only restart from gridinput.bin, src/io.c:4-65): the grids,
 * every replica's RNG state and optionally the committor fates, with the
 * caller's sweep counter.  Loading into handles of the same L, ngrids and RNG
 * kind continues every replica's trajectory bit for bit.  A driver run
 * resumed from a checkpoint taken at a check boundary reproduces the rest of
 * an uninterrupted run, with its isweep counted from 0 again.
 * gasp_checkpoint_info reads the header so the caller can create the handles. */
int gasp_checkpoint_save(const char *path, gasp_grids_t *grids, gasp_rng_t *rng,
                         const int *fates, int isweep);
int gasp_checkpoint_info(const char *path, int *L_out, int *ngrids_out, int *rng_kind_out,
                         int *isweep_out, int *has_fates_out);
int gasp_checkpoint_load(const char *path, gasp_grids_t *grids, gasp_rng_t *rng,
                         int *fates_out, int *isweep_out);

/* Replaces bootstrap_errbar (include/bootstrap.h:5, src/bootstrap.c:6-65):
 * m resamples with libc rand()%ngrids, population standard deviation.
 * Negative return on allocation failure, as the reference. */
double gasp_bootstrap_errbar(int ngrids, int m, const int *grid_fate);

/* pB per contiguous input block from fates (src/mc_gpu.cu:812-826). */
int gasp_committor_from_fates(int ngrids, int ninputs, const int *grid_fate, float *pB);

#ifdef __cplusplus
}
#endif
#endif /* GASP_H */
