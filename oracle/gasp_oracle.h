/*
 * gasp_oracle.h -- CPU restatement of the GASP hot path, used ONLY as a test
 * checker (tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg).
 * Nothing in the product library links or calls this code.
 *
 * Every function cites the reference file:line whose behaviour it restates.
 * Spin grids are int32, values +1/-1, laid out [grid][row][col] exactly as the
 * reference's host arrays (src/grid.c:10).
 */
#ifndef GASP_ORACLE_H
#define GASP_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Acceptance tables indexed 5*(s+1) + nsum + 4 (20 slots, even ones used). */
void orc_probs_cpu(double beta, double h, double P[20]);  /* src/mc_cpu.c:14-38 */
void orc_probs_gpu(double beta, double h, float P[20]);   /* src/mc_gpu.cu:21-37 */

/* One replica, CPU arithmetic (src/mc_cpu.c:41-89): each attempt consumes
 * three doubles from `stream` (row-u, col-u, xi).  Returns attempts done. */
long long orc_sweep_cpu_stream(int L, int *grid, long long nattempts,
                               const double *stream, const double P[20]);

/* One replica, GPU arithmetic (src/mc_gpu.cu:315-340, identical in
 * src/mc_gpu.cu:106-141 and :220-256): each attempt consumes two floats
 * (u1 -> site via floor(fl((1-FLT_EPSILON)*N) * u1), u2 -> accept if u2 < P). */
long long orc_sweep_gpu_stream(int L, int *grid, long long nattempts,
                               const float *ustream, const float P[20]);

/* Production stream (MWC64X; no reference counterpart).  One replica, one
 * stream (x, c in/out): site = (r * L*L) >> 32 of a draw r, accept iff the
 * next draw u <= thr[5*(spin up) + (# up neighbours)]; attempts in order. */
long long orc_sweep_mwc(int L, int *grid, long long nattempts, uint32_t *x, uint32_t *c,
                        const uint32_t thr[10]);
/* The one-warp-per-replica sweep (variant 6) restated serially: 32 lane
 * substreams (X * mul[j] mod M), the window and conflict rule that fix which
 * lane draws each attempt, attempts applied one at a time in window order,
 * and the replica's state afterwards (x, c in/out).  order (optional) gets
 * (site, u) of every attempt in the order applied.  Returns attempts. */
long long orc_sweep_tail(int L, int *grid, int nsweeps, uint32_t *x, uint32_t *c,
                         const uint32_t thr[10], const uint64_t mul[32], const uint64_t inv[32],
                         uint32_t *order);

/* The multispin shared-site sweep (variant 7) restated serially for one tile
 * of nrep <= 32 replicas: per batch of nrep attempts each replica draws one
 * site and attempt j uses replica j's; then every replica draws its
 * acceptance.  grids [nrep][L*L], x/c [nrep] in/out.  Returns attempts. */
long long orc_sweep_shared(int L, int nrep, int *grids, int nsweeps, uint32_t *x, uint32_t *c,
                           const uint32_t thr[10]);

/* Magnetisation, GPU flavour: float running sum / (float)(L*L)
 * (src/mc_gpu.cu:437-455). */
float orc_magnetisation_gpu(int L, const int *grid);
/* CPU flavour: double sum, (float)(m/(double)N) (src/mc_cpu.c:91-104). */
float orc_magnetisation_cpu(int L, const int *grid);
/* src/mc_cpu.c:310-364: largest periodic 4-connected cluster of `spin`. */
int orc_largest_cluster(int L, const int *grid, int spin);

/* gridstates.bin payload: all grids contiguous, row-major, LSB-first,
 * bit=1 iff spin==+1 (src/io.c:89-117).  Returns bytes written to `out`
 * (ceil(L*L*ngrids/8)); `out` must hold that many. */
long long orc_pack_frame(int L, int ngrids, const int *grids, uint8_t *out);
/* Inverse of orc_pack_frame (bit 1 -> +1, 0 -> -1). */
void orc_unpack_frame(int L, int ngrids, const uint8_t *in, int *grids);

/* Append one gridstates.bin frame: int32 L, int32 ngrids, int32 isweep,
 * then the packed payload (src/io.c:67-130).  0 on success, -1 on I/O error. */
int orc_write_frame(const char *path, int L, int ngrids, const int *grids, int isweep);

/* gridinput.bin: int32 L then ceil(L*L/8) LSB-first bytes; the one grid is
 * copied into all ngrids (src/io.c:4-65, intended semantics: only the first
 * L*L bits are used).  0 ok, -1 open/read error, -2 L mismatch. */
int orc_read_input_grid(const char *path, int L, int ngrids, int *grids);

/* Bootstrap error bar on pB from fates (src/bootstrap.c:6-65).  Uses the
 * process' libc rand() exactly as the reference does. */
double orc_bootstrap_errbar(int ngrids, int m, const int *fate);
/* Reset libc rand() (srand) so two bootstrap calls can be aligned. */
void orc_srand(unsigned int seed);

/* Driver-level committor result (src/mc_gpu.cu:812-826): pB per input block. */
void orc_committor_from_fates(int ngrids, int ninputs, const int *fate, float *pB);

#ifdef __cplusplus
}
#endif
#endif
