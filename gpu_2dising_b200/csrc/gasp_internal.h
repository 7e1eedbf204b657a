// gasp_internal.h -- shared host-side declarations of the gasp-b200 library.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>

#include "gasp.h"

namespace gasp {

// Lattice storage ("lane-interleaved bit planes").  Replicas are grouped in
// tiles of 32 (one warp, one replica per lane).  A replica's L*L spins are
// bit-packed row-major into W = ceil(L*L/32) words (site s -> word s>>5,
// bit s&31, bit 1 == spin +1).  Within a tile, word w of lane l sits at
// index w*32 + l, so a warp that reads "its own word w" touches 32
// consecutive words: one coalesced 128 B line in HBM and 32 distinct banks in
// shared memory whatever site each lane picked.
constexpr int kTile = 32;

inline int words_per_replica(int L) { return (L * L + 31) / 32; }
inline int tiles_for(int ngrids) { return (ngrids + kTile - 1) / kTile; }

// Per-replica XORWOW state in structure-of-arrays form: component k of
// replica r at state[k * stride + r], k = 0 (d), 1..5 (v[0..4]).
constexpr int kRngWords = 6;

// Production RNG: MWC64X (D. B. Thomas, "The MWC64X random number generator",
// 2011): state (x, c), step t = A*x + c, x' = t mod 2^32, c' = t >> 32,
// output x ^ c.  Equivalent to X -> X*A mod M with X = x*A + c and
// M = A*2^32 - 1, which gives the skip-ahead used to start replica r's stream
// r * 2^40 draws after the seed's base state (non-overlapping substreams).
constexpr uint32_t kMwcA = 4294883355u;
constexpr int kMwcWords = 2;  // SoA: x at [0*stride + r], c at [1*stride + r]
enum RngKind { kRngXorwow = 0, kRngMwc = 1 };

// Lane substreams of the one-warp-per-replica sweep (gasp_tail.cu): lane j
// starts at the replica's state X times mul[j] = A^(j * 2^35) mod M; a lane's
// end state times inv[j] = A^-(j * 2^35) mod M maps back to the replica's own
// stream.  Built once on the host (gasp_api.cu).
struct TailParams {
  uint64_t mul[32];
  uint64_t inv[32];
};
const TailParams &mwc_lane_params();
constexpr int kTailMaxL = 512;  // shared lattice + bitmap: 2 * W words per warp

void set_error(const char *fmt, ...);
int cuda_fail(cudaError_t e, const char *what, const char *file, int line);

#define GASP_CUDA(call)                                                             \
  do {                                                                              \
    cudaError_t e_ = (call);                                                        \
    if (e_ != cudaSuccess) return ::gasp::cuda_fail(e_, #call, __FILE__, __LINE__); \
  } while (0)

cudaStream_t current_stream();

// Thresholds for the integer acceptance test: replica accepts iff its raw
// 32-bit XORWOW draw x <= thr[class], class = 5*spin01 + (# up neighbours).
// Built on the device from the float table so the comparison is exactly
// "_curand_uniform(x) < P" (see k_build_thresholds).
struct AcceptTable {
  float pacc[20];        // reference float table (src/mc_gpu.cu:21-37)
  double pacc_cpu[20];   // reference double table (src/mc_cpu.c:14-38)
};

struct SweepLaunch {
  uint32_t *lat;          // home lattice words [ntiles][W][32]
  uint32_t *rng;          // SoA XORWOW states
  int rng_stride;         // component stride of rng (>= ngrids)
  const int *active;      // optional replica id list (nullptr: identity)
  int n_active;           // replicas to sweep (slots)
  int L;
  int nsweeps;
  int ngrids;             // replicas in the set
  const uint32_t *thr;    // 10 device thresholds (exact mode)
  const float *pacc_f;    // 20 floats (exact mode, float comparison)
  const double *stream;   // trace mode: per-replica double stream
  const double *pacc_cpu; // trace mode: 20 doubles (device)
  float *mag_out;         // optional: magnetisation after the batch [ngrids]
  int float_compare;      // exact mode: compare in float (thresholds unusable)
  int warps_per_cta;      // launch shape (0: default)
  int variant;            // GASP_OPT_SWEEP_VARIANT (0: fastest kernel for L)
  int rng_kind;           // RngKind of p.rng
  const int *n_active_dev;// optional device count overriding n_active (graph replays)
  int lattice_in_global;  // L beyond shared memory: sweep the lattice in place in HBM
  int tail_split;         // > 0: with n live replicas, the one-warp-per-replica kernel runs
                          // only when n <= tail_split and the other kernels only when
                          // n > tail_split (both are enqueued; the choice is made on the
                          // device, so runs do not depend on host timing)
};

// Sweep parameters of a replica set + RNG whose tables are ready
// (prepare_tables called for the set's beta, h); gasp_api.cu.
SweepLaunch launch_for(gasp_grids_t *g, gasp_rng_t *r);
// Re-seeds an RNG state set in place (gasp_api.cu); its buffer is kept, so
// graphs that captured it stay valid.
int rng_reseed(gasp_rng_t *r, unsigned long long seed);
int prepare_tables(gasp_grids_t *g, double beta, double h);

// Device-side committor check + compaction (gasp_batch.cu): fates of active
// replicas past a threshold, survivors copied in order from active_in to
// active_out (distinct arrays), count and attempts updated on the device.
// max_active bounds *n_active; cnt holds fate_compact_blocks(max_active) + 1
// ints of scratch.
int fate_compact_blocks(int max_active);
int launch_fate_compact(const float *colvar, int *fates, const int *active_in, int *active_out,
                        int *n_active, int *cnt, int max_active, double up_thr, double dn_thr,
                        long long *attempts, long long attempts_per_replica, cudaStream_t s);

// Device-side check + compaction of one replica group (gasp_batch.cu).
int launch_check_compact(const float *mag, int *active, int *n_active, int ngrids,
                         double up_thr, int *counts, int *interval, int max_intervals,
                         cudaStream_t s);

// kernel launchers (gasp_kernels.cu); each returns a GASP status.
int launch_rng_init(uint32_t *rng, int ngrids, int stride, unsigned long long seed, cudaStream_t s);
int launch_build_thresholds(const float *d_pacc20, uint32_t *d_thr10, int *d_flags, cudaStream_t s);
int launch_sweep_exact(const SweepLaunch &p, cudaStream_t s);
int launch_sweep_trace_cpu(const SweepLaunch &p, cudaStream_t s);
// One launch over several groups (gasp_kernels.cu k_sweep_multi): d_groups
// [ngroups] sweep parameters in device memory, d_tile_begin [ngroups + 1] the
// first CTA of each group; integer thresholds, one RNG kind for all.
int launch_sweep_multi(const SweepLaunch *d_groups, const int *d_tile_begin, int ngroups,
                       int total_tiles, int max_L, int rng_kind, cudaStream_t s);
// One warp per replica, either stream (gasp_tail.cu); p.n_active is the
// launch shape (an upper bound of *p.n_active_dev when that is set).
int launch_sweep_tail(const SweepLaunch &p, cudaStream_t s);
// Multispin shared-site sweep, MWC64X stream, no active list (gasp_shared.cu).
int launch_sweep_shared(const SweepLaunch &p, cudaStream_t s);
int launch_measure(const uint32_t *lat, int L, int ngrids, float *mag, cudaStream_t s);
int launch_pack_grids(const int *grids32, uint32_t *lat, int L, int ngrids, cudaStream_t s,
                      int per_input = 0);
int launch_unpack_grids(const uint32_t *lat, int *grids32, int L, int ngrids, cudaStream_t s);
int launch_pack_frame(const uint32_t *lat, uint8_t *frame, int L, int ngrids, cudaStream_t s);
int max_shared_L(int device);

// Largest cluster of `spin` sites per replica (gasp_cluster.cu).  work_bytes
// from largest_cluster_work_bytes: 0 when the labels fit shared memory,
// otherwise the size of the global work area the launcher needs.
size_t largest_cluster_work_bytes(int L, int ngrids, int device);
int launch_largest_cluster(const uint32_t *lat, int L, int ngrids, int spin, int *work,
                           size_t work_bytes, float *out, cudaStream_t s);

}  // namespace gasp

// Opaque handle definitions.
struct gasp_grids {
  int device;
  int L, N, W;
  int ngrids, ntiles;
  uint32_t *d_lat;       // ntiles * W * 32 words
  float *d_mag;          // ngrids
  uint8_t *d_frame;      // frame payload buffer (lazily allocated)
  size_t frame_bytes;
  int *d_scratch32;      // int32 staging (lazily allocated), ngrids*N
  int global_lattice;    // L exceeds the shared-memory sweep: use the HBM path
};

struct gasp_rng {
  int device;
  int ngrids, stride;
  int kind;              // gasp::RngKind
  uint32_t *d_state;     // kRngWords (XORWOW) or kMwcWords (MWC64X) * stride
};
