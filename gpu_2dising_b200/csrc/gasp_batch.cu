// gasp_batch.cu -- several replica groups of uneven L, beta and h driven
// together (the reference runs one (L, beta, h) per process).
//
// GASP_BATCH_GRAPH: each check interval is one CUDA graph.  Every group has a
// parallel branch [sweep kernel over its active replicas -> device-side
// check + compaction], so all groups share the GPU at once; replicas that
// have nucleated (magnetisation > up_thr at a check, absorbing) leave the
// active list and are never swept again.  The active counts live on the
// device, so the host only replays the graph: no per-interval sync.
// GASP_BATCH_PLAIN: one launch per group per interval over all of its
// replicas, groups one after another, checks on the host (the comparison
// path: what running each group with the single-group driver amounts to).
#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstring>
#include <vector>

#include "gasp_internal.h"

namespace gasp {
namespace {

constexpr int kCheckThreads = 1024;
constexpr int kCheckPerThread = 16;

// Block-wide exclusive scan of one int per thread (1024 threads).
__device__ __forceinline__ int block_exclusive_scan(int v, int *warp_sums, int *total) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) warp_sums[warp] = x;
  __syncthreads();
  if (warp == 0) {
    int w = warp_sums[lane];
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, w, o);
      if (lane >= o) w += y;
    }
    warp_sums[lane] = w;  // inclusive
    if (lane == 31) *total = w;
  }
  __syncthreads();
  const int before = warp > 0 ? warp_sums[warp - 1] : 0;
  return before + x - v;
}

// Stable in-place compaction of the active list: replicas whose magnetisation
// exceeds up_thr are finished.  Each round reads its entries into registers
// before any thread writes, and writes never pass the read cursor.
__global__ void __launch_bounds__(kCheckThreads)
    k_check_compact(const float *mag, int *active, int *n_active, int ngrids, double up_thr,
                    int *counts, int *interval, int max_intervals) {
  __shared__ int warp_sums[32];
  __shared__ int round_total;
  __shared__ int out_base;
  const int n = *n_active;
  if (threadIdx.x == 0) out_base = 0;
  __syncthreads();
  for (int start = 0; start < n; start += kCheckThreads * kCheckPerThread) {
    int ids[kCheckPerThread];
    int keep = 0;
    const int first = start + threadIdx.x * kCheckPerThread;
#pragma unroll
    for (int j = 0; j < kCheckPerThread; ++j) {
      const int i = first + j;
      int id = -1;
      if (i < n) {
        id = active[i];
        if (!((double)mag[id] > up_thr)) keep++;
        else id = -1;
      }
      ids[j] = id;
    }
    const int off = block_exclusive_scan(keep, warp_sums, &round_total);
    const int base = out_base;
    int o = base + off;
#pragma unroll
    for (int j = 0; j < kCheckPerThread; ++j)
      if (ids[j] >= 0) active[o++] = ids[j];
    __syncthreads();
    if (threadIdx.x == 0) out_base = base + round_total;
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    *n_active = out_base;
    const int iv = *interval;
    if (iv < max_intervals) counts[iv] = ngrids - out_base;
    *interval = iv + 1;
  }
}

// Committor check on the device (the driver's itask-1 check, src/mc_gpu.cu:
// 744-750): every active replica whose colvar is above up_thr (B) or below
// dn_thr (A) gets its fate and leaves the active list, which is compacted
// stably from active_in to active_out by many CTAs in two kernels.
// k_fate_count: each CTA takes 4096 consecutive entries, records the fates
// and counts its survivors (cnt[b]); CTA 0 also keeps the live count it saw
// in cnt[nblocks], so the scatter needs no read of *n_active while CTA 0
// rewrites it.  k_fate_scatter: each CTA sums the counts of the CTAs before
// it and writes its survivors, in order, at that offset; CTA 0 sets the new
// count and adds the attempts of the sweep that follows (survivors x
// attempts_per_replica).
constexpr int kFateThreads = 1024;
constexpr int kFatePer = 4;
constexpr int kFateChunk = kFateThreads * kFatePer;

__device__ __forceinline__ bool fate_keep(float colvar, double up_thr, double dn_thr) {
  const double m = (double)colvar;
  return !(m > up_thr) && !(m < dn_thr);
}

__global__ void __launch_bounds__(kFateThreads)
    k_fate_count(const float *colvar, int *fates, const int *active, const int *n_active,
                 double up_thr, double dn_thr, int *cnt) {
  __shared__ int warp_sums[32];
  __shared__ int total;
  const int n = *n_active;
  const int first = blockIdx.x * kFateChunk + threadIdx.x * kFatePer;
  int keep = 0;
#pragma unroll
  for (int j = 0; j < kFatePer; ++j) {
    const int i = first + j;
    if (i < n) {
      const int id = active[i];
      const double m = (double)colvar[id];
      if (m > up_thr) fates[id] = 1;
      else if (m < dn_thr) fates[id] = 0;
      else ++keep;
    }
  }
  block_exclusive_scan(keep, warp_sums, &total);
  if (threadIdx.x == 0) {
    cnt[blockIdx.x] = total;
    if (blockIdx.x == 0) cnt[gridDim.x] = n;
  }
}

__global__ void __launch_bounds__(kFateThreads)
    k_fate_scatter(const float *colvar, const int *active_in, int *active_out, int *n_active,
                   const int *cnt, double up_thr, double dn_thr, long long *attempts,
                   long long attempts_per_replica) {
  __shared__ int warp_sums[32];
  __shared__ int total;
  __shared__ int base;
  const int n = cnt[gridDim.x];
  const int lane = threadIdx.x & 31;
  if (threadIdx.x < 32) {  // survivors of the CTAs before this one
    int sum = 0;
    for (int b = lane; b < (int)blockIdx.x; b += 32) sum += cnt[b];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, o);
    if (lane == 0) base = sum;
  }
  const int first = blockIdx.x * kFateChunk + threadIdx.x * kFatePer;
  int ids[kFatePer];
  int keep = 0;
#pragma unroll
  for (int j = 0; j < kFatePer; ++j) {
    const int i = first + j;
    ids[j] = -1;
    if (i < n) {
      const int id = active_in[i];
      if (fate_keep(colvar[id], up_thr, dn_thr)) {
        ids[j] = id;
        ++keep;
      }
    }
  }
  const int off = block_exclusive_scan(keep, warp_sums, &total);  // also orders `base`
  int o = base + off;
#pragma unroll
  for (int j = 0; j < kFatePer; ++j)
    if (ids[j] >= 0) active_out[o++] = ids[j];
  if (blockIdx.x == 0 && threadIdx.x < 32) {
    int sum = 0;
    for (int b = lane; b < (int)gridDim.x; b += 32) sum += cnt[b];
#pragma unroll
    for (int o2 = 16; o2 > 0; o2 >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, o2);
    if (lane == 0) {
      *n_active = sum;
      *attempts += (long long)sum * attempts_per_replica;
    }
  }
}

__global__ void k_iota(int *a, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) a[i] = i;
}

}  // namespace

int fate_compact_blocks(int max_active) { return (max_active + kFateChunk - 1) / kFateChunk; }

int launch_fate_compact(const float *colvar, int *fates, const int *active_in, int *active_out,
                        int *n_active, int *cnt, int max_active, double up_thr, double dn_thr,
                        long long *attempts, long long attempts_per_replica, cudaStream_t s) {
  const int nblk = fate_compact_blocks(max_active);
  if (nblk <= 0) return GASP_OK;
  k_fate_count<<<nblk, kFateThreads, 0, s>>>(colvar, fates, active_in, n_active, up_thr, dn_thr,
                                             cnt);
  GASP_CUDA(cudaGetLastError());
  k_fate_scatter<<<nblk, kFateThreads, 0, s>>>(colvar, active_in, active_out, n_active, cnt,
                                               up_thr, dn_thr, attempts, attempts_per_replica);
  GASP_CUDA(cudaGetLastError());
  return GASP_OK;
}

int launch_check_compact(const float *mag, int *active, int *n_active, int ngrids, double up_thr,
                         int *counts, int *interval, int max_intervals, cudaStream_t s) {
  k_check_compact<<<1, kCheckThreads, 0, s>>>(mag, active, n_active, ngrids, up_thr, counts,
                                              interval, max_intervals);
  GASP_CUDA(cudaGetLastError());
  return GASP_OK;
}

}  // namespace gasp

using namespace gasp;

struct gasp_batch {
  int device;
  int ngroups;
  unsigned long long seed;
  int rng_kind;
  std::vector<gasp_group_t> groups;
  std::vector<gasp_grids_t *> grids;
  std::vector<gasp_rng_t *> rngs;
  std::vector<int *> d_active;
  int *d_small = nullptr;   // per group: [n_active, interval]
  int *d_counts = nullptr;  // [ngroups][max_intervals]
  int max_intervals = 0;
  std::vector<cudaStream_t> streams;
  std::vector<cudaEvent_t> events;  // fork + one join per group
  cudaStream_t origin = nullptr;    // capture/launch stream (never the legacy default)
  cudaGraphExec_t exec = nullptr;
  int graph_check_int = -1;
  double graph_up = 0.0;
  int graph_layout = -1;
  // Sweep layout of the graph: 0 one kernel per group (concurrent branches),
  // 1 all groups in one persistent launch (k_sweep_multi).  Set by the autotuner.
  int layout = 0;
  SweepLaunch *d_multi = nullptr;  // [ngroups] sweep parameters, largest L first
  int *d_tile_begin = nullptr;     // [ngroups + 1]
  int multi_tiles = 0, multi_max_L = 0;
  float layout_ms[2] = {-1.f, -1.f};  // autotuner's timing of the two layouts
};

namespace {

struct StreamRestore {
  cudaStream_t prev = current_stream();
  ~StreamRestore() { gasp_set_stream(prev); }
};

int batch_release(gasp_batch *b) {
  if (!b) return GASP_OK;
  if (b->exec) cudaGraphExecDestroy(b->exec);
  for (auto *g : b->grids) gasp_free_grid(g);
  for (auto *r : b->rngs) gasp_free_rand(r);
  for (auto *a : b->d_active) cudaFree(a);
  cudaFree(b->d_small);
  cudaFree(b->d_counts);
  cudaFree(b->d_multi);
  cudaFree(b->d_tile_begin);
  for (auto s : b->streams) cudaStreamDestroy(s);
  if (b->origin) cudaStreamDestroy(b->origin);
  for (auto e : b->events) cudaEventDestroy(e);
  delete b;
  return GASP_OK;
}

// Fresh start for a run: all spins -1, RNG streams re-seeded, all replicas
// active, interval counters zero.
int batch_reset(gasp_batch *b, cudaStream_t s) {
  for (int g = 0; g < b->ngroups; ++g) {
    gasp_grids_t *gr = b->grids[g];
    const size_t words = (size_t)gr->ntiles * gr->W * kTile;
    GASP_CUDA(cudaMemsetAsync(gr->d_lat, 0, words * sizeof(uint32_t), s));
    // re-seeded in place: a captured graph keeps pointing at these states
    gasp_set_stream(s);
    const unsigned long long seed = b->seed + 1000003ull * (unsigned)g;
    const int rc = b->rngs[g] ? rng_reseed(b->rngs[g], seed)
                              : gasp_init_rand_mode(gr->ngrids, 32, seed, b->rng_kind, &b->rngs[g]);
    if (rc) return rc;
    k_iota<<<(gr->ngrids + 255) / 256, 256, 0, s>>>(b->d_active[g], gr->ngrids);
    GASP_CUDA(cudaGetLastError());
  }
  std::vector<int> small((size_t)2 * b->ngroups, 0);
  for (int g = 0; g < b->ngroups; ++g) small[2 * g] = b->groups[g].ngrids;
  GASP_CUDA(cudaMemcpyAsync(b->d_small, small.data(), small.size() * sizeof(int),
                            cudaMemcpyHostToDevice, s));
  GASP_CUDA(cudaStreamSynchronize(s));
  return GASP_OK;
}

SweepLaunch group_launch(gasp_batch *b, int g, int nsweeps) {
  SweepLaunch p = launch_for(b->grids[g], b->rngs[g]);
  p.nsweeps = nsweeps;
  // The groups' kernels run side by side on the SMs: the row kernels' compact
  // form (one block of attempts per loop iteration) keeps their code within
  // the instruction cache.  Five-group uneven batch, 1000 sweeps: graph
  // 1.10 s compact against 1.26 s with the two-block form, one persistent
  // launch 1.04 s against 1.20 s (plain per-group launches, which run one
  // kernel at a time, keep the two-block form: 2.08 s).
  if (p.variant == 0) p.variant = 10;
  p.active = b->d_active[g];
  p.n_active = b->groups[g].ngrids;  // grid size; the live count is read on the device
  p.n_active_dev = b->d_small + 2 * g;
  p.mag_out = b->grids[g]->d_mag;
  return p;
}

// Can every group run in one persistent launch?  (integer thresholds and
// lattices in shared memory; the tables must be prepared)
bool multi_possible(gasp_batch *b) {
  for (int g = 0; g < b->ngroups; ++g) {
    const SweepLaunch p = launch_for(b->grids[g], b->rngs[g]);
    if (p.float_compare || p.lattice_in_global) return false;
  }
  return true;
}

// Uploads the groups' sweep parameters for k_sweep_multi, largest L first
// (longest chains start first).  Synchronous; not while capturing.
int batch_prepare_multi(gasp_batch *b, int check_int, cudaStream_t s) {
  std::vector<int> order((size_t)b->ngroups);
  for (int g = 0; g < b->ngroups; ++g) order[(size_t)g] = g;
  std::stable_sort(order.begin(), order.end(),
                   [&](int x, int y) { return b->groups[x].L > b->groups[y].L; });
  std::vector<SweepLaunch> ps;
  std::vector<int> begin(1, 0);
  int max_L = 0;
  for (int g : order) {
    ps.push_back(group_launch(b, g, check_int));
    begin.push_back(begin.back() + tiles_for(b->groups[g].ngrids));
    if (b->groups[g].L > max_L) max_L = b->groups[g].L;
  }
  if (!b->d_multi) {
    GASP_CUDA(cudaMalloc(&b->d_multi, (size_t)b->ngroups * sizeof(SweepLaunch)));
    GASP_CUDA(cudaMalloc(&b->d_tile_begin, (size_t)(b->ngroups + 1) * sizeof(int)));
  }
  GASP_CUDA(cudaMemcpyAsync(b->d_multi, ps.data(), ps.size() * sizeof(SweepLaunch),
                            cudaMemcpyHostToDevice, s));
  GASP_CUDA(cudaMemcpyAsync(b->d_tile_begin, begin.data(), begin.size() * sizeof(int),
                            cudaMemcpyHostToDevice, s));
  GASP_CUDA(cudaStreamSynchronize(s));
  b->multi_tiles = begin.back();
  b->multi_max_L = max_L;
  return GASP_OK;
}

// One interval of all groups, issued on the per-group streams (captured into
// the graph by the caller).  layout 1: the sweeps of all groups are one
// k_sweep_multi launch on the origin stream (batch_prepare_multi first), the
// checks still one branch per group.
int batch_issue_interval(gasp_batch *b, cudaStream_t origin, int check_int, double up,
                         int layout) {
  if (layout == 1) {
    const int rc = launch_sweep_multi(b->d_multi, b->d_tile_begin, b->ngroups, b->multi_tiles,
                                      b->multi_max_L, b->rng_kind == GASP_RNG_MWC64X ? kRngMwc
                                                                                     : kRngXorwow,
                                      origin);
    if (rc) return rc;
  }
  GASP_CUDA(cudaEventRecord(b->events[0], origin));
  for (int g = 0; g < b->ngroups; ++g) {
    cudaStream_t sg = b->streams[g];
    GASP_CUDA(cudaStreamWaitEvent(sg, b->events[0], 0));
    int rc = GASP_OK;
    if (layout != 1) {
      const SweepLaunch p = group_launch(b, g, check_int);
      rc = launch_sweep_exact(p, sg);
      if (rc) return rc;
    }
    rc = launch_check_compact(b->grids[g]->d_mag, b->d_active[g], b->d_small + 2 * g,
                              b->groups[g].ngrids, up, b->d_counts + (size_t)g * b->max_intervals,
                              b->d_small + 2 * g + 1, b->max_intervals, sg);
    if (rc) return rc;
    GASP_CUDA(cudaEventRecord(b->events[1 + g], sg));
    GASP_CUDA(cudaStreamWaitEvent(origin, b->events[1 + g], 0));
  }
  return GASP_OK;
}

// The interval graph for (check_int, up, layout), captured once and cached.
// Leaves the batch reset (an uncaptured warm-up interval sets the kernels'
// launch attributes first).  The tables must be prepared.
int batch_build_graph(gasp_batch *b, cudaStream_t s, int check_int, double up, int layout) {
  if (b->exec && b->graph_check_int == check_int && b->graph_up == up &&
      b->graph_layout == layout)
    return GASP_OK;
  if (b->exec) {
    cudaGraphExecDestroy(b->exec);
    b->exec = nullptr;
  }
  int rc;
  if (layout == 1 && (rc = batch_prepare_multi(b, check_int, s))) return rc;
  if ((rc = batch_issue_interval(b, s, check_int, up, layout))) return rc;
  GASP_CUDA(cudaStreamSynchronize(s));
  cudaGraph_t graph;
  GASP_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeRelaxed));
  rc = batch_issue_interval(b, s, check_int, up, layout);
  cudaError_t e = cudaStreamEndCapture(s, &graph);
  if (rc) return rc;
  if (e != cudaSuccess) return cuda_fail(e, "graph capture", __FILE__, __LINE__);
  e = cudaGraphInstantiate(&b->exec, graph, 0);
  cudaGraphDestroy(graph);
  if (e != cudaSuccess) return cuda_fail(e, "graph instantiate", __FILE__, __LINE__);
  b->graph_check_int = check_int;
  b->graph_up = up;
  b->graph_layout = layout;
  return batch_reset(b, s);  // restart from a clean state after the warm-up interval
}

}  // namespace

extern "C" {

int gasp_batch_create(const gasp_group_t *groups, int ngroups, unsigned long long seed,
                      int rng_kind, gasp_batch_t **out) {
  if (!groups || ngroups <= 0 || !out) return GASP_ERR_INVALID;
  *out = nullptr;
  gasp_batch *b = new (std::nothrow) gasp_batch();
  if (!b) return GASP_ERR_ALLOC;
  cudaGetDevice(&b->device);
  b->ngroups = ngroups;
  b->seed = seed;
  b->rng_kind = rng_kind;
  b->groups.assign(groups, groups + ngroups);
  int rc = GASP_OK;
  for (int g = 0; g < ngroups && rc == GASP_OK; ++g) {
    gasp_grids_t *gr = nullptr;
    rc = gasp_init_grid(groups[g].L, groups[g].ngrids, 32, nullptr, &gr);
    if (rc) break;
    b->grids.push_back(gr);
    b->rngs.push_back(nullptr);
    int *a = nullptr;
    if (cudaMalloc(&a, (size_t)groups[g].ngrids * sizeof(int)) != cudaSuccess) {
      rc = GASP_ERR_ALLOC;
      break;
    }
    b->d_active.push_back(a);
    cudaStream_t s;
    if (cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess) {
      rc = GASP_ERR_CUDA;
      break;
    }
    b->streams.push_back(s);
  }
  for (int e = 0; rc == GASP_OK && e <= ngroups; ++e) {
    cudaEvent_t ev;
    if (cudaEventCreateWithFlags(&ev, cudaEventDisableTiming) != cudaSuccess) rc = GASP_ERR_CUDA;
    else b->events.push_back(ev);
  }
  if (rc == GASP_OK && cudaStreamCreateWithFlags(&b->origin, cudaStreamNonBlocking) != cudaSuccess)
    rc = GASP_ERR_CUDA;
  if (rc == GASP_OK && cudaMalloc(&b->d_small, (size_t)2 * ngroups * sizeof(int)) != cudaSuccess)
    rc = GASP_ERR_ALLOC;
  if (rc) {
    batch_release(b);
    set_error("gasp_batch_create failed: %s", gasp_last_error());
    return rc;
  }
  *out = b;
  return GASP_OK;
}

int gasp_batch_free(gasp_batch_t *b) { return batch_release(b); }

int gasp_batch_swarm(gasp_batch_t *b, int tot_nsweeps, int check_int, double up_thr, int mode,
                     int *counts_out, long long *attempts_out, double *elapsed_out) {
  if (!b || tot_nsweeps < 0 || check_int <= 0 ||
      (mode != GASP_BATCH_PLAIN && mode != GASP_BATCH_GRAPH && mode != GASP_BATCH_MULTI))
    return GASP_ERR_INVALID;
  const int nint = tot_nsweeps / check_int;
  int rc;
  // All batch work runs on the batch's own stream; the caller's stream
  // choice is restored on return.
  const StreamRestore restore_stream;
  cudaStream_t s = b->origin;
  GASP_CUDA(cudaStreamSynchronize(restore_stream.prev));
  if (nint > b->max_intervals) {
    cudaFree(b->d_counts);
    b->d_counts = nullptr;
    GASP_CUDA(cudaMalloc(&b->d_counts, (size_t)b->ngroups * (nint > 0 ? nint : 1) * sizeof(int)));
    b->max_intervals = nint;
    if (b->exec) {
      cudaGraphExecDestroy(b->exec);
      b->exec = nullptr;
    }
  }
  if ((rc = batch_reset(b, s))) return rc;
  for (int g = 0; g < b->ngroups; ++g) {
    if ((rc = prepare_tables(b->grids[g], b->groups[g].beta, b->groups[g].h))) return rc;
  }
  std::vector<int> counts((size_t)b->ngroups * nint, 0);
  long long attempts = 0;
  const auto t0 = std::chrono::steady_clock::now();
  if (mode == GASP_BATCH_GRAPH || mode == GASP_BATCH_MULTI) {
    const int layout = mode == GASP_BATCH_MULTI ? 1 : b->layout;
    if (layout == 1 && !multi_possible(b)) {
      set_error("gasp_batch_swarm: one persistent launch needs integer thresholds and "
                "lattices in shared memory for every group");
      return GASP_ERR_UNSUPPORTED;
    }
    if ((rc = batch_build_graph(b, s, check_int, up_thr, layout))) return rc;
    for (int i = 0; i < nint; ++i) GASP_CUDA(cudaGraphLaunch(b->exec, s));
    GASP_CUDA(cudaStreamSynchronize(s));
    for (int g = 0; g < b->ngroups; ++g) {
      std::vector<int> c((size_t)nint, 0);
      if (nint > 0)
        GASP_CUDA(cudaMemcpy(c.data(), b->d_counts + (size_t)g * b->max_intervals,
                             (size_t)nint * sizeof(int), cudaMemcpyDeviceToHost));
      for (int i = 0; i < nint; ++i) counts[(size_t)i * b->ngroups + g] = c[i];
    }
  } else {
    for (int g = 0; g < b->ngroups; ++g) {
      gasp_grids_t *gr = b->grids[g];
      const int n = gr->ngrids;
      std::vector<char> done((size_t)n, 0);
      std::vector<float> mag((size_t)n);
      int ndone = 0;
      for (int i = 0; i < nint; ++i) {
        if ((rc = gasp_sweep(gr, b->rngs[g], b->groups[g].beta, b->groups[g].h, check_int, 2)))
          return rc;
        GASP_CUDA(cudaMemcpyAsync(mag.data(), gr->d_mag, (size_t)n * sizeof(float),
                                  cudaMemcpyDeviceToHost, s));
        GASP_CUDA(cudaStreamSynchronize(s));
        for (int r = 0; r < n; ++r)
          if (!done[r] && (double)mag[r] > up_thr) {
            done[r] = 1;
            ndone++;
          }
        counts[(size_t)i * b->ngroups + g] = ndone;
      }
    }
  }
  const double elapsed =
      std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  // Workload-defined attempts: each replica is credited until the check at
  // which it finished (identical for both modes).
  for (int g = 0; g < b->ngroups; ++g) {
    const long long N = (long long)b->groups[g].L * b->groups[g].L;
    int prev_done = 0;
    for (int i = 0; i < nint; ++i) {
      attempts += (long long)(b->groups[g].ngrids - prev_done) * N * check_int;
      prev_done = counts[(size_t)i * b->ngroups + g];
    }
  }
  if (counts_out) memcpy(counts_out, counts.data(), counts.size() * sizeof(int));
  if (attempts_out) *attempts_out = attempts;
  if (elapsed_out) *elapsed_out = elapsed;
  return GASP_OK;
}

int gasp_batch_autotune(gasp_batch_t *b, int nsweeps, int *choice_out) {
  if (!b || nsweeps <= 0) return GASP_ERR_INVALID;
  // All batch work runs on the batch's own stream; the caller's stream
  // choice is restored on return.
  const StreamRestore restore_stream;
  cudaStream_t s = b->origin;
  GASP_CUDA(cudaStreamSynchronize(restore_stream.prev));
  cudaEvent_t e0, e1;
  GASP_CUDA(cudaEventCreate(&e0));
  GASP_CUDA(cudaEventCreate(&e1));
  int rc = batch_reset(b, s);
  for (int g = 0; g < b->ngroups && rc == GASP_OK; ++g) {
    gasp_grids_t *gr = b->grids[g];
    if ((rc = prepare_tables(gr, b->groups[g].beta, b->groups[g].h))) break;
    const int L = b->groups[g].L;
    const bool rows = (L == 32 || L == 64 || L == 96 || L == 128);
    // candidates: (variant, warps_per_cta).  One warp per replica (variant 6)
    // is not one: timed alone it halves a small group's sweep (L=128, 512
    // replicas, XORWOW), but it spends ~20x the issue slots per attempt, and
    // in the concurrent graph that slows the other groups by more than it saves.
    std::vector<std::pair<int, int>> cand;
    if (rows) cand = {{0, 1}, {2, 1}};
    else cand = {{0, 1}, {0, 2}, {0, 4}};
    float best = 1e30f;
    int best_i = 0;
    for (size_t i = 0; i < cand.size(); ++i) {
      gasp_grids_set_option(gr, GASP_OPT_SWEEP_VARIANT, cand[i].first);
      gasp_grids_set_option(gr, GASP_OPT_WARPS_PER_CTA, cand[i].second);
      float ms = 0.f;
      for (int rep = 0; rep < 2; ++rep) {  // first run warms up
        GASP_CUDA(cudaEventRecord(e0, s));
        if ((rc = gasp_sweep(gr, b->rngs[g], b->groups[g].beta, b->groups[g].h, nsweeps, 2))) break;
        GASP_CUDA(cudaEventRecord(e1, s));
        GASP_CUDA(cudaEventSynchronize(e1));
        GASP_CUDA(cudaEventElapsedTime(&ms, e0, e1));
      }
      if (rc) break;
      if (ms < best) {
        best = ms;
        best_i = (int)i;
      }
    }
    if (rc) break;
    gasp_grids_set_option(gr, GASP_OPT_SWEEP_VARIANT, cand[best_i].first);
    gasp_grids_set_option(gr, GASP_OPT_WARPS_PER_CTA, cand[best_i].second);
    if (choice_out) {
      choice_out[2 * g] = cand[best_i].first;
      choice_out[2 * g + 1] = cand[best_i].second;
    }
  }
  // Layout of the interval graph: one kernel per group (concurrent branches)
  // or every group in one persistent launch.  Each is timed on intervals of
  // max(nsweeps, 20) sweeps in which no replica finishes (up = 2), at three
  // live fractions of every group (all, half, 15 %: a swarm's intervals run
  // with more and more of each group compacted out), two intervals each.
  b->layout = 0;
  b->layout_ms[0] = b->layout_ms[1] = -1.f;
  if (rc == GASP_OK && b->exec) {  // kernel choices changed: recapture
    cudaGraphExecDestroy(b->exec);
    b->exec = nullptr;
  }
  if (rc == GASP_OK && multi_possible(b)) {
    const double fracs[3] = {1.0, 0.5, 0.15};
    std::vector<int> small((size_t)2 * b->ngroups, 0);
    for (int layout = 0; layout < 2 && rc == GASP_OK; ++layout) {
      if ((rc = batch_build_graph(b, s, nsweeps > 20 ? nsweeps : 20, 2.0, layout))) break;
      GASP_CUDA(cudaGraphLaunch(b->exec, s));  // warm-up replay
      float total = 0.f;
      for (double f : fracs) {
        for (int g = 0; g < b->ngroups; ++g) {
          const int n = (int)(f * b->groups[g].ngrids);
          small[(size_t)2 * g] = n > 1 ? n : 1;  // live count; the active list is 0..n-1
          small[(size_t)2 * g + 1] = 0;
        }
        GASP_CUDA(cudaMemcpyAsync(b->d_small, small.data(), small.size() * sizeof(int),
                                  cudaMemcpyHostToDevice, s));
        GASP_CUDA(cudaEventRecord(e0, s));
        for (int i = 0; i < 2; ++i) GASP_CUDA(cudaGraphLaunch(b->exec, s));
        GASP_CUDA(cudaEventRecord(e1, s));
        GASP_CUDA(cudaEventSynchronize(e1));
        float ms = 0.f;
        GASP_CUDA(cudaEventElapsedTime(&ms, e0, e1));
        total += ms;
      }
      b->layout_ms[layout] = total;
    }
    if (rc == GASP_OK && b->layout_ms[1] < b->layout_ms[0]) b->layout = 1;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (b->exec) {  // built for timing only: the next run captures its own
    cudaGraphExecDestroy(b->exec);
    b->exec = nullptr;
  }
  if (rc == GASP_OK) rc = batch_reset(b, s);
  return rc;
}

int gasp_batch_layout(const gasp_batch_t *b, float *ms_per_group_kernels, float *ms_one_launch) {
  if (!b) return -1;
  if (ms_per_group_kernels) *ms_per_group_kernels = b->layout_ms[0];
  if (ms_one_launch) *ms_one_launch = b->layout_ms[1];
  return b->layout;
}

}  // extern "C"
