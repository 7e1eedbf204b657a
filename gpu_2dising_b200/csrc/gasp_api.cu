// gasp_api.cu -- host implementation of the gasp-b200 C ABI (include/gasp.h):
// device set-up, replica sets, RNG states, single sweep batches and the
// reference-compatible driver loop (replaces mc_driver_gpu,
// src/mc_gpu.cu:530-831).
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <chrono>
#include <string>
#include <vector>

#include "gasp_internal.h"

namespace gasp {

static thread_local std::string g_err;
static thread_local cudaStream_t g_stream = nullptr;

void set_error(const char *fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  g_err = buf;
}

int cuda_fail(cudaError_t e, const char *what, const char *file, int line) {
  set_error("%s: %s (%s:%d)", what, cudaGetErrorString(e), file, line);
  if (e == cudaErrorMemoryAllocation) return GASP_ERR_ALLOC;
  if (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver) return GASP_ERR_NO_DEVICE;
  return GASP_ERR_CUDA;
}

cudaStream_t current_stream() { return g_stream; }

}  // namespace gasp

using namespace gasp;

namespace {

// Device-side table block of a replica set: thresholds, float and double
// acceptance tables, flags.
struct TableBlock {
  uint32_t thr[16];
  float pacc[20];
  float pad_[12];
  double pacc_cpu[20];
  int flags[4];
};

// Committor shooting on the MWC64X stream switches to the one-warp-per-replica
// sweep once at most this many replicas are undecided (GASP_OPT_TAIL_REPLICAS).
// Live replicas at which device-side committor shooting hands its last
// undecided replicas to the one-warp-per-replica kernel, per stream (the
// XORWOW kernel draws its attempts in order, one warp-wide step per draw,
// so its throughput crosses the row kernel's at fewer replicas).
constexpr int kTailReplicasMwc = 4096;
constexpr int kTailReplicasXorwow = 1024;

struct GridsExtra {
  TableBlock *d_tab = nullptr;
  double beta = NAN, h = NAN;
  int float_cmp = 0;
  double *d_stream = nullptr;
  size_t stream_cap = 0;
  float *d_mag2 = nullptr;  // second magnetisation buffer for the driver
  int *d_active = nullptr;
  float *d_lclus = nullptr; // largest-cluster sizes [ngrids]
  int *d_cwork = nullptr;   // largest-cluster global work area (large L only)
  size_t cwork_bytes = 0;
  int variant = 0;          // GASP_OPT_SWEEP_VARIANT
  int warps_per_cta = 1;    // GASP_OPT_WARPS_PER_CTA
  int tail_replicas = -1;   // GASP_OPT_TAIL_REPLICAS (-1: the stream's default)
  int *d_upchunk = nullptr; // int32 staging of whole-set uploads, kUploadChunk replicas
};

// Replicas per chunk of a whole-set upload without the set's int32 buffer
// (16 MiB at L=64): allocating a set-sized int32 buffer (512 MiB at L=64 x
// 32768) cost 5-30 ms on a B200, two to three times the copy itself.
constexpr int kUploadChunk = 1024;

// Extra state kept beside the public struct (allocated with it).
struct GridsImpl {
  gasp_grids pub;
  GridsExtra x;
};

GridsImpl *impl(gasp_grids_t *g) { return reinterpret_cast<GridsImpl *>(g); }

void host_probs_gpu(double beta, double h, float P[20]) {
  // src/mc_gpu.cu:21-37, with the host expf.
  for (int i = 0; i < 20; ++i) P[i] = 0.f;
  for (int s = -1; s < 2; s += 2)
    for (int nsum = -4; nsum < 5; nsum += 2) {
      const int index = 5 * (s + 1) + nsum + 4;
      const float de = 2.0f * (float)s * ((float)nsum + (float)h);
      P[index] = expf(-(float)beta * de);
    }
}

void host_probs_cpu(double beta, double h, double P[20]) {
  // src/mc_cpu.c:14-38.
  for (int i = 0; i < 20; ++i) P[i] = 0.0;
  for (int s = -1; s < 2; s += 2)
    for (int nsum = -4; nsum < 5; nsum += 2) {
      const int index = 5 * (s + 1) + nsum + 4;
      P[index] = exp(-beta * (2.0 * (double)s * ((double)nsum + h)));
    }
}

// Makes the replica set's tables match (beta, h).  Synchronous on change.
int ensure_tables(gasp_grids_t *g, double beta, double h) {
  GridsExtra &x = impl(g)->x;
  if (x.d_tab && x.beta == beta && x.h == h) return GASP_OK;
  if (!x.d_tab) GASP_CUDA(cudaMalloc(&x.d_tab, sizeof(TableBlock)));
  TableBlock hb;
  memset(&hb, 0, sizeof hb);
  host_probs_gpu(beta, h, hb.pacc);
  host_probs_cpu(beta, h, hb.pacc_cpu);
  cudaStream_t s = current_stream();
  GASP_CUDA(cudaMemcpyAsync(x.d_tab, &hb, sizeof hb, cudaMemcpyHostToDevice, s));
  int rc = launch_build_thresholds(x.d_tab->pacc, x.d_tab->thr, x.d_tab->flags, s);
  if (rc) return rc;
  int flags[4];
  GASP_CUDA(cudaMemcpyAsync(flags, x.d_tab->flags, sizeof flags, cudaMemcpyDeviceToHost, s));
  GASP_CUDA(cudaStreamSynchronize(s));
  x.float_cmp = flags[0] != 0;
  x.beta = beta;
  x.h = h;
  return GASP_OK;
}

int check_device_of(int dev) {
  int cur = -1;
  GASP_CUDA(cudaGetDevice(&cur));
  if (cur != dev) GASP_CUDA(cudaSetDevice(dev));
  return GASP_OK;
}

int validate_L(int L, int device) {
  if (L < 2) {
    set_error("L must be >= 2 (got %d)", L);
    return GASP_ERR_INVALID;
  }
  (void)device;
  if (L > 8192) {  // the reference's MAXL (include/mc_gpu.h:59)
    set_error("L=%d exceeds the maximum lattice side 8192", L);
    return GASP_ERR_UNSUPPORTED;
  }
  return GASP_OK;
}

}  // namespace

extern "C" {

const char *gasp_status_string(int status) {
  switch (status) {
    case GASP_OK: return "ok";
    case GASP_ERR_INVALID: return "invalid argument";
    case GASP_ERR_CUDA: return "CUDA error";
    case GASP_ERR_NO_DEVICE: return "no CUDA device";
    case GASP_ERR_ALLOC: return "allocation failed";
    case GASP_ERR_IO: return "I/O error";
    case GASP_ERR_FORMAT: return "file format mismatch";
    case GASP_ERR_CALLBACK: return "output callback failed";
    case GASP_ERR_UNSUPPORTED: return "unsupported configuration";
    case GASP_ERR_TIMEOUT: return "device wait timed out";
    default: return "unknown status";
  }
}

const char *gasp_last_error(void) { return g_err.c_str(); }
const char *gasp_version(void) { return "gasp-b200 0.1 (sm_100a)"; }

int gasp_set_stream(void *stream) {
  g_stream = reinterpret_cast<cudaStream_t>(stream);
  return GASP_OK;
}

int gasp_init_device(int device_index, int verbose, int *device_out, int *nsms_out) {
  int count = 0;
  cudaError_t e = cudaGetDeviceCount(&count);
  if (e != cudaSuccess || count == 0) {
    if (verbose) fprintf(stdout, "No CUDA supported devices are available in this system.\n");
    set_error("no CUDA device (%s)", cudaGetErrorString(e));
    return GASP_ERR_NO_DEVICE;
  }
  if (verbose) {
    // The reference's device summary (src/gpu_tools.cu:31-76).
    fprintf(stdout, "Found %d CUDA devices in this system\n", count);
    for (int d = 0; d < count; ++d) {
      cudaDeviceProp prop;
      GASP_CUDA(cudaGetDeviceProperties(&prop, d));
      int optin = 0;
      GASP_CUDA(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, d));
      fprintf(stdout, "Device %d : %s\n", d, prop.name);
      fprintf(stdout, "================================\n");
      fprintf(stdout, "Number of SMs       : %d\n", prop.multiProcessorCount);
      fprintf(stdout, "Max SHMEM per block : %ld KB\n", (long)(prop.sharedMemPerBlock / 1024));
      fprintf(stdout, "Max Opt in shared   : %d KB\n", optin / 1024);
      fprintf(stdout, "Recommended ngrids  : %d\n", 4 * prop.warpSize * prop.multiProcessorCount);
      fprintf(stdout, "\n");
      fprintf(stdout, "Estimated largest L for shared memory code path : %d\n", max_shared_L(d));
      fprintf(stdout, "(Assumes threadsPerBlock = 32)\n");
      fprintf(stdout, "\n");
    }
  }
  if (device_index != -1) {
    if (device_index < 0 || device_index >= count) {
      set_error("device index %d out of range (%d devices)", device_index, count);
      return GASP_ERR_INVALID;
    }
    GASP_CUDA(cudaSetDevice(device_index));
  }
  int dev = 0;
  GASP_CUDA(cudaGetDevice(&dev));
  if (verbose) {
    fprintf(stdout, "Using CUDA device : %d\n", dev);
    fflush(stdout);
  }
  cudaDeviceProp prop;
  GASP_CUDA(cudaGetDeviceProperties(&prop, dev));
  if (device_out) *device_out = dev;
  if (nsms_out) *nsms_out = prop.multiProcessorCount;
  return GASP_OK;
}

int gasp_select_gpu_method(int L, int ngrids, int threads_per_block, int gpu_device,
                           int *method_out) {
  (void)ngrids;
  if (!method_out || threads_per_block <= 0) {
    set_error("invalid arguments to gasp_select_gpu_method");
    return GASP_ERR_INVALID;
  }
  int dev = gpu_device;
  if (dev < 0) GASP_CUDA(cudaGetDevice(&dev));
  cudaDeviceProp prop;
  GASP_CUDA(cudaGetDeviceProperties(&prop, dev));
  // src/gpu_tools.cu:211-224, the same arithmetic.
  const int max_shmem = (int)prop.sharedMemPerBlock;
  const double value = (8.0 * max_shmem) / threads_per_block;
  int maxL = (int)sqrt(value);
  maxL = (int)sqrt(32 * (maxL * maxL / 32));
  *method_out = (L <= maxL) ? 2 : 0;
  return GASP_OK;
}

int gasp_acceptance_table(double beta, double h, float table_out[20]) {
  if (!table_out) return GASP_ERR_INVALID;
  host_probs_gpu(beta, h, table_out);
  return GASP_OK;
}

int gasp_max_shared_L(int device, int *maxL_out) {
  if (!maxL_out) return GASP_ERR_INVALID;
  int dev = device;
  if (dev < 0) GASP_CUDA(cudaGetDevice(&dev));
  *maxL_out = max_shared_L(dev);
  return GASP_OK;
}

size_t gasp_frame_bytes(int L, int ngrids) {
  return (size_t)(((long long)L * L * ngrids + 7) / 8);
}

int gasp_init_grid(int L, int ngrids, int threads_per_block, const int *host_grids,
                   gasp_grids_t **grids_out) {
  (void)threads_per_block;
  if (!grids_out || ngrids <= 0) {
    set_error("gasp_init_grid: ngrids must be positive and grids_out non-NULL");
    return GASP_ERR_INVALID;
  }
  *grids_out = nullptr;
  int dev = 0;
  GASP_CUDA(cudaGetDevice(&dev));
  int rc = validate_L(L, dev);
  if (rc) return rc;
  GridsImpl *im = new (std::nothrow) GridsImpl();
  if (!im) return GASP_ERR_ALLOC;
  gasp_grids &g = im->pub;
  g.device = dev;
  g.L = L;
  g.N = L * L;
  g.W = words_per_replica(L);
  g.ngrids = ngrids;
  g.ntiles = tiles_for(ngrids);
  g.frame_bytes = gasp_frame_bytes(L, ngrids);
  g.global_lattice = L > max_shared_L(dev) ? 1 : 0;
  const size_t words = (size_t)g.ntiles * g.W * kTile;
  cudaError_t e = cudaMalloc(&g.d_lat, words * sizeof(uint32_t));
  if (e == cudaSuccess) e = cudaMalloc(&g.d_mag, (size_t)g.ntiles * kTile * sizeof(float));
  if (e == cudaSuccess) e = cudaMemsetAsync(g.d_lat, 0, words * sizeof(uint32_t), current_stream());
  if (e != cudaSuccess) {
    cudaFree(g.d_lat);
    cudaFree(g.d_mag);
    delete im;
    return cuda_fail(e, "gasp_init_grid allocation", __FILE__, __LINE__);
  }
  *grids_out = &g;
  if (host_grids) return gasp_grids_upload(&g, host_grids);
  return GASP_OK;
}

int gasp_free_grid(gasp_grids_t *g) {
  if (!g) return GASP_OK;
  GridsImpl *im = impl(g);
  cudaFree(g->d_lat);
  cudaFree(g->d_mag);
  cudaFree(g->d_frame);
  cudaFree(g->d_scratch32);
  cudaFree(im->x.d_tab);
  cudaFree(im->x.d_stream);
  cudaFree(im->x.d_mag2);
  cudaFree(im->x.d_active);
  cudaFree(im->x.d_lclus);
  cudaFree(im->x.d_cwork);
  cudaFree(im->x.d_upchunk);
  delete im;
  return GASP_OK;
}

static int ensure_scratch32(gasp_grids_t *g) {
  if (!g->d_scratch32)
    GASP_CUDA(cudaMalloc(&g->d_scratch32, (size_t)g->ngrids * g->N * sizeof(int)));
  return GASP_OK;
}

int gasp_grids_upload(gasp_grids_t *g, const int *host_grids) {
  if (!g || !host_grids) return GASP_ERR_INVALID;
  int rc = check_device_of(g->device);
  if (rc) return rc;
  cudaStream_t s = current_stream();
  if (!g->d_scratch32) {
    // No set-sized int32 buffer yet: upload in chunks of kUploadChunk
    // replicas through one reusable staging buffer, each chunk copied then
    // packed into its tiles (stream order keeps a chunk's copy behind the
    // previous chunk's pack); the copies run at the full host-to-device rate.
    GridsExtra &x = impl(g)->x;
    const int chunk = g->ngrids < kUploadChunk ? g->ngrids : kUploadChunk;
    if (!x.d_upchunk) GASP_CUDA(cudaMalloc(&x.d_upchunk, (size_t)chunk * g->N * sizeof(int)));
    for (int r0 = 0; r0 < g->ngrids; r0 += chunk) {
      const int n = g->ngrids - r0 < chunk ? g->ngrids - r0 : chunk;
      GASP_CUDA(cudaMemcpyAsync(x.d_upchunk, host_grids + (size_t)r0 * g->N,
                                (size_t)n * g->N * sizeof(int), cudaMemcpyHostToDevice, s));
      // kUploadChunk is a multiple of the 32-replica tile: chunks start on tiles
      rc = launch_pack_grids(x.d_upchunk, g->d_lat + (size_t)(r0 / kTile) * g->W * kTile, g->L,
                             n, s);
      if (rc) break;
    }
    const cudaError_t se = cudaStreamSynchronize(s);
    if (rc) return rc;
    if (se != cudaSuccess) return cuda_fail(se, "cudaStreamSynchronize", __FILE__, __LINE__);
    return GASP_OK;
  }
  GASP_CUDA(cudaMemcpyAsync(g->d_scratch32, host_grids, (size_t)g->ngrids * g->N * sizeof(int),
                            cudaMemcpyHostToDevice, s));
  rc = launch_pack_grids(g->d_scratch32, g->d_lat, g->L, g->ngrids, s);
  if (rc) return rc;
  GASP_CUDA(cudaStreamSynchronize(s));
  return GASP_OK;
}

int gasp_grids_upload_inputs(gasp_grids_t *g, const int *inputs, int ninputs) {
  if (!g || !inputs || ninputs <= 0 || g->ngrids % ninputs != 0) {
    set_error("gasp_grids_upload_inputs: ngrids must be a multiple of ninputs");
    return GASP_ERR_INVALID;
  }
  int rc = check_device_of(g->device);
  if (rc) return rc;
  // Stage in the set's int32 buffer if it has one, else in a buffer sized
  // for the inputs only (the set-sized buffer is 32x the lattice).
  const size_t bytes = (size_t)ninputs * g->N * sizeof(int);
  int *stage = g->d_scratch32, *owned = nullptr;
  if (!stage) {
    GASP_CUDA(cudaMalloc(&owned, bytes));
    stage = owned;
  }
  cudaStream_t s = current_stream();
  cudaError_t e = cudaMemcpyAsync(stage, inputs, bytes, cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) {
    rc = launch_pack_grids(stage, g->d_lat, g->L, g->ngrids, s, g->ngrids / ninputs);
    e = cudaStreamSynchronize(s);
  }
  if (owned) cudaFree(owned);
  if (rc) return rc;
  GASP_CUDA(e);
  return GASP_OK;
}

int gasp_grids_download(gasp_grids_t *g, int *host_grids) {
  if (!g || !host_grids) return GASP_ERR_INVALID;
  int rc = check_device_of(g->device);
  if (rc) return rc;
  if ((rc = ensure_scratch32(g))) return rc;
  cudaStream_t s = current_stream();
  rc = launch_unpack_grids(g->d_lat, g->d_scratch32, g->L, g->ngrids, s);
  if (rc) return rc;
  GASP_CUDA(cudaMemcpyAsync(host_grids, g->d_scratch32, (size_t)g->ngrids * g->N * sizeof(int),
                            cudaMemcpyDeviceToHost, s));
  GASP_CUDA(cudaStreamSynchronize(s));
  return GASP_OK;
}

int gasp_grids_set_option(gasp_grids_t *g, int option, int value) {
  if (!g) return GASP_ERR_INVALID;
  GridsExtra &x = impl(g)->x;
  // Variants 3, 4 and 8 (pairwise speculation, acceptance mask, two tiles
  // per warp) were measured slower than variant 0 and have been retired.
  if (option == GASP_OPT_SWEEP_VARIANT && value >= 0 && value <= 10 && value != 3 &&
      value != 4 && value != 8) {
    x.variant = value;
    return GASP_OK;
  }
  if (option == GASP_OPT_WARPS_PER_CTA && value >= 1 && value <= 8) {
    x.warps_per_cta = value;
    return GASP_OK;
  }
  if (option == GASP_OPT_TAIL_REPLICAS && value >= 0) {
    x.tail_replicas = value;
    return GASP_OK;
  }
  set_error("unknown option %d or bad value %d", option, value);
  return GASP_ERR_INVALID;
}

int gasp_grids_shape(const gasp_grids_t *g, int *L_out, int *ngrids_out) {
  if (!g) return GASP_ERR_INVALID;
  if (L_out) *L_out = g->L;
  if (ngrids_out) *ngrids_out = g->ngrids;
  return GASP_OK;
}

}  // extern "C"

namespace {

uint64_t splitmix64(uint64_t &z) {
  // Steele, Lea & Flood (2014) SplitMix64 finaliser, used only to spread the
  // user's seed over the MWC64X state space.
  uint64_t v = (z += 0x9E3779B97F4A7C15ull);
  v = (v ^ (v >> 30)) * 0xBF58476D1CE4E5B9ull;
  v = (v ^ (v >> 27)) * 0x94D049BB133111EBull;
  return v ^ (v >> 31);
}

uint64_t mulmod64(uint64_t a, uint64_t b, uint64_t m) {
  return (uint64_t)((unsigned __int128)a * b % m);
}

uint64_t powmod64(uint64_t a, uint64_t e, uint64_t m) {
  uint64_t r = 1 % m;
  a %= m;
  while (e) {
    if (e & 1) r = mulmod64(r, a, m);
    a = mulmod64(a, a, m);
    e >>= 1;
  }
  return r;
}

// MWC64X states for ngrids replicas: the seed picks a base state X0 in
// [1, M-1]; replica r starts at X0 * A^(r * 2^40) mod M, i.e. 2^40 draws
// after replica r-1 (a run uses < 2^32 draws per replica, so streams never
// overlap).  Layout: x at [r], c at [stride + r].
void mwc_seed_states(uint64_t seed, int ngrids, int stride, std::vector<uint32_t> &out) {
  const uint64_t A = kMwcA;
  const uint64_t M = (A << 32) - 1;
  uint64_t z = seed;
  const uint64_t X0 = 1 + splitmix64(z) % (M - 1);
  const uint64_t P = powmod64(A, 1ull << 40, M);
  out.assign((size_t)kMwcWords * stride, 0u);
  uint64_t X = X0;
  for (int r = 0; r < ngrids; ++r) {
    out[r] = (uint32_t)(X / A);
    out[(size_t)stride + r] = (uint32_t)(X % A);
    X = mulmod64(X, P, M);
  }
}

}  // namespace

const TailParams &gasp::mwc_lane_params() {
  static const TailParams t = [] {
    TailParams q;
    const uint64_t A = kMwcA;
    const uint64_t M = (A << 32) - 1;
    const uint64_t Ainv = 1ull << 32;  // A * 2^32 = M + 1
    for (int j = 0; j < 32; ++j) {
      q.mul[j] = powmod64(A, (uint64_t)j << 35, M);
      q.inv[j] = powmod64(Ainv, (uint64_t)j << 35, M);
    }
    return q;
  }();
  return t;
}

namespace gasp {
// Seeds the states of r in place (the same streams gasp_init_rand_mode gives
// for this seed) on the current stream, and waits for them.
int rng_reseed(gasp_rng_t *r, unsigned long long seed) {
  cudaStream_t s = current_stream();
  int rc = GASP_OK;
  if (r->kind == kRngMwc) {
    std::vector<uint32_t> host;
    mwc_seed_states(seed, r->ngrids, r->stride, host);
    const cudaError_t e = cudaMemcpyAsync(r->d_state, host.data(), host.size() * sizeof(uint32_t),
                                          cudaMemcpyHostToDevice, s);
    if (e != cudaSuccess) return cuda_fail(e, "gasp_init_rand upload", __FILE__, __LINE__);
  } else {
    rc = launch_rng_init(r->d_state, r->ngrids, r->stride, seed, s);
    if (rc) return rc;
  }
  const cudaError_t e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return cuda_fail(e, "gasp_init_rand", __FILE__, __LINE__);
  return GASP_OK;
}
}  // namespace gasp

extern "C" {

int gasp_init_rand_mode(int ngrids, int threads_per_block, unsigned long long seed, int kind,
                        gasp_rng_t **rng_out) {
  (void)threads_per_block;
  if (!rng_out || ngrids <= 0 || (kind != GASP_RNG_XORWOW && kind != GASP_RNG_MWC64X)) {
    set_error("gasp_init_rand: ngrids must be positive, kind valid and rng_out non-NULL");
    return GASP_ERR_INVALID;
  }
  *rng_out = nullptr;
  gasp_rng *r = new (std::nothrow) gasp_rng();
  if (!r) return GASP_ERR_ALLOC;
  cudaError_t e = cudaGetDevice(&r->device);
  r->ngrids = ngrids;
  r->stride = tiles_for(ngrids) * kTile;
  r->kind = kind == GASP_RNG_MWC64X ? kRngMwc : kRngXorwow;
  const int words = r->kind == kRngMwc ? kMwcWords : kRngWords;
  if (e == cudaSuccess)
    e = cudaMalloc(&r->d_state, (size_t)words * r->stride * sizeof(uint32_t));
  if (e != cudaSuccess) {
    delete r;
    return cuda_fail(e, "gasp_init_rand allocation", __FILE__, __LINE__);
  }
  const int rc = rng_reseed(r, seed);
  if (rc) {
    cudaFree(r->d_state);
    delete r;
    return rc;
  }
  *rng_out = r;
  return GASP_OK;
}

int gasp_acceptance_thresholds(gasp_grids_t *g, double beta, double h, uint32_t *thr10,
                               int *float_compare) {
  if (!g || !thr10) return GASP_ERR_INVALID;
  int rc = check_device_of(g->device);
  if (rc) return rc;
  if ((rc = ensure_tables(g, beta, h))) return rc;
  GridsExtra &x = impl(g)->x;
  cudaStream_t s = current_stream();
  GASP_CUDA(cudaMemcpyAsync(thr10, x.d_tab->thr, 10 * sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
  GASP_CUDA(cudaStreamSynchronize(s));
  if (float_compare) *float_compare = x.float_cmp;
  return GASP_OK;
}

int gasp_mwc64x_lane_multipliers(uint64_t *mul32, uint64_t *inv32) {
  if (!mul32 || !inv32) return GASP_ERR_INVALID;
  const TailParams &t = mwc_lane_params();
  memcpy(mul32, t.mul, sizeof t.mul);
  memcpy(inv32, t.inv, sizeof t.inv);
  return GASP_OK;
}

int gasp_rng_read_states(const gasp_rng_t *r, uint32_t *out, long long nwords) {
  if (!r || !out) return GASP_ERR_INVALID;
  const long long need = (long long)(r->kind == kRngMwc ? kMwcWords : kRngWords) * r->stride;
  if (nwords < need) {
    set_error("gasp_rng_read_states: %lld words needed, %lld given", need, nwords);
    return GASP_ERR_INVALID;
  }
  int rc = check_device_of(r->device);
  if (rc) return rc;
  cudaStream_t s = current_stream();
  GASP_CUDA(cudaMemcpyAsync(out, r->d_state, (size_t)need * sizeof(uint32_t),
                            cudaMemcpyDeviceToHost, s));
  GASP_CUDA(cudaStreamSynchronize(s));
  return GASP_OK;
}

int gasp_mwc64x_seed_states(unsigned long long seed, int ngrids, int stride, uint32_t *out) {
  if (!out || ngrids <= 0 || stride < ngrids) return GASP_ERR_INVALID;
  std::vector<uint32_t> host;
  mwc_seed_states(seed, ngrids, stride, host);
  memcpy(out, host.data(), host.size() * sizeof(uint32_t));
  return GASP_OK;
}

int gasp_init_rand(int ngrids, int threads_per_block, unsigned long long seed,
                   gasp_rng_t **rng_out) {
  return gasp_init_rand_mode(ngrids, threads_per_block, seed, GASP_RNG_XORWOW, rng_out);
}

int gasp_free_rand(gasp_rng_t *r) {
  if (!r) return GASP_OK;
  cudaFree(r->d_state);
  delete r;
  return GASP_OK;
}

}  // extern "C"

namespace {

SweepLaunch base_launch(gasp_grids_t *g) {
  SweepLaunch p;
  memset(&p, 0, sizeof p);
  GridsExtra &x = impl(g)->x;
  p.lat = g->d_lat;
  p.L = g->L;
  p.ngrids = g->ngrids;
  p.n_active = g->ngrids;
  p.thr = x.d_tab->thr;
  p.pacc_f = x.d_tab->pacc;
  p.pacc_cpu = x.d_tab->pacc_cpu;
  p.float_compare = x.float_cmp;
  p.variant = x.variant;
  p.lattice_in_global = g->global_lattice;
  p.warps_per_cta = x.warps_per_cta;
  return p;
}

int check_sweep_args(gasp_grids_t *g, gasp_rng_t *r, int nsweeps, int method) {
  if (!g || !r) {
    set_error("NULL grid set or RNG");
    return GASP_ERR_INVALID;
  }
  if (r->ngrids < g->ngrids) {
    set_error("RNG has %d states for %d grids", r->ngrids, g->ngrids);
    return GASP_ERR_INVALID;
  }
  if (nsweeps < 0) {
    set_error("nsweeps must be >= 0");
    return GASP_ERR_INVALID;
  }
  if (method < 0 || method > 2) {
    set_error("gpu_method must be 0, 1 or 2 (got %d)", method);
    return GASP_ERR_INVALID;
  }
  return check_device_of(g->device);
}

}  // namespace

namespace gasp {

SweepLaunch launch_for(gasp_grids_t *g, gasp_rng_t *r) {
  SweepLaunch p = base_launch(g);
  p.rng = r->d_state;
  p.rng_stride = r->stride;
  p.rng_kind = r->kind;
  return p;
}

int prepare_tables(gasp_grids_t *g, double beta, double h) { return ensure_tables(g, beta, h); }

}  // namespace gasp

extern "C" {

int gasp_sweep(gasp_grids_t *g, gasp_rng_t *r, double beta, double h, int nsweeps, int gpu_method) {
  int rc = check_sweep_args(g, r, nsweeps, gpu_method);
  if (rc) return rc;
  if ((rc = ensure_tables(g, beta, h))) return rc;
  if (nsweeps == 0) return GASP_OK;
  SweepLaunch p = base_launch(g);
  p.rng = r->d_state;
  p.rng_stride = r->stride;
  p.rng_kind = r->kind;
  p.nsweeps = nsweeps;
  p.mag_out = g->d_mag;
  return launch_sweep_exact(p, current_stream());
}

int gasp_sweep_trace_cpu(gasp_grids_t *g, const double *stream, double beta, double h,
                         int nsweeps) {
  if (!g || !stream || nsweeps < 0) return GASP_ERR_INVALID;
  int rc = check_device_of(g->device);
  if (rc) return rc;
  if ((rc = ensure_tables(g, beta, h))) return rc;
  if (nsweeps == 0) return GASP_OK;
  GridsExtra &x = impl(g)->x;
  const size_t n = (size_t)g->ngrids * 3 * (size_t)g->N * nsweeps;
  cudaPointerAttributes attr;
  const double *dptr = stream;
  cudaStream_t s = current_stream();
  if (cudaPointerGetAttributes(&attr, stream) != cudaSuccess || attr.type != cudaMemoryTypeDevice) {
    cudaGetLastError();
    if (x.stream_cap < n) {
      cudaFree(x.d_stream);
      x.d_stream = nullptr;
      x.stream_cap = 0;
      GASP_CUDA(cudaMalloc(&x.d_stream, n * sizeof(double)));
      x.stream_cap = n;
    }
    GASP_CUDA(cudaMemcpyAsync(x.d_stream, stream, n * sizeof(double), cudaMemcpyHostToDevice, s));
    dptr = x.d_stream;
  }
  SweepLaunch p = base_launch(g);
  p.stream = dptr;
  p.nsweeps = nsweeps;
  p.mag_out = g->d_mag;
  rc = launch_sweep_trace_cpu(p, s);
  if (rc) return rc;
  GASP_CUDA(cudaStreamSynchronize(s));
  return GASP_OK;
}

int gasp_magnetisation(gasp_grids_t *g, float *host_mag) {
  if (!g || !host_mag) return GASP_ERR_INVALID;
  int rc = check_device_of(g->device);
  if (rc) return rc;
  cudaStream_t s = current_stream();
  rc = launch_measure(g->d_lat, g->L, g->ngrids, g->d_mag, s);
  if (rc) return rc;
  GASP_CUDA(cudaMemcpyAsync(host_mag, g->d_mag, (size_t)g->ngrids * sizeof(float),
                            cudaMemcpyDeviceToHost, s));
  GASP_CUDA(cudaStreamSynchronize(s));
  return GASP_OK;
}

static int ensure_frame(gasp_grids_t *g) {
  if (!g->d_frame) GASP_CUDA(cudaMalloc(&g->d_frame, (g->frame_bytes + 15) & ~(size_t)15));
  return GASP_OK;
}

int gasp_pack_frame(gasp_grids_t *g, uint8_t *host_out) {
  if (!g || !host_out) return GASP_ERR_INVALID;
  int rc = check_device_of(g->device);
  if (rc) return rc;
  if ((rc = ensure_frame(g))) return rc;
  cudaStream_t s = current_stream();
  rc = launch_pack_frame(g->d_lat, g->d_frame, g->L, g->ngrids, s);
  if (rc) return rc;
  GASP_CUDA(cudaMemcpyAsync(host_out, g->d_frame, g->frame_bytes, cudaMemcpyDeviceToHost, s));
  GASP_CUDA(cudaStreamSynchronize(s));
  return GASP_OK;
}

}  // extern "C"

// Largest cluster of `spin` sites of every replica into x.d_lclus (on s).
static int measure_largest_cluster(gasp_grids_t *g, int spin, cudaStream_t s) {
  GridsExtra &x = impl(g)->x;
  if (!x.d_lclus) GASP_CUDA(cudaMalloc(&x.d_lclus, (size_t)g->ngrids * sizeof(float)));
  if (spin != 1 && spin != -1) {  // no site holds such a spin
    GASP_CUDA(cudaMemsetAsync(x.d_lclus, 0, (size_t)g->ngrids * sizeof(float), s));
    return GASP_OK;
  }
  const size_t need = largest_cluster_work_bytes(g->L, g->ngrids, g->device);
  if (need > x.cwork_bytes) {
    cudaFree(x.d_cwork);
    x.d_cwork = nullptr;
    x.cwork_bytes = 0;
    GASP_CUDA(cudaMalloc(&x.d_cwork, need));
    x.cwork_bytes = need;
  }
  return launch_largest_cluster(g->d_lat, g->L, g->ngrids, spin, x.d_cwork, need, x.d_lclus, s);
}

extern "C" int gasp_largest_cluster(gasp_grids_t *g, int spin, float *host_out) {
  if (!g || !host_out) return GASP_ERR_INVALID;
  int rc = check_device_of(g->device);
  if (rc) return rc;
  cudaStream_t s = current_stream();
  if ((rc = measure_largest_cluster(g, spin, s))) return rc;
  GASP_CUDA(cudaMemcpyAsync(host_out, impl(g)->x.d_lclus, (size_t)g->ngrids * sizeof(float),
                            cudaMemcpyDeviceToHost, s));
  GASP_CUDA(cudaStreamSynchronize(s));
  return GASP_OK;
}

// ===========================================================================
// Checkpoint files (no reference counterpart): "GASPCKP1", int32 L, ngrids,
// rng kind, RNG words per replica, isweep, has_fates; the grids as one
// gridstates.bin payload (ceil(L*L*ngrids/8) bytes); the RNG words
// component-major (uint32 [words][ngrids]); int32 fates[ngrids] if present.
// ===========================================================================
namespace {

const char kCkptMagic[8] = {'G', 'A', 'S', 'P', 'C', 'K', 'P', '1'};

// gridstates.bin payload bits -> int32 spins (bit 1 -> +1).
void expand_frame(const uint8_t *payload, int *grids, long long nbits) {
  for (long long i = 0; i < nbits; ++i) grids[i] = ((payload[i >> 3] >> (i & 7)) & 1) ? 1 : -1;
}

int rng_words(const gasp_rng_t *r) { return r->kind == kRngMwc ? kMwcWords : kRngWords; }

struct FileCloser {
  FILE *f;
  ~FileCloser() {
    if (f) fclose(f);
  }
};

int read_ckpt_header(FILE *f, int hdr[6]) {
  char magic[8];
  if (fread(magic, 1, 8, f) != 8 || fread(hdr, sizeof(int), 6, f) != 6) {
    set_error("checkpoint: truncated header");
    return GASP_ERR_IO;
  }
  if (memcmp(magic, kCkptMagic, 8) != 0 || hdr[0] < 2 || hdr[1] <= 0 ||
      (hdr[2] != kRngXorwow && hdr[2] != kRngMwc) ||
      hdr[3] != (hdr[2] == kRngMwc ? kMwcWords : kRngWords)) {
    set_error("checkpoint: not a gasp checkpoint or unknown version");
    return GASP_ERR_FORMAT;
  }
  return GASP_OK;
}

}  // namespace

extern "C" int gasp_checkpoint_save(const char *path, gasp_grids_t *g, gasp_rng_t *r,
                                    const int *fates, int isweep) {
  if (!path || !g || !r) return GASP_ERR_INVALID;
  if (r->ngrids < g->ngrids) {
    set_error("checkpoint: %d RNG states for %d replicas", r->ngrids, g->ngrids);
    return GASP_ERR_INVALID;
  }
  int rc = check_device_of(g->device);
  if (rc) return rc;
  if ((rc = ensure_frame(g))) return rc;
  const int ng = g->ngrids, words = rng_words(r);
  std::vector<uint8_t> payload(g->frame_bytes);
  std::vector<uint32_t> rs((size_t)words * ng);
  cudaStream_t s = current_stream();
  if ((rc = launch_pack_frame(g->d_lat, g->d_frame, g->L, ng, s))) return rc;
  GASP_CUDA(cudaMemcpyAsync(payload.data(), g->d_frame, g->frame_bytes, cudaMemcpyDeviceToHost, s));
  for (int k = 0; k < words; ++k)
    GASP_CUDA(cudaMemcpyAsync(rs.data() + (size_t)k * ng, r->d_state + (size_t)k * r->stride,
                              (size_t)ng * sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
  GASP_CUDA(cudaStreamSynchronize(s));
  FileCloser fc{fopen(path, "wb")};
  if (!fc.f) {
    set_error("checkpoint: cannot open %s for writing", path);
    return GASP_ERR_IO;
  }
  const int hdr[6] = {g->L, ng, r->kind, words, isweep, fates ? 1 : 0};
  bool ok = fwrite(kCkptMagic, 1, 8, fc.f) == 8 && fwrite(hdr, sizeof(int), 6, fc.f) == 6 &&
            fwrite(payload.data(), 1, payload.size(), fc.f) == payload.size() &&
            fwrite(rs.data(), sizeof(uint32_t), rs.size(), fc.f) == rs.size();
  if (ok && fates) ok = fwrite(fates, sizeof(int), (size_t)ng, fc.f) == (size_t)ng;
  ok = (fclose(fc.f) == 0) && ok;
  fc.f = nullptr;
  if (!ok) {
    set_error("checkpoint: write to %s failed", path);
    return GASP_ERR_IO;
  }
  return GASP_OK;
}

extern "C" int gasp_checkpoint_info(const char *path, int *L_out, int *ngrids_out,
                                    int *rng_kind_out, int *isweep_out, int *has_fates_out) {
  if (!path) return GASP_ERR_INVALID;
  FileCloser fc{fopen(path, "rb")};
  if (!fc.f) {
    set_error("checkpoint: cannot open %s", path);
    return GASP_ERR_IO;
  }
  int hdr[6];
  int rc = read_ckpt_header(fc.f, hdr);
  if (rc) return rc;
  if (L_out) *L_out = hdr[0];
  if (ngrids_out) *ngrids_out = hdr[1];
  if (rng_kind_out) *rng_kind_out = hdr[2];
  if (isweep_out) *isweep_out = hdr[4];
  if (has_fates_out) *has_fates_out = hdr[5];
  return GASP_OK;
}

extern "C" int gasp_checkpoint_load(const char *path, gasp_grids_t *g, gasp_rng_t *r,
                                    int *fates_out, int *isweep_out) {
  if (!path || !g || !r) return GASP_ERR_INVALID;
  FileCloser fc{fopen(path, "rb")};
  if (!fc.f) {
    set_error("checkpoint: cannot open %s", path);
    return GASP_ERR_IO;
  }
  int hdr[6];
  int rc = read_ckpt_header(fc.f, hdr);
  if (rc) return rc;
  if (hdr[0] != g->L || hdr[1] != g->ngrids || hdr[2] != r->kind || r->ngrids < hdr[1]) {
    set_error("checkpoint: file holds L=%d ngrids=%d rng kind %d; the handles differ", hdr[0],
              hdr[1], hdr[2]);
    return GASP_ERR_FORMAT;
  }
  if ((rc = check_device_of(g->device))) return rc;
  const int ng = hdr[1], words = hdr[3];
  std::vector<uint8_t> payload(g->frame_bytes);
  std::vector<uint32_t> rs((size_t)words * ng);
  std::vector<int> fates(hdr[5] ? (size_t)ng : 0);
  bool ok = fread(payload.data(), 1, payload.size(), fc.f) == payload.size() &&
            fread(rs.data(), sizeof(uint32_t), rs.size(), fc.f) == rs.size();
  if (ok && hdr[5]) ok = fread(fates.data(), sizeof(int), (size_t)ng, fc.f) == (size_t)ng;
  if (!ok) {
    set_error("checkpoint: %s is truncated", path);
    return GASP_ERR_IO;
  }
  std::vector<int> grids((size_t)g->N * ng);
  expand_frame(payload.data(), grids.data(), (long long)g->N * ng);
  if ((rc = gasp_grids_upload(g, grids.data()))) return rc;
  cudaStream_t s = current_stream();
  for (int k = 0; k < words; ++k)
    GASP_CUDA(cudaMemcpyAsync(r->d_state + (size_t)k * r->stride, rs.data() + (size_t)k * ng,
                              (size_t)ng * sizeof(uint32_t), cudaMemcpyHostToDevice, s));
  GASP_CUDA(cudaStreamSynchronize(s));
  if (fates_out) {
    if (hdr[5]) memcpy(fates_out, fates.data(), (size_t)ng * sizeof(int));
    else for (int i = 0; i < ng; ++i) fates_out[i] = -1;
  }
  if (isweep_out) *isweep_out = hdr[4];
  return GASP_OK;
}

// ===========================================================================
// Driver
// ===========================================================================
namespace {

struct PinnedBuf {
  void *p = nullptr;
  ~PinnedBuf() {
    if (p) cudaFreeHost(p);
  }
};


}  // namespace

namespace {

// Committor shooting with the checks on the device: the itask-1 loop of the
// driver (check at every isweep % mag_int == 0, then spc sweeps of the
// replicas still undecided) with fates, compaction and attempt counts kept
// in device memory, so intervals are enqueued back to back and the host only
// polls the number of undecided replicas now and then.  Same fates as the
// host loop: the same thresholds are applied to the same states.
int committor_on_device(gasp_grids_t *g, gasp_rng_t *r, int tot, int mag_int, int spc,
                        double up, double dn, int *grid_fate, long long *attempts_out) {
  GridsExtra &x = impl(g)->x;
  const int ngrids = g->ngrids, N = g->N;
  cudaStream_t s = current_stream();
  if (!x.d_active) GASP_CUDA(cudaMalloc(&x.d_active, (size_t)ngrids * sizeof(int)));
  struct DevBuf {
    void *p = nullptr;
    ~DevBuf() {
      if (p) cudaFree(p);
    }
  } fates_b, small_b, act2_b, cnt_b;
  GASP_CUDA(cudaMalloc(&fates_b.p, (size_t)ngrids * sizeof(int)));
  // the compaction writes survivors to the other list of a ping-pong pair
  GASP_CUDA(cudaMalloc(&act2_b.p, (size_t)ngrids * sizeof(int)));
  GASP_CUDA(cudaMalloc(&cnt_b.p, (size_t)(fate_compact_blocks(ngrids) + 1) * sizeof(int)));
  int *act[2] = {x.d_active, static_cast<int *>(act2_b.p)};
  int cur = 0;
  GASP_CUDA(cudaMalloc(&small_b.p, 64));
  int *d_fates = static_cast<int *>(fates_b.p);
  int *d_n = static_cast<int *>(small_b.p);
  long long *d_att = reinterpret_cast<long long *>(static_cast<char *>(small_b.p) + 8);
  PinnedBuf hpoll_b;  // read behind events while the host runs ahead: pinned
  GASP_CUDA(cudaMallocHost(&hpoll_b.p, 64 * sizeof(int)));
  std::vector<int> hact_v((size_t)ngrids);
  int *hact = hact_v.data();
  volatile int *hpoll = static_cast<volatile int *>(hpoll_b.p);
  int n0 = 0;
  for (int i = 0; i < ngrids; ++i)
    if (grid_fate[i] == -1) hact[n0++] = i;
  const long long zero = 0;
  GASP_CUDA(cudaMemcpyAsync(d_fates, grid_fate, (size_t)ngrids * sizeof(int),
                            cudaMemcpyHostToDevice, s));
  if (n0 > 0)
    GASP_CUDA(cudaMemcpyAsync(x.d_active, hact, (size_t)n0 * sizeof(int), cudaMemcpyHostToDevice,
                              s));
  GASP_CUDA(cudaMemcpyAsync(d_n, &n0, sizeof(int), cudaMemcpyHostToDevice, s));
  GASP_CUDA(cudaMemcpyAsync(d_att, &zero, sizeof(long long), cudaMemcpyHostToDevice, s));
  int rc = launch_measure(g->d_lat, g->L, ngrids, g->d_mag, s);
  if (rc) return rc;

  SweepLaunch p = base_launch(g);
  p.rng = r->d_state;
  p.rng_stride = r->stride;
  p.rng_kind = r->kind;
  p.nsweeps = spc;
  p.active = x.d_active;
  p.n_active = ngrids;  // launch shape; the kernels read the live count from d_n
  p.n_active_dev = d_n;
  p.mag_out = g->d_mag;

  // Poll ring: every kPollEvery checks the live count is copied to pinned
  // memory behind an event; the host looks at completed polls without
  // waiting and stays at most kAhead polls ahead of the device.
  constexpr int kPollEvery = 8, kRing = 16, kAhead = 4;
  cudaEvent_t ev[kRing];
  int nev = 0;
  for (; nev < kRing; ++nev)
    if (cudaEventCreateWithFlags(&ev[nev], cudaEventDisableTiming) != cudaSuccess) break;
  struct EvGuard {
    cudaEvent_t *e;
    int n;
    ~EvGuard() {
      for (int i = 0; i < n; ++i) cudaEventDestroy(e[i]);
    }
  } evg{ev, nev};
  if (nev < kRing) GASP_CUDA(cudaGetLastError());
  long long polls_issued = 0, polls_seen = 0;
  bool done = n0 == 0;
  int checks = 0;
  // Once few replicas are undecided, each gets a warp of its own
  // (k_sweep_tail).  Both kernels are enqueued every interval and each checks
  // the device count, so the switch happens at the same interval whatever the
  // host's timing.  On the XORWOW stream the tail kernel draws every attempt
  // in the replica's own order, so the trajectories stay the reference's.
  const int tail_n = x.tail_replicas >= 0 ? x.tail_replicas
                     : r->kind == kRngMwc ? kTailReplicasMwc : kTailReplicasXorwow;
  const bool tail_ok = tail_n > 0 && !g->global_lattice && g->L >= 3 && g->L <= kTailMaxL;
  SweepLaunch q = p;
  if (tail_ok) {
    p.tail_split = q.tail_split = tail_n;
    q.variant = 6;
    q.n_active = tail_n < ngrids ? tail_n : ngrids;
  }
  for (int isweep = 0; isweep < tot && !done; isweep += spc) {
    if (isweep % mag_int == 0) {
      // sweeps from this check to the next one (or to the end of the run)
      long long span = 0;
      for (int j = isweep; j < tot && (j == isweep || j % mag_int != 0); j += spc) span += spc;
      if ((rc = launch_fate_compact(g->d_mag, d_fates, act[cur], act[cur ^ 1], d_n,
                                    static_cast<int *>(cnt_b.p), ngrids, up, dn, d_att,
                                    (long long)N * span, s)))
        return rc;
      cur ^= 1;
      p.active = q.active = act[cur];
      if (++checks % kPollEvery == 0) {
        const int slot = (int)(polls_issued % kRing);
        GASP_CUDA(cudaMemcpyAsync(const_cast<int *>(hpoll) + slot, d_n, sizeof(int),
                                  cudaMemcpyDeviceToHost, s));
        GASP_CUDA(cudaEventRecord(ev[slot], s));
        ++polls_issued;
      }
    }
    if ((rc = launch_sweep_exact(p, s))) return rc;
    if (tail_ok && (rc = launch_sweep_exact(q, s))) return rc;
    // look at finished polls; wait only when too far ahead
    while (polls_seen < polls_issued) {
      const int slot = (int)(polls_seen % kRing);
      cudaError_t q = polls_issued - polls_seen > kAhead ? cudaEventSynchronize(ev[slot])
                                                          : cudaEventQuery(ev[slot]);
      if (q == cudaErrorNotReady) break;
      GASP_CUDA(q);
      ++polls_seen;
      if (hpoll[slot] == 0) {
        done = true;
        break;
      }
    }
  }
  long long att = 0;
  GASP_CUDA(cudaMemcpyAsync(grid_fate, d_fates, (size_t)ngrids * sizeof(int),
                            cudaMemcpyDeviceToHost, s));
  GASP_CUDA(cudaMemcpyAsync(&att, d_att, sizeof(long long), cudaMemcpyDeviceToHost, s));
  GASP_CUDA(cudaStreamSynchronize(s));
  if (attempts_out) *attempts_out = att;
  return GASP_OK;
}

}  // namespace

extern "C" int gasp_mc_driver_gpu_ex(gasp_gpu_grids_t grids, double beta, double h, int *grid_fate,
                                     gasp_sampler_t samples, gasp_function_t calc,
                                     gasp_gpu_run_t gpu_state, gasp_grid_output_fn outfunc,
                                     const gasp_driver_opts_t *opts) {
  gasp_driver_opts_t o;
  memset(&o, 0, sizeof o);
  if (opts) o = *opts;
  gasp_grids_t *g = grids.d_grids;
  gasp_rng_t *r = gpu_state.d_state;
  const int tot = samples.tot_nsweeps, mag_int = samples.mag_output_int,
            grid_int = samples.grid_output_int;
  if (!g || !r) {
    set_error("driver: device grid set and RNG states are required");
    return GASP_ERR_INVALID;
  }
  if (grids.L != g->L || grids.ngrids != g->ngrids) {
    set_error("driver: grids.L/ngrids (%d, %d) do not match the device set (%d, %d)", grids.L,
              grids.ngrids, g->L, g->ngrids);
    return GASP_ERR_INVALID;
  }
  if (mag_int <= 0 || grid_int <= 0 || tot < 0) {
    set_error("driver: output intervals must be positive and tot_nsweeps >= 0");
    return GASP_ERR_INVALID;
  }
  if (calc.itask != 0 && calc.itask != 1) {
    set_error("Error: itask must be 0 or 1!");
    return GASP_ERR_INVALID;
  }
  const int ninputs = calc.ninputs > 0 ? calc.ninputs : 1;
  if (g->ngrids % ninputs != 0) {
    set_error("Error: ngrids must be divisible by ninputs!");
    return GASP_ERR_INVALID;
  }
  const bool use_lclus = calc.cv && strcmp(calc.cv, "largest_cluster") == 0;
  if (calc.cv && !use_lclus && strcmp(calc.cv, "magnetisation") != 0) {
    set_error("driver: cv must be 'magnetisation' or 'largest_cluster' (got '%s')", calc.cv);
    return GASP_ERR_UNSUPPORTED;
  }
  if (calc.itask == 1 && !grid_fate) {
    set_error("driver: itask 1 needs a grid_fate array");
    return GASP_ERR_INVALID;
  }
  if (outfunc && !grids.ising_grids) {
    set_error("driver: outfunc needs the host grids array (grids.ising_grids)");
    return GASP_ERR_INVALID;
  }
  int rc = check_sweep_args(g, r, 0, gpu_state.gpu_method < 0 ? 0 : gpu_state.gpu_method % 3);
  if (rc) return rc;
  if ((rc = ensure_tables(g, beta, h))) return rc;

  GridsExtra &x = impl(g)->x;
  const int ngrids = g->ngrids, N = g->N, L = g->L;
  const int itask = calc.itask;
  const double up = calc.up_thr, dn = calc.dn_thr;
  const int spc = mag_int < grid_int ? mag_int : grid_int;
  const int nres = itask == 0 ? tot / mag_int : ninputs;
  std::vector<float> result((size_t)nres, itask == 0 ? 1.0f : 0.0f);
  const bool dumps = outfunc != nullptr || o.packed_out != nullptr;
  const bool compact = o.compact && itask == 1;
  char *cv = const_cast<char *>(calc.cv ? calc.cv : "magnetisation");
  char *fname = const_cast<char *>(calc.filename ? calc.filename : "gridstates.bin");

  if (compact && !dumps && o.verbosity == 0 && !use_lclus) {
    // Nothing to report per check: run the shooting loop on the device.
    long long attempts = 0;
    const auto t0 = std::chrono::steady_clock::now();
    int rc2 = committor_on_device(g, r, tot, mag_int, spc, up, dn, grid_fate, &attempts);
    if (rc2) return rc2;
    const double elapsed =
        std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    const int sub = ngrids / ninputs;
    for (int i = 0; i < ninputs; ++i) {  // src/mc_gpu.cu:812-826
      int nBb = 0, nF = 0;
      for (int j = 0; j < sub; ++j) {
        const int f = grid_fate[i * sub + j];
        if (f > -1) nBb += f;
        else nF += 1;
      }
      result[i] = (float)nBb / (float)(sub - nF);
    }
    if (calc.result)
      for (int i = 0; i < nres; ++i) calc.result[i] = result[i];
    if (o.elapsed_s) *o.elapsed_s = elapsed;
    if (o.attempts) *o.attempts = attempts;
    return GASP_OK;
  }

  cudaStream_t s = current_stream();
  if (!x.d_mag2) GASP_CUDA(cudaMalloc(&x.d_mag2, (size_t)g->ntiles * kTile * sizeof(float)));
  if (compact && !x.d_active) GASP_CUDA(cudaMalloc(&x.d_active, (size_t)ngrids * sizeof(int)));
  if (dumps && (rc = ensure_frame(g))) return rc;
  // Host staging is pageable: the loop waits on every read-back anyway, and
  // page-locking (16 MiB for a frame at L=64 x 32768) can cost more than the
  // copies it would speed up.
  std::vector<float> hmag_v((size_t)ngrids);
  float *hmag = hmag_v.data();
  std::vector<float> mag_last((size_t)ngrids, 0.0f);
  // Collective variable compared with the thresholds: the magnetisation or
  // the largest cluster of spins opposite to initial_spin (src/mc_gpu.cu:586-605).
  std::vector<float> lclus_last(use_lclus ? (size_t)ngrids : 0, 0.0f);
  std::vector<float> hlclus_v(use_lclus ? (size_t)ngrids : 0);
  float *hlclus = use_lclus ? hlclus_v.data() : nullptr;
  const float *colvar = use_lclus ? lclus_last.data() : mag_last.data();
  auto take_check = [&]() {
    memcpy(mag_last.data(), hmag, (size_t)ngrids * sizeof(float));
    if (use_lclus) memcpy(lclus_last.data(), hlclus, (size_t)ngrids * sizeof(float));
  };
  std::vector<uint8_t> hframe_v(dumps ? g->frame_bytes : 0);
  std::vector<int> hact_v(compact ? (size_t)ngrids : 0);
  uint8_t *hframe = dumps ? hframe_v.data() : nullptr;
  int *hact = compact ? hact_v.data() : nullptr;

  float *d_mag_cur = g->d_mag, *d_mag_next = x.d_mag2;
  SweepLaunch p = base_launch(g);
  p.rng = r->d_state;
  p.rng_stride = r->stride;
  p.rng_kind = r->kind;
  p.nsweeps = spc;

  long long attempts = 0;
  int n_active = ngrids;
  // A check's read-backs (magnetisation, cluster sizes, frame) go on a side
  // stream once the state they read has been produced (`ready`, recorded on
  // the sweep stream before the interval's sweep is launched), so the copies
  // overlap that sweep and the sweeps queue back to back; the host waits on
  // `copied` for the data it reads.  The next write of a buffer being copied
  // (the other half of the magnetisation pair, the frame) is launched only
  // after the host has waited.
  cudaStream_t rs = nullptr;
  cudaEvent_t ready = nullptr, copied = nullptr;
  struct SideGuard {
    cudaStream_t &st;
    cudaEvent_t &a, &b;
    ~SideGuard() {
      if (st) { cudaStreamSynchronize(st); cudaStreamDestroy(st); }
      if (a) cudaEventDestroy(a);
      if (b) cudaEventDestroy(b);
    }
  } side_guard{rs, ready, copied};
  GASP_CUDA(cudaStreamCreateWithFlags(&rs, cudaStreamNonBlocking));
  GASP_CUDA(cudaEventCreateWithFlags(&ready, cudaEventDisableTiming));
  GASP_CUDA(cudaEventCreateWithFlags(&copied, cudaEventDisableTiming));
  const auto t0 = std::chrono::steady_clock::now();
  if ((rc = launch_measure(g->d_lat, L, ngrids, d_mag_cur, s))) return rc;

  if (o.first_up)
    for (int i = 0; i < ngrids; ++i) o.first_up[i] = -1;
  int isweep = 0;
  bool have_frame = false;
  while (isweep < tot) {
    const bool dump_now = dumps && (isweep % grid_int == 0);
    const bool mag_now = isweep % mag_int == 0;
    if (dump_now)
      if ((rc = launch_pack_frame(g->d_lat, g->d_frame, L, ngrids, s))) return rc;
    if (mag_now && use_lclus)  // on the lattice before this interval's sweeps
      if ((rc = measure_largest_cluster(g, -calc.initial_spin, s))) return rc;
    bool fates_done = false;
    int nA = 0, nB = 0;
    if (compact && mag_now) {
      // Fates at this check decide which replicas the next batch simulates:
      // read back on the sweep stream and wait before launching it.
      GASP_CUDA(cudaMemcpyAsync(hmag, d_mag_cur, (size_t)ngrids * sizeof(float),
                                cudaMemcpyDeviceToHost, s));
      if (use_lclus)
        GASP_CUDA(cudaMemcpyAsync(hlclus, x.d_lclus, (size_t)ngrids * sizeof(float),
                                  cudaMemcpyDeviceToHost, s));
      GASP_CUDA(cudaStreamSynchronize(s));
      take_check();
      n_active = 0;
      for (int i = 0; i < ngrids; ++i) {
        if (grid_fate[i] == -1) {
          const double m = (double)colvar[i];
          if (m > up) grid_fate[i] = 1;
          else if (m < dn) grid_fate[i] = 0;
        }
        if (grid_fate[i] == 0) nA++;
        else if (grid_fate[i] == 1) nB++;
        else hact[n_active++] = i;
      }
      fates_done = true;
      if (n_active > 0)
        GASP_CUDA(cudaMemcpyAsync(x.d_active, hact, (size_t)n_active * sizeof(int),
                                  cudaMemcpyHostToDevice, s));
    }
    // The batch isweep -> isweep+spc; its epilogue measures the state the
    // next check will read.
    const int next = isweep + spc;
    const bool mag_next = next % mag_int == 0;
    if (n_active > 0) {
      p.active = compact ? x.d_active : nullptr;
      p.n_active = n_active;
      p.mag_out = mag_next ? d_mag_next : nullptr;
      if (compact && mag_next) {
        // Resolved replicas are not swept; keep their last magnetisation.
        GASP_CUDA(cudaMemcpyAsync(d_mag_next, d_mag_cur, (size_t)ngrids * sizeof(float),
                                  cudaMemcpyDeviceToDevice, s));
      }
      GASP_CUDA(cudaEventRecord(ready, s));  // this check's state (before the sweep below)
      if ((rc = launch_sweep_exact(p, s))) return rc;
      attempts += (long long)n_active * N * spc;
    } else {
      GASP_CUDA(cudaEventRecord(ready, s));
    }
    if (dump_now || (mag_now && !fates_done)) {
      // the check's read-backs, on the side stream while the sweep runs
      GASP_CUDA(cudaStreamWaitEvent(rs, ready, 0));
      if (dump_now)
        GASP_CUDA(cudaMemcpyAsync(hframe, g->d_frame, g->frame_bytes, cudaMemcpyDeviceToHost, rs));
      if (mag_now && !fates_done) {
        GASP_CUDA(cudaMemcpyAsync(hmag, d_mag_cur, (size_t)ngrids * sizeof(float),
                                  cudaMemcpyDeviceToHost, rs));
        if (use_lclus)
          GASP_CUDA(cudaMemcpyAsync(hlclus, x.d_lclus, (size_t)ngrids * sizeof(float),
                                    cudaMemcpyDeviceToHost, rs));
      }
      GASP_CUDA(cudaEventRecord(copied, rs));
    }
    if (dump_now || (dumps && isweep == tot - 1)) {
      GASP_CUDA(cudaEventSynchronize(copied));
      if (dump_now) {
        have_frame = true;
        if (outfunc) expand_frame(hframe, grids.ising_grids, (long long)N * ngrids);
      }
      if (mag_now && !fates_done) take_check();
      if (have_frame) {
        if (outfunc && outfunc(L, ngrids, grids.ising_grids, isweep, mag_last.data(),
                               use_lclus ? lclus_last.data() : nullptr, cv, dn, up, fname) != 0) {
          cudaStreamSynchronize(s);
          set_error("output callback returned non-zero at isweep %d", isweep);
          return GASP_ERR_CALLBACK;
        }
        if (o.packed_out && o.packed_out(L, ngrids, hframe, g->frame_bytes, isweep,
                                         mag_last.data(), o.packed_user) != 0) {
          cudaStreamSynchronize(s);
          set_error("packed output callback returned non-zero at isweep %d", isweep);
          return GASP_ERR_CALLBACK;
        }
      }
    }
    bool stop = false;
    if (mag_now || isweep == tot - 1) {
      if (mag_now && !fates_done) {
        GASP_CUDA(cudaEventSynchronize(copied));
        take_check();
      }
      if (itask == 0) {
        int nnuc = 0;
        for (int i = 0; i < ngrids; ++i) nnuc += ((double)colvar[i] > up) ? 1 : 0;
        if (o.first_up)
          for (int i = 0; i < ngrids; ++i)
            if (o.first_up[i] < 0 && (double)colvar[i] > up) o.first_up[i] = isweep;
        const int idx = isweep / mag_int;
        if (idx < nres) result[idx] = (float)((double)nnuc / (double)ngrids);
        if (o.verbosity == 1) {  // CLI (src/mc_gpu.cu:726)
          fprintf(stdout, "%10d  %12.6f\n", isweep, (double)nnuc / (double)ngrids);
          fflush(stdout);
        } else if (o.verbosity == 2) {  // PyGASP progress (src/mc_gpu.cu:730-731)
          fprintf(stdout, "\r Sweep : %10d, Reached cv = %6.2f : %4d , Unresolved : %4d", isweep,
                  up, nnuc, ngrids - nnuc);
          fflush(stdout);
        }
        stop = nnuc == ngrids;
      } else {
        if (!fates_done) {
          nA = nB = 0;
          for (int i = 0; i < ngrids; ++i) {
            if (grid_fate[i] == 0) {
              nA++;
            } else if (grid_fate[i] == 1) {
              nB++;
            } else {
              const double m = (double)colvar[i];
              if (m > up) { grid_fate[i] = 1; nB++; }
              else if (m < dn) { grid_fate[i] = 0; nA++; }
            }
          }
        }
        if (o.verbosity >= 1) {
          fprintf(stdout,
                  "\r Sweep : %10d, Reached cv = %6.2f : %4d , Reached cv = %6.2f : %4d , "
                  "Unresolved : %4d",
                  isweep, dn, nA, up, nB, ngrids - nA - nB);
          fflush(stdout);
        }
        stop = nA + nB == ngrids;
      }
    }
    if (mag_next) {
      float *t = d_mag_cur;
      d_mag_cur = d_mag_next;
      d_mag_next = t;
    }
    if (stop) break;
    isweep = next;
  }
  GASP_CUDA(cudaStreamSynchronize(s));
  // Keep the set's magnetisation buffer pointing at the freshest values.
  if (d_mag_cur != g->d_mag) {
    x.d_mag2 = g->d_mag;
    g->d_mag = d_mag_cur;
  }
  const double elapsed =
      std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  if (itask == 1) {
    const int sub = ngrids / ninputs;
    for (int i = 0; i < ninputs; ++i) {
      int nBb = 0, nF = 0;
      for (int j = 0; j < sub; ++j) {
        const int f = grid_fate[i * sub + j];
        if (f > -1) nBb += f;
        else nF += 1;
      }
      result[i] = (float)nBb / (float)(sub - nF);
    }
  }
  if (o.verbosity == 1) {  // src/mc_gpu.cu:786-787
    fprintf(stdout, "\n# Time taken on GPU = %f seconds\n", elapsed);
    if (itask == 1) fprintf(stdout, "pB estimate : %10.6f\n", nres > 0 ? (double)result[0] : 0.0);
    fflush(stdout);
  } else if (o.verbosity == 2) {
    fprintf(stdout, "\n");
    fflush(stdout);
  }
  if (calc.result)
    for (int i = 0; i < nres; ++i) calc.result[i] = result[i];
  if (o.elapsed_s) *o.elapsed_s = elapsed;
  if (o.attempts) *o.attempts = attempts;
  return GASP_OK;
}

extern "C" int gasp_mc_driver_gpu(gasp_gpu_grids_t grids, double beta, double h, int *grid_fate,
                                  gasp_sampler_t samples, gasp_function_t calc,
                                  gasp_gpu_run_t gpu_state, gasp_grid_output_fn outfunc) {
  return gasp_mc_driver_gpu_ex(grids, beta, h, grid_fate, samples, calc, gpu_state, outfunc,
                               nullptr);
}
