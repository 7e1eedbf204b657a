// gasp_kernels.cu -- sm_100a device code of gasp-b200.
//
// Hot kernel: k_sweep_exact, the reference-exact random-site Metropolis sweep
// (reproduces mc_sweep_gpu / _bitrep / _bitmap32, src/mc_gpu.cu:88-356).
// Design (B200 first, not a translation):
//   * one warp = one tile of 32 replicas, one replica per lane;
//   * each replica's lattice is a private bitmap in shared memory, stored
//     lane-interleaved (word w of lane l at w*32+l): every shared load or
//     store a warp issues hits 32 distinct banks, whatever sites the lanes
//     drew, so the random-site gathers of the reference (3-4 way bank
//     conflicts plus an atomicXor per flip) become single-wavefront accesses
//     and a flip is a plain store to a word only its lane owns;
//   * the XORWOW state lives in registers for the whole batch and is drawn
//     with the cuRAND device API (curand / _curand_uniform), so the stream is
//     the reference's own;
//   * the acceptance test u2 < P is replaced by an exactly equivalent integer
//     test x2 <= thr[class] on the raw draw; thresholds are found on the
//     device by bisection over the same _curand_uniform, which is monotone;
//   * the magnetisation of the batch's final state is a popcount of the
//     lane's own words, fused into the epilogue.
#include <cfloat>
#include <cstdio>

#include <curand_kernel.h>

#include "gasp_internal.h"

namespace gasp {
namespace {

constexpr int kHeaderWords = 64;  // per-CTA shared header: tables (256 B)

__device__ __forceinline__ void load_rng(curandStateXORWOW &st, const uint32_t *rng,
                                         int stride, int rep) {
  st.d = rng[rep];
#pragma unroll
  for (int k = 0; k < 5; ++k) st.v[k] = rng[(k + 1) * stride + rep];
  st.boxmuller_flag = 0;
  st.boxmuller_flag_double = 0;
  st.boxmuller_extra = 0.f;
  st.boxmuller_extra_double = 0.0;
}

__device__ __forceinline__ void store_rng(const curandStateXORWOW &st, uint32_t *rng,
                                          int stride, int rep) {
  rng[rep] = st.d;
#pragma unroll
  for (int k = 0; k < 5; ++k) rng[(k + 1) * stride + rep] = st.v[k];
}

// RNG policies of the sweep kernels.
//   RngXorwow: the reference stream (cuRAND XORWOW, curand_uniform site
//              arithmetic of src/mc_gpu.cu:311,317).
//   RngMwc:    the production stream (MWC64X, two instructions per 32-bit
//              draw; site = the draw's top bits scaled to [0, N)).
template <int kKind>
struct RngPolicy;

template <>
struct RngPolicy<kRngXorwow> {
  static constexpr int kKind = kRngXorwow;
  curandStateXORWOW st;
  __device__ __forceinline__ void load(const uint32_t *rng, int stride, int rep) {
    load_rng(st, rng, stride, rep);
  }
  __device__ __forceinline__ void store(uint32_t *rng, int stride, int rep) const {
    store_rng(st, rng, stride, rep);
  }
  __device__ __forceinline__ uint32_t next() { return curand(&st); }
  template <int N>
  __device__ __forceinline__ uint32_t site(float shrink, int /*n_runtime*/) {
    return (uint32_t)__float2int_rd(shrink * _curand_uniform(curand(&st)));
  }
};

template <>
struct RngPolicy<kRngMwc> {
  static constexpr int kKind = kRngMwc;
  uint32_t x, c;
  __device__ __forceinline__ void load(const uint32_t *rng, int stride, int rep) {
    x = rng[rep];
    c = rng[stride + rep];
  }
  __device__ __forceinline__ void store(uint32_t *rng, int stride, int rep) const {
    rng[rep] = x;
    rng[stride + rep] = c;
  }
  __device__ __forceinline__ uint32_t next() {
    const uint32_t r = x ^ c;
    const unsigned long long t = (unsigned long long)x * kMwcA + c;
    x = (uint32_t)t;
    c = (uint32_t)(t >> 32);
    return r;
  }
  template <int N>
  __device__ __forceinline__ uint32_t site(float, int n_runtime) {
    const uint32_t r = next();
    if constexpr (N > 0 && (N & (N - 1)) == 0) {
      return r >> (32 - __builtin_ctz((unsigned)N));
    } else {
      return __umulhi(r, (uint32_t)(N > 0 ? N : n_runtime));
    }
  }
};

// Replicas to sweep: the device count when there is one, zero when a
// one-warp-per-replica launch takes over at this count (p.tail_split).
__device__ __forceinline__ int live_count(const SweepLaunch &p) {
  const int n = p.n_active_dev ? *p.n_active_dev : p.n_active;
  return p.tail_split > 0 && n <= p.tail_split ? 0 : n;
}

// Shared-memory staging of one tile (identity order) or of 32 listed replicas.
__device__ __forceinline__ void stage_in(uint32_t *lat_s, const SweepLaunch &p, int W,
                                         int tile, int lane, bool live, int rep) {
  if (p.active == nullptr) {
    const uint32_t *src = p.lat + (size_t)tile * W * kTile + lane;
    for (int w = 0; w < W; ++w) lat_s[w * kTile + lane] = src[(size_t)w * kTile];
  } else {
    const uint32_t *src = p.lat + (size_t)(rep >> 5) * W * kTile + (rep & 31);
    for (int w = 0; w < W; ++w) lat_s[w * kTile + lane] = live ? src[(size_t)w * kTile] : 0u;
  }
}

__device__ __forceinline__ void stage_out(const uint32_t *lat_s, const SweepLaunch &p, int W,
                                          int tile, int lane, bool live, int rep) {
  if (p.active == nullptr) {
    uint32_t *dst = p.lat + (size_t)tile * W * kTile + lane;
    for (int w = 0; w < W; ++w) dst[(size_t)w * kTile] = lat_s[w * kTile + lane];
  } else if (live) {
    uint32_t *dst = p.lat + (size_t)(rep >> 5) * W * kTile + (rep & 31);
    for (int w = 0; w < W; ++w) dst[(size_t)w * kTile] = lat_s[w * kTile + lane];
  }
}

// Bulk-copy staging (sweep variant 9).  In identity order a tile's W*32 words
// are contiguous in HBM and in shared memory, so one cp.async.bulk of the
// whole tile, its completion counted on an mbarrier, replaces the per-lane
// loads, and one bulk shared->global copy the write-back.  Every wait is
// bounded: a load that has not completed after kStagePolls polls (and as many
// again) sets g_stage_timeout, the tile is neither swept nor written back,
// and the host turns the flag into GASP_ERR_TIMEOUT.
__device__ int g_stage_timeout;
constexpr int kStagePolls = 1 << 22;

__device__ __forceinline__ bool stage_wait(uint32_t bar) {
  for (int i = 0; i < kStagePolls; ++i) {
    uint32_t done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], 0;\n"
        " selp.u32 %0, 1, 0, p;\n}"
        : "=r"(done)
        : "r"(bar)
        : "memory");
    if (done) return true;
  }
  return false;
}

// Returns false (on every lane) when the copy did not complete in time.
__device__ __forceinline__ bool bulk_stage_in(uint32_t *lat_s, const uint32_t *src, uint32_t bytes,
                                              uint64_t *bar, int lane) {
  const uint32_t b = (uint32_t)__cvta_generic_to_shared(bar);
  if (lane == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(b) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(b), "r"(bytes)
                 : "memory");
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            (uint32_t)__cvta_generic_to_shared(lat_s)),
        "l"(src), "r"(bytes), "r"(b)
        : "memory");
  }
  __syncwarp();
  bool ok = stage_wait(b);
  if (!ok) {
    if (lane == 0) atomicOr(&g_stage_timeout, 1);
    stage_wait(b);  // give the copy in flight a second bounded wait before the CTA moves on
  }
  return __all_sync(0xffffffffu, ok);
}

__device__ __forceinline__ void bulk_stage_out(uint32_t *dst, const uint32_t *lat_s, uint32_t bytes,
                                               int lane) {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");  // the sweep's writes, to the copy
  __syncwarp();
  if (lane == 0) {
    asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;" ::"l"(dst),
                 "r"((uint32_t)__cvta_generic_to_shared(lat_s)), "r"(bytes)
                 : "memory");
    asm volatile("cp.async.bulk.commit_group;" ::: "memory");
    asm volatile("cp.async.bulk.wait_group 0;" ::: "memory");
  }
  __syncwarp();
}

__device__ __forceinline__ uint32_t bit_at(const uint32_t *my, int s) {
  return (my[(s >> 5) * kTile] >> (s & 31)) & 1u;
}

// Five opaque register constants materialised at the top of each block.
// They take no part in the arithmetic; they change how the compiler orders
// a block's draws against the previous block's applies.  Measured: 4.57-4.59e11
// attempts/s with them, 4.48e11 without, 4.47-4.55e11 with 1, 2, 3 or 8 of
// them or with an empty asm statement or a memory clobber instead.  Results
// are bit-identical either way.
__device__ __forceinline__ void block_marks() {
  [[maybe_unused]] uint32_t m0, m1, m2, m3, m4;
  asm volatile("mov.u32 %0, 16;" : "=r"(m0));
  asm volatile("mov.u32 %0, 2;" : "=r"(m1));
  asm volatile("mov.u32 %0, 1073741824;" : "=r"(m2));
  asm volatile("mov.u32 %0, 1;" : "=r"(m3));
  asm volatile("mov.u32 %0, 362437;" : "=r"(m4));
}

__device__ __forceinline__ void epilogue_mag(const uint32_t *my, const SweepLaunch &p, int N,
                                             int W, bool live, int rep) {
  if (p.mag_out != nullptr && live) {
    int pc = 0;
    for (int w = 0; w < W; ++w) pc += __popc(my[w * kTile]);
    // (float)(sum of +-1 spins) / (float)N, the sum being exact in float.
    p.mag_out[rep] = (float)(2 * pc - N) / (float)N;
  }
}

// One lane's attempts of a generic-kernel batch on its staged lattice `my`
// (word w at my[w*32]); L_ > 0 compile-time side length, else L.
template <int L_, bool kFloatCmp, int kRng, bool kStoreAlways>
__device__ __forceinline__ void exact_run(const SweepLaunch &p, int rep, uint32_t *my, int L,
                                          const uint32_t *thr_s, const float *pacc_s) {
  const int N = L * L;
  RngPolicy<kRng> rg;
  rg.load(p.rng, p.rng_stride, rep);
  const float shrink = (1.0f - FLT_EPSILON) * (float)N;
  // MWC64X stream: attempts in blocks of 16, the block's 32 draws first (see
  // row_draw64), flat over all attempts of the batch.  Measured against the
  // per-sweep loop below: L=20 +9 %, L=48 +2 to +5 %, L=100 +18 % (4096 and
  // 32768 replicas); on the XORWOW stream the blocks were slower (L=48 -29 %,
  // L=100 -2 %), so that stream keeps the loop below.
  if constexpr (!kFloatCmp && kRng == kRngMwc) {
    const int total = N * p.nsweeps;
    int a = 0;
    for (; a + 16 <= total; a += 16) {
      uint32_t ss[16], xx[16];
      block_marks();
#pragma unroll
      for (int j = 0; j < 16; ++j) {
        ss[j] = rg.template site<(L_ > 0 ? L_ * L_ : 0)>(shrink, N);
        xx[j] = rg.next();
      }
#pragma unroll
      for (int j = 0; j < 16; ++j) {
        const int s = (int)ss[j];
        const int row = s / L;
        const int col = s - row * L;
        const int su = row == 0 ? s + N - L : s - L;
        const int sd = row == L - 1 ? s - N + L : s + L;
        const int sl = col == 0 ? s + L - 1 : s - 1;
        const int sr = col == L - 1 ? s - L + 1 : s + 1;
        const uint32_t wc = my[(s >> 5) * kTile];
        const uint32_t bs = (wc >> (s & 31)) & 1u;
        const uint32_t k = bit_at(my, su) + bit_at(my, sd) + bit_at(my, sl) + bit_at(my, sr);
        const uint32_t cls = 5u * bs + k;
        const bool acc = xx[j] <= thr_s[cls];
        if constexpr (kStoreAlways) {
          my[(s >> 5) * kTile] = acc ? wc ^ (1u << (s & 31)) : wc;
        } else {
          if (acc) my[(s >> 5) * kTile] = wc ^ (1u << (s & 31));
        }
      }
    }
    for (; a < total; ++a) {
      const int s = (int)rg.template site<(L_ > 0 ? L_ * L_ : 0)>(shrink, N);
      const int row = s / L;
      const int col = s - row * L;
      const int su = row == 0 ? s + N - L : s - L;
      const int sd = row == L - 1 ? s - N + L : s + L;
      const int sl = col == 0 ? s + L - 1 : s - 1;
      const int sr = col == L - 1 ? s - L + 1 : s + 1;
      const uint32_t wc = my[(s >> 5) * kTile];
      const uint32_t bs = (wc >> (s & 31)) & 1u;
      const uint32_t k = bit_at(my, su) + bit_at(my, sd) + bit_at(my, sl) + bit_at(my, sr);
      const uint32_t cls = 5u * bs + k;
      const uint32_t x2 = rg.next();
      const bool acc = x2 <= thr_s[cls];
      if constexpr (kStoreAlways) {
        my[(s >> 5) * kTile] = acc ? wc ^ (1u << (s & 31)) : wc;
      } else {
        if (acc) my[(s >> 5) * kTile] = wc ^ (1u << (s & 31));
      }
    }
  } else {
    for (int sw = 0; sw < p.nsweeps; ++sw) {
      // unroll 4: 1.2-1.5x over the compiler's choice on the reference stream
      // (L=48: 2.45e11 vs 2.04e11 attempts/s at 32768 replicas; L=100: 3.3e10 vs 2.2e10)
#pragma unroll 4
      for (int a = 0; a < N; ++a) {
        const int s = (int)rg.template site<(L_ > 0 ? L_ * L_ : 0)>(shrink, N);
        const int row = s / L;
        const int col = s - row * L;
        const int su = row == 0 ? s + N - L : s - L;
        const int sd = row == L - 1 ? s - N + L : s + L;
        const int sl = col == 0 ? s + L - 1 : s - 1;
        const int sr = col == L - 1 ? s - L + 1 : s + 1;
        const uint32_t wc = my[(s >> 5) * kTile];
        const uint32_t bs = (wc >> (s & 31)) & 1u;
        const uint32_t k = bit_at(my, su) + bit_at(my, sd) + bit_at(my, sl) + bit_at(my, sr);
        const uint32_t cls = 5u * bs + k;
        const uint32_t x2 = rg.next();
        bool acc;
        if (kFloatCmp) {
          acc = _curand_uniform(x2) < pacc_s[2 * cls];  // index 10*bs + 2k
        } else {
          acc = x2 <= thr_s[cls];
        }
        if constexpr (kStoreAlways) {  // written back unchanged when rejected: no branch
          my[(s >> 5) * kTile] = acc ? wc ^ (1u << (s & 31)) : wc;
        } else {
          if (acc) my[(s >> 5) * kTile] = wc ^ (1u << (s & 31));
        }
      }
    }
  }
  rg.store(p.rng, p.rng_stride, rep);
}

// ---------------------------------------------------------------------------
// Exact sweep.  L_ > 0: compile-time side length; L_ == 0: runtime p.L.
// ---------------------------------------------------------------------------
template <int L_, bool kFloatCmp, int kRng, bool kStoreAlways = false>
__global__ void __launch_bounds__(256) k_sweep_exact(SweepLaunch p) {
  const int L = L_ > 0 ? L_ : p.L;
  const int N = L * L;
  const int W = (N + 31) >> 5;
  extern __shared__ __align__(16) uint32_t smem[];
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  const int nwarps = blockDim.x >> 5;

  uint32_t *thr_s = smem;                                  // [10]
  float *pacc_s = reinterpret_cast<float *>(smem + 16);    // [20]
  if (threadIdx.x < 10) thr_s[threadIdx.x] = p.thr[threadIdx.x];
  if (threadIdx.x < 20) pacc_s[threadIdx.x] = p.pacc_f[threadIdx.x];

  const int n_act = live_count(p);
  const int tile = blockIdx.x * nwarps + warp;
  const int slot = tile * kTile + lane;
  const bool tile_live = tile * kTile < n_act;
  const bool live = slot < n_act;
  const int rep = live ? (p.active ? p.active[slot] : slot) : 0;
  uint32_t *lat_s = smem + kHeaderWords + warp * (W * kTile);
  if (tile_live) stage_in(lat_s, p, W, tile, lane, live, rep);
  __syncthreads();
  if (!tile_live) return;

  uint32_t *my = lat_s + lane;
  if (live) exact_run<L_, kFloatCmp, kRng, kStoreAlways>(p, rep, my, L, thr_s, pacc_s);
  __syncwarp();
  epilogue_mag(my, p, N, W, live, rep);
  stage_out(lat_s, p, W, tile, lane, live, rep);
}

// ---------------------------------------------------------------------------
// The same sweep for lattices larger than shared memory holds (the role of
// the reference's global-memory method 0): each lane works on its replica's
// interleaved words in place in HBM (the L2 keeps the active lines).
// ---------------------------------------------------------------------------
template <bool kFloatCmp, int kRng>
__global__ void __launch_bounds__(128) k_sweep_global(SweepLaunch p) {
  const int L = p.L;
  const int N = L * L;
  const int W = (N + 31) >> 5;
  __shared__ uint32_t thr_s[16];
  __shared__ float pacc_s[20];
  if (threadIdx.x < 10) thr_s[threadIdx.x] = p.thr[threadIdx.x];
  if (threadIdx.x < 20) pacc_s[threadIdx.x] = p.pacc_f[threadIdx.x];
  __syncthreads();
  const int n_act = live_count(p);
  const int slot = blockIdx.x * blockDim.x + threadIdx.x;
  if (slot >= n_act) return;
  const int rep = p.active ? p.active[slot] : slot;
  uint32_t *my = p.lat + (size_t)(rep >> 5) * W * kTile + (rep & 31);
  RngPolicy<kRng> rg;
  rg.load(p.rng, p.rng_stride, rep);
  const float shrink = (1.0f - FLT_EPSILON) * (float)N;
  for (int sw = 0; sw < p.nsweeps; ++sw) {
    // unroll 4: L=300, 2048 replicas, 4.3e9 vs 2.4e9 attempts/s (exact stream),
    // 4.4e9 vs 3.7e9 (MWC64X)
#pragma unroll 4
    for (int a = 0; a < N; ++a) {
      const int s = (int)rg.template site<0>(shrink, N);
      const int row = s / L;
      const int col = s - row * L;
      const int su = row == 0 ? s + N - L : s - L;
      const int sd = row == L - 1 ? s - N + L : s + L;
      const int sl = col == 0 ? s + L - 1 : s - 1;
      const int sr = col == L - 1 ? s - L + 1 : s + 1;
      const uint32_t wc = my[(size_t)(s >> 5) * kTile];
      const uint32_t bs = (wc >> (s & 31)) & 1u;
      const uint32_t k = bit_at(my, su) + bit_at(my, sd) + bit_at(my, sl) + bit_at(my, sr);
      const uint32_t cls = 5u * bs + k;
      const uint32_t x2 = rg.next();
      const bool acc = kFloatCmp ? (_curand_uniform(x2) < pacc_s[2 * cls]) : (x2 <= thr_s[cls]);
      if (acc) my[(size_t)(s >> 5) * kTile] = wc ^ (1u << (s & 31));
    }
  }
  rg.store(p.rng, p.rng_stride, rep);
  epilogue_mag(my, p, N, W, true, rep);
}

// ---------------------------------------------------------------------------
// Exact sweep specialised for L a power of two and a multiple of 32 (32, 64,
// 128): a row is R = L/32 whole words, so
//   * up/down neighbours are the words R rows-words away, at the same bit,
//     and their byte offsets wrap with a mask (4N is a power of two);
//   * left/right neighbours sit in the centre word except at bit 0 / 31,
//     where they are in the row's edge word (for R == 2 simply word w^1);
//   * one funnel shift of (hi:lo) brings left/centre/right to bits 2..4 and
//     two rotates bring up/down to bits 5..6, giving pattern*4 directly as a
//     byte offset into a 32-entry threshold table indexed by the 5 spins.
// Same arithmetic, stream consumption and result as k_sweep_exact.
// ---------------------------------------------------------------------------
template <int Words, bool kStatic>
struct LatticeStore;

template <int Words>
struct LatticeStore<Words, true> {
  __device__ __forceinline__ static uint32_t *get(uint32_t *) {
    __shared__ __align__(128) uint32_t lat[Words];
    return lat;
  }
};

template <int Words>
struct LatticeStore<Words, false> {
  __device__ __forceinline__ static uint32_t *get(uint32_t *dyn) { return dyn; }
};

// One attempt of k_sweep_rows on site s.  kLookahead: also draw the next
// attempt's site (after this attempt's acceptance draw, as the reference's
// stream order requires) so its conversion overlaps this attempt's
// shared-memory round trips.
template <int L, bool kFloatCmp, bool kLookahead, bool kStoreAlways, typename Rng>
__device__ __forceinline__ void row_attempt(uint32_t &s, Rng &rg, const char *latb,
                                            const char *thrb, const char *paccb, uint32_t lane4,
                                            float shrink) {
  constexpr int N = L * L;
  constexpr int R = L / 32;
  constexpr bool kPow2 = (L & (L - 1)) == 0;
  constexpr uint32_t kMask = (uint32_t)(4 * N - 1) & ~127u;  // word part of a byte offset
  const uint32_t b = s & 31u;
  uint32_t offc, offu, offd;
  if constexpr (kPow2) {
    offc = ((s << 2) & kMask) | lane4;
    offu = ((offc - 128u * R) & kMask) | lane4;
    offd = ((offc + 128u * R) & kMask) | lane4;
  } else {  // rows of R words, R not a power of two: wrap by compare (4N bytes per tile)
    offc = ((s << 2) & ~127u) | lane4;
    offu = offc >= 128u * R ? offc - 128u * R : offc + (4u * N - 128u * R);
    offd = offc + 128u * R < 4u * N ? offc + 128u * R : offc - (4u * N - 128u * R);
  }
  const uint32_t wu = *reinterpret_cast<const uint32_t *>(latb + offu);
  const uint32_t wd = *reinterpret_cast<const uint32_t *>(latb + offd);
  uint32_t wc, lo, hi;
  if constexpr (R == 1) {
    wc = *reinterpret_cast<const uint32_t *>(latb + offc);
    lo = hi = wc;
  } else if constexpr (R == 2) {
    wc = *reinterpret_cast<const uint32_t *>(latb + offc);
    const uint32_t wx = *reinterpret_cast<const uint32_t *>(latb + (offc ^ 128u));
    if constexpr (Rng::kKind == kRngXorwow) {
      // The row is the circular 64 bits (wx:wc) seen from the site's word: for
      // b >= 3 the bits b-1..b+1 sit in (wx:wc) >> (b-3) (b = 31 reaches wx
      // bit 0); for b < 3 the left neighbour wraps to the top of wx, so the
      // pair is read as (wc:wx), whose shift by b+29 lands on the same bits.
      // One compare instead of two: 4.23e11 vs 4.11e11 attempts/s.
      const bool wrap = b < 3u;
      lo = wrap ? wx : wc;
      hi = wrap ? wc : wx;
    } else {  // with the MWC64X stream the two-compare form schedules better (4.96e11 vs 4.89e11)
      lo = (b == 0u) ? wx : wc;
      hi = (b == 31u) ? wx : wc;
    }
  } else {
    // word of the site within its row
    const uint32_t wi = kPow2 ? (offc >> 7) & (uint32_t)(R - 1) : (s >> 5) % (uint32_t)R;
    const uint32_t offl = (b == 0u) ? (wi == 0u ? offc + 128u * (R - 1) : offc - 128u) : offc;
    const uint32_t offr =
        (b == 31u) ? (wi == (uint32_t)(R - 1) ? offc - 128u * (R - 1) : offc + 128u) : offc;
    lo = *reinterpret_cast<const uint32_t *>(latb + offl);
    hi = *reinterpret_cast<const uint32_t *>(latb + offr);
    wc = (b == 0u) ? hi : lo;
  }
  const uint32_t t = __funnelshift_r(lo, hi, b + 29u);  // bits 2,3,4: left, centre, right
  const uint32_t u = __funnelshift_r(wu, wu, b + 27u);  // bit 5: up
  const uint32_t d = __funnelshift_r(wd, wd, b + 26u);  // bit 6: down
  const uint32_t p4 = (t & 0x1Cu) | (u & 0x20u) | (d & 0x40u);
  const uint32_t x2 = rg.next();
  const uint32_t sc = s;
  if constexpr (kLookahead) s = rg.template site<N>(shrink, N);
  bool acc;
  if constexpr (kFloatCmp) {
    acc = _curand_uniform(x2) < *reinterpret_cast<const float *>(paccb + p4);
  } else {
    acc = x2 <= *reinterpret_cast<const uint32_t *>(thrb + p4);
  }
  uint32_t *dst = reinterpret_cast<uint32_t *>(const_cast<char *>(latb) + offc);
  if constexpr (kStoreAlways) {
    *dst = acc ? wc ^ (1u << (sc & 31u)) : wc;  // rejected: the word written back unchanged
  } else {
    if (acc) *dst = wc ^ (1u << (sc & 31u));
  }
}

// Threshold and float tables of the row kernels, indexed by the 5-spin
// pattern (bits 0 left, 1 centre, 2 right, 3 up, 4 down; 1 == spin +1).
__device__ __forceinline__ void pattern_tables(const SweepLaunch &p, uint32_t *thrP, float *paccP,
                                               int lane) {
  const int c = (lane >> 1) & 1;
  const int cls = 5 * c + __popc(lane & 0x1D);
  thrP[lane] = p.thr[cls];
  paccP[lane] = p.pacc_f[2 * cls];
}

// The L=64 row kernel (integer thresholds, centre word written back on every
// attempt; both streams) runs its attempts in blocks of K, each
// in two phases: row_draw64 takes the block's 2K draws in the reference's
// order (site, acceptance, site, ...) and each site's word offset, then
// row_apply64 applies the K attempts in order.  The applies form a chain of
// shared-memory round trips with only their own arithmetic in between, and
// the draws are independent work the scheduler can issue back to back; the
// trajectory is the row_attempt loop's (same draws, same attempts, same
// order).
//   The site is floor(fl(shrink * u)) as in the reference.  With f =
// fl(shrink * u) in [0, N), the sum f + 2^23 rounded down is 2^23 + floor(f)
// (the floats in [2^23, 2^24) are the integers), whose bit pattern is
// sb = 0x4B000000 + floor(f).  0x4B000000 has no bit below bit 24, so sb
// stands in for the site wherever only its low bits count: the word offset
// (sb << 2 masked), the funnel-shift amounts (taken mod 32), the flip bit
// (a funnel shift, also mod 32) and the wrap test on the bit position
// (sb << 27 keeps the five low bits on top).
// Measured on the headline workload (32768 replicas, 100 sweeps per launch,
// exact stream, one B200): 4.78-4.80e11 attempts/s with two blocks per loop
// iteration and the site's row loaded before the up/down words (one block
// per iteration: 4.58e11, 4.62e11 with the row first; the unrolled
// row_attempt loop: 4.41e11).  Blocks of 8 or 32, the up/down offsets
// computed in the draw phase, the next block's draws interleaved with this
// block's applies, and starting odd tiles half a block ahead were all
// slower.  On the MWC64X stream (site = the draw's top 12 bits, an exact
// integer already): 5.11e11 against 4.91e11 for its unrolled loop (one block
// per iteration without the marks had been slower, 4.87e11).  With the
// marks below, blocks of 8 (4.50e11) or 32
// (4.46e11), a second set of marks before the applies (4.50e11), a store
// only on acceptance (4.35e11), a two-compare row window (4.51e11), four
// blocks per iteration (2.7e11) and a register cap of 80 (4.42e11) were
// slower.


template <int L, int K, typename Rng>
__device__ __forceinline__ void row_draw64(Rng &rg, uint32_t (&offc)[K], uint32_t (&sbits)[K],
                                           uint32_t (&x2)[K], uint32_t lane4, float shrink) {
  static_assert(L == 64, "rows of two words");
  constexpr int N = L * L;
  constexpr uint32_t kMask = (uint32_t)(4 * N - 1) & ~127u;  // word part of a byte offset
  block_marks();
#pragma unroll
  for (int j = 0; j < K; ++j) {
    uint32_t sb;
    if constexpr (Rng::kKind == kRngXorwow)
      sb = __float_as_uint(__fadd_rd(shrink * _curand_uniform(rg.next()), 8388608.0f));
    else  // MWC64X: the draw's top 12 bits (N = 4096)
      sb = rg.template site<N>(shrink, N);
    x2[j] = rg.next();
    offc[j] = ((sb << 2) & kMask) | lane4;
    sbits[j] = sb;
  }
}

template <int L, int K>
__device__ __forceinline__ void row_apply64(const uint32_t (&offc)[K], const uint32_t (&sbits)[K],
                                            const uint32_t (&x2)[K], const char *latb,
                                            const char *thrb, uint32_t lane4) {
  constexpr int N = L * L;
  constexpr uint32_t kMask = (uint32_t)(4 * N - 1) & ~127u;
#pragma unroll
  for (int j = 0; j < K; ++j) {
    const uint32_t oc = offc[j], sb = sbits[j];
    // the site's row first (its words end the chain's critical path soonest)
    const uint32_t wc = *reinterpret_cast<const uint32_t *>(latb + oc);
    const uint32_t wx = *reinterpret_cast<const uint32_t *>(latb + (oc ^ 128u));
    const uint32_t wu = *reinterpret_cast<const uint32_t *>(latb + (((oc - 256u) & kMask) | lane4));
    const uint32_t wd = *reinterpret_cast<const uint32_t *>(latb + (((oc + 256u) & kMask) | lane4));
    // the row's circular 64 bits seen from the site's word (see row_attempt):
    // bit position b = sb mod 32 below 3 reads the pair the other way round
    const bool wrap = (sb << 27) < (3u << 27);
    const uint32_t lo = wrap ? wx : wc;
    const uint32_t hi = wrap ? wc : wx;
    const uint32_t t = __funnelshift_r(lo, hi, sb + 29u);  // bits 2,3,4: left, centre, right
    const uint32_t u = __funnelshift_r(wu, wu, sb + 27u);  // bit 5: up
    const uint32_t d = __funnelshift_r(wd, wd, sb + 26u);  // bit 6: down
    const uint32_t p4 = (t & 0x1Cu) | (u & 0x20u) | (d & 0x40u);
    const bool acc = x2[j] <= *reinterpret_cast<const uint32_t *>(thrb + p4);
    const uint32_t bit = __funnelshift_l(0u, 1u, sb);  // 1 << b
    *reinterpret_cast<uint32_t *>(const_cast<char *>(latb) + oc) = acc ? wc ^ bit : wc;
  }
}

// The same blocks for the other row-kernel sides (L = 32, 96, 128) on the
// reference stream: row_draw / row_apply below are the L=64 pair written for
// rows of one, two or more words.  L=64 keeps its own pair: compiled from the
// generic source its schedule came out 4 % slower (4.41e11 against 4.59e11).
// Measured against the unrolled row_attempt loop, one block per iteration:
// L=96 +8.7 % (2048 and 32768 replicas), L=128 +2.9 % (512 and 16384), L=32
// +3.6 % (32768; 16384: -0.3 %); the uneven batch 3 % faster on both its
// paths.  Two blocks per iteration then gave L=32 a further 3.9 % and, with
// the site's row loaded first, L=128 3.3 %; L=96 lost 4-10 % with either.
// On the MWC64X stream the final form gives L=32 +5 % (16384 replicas) to
// +9 % (32768) and L=128 +2 % over the unrolled loop; L=96 keeps that loop
// (blocks: -1.9 %).

// Word part of a byte offset into a tile image of 4N bytes, rounded up to a
// power of two (the offset of the site's word is (site << 2) under it).
template <int L>
__host__ __device__ constexpr uint32_t row_word_mask() {
  uint32_t m = 128;
  while (m < 4u * L * L) m <<= 1;
  return (m - 1) & ~127u;
}

template <int L, int K, typename Rng>
__device__ __forceinline__ void row_draw(Rng &rg, uint32_t (&offc)[K], uint32_t (&sbits)[K],
                                         uint32_t (&x2)[K], uint32_t lane4, float shrink) {
  static_assert(L * L <= (1 << 15), "site bits and word offsets below 2^17");
  constexpr int N = L * L;
  constexpr uint32_t kMaskD = row_word_mask<L>();
  block_marks();
#pragma unroll
  for (int j = 0; j < K; ++j) {
    uint32_t sb;
    if constexpr (Rng::kKind == kRngXorwow)
      sb = __float_as_uint(__fadd_rd(shrink * _curand_uniform(rg.next()), 8388608.0f));
    else  // MWC64X: the exact integer site (power-of-two N: top bits; L=96: high product)
      sb = rg.template site<N>(shrink, N);
    x2[j] = rg.next();
    offc[j] = ((sb << 2) & kMaskD) | lane4;
    sbits[j] = sb;
  }
}

template <int L, int K>
__device__ __forceinline__ void row_apply(const uint32_t (&offc)[K], const uint32_t (&sbits)[K],
                                          const uint32_t (&x2)[K], const char *latb,
                                          const char *thrb, uint32_t lane4) {
  constexpr int N = L * L;
  constexpr int R = L / 32;
  constexpr bool kPow2 = (L & (L - 1)) == 0;
  constexpr uint32_t kMask = (uint32_t)(4 * N - 1) & ~127u;
#pragma unroll
  for (int j = 0; j < K; ++j) {
    const uint32_t oc = offc[j], sb = sbits[j];
    const uint32_t bt = sb << 27;  // bit position b on top
    uint32_t offu, offd;
    if constexpr (kPow2) {
      offu = ((oc - 128u * R) & kMask) | lane4;
      offd = ((oc + 128u * R) & kMask) | lane4;
    } else {  // rows of R words, R not a power of two: wrap by compare
      offu = oc >= 128u * R ? oc - 128u * R : oc + (4u * N - 128u * R);
      offd = oc + 128u * R < 4u * N ? oc + 128u * R : oc - (4u * N - 128u * R);
    }
    // L=128 loads the site's row before the up/down words (3.3 % faster; the
    // other sides keep up/down first)
    constexpr bool kRowFirst = L == 128;
    uint32_t wu = 0, wd = 0;
    if constexpr (!kRowFirst) {
      wu = *reinterpret_cast<const uint32_t *>(latb + offu);
      wd = *reinterpret_cast<const uint32_t *>(latb + offd);
    }
    uint32_t wc, lo, hi;
    if constexpr (R == 1) {
      wc = *reinterpret_cast<const uint32_t *>(latb + oc);
      lo = hi = wc;
    } else if constexpr (R == 2) {
      // the row's circular 64 bits seen from the site's word (see row_attempt):
      // b below 3 reads the pair the other way round
      wc = *reinterpret_cast<const uint32_t *>(latb + oc);
      const uint32_t wx = *reinterpret_cast<const uint32_t *>(latb + (oc ^ 128u));
      const bool wrap = bt < (3u << 27);
      lo = wrap ? wx : wc;
      hi = wrap ? wc : wx;
    } else {
      // word of the site within its row; at b = 0 / 31 the left / right
      // neighbour is in the previous / next word of the row (circularly)
      const uint32_t wi =
          kPow2 ? (oc >> 7) & (uint32_t)(R - 1) : ((sb & 0x7FFFFFu) >> 5) % (uint32_t)R;
      const uint32_t offl = (bt == 0u) ? (wi == 0u ? oc + 128u * (R - 1) : oc - 128u) : oc;
      const uint32_t offr =
          (bt == (31u << 27)) ? (wi == (uint32_t)(R - 1) ? oc - 128u * (R - 1) : oc + 128u) : oc;
      lo = *reinterpret_cast<const uint32_t *>(latb + offl);
      hi = *reinterpret_cast<const uint32_t *>(latb + offr);
      wc = (bt == 0u) ? hi : lo;
    }
    if constexpr (kRowFirst) {
      wu = *reinterpret_cast<const uint32_t *>(latb + offu);
      wd = *reinterpret_cast<const uint32_t *>(latb + offd);
    }
    const uint32_t t = __funnelshift_r(lo, hi, sb + 29u);  // bits 2,3,4: left, centre, right
    const uint32_t u = __funnelshift_r(wu, wu, sb + 27u);  // bit 5: up
    const uint32_t d = __funnelshift_r(wd, wd, sb + 26u);  // bit 6: down
    const uint32_t p4 = (t & 0x1Cu) | (u & 0x20u) | (d & 0x40u);
    const bool acc = x2[j] <= *reinterpret_cast<const uint32_t *>(thrb + p4);
    const uint32_t bit = __funnelshift_l(0u, 1u, sb);  // 1 << b
    *reinterpret_cast<uint32_t *>(const_cast<char *>(latb) + oc) = acc ? wc ^ bit : wc;
  }
}

// One lane's attempts of a row-kernel batch (N * nsweeps of them) on its
// staged lattice, software-pipelined: draw order x1(a), x2(a), x1(a+1), ...
// as in the reference.  The host keeps N*nsweeps < 2^31.
// kCompact: one block of attempts per loop iteration at every side (half the
// loop's code; for launches whose kernels share an SM's instruction cache
// with other kernels, the batched groups).
template <int L, bool kFloatCmp, bool kStoreAlways, int kRng, bool kCompact = false>
__device__ __forceinline__ void rows_run(const SweepLaunch &p, int rep, const uint32_t *lat,
                                         const uint32_t *thrP, const float *paccP, int lane) {
  constexpr int N = L * L;
  const char *latb = reinterpret_cast<const char *>(lat);
  const char *thrb = reinterpret_cast<const char *>(thrP);
  const char *paccb = reinterpret_cast<const char *>(paccP);
  RngPolicy<kRng> rg;
  rg.load(p.rng, p.rng_stride, rep);
  const float shrink = (1.0f - FLT_EPSILON) * (float)N;
  const uint32_t lane4 = (uint32_t)lane << 2;
  const int total = N * p.nsweeps;
  if constexpr (L == 64 && !kFloatCmp && kStoreAlways) {
    // the default L=64 kernel on the reference stream: blocks of 16 attempts
    // (total = 4096 * nsweeps is a multiple of 16)
    uint32_t offc[16], sbits[16], x2[16];
    if constexpr (kCompact) {
      for (int a = 0; a < total; a += 16) {
        row_draw64<L, 16>(rg, offc, sbits, x2, lane4, shrink);
        row_apply64<L, 16>(offc, sbits, x2, latb, thrb, lane4);
      }
    } else {
      // two blocks per loop iteration (4 blocks: 2.7e11, the body outgrows
      // the instruction cache)
#pragma unroll 2
      for (int a = 0; a < total; a += 16) {
        row_draw64<L, 16>(rg, offc, sbits, x2, lane4, shrink);
        row_apply64<L, 16>(offc, sbits, x2, latb, thrb, lane4);
      }
    }
    rg.store(p.rng, p.rng_stride, rep);
    return;
  }
  // (MWC64X at L=96 keeps the unrolled loop: blocks -1.9 %)
  if constexpr (L != 64 && (kRng == kRngXorwow || L != 96) && !kFloatCmp && kStoreAlways) {
    // blocks of 16 attempts (total = L * L * nsweeps, a multiple of 16 for
    // L = 32, 96, 128)
    uint32_t offc[16], sbits[16], x2[16];
    if constexpr (L == 96 || kCompact) {  // one block per iteration (L=96, two: -4 to -10 %)
      for (int a = 0; a < total; a += 16) {
        row_draw<L, 16>(rg, offc, sbits, x2, lane4, shrink);
        row_apply<L, 16>(offc, sbits, x2, latb, thrb, lane4);
      }
    } else {  // two blocks per iteration: L=32 +3.9 %, L=128 +3.3 % (with the row first)
#pragma unroll 2
      for (int a = 0; a < total; a += 16) {
        row_draw<L, 16>(rg, offc, sbits, x2, lane4, shrink);
        row_apply<L, 16>(offc, sbits, x2, latb, thrb, lane4);
      }
    }
    rg.store(p.rng, p.rng_stride, rep);
    return;
  }
  uint32_t s = rg.template site<N>(shrink, N);
  if constexpr (L == 64 && kRng == kRngXorwow) {
    // unroll measured at L=64 on the reference stream: 8 -> 4.40e11, 5 -> 4.23e11,
    // 16 -> 4.36e11, 10 -> 4.28e11 attempts/s (the MWC64X stream is fastest at 5)
#pragma unroll 8
    for (int a = 0; a < total - 1; ++a)
      row_attempt<L, kFloatCmp, true, kStoreAlways>(s, rg, latb, thrb, paccb, lane4, shrink);
    row_attempt<L, kFloatCmp, false, kStoreAlways>(s, rg, latb, thrb, paccb, lane4, shrink);
  } else if constexpr (L == 128 || (L == 32 && kRng == kRngXorwow) ||
                       (L == 96 && kRng == kRngMwc)) {
    // unroll 16 measured 2-4 % faster than 5 for these (L, stream) pairs
    // (e.g. L=128, 16384 replicas: 1.27e11 vs 1.23e11 exact, 1.45e11 vs 1.42e11
    // MWC64X; L=32 exact, 16384 replicas: 2.85e11 vs 2.74e11) and slower for the others
#pragma unroll 16
    for (int a = 0; a < total - 1; ++a)
      row_attempt<L, kFloatCmp, true, kStoreAlways>(s, rg, latb, thrb, paccb, lane4, shrink);
    row_attempt<L, kFloatCmp, false, kStoreAlways>(s, rg, latb, thrb, paccb, lane4, shrink);
  } else {
#pragma unroll 5
    for (int a = 0; a < total - 1; ++a)
      row_attempt<L, kFloatCmp, true, kStoreAlways>(s, rg, latb, thrb, paccb, lane4, shrink);
    row_attempt<L, kFloatCmp, false, kStoreAlways>(s, rg, latb, thrb, paccb, lane4, shrink);
  }
  rg.store(p.rng, p.rng_stride, rep);
}

template <int L, bool kStatic, bool kFloatCmp, int kRng, bool kStoreAlways = false,
          bool kBulk = false, bool kCompact = false>
__global__ void __launch_bounds__(32) k_sweep_rows(SweepLaunch p) {
  static_assert(L % 32 == 0, "rows of whole words");
  constexpr int N = L * L;
  constexpr int W = N / 32;
  __shared__ __align__(16) uint32_t thrP[32];   // threshold by 5-spin pattern
  __shared__ __align__(16) float paccP[32];     // float table by pattern
  extern __shared__ __align__(16) uint32_t dyn[];
  uint32_t *lat = LatticeStore<W * kTile, kStatic>::get(dyn);

  const int lane = threadIdx.x;
  pattern_tables(p, thrP, paccP, lane);
  const int n_act = live_count(p);
  const int tile = blockIdx.x;
  if (tile * kTile >= n_act) return;  // whole CTA (one warp) idle this batch
  const int slot = tile * kTile + lane;
  const bool live = slot < n_act;
  const int rep = live ? (p.active ? p.active[slot] : slot) : 0;
  constexpr uint32_t kTileBytes = W * kTile * sizeof(uint32_t);
  bool staged = true;
  if constexpr (kBulk) {
    __shared__ __align__(8) uint64_t stage_bar;
    if (p.active == nullptr)
      staged = bulk_stage_in(lat, p.lat + (size_t)tile * W * kTile, kTileBytes, &stage_bar, lane);
    else
      stage_in(lat, p, W, tile, lane, live, rep);
  } else {
    stage_in(lat, p, W, tile, lane, live, rep);
  }
  __syncwarp();

  if (live && staged && p.nsweeps > 0)
    rows_run<L, kFloatCmp, kStoreAlways, kRng, kCompact>(p, rep, lat, thrP, paccP, lane);
  __syncwarp();
  if (!staged) return;  // the bulk load timed out: flagged, nothing written back
  epilogue_mag(lat + lane, p, N, W, live, rep);
  if constexpr (kBulk) {
    if (p.active == nullptr)
      bulk_stage_out(p.lat + (size_t)tile * W * kTile, lat, kTileBytes, lane);
    else
      stage_out(lat, p, W, tile, lane, live, rep);
  } else {
    stage_out(lat, p, W, tile, lane, live, rep);
  }
}

// ---------------------------------------------------------------------------
// Several replica groups of different L in one launch (the batched path).
// CTA b sweeps tile b - tile_begin[g] of the group g whose CTA range holds b,
// with that group's L-specialised attempt loop (the row loop for L = 32, 64,
// 96, 128; the generic loop otherwise) and its own tables, RNG states, active
// list and device live count.  Integer thresholds only.  The dynamic shared
// memory is the largest group's tile; the host orders groups by decreasing
// work per tile, so the longest chains start first.
// ---------------------------------------------------------------------------
template <int kRng>
__global__ void __launch_bounds__(32) k_sweep_multi(const SweepLaunch *groups,
                                                    const int *tile_begin, int ngroups) {
  __shared__ __align__(16) uint32_t thrP[32];
  __shared__ __align__(16) float paccP[32];
  extern __shared__ __align__(16) uint32_t dyn[];
  int g = 0;
  while (g + 1 < ngroups && (int)blockIdx.x >= tile_begin[g + 1]) ++g;
  const SweepLaunch &p = groups[g];
  const int lane = threadIdx.x;
  const int L = p.L, N = L * L, W = (N + 31) >> 5;
  const int n_act = live_count(p);
  const int tile = (int)blockIdx.x - tile_begin[g];
  if (tile * kTile >= n_act) return;  // whole CTA idle this batch
  const int slot = tile * kTile + lane;
  const bool live = slot < n_act;
  const int rep = live ? (p.active ? p.active[slot] : slot) : 0;
  const bool rows = L == 32 || L == 64 || L == 96 || L == 128;
  if (rows) pattern_tables(p, thrP, paccP, lane);
  else if (lane < 10) thrP[lane] = p.thr[lane];
  stage_in(dyn, p, W, tile, lane, live, rep);
  __syncwarp();
  if (live && p.nsweeps > 0) {
    switch (L) {
      case 32: rows_run<32, false, true, kRng, true>(p, rep, dyn, thrP, paccP, lane); break;
      case 64: rows_run<64, false, true, kRng, true>(p, rep, dyn, thrP, paccP, lane); break;
      case 96: rows_run<96, false, true, kRng, true>(p, rep, dyn, thrP, paccP, lane); break;
      case 128: rows_run<128, false, true, kRng, true>(p, rep, dyn, thrP, paccP, lane); break;
      case 48: exact_run<48, false, kRng, false>(p, rep, dyn + lane, L, thrP, paccP); break;
      default: exact_run<0, false, kRng, false>(p, rep, dyn + lane, L, thrP, paccP); break;
    }
  }
  __syncwarp();
  epilogue_mag(dyn + lane, p, N, W, live, rep);
  stage_out(dyn, p, W, tile, lane, live, rep);
}

// ---------------------------------------------------------------------------
// CPU-trace sweep: mc_sweep_cpu arithmetic (src/mc_cpu.c:41-89) on a replayed
// stream of doubles (row-u, col-u, xi) per attempt.
// ---------------------------------------------------------------------------
template <int L_>
__global__ void __launch_bounds__(256) k_sweep_trace_cpu(SweepLaunch p) {
  const int L = L_ > 0 ? L_ : p.L;
  const int N = L * L;
  const int W = (N + 31) >> 5;
  extern __shared__ __align__(16) uint32_t smem[];
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  const int nwarps = blockDim.x >> 5;
  double *pacc_s = reinterpret_cast<double *>(smem);  // [20] (160 B < header)
  if (threadIdx.x < 20) pacc_s[threadIdx.x] = p.pacc_cpu[threadIdx.x];
  const int n_act = live_count(p);
  const int tile = blockIdx.x * nwarps + warp;
  const int slot = tile * kTile + lane;
  const bool tile_live = tile * kTile < n_act;
  const bool live = slot < n_act;
  const int rep = live ? (p.active ? p.active[slot] : slot) : 0;
  uint32_t *lat_s = smem + kHeaderWords + warp * (W * kTile);
  if (tile_live) stage_in(lat_s, p, W, tile, lane, live, rep);
  __syncthreads();
  if (!tile_live) return;
  uint32_t *my = lat_s + lane;
  if (live) {
    const double *str = p.stream + (size_t)rep * 3 * (size_t)N * p.nsweeps;
    const long long total = (long long)N * p.nsweeps;
    for (long long a = 0; a < total; ++a) {
      const double ur = str[3 * a + 0], uc = str[3 * a + 1], xi = str[3 * a + 2];
      const int row = (int)floor(L * ur);
      const int col = (int)floor(L * uc);
      const int s = L * row + col;
      const int su = L * ((row + L - 1) % L) + col;
      const int sd = L * ((row + 1) % L) + col;
      const int sr = L * row + (col + 1) % L;
      const int sl = L * row + (col + L - 1) % L;
      const uint32_t wc = my[(s >> 5) * kTile];
      const uint32_t bs = (wc >> (s & 31)) & 1u;
      const uint32_t k = bit_at(my, su) + bit_at(my, sd) + bit_at(my, sl) + bit_at(my, sr);
      // reference index 5*(spin+1) + nsum + 4 == 10*bs + 2*k
      if (xi < pacc_s[10 * bs + 2 * k]) my[(s >> 5) * kTile] = wc ^ (1u << (s & 31));
    }
  }
  __syncwarp();
  epilogue_mag(my, p, N, W, live, rep);
  stage_out(lat_s, p, W, tile, lane, live, rep);
}

// ---------------------------------------------------------------------------
__global__ void k_rng_init(uint32_t *rng, int ngrids, int stride, unsigned long long seed) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= ngrids) return;
  curandStateXORWOW st;
  curand_init(seed, (unsigned long long)r, 0ull, &st);  // as src/gpu_tools.cu:130-133
  store_rng(st, rng, stride, r);
}

// thr[c] = T-1 with T = min{x in [0,2^32] : !(_curand_uniform(x) < P[2c])}.
// _curand_uniform is monotone non-decreasing in x (a rounded conversion then a
// fused multiply-add by a positive constant), so "x <= thr[c]" is exactly
// "_curand_uniform(x) < P[2c]" for every 32-bit x.  flags[0] is set when some
// class can never accept (T == 0); the host then uses the float comparison.
__global__ void k_build_thresholds(const float *pacc20, uint32_t *thr10, int *flags) {
  const int c = threadIdx.x;
  if (c >= 10) return;
  const float P = pacc20[2 * c];
  unsigned long long lo = 0ull, hi = 1ull << 32;
  while (lo < hi) {
    const unsigned long long mid = (lo + hi) >> 1;
    if (_curand_uniform((unsigned int)mid) < P) lo = mid + 1;
    else hi = mid;
  }
  if (lo == 0ull) atomicExch(flags, 1);
  thr10[c] = (uint32_t)(lo - 1ull);
}

__global__ void k_measure(const uint32_t *lat, int L, int ngrids, float *mag) {
  const int rep = blockIdx.x * blockDim.x + threadIdx.x;
  if (rep >= ngrids) return;
  const int N = L * L, W = (N + 31) >> 5;
  const uint32_t *src = lat + (size_t)(rep >> 5) * W * kTile + (rep & 31);
  int pc = 0;
  for (int w = 0; w < W; ++w) pc += __popc(src[(size_t)w * kTile]);
  mag[rep] = (float)(2 * pc - N) / (float)N;
}

// int32 grids [ngrids][N] -> lattice words; one thread per (tile, w, lane).
// per_input > 0: g holds ngrids/per_input input grids and replica r takes
// input r / per_input (the layout of init_grids_from_array, src/grid.c:59-67).
__global__ void k_pack_grids(const int *g, uint32_t *lat, int L, int ngrids, long long total,
                             int per_input) {
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= total) return;
  const int N = L * L, W = (N + 31) >> 5;
  const int lane = (int)(idx & 31);
  const long long tw = idx >> 5;
  const int w = (int)(tw % W);
  const long long tile = tw / W;
  const long long rep = tile * kTile + lane;
  uint32_t word = 0u;
  if (rep < ngrids) {
    const int *src = g + (per_input > 0 ? rep / per_input : rep) * N;
    const int s0 = w * 32;
    const int nb = min(32, N - s0);
    for (int b = 0; b < nb; ++b) word |= (src[s0 + b] == 1 ? 1u : 0u) << b;
  }
  lat[idx] = word;
}

// lattice words -> int32 grids; one thread per (replica, w).
__global__ void k_unpack_grids(const uint32_t *lat, int *g, int L, int ngrids, long long total) {
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= total) return;
  const int N = L * L, W = (N + 31) >> 5;
  const long long rep = idx / W;
  const int w = (int)(idx % W);
  const uint32_t word = lat[(rep >> 5) * W * kTile + (size_t)w * kTile + (rep & 31)];
  int *dst = g + rep * N;
  const int s0 = w * 32;
  const int nb = min(32, N - s0);
  for (int b = 0; b < nb; ++b) dst[s0 + b] = ((word >> b) & 1u) ? 1 : -1;
}

// gridstates.bin payload, N % 32 == 0: output word k is lattice word
// (rep = k / W, w = k % W): a per-tile transpose.
// gridstates.bin payload for L*L % 32 == 0: replica r's word w is word w of
// lane r%32 of tile r/32.  Each 32 x 8 block moves a 32-word x 32-replica
// square through a padded shared array: the tile's words are read as
// 128-byte rows, and each replica's 32 words are written as one 128-byte run.
__global__ void __launch_bounds__(256) k_pack_frame32t(const uint32_t *lat, uint32_t *out, int W,
                                                        int ngrids, int nchunks) {
  __shared__ uint32_t sq[32][33];
  const int tile = (int)(blockIdx.x / (unsigned)nchunks);
  const int w0 = (int)(blockIdx.x % (unsigned)nchunks) * 32;
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;  // 32 x 8
  const uint32_t *src = lat + (size_t)tile * W * kTile;
#pragma unroll
  for (int j = ty; j < 32; j += 8)
    if (w0 + j < W) sq[j][tx] = src[(size_t)(w0 + j) * kTile + tx];
  __syncthreads();
#pragma unroll
  for (int j = ty; j < 32; j += 8) {  // j: replica of the tile, tx: word of the square
    const int rep = tile * kTile + j;
    if (rep < ngrids && w0 + tx < W) out[(size_t)rep * W + w0 + tx] = sq[tx][j];
  }
}


// General payload: one thread per output byte, bit cursor over all spins.
__global__ void k_pack_frame8(const uint32_t *lat, uint8_t *out, int L, long long nbits,
                              long long nbytes) {
  const long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= nbytes) return;
  const int N = L * L, W = (N + 31) >> 5;
  uint32_t byte = 0u;
  for (int b = 0; b < 8; ++b) {
    const long long pbit = j * 8 + b;
    if (pbit >= nbits) break;
    const long long rep = pbit / N;
    const int s = (int)(pbit % N);
    const uint32_t word = lat[(rep >> 5) * W * kTile + (size_t)(s >> 5) * kTile + (rep & 31)];
    byte |= ((word >> (s & 31)) & 1u) << b;
  }
  out[j] = (uint8_t)byte;
}

template <typename Kern>
int launch_tiles(Kern kern, const SweepLaunch &p, cudaStream_t s) {
  const int W = words_per_replica(p.L);
  const int nwarps = p.warps_per_cta > 0 ? p.warps_per_cta : 1;
  const int tiles = tiles_for(p.n_active);
  if (tiles == 0) return GASP_OK;
  const size_t smem = (size_t)(kHeaderWords + nwarps * W * kTile) * sizeof(uint32_t);
  GASP_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  const int blocks = (tiles + nwarps - 1) / nwarps;
  kern<<<blocks, nwarps * 32, smem, s>>>(p);
  GASP_CUDA(cudaGetLastError());
  return GASP_OK;
}

// One warp per CTA; the lattice is static shared memory (kStatic) or dynamic.
template <typename Kern>
int launch_rows(Kern kern, const SweepLaunch &p, size_t dyn_smem, cudaStream_t s) {
  const int tiles = tiles_for(p.n_active);
  if (tiles == 0) return GASP_OK;
  if (dyn_smem > 0)
    GASP_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dyn_smem));
  kern<<<tiles, 32, dyn_smem, s>>>(p);
  GASP_CUDA(cudaGetLastError());
  return GASP_OK;
}

template <bool F, int K>
int dispatch_kind(const SweepLaunch &p, cudaStream_t s) {
  if (p.lattice_in_global) {
    if (p.n_active == 0) return GASP_OK;
    k_sweep_global<F, K><<<(p.n_active + 127) / 128, 128, 0, s>>>(p);
    GASP_CUDA(cudaGetLastError());
    return GASP_OK;
  }
  if (p.variant == 6) return launch_sweep_tail(p, s);    // one warp per replica (MWC64X)
  if (p.variant == 7) return launch_sweep_shared(p, s);  // shared site per tile (MWC64X)
  if (p.variant == 1) {  // the generic kernel, kept selectable for comparisons
    return launch_tiles(p.L == 64 ? k_sweep_exact<64, F, K> : k_sweep_exact<0, F, K>, p, s);
  }
  const size_t dyn128 = (size_t)words_per_replica(128) * kTile * sizeof(uint32_t);
  const size_t dyn96 = (size_t)words_per_replica(96) * kTile * sizeof(uint32_t);
  if (p.variant == 9) {  // variant 0 with bulk-copy staging of the tiles (measured slower)
    switch (p.L) {
      case 32: return launch_rows(k_sweep_rows<32, true, F, K, true, true>, p, 0, s);
      case 64: return launch_rows(k_sweep_rows<64, true, F, K, true, true>, p, 0, s);
      case 96: return launch_rows(k_sweep_rows<96, false, F, K, true, true>, p, dyn96, s);
      case 128:
        return launch_rows(k_sweep_rows<128, false, F, K, true, true>, p, dyn128, s);
      default: break;  // other L: the default kernels
    }
  }
  if (p.variant == 10) {  // variant 0 with one block per loop iteration
    switch (p.L) {
      case 32: return launch_rows(k_sweep_rows<32, true, F, K, true, false, true>, p, 0, s);
      case 64: return launch_rows(k_sweep_rows<64, true, F, K, true, false, true>, p, 0, s);
      case 96: return launch_rows(k_sweep_rows<96, false, F, K, true, false, true>, p, dyn96, s);
      case 128:
        return launch_rows(k_sweep_rows<128, false, F, K, true, false, true>, p, dyn128, s);
      default: break;
    }
  }
  if (p.variant == 0 || p.variant == 10) {  // the row kernel writing the centre word back on every attempt
    switch (p.L) {
      case 32: return launch_rows(k_sweep_rows<32, true, F, K, true>, p, 0, s);
      case 64: return launch_rows(k_sweep_rows<64, true, F, K, true>, p, 0, s);
      case 96: return launch_rows(k_sweep_rows<96, false, F, K, true>, p, dyn96, s);
      case 128: return launch_rows(k_sweep_rows<128, false, F, K, true>, p, dyn128, s);
      default: break;
    }
  }
  switch (p.L) {  // variant 2 (and other L): the software-pipelined row kernel
    case 16: return launch_tiles(k_sweep_exact<16, F, K>, p, s);
    case 32: return launch_rows(k_sweep_rows<32, true, F, K>, p, 0, s);
    case 48: return p.variant == 5 ? launch_tiles(k_sweep_exact<48, F, K, true>, p, s)
                                   : launch_tiles(k_sweep_exact<48, F, K>, p, s);
    case 64: return launch_rows(k_sweep_rows<64, true, F, K>, p, 0, s);
    case 96: return p.variant == 5 ? launch_tiles(k_sweep_exact<96, F, K, true>, p, s)
                                   : launch_rows(k_sweep_rows<96, false, F, K>, p, dyn96, s);
    case 128: return launch_rows(k_sweep_rows<128, false, F, K>, p, dyn128, s);
    default: return launch_tiles(k_sweep_exact<0, F, K>, p, s);
  }
}

template <bool F>
int dispatch_exact(const SweepLaunch &p, cudaStream_t s) {
  return p.rng_kind == kRngMwc ? dispatch_kind<F, kRngMwc>(p, s)
                               : dispatch_kind<F, kRngXorwow>(p, s);
}

}  // namespace

int max_shared_L(int device) {
  int optin = 0;
  if (cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, device) != cudaSuccess)
    return 0;
  const int words = optin / 4 - kHeaderWords;  // one warp per CTA
  int L = 1;
  while (words_per_replica(L + 1) * kTile <= words) ++L;
  return L;
}

int launch_rng_init(uint32_t *rng, int ngrids, int stride, unsigned long long seed, cudaStream_t s) {
  if (ngrids <= 0) return GASP_OK;
  k_rng_init<<<(ngrids + 127) / 128, 128, 0, s>>>(rng, ngrids, stride, seed);
  GASP_CUDA(cudaGetLastError());
  return GASP_OK;
}

int launch_build_thresholds(const float *d_pacc20, uint32_t *d_thr10, int *d_flags, cudaStream_t s) {
  k_build_thresholds<<<1, 32, 0, s>>>(d_pacc20, d_thr10, d_flags);
  GASP_CUDA(cudaGetLastError());
  return GASP_OK;
}

int launch_sweep_exact(const SweepLaunch &p, cudaStream_t s) {
  // Kernels count a batch's attempts in 32-bit integers: split long batches.
  const int N = p.L * p.L;
  const int max_chunk = (1 << 30) / N;
  SweepLaunch q = p;
  int left = p.nsweeps;
  while (left > 0) {
    q.nsweeps = left < max_chunk ? left : max_chunk;
    left -= q.nsweeps;
    q.mag_out = left == 0 ? p.mag_out : nullptr;
    const int rc = p.float_compare ? dispatch_exact<true>(q, s) : dispatch_exact<false>(q, s);
    if (rc) return rc;
  }
  if (p.variant == 9) {  // bulk staging: report a timed-out copy (not while a graph is captured)
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    GASP_CUDA(cudaStreamIsCapturing(s, &cs));
    if (cs == cudaStreamCaptureStatusNone) {
      int flag = 0;
      GASP_CUDA(cudaMemcpyFromSymbolAsync(&flag, g_stage_timeout, sizeof(int), 0,
                                          cudaMemcpyDeviceToHost, s));
      GASP_CUDA(cudaStreamSynchronize(s));
      if (flag) {
        const int zero = 0;
        GASP_CUDA(cudaMemcpyToSymbolAsync(g_stage_timeout, &zero, sizeof(int), 0,
                                          cudaMemcpyHostToDevice, s));
        GASP_CUDA(cudaStreamSynchronize(s));
        return GASP_ERR_TIMEOUT;
      }
    }
  }
  return GASP_OK;
}

int launch_sweep_multi(const SweepLaunch *d_groups, const int *d_tile_begin, int ngroups,
                       int total_tiles, int max_L, int rng_kind, cudaStream_t s) {
  if (total_tiles <= 0) return GASP_OK;
  const size_t smem = (size_t)words_per_replica(max_L) * kTile * sizeof(uint32_t);
  auto kern = rng_kind == kRngMwc ? k_sweep_multi<kRngMwc> : k_sweep_multi<kRngXorwow>;
  GASP_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  kern<<<total_tiles, 32, smem, s>>>(d_groups, d_tile_begin, ngroups);
  GASP_CUDA(cudaGetLastError());
  return GASP_OK;
}

int launch_sweep_trace_cpu(const SweepLaunch &p, cudaStream_t s) {
  switch (p.L) {
    case 16: return launch_tiles(k_sweep_trace_cpu<16>, p, s);
    case 64: return launch_tiles(k_sweep_trace_cpu<64>, p, s);
    default: return launch_tiles(k_sweep_trace_cpu<0>, p, s);
  }
}

int launch_measure(const uint32_t *lat, int L, int ngrids, float *mag, cudaStream_t s) {
  if (ngrids <= 0) return GASP_OK;
  k_measure<<<(ngrids + 127) / 128, 128, 0, s>>>(lat, L, ngrids, mag);
  GASP_CUDA(cudaGetLastError());
  return GASP_OK;
}

int launch_pack_grids(const int *g, uint32_t *lat, int L, int ngrids, cudaStream_t s,
                      int per_input) {
  const long long total = (long long)tiles_for(ngrids) * words_per_replica(L) * kTile;
  if (total == 0) return GASP_OK;
  k_pack_grids<<<(unsigned)((total + 255) / 256), 256, 0, s>>>(g, lat, L, ngrids, total,
                                                               per_input);
  GASP_CUDA(cudaGetLastError());
  return GASP_OK;
}

int launch_unpack_grids(const uint32_t *lat, int *g, int L, int ngrids, cudaStream_t s) {
  const long long total = (long long)ngrids * words_per_replica(L);
  if (total == 0) return GASP_OK;
  k_unpack_grids<<<(unsigned)((total + 255) / 256), 256, 0, s>>>(lat, g, L, ngrids, total);
  GASP_CUDA(cudaGetLastError());
  return GASP_OK;
}

int launch_pack_frame(const uint32_t *lat, uint8_t *frame, int L, int ngrids, cudaStream_t s) {
  const long long N = (long long)L * L;
  const long long nbits = N * ngrids;
  if (nbits == 0) return GASP_OK;
  if (N % 32 == 0) {
    const int W = (int)(N / 32), nchunks = (W + 31) / 32;
    const long long blocks = (long long)tiles_for(ngrids) * nchunks;
    if (blocks > 0x7fffffffLL) {
      set_error("gridstates frame of %d replicas of L=%d is too large to pack", ngrids, L);
      return GASP_ERR_UNSUPPORTED;
    }
    k_pack_frame32t<<<(unsigned)blocks, 256, 0, s>>>(lat, reinterpret_cast<uint32_t *>(frame), W,
                                                      ngrids, nchunks);
  } else {
    const long long nbytes = (nbits + 7) / 8;
    k_pack_frame8<<<(unsigned)((nbytes + 255) / 256), 256, 0, s>>>(lat, frame, L, nbits, nbytes);
  }
  GASP_CUDA(cudaGetLastError());
  return GASP_OK;
}

}  // namespace gasp
