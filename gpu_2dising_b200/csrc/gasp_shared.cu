// gasp_shared.cu -- the multispin shared-site sweep (sweep variant 7,
// production MWC64X stream; no reference counterpart).
//
// A warp sweeps a tile of 32 replicas that share every attempt's site:
//   * the tile is held transposed in shared memory, one 32-bit word per site
//     whose bit l is replica l's spin (the layout of the reference's
//     mc_sweep_gpu_bitmap32, src/mc_gpu.cu:279-356), so an attempt's five
//     words are broadcast loads (one wavefront each);
//   * the up-neighbour counts of all 32 replicas come from bitwise full
//     adders on the four neighbour words (three bit planes of the count);
//   * each lane draws its replica's acceptance from its own stream and
//     compares it with the integer threshold of its class;
//   * __ballot_sync gives the flip mask and the centre word is stored once
//     (every lane writes the same value, so each lane's next load of that word
//     sees it without a warp barrier).
// Sites come in batches: at the start of a batch every live lane draws one
// site from its own stream, and attempt j of the batch uses lane j's site
// (__shfl_sync), so a site costs 1/32 of a draw per lane.  Replicas of a tile
// therefore follow the same site sequence (correlated, each one an exact
// random-site Metropolis chain); error bars over replicas need blocks of 32.
// The tile is transposed with ballots on the way in and bit gathers on the
// way out; the home lattice keeps the lane-interleaved layout of the other
// sweep kernels.
#include "gasp_internal.h"

namespace gasp {
namespace {

constexpr unsigned kFull = 0xffffffffu;
constexpr int kSharedHeaderWords = 64;

template <int L_>
__global__ void __launch_bounds__(32) k_sweep_shared(SweepLaunch p) {
  const int L = L_ > 0 ? L_ : p.L;
  const int N = L * L;
  const int W = (N + 31) >> 5;
  extern __shared__ __align__(16) uint32_t smem[];
  const int lane = threadIdx.x;
  uint32_t *thr_s = smem;
  if (lane < 10) thr_s[lane] = p.thr[lane];
  const int n_act = p.n_active_dev ? *p.n_active_dev : p.n_active;
  const int tile = blockIdx.x;
  const int first = tile * kTile;
  if (first >= n_act) return;  // whole warp
  const int nlive = n_act - first < kTile ? n_act - first : kTile;
  const bool live = lane < nlive;
  const int rep = first + lane;
  uint32_t *T = smem + kSharedHeaderWords;  // T[site], bit l = replica l
  uint32_t *home = p.lat + (size_t)tile * W * kTile + lane;

  // transpose in: word w of lane l holds sites 32w..32w+31 of replica l
  for (int w = 0; w < W; ++w) {
    const uint32_t v = live ? home[(size_t)w * kTile] : 0u;
    uint32_t mine = 0u;
#pragma unroll 8
    for (int b = 0; b < 32; ++b) {
      const uint32_t t = __ballot_sync(kFull, (v >> b) & 1u);
      if (lane == b) mine = t;
    }
    T[w * 32 + lane] = mine;
  }
  __syncwarp();

  uint32_t x = live ? p.rng[rep] : 0u, c = live ? p.rng[p.rng_stride + rep] : 0u;
  auto next = [&]() -> uint32_t {
    const uint32_t r = x ^ c;
    const uint64_t t = (uint64_t)x * kMwcA + c;
    x = (uint32_t)t;
    c = (uint32_t)(t >> 32);
    return r;
  };
  auto site_of = [&](uint32_t r) -> uint32_t {
    if constexpr (L_ > 0 && ((L_ * L_) & (L_ * L_ - 1)) == 0)
      return r >> (32 - __builtin_ctz((unsigned)(L_ * L_)));
    else
      return __umulhi(r, (uint32_t)N);
  };

  const int Q = p.nsweeps * N;  // < 2^30 (launch_sweep_exact splits longer batches)
  uint32_t sb = 0u;
  int j = 0;
  for (int a = 0; a < Q; ++a) {
    if (j == 0 && live) sb = site_of(next());
    const uint32_t s = __shfl_sync(kFull, sb, j);
    j = j + 1 == nlive ? 0 : j + 1;
    const uint32_t row = s / (uint32_t)L, col = s - row * (uint32_t)L;
    const uint32_t su = row == 0 ? s + N - L : s - L;
    const uint32_t sd = row == (uint32_t)L - 1 ? s - N + L : s + L;
    const uint32_t sl = col == 0 ? s + L - 1 : s - 1;
    const uint32_t sr = col == (uint32_t)L - 1 ? s - L + 1 : s + 1;
    const uint32_t wc = T[s], wu = T[su], wd = T[sd], wl = T[sl], wr = T[sr];
    // bit planes of (# up neighbours) for all 32 replicas: u+d = x1 + 2 a1,
    // l+r = x2 + 2 a2; total = b0 + 2 (k0 + a1 + a2) with k0 + a1 + a2 <= 2
    const uint32_t x1 = wu ^ wd, a1 = wu & wd, x2 = wl ^ wr, a2 = wl & wr;
    const uint32_t b0 = x1 ^ x2, k0 = x1 & x2;
    const uint32_t b1 = k0 ^ a1 ^ a2, b2 = a1 & a2;
    const uint32_t nb = ((b0 >> lane) & 1u) | (((b1 >> lane) & 1u) << 1) | (((b2 >> lane) & 1u) << 2);
    const uint32_t cls = 5u * ((wc >> lane) & 1u) + nb;
    bool acc = false;
    if (live) acc = next() <= thr_s[cls];
    const uint32_t m = __ballot_sync(kFull, acc);
    T[s] = wc ^ m;  // the same value from every lane
  }
  __syncwarp();

  // transpose out and magnetisation
  int pc = 0;
  for (int w = 0; w < W; ++w) {
    uint32_t v = 0u;
#pragma unroll 8
    for (int b = 0; b < 32; ++b) v |= ((T[w * 32 + b] >> lane) & 1u) << b;
    if (live) home[(size_t)w * kTile] = v;
    pc += __popc(v);
  }
  if (live) {
    p.rng[rep] = x;
    p.rng[p.rng_stride + rep] = c;
    if (p.mag_out != nullptr) p.mag_out[rep] = (float)(2 * pc - N) / (float)N;
  }
}

template <int L_>
int launch_shared_kernel(const SweepLaunch &p, cudaStream_t s) {
  const int W = words_per_replica(p.L);
  const size_t smem = (size_t)(kSharedHeaderWords + W * kTile) * sizeof(uint32_t);
  auto kern = k_sweep_shared<L_>;
  GASP_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  kern<<<tiles_for(p.n_active), 32, smem, s>>>(p);
  GASP_CUDA(cudaGetLastError());
  return GASP_OK;
}

}  // namespace

int launch_sweep_shared(const SweepLaunch &p, cudaStream_t s) {
  if (p.rng_kind != kRngMwc || p.lattice_in_global || p.active != nullptr || p.L < 3 ||
      p.float_compare) {
    set_error("the shared-site sweep needs the MWC64X stream, 3 <= L within shared memory, "
              "integer thresholds and no active-replica list");
    return GASP_ERR_UNSUPPORTED;
  }
  if (p.n_active <= 0 || p.nsweeps <= 0) return GASP_OK;
  switch (p.L) {
    case 32: return launch_shared_kernel<32>(p, s);
    case 64: return launch_shared_kernel<64>(p, s);
    case 128: return launch_shared_kernel<128>(p, s);
    default: return launch_shared_kernel<0>(p, s);
  }
}

}  // namespace gasp
