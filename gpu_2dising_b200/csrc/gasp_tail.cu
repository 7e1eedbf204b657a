// gasp_tail.cu -- one warp per replica: the latency-bound end of a committor
// run, on the production (MWC64X) stream and on the reference (XORWOW) one.
//
// Near the end of a shooting run only a few trajectories are undecided.  The
// row kernels give each replica one lane, and a lane's attempts form one
// dependency chain (draw -> shared loads -> threshold -> store), about 100
// cycles per attempt, so a lone replica needs ~0.2 ms per L=64 sweep however
// idle the GPU is.  Here the 32 lanes of a warp work on ONE replica:
//
//   * the warp keeps a window of 32 pending attempts (site, acceptance draw)
//     in first-in-first-out order, one per lane; the window position of lane
//     l is (l - head) mod 32;
//   * each round every pending site is marked in a per-warp occupancy bitmap
//     (atomicOr; a lane that finds its bit already set also marks the site in
//     a duplicates bitmap); a lane is flagged when its site is a duplicate or
//     one of its four neighbours is occupied -- a symmetric relation;
//   * with f the first flagged window position, positions 0..f are applied at
//     once (all 32 when none is flagged): positions before f have no partner at
//     all and f's partners all come later, so no applied attempt touches the
//     site or the neighbours of another, and applying them together gives
//     exactly the lattice that applying them one after the other in window
//     order gives;
//   * the lanes whose attempts were applied draw the next attempts into the
//     back of the window, so every drawn attempt is applied, in the order
//     drawn: the dynamics is random-site Metropolis with i.i.d. uniform sites
//     and acceptance draws, the same Markov chain as the row kernels.
//
// At L=64 about 22 attempts are applied per round.  On the XORWOW stream the
// whole warp steps the replica's one state and hands the refilled lanes their
// draws in order, so the attempts are the row kernel's, bit for bit.  On
// MWC64X lane j draws from the replica's stream skipped ahead by j * 2^35
// (a one-off 64-bit modular multiply per lane and launch); after the launch
// the replica's state is set past the longest lane segment used, so later
// launches never reuse a draw.
// Per warp, shared memory holds the lattice (W words) and two sets of marks
// (occupancy + duplicates, W words each) used in alternate rounds, so a
// round's marks are cleared during the next round without a third warp
// barrier.  Each lane draws its next attempt one assignment ahead.  The
// replica is read from and written back to its lane-interleaved home words
// like the other sweep kernels.
#include <cfloat>

#include <curand_kernel.h>

#include "gasp_internal.h"

namespace gasp {
namespace {

constexpr unsigned kFull = 0xffffffffu;
constexpr int kTailHeaderWords = 64;  // thresholds (10) and float table (20)
constexpr uint64_t kMwcM = ((uint64_t)kMwcA << 32) - 1;
constexpr int kTailWordsPerW = 5;     // shared words per warp, in units of W

// (a + b) mod M for a, b < M < 2^64.
__device__ __forceinline__ uint64_t addmod_m(uint64_t a, uint64_t b) {
  uint64_t t = a + b;
  if (t < a || t >= kMwcM) t -= kMwcM;
  return t;
}

// (a * b) mod M by binary double-and-add (once per lane and launch).
__device__ uint64_t mulmod_m(uint64_t a, uint64_t b) {
  uint64_t r = 0;
  for (int i = 63; i >= 0; --i) {
    r = addmod_m(r, r);
    if ((b >> i) & 1ull) r = addmod_m(r, a);
  }
  return r;
}

__device__ __forceinline__ uint32_t bit_of(const uint32_t *words, uint32_t s) {
  return (words[s >> 5] >> (s & 31u)) & 1u;
}

template <int L_, bool kFloatCmp, int kRng>
__global__ void __launch_bounds__(128) k_sweep_tail(SweepLaunch p, TailParams tp) {
  const int L = L_ > 0 ? L_ : p.L;
  const int N = L * L;
  const int W = (N + 31) >> 5;
  extern __shared__ __align__(16) uint32_t smem[];
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  const int nwarps = blockDim.x >> 5;
  uint32_t *thr_s = smem;
  float *pacc_s = reinterpret_cast<float *>(smem + 16);
  if (threadIdx.x < 10) thr_s[threadIdx.x] = p.thr[threadIdx.x];
  if (threadIdx.x < 20) pacc_s[threadIdx.x] = p.pacc_f[threadIdx.x];
  __syncthreads();

  int n_act = p.n_active_dev ? *p.n_active_dev : p.n_active;
  if (p.tail_split > 0 && n_act > p.tail_split) n_act = 0;  // the row kernels' turn
  const int slot = blockIdx.x * nwarps + warp;
  if (slot >= n_act) return;  // whole warp
  const int rep = p.active ? p.active[slot] : slot;
  // per warp: lattice [W], then two mark buffers, each occupancy [W] + duplicates [W]
  uint32_t *lat_s = smem + kTailHeaderWords + (size_t)warp * kTailWordsPerW * W;
  uint32_t *marks = lat_s + W;
  uint32_t *home = p.lat + (size_t)(rep >> 5) * W * kTile + (rep & 31);
  for (int w = lane; w < W; w += 32) {
    lat_s[w] = home[(size_t)w * kTile];
    marks[w] = marks[W + w] = marks[2 * W + w] = marks[3 * W + w] = 0u;
  }

  // MWC64X: lane j's stream is the replica's state advanced by j * 2^35 draws.
  // XORWOW: every lane holds the replica's one state and steps it in
  // lockstep, so the attempts are drawn in the replica's own order (site,
  // acceptance, site, ...) exactly as the row kernels draw them.
  uint32_t x = 0u, c = 0u;
  curandStateXORWOW st;
  if constexpr (kRng == kRngMwc) {
    const uint64_t X = (uint64_t)p.rng[rep] * kMwcA + p.rng[p.rng_stride + rep];
    const uint64_t Xj = mulmod_m(X, tp.mul[lane]);
    x = (uint32_t)(Xj / kMwcA);
    c = (uint32_t)(Xj % kMwcA);
  } else {
    st.d = p.rng[rep];
#pragma unroll
    for (int k = 0; k < 5; ++k) st.v[k] = p.rng[(k + 1) * p.rng_stride + rep];
    st.boxmuller_flag = 0;
    st.boxmuller_flag_double = 0;
    st.boxmuller_extra = 0.f;
    st.boxmuller_extra_double = 0.0;
  }
  uint32_t ndraw = 0;
  auto next = [&]() -> uint32_t {
    const uint32_t r = x ^ c;
    const uint64_t t = (uint64_t)x * kMwcA + c;
    x = (uint32_t)t;
    c = (uint32_t)(t >> 32);
    ++ndraw;
    return r;
  };
  // site of a draw: MWC64X, its top bits scaled to [0, N); XORWOW, the
  // reference's float arithmetic (src/mc_gpu.cu:311,317), as the row kernels
  const float shrink = (1.0f - FLT_EPSILON) * (float)N;
  auto site_of = [&](uint32_t r) -> uint32_t {
    if constexpr (kRng == kRngXorwow)
      return (uint32_t)__float2int_rd(shrink * _curand_uniform(r));
    else if constexpr (L_ > 0 && ((L_ * L_) & (L_ * L_ - 1)) == 0)
      return r >> (32 - __builtin_ctz((unsigned)(L_ * L_)));
    else
      return __umulhi(r, (uint32_t)N);
  };
  // XORWOW refill: the warp draws the next `nnew` attempts in order (warp-
  // uniform loop); the lane whose attempt is the q-th of them keeps its pair.
  auto draw_in_order = [&](int nnew, int q, uint32_t &s_out, uint32_t &u_out) {
    uint32_t a = 0u, b = 0u;
    for (int j = 0; j < nnew; ++j) {
      const uint32_t r0 = curand(&st);
      const uint32_t r1 = curand(&st);
      if (j == q) {
        a = r0;
        b = r1;
      }
    }
    if (q >= 0 && q < nnew) {
      s_out = site_of(a);
      u_out = b;
    }
  };
  // MWC64X: every lane holds its next attempt ready (drawn one assignment
  // ahead), so a refill is a register move and the draws stay off the
  // round's chain.
  uint32_t ns = 0u, nu = 0u;
  if constexpr (kRng == kRngMwc) {
    ns = site_of(next());
    nu = next();
  }
  __syncwarp();

  const int Q = p.nsweeps * N;  // attempts of this launch (< 2^30)
  int drawn = Q < 32 ? Q : 32;
  bool valid = lane < drawn;
  uint32_t s = 0u, u = 0u;
  if constexpr (kRng == kRngMwc) {
    if (valid) {
      s = ns;
      u = nu;
      ns = site_of(next());
      nu = next();
    }
  } else {
    draw_in_order(drawn, lane, s, u);
  }
  int head = 0, pend = drawn, done = 0, rnd = 0;
  bool pvalid = false;  // this lane's mark of the previous round, to clear
  uint32_t ps = 0u;
  while (done < Q) {
    uint32_t *occ = marks + (rnd & 1) * 2 * W;
    uint32_t *dup = occ + W;
    // the previous round's marks (other buffer) were read before its closing
    // __syncwarp and are next written after this round's: clear them now
    if (pvalid) {
      uint32_t *pocc = marks + ((rnd + 1) & 1) * 2 * W;
      pocc[ps >> 5] = 0u;
      pocc[W + (ps >> 5)] = 0u;
    }
    const uint32_t bit = 1u << (s & 31u);
    if (valid) {
      const uint32_t old = atomicOr(&occ[s >> 5], bit);
      if (old & bit) atomicOr(&dup[s >> 5], bit);  // a second attempt on this site
    }
    __syncwarp();
    uint32_t su, sd, sl, sr;
    {
      const uint32_t row = s / (uint32_t)L, col = s - row * (uint32_t)L;
      su = row == 0 ? s + N - L : s - L;
      sd = row == (uint32_t)L - 1 ? s - N + L : s + L;
      sl = col == 0 ? s + L - 1 : s - 1;
      sr = col == (uint32_t)L - 1 ? s - L + 1 : s + 1;
    }
    // marks and lattice are read together; the acceptance is decided for every
    // pending attempt and used only by those applied this round
    const uint32_t m = bit_of(occ, su) | bit_of(occ, sd) | bit_of(occ, sl) | bit_of(occ, sr) |
                       ((dup[s >> 5] & bit) != 0u);
    const uint32_t wc = lat_s[s >> 5];
    const uint32_t nb = bit_of(lat_s, su) + bit_of(lat_s, sd) + bit_of(lat_s, sl) +
                        bit_of(lat_s, sr);
    const uint32_t cls = 5u * ((wc & bit) != 0u) + nb;
    bool acc;
    if constexpr (kFloatCmp) {
      acc = _curand_uniform(u) < pacc_s[2 * cls];
    } else {
      acc = u <= thr_s[cls];
    }
    const unsigned fm = __ballot_sync(kFull, valid && m != 0u);
    const unsigned fr = __funnelshift_r(fm, fm, (unsigned)head);  // bit i: window position i
    int k = fr ? __ffs(fr) : 32;
    if (k > pend) k = pend;
    if (k <= 0) break;  // cannot happen (pend >= 1 while done < Q); keeps the loop bounded
    const int pos = (lane - head) & 31;
    if (pos < k && acc) atomicXor(&lat_s[s >> 5], bit);
    __syncwarp();
    pvalid = valid;
    ps = s;
    ++rnd;
    done += k;
    head = (head + k) & 31;
    pend -= k;
    const int room = 32 - pend, left = Q - drawn;
    const int nnew = room < left ? room : left;
    const int pos2 = (lane - head) & 31;
    if (pos2 >= pend) valid = pos2 - pend < nnew;
    if constexpr (kRng == kRngMwc) {
      if (pos2 >= pend && valid) {
        s = ns;
        u = nu;
        ns = site_of(next());
        nu = next();
      }
    } else {
      draw_in_order(nnew, pos2 - pend, s, u);  // lanes still pending keep theirs (q < 0)
    }
    pend += nnew;
    drawn += nnew;
  }

  if constexpr (kRng == kRngMwc) {
    // the replica's stream continues past the longest lane segment used
    const uint32_t most = __reduce_max_sync(kFull, ndraw);
    const int jstar = __ffs(__ballot_sync(kFull, ndraw == most)) - 1;
    if (lane == jstar) {
      const uint64_t Xe = (uint64_t)x * kMwcA + c;
      const uint64_t Xb = mulmod_m(Xe, tp.inv[lane]);
      p.rng[rep] = (uint32_t)(Xb / kMwcA);
      p.rng[p.rng_stride + rep] = (uint32_t)(Xb % kMwcA);
    }
  } else if (lane == 0) {  // 2 draws per attempt consumed, as by the row kernels
    p.rng[rep] = st.d;
#pragma unroll
    for (int k = 0; k < 5; ++k) p.rng[(k + 1) * p.rng_stride + rep] = st.v[k];
  }
  __syncwarp();
  int pc = 0;
  for (int w = lane; w < W; w += 32) {
    const uint32_t v = lat_s[w];
    pc += __popc(v);
    home[(size_t)w * kTile] = v;
  }
  pc = (int)__reduce_add_sync(kFull, (unsigned)pc);
  if (lane == 0 && p.mag_out != nullptr) p.mag_out[rep] = (float)(2 * pc - N) / (float)N;
}

template <int L_, bool F, int K>
int launch_tail_kernel(const SweepLaunch &p, cudaStream_t s) {
  const int W = words_per_replica(p.L);
  const int nwarps = kTailWordsPerW * W <= 4096 ? 4 : 1;
  const size_t smem = (size_t)(kTailHeaderWords + nwarps * kTailWordsPerW * W) * sizeof(uint32_t);
  auto kern = k_sweep_tail<L_, F, K>;
  if (smem > 48 * 1024)
    GASP_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  const int blocks = (p.n_active + nwarps - 1) / nwarps;
  kern<<<blocks, nwarps * 32, smem, s>>>(p, mwc_lane_params());
  GASP_CUDA(cudaGetLastError());
  return GASP_OK;
}

}  // namespace

template <int K>
int launch_tail_kind(const SweepLaunch &p, cudaStream_t s) {
  if (p.L == 64)
    return p.float_compare ? launch_tail_kernel<64, true, K>(p, s)
                           : launch_tail_kernel<64, false, K>(p, s);
  return p.float_compare ? launch_tail_kernel<0, true, K>(p, s)
                         : launch_tail_kernel<0, false, K>(p, s);
}

int launch_sweep_tail(const SweepLaunch &p, cudaStream_t s) {
  if (p.lattice_in_global || p.L < 3 || p.L > kTailMaxL) {
    set_error("the one-warp-per-replica sweep needs 3 <= L <= %d (shared-memory lattices)",
              kTailMaxL);
    return GASP_ERR_UNSUPPORTED;
  }
  if (p.n_active <= 0 || p.nsweeps <= 0) return GASP_OK;
  return p.rng_kind == kRngMwc ? launch_tail_kind<kRngMwc>(p, s)
                               : launch_tail_kind<kRngXorwow>(p, s);
}

}  // namespace gasp
