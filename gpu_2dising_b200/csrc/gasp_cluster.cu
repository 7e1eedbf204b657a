// gasp_cluster.cu -- largest-cluster collective variable on the bit-packed
// lattice.
//
// Reference: compute_largest_cluster_gpu (src/mc_gpu.cu:457-526) and
// compute_largest_cluster_cpu (src/mc_cpu.c:310-364): per replica, the size
// of the largest 4-connected (periodic) cluster of sites whose spin equals
// `spin`, returned as a float.  The reference runs one breadth-first search
// per thread over an int32 grid in HBM with a 2*L*L int work area per
// replica.  Here one CTA labels one replica with the lock-free union-find of
// O. Kalentev et al. / D. P. Playne and K. Hawick ("A New Algorithm for
// Parallel Connected-Component Labelling on GPUs", IEEE TPDS 29(6), 2018):
//   1. every matching site is its own root;
//   2. each matching site unions itself with its matching right and down
//      neighbours (periodic), roots always pointing at smaller indices, links
//      made with atomicMin and retried when another thread got there first;
//   3. each matching site adds one to the counter of its root;
//   4. block max over the counters.
// The labels and counters live in shared memory while 2*L*L*4 bytes fit
// (L <= 170 at 227 KiB per CTA); beyond that they live in a global work area
// and replicas are processed in chunks that fit it.
#include <stdint.h>

#include "gasp_internal.h"

namespace gasp {
namespace {

constexpr int kClusterThreads = 512;
constexpr size_t kClusterWorkBudget = (size_t)256 << 20;  // global work area cap (bytes)

__device__ __forceinline__ int uf_find(const int *P, int a) {
  const volatile int *vp = P;
  int p = vp[a];
  while (p != a) {
    a = p;
    p = vp[a];
  }
  return a;
}

__device__ __forceinline__ void uf_union(int *P, int a, int b) {
  for (;;) {
    a = uf_find(P, a);
    b = uf_find(P, b);
    if (a == b) return;
    if (b < a) {
      const int old = atomicMin(&P[a], b);
      if (old == a) return;
      a = old;
    } else {
      const int old = atomicMin(&P[b], a);
      if (old == b) return;
      b = old;
    }
  }
}

// One CTA per replica rep0 + blockIdx.x.  Lattice words of replica r are
// lat[((r/32)*W + w)*32 + r%32] (lane-interleaved tiles).
template <bool kShared>
__global__ void __launch_bounds__(kClusterThreads)
k_largest_cluster(const uint32_t *__restrict__ lat, int L, int ngrids, int rep0, int want_up,
                  int *__restrict__ work, float *__restrict__ out) {
  extern __shared__ int sm[];
  const int rep = rep0 + blockIdx.x;
  if (rep >= ngrids) return;  // uniform over the block
  const int N = L * L, W = (N + 31) >> 5;
  const uint32_t flip = want_up ? 0u : 0xffffffffu;
  const uint32_t *src = lat + (size_t)(rep >> 5) * W * kTile + (rep & 31);
  int *P, *cnt;
  const uint32_t *bits;
  int bstride;
  if (kShared) {
    P = sm;
    cnt = sm + N;
    uint32_t *b = reinterpret_cast<uint32_t *>(sm + 2 * N);
    for (int w = threadIdx.x; w < W; w += blockDim.x) b[w] = src[(size_t)w * kTile] ^ flip;
    bits = b;
    bstride = 1;
  } else {
    P = work + (size_t)blockIdx.x * 2 * N;
    cnt = P + N;
    bits = src;
    bstride = kTile;
  }
  const uint32_t xflip = kShared ? 0u : flip;
  auto on = [&](int s) -> bool {
    return ((bits[(size_t)(s >> 5) * bstride] ^ xflip) >> (s & 31)) & 1u;
  };
  if (kShared) __syncthreads();
  for (int s = threadIdx.x; s < N; s += blockDim.x) {
    P[s] = s;
    cnt[s] = 0;
  }
  __syncthreads();
  for (int s = threadIdx.x; s < N; s += blockDim.x) {
    if (!on(s)) continue;
    const int y = s / L, x = s - y * L;
    const int right = y * L + (x + 1 == L ? 0 : x + 1);
    const int down = (y + 1 == L ? 0 : y + 1) * L + x;
    if (on(right)) uf_union(P, s, right);
    if (on(down)) uf_union(P, s, down);
  }
  __syncthreads();
  // No unions are running any more: compressing a path with plain stores is
  // safe now (every value written is the root, a valid ancestor).
  for (int s = threadIdx.x; s < N; s += blockDim.x) {
    if (!on(s)) continue;
    const int r = uf_find(P, s);
    atomicAdd(&cnt[r], 1);
    P[s] = r;
  }
  __syncthreads();
  int best = 0;
  for (int s = threadIdx.x; s < N; s += blockDim.x) best = max(best, cnt[s]);
  for (int o = 16; o > 0; o >>= 1) best = max(best, __shfl_xor_sync(0xffffffffu, best, o));
  __shared__ int warp_best[kClusterThreads / 32];
  if ((threadIdx.x & 31) == 0) warp_best[threadIdx.x >> 5] = best;
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int i = 1; i < (int)(blockDim.x >> 5); ++i) best = max(best, warp_best[i]);
    out[rep] = (float)best;
  }
}

size_t cluster_smem_bytes(int L) {
  const size_t N = (size_t)L * L;
  return 2 * N * sizeof(int) + (size_t)words_per_replica(L) * sizeof(uint32_t);
}

}  // namespace

size_t largest_cluster_work_bytes(int L, int ngrids, int device) {
  int optin = 0;
  if (cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, device) !=
      cudaSuccess) {
    cudaGetLastError();
    optin = 48 * 1024;
  }
  if (cluster_smem_bytes(L) + 1024 <= (size_t)optin) return 0;  // + static shared memory
  const size_t per = 2 * (size_t)L * L * sizeof(int);
  size_t chunk = kClusterWorkBudget / per;
  if (chunk < 1) chunk = 1;
  if (chunk > (size_t)ngrids) chunk = (size_t)ngrids;
  return chunk * per;
}

int launch_largest_cluster(const uint32_t *lat, int L, int ngrids, int spin, int *work,
                           size_t work_bytes, float *out, cudaStream_t s) {
  if (ngrids <= 0) return GASP_OK;
  const int want_up = spin > 0 ? 1 : 0;
  if (work_bytes == 0) {
    const size_t smem = cluster_smem_bytes(L);
    GASP_CUDA(cudaFuncSetAttribute(k_largest_cluster<true>,
                                   cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    k_largest_cluster<true><<<ngrids, kClusterThreads, smem, s>>>(lat, L, ngrids, 0, want_up,
                                                                  nullptr, out);
    GASP_CUDA(cudaGetLastError());
    return GASP_OK;
  }
  if (!work) {
    set_error("largest cluster: L=%d needs a work area", L);
    return GASP_ERR_INVALID;
  }
  const size_t per = 2 * (size_t)L * L * sizeof(int);
  const int chunk = (int)(work_bytes / per);
  if (chunk < 1) {
    set_error("largest cluster: work area of %zu bytes is below one replica's %zu", work_bytes,
              per);
    return GASP_ERR_INVALID;
  }
  for (int r0 = 0; r0 < ngrids; r0 += chunk) {
    const int n = ngrids - r0 < chunk ? ngrids - r0 : chunk;
    k_largest_cluster<false><<<n, kClusterThreads, 0, s>>>(lat, L, ngrids, r0, want_up, work, out);
    GASP_CUDA(cudaGetLastError());
  }
  return GASP_OK;
}

}  // namespace gasp
