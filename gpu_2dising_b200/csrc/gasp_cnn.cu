// gasp_cnn.cu -- the committor surrogate network on sm_100a (no reference
// counterpart).  4 circular 3x3 convolutions (1->32, 32->32 x3) + ReLU,
// global average pool, 32->1 linear, sigmoid; binomial cross-entropy; Adam.
//
// Convolutions (forward, and the data gradient of the backward pass) are
// implicit GEMMs on the 5th-generation tensor cores: per CTA a 128-pixel tile,
// D[128 x 32] (FP32, in TMEM) = A[128 x K] (BF16) * B[32 x K]^T (weights,
// BF16), K = 9 taps * 32 channels = 288 (16 for the first layer).  A is an
// im2col buffer (k_conv_tc) or, for the 32-channel layers, shifted windows
// over the tile's staged input rows (k_conv_win, k_conv_gh64).  The first
// layer (one input channel of +-1 spins) has only 512 distinct input
// neighbourhoods: k_conv_tc computes their activations once per call and
// k_conv1_lookup writes each pixel's row of that table.  Operands are K-major in
// shared memory in the no-swizzle interleaved layout (8-row x 16-byte core
// matrices); one thread issues K/16 tcgen05.mma (kind::f16, M=128, N=32), a
// tcgen05.commit arrives on an mbarrier, and every warp reads its 32 rows of D
// with tcgen05.ld.  Weight gradients are tcgen05 GEMMs too, reducing over the
// batch's pixels with both operands MN-major (k_conv_dw_win, k_conv_dw1_tc).
//
// Activations: BF16, [image][pixel][32 channels] (pixel = row*L + col).
#include <cuda_bf16.h>

#include <cmath>
#include <cstdlib>
#include <cstdio>
#include <cstring>
#include <vector>

#include "gasp_internal.h"

namespace gasp {
namespace {

constexpr int kC = 32;
constexpr int kTileM = 128;
constexpr int kWaitLimit = 1 << 26;  // bounded mbarrier wait (iterations)

// Flat FP32 parameter offsets (same order as the CPU oracle).
constexpr int kOffW1 = 0, kOffB1 = 288, kOffW2 = 320, kOffB2 = 320 + 9216;
constexpr int kOffW3 = kOffB2 + 32, kOffB3 = kOffW3 + 9216;
constexpr int kOffW4 = kOffB3 + 32, kOffB4 = kOffW4 + 9216;
constexpr int kOffWf = kOffB4 + 32, kOffBf = kOffWf + 32;
constexpr int kNParam = kOffBf + 1;  // 28097
static_assert(kNParam == 28097, "parameter count");

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

// UMMA shared-memory descriptor: no swizzle, K-major interleaved layout.
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr >> 4) & 0x3FFFu);
  d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
  d |= (uint64_t)1u << 46;  // descriptor version for sm_100
  return d;                 // base offset 0, layout type 0 (no swizzle)
}

// Instruction descriptor: D F32, A/B BF16, both K-major, N=32, M=128.
constexpr uint32_t kIdesc = (1u << 4) | (1u << 7) | (1u << 10) | ((32u >> 3) << 17) |
                            ((128u >> 4) << 24);

__device__ __forceinline__ void umma_bf16(uint32_t tmem_d, uint64_t da, uint64_t db,
                                          uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem_d),
      "l"(da), "l"(db), "r"(kIdesc), "r"(accumulate));
}

__device__ __forceinline__ void umma_commit(uint32_t mbar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                   mbar)
               : "memory");
}

__device__ __forceinline__ void mbar_init(uint32_t mbar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(mbar), "r"(count) : "memory");
}

// Bounded wait for phase `parity` of an mbarrier; false on timeout.
__device__ __forceinline__ bool mbar_wait(uint32_t mbar, uint32_t parity) {
  for (int it = 0; it < kWaitLimit; ++it) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred P1;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, P1;\n\t}\n"
        : "=r"(done)
        : "r"(mbar), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

// 16-byte global -> shared copy that does not pass through registers, so a
// thread keeps all of its im2col gathers in flight at once.
__device__ __forceinline__ void cp_async16(uint32_t dst, const void *src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(dst), "l"(src) : "memory");
}

__device__ __forceinline__ void cp_async_wait_all() {
  asm volatile("cp.async.commit_group;\n\tcp.async.wait_group 0;" ::: "memory");
}

__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float (&v)[32]) {
  uint32_t r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,"
      "%14,%15,%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]),
        "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]),
        "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]),
        "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]),
        "=r"(r[31])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}

// Byte offset of element (row, k) in the interleaved K-major layout.
__device__ __forceinline__ uint32_t il_off(int row, int k, int sbo) {
  return (uint32_t)((row >> 3) * sbo + (k >> 3) * 128 + (row & 7) * 16 + (k & 7) * 2);
}

__device__ __forceinline__ int nbr(int p, int tap, int L) {
  const int y = p / L, x = p - y * L;
  const int dy = tap / 3 - 1, dx = tap % 3 - 1;
  const int yy = (y + dy + L) % L, xx = (x + dx + L) % L;
  return yy * L + xx;
}

// kTab1: layer 1 on the 512 patterns of a 3x3 spin neighbourhood (row q of
// A holds +1 for tap k where bit k of q is set, -1 elsewhere); its outputs are
// the first layer's activation table (k_conv1_lookup).
enum { kFwd = 1, kBwd = 2, kTab1 = 3 };
constexpr int kNPatterns = 512;

struct ConvArgs {
  int L;
  const int8_t *spins;           // layer 1 (k_conv1_lookup): [B][N]
  const __nv_bfloat16 *x;        // kFwd: activations in; kBwd: dZ of this layer
  const __nv_bfloat16 *w;        // [32][K] (kBwd: transposed weights)
  const float *bias;             // kTab1/kFwd
  __nv_bfloat16 *y;              // kFwd: activations out; kBwd: dZ of the previous layer
  const __nv_bfloat16 *mask_src; // kBwd: activations of the previous layer (ReLU mask)
  float *pool;                   // layer 4 forward: per-image channel sums [B][32]
  int *err;                      // set on a timed-out wait
  int ntiles;                    // images * (L*L / 128)
};

// Persistent: each CTA allocates its TMEM columns and stages the weights once,
// then loops over 128-pixel tiles (tile = image * tiles_per_image + index).
template <int MODE>
__global__ void __launch_bounds__(128) k_conv_tc(ConvArgs a) {
  constexpr int K = MODE == kTab1 ? 16 : 9 * kC;
  constexpr int SBO = K * 16;  // bytes between 8-row groups
  extern __shared__ __align__(1024) unsigned char smem[];
  unsigned char *sA = smem;                               // 128 x K bf16
  unsigned char *sB = smem + kTileM * K * 2;              // 32 x K bf16
  uint64_t *mbar = reinterpret_cast<uint64_t *>(sB + kC * K * 2);
  uint32_t *tslot = reinterpret_cast<uint32_t *>(mbar + 1);
  float *red = reinterpret_cast<float *>(tslot + 4);     // [128][33] (pool)

  const int L = a.L, N = MODE == kTab1 ? kNPatterns : L * L;
  const int tid = threadIdx.x, warp = tid >> 5;
  const int tiles_per_img = N / kTileM;

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(tslot)),
                 "r"(32)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (tid == 0) {
    mbar_init(smem_u32(mbar), 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  // ---- stage B (32 x K weights), once ----
  for (int i = tid; i < kC * (K / 8); i += blockDim.x) {
    const int n = i / (K / 8), kc = i % (K / 8);
    cp_async16(smem_u32(sB + il_off(n, kc * 8, SBO)), a.w + (size_t)n * K + kc * 8);
  }
  cp_async_wait_all();
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t taddr = *tslot;

  uint32_t phase = 0;
  for (int tile = blockIdx.x; tile < a.ntiles; tile += gridDim.x) {
    const int img = tile / tiles_per_img;
    const int p0 = (tile % tiles_per_img) * kTileM;
    const int p = p0 + tid;  // this thread's pixel in the epilogue

    // ---- stage A (im2col rows of the tile) ----
    if constexpr (MODE == kTab1) {
      __align__(16) __nv_bfloat16 v[16];
#pragma unroll
      for (int k = 0; k < 16; ++k)
        v[k] = __float2bfloat16_rn(k < 9 ? ((p >> k) & 1 ? 1.0f : -1.0f) : 0.0f);
      *reinterpret_cast<uint4 *>(sA + il_off(tid, 0, SBO)) = *reinterpret_cast<uint4 *>(&v[0]);
      *reinterpret_cast<uint4 *>(sA + il_off(tid, 8, SBO)) = *reinterpret_cast<uint4 *>(&v[8]);
    } else {
      // Four consecutive threads copy the four 16-byte channel chunks of one
      // neighbour pixel, so a warp reads 8 whole pixels (512 contiguous bytes
      // within an image row) per instruction.
      const __nv_bfloat16 *x = a.x + (size_t)img * N * kC;
      const int c = tid & 3;
#pragma unroll
      for (int tap = 0; tap < 9; ++tap) {
        // forward reads the tap's neighbour; the data gradient the opposite one
        const int t = MODE == kBwd ? 8 - tap : tap;
#pragma unroll
        for (int it = 0; it < kTileM / 32; ++it) {
          const int r = it * 32 + (tid >> 2);  // tile row (pixel) handled by this thread
          const int pp = p0 + r;
          const int y = pp / L, xc = pp - y * L;
          const int yy = y + t / 3 - 1, xx = xc + t % 3 - 1;
          const int q = (yy < 0 ? yy + L : (yy >= L ? yy - L : yy)) * L +
                        (xx < 0 ? xx + L : (xx >= L ? xx - L : xx));
          const char *src = reinterpret_cast<const char *>(x + (size_t)q * kC) + 16 * c;
          cp_async16(smem_u32(sA + il_off(r, tap * kC + 8 * c, SBO)), src);
        }
      }
      cp_async_wait_all();
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");

    if (tid == 0) {
      const uint32_t a0 = smem_u32(sA), b0 = smem_u32(sB);
#pragma unroll
      for (int j = 0; j < K / 16; ++j)
        umma_bf16(taddr, umma_desc(a0 + j * 256, 128, SBO), umma_desc(b0 + j * 256, 128, SBO),
                  j > 0 ? 1u : 0u);
      umma_commit(smem_u32(mbar));
    }
    // One thread polls the MMA barrier; the CTA barrier passes the result on
    // (127 spinning threads would keep the shared-memory pipe busy).
    bool waited = true;
    if (tid == 0) waited = mbar_wait(smem_u32(mbar), phase);
    const bool ok = __syncthreads_and(waited ? 1 : 0) != 0;
    phase ^= 1u;
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    float acc[32];
    tmem_ld32(taddr + ((uint32_t)(warp * 32) << 16), acc);

    // ---- epilogue: this thread owns pixel p's 32 channels ----
    if (ok) {
      __align__(16) __nv_bfloat16 o[32];
      if constexpr (MODE == kBwd) {
        // the pixel's 32 mask activations as four 16-byte loads
        __align__(16) __nv_bfloat16 m[32];
        const uint4 *msrc =
            reinterpret_cast<const uint4 *>(a.mask_src + ((size_t)img * N + p) * kC);
#pragma unroll
        for (int c = 0; c < 4; ++c) reinterpret_cast<uint4 *>(m)[c] = msrc[c];
#pragma unroll
        for (int c = 0; c < 32; ++c)
          o[c] = __float2bfloat16_rn(__bfloat162float(m[c]) > 0.0f ? acc[c] : 0.0f);
      } else {
#pragma unroll
        for (int c = 0; c < 32; ++c) {
          const float z = acc[c] + a.bias[c];
          acc[c] = z > 0.0f ? z : 0.0f;
          o[c] = __float2bfloat16_rn(acc[c]);
        }
      }
      if (a.y != nullptr) {  // prediction does not keep the last layer's activations
        uint4 *dst = reinterpret_cast<uint4 *>(a.y + ((size_t)img * N + p) * kC);
#pragma unroll
        for (int c = 0; c < 4; ++c) dst[c] = reinterpret_cast<uint4 *>(o)[c];
      }
      if (MODE == kFwd && a.pool != nullptr) {
        // channel sums of the rounded activations over the tile
#pragma unroll
        for (int c = 0; c < 32; ++c) red[tid * 33 + c] = __bfloat162float(o[c]);
      }
    }
    if (MODE == kFwd && a.pool != nullptr) {
      __syncthreads();
      if (ok && tid < 32) {
        float sum = 0.f;
        for (int r = 0; r < kTileM; ++r) sum += red[r * 33 + tid];
        atomicAdd(&a.pool[img * kC + tid], sum);
      }
    }
    // every TMEM read and shared-memory use of this tile is done before the
    // next tile's staging and MMA
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    const int bad = __syncthreads_or(ok ? 0 : 1);
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (bad) {
      if (tid == 0 && a.err) atomicExch(a.err, 1);
      break;
    }
  }
  if (warp == 0) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(32)
                 : "memory");
  }
}

// The first layer from its activation table: pixel p's 32 BF16 activations
// are row q of the table, q the pattern of its 3x3 neighbourhood (bit
// (dy+1)*3 + (dx+1) set where that spin is +1).  k_conv_tc<kTab1> fills the
// table with the same A rows (+-1 per tap, zero padding to K = 16), weights,
// MMA and epilogue as a per-pixel first layer, so the activations equal
// those of the im2col form (checked byte for byte on the GPU), which has to
// stage and multiply every pixel of the batch.  This kernel only writes 64
// bytes per pixel (HBM bound): lane l finds the pattern of pixel base + l,
// then the warp writes its 32 rows as four 512-byte stretches, lane l taking
// 16-byte chunk l % 4 of pixel base + 8 i + l / 4 in step i.  Spins other
// than +1 count as -1.  Grid: x over 256-pixel blocks of an image, y over
// images (strided when the batch exceeds gridDim.y).
__global__ void __launch_bounds__(256) k_conv1_lookup(const int8_t *spins,
                                                      const __nv_bfloat16 *tab,
                                                      __nv_bfloat16 *y, int L, int batch) {
  const int N = L * L;
  const int lane = threadIdx.x & 31;
  const int base = blockIdx.x * blockDim.x + (threadIdx.x & ~31);  // the warp's first pixel
  if (base >= N) return;
  const int p = base + lane;
  const bool own = p < N;
  const int pc = own ? p : N - 1;
  const int r = pc / L, col = pc - r * L;
  const int rows[3] = {(r == 0 ? L - 1 : r - 1) * L, r * L, (r == L - 1 ? 0 : r + 1) * L};
  const int cols[3] = {col == 0 ? L - 1 : col - 1, col, col == L - 1 ? 0 : col + 1};
  const uint4 *tab16 = reinterpret_cast<const uint4 *>(tab);
  for (int img = blockIdx.y; img < batch; img += gridDim.y) {
    const int8_t *sp = spins + (size_t)img * N;
    int q = 0;
#pragma unroll
    for (int k = 0; k < 9; ++k) q |= (sp[rows[k / 3] + cols[k % 3]] > 0 ? 1 : 0) << k;
    uint4 *dst = reinterpret_cast<uint4 *>(y + ((size_t)img * N + base) * kC);
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const int j = 8 * i + (lane >> 2);  // pixel base + j, chunk lane % 4
      const int qj = __shfl_sync(0xffffffffu, q, j);
      if (base + j < N) dst[4 * j + (lane & 3)] = tab16[4 * qj + (lane & 3)];
    }
  }
}

// The 32-channel layers without an im2col buffer.  A tile's 128 output
// pixels p0..p0+127 need input pixels p0-L .. p0+127+L (a window of
// W = 128 + 2L consecutive pixels, row-major, rows wrapping); the window is
// staged three times, rotated by dx = -1, 0, +1 within each image row, so
// the A operand of tap (dy, dx) is the rotated copy dx starting (dy+1)*L
// pixels into the window: 128 consecutive pixels at a 16-byte stride, which a
// UMMA descriptor addresses directly (8-pixel groups 128 B apart, 8-channel
// chunks W*16 B apart).  Shared memory per tile: 3 * W * 64 B (48 KB at L=64)
// instead of the 72 KB im2col, and every input pixel is read from L2 once per
// tile instead of nine times.  Same arithmetic as k_conv_tc (same K order:
// tap-major, 32 channels per tap; same FP32 accumulation order per MMA).
//
// LT > 0 (L = 32, 64, 128, dividing the 128-pixel tile): the window is whole
// image rows, so each thread loads its 16-byte chunks once from global memory
// into registers and stores them to the three rotated copies itself (one L2
// read per input chunk); LT == 0: any L, three cp.async per chunk.
template <int MODE, int LT>
__global__ void __launch_bounds__(128) k_conv_win(ConvArgs a) {
  static_assert(MODE == kFwd || MODE == kBwd, "32-channel layers only");
  static_assert(LT == 0 || (kTileM % (LT > 0 ? LT : 1) == 0 && (LT & (LT - 1)) == 0),
                "LT divides the tile");
  constexpr int K = 9 * kC;
  constexpr int SBO_B = K * 16;  // weights: bytes between 8-row groups
  extern __shared__ __align__(1024) unsigned char smem[];
  const int L = a.L, N = L * L;
  const int W = kTileM + 2 * L;          // window pixels
  const uint32_t lbo = (uint32_t)W * 16; // bytes between 8-channel chunks
  const uint32_t vstride = 4u * lbo;     // bytes between the three rotated copies
  unsigned char *sA = smem;                             // [3][4][W][16 B]
  unsigned char *sB = smem + 3 * vstride;               // 32 x K bf16 (interleaved)
  uint64_t *mbar = reinterpret_cast<uint64_t *>(sB + kC * K * 2);
  uint32_t *tslot = reinterpret_cast<uint32_t *>(mbar + 1);
  float *red = reinterpret_cast<float *>(tslot + 4);   // [128][33] (pool)

  const int tid = threadIdx.x, warp = tid >> 5;
  const int tiles_per_img = N / kTileM;

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(tslot)),
                 "r"(32)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (tid == 0) {
    mbar_init(smem_u32(mbar), 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  for (int i = tid; i < kC * (K / 8); i += blockDim.x) {
    const int n = i / (K / 8), kc = i % (K / 8);
    cp_async16(smem_u32(sB + il_off(n, kc * 8, SBO_B)), a.w + (size_t)n * K + kc * 8);
  }
  cp_async_wait_all();
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t taddr = *tslot;

  // LT > 0: a tile's window is loaded into registers one tile ahead, so the
  // global loads of tile i+1 are in flight during the MMA and epilogue of i.
  constexpr int LR0 = LT > 0 ? LT : 1;
  constexpr int kPerW = (kTileM + 2 * LR0) * 4 / 128;  // 16-byte chunks per thread
  uint4 v4[kPerW];
  auto load_window = [&](int t) {
    const int timg = t / tiles_per_img;
    const int y0 = ((t % tiles_per_img) * kTileM) / LR0;  // first output row of the tile
    const __nv_bfloat16 *xs = a.x + (size_t)timg * N * kC;
#pragma unroll
    for (int j = 0; j < kPerW; ++j) {
      // a quarter-warp (8 lanes) takes one 16-byte channel chunk of 8
      // consecutive pixels: each rotated-copy store is one 128-byte row per
      // quarter-warp (no bank conflict); the warp still reads 512 contiguous bytes
      const int c = (tid & 31) >> 3, w = j * 32 + (tid >> 5) * 8 + (tid & 7);
      int row = y0 - 1 + w / LR0;
      row = row < 0 ? row + LR0 : (row >= LR0 ? row - LR0 : row);
      v4[j] = *reinterpret_cast<const uint4 *>(xs + ((size_t)row * LR0 + (w % LR0)) * kC + 8 * c);
    }
  };
  if constexpr (LT > 0) {
    if ((int)blockIdx.x < a.ntiles) load_window(blockIdx.x);
  }

  uint32_t phase = 0;
  for (int tile = blockIdx.x; tile < a.ntiles; tile += gridDim.x) {
    const int img = tile / tiles_per_img;
    const int p0 = (tile % tiles_per_img) * kTileM;
    const int p = p0 + tid;
    const __nv_bfloat16 *x = a.x + (size_t)img * N * kC;

    // ---- stage the three rotated windows (16-byte chunks, channel chunk fastest) ----
    if constexpr (LT > 0) {
#pragma unroll
      for (int j = 0; j < kPerW; ++j) {  // the registers hold this tile's window
        const int c = (tid & 31) >> 3, w = j * 32 + (tid >> 5) * 8 + (tid & 7);
        const int col = w % LR0, rbase = w - col;
#pragma unroll
        for (int v = 0; v < 3; ++v) {  // copy v holds, at column col', input column col' + v - 1
          const int cd = (col - (v - 1) + LR0) % LR0;
          *reinterpret_cast<uint4 *>(sA + v * vstride + c * lbo + (uint32_t)(rbase + cd) * 16) =
              v4[j];
        }
      }
    } else {
      for (int i = tid; i < 3 * W * 4; i += blockDim.x) {
        const int c = i & 3;
        const int w = (i >> 2) % W;
        const int v = (i >> 2) / W;                // rotation dx = v - 1
        int q = p0 - L + w;
        q = q < 0 ? q + N : (q >= N ? q - N : q);  // window pixel (rows wrap)
        const int r = q / L, col = q - r * L;
        int cs = col + v - 1;
        cs = cs < 0 ? cs + L : (cs >= L ? cs - L : cs);
        const char *src = reinterpret_cast<const char *>(x + ((size_t)r * L + cs) * kC) + 16 * c;
        cp_async16(smem_u32(sA + v * vstride + c * lbo + (uint32_t)w * 16), src);
      }
      cp_async_wait_all();
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");

    if (tid == 0) {
      const uint32_t a0 = smem_u32(sA), b0 = smem_u32(sB);
#pragma unroll
      for (int tap = 0; tap < 9; ++tap) {
        // forward reads the tap's neighbour; the data gradient the opposite one
        const int t = MODE == kBwd ? 8 - tap : tap;
        const int dy = t / 3 - 1, dx = t % 3 - 1;
        const uint32_t abase = a0 + (uint32_t)(dx + 1) * vstride + (uint32_t)((dy + 1) * L) * 16;
#pragma unroll
        for (int j = 0; j < 2; ++j)
          umma_bf16(taddr, umma_desc(abase + 2u * j * lbo, lbo, 128),
                    umma_desc(b0 + (uint32_t)(tap * 2 + j) * 256, 128, SBO_B),
                    (tap | j) ? 1u : 0u);
      }
      umma_commit(smem_u32(mbar));
    }
    if constexpr (LT > 0) {  // the next tile's loads overlap this tile's MMA and epilogue
      const int nt = tile + (int)gridDim.x;
      if (nt < a.ntiles) load_window(nt);
    }
    // One thread polls the MMA barrier; the CTA barrier passes the result on
    // (127 spinning threads would keep the shared-memory pipe busy).
    bool waited = true;
    if (tid == 0) waited = mbar_wait(smem_u32(mbar), phase);
    const bool ok = __syncthreads_and(waited ? 1 : 0) != 0;
    phase ^= 1u;
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    float acc[32];
    tmem_ld32(taddr + ((uint32_t)(warp * 32) << 16), acc);

    if (ok) {
      __align__(16) __nv_bfloat16 o[32];
      if constexpr (MODE == kBwd) {
        // the pixel's 32 mask activations as four 16-byte loads
        __align__(16) __nv_bfloat16 m[32];
        const uint4 *msrc =
            reinterpret_cast<const uint4 *>(a.mask_src + ((size_t)img * N + p) * kC);
#pragma unroll
        for (int c = 0; c < 4; ++c) reinterpret_cast<uint4 *>(m)[c] = msrc[c];
#pragma unroll
        for (int c = 0; c < 32; ++c)
          o[c] = __float2bfloat16_rn(__bfloat162float(m[c]) > 0.0f ? acc[c] : 0.0f);
      } else {
#pragma unroll
        for (int c = 0; c < 32; ++c) {
          const float z = acc[c] + a.bias[c];
          acc[c] = z > 0.0f ? z : 0.0f;
          o[c] = __float2bfloat16_rn(acc[c]);
        }
      }
      if (a.y != nullptr) {  // prediction does not keep the last layer's activations
        uint4 *dst = reinterpret_cast<uint4 *>(a.y + ((size_t)img * N + p) * kC);
#pragma unroll
        for (int c = 0; c < 4; ++c) dst[c] = reinterpret_cast<uint4 *>(o)[c];
      }
      if (MODE == kFwd && a.pool != nullptr) {
#pragma unroll
        for (int c = 0; c < 32; ++c) red[tid * 33 + c] = __bfloat162float(o[c]);
      }
    }
    if (MODE == kFwd && a.pool != nullptr) {
      __syncthreads();
      if (ok && tid < 32) {
        float sum = 0.f;
        for (int r = 0; r < kTileM; ++r) sum += red[r * 33 + tid];
        atomicAdd(&a.pool[img * kC + tid], sum);
      }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    const int bad = __syncthreads_or(ok ? 0 : 1);
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (bad) {
      if (tid == 0 && a.err) atomicExch(a.err, 1);
      break;
    }
  }
  if (warp == 0) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(32)
                 : "memory");
  }
}

// ---------------------------------------------------------------------------
// The 32-channel forward layers at L = 64 with one staged copy of the window.
// Positions run in rows of kGhP = 66: a ghost column on each side of the 64
// pixels holds the circularly wrapped neighbour (left ghost = pixel 63 of the
// row, right ghost = pixel 0), so the A operand of tap (dy, dx) for 128
// consecutive positions is 128 consecutive window positions (1 + dy) * 66 +
// dx + 1 further on -- a plain descriptor offset, with no rotated copies.  An
// image is 64 * 66 = 33 * 128 positions: 33 M tiles of 128 consecutive
// positions, whose ghost outputs (3 %) are computed and dropped.  A tile's
// window is the 262 positions from 67 before its first position, staged once
// (4 x 264 x 16 B = 17 KB against k_conv_win's three rotated copies, 48 KB).
// Same arithmetic as k_conv_win (same K order: tap-major, 32 channels per
// tap; same FP32 accumulation per MMA), so the same outputs.
// Measured (one B200, prediction of 100 000 grids, bench.py --workload cnn):
// 1.163M grids/s against 1.036M with k_conv_win's rotated copies (one
// buffer, no double buffering: 1.098M); per 1024-image layer 244 us against
// 277 us (ncu), shared-memory stores 5.8 M wavefronts against 14.1 M, the
// tensor core's operand reads (24.3 M wavefronts) now the bulk of l1tex 75 %.
// ---------------------------------------------------------------------------
constexpr int kGhP = 66;                 // positions per padded row
constexpr int kGhTiles = 64 * kGhP / kTileM;  // 33 M tiles per image
constexpr int kGhLead = kGhP + 1;        // window positions before the tile's first
constexpr int kGhWin = 264;              // window positions staged (262, rounded up to 8)
static_assert(kGhTiles * kTileM == 64 * kGhP, "whole tiles per image");
static_assert(kGhWin >= kTileM + 2 * kGhLead, "window covers every tap");

size_t conv_gh64_smem(bool pool) {
  return 2 * 4 * (size_t)kGhWin * 16 + (size_t)kC * 9 * kC * 2 + 64 +
         (pool ? (size_t)kTileM * 33 * 4 : 0);
}

// Two window buffers and two TMEM accumulators: while the epilogue of tile
// i reads accumulator i % 2, the MMAs of tile i+1 (staged into the other
// buffer just before) run into the other accumulator.  A buffer is
// restaged only after the MMAs that read it have completed (waited for one
// iteration earlier), an accumulator is rewritten only after its epilogue's
// tcgen05.ld (also one iteration earlier).
__global__ void __launch_bounds__(128) k_conv_gh64(ConvArgs a) {
  constexpr int L = 64, N = L * L;
  constexpr int K = 9 * kC;
  constexpr int SBO_B = K * 16;                    // weights: bytes between 8-row groups
  constexpr uint32_t lbo = (uint32_t)kGhWin * 16;  // bytes between 8-channel chunks
  constexpr uint32_t kBuf = 4 * lbo;               // bytes per window buffer
  constexpr int kPerW = (kGhWin * 4 + 127) / 128;  // 16-byte chunks per thread (9)
  extern __shared__ __align__(1024) unsigned char smem[];
  unsigned char *sA = smem;                        // [2][4][kGhWin][16 B]
  unsigned char *sB = smem + 2 * kBuf;             // 32 x K bf16 (interleaved)
  uint64_t *mbar = reinterpret_cast<uint64_t *>(sB + kC * K * 2);  // [2]
  uint32_t *tslot = reinterpret_cast<uint32_t *>(mbar + 2);
  float *red = reinterpret_cast<float *>(tslot + 4);  // [128][33] (pool)

  const int tid = threadIdx.x, warp = tid >> 5;

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(tslot)),
                 "r"(64)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (tid == 0) {
    mbar_init(smem_u32(&mbar[0]), 1);
    mbar_init(smem_u32(&mbar[1]), 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  for (int i = tid; i < kC * (K / 8); i += blockDim.x) {
    const int n = i / (K / 8), kc = i % (K / 8);
    cp_async16(smem_u32(sB + il_off(n, kc * 8, SBO_B)), a.w + (size_t)n * K + kc * 8);
  }
  cp_async_wait_all();
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t taddr = *tslot;

  // A tile's window is loaded into registers ahead of its staging, so the
  // global loads are in flight during the MMAs and epilogue before it.  A
  // quarter-warp (8 lanes) takes one 16-byte channel chunk of 8 consecutive
  // positions: each shared store is one conflict-free 128-byte row.
  uint4 v4[kPerW];
  auto load_window = [&](int t) {
    const int timg = t / kGhTiles, m = t - timg * kGhTiles;
    const __nv_bfloat16 *xs = a.x + (size_t)timg * N * kC;
    const int c = (tid & 31) >> 3;
#pragma unroll
    for (int j = 0; j < kPerW; ++j) {
      const int w = j * 32 + (tid >> 5) * 8 + (tid & 7);
      if (w < kGhWin) {
        int q = m * kTileM - kGhLead + w;  // padded position, rows wrap
        q = q < 0 ? q + L * kGhP : (q >= L * kGhP ? q - L * kGhP : q);
        const int r = q / kGhP, col = q - r * kGhP;
        const int pc = col == 0 ? L - 1 : (col == kGhP - 1 ? 0 : col - 1);
        v4[j] = *reinterpret_cast<const uint4 *>(xs + ((size_t)r * L + pc) * kC + 8 * c);
      }
    }
  };
  // stage the registers' window into buffer b, then (one thread) issue the
  // tile's 18 MMAs into accumulator b with a commit to mbar[b]
  auto stage_and_issue = [&](int b) {
    const int c = (tid & 31) >> 3;
    unsigned char *buf = sA + b * kBuf;
#pragma unroll
    for (int j = 0; j < kPerW; ++j) {
      const int w = j * 32 + (tid >> 5) * 8 + (tid & 7);
      if (w < kGhWin) *reinterpret_cast<uint4 *>(buf + c * lbo + (uint32_t)w * 16) = v4[j];
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (tid == 0) {
      const uint32_t a0 = smem_u32(buf), b0 = smem_u32(sB);
#pragma unroll
      for (int tap = 0; tap < 9; ++tap) {
        const int dy = tap / 3 - 1, dx = tap % 3 - 1;
        const uint32_t abase = a0 + (uint32_t)(kGhLead + dy * kGhP + dx) * 16u;
#pragma unroll
        for (int j = 0; j < 2; ++j)
          umma_bf16(taddr + (uint32_t)(b * 32), umma_desc(abase + 2u * j * lbo, lbo, 128),
                    umma_desc(b0 + (uint32_t)(tap * 2 + j) * 256, 128, SBO_B),
                    (tap | j) ? 1u : 0u);
      }
      umma_commit(smem_u32(&mbar[b]));
    }
  };

  // thread 0's view: bit b of `phase` is the parity of mbar[b]'s next
  // completion; bit b of `outstanding` marks MMAs committed to mbar[b] and
  // not yet waited for
  uint32_t phase = 0, outstanding = 0;
  int tile = blockIdx.x;
  if (tile < a.ntiles) {
    load_window(tile);
    stage_and_issue(0);
    outstanding |= 1u;
    if (tile + (int)gridDim.x < a.ntiles) load_window(tile + (int)gridDim.x);
  }
  for (int it = 0; tile < a.ntiles; tile += gridDim.x, ++it) {
    const int cur = it & 1;
    const int img = tile / kGhTiles, m = tile - img * kGhTiles;
    const int nt = tile + (int)gridDim.x;
    if (nt < a.ntiles) {  // the next tile's MMAs run during this tile's epilogue
      stage_and_issue(cur ^ 1);
      outstanding |= 1u << (cur ^ 1);
      if (nt + (int)gridDim.x < a.ntiles) load_window(nt + (int)gridDim.x);
    }
    // One thread polls the MMA barrier; the CTA barrier passes the result on.
    bool waited = true;
    if (tid == 0) {
      waited = mbar_wait(smem_u32(&mbar[cur]), (phase >> cur) & 1u);
      if (waited) {
        phase ^= 1u << cur;
        outstanding &= ~(1u << cur);
      }
    }
    const bool ok = __syncthreads_and(waited ? 1 : 0) != 0;
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    float acc[32];
    tmem_ld32(taddr + ((uint32_t)(warp * 32) << 16) + (uint32_t)(cur * 32), acc);

    const int q = m * kTileM + tid;  // this thread's padded position
    const int r = q / kGhP, col = q - r * kGhP;
    const bool pixel = col >= 1 && col <= L;
    if (ok) {
      __align__(16) __nv_bfloat16 o[32];
#pragma unroll
      for (int c = 0; c < 32; ++c) {
        const float z = acc[c] + a.bias[c];
        acc[c] = z > 0.0f ? z : 0.0f;
        o[c] = __float2bfloat16_rn(acc[c]);
      }
      if (a.y != nullptr && pixel) {  // prediction does not keep the last layer's activations
        uint4 *dst = reinterpret_cast<uint4 *>(a.y + ((size_t)img * N + r * L + col - 1) * kC);
#pragma unroll
        for (int c = 0; c < 4; ++c) dst[c] = reinterpret_cast<uint4 *>(o)[c];
      }
      if (a.pool != nullptr) {
#pragma unroll
        for (int c = 0; c < 32; ++c) red[tid * 33 + c] = pixel ? __bfloat162float(o[c]) : 0.0f;
      }
    }
    if (a.pool != nullptr) {
      __syncthreads();
      if (ok && tid < 32) {
        float sum = 0.f;
        for (int rr = 0; rr < kTileM; ++rr) sum += red[rr * 33 + tid];
        atomicAdd(&a.pool[img * kC + tid], sum);
      }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    const int bad = __syncthreads_or(ok ? 0 : 1);
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (bad) {
      if (tid == 0 && a.err) atomicExch(a.err, 1);
      break;
    }
  }
  // After an abort MMAs may still be in flight into either accumulator: wait
  // for their commits (bounded) before the columns are released.
  if (tid == 0) {
    for (int b = 0; b < 2; ++b)
      if ((outstanding >> b) & 1u) mbar_wait(smem_u32(&mbar[b]), (phase >> b) & 1u);
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(64)
                 : "memory");
  }
}

// ---------------------------------------------------------------------------
// Inference forward of the whole network for L = 64 in one kernel.  A work
// item is an image band of kFzRows output rows; the four layers run back to
// back on the chip and only the band's spins come from HBM (the pooled sums
// go out by atomicAdd): layer l computes its rows of the band plus the halo
// the next layer needs (a1: 14 rows, a2: 12, a3: 10, a4: 8, pooled).
// Activations stay in shared memory, K-major like k_conv_win's windows
// ([channel chunk][position][16 B]), in rows of kFzPitch = 66 positions: a
// ghost column, the 64 pixels, a ghost column, the ghosts holding the
// circularly wrapped neighbours.  With that pitch the A operand of tap
// (dy, dx) for 128 consecutive output positions is 128 consecutive input
// positions starting (1 + dy) * 66 + dx further on, a plain descriptor offset;
// an M tile covers 128 padded positions, and its ghost positions (3 %) are
// computed and dropped.  Two TMEM accumulators: while one 4-warp group runs
// the epilogue of tile t (bias, ReLU, BF16 rounding, stores into the next
// layer's buffer and the ghost copies, or the pool sums), warp 8 issues the
// MMAs of tile t + 1.  Same arithmetic as the layer-by-layer kernels (BF16
// activations, FP32 accumulation, the same K order).
// ---------------------------------------------------------------------------
constexpr int kFzRows = 8;     // output rows per band
constexpr int kFzPitch = 66;   // positions per padded row
constexpr int kFzLead = 8;     // positions before position 0 (tap reads reach -1)
constexpr int kFzPosA = 1048;  // positions per chunk, buffer A (a1: 14 rows, a3: 10)
constexpr int kFzPosB = 912;   // buffer B (a2: 12 rows)
constexpr int kFzIm = 1024;    // layer-1 im2col rows (8 tiles of 128)
constexpr int kFzGroups = 4;                    // TMEM accumulators = epilogue groups of 4 warps
constexpr int kFzThreads = (4 * kFzGroups + 1) * 32;  // + one MMA-issue warp (the last)
constexpr int kFzTilesMax = 8;                  // M tiles per layer and band, at most
// shared-memory layout (bytes)
constexpr uint32_t kFzW = 0;                                 // W2..W4, 3 x 32 x 288 bf16
constexpr uint32_t kFzW1 = kFzW + 3u * kC * 288 * 2;         // W1, 32 x 16 bf16
constexpr uint32_t kFzBufA = kFzW1 + (uint32_t)kC * 16 * 2;  // [4][kFzPosA][16 B]
constexpr uint32_t kFzBufB = kFzBufA + 4u * kFzPosA * 16;    // [4][kFzPosB][16 B]
constexpr uint32_t kFzImB = kFzBufB + 4u * kFzPosB * 16;     // im2col, 1024 x 16 bf16
constexpr uint32_t kFzSp = kFzImB + (uint32_t)kFzIm * 16 * 2;  // spins, 16 rows x 66 (+pad)
constexpr uint32_t kFzBias = kFzSp + 16u * kFzPitch + 32;      // 4 x 32 floats
constexpr uint32_t kFzPool = kFzBias + 4u * kC * 4;            // 32 floats
// mbarriers: mma_done[4], acc_free[4], tile_done[4 layers][8]; then the TMEM
// slot and the abort flag
constexpr uint32_t kFzBar = kFzPool + (uint32_t)kC * 4;
constexpr uint32_t kFzNBar = 2 * kFzGroups + 4 * kFzTilesMax;
constexpr size_t kFzSmem = kFzBar + kFzNBar * 8 + 16;
static_assert(kFzSmem <= 227 * 1024, "fused kernel shared memory");
static_assert(kFzBufA % 16 == 0 && kFzBufB % 16 == 0 && kFzImB % 16 == 0, "16-byte operands");

struct FusedArgs {
  const int8_t *spins;           // [B][4096]
  const __nv_bfloat16 *w1;       // [32][16] (taps padded)
  const __nv_bfloat16 *w;        // W2..W4 [3][32][288]
  const float *params;           // biases (kOffB1.. in the flat parameter vector)
  float *pool;                   // [B][32] channel sums of a4 (added to)
  int *err;                      // set on a timed-out wait
  int nbands;                    // B * (64 / kFzRows)
};

__global__ void __launch_bounds__(kFzThreads, 1) k_cnn_fused64(FusedArgs a) {
  constexpr int L = 64, N = L * L;
  constexpr int K = 9 * kC;       // 288
  constexpr int SBO_W = K * 16;   // weights: bytes between 8-row groups
  constexpr int kBands = L / kFzRows;
  constexpr int kIssuer = 4 * kFzGroups;  // the MMA warp
  extern __shared__ __align__(1024) unsigned char smem[];
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  uint64_t *bar = reinterpret_cast<uint64_t *>(smem + kFzBar);
  uint64_t *mma_done = bar;                        // [kFzGroups], one commit each
  uint64_t *acc_free = bar + kFzGroups;            // [kFzGroups], one arrival per warp
  uint64_t *tile_done = bar + 2 * kFzGroups;       // [4][kFzTilesMax], one arrival per warp
  uint32_t *tslot = reinterpret_cast<uint32_t *>(smem + kFzBar + kFzNBar * 8);
  volatile int *abort_flag = reinterpret_cast<volatile int *>(smem + kFzBar + kFzNBar * 8 + 8);
  float *bias = reinterpret_cast<float *>(smem + kFzBias);
  float *spool = reinterpret_cast<float *>(smem + kFzPool);
  int8_t *sp = reinterpret_cast<int8_t *>(smem + kFzSp);
  const uint32_t sbase = smem_u32(smem);

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(tslot)),
                 "r"(32 * kFzGroups)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (tid == 0) {
    for (int i = 0; i < kFzGroups; ++i) {
      mbar_init(smem_u32(&mma_done[i]), 1);
      mbar_init(smem_u32(&acc_free[i]), 4);
    }
    for (int i = 0; i < 4 * kFzTilesMax; ++i) mbar_init(smem_u32(&tile_done[i]), 4);
    *abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  // weights, once per CTA: W2..W4 as k_conv_win stages them, W1 as k_conv_tc
  for (int i = tid; i < 3 * kC * (K / 8); i += blockDim.x) {
    const int l = i / (kC * (K / 8)), r = i % (kC * (K / 8));
    const int n = r / (K / 8), kc = r % (K / 8);
    cp_async16(sbase + kFzW + (uint32_t)(l * kC * K * 2) + il_off(n, kc * 8, SBO_W),
               a.w + (size_t)l * kC * K + (size_t)n * K + kc * 8);
  }
  for (int i = tid; i < kC * 2; i += blockDim.x)
    cp_async16(sbase + kFzW1 + il_off(i >> 1, (i & 1) * 8, 256), a.w1 + (i >> 1) * 16 + (i & 1) * 8);
  for (int i = tid; i < 4 * kC; i += blockDim.x) {
    const int l = i / kC, c = i % kC;
    bias[i] = a.params[l == 0 ? kOffB1 + c : kOffB2 + (l - 1) * (9216 + 32) + c];
  }
  cp_async_wait_all();
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t taddr = *tslot;

  const int grp = warp >> 2, quad = warp & 3;  // epilogue warps (warp < kIssuer)
  uint32_t use[kFzGroups] = {};                // issuer: uses of each accumulator
  uint32_t my_use = 0;                         // epilogue: uses of its group's accumulator
  uint32_t my_base = 0;                        // tiles of earlier bands (accumulator = tile % 4)
  uint32_t nband = 0;                          // bands done (tile_done parity)

  for (int band = blockIdx.x; band < a.nbands; band += gridDim.x, ++nband) {
    const int img = band / kBands, y0 = (band % kBands) * kFzRows;
    // spins of image rows y0-4 .. y0+11, with the wrapped ghost columns
    const int8_t *sg = a.spins + (size_t)img * N;
    for (int i = tid; i < 16 * kFzPitch; i += blockDim.x) {
      const int r = i / kFzPitch, j = i - r * kFzPitch;
      const int x = (j - 1 + L) % L, y = (y0 - 4 + r + L) % L;
      sp[i] = sg[y * L + x];
    }
    if (tid < kC) spool[tid] = 0.f;
    __syncthreads();
    // layer-1 im2col: row q is a1 position q (local row q / 66, padded column q % 66)
    for (int q = tid; q < kFzIm; q += blockDim.x) {
      const int i = q / kFzPitch, j = q - i * kFzPitch;
      __align__(16) __nv_bfloat16 v[16];
#pragma unroll
      for (int k = 0; k < 16; ++k) {
        float f = 0.0f;
        if (k < 9) {
          const int r = min(i + 1 + k / 3 - 1, 15);
          const int jj = min(max(j + k % 3 - 1, 0), kFzPitch - 1);
          f = (float)sp[r * kFzPitch + jj];
        }
        v[k] = __float2bfloat16_rn(f);
      }
      *reinterpret_cast<uint4 *>(smem + kFzImB + il_off(q, 0, 256)) =
          *reinterpret_cast<const uint4 *>(&v[0]);
      *reinterpret_cast<uint4 *>(smem + kFzImB + il_off(q, 8, 256)) =
          *reinterpret_cast<const uint4 *>(&v[8]);
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    // The band's 26 M tiles, layer after layer (8, 7, 6, 5 tiles).  Tile t of
    // layer l reads layer l-1 positions up to 128 t + 260 (taps and ghost
    // columns), all written by tiles 0..t+2 of layer l-1, so it waits for
    // those tiles only: no barrier between layers.  The same bound keeps
    // every buffer write clear of the reads still in flight.
    if (warp == kIssuer) {
      if (lane == 0) {
        for (int layer = 0; layer < 4; ++layer) {
          const int ntiles = ((14 - 2 * layer) * kFzPitch + 127) / 128;
          const int nprev = layer > 0 ? ((16 - 2 * layer) * kFzPitch + 127) / 128 : 0;
          const uint32_t in_off = layer == 2 ? kFzBufB : kFzBufA;
          const uint32_t in_lbo = (layer == 2 ? kFzPosB : kFzPosA) * 16u;
          int ready = 0;
          for (int t = 0; t < ntiles; ++t) {
            const int g = (int)(use[0] + use[1] + use[2] + use[3]) & (kFzGroups - 1);
            if (use[g] > 0 && !*abort_flag &&
                !mbar_wait(smem_u32(&acc_free[g]), (use[g] - 1) & 1u))
              *abort_flag = 1;
            const int need = min(t + 3, nprev);
            for (; ready < need && !*abort_flag; ++ready)
              if (!mbar_wait(smem_u32(&tile_done[(layer - 1) * kFzTilesMax + ready]), nband & 1u))
                *abort_flag = 1;
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            if (!*abort_flag) {
              const uint32_t d = taddr + (uint32_t)(g * 32);
              if (layer == 0) {
                umma_bf16(d, umma_desc(sbase + kFzImB + (uint32_t)t * 4096u, 128, 256),
                          umma_desc(sbase + kFzW1, 128, 256), 0u);
              } else {
                // descriptors differ only in their start address (bits 0-13,
                // in 16-byte units): one base each, offsets added per MMA
                const uint64_t da0 =
                    umma_desc(sbase + in_off + (uint32_t)(kFzLead + 128 * t) * 16u, in_lbo, 128);
                const uint64_t db0 =
                    umma_desc(sbase + kFzW + (uint32_t)((layer - 1) * kC * K * 2), 128, SBO_W);
                const uint32_t lbo16 = in_lbo >> 4;
#pragma unroll
                for (int tap = 0; tap < 9; ++tap) {
                  const int pos = (tap / 3) * kFzPitch + tap % 3 - 1;  // >= -1; base is kFzLead in
#pragma unroll
                  for (int j = 0; j < 2; ++j)
                    umma_bf16(d, da0 + (uint64_t)(int64_t)(pos + (int)(2u * j * lbo16)),
                              db0 + (uint64_t)((tap * 2 + j) * 16), (tap | j) ? 1u : 0u);
                }
              }
              umma_commit(smem_u32(&mma_done[g]));
            }
            ++use[g];
          }
        }
      }
      __syncwarp();
    } else {
      uint32_t seqb = 0;  // tiles of this band so far
      for (int layer = 0; layer < 4; ++layer) {
        const int npos = (14 - 2 * layer) * kFzPitch;  // output positions of this layer
        const int ntiles = (npos + 127) / 128;
        // layer index 1 writes buffer B, 2 writes A, 3 (pooled) writes B; 0 writes A
        const uint32_t out_off = (layer & 1) ? kFzBufB : kFzBufA;
        const uint32_t out_lbo = ((layer & 1) ? kFzPosB : kFzPosA) * 16u;
        for (int t = 0; t < ntiles; ++t, ++seqb) {
          if ((int)((my_base + seqb) & (kFzGroups - 1)) != grp) continue;
          // one lane polls; the warp barrier passes it on
          if (lane == 0 && !*abort_flag && !mbar_wait(smem_u32(&mma_done[grp]), my_use & 1u))
            *abort_flag = 1;
          __syncwarp();
          ++my_use;
          asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
          float acc[32];
          tmem_ld32(taddr + ((uint32_t)(quad * 32) << 16) + (uint32_t)(grp * 32), acc);
          asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
          __syncwarp();
          // the accumulator is in registers: hand it back to the issuer now
          if (lane == 0)
            asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(&acc_free[grp]))
                         : "memory");
          const int q = 128 * t + quad * 32 + lane;
          const int i = q / kFzPitch, j = q - i * kFzPitch;
          if (!*abort_flag && q < npos && j >= 1 && j <= L) {  // a pixel (not a ghost) of the band
            const float *bl = bias + layer * kC;
            __align__(16) __nv_bfloat16 o[32];
#pragma unroll
            for (int c = 0; c < 32; ++c) {
              const float z = acc[c] + bl[c];
              o[c] = __float2bfloat16_rn(z > 0.0f ? z : 0.0f);
            }
            const uint32_t p0 = (uint32_t)(kFzLead + q) * 16u;
            const bool ghost = layer < 3 && (j == 1 || j == L);
            const uint32_t pg = (uint32_t)(kFzLead + i * kFzPitch + (j == 1 ? L + 1 : 0)) * 16u;
#pragma unroll
            for (int c = 0; c < 4; ++c) {
              const uint4 val = reinterpret_cast<const uint4 *>(o)[c];
              *reinterpret_cast<uint4 *>(smem + out_off + c * out_lbo + p0) = val;
              if (ghost) *reinterpret_cast<uint4 *>(smem + out_off + c * out_lbo + pg) = val;
            }
          }
          // this warp's rows of the tile are written: visible to the MMA (async proxy)
          asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
          __syncwarp();
          if (lane == 0)
            asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(
                             smem_u32(&tile_done[layer * kFzTilesMax + t]))
                         : "memory");
        }
      }
    }
    my_base += 26;  // tiles per band (8 + 7 + 6 + 5)
    __syncthreads();
    // pooled sums of the band's 8 rows of a4 (buffer B): thread (row, channel)
    if (tid < kFzRows * kC) {
      const int c = tid & (kC - 1), i = tid >> 5;
      const unsigned char *src = smem + kFzBufB + (c >> 3) * (kFzPosB * 16) +
                                 (kFzLead + i * kFzPitch + 1) * 16 + (c & 7) * 2;
      float sum = 0.f;
#pragma unroll 8
      for (int x = 0; x < L; ++x)
        sum += __bfloat162float(*reinterpret_cast<const __nv_bfloat16 *>(src + x * 16));
      atomicAdd(&spool[c], sum);
    }
    __syncthreads();
    if (tid < kC && !*abort_flag) atomicAdd(&a.pool[img * kC + tid], spool[tid]);
  }
  if (tid == 0 && *abort_flag && a.err) atomicExch(a.err, 1);
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr),
                 "r"(32 * kFzGroups)
                 : "memory");
  }
}

size_t conv_win_smem(int L, bool pool) {
  const size_t W = (size_t)kTileM + 2 * (size_t)L;
  return 3 * 4 * W * 16 + (size_t)kC * 9 * kC * 2 + 64 + (pool ? (size_t)kTileM * 33 * 4 : 0);
}

size_t conv_smem(int mode) {
  const int K = mode == kTab1 ? 16 : 9 * kC;
  return (size_t)kTileM * K * 2 + (size_t)kC * K * 2 + 64 + (size_t)kTileM * 33 * 4;
}

// FP32 weight gradient of a 32->32 layer for L other than 32, 64, 128 (the
// tcgen05 kernel k_conv_dw_win takes those), register-tiled: dW[co][k] +=
// sum_p dZ[p][co] * X[p, k] (k = tap*32 + ci, X the layer input at the tap's
// neighbour).  A block takes chunks of 32 pixels; thread t accumulates the 4
// output channels 4*(t/32).. and the 9 k values (t%32) + 32*j, so each pixel
// costs it 13 shared-memory loads for 36 FMAs (broadcast dZ, conflict-free X).
// The neighbour rows are gathered with 16-byte loads.  Partial sums go to dW
// with one atomicAdd per value and block.
__global__ void __launch_bounds__(256) k_conv_dw32(int L, int B, const __nv_bfloat16 *dz,
                                                   const __nv_bfloat16 *xin, float *dW,
                                                   float *db) {
  constexpr int K = 9 * kC;  // 288
  constexpr int P = 32;      // pixels per chunk
  __shared__ __align__(16) float s_x[P][K];
  __shared__ __align__(16) float s_dz[P][kC];
  const int N = L * L;
  const int tid = threadIdx.x;
  const int cog = (tid >> 5) * 4;  // first of this thread's 4 output channels
  const int kg = tid & 31;         // this thread's k values: kg + 32 j
  float acc[4][9];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 9; ++j) acc[i][j] = 0.f;
  float accb[4] = {0.f, 0.f, 0.f, 0.f};
  const long long nchunks = (long long)B * N / P;
  for (long long ch = blockIdx.x; ch < nchunks; ch += gridDim.x) {
    const long long pix0 = ch * P;
    const int img = (int)(pix0 / N);
    const int p0 = (int)(pix0 % N);
    // dZ rows: 32 pixels x 32 channels = 128 chunks of 8 bf16
    if (tid < P * 4) {
      const int r = tid >> 2, c8 = (tid & 3) * 8;
      const uint4 v = *reinterpret_cast<const uint4 *>(dz + ((size_t)img * N + p0 + r) * kC + c8);
      const __nv_bfloat16 *h = reinterpret_cast<const __nv_bfloat16 *>(&v);
#pragma unroll
      for (int e = 0; e < 8; ++e) s_dz[r][c8 + e] = __bfloat162float(h[e]);
    }
    // X at the 9 neighbours: 32 pixels x 9 taps x 4 chunks of 8 bf16
    for (int i = tid; i < P * 9 * 4; i += blockDim.x) {
      const int r = i / 36, rem = i - r * 36, tap = rem >> 2, c8 = (rem & 3) * 8;
      const int q = nbr(p0 + r, tap, L);
      const uint4 v = *reinterpret_cast<const uint4 *>(xin + ((size_t)img * N + q) * kC + c8);
      const __nv_bfloat16 *h = reinterpret_cast<const __nv_bfloat16 *>(&v);
      float4 lo, hi;
      lo.x = __bfloat162float(h[0]); lo.y = __bfloat162float(h[1]);
      lo.z = __bfloat162float(h[2]); lo.w = __bfloat162float(h[3]);
      hi.x = __bfloat162float(h[4]); hi.y = __bfloat162float(h[5]);
      hi.z = __bfloat162float(h[6]); hi.w = __bfloat162float(h[7]);
      *reinterpret_cast<float4 *>(&s_x[r][tap * kC + c8]) = lo;
      *reinterpret_cast<float4 *>(&s_x[r][tap * kC + c8 + 4]) = hi;
    }
    __syncthreads();
#pragma unroll 2
    for (int r = 0; r < P; ++r) {
      const float4 g = *reinterpret_cast<const float4 *>(&s_dz[r][cog]);
      float xv[9];
#pragma unroll
      for (int j = 0; j < 9; ++j) xv[j] = s_x[r][kg + 32 * j];
#pragma unroll
      for (int j = 0; j < 9; ++j) {
        acc[0][j] = fmaf(g.x, xv[j], acc[0][j]);
        acc[1][j] = fmaf(g.y, xv[j], acc[1][j]);
        acc[2][j] = fmaf(g.z, xv[j], acc[2][j]);
        acc[3][j] = fmaf(g.w, xv[j], acc[3][j]);
      }
      if (kg == 0) {
        accb[0] += g.x; accb[1] += g.y; accb[2] += g.z; accb[3] += g.w;
      }
    }
    __syncthreads();
  }
#pragma unroll
  for (int i = 0; i < 4; ++i) {
#pragma unroll
    for (int j = 0; j < 9; ++j) atomicAdd(&dW[(cog + i) * K + kg + 32 * j], acc[i][j]);
    if (kg == 0) atomicAdd(&db[cog + i], accb[i]);
  }
}

// ---------------------------------------------------------------------------
// Weight gradients on tcgen05.  dW[co][k] = sum_p dZ[p][co] * X[p][k] is a GEMM
// whose reduction runs over every pixel of the batch: D[m][n] = sum_k A[m][k]
// B[n][k] with k = pixel, n = co (N = 32) and m = the layer-input value a tap
// reads.  Both operands are MN-major in shared memory (no swizzle): a core
// matrix is 8 pixels (K) x 8 values (MN) = 8 rows of 16 bytes, 8-pixel groups
// 128 B apart (LBO), 8-value groups SBO apart.  dZ is staged [co chunk][pixel]
// [16 B] (SBO 2 KB).  FP32 accumulation in TMEM over all of a CTA's tiles;
// each CTA adds its partial sums to dW and db (one atomicAdd per value).
// ---------------------------------------------------------------------------
// Instruction descriptor: D F32, A/B BF16, both MN-major, N=32, M=128.
constexpr uint32_t kIdescMN = kIdesc | (1u << 15) | (1u << 16);

__device__ __forceinline__ void umma_bf16_mn(uint32_t tmem_d, uint64_t da, uint64_t db,
                                             uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem_d),
      "l"(da), "l"(db), "r"(kIdescMN), "r"(accumulate));
}

struct DwArgs {
  int L;
  const __nv_bfloat16 *x;   // layer input activations [B][N][32] (32->32 layers)
  const int8_t *spins;      // layer 1: the input grids [B][N]
  const __nv_bfloat16 *dz;  // this layer's output gradient (after the ReLU mask) [B][N][32]
  float *dW, *db;           // gradients, added to
  int *err;                 // set on a timed-out wait
  int ntiles;               // images * (L*L / 128)
};

// 32->32 layers, L = LT in {32, 64, 128}.  The A operand is the input window
// of k_conv_win: the tile's rows and one row above and below (W = 128 + 2L
// pixels), staged as copies rotated by dx = -1, 0, +1 within each image row,
// [copy][channel chunk][pixel][16 B]; read with pixels along K and channels
// along M, copy v's four channel chunks are M rows 32v..32v+31 (SBO = W*16,
// the chunk stride; copies follow one another at 4*W*16).  A fourth copy holds
// ones, so M rows 96..127 accumulate sum_p dZ[p][co] = db.  A tap's row offset
// dy is a start offset of (dy+1)*L pixels along K, and each dy has its own
// accumulator (TMEM columns 32*(dy+1)): per 128-pixel tile 3 x 8 MMAs of
// M=128, N=32, K=16 (the ones rows repeated for dy = 0, +1 are not used).
// The next tile's window and dZ rows are loaded into registers while the
// current tile's MMAs run.
template <int LT>
__global__ void __launch_bounds__(128) k_conv_dw_win(DwArgs a) {
  static_assert(LT == 32 || LT == 64 || LT == 128, "whole image rows per tile");
  constexpr int L = LT, N = L * L;
  constexpr int W = kTileM + 2 * L;             // window pixels
  constexpr uint32_t lbo = (uint32_t)W * 16;    // bytes between channel chunks
  constexpr uint32_t vstride = 4u * lbo;        // bytes between rotated copies
  constexpr int tiles_per_img = N / kTileM;
  extern __shared__ __align__(1024) unsigned char smem[];
  unsigned char *sA = smem;                      // [4][4][W][16 B]; copy 3 = ones
  unsigned char *sB = smem + 4 * vstride;        // dZ: [4][128][16 B]
  uint64_t *mbar = reinterpret_cast<uint64_t *>(sB + 4 * kTileM * 16);
  uint32_t *tslot = reinterpret_cast<uint32_t *>(mbar + 1);
  const int tid = threadIdx.x, warp = tid >> 5;

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(tslot)),
                 "r"(128)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (tid == 0) {
    mbar_init(smem_u32(mbar), 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  {
    const uint4 ones = make_uint4(0x3F803F80u, 0x3F803F80u, 0x3F803F80u, 0x3F803F80u);
    for (int i = tid; i < 4 * W; i += blockDim.x)
      *reinterpret_cast<uint4 *>(sA + 3 * vstride + (uint32_t)i * 16) = ones;
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t taddr = *tslot;

  constexpr int kPerW = W * 4 / 128;  // 16-byte window chunks per thread
  uint4 v4[kPerW];
  uint4 g4[4];
  auto load_tile = [&](int t) {
    const int timg = t / tiles_per_img;
    const int y0 = ((t % tiles_per_img) * kTileM) / L;  // first output row of the tile
    const __nv_bfloat16 *xs = a.x + (size_t)timg * N * kC;
#pragma unroll
    for (int j = 0; j < kPerW; ++j) {
      const int c = (tid & 31) >> 3, w = j * 32 + (tid >> 5) * 8 + (tid & 7);
      int row = y0 - 1 + w / L;
      row = row < 0 ? row + L : (row >= L ? row - L : row);
      v4[j] = *reinterpret_cast<const uint4 *>(xs + ((size_t)row * L + (w % L)) * kC + 8 * c);
    }
    const uint4 *gz = reinterpret_cast<const uint4 *>(
        a.dz + ((size_t)timg * N + (size_t)(t % tiles_per_img) * kTileM + tid) * kC);
#pragma unroll
    for (int c = 0; c < 4; ++c) g4[c] = gz[c];
  };
  if ((int)blockIdx.x < a.ntiles) load_tile(blockIdx.x);

  uint32_t phase = 0;
  bool first = true, ok = true;
  for (int tile = blockIdx.x; tile < a.ntiles; tile += gridDim.x) {
    if (!first) {  // the previous tile's MMAs still read the shared operands
      bool waited = true;
      if (tid == 0) waited = mbar_wait(smem_u32(mbar), phase);
      ok = __syncthreads_and(waited ? 1 : 0) != 0;
      phase ^= 1u;
      if (!ok) break;
    }
#pragma unroll
    for (int j = 0; j < kPerW; ++j) {
      const int c = (tid & 31) >> 3, w = j * 32 + (tid >> 5) * 8 + (tid & 7);
      const int col = w % L, rbase = w - col;
#pragma unroll
      for (int v = 0; v < 3; ++v) {  // copy v holds, at column col', input column col' + v - 1
        const int cd = (col - (v - 1) + L) % L;
        *reinterpret_cast<uint4 *>(sA + v * vstride + c * lbo + (uint32_t)(rbase + cd) * 16) =
            v4[j];
      }
    }
#pragma unroll
    for (int c = 0; c < 4; ++c)
      *reinterpret_cast<uint4 *>(sB + c * (kTileM * 16) + tid * 16) = g4[c];
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (tid == 0) {
      const uint32_t a0 = smem_u32(sA), b0 = smem_u32(sB);
#pragma unroll
      for (int dy = 0; dy < 3; ++dy) {
#pragma unroll
        for (int s = 0; s < kTileM / 16; ++s)
          umma_bf16_mn(taddr + (uint32_t)(dy * 32),
                       umma_desc(a0 + (uint32_t)(dy * L + 16 * s) * 16, 128, lbo),
                       umma_desc(b0 + (uint32_t)s * 256, 128, kTileM * 16),
                       (first && s == 0) ? 0u : 1u);
      }
      umma_commit(smem_u32(mbar));
    }
    first = false;
    const int nt = tile + (int)gridDim.x;
    if (nt < a.ntiles) load_tile(nt);
  }
  if (!first && ok) {  // the last tile's MMAs, then this CTA's sums
    bool waited = true;
    if (tid == 0) waited = mbar_wait(smem_u32(mbar), phase);
    ok = __syncthreads_and(waited ? 1 : 0) != 0;
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (ok) {
      const int lane = tid & 31;
#pragma unroll 1
      for (int dy = 0; dy < 3; ++dy) {
        float acc[32];
        tmem_ld32(taddr + ((uint32_t)(warp * 32) << 16) + (uint32_t)(dy * 32), acc);
        if (warp < 3) {  // copy v = warp: tap (dy, dx = v - 1), ci = lane
          const int k = (dy * 3 + warp) * kC + lane;
#pragma unroll
          for (int co = 0; co < kC; ++co) atomicAdd(&a.dW[co * 9 * kC + k], acc[co]);
        } else if (dy == 0 && lane == 0) {  // a row of ones: sum_p dZ[p][co]
#pragma unroll
          for (int co = 0; co < kC; ++co) atomicAdd(&a.db[co], acc[co]);
        }
      }
    }
  }
  if (!ok && tid == 0 && a.err) atomicExch(a.err, 1);
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(128)
                 : "memory");
  }
}

constexpr size_t dw_win_smem(int L) {
  return 4 * 4 * ((size_t)kTileM + 2 * (size_t)L) * 16 + 4 * (size_t)kTileM * 16 + 64;
}

// Layer 1 (one input channel, 9 taps): A rows are the taps, staged per pixel
// as two 16-byte MN groups (taps 0-7; tap 8 and seven zeros), then a group of
// ones (rows 16..23: db) and thirteen zero groups to fill M = 128 (SBO 2 KB:
// [group][pixel][16 B]).  One accumulator; 8 MMAs per 128-pixel tile.
__global__ void __launch_bounds__(128) k_conv_dw1_tc(DwArgs a) {
  constexpr int kGroups = 16;
  constexpr uint32_t sbo = kTileM * 16;  // 2 KB
  extern __shared__ __align__(1024) unsigned char smem[];
  unsigned char *sA = smem;                           // [16][128][16 B]
  unsigned char *sB = smem + kGroups * sbo;           // dZ: [4][128][16 B]
  uint64_t *mbar = reinterpret_cast<uint64_t *>(sB + 4 * sbo);
  uint32_t *tslot = reinterpret_cast<uint32_t *>(mbar + 1);
  const int L = a.L, N = L * L;
  const int tiles_per_img = N / kTileM;
  const int tid = threadIdx.x, warp = tid >> 5;

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(tslot)),
                 "r"(32)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (tid == 0) {
    mbar_init(smem_u32(mbar), 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  {
    const uint4 ones = make_uint4(0x3F803F80u, 0x3F803F80u, 0x3F803F80u, 0x3F803F80u);
    const uint4 zero = make_uint4(0u, 0u, 0u, 0u);
    for (int i = tid; i < (kGroups - 2) * kTileM; i += blockDim.x)
      *reinterpret_cast<uint4 *>(sA + 2 * sbo + (uint32_t)i * 16) = i < kTileM ? ones : zero;
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t taddr = *tslot;

  uint32_t phase = 0;
  bool first = true, ok = true;
  for (int tile = blockIdx.x; tile < a.ntiles; tile += gridDim.x) {
    const int img = tile / tiles_per_img;
    const int p = (tile % tiles_per_img) * kTileM + tid;
    const int8_t *sp = a.spins + (size_t)img * N;
    __align__(16) __nv_bfloat16 v[16];
#pragma unroll
    for (int k = 0; k < 16; ++k) v[k] = __float2bfloat16_rn(k < 9 ? (float)sp[nbr(p, k, L)] : 0.0f);
    const uint4 *gz = reinterpret_cast<const uint4 *>(a.dz + ((size_t)img * N + p) * kC);
    uint4 g4[4];
#pragma unroll
    for (int c = 0; c < 4; ++c) g4[c] = gz[c];
    if (!first) {
      bool waited = true;
      if (tid == 0) waited = mbar_wait(smem_u32(mbar), phase);
      ok = __syncthreads_and(waited ? 1 : 0) != 0;
      phase ^= 1u;
      if (!ok) break;
    }
    *reinterpret_cast<uint4 *>(sA + tid * 16) = *reinterpret_cast<const uint4 *>(&v[0]);
    *reinterpret_cast<uint4 *>(sA + sbo + tid * 16) = *reinterpret_cast<const uint4 *>(&v[8]);
#pragma unroll
    for (int c = 0; c < 4; ++c) *reinterpret_cast<uint4 *>(sB + c * sbo + tid * 16) = g4[c];
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (tid == 0) {
      const uint32_t a0 = smem_u32(sA), b0 = smem_u32(sB);
#pragma unroll
      for (int s = 0; s < kTileM / 16; ++s)
        umma_bf16_mn(taddr, umma_desc(a0 + (uint32_t)s * 256, 128, sbo),
                     umma_desc(b0 + (uint32_t)s * 256, 128, sbo), (first && s == 0) ? 0u : 1u);
      umma_commit(smem_u32(mbar));
    }
    first = false;
  }
  if (!first && ok) {
    bool waited = true;
    if (tid == 0) waited = mbar_wait(smem_u32(mbar), phase);
    ok = __syncthreads_and(waited ? 1 : 0) != 0;
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (ok && warp == 0) {  // rows 0..8: taps; row 16: ones
      const int lane = tid & 31;
      float acc[32];
      tmem_ld32(taddr, acc);
      if (lane < 9) {
#pragma unroll
        for (int co = 0; co < kC; ++co) atomicAdd(&a.dW[co * 9 + lane], acc[co]);
      } else if (lane == 16) {
#pragma unroll
        for (int co = 0; co < kC; ++co) atomicAdd(&a.db[co], acc[co]);
      }
    }
  }
  if (!ok && tid == 0 && a.err) atomicExch(a.err, 1);
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(32)
                 : "memory");
  }
}

constexpr size_t kDw1Smem = 16 * (size_t)kTileM * 16 + 4 * (size_t)kTileM * 16 + 64;

// Head: mean pool -> linear -> sigmoid -> cross-entropy; one warp per image,
// lane = channel.  Writes q, adds the mean loss, the head's gradients and
// dmean[b][c] = dL/d(pooled mean).
// Magnetisation of int8 +-1 grids, one warp per grid: 16-byte loads summed
// four bytes at a time with __dp4a; (float)sum / (float)N as the sweep
// kernels compute it (the sum is exact).  N is a multiple of 128.
__global__ void k_spin_mag(const int8_t *spins, int N, int batch, float *mag) {
  const int g = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  if (g >= batch) return;
  const int4 *src = reinterpret_cast<const int4 *>(spins + (size_t)g * N);
  int acc = 0;
  for (int i = lane; i < N / 16; i += 32) {
    const int4 v = src[i];
    acc = __dp4a(v.x, 0x01010101, acc);
    acc = __dp4a(v.y, 0x01010101, acc);
    acc = __dp4a(v.z, 0x01010101, acc);
    acc = __dp4a(v.w, 0x01010101, acc);
  }
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  if (lane == 0) mag[g] = (float)acc / (float)N;
}

__global__ void k_head(int B, int N, const float *pool, const float *params, const float *labels,
                       float *q_out, float *loss, float *grad, float *dmean) {
  const int b = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  const int c = threadIdx.x & 31;
  if (b >= B) return;
  const float m = pool[b * kC + c] / (float)N;
  float z = m * params[kOffWf + c];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) z += __shfl_xor_sync(0xffffffffu, z, o);
  z += params[kOffBf];
  const float q = 1.0f / (1.0f + expf(-z));
  if (q_out && c == 0) q_out[b] = q;
  if (labels) {
    const float y = labels[b];
    const float dz = (q - y) / (float)B;
    if (c == 0) {
      const float qc = fminf(fmaxf(q, 1e-7f), 1.0f - 1e-7f);
      atomicAdd(loss, -(y * logf(qc) + (1.0f - y) * logf(1.0f - qc)) / (float)B);
      atomicAdd(&grad[kOffBf], dz);
    }
    atomicAdd(&grad[kOffWf + c], dz * m);
    dmean[b * kC + c] = dz * params[kOffWf + c];
  }
}

// dZ4 = dmean / N on every pixel where the layer-4 activation is positive.
// One thread per 8 channels of a pixel (16-byte loads and stores); grid x
// over 256-chunk blocks of one image, y over images (strided when the batch
// exceeds gridDim.y).  A block divides its image's 32 dmean values once, in
// shared memory (the same division per value as per pixel, so the same
// bytes, for 32 divisions a block instead of 8 a thread).
__global__ void __launch_bounds__(256) k_dz4(int B, int N, const float *dmean,
                                             const __nv_bfloat16 *a4, __nv_bfloat16 *dz4) {
  __shared__ float q[kC];
  const int i = blockIdx.x * blockDim.x + threadIdx.x;  // chunk within the image
  const int c0 = (threadIdx.x & (kC / 8 - 1)) * 8;
  for (int b = blockIdx.y; b < B; b += gridDim.y) {
    __syncthreads();  // the previous image's quotients are no longer read
    if (threadIdx.x < kC) q[threadIdx.x] = dmean[(size_t)b * kC + threadIdx.x] / (float)N;
    __syncthreads();
    if (i < N * (kC / 8)) {
      const size_t at = (size_t)b * N * (kC / 8) + i;
      const uint4 av = reinterpret_cast<const uint4 *>(a4)[at];
      const __nv_bfloat16 *ah = reinterpret_cast<const __nv_bfloat16 *>(&av);
      __align__(16) __nv_bfloat16 o[8];
#pragma unroll
      for (int e = 0; e < 8; ++e)
        o[e] = __float2bfloat16_rn(__bfloat162float(ah[e]) > 0.0f ? q[c0 + e] : 0.0f);
      reinterpret_cast<uint4 *>(dz4)[at] = *reinterpret_cast<const uint4 *>(o);
    }
  }
}

// BF16 copies of the weights: W1 [32][16] (taps padded), W2..4 [32][288]
// (k = tap*32 + ci) and their transposes WT [ci][tap*32 + co].
__global__ void k_pack_weights(const float *params, __nv_bfloat16 *w1, __nv_bfloat16 *w,
                               __nv_bfloat16 *wt) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < kC * 16) {
    const int co = i / 16, k = i % 16;
    w1[i] = __float2bfloat16_rn(k < 9 ? params[kOffW1 + co * 9 + k] : 0.0f);
  }
  if (i < 3 * 9216) {
    const int l = i / 9216, r = i % 9216;
    const int co = r / 288, k = r % 288, tap = k / kC, ci = k % kC;
    const float v = params[kOffW2 + l * (9216 + 32) + r];
    w[i] = __float2bfloat16_rn(v);
    wt[l * 9216 + ci * 288 + tap * kC + co] = __float2bfloat16_rn(v);
  }
}

__global__ void k_adam(float *params, const float *grad, float *m, float *v, int n, float lr,
                       float b1, float b2, float eps, float c1, float c2) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float g = grad[i];
  const float mi = b1 * m[i] + (1.0f - b1) * g;
  const float vi = b2 * v[i] + (1.0f - b2) * g * g;
  m[i] = mi;
  v[i] = vi;
  params[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
}

}  // namespace
}  // namespace gasp

using namespace gasp;

struct gasp_cnn {
  int device, L, N, max_batch;
  float *d_params, *d_grad, *d_m, *d_v;
  __nv_bfloat16 *d_w1, *d_w, *d_wt;
  int8_t *d_spins;
  float *d_labels, *d_q, *d_pool, *d_dmean, *d_loss;
  float *d_mag;             // magnetisation of each predicted grid
  // chunked prediction (batches above max_batch): a second input buffer and
  // a copy stream, so the next chunk's upload overlaps this chunk's network
  int8_t *d_spins2;
  cudaStream_t copy_stream;
  cudaEvent_t ev_copied[2], ev_used[2];
  __nv_bfloat16 *d_act[4];  // a1..a4
  __nv_bfloat16 *d_tab;     // first-layer activations by neighbourhood pattern [512][32]
  __nv_bfloat16 *d_dz[2];   // ping-pong data gradients
  int *d_err;
  int adam_t;
  int fused;  // inference through k_cnn_fused64 (L = 64); gasp_cnn_set_fused, default off
};

namespace {

int cnn_upload(gasp_cnn *c, const int8_t *spins, const float *labels, int batch) {
  cudaStream_t s = current_stream();
  GASP_CUDA(cudaMemcpyAsync(c->d_spins, spins, (size_t)batch * c->N, cudaMemcpyHostToDevice, s));
  if (labels)
    GASP_CUDA(cudaMemcpyAsync(c->d_labels, labels, (size_t)batch * sizeof(float),
                              cudaMemcpyHostToDevice, s));
  return GASP_OK;
}

// Persistent launch of a convolution kernel: the grid is sized so that all
// of its CTAs are resident at once and share the tiles evenly.  CTAs per SM
// are bounded by shared memory (1 KiB reserved per CTA), registers, and TMEM
// (512 columns, 32 per CTA).
template <typename Kern>
int launch_persistent(Kern kern, size_t smem_max, size_t smem, const ConvArgs &b, cudaStream_t s,
                      int tmem_cols = 32) {
  GASP_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_max));
  int dev = 0, nsm = 0, smem_sm = 0;
  GASP_CUDA(cudaGetDevice(&dev));
  GASP_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
  GASP_CUDA(cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev));
  int per_sm = smem_sm / (int)(smem + 1024);
  cudaFuncAttributes fa;
  GASP_CUDA(cudaFuncGetAttributes(&fa, kern));
  const int by_regs = fa.numRegs > 0 ? 65536 / (fa.numRegs * 128) : 16;
  if (per_sm > by_regs) per_sm = by_regs;
  if (per_sm > 16) per_sm = 16;  // 2048 threads per SM
  // every resident CTA holds its TMEM columns until it exits (512 per SM)
  if (per_sm > 512 / tmem_cols) per_sm = 512 / tmem_cols;
  if (per_sm < 1) per_sm = 1;
  const int grid = b.ntiles < nsm * per_sm ? b.ntiles : nsm * per_sm;
  kern<<<grid, 128, smem, s>>>(b);
  GASP_CUDA(cudaGetLastError());
  return GASP_OK;
}

// Persistent launch of a weight-gradient kernel: all CTAs resident, at most
// 512 / tmem_cols per SM (TMEM), bounded by shared memory and registers.
template <typename Kern>
int launch_dw(Kern kern, size_t smem, int tmem_cols, const DwArgs &b, cudaStream_t s) {
  GASP_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  int dev = 0, nsm = 0, smem_sm = 0;
  GASP_CUDA(cudaGetDevice(&dev));
  GASP_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
  GASP_CUDA(cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev));
  int per_sm = smem_sm / (int)(smem + 1024);
  cudaFuncAttributes fa;
  GASP_CUDA(cudaFuncGetAttributes(&fa, kern));
  const int by_regs = fa.numRegs > 0 ? 65536 / (fa.numRegs * 128) : 16;
  if (per_sm > by_regs) per_sm = by_regs;
  if (per_sm > 512 / tmem_cols) per_sm = 512 / tmem_cols;
  if (per_sm < 1) per_sm = 1;
  const int grid = b.ntiles < nsm * per_sm ? b.ntiles : nsm * per_sm;
  kern<<<grid, 128, smem, s>>>(b);
  GASP_CUDA(cudaGetLastError());
  return GASP_OK;
}

// The ghost-column forward kernel at L = 64 (GASP_CNN_WINDOW_COPIES=3 selects
// k_conv_win's three rotated copies instead, for comparisons).  The data
// gradient keeps k_conv_win: the same ghost-column form of it gave the same
// bytes but measured 2 % slower (287 against 281 us per 1024-image layer).
bool conv_gh64_enabled() {
  static const bool on = [] {
    const char *e = getenv("GASP_CNN_WINDOW_COPIES");
    return !(e && e[0] == '3');
  }();
  return on;
}

// Largest shared-memory footprint the window kernel is used with.
constexpr size_t kWinSmemLimit = 110 * 1024;

template <int MODE>
int launch_conv(const ConvArgs &a, int batch, cudaStream_t s) {
  ConvArgs b = a;
  b.ntiles = batch * (a.L * a.L / kTileM);
  if constexpr (MODE == kFwd) {
    if (a.L == 64 && conv_gh64_enabled()) {  // one staged window copy (ghost columns)
      b.ntiles = batch * kGhTiles;
      return launch_persistent(k_conv_gh64, conv_gh64_smem(true), conv_gh64_smem(a.pool != nullptr),
                               b, s, 64);
    }
  }
  const size_t win_max = conv_win_smem(a.L, MODE == kFwd);
  if (win_max <= kWinSmemLimit) {
    const size_t sm = conv_win_smem(a.L, a.pool != nullptr);
    switch (a.L) {
      case 32: return launch_persistent(k_conv_win<MODE, 32>, win_max, sm, b, s);
      case 64: return launch_persistent(k_conv_win<MODE, 64>, win_max, sm, b, s);
      case 128: return launch_persistent(k_conv_win<MODE, 128>, win_max, sm, b, s);
      default: return launch_persistent(k_conv_win<MODE, 0>, win_max, sm, b, s);
    }
  }
  const size_t smem_max = conv_smem(MODE);
  // the pooling scratch at the end is only touched by the layer that pools
  const size_t smem = a.pool ? smem_max : smem_max - (size_t)kTileM * 33 * 4;
  return launch_persistent(k_conv_tc<MODE>, smem_max, smem, b, s);
}

// The first layer: its 512-row activation table (four tiles of k_conv_tc on
// the neighbourhood patterns), then one table row per pixel.
int launch_conv1(const ConvArgs &a, __nv_bfloat16 *tab, int batch, cudaStream_t s) {
  ConvArgs t = a;
  t.y = tab;
  t.pool = nullptr;
  t.ntiles = kNPatterns / kTileM;
  const size_t smem_max = conv_smem(kTab1);
  int rc = launch_persistent(k_conv_tc<kTab1>, smem_max, smem_max - (size_t)kTileM * 33 * 4, t,
                             s);
  if (rc) return rc;
  const int N = a.L * a.L;
  const dim3 grid((unsigned)((N + 255) / 256), (unsigned)(batch < 65535 ? batch : 65535));
  k_conv1_lookup<<<grid, 256, 0, s>>>(a.spins, tab, a.y, a.L, batch);
  GASP_CUDA(cudaGetLastError());
  return GASP_OK;
}

// keep_last: store the last layer's activations (training's ReLU mask); the
// prediction path only needs their pooled sums.
int cnn_forward(gasp_cnn *c, int batch, cudaStream_t s, const int8_t *spins = nullptr,
                bool keep_last = true) {
  int rc;
  const int B = batch;
  k_pack_weights<<<(3 * 9216 + 255) / 256, 256, 0, s>>>(c->d_params, c->d_w1, c->d_w, c->d_wt);
  GASP_CUDA(cudaGetLastError());
  GASP_CUDA(cudaMemsetAsync(c->d_pool, 0, (size_t)B * kC * sizeof(float), s));
  ConvArgs a;
  memset(&a, 0, sizeof a);
  a.L = c->L;
  a.err = c->d_err;
  a.spins = spins ? spins : c->d_spins;
  a.w = c->d_w1;
  a.bias = c->d_params + kOffB1;
  a.y = c->d_act[0];
  if ((rc = launch_conv1(a, c->d_tab, B, s))) return rc;
  for (int l = 0; l < 3; ++l) {
    a.x = c->d_act[l];
    a.w = c->d_w + l * 9216;
    a.bias = c->d_params + kOffB2 + l * (9216 + 32);
    a.y = (l == 2 && !keep_last) ? nullptr : c->d_act[l + 1];
    a.pool = (l == 2) ? c->d_pool : nullptr;
    if ((rc = launch_conv<kFwd>(a, B, s))) return rc;
  }
  return GASP_OK;
}

// Inference forward (pooled sums in d_pool): the fused whole-network kernel
// for L = 64 when switched on, the layer-by-layer kernels otherwise.
int cnn_infer(gasp_cnn *c, int batch, cudaStream_t s, const int8_t *spins = nullptr) {
  if (c->L != 64 || !c->fused) return cnn_forward(c, batch, s, spins, false);
  k_pack_weights<<<(3 * 9216 + 255) / 256, 256, 0, s>>>(c->d_params, c->d_w1, c->d_w, c->d_wt);
  GASP_CUDA(cudaGetLastError());
  GASP_CUDA(cudaMemsetAsync(c->d_pool, 0, (size_t)batch * kC * sizeof(float), s));
  FusedArgs f;
  f.spins = spins ? spins : c->d_spins;
  f.w1 = c->d_w1;
  f.w = c->d_w;
  f.params = c->d_params;
  f.pool = c->d_pool;
  f.err = c->d_err;
  f.nbands = batch * (64 / kFzRows);
  GASP_CUDA(cudaFuncSetAttribute(k_cnn_fused64, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)kFzSmem));
  int dev = 0, nsm = 0;
  GASP_CUDA(cudaGetDevice(&dev));
  GASP_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
  const int grid = f.nbands < nsm ? f.nbands : nsm;  // one CTA per SM, persistent
  k_cnn_fused64<<<grid, kFzThreads, kFzSmem, s>>>(f);
  GASP_CUDA(cudaGetLastError());
  return GASP_OK;
}

int cnn_check_err(gasp_cnn *c, cudaStream_t s) {
  int err = 0;
  GASP_CUDA(cudaMemcpyAsync(&err, c->d_err, sizeof(int), cudaMemcpyDeviceToHost, s));
  GASP_CUDA(cudaStreamSynchronize(s));
  if (err) {
    set_error("tensor-core wait timed out");
    return GASP_ERR_TIMEOUT;
  }
  return GASP_OK;
}

// Prediction of more grids than one batch holds: chunks of max_batch through
// two input buffers.  The copy stream uploads chunk i+1 (after the network of
// chunk i-1 has read that buffer) while the current stream runs chunk i, so
// the host-to-device copies hide behind the convolutions.
int predict_chunked(gasp_cnn *c, const int8_t *spins, int batch, float *q_out, float *mag_out,
                    cudaStream_t s) {
  if (!c->copy_stream) {  // first chunked call: all four pieces, or none of them
    int8_t *buf = nullptr;
    cudaStream_t cs = nullptr;
    cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
    cudaError_t e = cudaMalloc(&buf, (size_t)c->max_batch * c->N);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking);
    for (int i = 0; i < 4 && e == cudaSuccess; ++i)
      e = cudaEventCreateWithFlags(&ev[i], cudaEventDisableTiming);
    if (e != cudaSuccess) {
      for (cudaEvent_t x : ev)
        if (x) cudaEventDestroy(x);
      if (cs) cudaStreamDestroy(cs);
      cudaFree(buf);
      return cuda_fail(e, "gasp_cnn_predict_ex chunk buffers", __FILE__, __LINE__);
    }
    c->d_spins2 = buf;
    c->ev_copied[0] = ev[0];
    c->ev_copied[1] = ev[1];
    c->ev_used[0] = ev[2];
    c->ev_used[1] = ev[3];
    c->copy_stream = cs;
  }
  cudaStream_t cs = c->copy_stream;
  int8_t *buf[2] = {c->d_spins, c->d_spins2};
  const int mb = c->max_batch;
  const int nch = (batch + mb - 1) / mb;
  auto rows = [&](int i) { return batch - i * mb < mb ? batch - i * mb : mb; };
  // earlier work on s may still read either buffer
  for (int b = 0; b < 2; ++b) GASP_CUDA(cudaEventRecord(c->ev_used[b], s));
  GASP_CUDA(cudaStreamWaitEvent(cs, c->ev_used[0], 0));
  GASP_CUDA(cudaMemcpyAsync(buf[0], spins, (size_t)rows(0) * c->N, cudaMemcpyHostToDevice, cs));
  GASP_CUDA(cudaEventRecord(c->ev_copied[0], cs));
  int rc;
  for (int i = 0; i < nch; ++i) {
    const int b = i & 1, n = rows(i);
    GASP_CUDA(cudaStreamWaitEvent(s, c->ev_copied[b], 0));
    if ((rc = cnn_infer(c, n, s, buf[b]))) return rc;
    k_head<<<(n + 7) / 8, 256, 0, s>>>(n, c->N, c->d_pool, c->d_params, nullptr, c->d_q, nullptr,
                                       nullptr, nullptr);
    GASP_CUDA(cudaGetLastError());
    if (mag_out) {
      k_spin_mag<<<(n + 7) / 8, 256, 0, s>>>(buf[b], c->N, n, c->d_mag);
      GASP_CUDA(cudaGetLastError());
    }
    GASP_CUDA(cudaEventRecord(c->ev_used[b], s));
    if (i + 1 < nch) {
      const int nb = (i + 1) & 1;
      GASP_CUDA(cudaStreamWaitEvent(cs, c->ev_used[nb], 0));
      GASP_CUDA(cudaMemcpyAsync(buf[nb], spins + (size_t)(i + 1) * mb * c->N,
                                (size_t)rows(i + 1) * c->N, cudaMemcpyHostToDevice, cs));
      GASP_CUDA(cudaEventRecord(c->ev_copied[nb], cs));
    }
    GASP_CUDA(cudaMemcpyAsync(q_out + (size_t)i * mb, c->d_q, (size_t)n * sizeof(float),
                              cudaMemcpyDeviceToHost, s));
    if (mag_out)
      GASP_CUDA(cudaMemcpyAsync(mag_out + (size_t)i * mb, c->d_mag, (size_t)n * sizeof(float),
                                cudaMemcpyDeviceToHost, s));
  }
  return cnn_check_err(c, s);
}

// Forward + loss + all gradients (into d_grad) for the uploaded batch.
int cnn_backward(gasp_cnn *c, int batch, cudaStream_t s) {
  int rc;
  const int B = batch, N = c->N;
  GASP_CUDA(cudaMemsetAsync(c->d_grad, 0, kNParam * sizeof(float), s));
  GASP_CUDA(cudaMemsetAsync(c->d_loss, 0, sizeof(float), s));
  if ((rc = cnn_forward(c, B, s))) return rc;
  k_head<<<(B + 7) / 8, 256, 0, s>>>(B, N, c->d_pool, c->d_params, c->d_labels, c->d_q, c->d_loss,
                                     c->d_grad, c->d_dmean);
  GASP_CUDA(cudaGetLastError());
  const dim3 gz((unsigned)((N * (kC / 8) + 255) / 256), (unsigned)(B < 65535 ? B : 65535));
  k_dz4<<<gz, 256, 0, s>>>(B, N, c->d_dmean, c->d_act[3], c->d_dz[0]);
  GASP_CUDA(cudaGetLastError());
  int cur = 0;
  int dev = 0, nsm = 148;
  GASP_CUDA(cudaGetDevice(&dev));
  GASP_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
  const int dw_grid = nsm * 3;  // k_conv_dw32: 3 resident blocks per SM (registers)
  DwArgs d;
  memset(&d, 0, sizeof d);
  d.L = c->L;
  d.err = c->d_err;
  d.ntiles = B * (N / kTileM);
  for (int l = 3; l >= 1; --l) {  // layers 4, 3, 2 (0-based l)
    float *gW = c->d_grad + kOffW2 + (l - 1) * (9216 + 32);
    d.x = c->d_act[l - 1];
    d.dz = c->d_dz[cur];
    d.dW = gW;
    d.db = gW + 9216;
    switch (c->L) {
      case 32: rc = launch_dw(k_conv_dw_win<32>, dw_win_smem(32), 128, d, s); break;
      case 64: rc = launch_dw(k_conv_dw_win<64>, dw_win_smem(64), 128, d, s); break;
      case 128: rc = launch_dw(k_conv_dw_win<128>, dw_win_smem(128), 128, d, s); break;
      default:
        k_conv_dw32<<<dw_grid, 256, 0, s>>>(c->L, B, c->d_dz[cur], c->d_act[l - 1], gW,
                                            gW + 9216);
        GASP_CUDA(cudaGetLastError());
        rc = GASP_OK;
    }
    if (rc) return rc;
    ConvArgs a;
    memset(&a, 0, sizeof a);
    a.L = c->L;
    a.err = c->d_err;
    a.x = c->d_dz[cur];
    a.w = c->d_wt + (l - 1) * 9216;
    a.y = c->d_dz[cur ^ 1];
    a.mask_src = c->d_act[l - 1];
    if ((rc = launch_conv<kBwd>(a, B, s))) return rc;
    cur ^= 1;
  }
  d.x = nullptr;
  d.spins = c->d_spins;
  d.dz = c->d_dz[cur];
  d.dW = c->d_grad + kOffW1;
  d.db = c->d_grad + kOffB1;
  return launch_dw(k_conv_dw1_tc, kDw1Smem, 32, d, s);
}

}  // namespace

extern "C" {

int gasp_cnn_param_count(void) { return kNParam; }

int gasp_cnn_create(int L, int max_batch, gasp_cnn_t **out) {
  if (!out || max_batch <= 0 || L <= 0 || (L * L) % kTileM != 0) {
    set_error("gasp_cnn_create: L*L must be a multiple of 128 and max_batch positive");
    return GASP_ERR_INVALID;
  }
  *out = nullptr;
  gasp_cnn *c = new (std::nothrow) gasp_cnn();
  if (!c) return GASP_ERR_ALLOC;
  memset(c, 0, sizeof *c);
  cudaGetDevice(&c->device);
  c->L = L;
  c->N = L * L;
  c->max_batch = max_batch;
  c->fused = 0;  // the layer-by-layer path measured faster (1.0M vs 0.62M grids/s)
  const size_t act = (size_t)max_batch * c->N * kC * sizeof(__nv_bfloat16);
  cudaError_t e = cudaSuccess;
  auto A = [&](void **p, size_t n) {
    if (e == cudaSuccess) e = cudaMalloc(p, n);
  };
  A((void **)&c->d_params, kNParam * sizeof(float));
  A((void **)&c->d_grad, kNParam * sizeof(float));
  A((void **)&c->d_m, kNParam * sizeof(float));
  A((void **)&c->d_v, kNParam * sizeof(float));
  A((void **)&c->d_w1, 32 * 16 * sizeof(__nv_bfloat16));
  A((void **)&c->d_w, 3 * 9216 * sizeof(__nv_bfloat16));
  A((void **)&c->d_wt, 3 * 9216 * sizeof(__nv_bfloat16));
  A((void **)&c->d_spins, (size_t)max_batch * c->N);
  A((void **)&c->d_labels, (size_t)max_batch * sizeof(float));
  A((void **)&c->d_q, (size_t)max_batch * sizeof(float));
  A((void **)&c->d_mag, (size_t)max_batch * sizeof(float));
  A((void **)&c->d_pool, (size_t)max_batch * kC * sizeof(float));
  A((void **)&c->d_dmean, (size_t)max_batch * kC * sizeof(float));
  A((void **)&c->d_loss, sizeof(float));
  A((void **)&c->d_err, sizeof(int));
  A((void **)&c->d_tab, (size_t)kNPatterns * kC * sizeof(__nv_bfloat16));
  for (int i = 0; i < 4; ++i) A((void **)&c->d_act[i], act);
  for (int i = 0; i < 2; ++i) A((void **)&c->d_dz[i], act);
  if (e == cudaSuccess) e = cudaMemset(c->d_params, 0, kNParam * sizeof(float));
  if (e == cudaSuccess) e = cudaMemset(c->d_m, 0, kNParam * sizeof(float));
  if (e == cudaSuccess) e = cudaMemset(c->d_v, 0, kNParam * sizeof(float));
  if (e == cudaSuccess) e = cudaMemset(c->d_err, 0, sizeof(int));
  if (e != cudaSuccess) {
    gasp_cnn_free(c);
    return cuda_fail(e, "gasp_cnn_create", __FILE__, __LINE__);
  }
  *out = c;
  return GASP_OK;
}

int gasp_cnn_free(gasp_cnn_t *c) {
  if (!c) return GASP_OK;
  void *ptrs[] = {c->d_params, c->d_grad, c->d_m, c->d_v, c->d_w1, c->d_w, c->d_wt, c->d_spins,
                  c->d_labels, c->d_q, c->d_mag, c->d_pool, c->d_dmean, c->d_loss, c->d_err, c->d_tab,
                  c->d_act[0], c->d_act[1], c->d_act[2], c->d_act[3], c->d_dz[0], c->d_dz[1]};
  for (void *p : ptrs) cudaFree(p);
  if (c->copy_stream) {
    cudaStreamDestroy(c->copy_stream);
    for (int i = 0; i < 2; ++i) {
      cudaEventDestroy(c->ev_copied[i]);
      cudaEventDestroy(c->ev_used[i]);
    }
  }
  cudaFree(c->d_spins2);
  delete c;
  return GASP_OK;
}

int gasp_cnn_set_params(gasp_cnn_t *c, const float *params) {
  if (!c || !params) return GASP_ERR_INVALID;
  GASP_CUDA(cudaMemcpy(c->d_params, params, kNParam * sizeof(float), cudaMemcpyHostToDevice));
  GASP_CUDA(cudaMemset(c->d_m, 0, kNParam * sizeof(float)));
  GASP_CUDA(cudaMemset(c->d_v, 0, kNParam * sizeof(float)));
  c->adam_t = 0;
  return GASP_OK;
}

int gasp_cnn_get_params(gasp_cnn_t *c, float *params) {
  if (!c || !params) return GASP_ERR_INVALID;
  GASP_CUDA(cudaMemcpy(params, c->d_params, kNParam * sizeof(float), cudaMemcpyDeviceToHost));
  return GASP_OK;
}

int gasp_cnn_predict_ex(gasp_cnn_t *c, const int8_t *spins, int batch, float *q_out,
                        float *mag_out) {
  if (!c || !spins || !q_out || batch <= 0) return GASP_ERR_INVALID;
  cudaStream_t s = current_stream();
  int rc;
  if (batch > c->max_batch) return predict_chunked(c, spins, batch, q_out, mag_out, s);
  if ((rc = cnn_upload(c, spins, nullptr, batch))) return rc;
  if ((rc = cnn_infer(c, batch, s))) return rc;
  k_head<<<(batch + 7) / 8, 256, 0, s>>>(batch, c->N, c->d_pool, c->d_params, nullptr, c->d_q,
                                         nullptr, nullptr, nullptr);
  GASP_CUDA(cudaGetLastError());
  GASP_CUDA(cudaMemcpyAsync(q_out, c->d_q, (size_t)batch * sizeof(float), cudaMemcpyDeviceToHost, s));
  if (mag_out) {
    k_spin_mag<<<(batch + 7) / 8, 256, 0, s>>>(c->d_spins, c->N, batch, c->d_mag);
    GASP_CUDA(cudaGetLastError());
    GASP_CUDA(cudaMemcpyAsync(mag_out, c->d_mag, (size_t)batch * sizeof(float),
                              cudaMemcpyDeviceToHost, s));
  }
  return cnn_check_err(c, s);
}

int gasp_cnn_predict(gasp_cnn_t *c, const int8_t *spins, int batch, float *q_out) {
  return gasp_cnn_predict_ex(c, spins, batch, q_out, nullptr);
}

int gasp_cnn_set_fused(gasp_cnn_t *c, int on) {
  if (!c) return GASP_ERR_INVALID;
  c->fused = on != 0;
  return GASP_OK;
}

int gasp_cnn_gradients(gasp_cnn_t *c, const int8_t *spins, const float *labels, int batch,
                       float *loss_out, float *grad_out) {
  if (!c || !spins || !labels || batch <= 0 || batch > c->max_batch) return GASP_ERR_INVALID;
  cudaStream_t s = current_stream();
  int rc;
  if ((rc = cnn_upload(c, spins, labels, batch))) return rc;
  if ((rc = cnn_backward(c, batch, s))) return rc;
  if (loss_out) GASP_CUDA(cudaMemcpyAsync(loss_out, c->d_loss, sizeof(float), cudaMemcpyDeviceToHost, s));
  if (grad_out)
    GASP_CUDA(cudaMemcpyAsync(grad_out, c->d_grad, kNParam * sizeof(float), cudaMemcpyDeviceToHost, s));
  return cnn_check_err(c, s);
}

int gasp_cnn_train_step(gasp_cnn_t *c, const int8_t *spins, const float *labels, int batch,
                        float lr, float *loss_out) {
  if (!c || !spins || !labels || batch <= 0 || batch > c->max_batch) return GASP_ERR_INVALID;
  cudaStream_t s = current_stream();
  int rc;
  if ((rc = cnn_upload(c, spins, labels, batch))) return rc;
  if ((rc = cnn_backward(c, batch, s))) return rc;
  c->adam_t++;
  const float b1 = 0.9f, b2 = 0.999f;
  const float c1 = 1.0f - powf(b1, (float)c->adam_t), c2 = 1.0f - powf(b2, (float)c->adam_t);
  k_adam<<<(kNParam + 255) / 256, 256, 0, s>>>(c->d_params, c->d_grad, c->d_m, c->d_v, kNParam,
                                               lr, b1, b2, 1e-8f, c1, c2);
  GASP_CUDA(cudaGetLastError());
  if (loss_out) GASP_CUDA(cudaMemcpyAsync(loss_out, c->d_loss, sizeof(float), cudaMemcpyDeviceToHost, s));
  return cnn_check_err(c, s);
}

}  // extern "C"
