/*
 * gasp_oracle.c -- CPU restatement of the GASP hot path.  TEST INFRASTRUCTURE
 * ONLY: imported by tests/, __graft_entry__.smoke() and bench.py's CPU
 * baseline leg as the checker; the product library never links it.
 *
 * Parity of this file is pinned against the reference's own CPU code compiled
 * unmodified from its sources (oracle/Makefile -> oracle/_ref/) and against
 * the committed golden fixtures in tests/golden/.
 *
 * Build: gcc -O2 -ffp-contract=off -fPIC -shared (oracle/Makefile).  Float
 * arithmetic must stay single precision and uncontracted so that the GPU
 * flavour below rounds like the reference's device code.
 */
#include "gasp_oracle.h"

#include <float.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

/* src/mc_cpu.c:14-38 -- P[5(s+1)+nsum+4] = exp(-beta * 2 s (nsum + h)), double. */
void orc_probs_cpu(double beta, double h, double P[20]) {
  for (int i = 0; i < 20; ++i) P[i] = 0.0;
  for (int s = -1; s <= 1; s += 2) {
    for (int nsum = -4; nsum <= 4; nsum += 2) {
      int index = 5 * (s + 1) + nsum + 4;
      double de = 2.0 * (double)s * ((double)nsum + h);
      P[index] = exp(-beta * de);
    }
  }
}

/* src/mc_gpu.cu:21-37 -- same table in float: 2f*s*((float)nsum+(float)h),
 * then expf(-(float)beta * that) on the host. */
void orc_probs_gpu(double beta, double h, float P[20]) {
  for (int i = 0; i < 20; ++i) P[i] = 0.0f;
  for (int s = -1; s <= 1; s += 2) {
    for (int nsum = -4; nsum <= 4; nsum += 2) {
      int index = 5 * (s + 1) + nsum + 4;
      float de = 2.0f * (float)s * ((float)nsum + (float)h);
      P[index] = expf(-(float)beta * de);
    }
  }
}

/* Neighbour sum of the four periodic neighbours (src/mc_cpu.c:55-62). */
static inline int nsum4(const int *g, int L, int row, int col) {
  int up = L * ((row + L - 1) % L) + col;
  int dn = L * ((row + 1) % L) + col;
  int rt = L * row + (col + 1) % L;
  int lt = L * row + (col + L - 1) % L;
  return g[up] + g[dn] + g[lt] + g[rt];
}

/* src/mc_cpu.c:41-89.  The reference flips, draws xi, and reverts on reject;
 * the net effect is a conditional flip, which is what is done here. */
long long orc_sweep_cpu_stream(int L, int *grid, long long nattempts,
                               const double *stream, const double P[20]) {
  for (long long a = 0; a < nattempts; ++a) {
    double ur = stream[3 * a + 0];
    double uc = stream[3 * a + 1];
    double xi = stream[3 * a + 2];
    int row = (int)floor(L * ur);
    int col = (int)floor(L * uc);
    int my = L * row + col;
    int index = 5 * (grid[my] + 1) + nsum4(grid, L, row, col) + 4;
    if (xi < P[index]) grid[my] = -grid[my];
  }
  return nattempts;
}

/* src/mc_gpu.cu:310-340 (method 2), identical arithmetic in method 0
 * (src/mc_gpu.cu:98-129) and method 1 (src/mc_gpu.cu:216-253: the expression
 * (float)L*L*shrink*u evaluates as fl(fl(N*(1-eps))*u), the same value). */
long long orc_sweep_gpu_stream(int L, int *grid, long long nattempts,
                               const float *ustream, const float P[20]) {
  const int N = L * L;
  const float shrink = (1.0f - FLT_EPSILON) * (float)N;
  for (long long a = 0; a < nattempts; ++a) {
    float u1 = ustream[2 * a + 0];
    float u2 = ustream[2 * a + 1];
    float prod = shrink * u1;
    int my = (int)floorf(prod);
    int row = my / L, col = my % L;
    int spin = grid[my];
    int n1 = grid[L * ((row + 1) % L) + col];
    int n2 = grid[L * ((row + L - 1) % L) + col];
    int n3 = grid[L * row + (col + 1) % L];
    int n4 = grid[L * row + (col + L - 1) % L];
    int index = 5 * (spin + 1) + n1 + n2 + n3 + n4 + 4;
    if (u2 < P[index]) grid[my] = -spin;
  }
  return nattempts;
}

/* src/mc_gpu.cu:437-455: float accumulation of the int spins (exact for
 * N <= 2^24), then one float division. */
float orc_magnetisation_gpu(int L, const int *grid) {
  float m = 0.0f;
  for (int i = 0; i < L * L; ++i) m += (float)grid[i];
  return m / (float)(L * L);
}

/* src/mc_cpu.c:91-104. */
float orc_magnetisation_cpu(int L, const int *grid) {
  double m = 0.0;
  for (int i = 0; i < L * L; ++i) m += (double)grid[i];
  return (float)(m / (double)(L * L));
}

/* src/mc_cpu.c:310-364 (and its GPU twin src/mc_gpu.cu:457-526): size of the
 * largest 4-connected cluster of sites equal to `spin`, periodic in both
 * directions, found by flood fill from every unvisited matching site.
 * Returns -1 if the work arrays cannot be allocated. */
int orc_largest_cluster(int L, const int *grid, int spin) {
  const int N = L * L;
  unsigned char *seen = (unsigned char *)calloc((size_t)N, 1);
  int *todo = (int *)malloc((size_t)N * sizeof(int));
  if (!seen || !todo) {
    free(seen);
    free(todo);
    return -1;
  }
  int best = 0;
  for (int start = 0; start < N; ++start) {
    if (grid[start] != spin || seen[start]) continue;
    int head = 0, tail = 0, size = 0;
    seen[start] = 1;
    todo[tail++] = start;
    while (head < tail) {
      const int s = todo[head++];
      ++size;
      const int r = s / L, c = s % L;
      const int nb[4] = {r * L + (c + L - 1) % L, r * L + (c + 1) % L,
                         ((r + L - 1) % L) * L + c, ((r + 1) % L) * L + c};
      for (int k = 0; k < 4; ++k)
        if (grid[nb[k]] == spin && !seen[nb[k]]) {
          seen[nb[k]] = 1;
          todo[tail++] = nb[k];
        }
    }
    if (size > best) best = size;
  }
  free(seen);
  free(todo);
  return best;
}

/* src/io.c:89-117: one running bit cursor over all L*L*ngrids spins. */
long long orc_pack_frame(int L, int ngrids, const int *grids, uint8_t *out) {
  long long nbits = (long long)L * L * ngrids;
  long long nbytes = (nbits + 7) / 8;
  memset(out, 0, (size_t)nbytes);
  for (long long i = 0; i < nbits; ++i)
    if (grids[i] == 1) out[i >> 3] |= (uint8_t)(1u << (i & 7));
  return nbytes;
}

void orc_unpack_frame(int L, int ngrids, const uint8_t *in, int *grids) {
  long long nbits = (long long)L * L * ngrids;
  for (long long i = 0; i < nbits; ++i)
    grids[i] = ((in[i >> 3] >> (i & 7)) & 1) ? 1 : -1;
}

/* src/io.c:67-130 (append mode, 3 int32 header words, packed payload). */
int orc_write_frame(const char *path, int L, int ngrids, const int *grids, int isweep) {
  FILE *f = fopen(path, "ab");
  if (!f) return -1;
  int hdr[3] = {L, ngrids, isweep};
  long long nbytes = ((long long)L * L * ngrids + 7) / 8;
  uint8_t *buf = (uint8_t *)malloc((size_t)nbytes);
  if (!buf) { fclose(f); return -1; }
  orc_pack_frame(L, ngrids, grids, buf);
  int ok = fwrite(hdr, sizeof(int), 3, f) == 3 &&
           fwrite(buf, 1, (size_t)nbytes, f) == (size_t)nbytes;
  free(buf);
  fclose(f);
  return ok ? 0 : -1;
}

/* src/io.c:4-65 with the intended semantics: only the first L*L bits are
 * spins (the reference also writes padding bits past each grid when
 * L*L % 8 != 0, src/io.c:47-58). */
int orc_read_input_grid(const char *path, int L, int ngrids, int *grids) {
  FILE *f = fopen(path, "rb");
  if (!f) return -1;
  int Lcheck = 0;
  if (fread(&Lcheck, sizeof(int), 1, f) != 1) { fclose(f); return -1; }
  if (Lcheck != L) { fclose(f); return -2; }
  int N = L * L;
  int nbytes = (N + 7) / 8;
  uint8_t *buf = (uint8_t *)malloc((size_t)nbytes);
  if (!buf) { fclose(f); return -1; }
  size_t got = fread(buf, 1, (size_t)nbytes, f);
  fclose(f);
  if (got != (size_t)nbytes) { free(buf); return -1; }
  for (int s = 0; s < N; ++s) {
    int v = ((buf[s >> 3] >> (s & 7)) & 1) ? 1 : -1;
    for (int g = 0; g < ngrids; ++g) grids[(long long)g * N + s] = v;
  }
  free(buf);
  return 0;
}

/* src/bootstrap.c:6-65: m resamples of ngrids indices drawn with
 * rand()%ngrids (all indices of one resample drawn first), pending fates
 * ignored, population standard deviation (divide by m). */
double orc_bootstrap_errbar(int ngrids, int m, const int *fate) {
  int *ind = (int *)malloc(sizeof(int) * (size_t)ngrids);
  double *pb = (double *)malloc(sizeof(double) * (size_t)m);
  if (!ind || !pb) { free(ind); free(pb); return -1.0; }
  for (int im = 0; im < m; ++im) {
    int nA = 0, nB = 0;
    for (int i = 0; i < ngrids; ++i) ind[i] = rand() % ngrids;
    for (int i = 0; i < ngrids; ++i) {
      int f = fate[ind[i]];
      if (f == 0) nA++;
      else if (f == 1) nB++;
    }
    pb[im] = (double)nB / (double)(nA + nB);
  }
  double mean = 0.0, num = 0.0;
  for (int im = 0; im < m; ++im) mean += pb[im];
  mean /= m;
  for (int im = 0; im < m; ++im) num += (pb[im] - mean) * (pb[im] - mean);
  free(ind);
  free(pb);
  return sqrt(num / m);
}

void orc_srand(unsigned int seed) { srand(seed); }

/* src/mc_gpu.cu:812-826: pB = nB / (sub - nPending) per contiguous block. */
void orc_committor_from_fates(int ngrids, int ninputs, const int *fate, float *pB) {
  int sub = ngrids / ninputs;
  for (int i = 0; i < ninputs; ++i) {
    int nB = 0, nF = 0;
    for (int j = 0; j < sub; ++j) {
      int f = fate[i * sub + j];
      if (f > -1) nB += f;
      else nF += 1;
    }
    pB[i] = (float)nB / (float)(sub - nF);
  }
}

/* ------------------------------------------------------------------------
 * Production stream (MWC64X) sweeps.  No reference counterpart: the
 * reference has only cuRAND XORWOW.  Attempt semantics follow
 * src/mc_gpu.cu:311-340 (random site, accept on a uniform draw below the
 * table entry) with integer draws: site = (r * N) >> 32 of a 32-bit draw r,
 * accept iff the next draw u <= thr[5*(spin up) + (# up neighbours)], where
 * thr[] comes from the product's gasp_acceptance_thresholds.
 * ---------------------------------------------------------------------- */
#define ORC_MWC_A 4294883355ull

static inline uint32_t orc_mwc_next(uint32_t *x, uint32_t *c) {
  uint32_t r = *x ^ *c;
  uint64_t t = (uint64_t)(*x) * ORC_MWC_A + *c;
  *x = (uint32_t)t;
  *c = (uint32_t)(t >> 32);
  return r;
}

static inline void orc_apply_int(int L, int *grid, uint32_t s, uint32_t u, const uint32_t thr[10]) {
  int row = (int)s / L, col = (int)s % L;
  int up = 0;
  up += grid[L * ((row + 1) % L) + col] > 0;
  up += grid[L * ((row + L - 1) % L) + col] > 0;
  up += grid[L * row + (col + 1) % L] > 0;
  up += grid[L * row + (col + L - 1) % L] > 0;
  int cls = 5 * (grid[s] > 0) + up;
  if (u <= thr[cls]) grid[s] = -grid[s];
}

/* One replica, one MWC64X stream (x, c updated in place), attempts applied
 * one at a time: the row kernels' production mode. */
long long orc_sweep_mwc(int L, int *grid, long long nattempts, uint32_t *x, uint32_t *c,
                        const uint32_t thr[10]) {
  const uint64_t N = (uint64_t)L * L;
  for (long long a = 0; a < nattempts; ++a) {
    uint32_t s = (uint32_t)(((uint64_t)orc_mwc_next(x, c) * N) >> 32);
    uint32_t u = orc_mwc_next(x, c);
    orc_apply_int(L, grid, s, u, thr);
  }
  return nattempts;
}

static inline uint64_t orc_mulmod(uint64_t a, uint64_t b, uint64_t m) {
  return (uint64_t)((unsigned __int128)a * b % m);
}

static inline int orc_adjacent(int L, uint32_t a, uint32_t b) {
  int ra = (int)a / L, ca = (int)a % L, rb = (int)b / L, cb = (int)b % L;
  if (ra == rb) return cb == (ca + 1) % L || ca == (cb + 1) % L;
  if (ca == cb) return rb == (ra + 1) % L || ra == (rb + 1) % L;
  return 0;
}

/* The one-warp-per-replica sweep (sweep variant 6), restated serially: the
 * window of 32 pending attempts (lane l at position (l - head) mod 32), the
 * rule fixing how many are applied per round (up to and including the first
 * position whose site, or a neighbour of it, holds another pending attempt),
 * which lane's substream draws each new attempt (every lane keeps its next
 * attempt drawn one assignment ahead), and the replica's stream state
 * afterwards.  Attempts are applied one at a time in window order; the kernel
 * applies each round's at once, which must give the same lattice.
 * x/c: the replica's state (in/out); mul/inv: gasp_mwc64x_lane_multipliers.
 * order (optional, 2 * nsweeps * L*L words) receives (site, u) of every
 * attempt in the order applied. */
long long orc_sweep_tail(int L, int *grid, int nsweeps, uint32_t *x, uint32_t *c,
                         const uint32_t thr[10], const uint64_t mul[32], const uint64_t inv[32],
                         uint32_t *order) {
  const uint64_t A = ORC_MWC_A, M = (A << 32) - 1;
  const uint64_t N = (uint64_t)L * L;
  const long long Q = (long long)nsweeps * (long long)N;
  uint32_t lx[32], lc[32], site[32], uu[32], nsite[32], nuu[32];
  unsigned nd[32];
  int valid[32], flag[32];
  const uint64_t X = (uint64_t)(*x) * A + *c;
  for (int j = 0; j < 32; ++j) {
    uint64_t Xj = orc_mulmod(X, mul[j], M);
    lx[j] = (uint32_t)(Xj / A);
    lc[j] = (uint32_t)(Xj % A);
    nsite[j] = (uint32_t)(((uint64_t)orc_mwc_next(&lx[j], &lc[j]) * N) >> 32);
    nuu[j] = orc_mwc_next(&lx[j], &lc[j]);
    nd[j] = 2;
  }
#define ORC_TAIL_TAKE(j)                                                          \
  do {                                                                            \
    site[j] = nsite[j];                                                           \
    uu[j] = nuu[j];                                                               \
    nsite[j] = (uint32_t)(((uint64_t)orc_mwc_next(&lx[j], &lc[j]) * N) >> 32);    \
    nuu[j] = orc_mwc_next(&lx[j], &lc[j]);                                        \
    nd[j] += 2;                                                                   \
  } while (0)
  long long drawn = Q < 32 ? Q : 32, done = 0, applied = 0;
  for (int j = 0; j < 32; ++j) {
    valid[j] = j < drawn;
    if (valid[j]) ORC_TAIL_TAKE(j);
  }
  int head = 0;
  long long pend = drawn;
  while (done < Q) {
    for (int j = 0; j < 32; ++j) {
      flag[j] = 0;
      if (!valid[j]) continue;
      for (int i = 0; i < 32; ++i)
        if (i != j && valid[i] && (site[i] == site[j] || orc_adjacent(L, site[i], site[j])))
          flag[j] = 1;
    }
    long long k = 32;
    for (int p = 0; p < 32; ++p) {
      int j = (head + p) & 31;
      if (flag[j]) {
        k = p + 1;
        break;
      }
    }
    if (k > pend) k = pend;
    for (int p = 0; p < k; ++p) {
      int j = (head + p) & 31;
      orc_apply_int(L, grid, site[j], uu[j], thr);
      if (order) {
        order[2 * applied] = site[j];
        order[2 * applied + 1] = uu[j];
      }
      ++applied;
    }
    done += k;
    head = (int)((head + k) & 31);
    pend -= k;
    long long room = 32 - pend, left = Q - drawn;
    long long nnew = room < left ? room : left;
    for (int j = 0; j < 32; ++j) {
      int p2 = (j - head) & 31;
      if (p2 >= pend) {
        valid[j] = p2 - pend < nnew;
        if (valid[j]) ORC_TAIL_TAKE(j);
      }
    }
    pend += nnew;
    drawn += nnew;
  }
#undef ORC_TAIL_TAKE
  int js = 0;
  for (int j = 1; j < 32; ++j)
    if (nd[j] > nd[js]) js = j;
  uint64_t Xe = (uint64_t)lx[js] * A + lc[js];
  uint64_t Xb = orc_mulmod(Xe, inv[js], M);
  *x = (uint32_t)(Xb / A);
  *c = (uint32_t)(Xb % A);
  return applied;
}

/* The multispin shared-site sweep (sweep variant 7) restated serially for
 * one tile of nrep <= 32 replicas (grids [nrep][L*L], streams x/c in/out):
 * sites come in batches -- at the start of a batch each replica draws one
 * site from its own stream, and attempt j of the batch uses replica j's site;
 * every replica then draws its acceptance and flips on u <= thr[class]. */
long long orc_sweep_shared(int L, int nrep, int *grids, int nsweeps, uint32_t *x, uint32_t *c,
                           const uint32_t thr[10]) {
  const uint64_t N = (uint64_t)L * L;
  const long long Q = (long long)nsweeps * (long long)N;
  uint32_t sites[32];
  int j = 0;
  for (long long a = 0; a < Q; ++a) {
    if (j == 0)
      for (int r = 0; r < nrep; ++r)
        sites[r] = (uint32_t)(((uint64_t)orc_mwc_next(&x[r], &c[r]) * N) >> 32);
    const uint32_t s = sites[j];
    j = j + 1 == nrep ? 0 : j + 1;
    for (int r = 0; r < nrep; ++r) {
      uint32_t u = orc_mwc_next(&x[r], &c[r]);
      orc_apply_int(L, grids + (size_t)r * N, s, u, thr);
    }
  }
  return Q;
}
