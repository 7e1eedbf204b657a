/*
 * gasp_host.c -- host-side helpers of the gasp-b200 C ABI: initial grids
 * (src/grid.c), the gridinput.bin / gridstates.bin formats (src/io.c:4-130),
 * the committor per input block (src/mc_gpu.cu:812-826) and the bootstrap
 * error bar (src/bootstrap.c:6-65).  Errors are returned, never exit().
 */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "gasp.h"

int gasp_init_grids_uniform(int L, int ngrids, int spin, int *out) {
  if (L <= 0 || ngrids <= 0 || !out) return GASP_ERR_INVALID;
  const size_t n = (size_t)L * L * ngrids;
  for (size_t i = 0; i < n; ++i) out[i] = spin;
  return GASP_OK;
}

int gasp_read_input_grid(const char *path, int L, int ngrids, int *out) {
  if (L <= 0 || ngrids <= 0 || !out) return GASP_ERR_INVALID;
  FILE *f = fopen(path ? path : "gridinput.bin", "rb");
  if (!f) return GASP_ERR_IO;
  int Lcheck = 0;
  if (fread(&Lcheck, sizeof(int), 1, f) != 1) {
    fclose(f);
    return GASP_ERR_IO;
  }
  if (Lcheck != L) {  /* src/io.c:25-28 */
    fclose(f);
    return GASP_ERR_FORMAT;
  }
  const int N = L * L;
  const size_t nbytes = (size_t)(N + 7) / 8;
  unsigned char *buf = (unsigned char *)malloc(nbytes);
  if (!buf) {
    fclose(f);
    return GASP_ERR_ALLOC;
  }
  const size_t got = fread(buf, 1, nbytes, f);
  fclose(f);
  if (got != nbytes) {
    free(buf);
    return GASP_ERR_IO;
  }
  /* LSB-first, bit 1 -> +1, row-major; only the first L*L bits are spins. */
  for (int s = 0; s < N; ++s) out[s] = ((buf[s >> 3] >> (s & 7)) & 1) ? 1 : -1;
  free(buf);
  for (int g = 1; g < ngrids; ++g) memcpy(out + (size_t)g * N, out, sizeof(int) * (size_t)N);
  return GASP_OK;
}

int gasp_init_grids_from_file(const char *path, int L, int ngrids, int *out) {
  return gasp_read_input_grid(path, L, ngrids, out);
}

int gasp_init_grids_from_array(int L, int ngrids, int ninputs, const int *array, int *out) {
  if (L <= 0 || ngrids <= 0 || ninputs <= 0 || !array || !out) return GASP_ERR_INVALID;
  if (ngrids % ninputs != 0) return GASP_ERR_INVALID; /* src/grid.c:51-54 */
  const size_t N = (size_t)L * L;
  const int per = ngrids / ninputs;
  for (int m = 0; m < ninputs; ++m)
    for (int i = 0; i < per; ++i)
      memcpy(out + ((size_t)m * per + i) * N, array + (size_t)m * N, sizeof(int) * N);
  return GASP_OK;
}

int gasp_init_fates(int ngrids, int *out) {
  if (ngrids <= 0 || !out) return GASP_ERR_INVALID;
  for (int i = 0; i < ngrids; ++i) out[i] = -1;
  return GASP_OK;
}

int gasp_write_packed_frame(const char *path, int L, int ngrids, int isweep,
                            const uint8_t *payload, size_t nbytes) {
  if (!path || !payload) return GASP_ERR_INVALID;
  FILE *f = fopen(path, "ab");
  if (!f) return GASP_ERR_IO;
  const int hdr[3] = {L, ngrids, isweep};
  int ok = fwrite(hdr, sizeof(int), 3, f) == 3 && fwrite(payload, 1, nbytes, f) == nbytes;
  ok = (fclose(f) == 0) && ok;
  return ok ? GASP_OK : GASP_ERR_IO;
}

int gasp_read_frame(const char *path, int iframe, int *L_out, int *ngrids_out, int *isweep_out,
                    int *grids_out, long long grids_cap) {
  if (!path || iframe < 0) return GASP_ERR_INVALID;
  FILE *f = fopen(path, "rb");
  if (!f) return GASP_ERR_IO;
  int hdr[3] = {0, 0, 0};
  long long payload = 0;
  for (int k = 0;; ++k) {
    if (fread(hdr, sizeof(int), 3, f) != 3 || hdr[0] <= 0 || hdr[1] <= 0) {
      fclose(f);
      return GASP_ERR_IO; /* fewer than iframe+1 frames, or a damaged header */
    }
    payload = ((long long)hdr[0] * hdr[0] * hdr[1] + 7) / 8;
    if (k == iframe) break;
    if (fseek(f, (long)payload, SEEK_CUR) != 0) {
      fclose(f);
      return GASP_ERR_IO;
    }
  }
  if (L_out) *L_out = hdr[0];
  if (ngrids_out) *ngrids_out = hdr[1];
  if (isweep_out) *isweep_out = hdr[2];
  int rc = GASP_OK;
  if (grids_out) {
    const long long nbits = (long long)hdr[0] * hdr[0] * hdr[1];
    uint8_t *buf = NULL;
    if (grids_cap < nbits) {
      rc = GASP_ERR_INVALID;
    } else if (!(buf = (uint8_t *)malloc((size_t)payload))) {
      rc = GASP_ERR_ALLOC;
    } else if (fread(buf, 1, (size_t)payload, f) != (size_t)payload) {
      rc = GASP_ERR_IO;
    } else {
      for (long long i = 0; i < nbits; ++i) grids_out[i] = ((buf[i >> 3] >> (i & 7)) & 1) ? 1 : -1;
    }
    free(buf);
  }
  fclose(f);
  return rc;
}

int gasp_write_input_grid(const char *path, int L, const int *grid) {
  if (L <= 0 || !grid) return GASP_ERR_INVALID;
  const int N = L * L;
  const size_t nbytes = (size_t)(N + 7) / 8;
  uint8_t *buf = (uint8_t *)calloc(nbytes, 1);
  if (!buf) return GASP_ERR_ALLOC;
  for (int s = 0; s < N; ++s)
    if (grid[s] == 1) buf[s >> 3] |= (uint8_t)(1u << (s & 7));
  FILE *f = fopen(path ? path : "gridinput.bin", "wb");
  if (!f) {
    free(buf);
    return GASP_ERR_IO;
  }
  int ok = fwrite(&L, sizeof(int), 1, f) == 1 && fwrite(buf, 1, nbytes, f) == nbytes;
  ok = (fclose(f) == 0) && ok;
  free(buf);
  return ok ? GASP_OK : GASP_ERR_IO;
}

int gasp_write_ising_grids(int L, int ngrids, int *ising_grids, int isweep,
                           float *magnetisation, float *lclus_size, char *cv,
                           double dn_thr, double up_thr, char *filename) {
  (void)magnetisation; (void)lclus_size; (void)cv; (void)dn_thr; (void)up_thr;
  if (!ising_grids || L <= 0 || ngrids <= 0) return GASP_ERR_INVALID;
  const long long nbits = (long long)L * L * ngrids;
  const size_t nbytes = (size_t)((nbits + 7) / 8);
  uint8_t *buf = (uint8_t *)calloc(nbytes, 1);
  if (!buf) return GASP_ERR_ALLOC;
  for (long long i = 0; i < nbits; ++i)
    if (ising_grids[i] == 1) buf[i >> 3] |= (uint8_t)(1u << (i & 7));
  int rc = gasp_write_packed_frame(filename ? filename : "gridstates.bin", L, ngrids, isweep,
                                   buf, nbytes);
  free(buf);
  return rc;
}

double gasp_bootstrap_errbar(int ngrids, int m, const int *grid_fate) {
  if (ngrids <= 0 || m <= 0 || !grid_fate) return -1.0;
  int *ind = (int *)malloc(sizeof(int) * (size_t)ngrids);
  double *pb = (double *)malloc(sizeof(double) * (size_t)m);
  if (!ind || !pb) {
    free(ind);
    free(pb);
    return -1.0;
  }
  for (int im = 0; im < m; ++im) {
    int nA = 0, nB = 0;
    for (int i = 0; i < ngrids; ++i) ind[i] = rand() % ngrids;
    for (int i = 0; i < ngrids; ++i) {
      const int f = grid_fate[ind[i]];
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

int gasp_committor_from_fates(int ngrids, int ninputs, const int *grid_fate, float *pB) {
  if (ngrids <= 0 || ninputs <= 0 || ngrids % ninputs != 0 || !grid_fate || !pB)
    return GASP_ERR_INVALID;
  const int sub = ngrids / ninputs;
  for (int i = 0; i < ninputs; ++i) {
    int nB = 0, nF = 0;
    for (int j = 0; j < sub; ++j) {
      const int f = grid_fate[i * sub + j];
      if (f > -1) nB += f;
      else nF += 1;
    }
    pB[i] = (float)nB / (float)(sub - nF);
  }
  return GASP_OK;
}
