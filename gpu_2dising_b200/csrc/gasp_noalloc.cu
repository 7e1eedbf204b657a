// gasp_noalloc.cu -- gasp_grids_upload_inputs_noalloc: the start-from-inputs
// upload of gasp_grids_upload_inputs without any device allocation.
//
// gasp_grids_upload_inputs stages the int32 input grids in a per-set buffer
// that it allocates on first use, sized for the whole set (ngrids * L * L
// int32, 32x the bit-packed lattice).  This form stages them instead in one
// fixed file-scope device array, so a set can be re-seeded from new inputs
// (committor shooting rounds) when the device has no room for that buffer or
// when the caller must not let cudaMalloc/cudaFree synchronise the device
// under work running on other streams.
#include <mutex>

#include "gasp_internal.h"

namespace {

// The staging array.  Nothing in it has to start at zero: every call
// overwrites the ninputs * L * L entries that its pack kernel reads.
__device__ __align__(256) int g_stage[GASP_NOALLOC_MAX_INPUT_INTS];

constexpr int kMaxDevices = 64;
std::mutex g_stage_mu;
int *g_stage_addr[kMaxDevices];  // device address of g_stage, per device

// Looks up the device address of g_stage once per device, with that device
// current (the address is per device; host code never uses the symbol name
// as a device pointer).
int stage_address(int dev, int **out) {
  if (dev < 0 || dev >= kMaxDevices) {
    gasp::set_error("gasp_grids_upload_inputs_noalloc: device %d out of range", dev);
    return GASP_ERR_INVALID;
  }
  std::lock_guard<std::mutex> lock(g_stage_mu);
  if (!g_stage_addr[dev]) {
    int *p = nullptr;
    cudaError_t e = cudaGetSymbolAddress((void **)&p, g_stage);
    if (e != cudaSuccess)
      return gasp::cuda_fail(e, "cudaGetSymbolAddress(g_stage)", __FILE__, __LINE__);
    g_stage_addr[dev] = p;
  }
  *out = g_stage_addr[dev];
  return GASP_OK;
}

}  // namespace

extern "C" int gasp_grids_upload_inputs_noalloc(gasp_grids_t *g, const int *inputs,
                                                int ninputs) {
  if (!g || !inputs || ninputs <= 0 || g->ngrids % ninputs != 0) {
    gasp::set_error("gasp_grids_upload_inputs_noalloc: ngrids must be a multiple of ninputs");
    return GASP_ERR_INVALID;
  }
  const long long need = (long long)ninputs * g->N;
  if (need > (long long)GASP_NOALLOC_MAX_INPUT_INTS) {
    gasp::set_error(
        "gasp_grids_upload_inputs_noalloc: %d inputs of %dx%d need %lld int32, above the "
        "fixed stage of %d (GASP_NOALLOC_MAX_INPUT_INTS); use gasp_grids_upload_inputs",
        ninputs, g->L, g->L, need, (int)GASP_NOALLOC_MAX_INPUT_INTS);
    return GASP_ERR_INVALID;
  }
  int cur = -1;
  GASP_CUDA(cudaGetDevice(&cur));
  if (cur != g->device) GASP_CUDA(cudaSetDevice(g->device));
  int *stage = nullptr;
  int rc = stage_address(g->device, &stage);
  if (rc) return rc;
  cudaStream_t s = gasp::current_stream();
  GASP_CUDA(cudaMemcpyAsync(stage, inputs, (size_t)need * sizeof(int), cudaMemcpyHostToDevice, s));
  rc = gasp::launch_pack_grids(stage, g->d_lat, g->L, g->ngrids, s, g->ngrids / ninputs);
  // The stage is free for the next call once this returns: wait for the copy
  // on the error path too, then report the first error.
  const cudaError_t se = cudaStreamSynchronize(s);
  if (rc) return rc;
  if (se != cudaSuccess) return gasp::cuda_fail(se, "cudaStreamSynchronize", __FILE__, __LINE__);
  return GASP_OK;
}
