"""Python host layer over the gasp-b200 C ABI.

Thin objects owning the native handles: ``DeviceGrids`` (replaces the
reference's device grid array, src/gpu_tools.cu:143-159), ``RngStates``
(replaces the curandState array, src/gpu_tools.cu:162-174) and ``run_driver``
(replaces mc_driver_gpu, src/mc_gpu.cu:530-831).  Every call goes to the CUDA
library; a missing library or device raises.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _native as nat
from ._native import check, lib


def init_device(device_index=-1, verbose=False):
    """Selects a device; returns (device, n_SMs).  src/gpu_tools.cu:18-99."""
    dev, nsms = C.c_int(), C.c_int()
    check(lib().gasp_init_device(int(device_index), int(bool(verbose)), C.byref(dev),
                                 C.byref(nsms)), "gasp_init_device")
    return dev.value, nsms.value


def select_gpu_method(L, ngrids, threads_per_block=32, device=-1):
    """The reference's method auto-selection rule (src/gpu_tools.cu:205-232)."""
    m = C.c_int()
    check(lib().gasp_select_gpu_method(L, ngrids, threads_per_block, device, C.byref(m)),
          "gasp_select_gpu_method")
    return m.value


def acceptance_table(beta, h):
    """float32[20] table of preComputeProbs_gpu (src/mc_gpu.cu:21-37)."""
    out = np.zeros(20, np.float32)
    check(lib().gasp_acceptance_table(float(beta), float(h), out), "gasp_acceptance_table")
    return out


def max_shared_L(device=-1):
    v = C.c_int()
    check(lib().gasp_max_shared_L(device, C.byref(v)), "gasp_max_shared_L")
    return v.value


def set_stream(stream_handle):
    """Route this thread's device work to a cudaStream_t (int handle or 0)."""
    check(lib().gasp_set_stream(C.c_void_p(int(stream_handle) if stream_handle else None)))


class RngStates:
    """Per-replica cuRAND XORWOW states, seeded as gpuInitRand."""

    def __init__(self, ngrids, seed, threads_per_block=32, kind="xorwow"):
        """kind: "xorwow" (the reference's cuRAND stream, bit-exact) or
        "mwc64x" (the production stream, statistically equivalent)."""
        self.ngrids = int(ngrids)
        self.kind = kind
        k = {"xorwow": nat.RNG_XORWOW, "mwc64x": nat.RNG_MWC64X}[kind]
        self._h = C.c_void_p()
        check(lib().gasp_init_rand_mode(self.ngrids, threads_per_block, C.c_ulonglong(int(seed)),
                                        k, C.byref(self._h)), "gasp_init_rand")

    @property
    def handle(self):
        return self._h

    @property
    def stride(self):
        return (self.ngrids + 31) // 32 * 32

    def read_states(self):
        """Device states as (words, stride) uint32: MWC64X x / carry rows, or
        the six XORWOW words."""
        words = 2 if self.kind == "mwc64x" else 6
        out = np.zeros(words * self.stride, np.uint32)
        check(lib().gasp_rng_read_states(self._h, out, out.size), "gasp_rng_read_states")
        return out.reshape(words, self.stride)

    def close(self):
        if self._h:
            lib().gasp_free_rand(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class DeviceGrids:
    """A device-resident set of ngrids LxL replicas (bit-packed)."""

    def __init__(self, L, ngrids, host_grids=None, threads_per_block=32):
        self.L, self.ngrids = int(L), int(ngrids)
        self._h = C.c_void_p()
        check(lib().gasp_init_grid(self.L, self.ngrids, threads_per_block, None,
                                   C.byref(self._h)), "gasp_init_grid")
        if host_grids is not None:
            self.upload(host_grids)

    @property
    def handle(self):
        return self._h

    def upload(self, grids):
        g = np.ascontiguousarray(grids, dtype=np.int32).reshape(-1)
        if g.size != self.L * self.L * self.ngrids:
            raise ValueError("grid array has the wrong size")
        check(lib().gasp_grids_upload(self._h, g), "gasp_grids_upload")

    def upload_inputs(self, inputs):
        """Replica r starts from inputs[r // (ngrids // len(inputs))]
        (init_grids_from_array); only the distinct inputs are copied."""
        x = np.ascontiguousarray(inputs, dtype=np.int32).reshape(-1, self.L * self.L)
        check(lib().gasp_grids_upload_inputs(self._h, x.reshape(-1), x.shape[0]),
              "gasp_grids_upload_inputs")

    def set_option(self, option, value):
        """Launch tuning, see gasp_grids_set_option.  Results never depend on
        it, except that sweep variant 6 and the committor tail threshold assign
        the MWC64X stream's draws differently (same dynamics)."""
        check(lib().gasp_grids_set_option(self._h, int(option), int(value)), "gasp_grids_set_option")

    def thresholds(self, beta, h):
        """(thr uint32[10], float_compare): the integer acceptance test of the
        sweep kernels, u <= thr[5*(spin up) + (# up neighbours)]."""
        thr = np.zeros(10, np.uint32)
        fc = C.c_int(0)
        check(lib().gasp_acceptance_thresholds(self._h, float(beta), float(h), thr, C.byref(fc)),
              "gasp_acceptance_thresholds")
        return thr, bool(fc.value)

    def download(self):
        out = np.empty(self.L * self.L * self.ngrids, np.int32)
        check(lib().gasp_grids_download(self._h, out), "gasp_grids_download")
        return out.reshape(self.ngrids, self.L, self.L)

    def magnetisation(self):
        out = np.empty(self.ngrids, np.float32)
        check(lib().gasp_magnetisation(self._h, out), "gasp_magnetisation")
        return out

    def largest_cluster(self, spin):
        """Largest periodic 4-connected cluster of `spin` per replica (float32)."""
        out = np.empty(self.ngrids, np.float32)
        check(lib().gasp_largest_cluster(self._h, int(spin), out), "gasp_largest_cluster")
        return out

    def pack_frame(self):
        n = lib().gasp_frame_bytes(self.L, self.ngrids)
        out = np.empty(n, np.uint8)
        check(lib().gasp_pack_frame(self._h, out), "gasp_pack_frame")
        return out

    def sweep(self, rng, beta, h, nsweeps, gpu_method=2):
        check(lib().gasp_sweep(self._h, rng.handle, float(beta), float(h), int(nsweeps),
                               int(gpu_method)), "gasp_sweep")

    def sweep_trace_cpu(self, stream, beta, h, nsweeps):
        s = np.ascontiguousarray(stream, np.float64)
        need = self.ngrids * 3 * self.L * self.L * nsweeps
        if s.size < need:
            raise ValueError(f"trace stream too short ({s.size} < {need})")
        check(lib().gasp_sweep_trace_cpu(self._h, s, float(beta), float(h), int(nsweeps)),
              "gasp_sweep_trace_cpu")

    def close(self):
        if self._h:
            lib().gasp_free_grid(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def run_driver(dgrids, rng, beta, h, tot_nsweeps, mag_output_int, grid_output_int, itask=0,
               dn_thr=-0.9, up_thr=0.9, ninputs=1, host_grids=None, fates=None,
               outfunc=None, packed_out=None, verbosity=0, compact=False,
               threads_per_block=32, gpu_method=2, filename="gridstates.bin", first_up=None,
               cv="magnetisation", initial_spin=-1):
    """Runs gasp_mc_driver_gpu_ex; returns (result, fates, elapsed_s, attempts).

    ``cv``: "magnetisation" or "largest_cluster" (largest cluster of spins
    -initial_spin, compared with the thresholds as a number of sites).
    ``first_up`` (int32[ngrids], optional) receives each replica's first check
    isweep with the cv above up_thr (-1: never).
    ``outfunc(L, ngrids, grids_int32[ngrids,L,L], isweep, mag)`` mirrors the
    reference's GridOutputFunc (with cv "largest_cluster" it gets the cluster
    sizes as a sixth argument); ``packed_out(L, ngrids, payload_u8, isweep,
    mag)`` receives gridstates.bin payloads.  Either returns 0 on success.
    """
    L, ngrids = dgrids.L, dgrids.ngrids
    nres = tot_nsweeps // mag_output_int if itask == 0 else ninputs
    result = np.zeros(max(nres, 1), np.float32)
    if host_grids is None and outfunc is not None:
        host_grids = np.empty((ngrids, L, L), np.int32)
    hg_ptr = None
    if host_grids is not None:
        host_grids = np.ascontiguousarray(host_grids, np.int32)
        hg_ptr = host_grids.ctypes.data_as(C.POINTER(C.c_int))
    if itask == 1 and fates is None:
        fates = np.full(ngrids, -1, np.int32)
    fate_ptr = fates.ctypes.data_as(C.c_void_p) if fates is not None else None

    def _outfunc(L_, ng_, gptr, isweep, magp, lcp, cv, dn, up, fn):
        try:
            g = np.ctypeslib.as_array(gptr, shape=(ng_ * L_ * L_,)).reshape(ng_, L_, L_)
            m = np.ctypeslib.as_array(magp, shape=(ng_,))
            if lcp:
                lc = np.ctypeslib.as_array(lcp, shape=(ng_,))
                return int(outfunc(L_, ng_, g, isweep, m, lc) or 0)
            return int(outfunc(L_, ng_, g, isweep, m) or 0)
        except Exception:  # a Python error stops the driver
            return 1

    def _packed(L_, ng_, payload, nbytes, isweep, magp, user):
        try:
            b = np.ctypeslib.as_array(payload, shape=(nbytes,))
            m = np.ctypeslib.as_array(magp, shape=(ng_,))
            return int(packed_out(L_, ng_, b, isweep, m) or 0)
        except Exception:
            return 1

    cb = nat.GRID_OUTPUT_FN(_outfunc) if outfunc is not None else nat.GRID_OUTPUT_FN()
    pcb = nat.PACKED_OUTPUT_FN(_packed) if packed_out is not None else nat.PACKED_OUTPUT_FN()
    elapsed = C.c_double(0.0)
    attempts = C.c_longlong(0)
    fu_ptr = None
    if first_up is not None:
        assert first_up.dtype == np.int32 and first_up.size >= ngrids and first_up.flags.c_contiguous
        fu_ptr = first_up.ctypes.data_as(C.POINTER(C.c_int))
    opts = nat.DriverOptsT(verbosity, int(bool(compact)), pcb, None,
                           C.pointer(elapsed), C.pointer(attempts), fu_ptr)
    grids_t = nat.GpuGridsT(L, ngrids, hg_ptr, dgrids.handle)
    samp = nat.SamplerT(tot_nsweeps, mag_output_int, grid_output_int)
    calc = nat.FunctionT(itask, dn_thr, up_thr, ninputs, int(initial_spin), cv.encode(),
                         result.ctypes.data_as(C.POINTER(C.c_float)), filename.encode())
    run = nat.GpuRunT(rng.handle, threads_per_block, gpu_method)
    check(lib().gasp_mc_driver_gpu_ex(grids_t, float(beta), float(h), fate_ptr, samp, calc, run,
                                      cb, C.byref(opts)), "gasp_mc_driver_gpu")
    return result[:nres], fates, elapsed.value, attempts.value


# ---- checkpoints and gridstates.bin frames ---------------------------------
_RNG_NAMES = {nat.RNG_XORWOW: "xorwow", nat.RNG_MWC64X: "mwc64x"}


def checkpoint_info(path):
    """Header of a checkpoint: dict(L, ngrids, rng, isweep, has_fates)."""
    v = [C.c_int() for _ in range(5)]
    check(lib().gasp_checkpoint_info(str(path).encode(), *[C.byref(x) for x in v]),
          "gasp_checkpoint_info")
    return {"L": v[0].value, "ngrids": v[1].value, "rng": _RNG_NAMES[v[2].value],
            "isweep": v[3].value, "has_fates": bool(v[4].value)}


def save_checkpoint(path, dgrids, rng, fates=None, isweep=0):
    """Grids, RNG states and (optionally) fates of a run, to one file."""
    fp = None
    if fates is not None:
        fates = np.ascontiguousarray(fates, np.int32)
        assert fates.size == dgrids.ngrids
        fp = fates.ctypes.data_as(C.c_void_p)
    check(lib().gasp_checkpoint_save(str(path).encode(), dgrids.handle, rng.handle, fp,
                                     int(isweep)), "gasp_checkpoint_save")


def load_checkpoint(path, seed=0):
    """New (DeviceGrids, RngStates, fates or None, isweep) from a checkpoint;
    every replica continues its trajectory exactly."""
    info = checkpoint_info(path)
    dg = DeviceGrids(info["L"], info["ngrids"])
    rng = RngStates(info["ngrids"], seed, kind=info["rng"])
    fates = np.empty(info["ngrids"], np.int32)
    isweep = C.c_int()
    check(lib().gasp_checkpoint_load(str(path).encode(), dg.handle, rng.handle,
                                     fates.ctypes.data_as(C.c_void_p), C.byref(isweep)),
          "gasp_checkpoint_load")
    return dg, rng, (fates if info["has_fates"] else None), isweep.value


def read_frame(path, iframe, grids=True):
    """Frame `iframe` of a gridstates.bin file: (L, ngrids, isweep, int32
    grids [ngrids, L, L] or None).  Host only."""
    L, ng, isw = C.c_int(), C.c_int(), C.c_int()
    check(lib().gasp_read_frame(str(path).encode(), int(iframe), C.byref(L), C.byref(ng),
                                C.byref(isw), None, 0), "gasp_read_frame")
    if not grids:
        return L.value, ng.value, isw.value, None
    out = np.empty((ng.value, L.value, L.value), np.int32)
    check(lib().gasp_read_frame(str(path).encode(), int(iframe), C.byref(L), C.byref(ng),
                                C.byref(isw), out.ctypes.data_as(C.c_void_p), out.size),
          "gasp_read_frame")
    return L.value, ng.value, isw.value, out


def write_input_grid(path, grid):
    """One LxL grid (+1/-1) as gridinput.bin.  Host only."""
    g = np.ascontiguousarray(grid, np.int32)
    assert g.ndim == 2 and g.shape[0] == g.shape[1]
    check(lib().gasp_write_input_grid(str(path).encode(), g.shape[0], g.reshape(-1)),
          "gasp_write_input_grid")
