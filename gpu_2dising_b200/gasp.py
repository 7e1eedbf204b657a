"""Drop-in mirror of the reference's PyGASP module ``gasp``
(src/ising_ext.cu:522-1264), running on the gasp-b200 CUDA library.

    from gpu_2dising_b200 import gasp
    frac = gasp.run_nucleation_swarm(64, 1024, 10000, 0.54, 0.07)
    pB = gasp.run_committor_calc(64, 1024, 20000, 0.54, 0.07, grid_input="NumPy",
                                 grid_array=[g0, g1])

Same entry points, keyword names, defaults, validation errors and return
values; the module-level ``grids`` / ``magnetisation`` / ``largest_cluster``
lists and ``gpu_nsms`` behave as in the reference, and every grid dump is
written to the HDF5 side file (gridstates.hdf5 for swarms, pBgrids.hdf5 for
committor runs, created at the start of each run) by the library's own
writer, which follows the HDF5 file format specification without libhdf5
(src/io.c:132-301).  Differences, all deliberate:

* there is no CPU fallback: without a CUDA device the calls raise;
* a failed HDF5 write stops the run and raises RuntimeError("Error writing
  HDF5 file"); the reference sets the same error and lets its driver run on,
  since it ignores the output callback's return (src/ising_ext.cu:360-366);
* with ``cv='largest_cluster'`` and thresholds below 2 in magnitude a
  UserWarning is issued through ``warnings`` (the reference sets the warning
  as a pending exception, src/ising_ext.cu:572-577);
* ``seed`` (default: the clock, as the reference) and ``compact`` (committor
  runs stop simulating replicas whose fate is decided; pB and fates are
  unchanged) are extra keywords;
* ``grid_input='gridstates.bin'`` reads gridinput.bin, the intended
  behaviour of src/ising_ext.cu:971-972 (the reference dereferences a NULL
  grid_array there).
"""
from __future__ import annotations

import copy
import os
import sys
import time
import warnings

import numpy as np

from . import engine
from ._native import GaspError, check, lib

# ---- module state (src/ising_ext.cu:61-64, :1192-1260) ---------------------
grids: list = []
magnetisation: list = []
largest_cluster: list = []
gpu_nsms: int = 0
_device_error = None

try:
    _dev, gpu_nsms = engine.init_device(-1)
except Exception as e:  # no device: calls raise later, import still works
    _device_error = e


class GridSnapObject:
    """A grid snapshot (src/ising_ext.cu:74-207): isweep, igrid, an int8 LxL
    ``grid`` and the float members magnetisation / lclus_size / committor."""

    __slots__ = ("isweep", "igrid", "_grid", "magnetisation", "lclus_size", "committor")

    def __init__(self, isweep, igrid, grid):
        if not isinstance(grid, np.ndarray):
            raise TypeError("Third argument must be a NumPy array.")
        if grid.dtype != np.int8 or grid.ndim != 2:
            raise TypeError("NumPy array must be 2D with 8-bit integer elements.")
        self.isweep = int(isweep)
        self.igrid = int(igrid)
        self._grid = grid
        self.magnetisation = 0.0
        self.lclus_size = -1.0
        self.committor = -1.0

    @property
    def grid(self):
        return self._grid

    @grid.setter
    def grid(self, value):
        if not isinstance(value, np.ndarray):
            raise TypeError("grid must be a numpy array")
        self._grid = value

    def __deepcopy__(self, memo):
        new = GridSnapObject(self.isweep, self.igrid, self._grid.copy())
        new.magnetisation = self.magnetisation
        new.lclus_size = self.lclus_size
        new.committor = self.committor
        return new

    def __repr__(self):
        return (f"GridSnapObject(isweep={self.isweep}, igrid={self.igrid}, "
                f"magnetisation={self.magnetisation:.4f}, committor={self.committor})")


def _reset_lists():
    """src/ising_ext.cu:216-275: fresh module-level lists."""
    global grids, magnetisation, largest_cluster
    grids = []
    magnetisation = []
    largest_cluster = []


class _History:
    """The grid-output callback of PyGASP, append_grids_list
    (src/ising_ext.cu:280-463): module lists, the HDF5 side file, the
    snapshot store."""

    def __init__(self, keep, maxhist, L, cv="magnetisation", h5file=None):
        self.keep, self.maxhist, self.L = keep, maxhist, L
        self.cv, self.h5file = cv, h5file
        self.ihist = 0
        self.error = None

    def __call__(self, L, ngrids, g, isweep, mag, dn, up, lclus=None):
        magnetisation.append([float(x) for x in mag])
        if lclus is not None:  # recorded only when it is the cv (src/ising_ext.cu:331-357)
            largest_cluster.append([float(x) for x in lclus])
        if self.h5file is not None:  # always written (src/ising_ext.cu:360-366)
            mag32 = np.ascontiguousarray(mag, np.float32)
            lc32 = None if lclus is None else np.ascontiguousarray(lclus, np.float32)
            rc = lib().gasp_write_ising_grids_hdf5(
                L, ngrids, np.ascontiguousarray(g, np.int32).reshape(-1), isweep,
                mag32.ctypes.data, None if lc32 is None else lc32.ctypes.data,
                self.cv.encode(), dn, up, self.h5file.encode())
            if rc != 0:
                self.error = RuntimeError("Error writing HDF5 file")
                return 1
        if not self.keep or self.ihist >= self.maxhist:
            return 0
        snaps = []
        cvv = (mag if lclus is None else lclus).astype(np.float64)
        sel = np.nonzero((cvv > dn) & (cvv < up))[0]
        for i in sel:
            snap = GridSnapObject(isweep, int(i), g[i].astype(np.int8))
            snap.magnetisation = float(mag[i])
            if lclus is not None:
                snap.lclus_size = float(lclus[i])
            snap.committor = -1.0
            snaps.append(snap)
            self.ihist += 1
            if self.ihist == self.maxhist:
                sys.stderr.write("\nWARNING: Maximum history reached, not storing more "
                                 "snapshots to grids object!\n\n")
                self.ihist += 1
                break
        if snaps:
            grids.append(snaps)
        return 0


def _create_h5(L, ngrid, tot_nsweeps, h, beta, itask, path):
    """create_ising_grids_hdf5 at the start of a run (src/ising_ext.cu:659-660,
    :1025-1026); a failure is reported on stderr and the run goes on, as in
    the reference."""
    lib().gasp_create_ising_grids_hdf5(L, ngrid, tot_nsweeps, h, beta, itask, path.encode())


def _run(hist, **kw):
    """engine.run_driver, raising the output callback's own error if it stopped
    the run."""
    try:
        return engine.run_driver(**kw)
    except GaspError:
        if hist.error is not None:
            raise hist.error from None
        raise


def _require_device():
    if _device_error is not None:
        raise GaspError(3, f"no CUDA device available ({_device_error})")


def _check_cv(cv, up, dn):
    if cv not in ("magnetisation", "largest_cluster"):
        raise ValueError("cv must be either 'magnetisation' or 'largest_cluster'")
    if cv == "largest_cluster" and (abs(up) < 2.0 or abs(dn) < 2.0):
        warnings.warn("For cv='largest_cluster', up_threshold and dn_threshold should have "
                      "magnitudes >= 2", UserWarning, stacklevel=3)


def _rng_kind(rng):
    if rng not in ("xorwow", "mwc64x"):
        raise ValueError(f"rng must be 'xorwow' or 'mwc64x' (got {rng!r})")
    return rng


def run_nucleation_swarm(L, ngrid, tot_nsweeps, beta, h, initial_spin=-1, cv="magnetisation",
                         up_threshold=0.90, dn_threshold=-0.95, mag_output_int=100,
                         grid_output_int=1000, keep_grids=True, max_keep_grids=0,
                         threadsPerBlock=32, gpu_method=0, seed=None, verbose=False,
                         rng="xorwow"):
    """Simulate a swarm of ngrid LxL replicas from a uniform ``initial_spin``
    start; returns float32[tot_nsweeps // mag_output_int], the fraction of
    replicas with cv > up_threshold at each check (src/ising_ext.cu:522-743).
    Default thresholds are those of the reference (computed there from the
    default initial_spin=-1: up 0.90, dn -0.95).  rng: "xorwow" (the
    reference's cuRAND stream, bit-identical trajectories) or "mwc64x" (the
    production stream: statistically equivalent, faster)."""
    _check_cv(cv, up_threshold, dn_threshold)
    if max_keep_grids < 0:
        raise ValueError("max_keep_grids must be a positive integer")
    _require_device()
    _rng_kind(rng)
    if os.path.exists("gridstates.bin"):
        os.remove("gridstates.bin")
    _reset_lists()
    nsnaps = tot_nsweeps // grid_output_int + 1
    maxhist = max_keep_grids if max_keep_grids else nsnaps * ngrid
    hist = _History(bool(keep_grids), maxhist, L, cv, "gridstates.hdf5")
    host = np.full((ngrid, L, L), int(initial_spin), np.int32)
    engine.select_gpu_method(L, ngrid, threadsPerBlock)  # evaluated, then ignored (as :678)
    seed = int(time.time()) if seed is None else int(seed)
    _create_h5(L, ngrid, tot_nsweeps, h, beta, 0, hist.h5file)
    dg = engine.DeviceGrids(L, ngrid, host)
    rng = engine.RngStates(ngrid, seed, kind=_rng_kind(rng))
    try:
        res, _, _, _ = _run(
            hist, dgrids=dg, rng=rng, beta=beta, h=h, tot_nsweeps=tot_nsweeps,
            mag_output_int=mag_output_int, grid_output_int=grid_output_int, itask=0,
            dn_thr=dn_threshold, up_thr=up_threshold, host_grids=host,
            outfunc=lambda L_, ng_, g, isweep, m, *lc: hist(L_, ng_, g, isweep, m, dn_threshold,
                                                             up_threshold, *lc),
            verbosity=2 if verbose else 0, threads_per_block=threadsPerBlock, cv=cv,
            initial_spin=initial_spin)
    finally:
        dg.close()
        rng.close()
    return np.asarray(res, np.float32)


def run_committor_calc(L, ngrid, tot_nsweeps, beta, h, initial_spin=-1, cv="magnetisation",
                       up_threshold=0.90, dn_threshold=-0.93, mag_output_int=100,
                       grid_output_int=1000, keep_grids=True, max_keep_grids=0,
                       threadsPerBlock=32, gpu_method=0, grid_input="gridstates.bin",
                       grid_array=None, nsms=None, seed=None, compact=False, verbose=False,
                       rng="xorwow"):
    """Committor pB of each input grid by shooting ngrid/len(grid_array)
    trajectories per input until cv > up_threshold (B) or < dn_threshold (A);
    returns [(pB, bootstrap error), ...] (src/ising_ext.cu:805-1130).  rng as
    for run_nucleation_swarm."""
    global gpu_nsms
    if nsms is None:
        nsms = gpu_nsms
    if nsms < 0:
        raise ValueError("nsms must be a non-negative integer")
    gpu_nsms = nsms
    _check_cv(cv, up_threshold, dn_threshold)
    if max_keep_grids < 0:
        raise ValueError("max_keep_grids must be a non-negative integer")
    count = 1
    if grid_array is not None:
        if not isinstance(grid_array, list):
            raise TypeError("grid_array must be a list of 2D NumPy arrays")
        count = len(grid_array)
        if count > gpu_nsms:
            raise ValueError("grid_array list length exceeds gpu_nsms")
        if count == 0:
            raise ValueError("grid_array list is empty")
        if gpu_nsms % count != 0:
            raise ValueError("grid_array list length must divide gpu_nsms exactly")
        if ngrid % gpu_nsms != 0:
            raise ValueError("ngrids must be a multiple of gpu_nsms")
        if ngrid % count != 0:
            raise ValueError("ngrids must be a multiple of grid_array list length")
        arrs = []
        for a in grid_array:
            if not isinstance(a, np.ndarray):
                raise TypeError("All items in grid_array must be NumPy arrays")
            if a.dtype != np.int8 or a.ndim != 2:
                raise TypeError("Each grid_array item must be a 2D NumPy array of type int8")
            if a.shape != (L, L):
                raise ValueError("Each grid_array item must have shape LxL")
            arrs.append(a.astype(np.int32))
    _require_device()
    _rng_kind(rng)
    if os.path.exists("gridstates.bin"):
        os.remove("gridstates.bin")
    _reset_lists()
    nsnaps = tot_nsweeps // grid_output_int + 1
    maxhist = max_keep_grids if max_keep_grids else nsnaps * ngrid
    hist = _History(bool(keep_grids), maxhist, L, cv, "pBgrids.hdf5")
    host = np.empty((ngrid, L, L), np.int32)
    if grid_input == "gridstates.bin":
        rc = lib().gasp_init_grids_from_file(b"gridinput.bin", L, ngrid, host.reshape(-1))
        check(rc, "reading gridinput.bin")
        count = 1
    elif grid_input == "NumPy" and grid_array is not None:
        check(lib().gasp_init_grids_from_array(L, ngrid, count,
                                               np.ascontiguousarray(np.stack(arrs)).reshape(-1),
                                               host.reshape(-1)), "init_grids_from_array")
    else:
        raise ValueError("Invalid grid_input option or no grid_array supplied")
    fates = np.full(ngrid, -1, np.int32)
    engine.select_gpu_method(L, ngrid, threadsPerBlock)
    seed = int(time.time()) if seed is None else int(seed)
    _create_h5(L, ngrid, tot_nsweeps, h, beta, 1, hist.h5file)
    dg = engine.DeviceGrids(L, ngrid, host)
    rng = engine.RngStates(ngrid, seed, kind=_rng_kind(rng))
    try:
        res, fates, _, _ = _run(
            hist, dgrids=dg, rng=rng, beta=beta, h=h, tot_nsweeps=tot_nsweeps,
            mag_output_int=mag_output_int, grid_output_int=grid_output_int, itask=1,
            dn_thr=dn_threshold, up_thr=up_threshold, ninputs=count, host_grids=host,
            fates=fates, compact=compact,
            outfunc=lambda L_, ng_, g, isweep, m, *lc: hist(L_, ng_, g, isweep, m, dn_threshold,
                                                             up_threshold, *lc),
            verbosity=2 if verbose else 0, threads_per_block=threadsPerBlock, cv=cv,
            initial_spin=initial_spin)
    finally:
        dg.close()
        rng.close()
    sub = ngrid // count
    out = []
    for i in range(count):
        block = np.ascontiguousarray(fates[i * sub:(i + 1) * sub])
        err = lib().gasp_bootstrap_errbar(sub, sub, block)
        if err < 0.0:
            raise RuntimeError("Error calculating bootstrap error bar")
        out.append((float(res[i]), float(err)))
    return out


__all__ = ["run_nucleation_swarm", "run_committor_calc", "GridSnapObject", "grids",
           "magnetisation", "largest_cluster", "gpu_nsms"]

_ = copy  # deepcopy support is through GridSnapObject.__deepcopy__
