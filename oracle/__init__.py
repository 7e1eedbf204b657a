"""CPU oracle for the GASP many-replica Metropolis path.

TEST INFRASTRUCTURE ONLY.  Only tests/, ``__graft_entry__.smoke()`` and the
CPU-baseline / ``--impl reference`` legs of bench.py import this package, and
only as the checker or the timed reference.  The product (``gpu_2dising_b200``)
never imports it.

Contents
--------
* ``liboracle.so`` (``gasp_oracle.c``): a C restatement of the reference's
  acceptance tables, single-replica sweeps (CPU and GPU arithmetic), the two
  magnetisation flavours, the gridstates.bin / gridinput.bin formats and the
  bootstrap error bar, each citing the reference file:line it follows.
* ``_ref/``: the reference's own sources compiled unmodified (``make ref``):
  ``libref_cpu.so`` (mc_cpu.c + mt19937ar.c + grid.c + bootstrap.c),
  ``libref_cpu_replay.so`` (mc_cpu.c driven by a replayed ``genrand_real3``
  stream), ``ref_cpu_bench`` and ``libref_gpu.so`` (mc_gpu.cu + gpu_tools.cu
  for sm_100a).
* Python restatements of the two drivers' check/dump/result timing
  (src/mc_cpu.c:189-267, src/mc_gpu.cu:654-778) used to validate the product
  driver on small cases.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass, field

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")

_i32p = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_f32p = np.ctypeslib.ndpointer(dtype=np.float32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_u8p = np.ctypeslib.ndpointer(dtype=np.uint8, flags="C_CONTIGUOUS")
_u32p = np.ctypeslib.ndpointer(dtype=np.uint32, flags="C_CONTIGUOUS")
_u64p = np.ctypeslib.ndpointer(dtype=np.uint64, flags="C_CONTIGUOUS")

_lib = None


def lib():
    """The restatement library (built by ``make -C oracle``)."""
    global _lib
    if _lib is None:
        path = os.path.join(HERE, "liboracle.so")
        if not os.path.exists(path):
            raise RuntimeError(f"oracle not built: {path} (run make -C oracle)")
        L = C.CDLL(path)
        L.orc_probs_cpu.argtypes = [C.c_double, C.c_double, _f64p]
        L.orc_probs_gpu.argtypes = [C.c_double, C.c_double, _f32p]
        L.orc_sweep_cpu_stream.argtypes = [C.c_int, _i32p, C.c_longlong, _f64p, _f64p]
        L.orc_sweep_cpu_stream.restype = C.c_longlong
        L.orc_sweep_gpu_stream.argtypes = [C.c_int, _i32p, C.c_longlong, _f32p, _f32p]
        L.orc_sweep_gpu_stream.restype = C.c_longlong
        L.orc_magnetisation_gpu.argtypes = [C.c_int, _i32p]
        L.orc_magnetisation_gpu.restype = C.c_float
        L.orc_magnetisation_cpu.argtypes = [C.c_int, _i32p]
        L.orc_magnetisation_cpu.restype = C.c_float
        L.orc_largest_cluster.argtypes = [C.c_int, _i32p, C.c_int]
        L.orc_largest_cluster.restype = C.c_int
        L.orc_pack_frame.argtypes = [C.c_int, C.c_int, _i32p, _u8p]
        L.orc_pack_frame.restype = C.c_longlong
        L.orc_unpack_frame.argtypes = [C.c_int, C.c_int, _u8p, _i32p]
        L.orc_write_frame.argtypes = [C.c_char_p, C.c_int, C.c_int, _i32p, C.c_int]
        L.orc_read_input_grid.argtypes = [C.c_char_p, C.c_int, C.c_int, _i32p]
        L.orc_bootstrap_errbar.argtypes = [C.c_int, C.c_int, _i32p]
        L.orc_bootstrap_errbar.restype = C.c_double
        L.orc_srand.argtypes = [C.c_uint]
        L.orc_committor_from_fates.argtypes = [C.c_int, C.c_int, _i32p, _f32p]
        L.orc_sweep_mwc.argtypes = [C.c_int, _i32p, C.c_longlong, C.POINTER(C.c_uint32),
                                    C.POINTER(C.c_uint32), _u32p]
        L.orc_sweep_mwc.restype = C.c_longlong
        L.orc_sweep_tail.argtypes = [C.c_int, _i32p, C.c_int, C.POINTER(C.c_uint32),
                                     C.POINTER(C.c_uint32), _u32p, _u64p, _u64p, C.c_void_p]
        L.orc_sweep_tail.restype = C.c_longlong
        L.orc_sweep_shared.argtypes = [C.c_int, C.c_int, _i32p, C.c_int, _u32p, _u32p, _u32p]
        L.orc_sweep_shared.restype = C.c_longlong
        _lib = L
    return _lib


# --------------------------------------------------------------------------
# thin numpy wrappers
# --------------------------------------------------------------------------
def probs_cpu(beta, h):
    P = np.zeros(20, np.float64)
    lib().orc_probs_cpu(beta, h, P)
    return P


def probs_gpu(beta, h):
    P = np.zeros(20, np.float32)
    lib().orc_probs_gpu(beta, h, P)
    return P


def sweep_cpu_stream(L, grid, stream, P):
    """In-place sweep of one int32 grid with CPU arithmetic (3 doubles/attempt)."""
    stream = np.ascontiguousarray(stream, np.float64)
    n = stream.size // 3
    lib().orc_sweep_cpu_stream(L, grid, n, stream, np.ascontiguousarray(P, np.float64))
    return n


def sweep_gpu_stream(L, grid, ustream, P):
    """In-place sweep of one int32 grid with GPU arithmetic (2 floats/attempt)."""
    ustream = np.ascontiguousarray(ustream, np.float32)
    n = ustream.size // 2
    lib().orc_sweep_gpu_stream(L, grid, n, ustream, np.ascontiguousarray(P, np.float32))
    return n


def sweep_mwc(L, grid, nattempts, x, c, thr):
    """In-place sweep of one int32 grid on one MWC64X stream (production
    row kernels); returns the stream state (x, c) afterwards."""
    xs, cs = C.c_uint32(int(x)), C.c_uint32(int(c))
    lib().orc_sweep_mwc(L, grid, int(nattempts), C.byref(xs), C.byref(cs),
                        np.ascontiguousarray(thr, np.uint32))
    return xs.value, cs.value


def sweep_tail(L, grid, nsweeps, x, c, thr, mul, inv, record=False):
    """In-place one-warp-per-replica sweep (variant 6) of one int32 grid,
    restated serially; returns (x, c) afterwards and, with record=True, the
    applied (site, u) pairs in order as uint32[n, 2]."""
    xs, cs = C.c_uint32(int(x)), C.c_uint32(int(c))
    order = np.zeros((nsweeps * L * L, 2), np.uint32) if record else None
    n = lib().orc_sweep_tail(L, grid, int(nsweeps), C.byref(xs), C.byref(cs),
                             np.ascontiguousarray(thr, np.uint32),
                             np.ascontiguousarray(mul, np.uint64),
                             np.ascontiguousarray(inv, np.uint64),
                             order.ctypes.data_as(C.c_void_p) if record else None)
    assert n == nsweeps * L * L
    return (xs.value, cs.value, order) if record else (xs.value, cs.value)


def sweep_shared(L, grids, nsweeps, x, c, thr):
    """In-place shared-site sweep (variant 7) of one tile of <= 32 int32
    grids; returns the streams (x, c) afterwards as uint32 arrays."""
    g = np.ascontiguousarray(grids, np.int32)
    assert g.ndim == 3 and g.shape[0] <= 32
    xs = np.array(x, np.uint32)
    cs = np.array(c, np.uint32)
    lib().orc_sweep_shared(L, g.shape[0], g.reshape(-1), int(nsweeps), xs, cs,
                           np.ascontiguousarray(thr, np.uint32))
    grids[...] = g
    return xs, cs


def magnetisation_gpu(L, grids):
    g = np.ascontiguousarray(grids, np.int32).reshape(-1, L * L)
    return np.array([lib().orc_magnetisation_gpu(L, np.ascontiguousarray(x)) for x in g], np.float32)


def magnetisation_cpu(L, grids):
    g = np.ascontiguousarray(grids, np.int32).reshape(-1, L * L)
    return np.array([lib().orc_magnetisation_cpu(L, np.ascontiguousarray(x)) for x in g], np.float32)


def largest_cluster(L, grids, spin):
    """Largest cluster size of `spin` per grid (float32, as the reference)."""
    g = np.ascontiguousarray(grids, np.int32).reshape(-1, L * L)
    return np.array([lib().orc_largest_cluster(L, np.ascontiguousarray(x), int(spin)) for x in g],
                    np.float32)


def pack_frame(L, grids):
    g = np.ascontiguousarray(grids, np.int32).reshape(-1)
    ngrids = g.size // (L * L)
    out = np.zeros((g.size + 7) // 8, np.uint8)
    lib().orc_pack_frame(L, ngrids, g, out)
    return out


def unpack_frame(L, ngrids, payload):
    out = np.zeros(L * L * ngrids, np.int32)
    lib().orc_unpack_frame(L, ngrids, np.ascontiguousarray(payload, np.uint8), out)
    return out.reshape(ngrids, L, L)


def write_frame(path, L, grids, isweep):
    g = np.ascontiguousarray(grids, np.int32).reshape(-1)
    return lib().orc_write_frame(path.encode(), L, g.size // (L * L), g, isweep)


def read_input_grid(path, L, ngrids):
    out = np.zeros(L * L * ngrids, np.int32)
    rc = lib().orc_read_input_grid(path.encode(), L, ngrids, out)
    return rc, out.reshape(ngrids, L, L)


def bootstrap_errbar(fates, m=None, seed=1):
    f = np.ascontiguousarray(fates, np.int32)
    lib().orc_srand(seed)
    return lib().orc_bootstrap_errbar(f.size, f.size if m is None else m, f)


def committor_from_fates(fates, ninputs):
    f = np.ascontiguousarray(fates, np.int32)
    out = np.zeros(ninputs, np.float32)
    lib().orc_committor_from_fates(f.size, ninputs, f, out)
    return out


def read_gridstates(path):
    """Parse a gridstates.bin file into [(L, ngrids, isweep, int32[ngrids,L,L])]
    following src/io.c:84-120 (one header + ceil(L*L*ngrids/8) bytes/frame)."""
    raw = np.fromfile(path, dtype=np.uint8)
    frames, pos = [], 0
    while pos + 12 <= raw.size:
        L, ng, isw = np.frombuffer(raw[pos:pos + 12].tobytes(), np.int32)
        nbytes = (int(L) * int(L) * int(ng) + 7) // 8
        payload = raw[pos + 12:pos + 12 + nbytes]
        frames.append((int(L), int(ng), int(isw), unpack_frame(int(L), int(ng), payload)))
        pos += 12 + nbytes
    return frames


# --------------------------------------------------------------------------
# MT19937 stream identical to the reference's init_genrand + genrand_real3
# (src/mt19937ar.c).  numpy's legacy RandomState(seed) seeds with the same
# init_genrand and its full-range uint32 draws are raw genrand_int32 outputs;
# tests pin this against the compiled reference (oracle/_ref).
# --------------------------------------------------------------------------
def mt_real3_stream(seed, n):
    rs = np.random.RandomState(int(seed) & 0xFFFFFFFF)
    x = rs.randint(0, 2 ** 32, size=n, dtype=np.uint64).astype(np.uint32)
    return (x.astype(np.float64) + 0.5) * (1.0 / 4294967296.0)


def mt_int32_stream(seed, n):
    rs = np.random.RandomState(int(seed) & 0xFFFFFFFF)
    return rs.randint(0, 2 ** 32, size=n, dtype=np.uint64).astype(np.uint32)


# --------------------------------------------------------------------------
# Driver restatements (check / dump / result timing)
# --------------------------------------------------------------------------
@dataclass
class DriverTrace:
    result: np.ndarray
    lines: list = field(default_factory=list)          # (isweep, fraction) printed
    dumps: list = field(default_factory=list)          # (isweep, grids copy, mag copy)
    mags: list = field(default_factory=list)           # (isweep, mag) per computed check
    fates: np.ndarray | None = None
    last_isweep: int = 0


def driver_cpu_semantics(grids, sweep_batch, mag_fn, tot, mag_int, grid_int, itask=0,
                         up=0.9, dn=-0.9, ninputs=1, fates=None):
    """Restatement of mc_driver_cpu's loop (src/mc_cpu.c:189-303).

    Order per iteration: check (magnetisation of all replicas, count or fate
    update, break) when isweep % mag_int == 0; dump when isweep % grid_int
    == 0; then ``sweep_batch(grids, batch_index, nsweeps)`` advances every
    replica in index order.  The CPU flavour has no ``isweep == tot-1``
    clauses and computes the magnetisation in double (src/mc_cpu.c:91-104).
    """
    ngrids = grids.shape[0]
    spc = min(mag_int, grid_int)
    if itask == 0:
        result = np.ones(tot // mag_int, np.float32)
    else:
        result = np.zeros(ninputs, np.float32)
        fates = np.full(ngrids, -1, np.int32) if fates is None else fates
    tr = DriverTrace(result=result, fates=fates)
    mag = np.zeros(ngrids, np.float32)
    isweep, batch = 0, 0
    while isweep < tot:
        if isweep % mag_int == 0:
            mag = mag_fn(grids)
            tr.mags.append((isweep, mag.copy()))
            m64 = mag.astype(np.float64)
            if itask == 0:
                nnuc = int(np.count_nonzero(m64 > up))
                tr.lines.append((isweep, nnuc / ngrids))
                result[isweep // mag_int] = np.float32(nnuc / ngrids)
                if nnuc == ngrids:
                    break
            else:
                pend = fates == -1
                fates[pend & (m64 > up)] = 1
                fates[pend & ~(m64 > up) & (m64 < dn)] = 0
                if int(np.count_nonzero(fates != -1)) == ngrids:
                    break
        if isweep % grid_int == 0:
            tr.dumps.append((isweep, grids.copy(), mag.copy()))
        sweep_batch(grids, batch, spc)
        batch += 1
        tr.last_isweep = isweep
        isweep += spc
    if itask == 1:
        sub = ngrids // ninputs
        for i in range(ninputs):
            f = fates[i * sub:(i + 1) * sub]
            nB = int(np.sum(f[f > -1]))
            nF = int(np.count_nonzero(f == -1))
            result[i] = np.float32(nB) / np.float32(sub - nF)
    return tr


class MTReal3:
    """Sequential genrand_real3 draws after init_genrand(seed)."""

    def __init__(self, seed):
        self.rs = np.random.RandomState(int(seed) & 0xFFFFFFFF)

    def take(self, n):
        x = self.rs.randint(0, 2 ** 32, size=n, dtype=np.uint64).astype(np.uint32)
        return (x.astype(np.float64) + 0.5) * (1.0 / 4294967296.0)

    def batch(self, ngrids, L, spc):
        """The doubles mc_driver_cpu consumes in one sweep batch: replicas in
        index order, 3 per attempt (src/mc_cpu.c:262-264, :51-52, :77).
        Shape [ngrids, 3*L*L*spc]."""
        return self.take(ngrids * 3 * L * L * spc).reshape(ngrids, 3 * L * L * spc)


def driver_gpu_semantics(grids, sweep, mag_fn, tot, mag_int, grid_int, itask=0,
                         up=0.9, dn=-0.9, ninputs=1, fates=None):
    """Restatement of mc_driver_gpu's loop (src/mc_gpu.cu:620-827).

    ``sweep(grids, nsweeps)`` advances all replicas in place; ``mag_fn(grids)``
    returns float32 magnetisations.  Grid copies for dumps are taken at
    ``isweep % grid_int == 0`` (:658-661); the callback fires at that condition
    or ``isweep == tot-1`` with the last copied grids (:709-711); checks use
    the most recently computed magnetisation (:714-769).
    """
    ngrids = grids.shape[0]
    spc = min(mag_int, grid_int)
    if itask == 0:
        nres = tot // mag_int
        result = np.ones(nres, np.float32)
    else:
        result = np.zeros(ninputs, np.float32)
        fates = np.full(ngrids, -1, np.int32) if fates is None else fates
    tr = DriverTrace(result=result, fates=fates)
    host_copy = grids.copy()
    mag = np.zeros(ngrids, np.float32)
    isweep = 0
    while isweep < tot:
        if isweep % grid_int == 0:
            host_copy = grids.copy()
        if isweep % mag_int == 0:
            mag = mag_fn(grids)
            tr.mags.append((isweep, mag.copy()))
        sweep(grids, spc)
        if isweep % grid_int == 0 or isweep == tot - 1:
            tr.dumps.append((isweep, host_copy.copy(), mag.copy()))
        stop = False
        if isweep % mag_int == 0 or isweep == tot - 1:
            if itask == 0:
                nnuc = int(np.count_nonzero(mag.astype(np.float64) > up))
                idx = isweep // mag_int
                if idx < result.size:
                    result[idx] = np.float32(nnuc / ngrids)
                tr.lines.append((isweep, nnuc / ngrids))
                stop = nnuc == ngrids
            else:
                m64 = mag.astype(np.float64)
                pend = fates == -1
                fates[pend & (m64 > up)] = 1
                fates[pend & ~(m64 > up) & (m64 < dn)] = 0
                stop = int(np.count_nonzero(fates != -1)) == ngrids
        tr.last_isweep = isweep
        if stop:
            break
        isweep += spc
    if itask == 1:
        sub = ngrids // ninputs
        for i in range(ninputs):
            f = fates[i * sub:(i + 1) * sub]
            nB = int(np.sum(f[f > -1]))
            nF = int(np.count_nonzero(f == -1))
            result[i] = np.float32(nB) / np.float32(sub - nF)
    return tr
