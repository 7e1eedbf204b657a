"""Generates the CPU golden fixtures in tests/golden/ from the reference's own
CPU code, compiled unmodified into oracle/_ref/ (``make -C oracle ref``).

    python tests/golden/make_golden.py

Fixtures (numpy .npz, small):
  ref_cpu_tables.npz   preComputeProbs_cpu (src/mc_cpu.c:14-38) for several (beta, h)
  ref_cpu_driver.npz   mc_driver_cpu runs (src/mc_cpu.c:106-308) seeded with
                       init_genrand: result, fates, callback frames, final grids
  ref_bootstrap.npz    bootstrap_errbar (src/bootstrap.c:6-65) after srand(1)
  ref_cluster.npz      compute_largest_cluster_cpu (src/mc_cpu.c:310-364) of
                       seeded grids (random densities around the percolation
                       threshold, wrapping stripes, checkerboards), both spins

    python tests/golden/make_golden.py cluster   # only ref_cluster.npz

The GPU parity tests compare with the reference's GPU kernels directly
(oracle/_ref/libref_gpu.so) instead of GPU fixtures.
"""
import ctypes as C
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, REPO)

import oracle  # noqa: E402

i32 = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
f32 = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
f64 = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")

TABLE_CASES = [(0.54, 0.07), (0.45, 0.03), (0.60, 0.12), (0.3, 0.0), (1.0, -0.5), (3.0, 0.4)]

# (name, L, ngrids, seed, beta, h, tot, mag, grid, itask, dn, up, ninputs, init)
DRIVER_CASES = [
    ("swarm_L16", 16, 6, 12345, 0.54, 0.07, 60, 10, 20, 0, -0.9, 0.9, 1, "down"),
    ("swarm_L16_fast", 16, 7, 31337, 0.50, 0.30, 120, 10, 30, 0, -0.9, -0.5, 1, "down"),
    ("swarm_L8_hot", 8, 5, 777, 0.30, 0.50, 40, 5, 10, 0, -0.9, 0.5, 1, "down"),
    ("swarm_L12_mixed", 12, 3, 4242, 0.40, 0.20, 45, 15, 9, 0, -0.9, 0.2, 1, "random"),
    ("committor_L16", 16, 8, 99, 0.54, 0.07, 400, 10, 50, 1, -0.93, 0.5, 2, "droplet"),
    ("committor_L10", 10, 6, 2024, 0.45, 0.10, 150, 5, 25, 1, -0.7, 0.2, 3, "droplet"),
]


def load_ref():
    p = os.path.join(REPO, "oracle", "_ref", "libref_cpu.so")
    lib = C.CDLL(p)
    lib.ref_driver_cpu.argtypes = [C.c_int, C.c_int, C.c_ulong, C.c_double, C.c_double, C.c_int,
                                   C.c_int, C.c_int, C.c_int, C.c_double, C.c_double, C.c_int,
                                   i32, C.c_void_p, f32, C.c_int, C.c_void_p, C.c_void_p,
                                   C.c_void_p]
    lib.ref_precompute_probs_cpu.argtypes = [C.c_double, C.c_double, f64]
    lib.ref_bootstrap_errbar.argtypes = [C.c_int, C.c_int, i32]
    lib.ref_bootstrap_errbar.restype = C.c_double
    return lib


def initial_grids(L, ngrids, ninputs, init, seed):
    rng = np.random.default_rng(seed)
    if init == "down":
        return -np.ones((ngrids, L, L), np.int32)
    if init == "random":
        return np.where(rng.random((ngrids, L, L)) < 0.5, 1, -1).astype(np.int32)
    # ninputs droplet inputs, each copied into ngrids/ninputs contiguous grids
    per = ngrids // ninputs
    out = []
    yy, xx = np.mgrid[0:L, 0:L]
    for m in range(ninputs):
        r = 3.0 + m
        g = np.where((yy - L / 2) ** 2 + (xx - L / 2) ** 2 <= r * r, 1, -1).astype(np.int32)
        out += [g] * per
    return np.stack(out).astype(np.int32)


def run_driver(lib, case):
    (name, L, ng, seed, beta, h, tot, mag, grid, itask, dn, up, ninputs, init) = case
    grids = initial_grids(L, ng, ninputs, init, seed)
    g = grids.reshape(-1).copy()
    fates = np.full(ng, -1, np.int32)
    nres = tot // mag if itask == 0 else ninputs
    result = np.zeros(max(nres, 1), np.float32)
    maxf = tot // min(mag, grid) + 2
    fg = np.zeros(maxf * ng * L * L, np.int32)
    fi = np.zeros(maxf, np.int32)
    fm = np.zeros(maxf * ng, np.float32)
    ncalls = lib.ref_driver_cpu(L, ng, seed, beta, h, tot, mag, grid, itask, dn, up, ninputs, g,
                                fates.ctypes.data if itask == 1 else None, result, maxf,
                                fg.ctypes.data, fi.ctypes.data, fm.ctypes.data)
    n = min(ncalls, maxf)
    return dict(L=L, ngrids=ng, seed=seed, beta=beta, h=h, tot=tot, mag=mag, grid=grid,
                itask=itask, dn=dn, up=up, ninputs=ninputs,
                initial=grids.astype(np.int8), final=g.reshape(ng, L, L).astype(np.int8),
                result=result[:nres], fates=fates,
                frame_isweep=fi[:n], frame_grids=fg[:n * ng * L * L].reshape(n, ng, L, L).astype(np.int8),
                frame_mag=fm[:n * ng].reshape(n, ng))


CLUSTER_LS = [2, 3, 5, 8, 16, 31, 64]


def cluster_grids(L, seed):
    """Seeded grids whose clusters wrap, percolate, or are all singletons."""
    rng = np.random.default_rng(seed)
    out = [np.where(rng.random((L, L)) < p, 1, -1) for p in (0.3, 0.5, 0.593, 0.7)]
    out.append(np.ones((L, L)))
    out.append(-np.ones((L, L)))
    stripe = -np.ones((L, L))
    stripe[L // 2, :] = 1  # one row: wraps around in x
    out.append(stripe)
    y, x = np.indices((L, L))
    out.append(np.where((x + y) % 2 == 0, 1, -1))  # checkerboard (odd L: seam)
    return np.stack(out).astype(np.int32)


def make_cluster(lib):
    lib.compute_largest_cluster_cpu.argtypes = [C.c_int, i32, C.c_int, C.c_int, f32]
    out = {"Ls": np.array(CLUSTER_LS)}
    for L in CLUSTER_LS:
        g = cluster_grids(L, 1000 + L)
        res = np.zeros((2, g.shape[0]), np.float32)
        flat = np.ascontiguousarray(g.reshape(-1))
        for k, spin in enumerate((1, -1)):
            for i in range(g.shape[0]):
                lib.compute_largest_cluster_cpu(L, flat, i, spin, res[k])
        out[f"L{L}_grids"] = g.astype(np.int8)
        out[f"L{L}_sizes"] = res  # [spin +1, spin -1][grid]
    np.savez_compressed(os.path.join(HERE, "ref_cluster.npz"), **out)


def main():
    lib = load_ref()
    make_cluster(lib)
    if sys.argv[1:] == ["cluster"]:
        print("ref_cluster.npz written to", HERE)
        return
    tabs = []
    for beta, h in TABLE_CASES:
        P = np.zeros(20, np.float64)
        lib.ref_precompute_probs_cpu(beta, h, P)
        tabs.append(P)
    np.savez_compressed(os.path.join(HERE, "ref_cpu_tables.npz"),
                        cases=np.array(TABLE_CASES), pacc=np.array(tabs))

    out = {}
    for case in DRIVER_CASES:
        d = run_driver(lib, case)
        for k, v in d.items():
            out[f"{case[0]}__{k}"] = np.asarray(v)
    out["names"] = np.array([c[0] for c in DRIVER_CASES])
    np.savez_compressed(os.path.join(HERE, "ref_cpu_driver.npz"), **out)

    rng = np.random.default_rng(5)
    fates_list, errs = [], []
    for n in (10, 37, 256):
        f = rng.choice([-1, 0, 1], size=n, p=[0.1, 0.5, 0.4]).astype(np.int32)
        oracle.lib().orc_srand(1)
        errs.append(lib.ref_bootstrap_errbar(n, n, f))
        fates_list.append(f)
    np.savez_compressed(os.path.join(HERE, "ref_bootstrap.npz"),
                        **{f"fates{i}": f for i, f in enumerate(fates_list)},
                        errbar=np.array(errs))
    print("golden CPU fixtures written to", HERE)


if __name__ == "__main__":
    main()
