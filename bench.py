"""Benchmark of the plain production swarm (L=64, 32768 replicas per GPU,
beta=0.54, h=0.07, all-down start, magnetisation check every 100 sweeps,
grid dump every 1000 sweeps) in the reference-exact mode (gpu_method 2
semantics, cuRAND XORWOW stream).

One step = one check interval: 100 sweeps of every replica (32768 * 4096 *
100 attempted flips) plus the fused magnetisation of the resulting state.

  python bench.py [--gpus N --steps K --warmup W] [--impl reference]
  python bench.py --workload {committor,batched,surrogate,cnn,rate,cluster,tail}

Prints one JSON line on rank 0.  Multi-GPU: replicas are independent, so each
rank runs its own 32768 replicas (weak scaling, no data-path collective); the
timing is the max over ranks.  `--gpus N` without a launcher starts the N
ranks itself (torch.distributed.run on this host); `--dry-run` runs the same
rank plumbing with a host stand-in for the sweep (gloo, no GPU).

The default line (N = 1) also carries
  * cpu_baseline: the reference's own mc_driver_cpu on every host core, on
    the CPU configuration of the same system (L=64, 1248 replicas, 5000
    sweeps, checks every 100);
  * secondary: the committor (64 droplet grids x 4096 shots, both streams,
    pB compared), the uneven batched launch against plain per-group launches,
    the full 50 000-sweep swarm's rate fit (k, t0, both streams) and the
    surrogate-screened committor against shooting alone -- each with its own
    clock record, run in a child process after the timed region.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, REPO)

from gpu_2dising_b200 import shards  # noqa: E402  (replica shards over ranks)

L, R, BETA, H = 64, 32768, 0.54, 0.07
SWEEPS_PER_STEP, MAG_INT, GRID_INT = 100, 100, 1000
SEED = 20240501
OPS_PER_ATTEMPT = 65  # canonical lane-op count of one exact-mode attempt
METRIC = "spin-flip attempts/s"
UNIT = "attempts/s"
CONFIG = {
    "workload": "plain production swarm, gpu_method 2 exact: L=64, 32768 replicas/GPU, "
                "beta=0.54, h=0.07, all-down start; step = 100 sweeps + magnetisation",
    "L": L, "replicas_per_gpu": R, "sweeps_per_step": SWEEPS_PER_STEP,
    "mag_output_int": MAG_INT, "grid_output_int": GRID_INT,
    "rng": "cuRAND XORWOW per replica (reference stream)",
    "l2": "flushed between timed steps (256 MiB device write)",
}
# The CPU configuration of the same system (the reference's mc_driver_cpu):
# L=64, 1248 replicas, 5000 sweeps, magnetisation checked every 100 sweeps.
CPU_CONFIG = {"L": 64, "replicas": 1248, "sweeps": 5000, "mag_output_int": 100}
CPU_MARK_INT = 50  # output-callback interval of the timing harness (step boundaries)


def load_peaks():
    p = os.path.join(REPO, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d.get("sm_max_mhz", 1965.0)), "measured"
    return 1965.0, "fallback"


class ClockSampler:
    """nvidia-smi clock / throttle-reason samples during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *a):
        self.out = ""
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.out, _ = self.proc.communicate(timeout=10)
            except subprocess.TimeoutExpired:
                self.proc.kill()
                self.out, _ = self.proc.communicate()

    def summary(self):
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in (self.out or "").splitlines():
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx.append(float(f[2]))
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx),
                "reasons": sorted(reasons), "samples": len(sm)}


def clocked(fn, *a, **kw):
    """fn(*a, **kw) -> dict, with the clock record of the GPU while it ran."""
    with ClockSampler(int(os.environ.get("LOCAL_RANK", "0"))) as clk:
        out = fn(*a, **kw)
    out["clocks"] = clk.summary()
    return out


def _cpu_cores():
    return sorted(os.sched_getaffinity(0))


def cpu_reference_run(replicas, sweeps, cores=None, seed=SEED):
    """The reference's own CPU driver (oracle/_ref/ref_cpu_bench: mc_cpu.c +
    mt19937ar.c compiled unmodified) on every host core: one process per core
    (its MT19937 state is a process global), each pinned to its core and
    given a contiguous, balanced share of the replicas and its own seed.
    Returns None when the harness is not built, else a dict with the attempts
    made, the wall time and, per process, the callback timestamps (every
    CPU_MARK_INT sweeps) that cut the run into steps."""
    exe = os.path.join(REPO, "oracle", "_ref", "ref_cpu_bench")
    if not os.path.exists(exe):
        return None
    cores = cores or _cpu_cores()
    nproc = max(1, min(len(cores), replicas))
    procs = []
    t0 = time.perf_counter()
    for i in range(nproc):
        _, count = shards.shard_range(replicas, nproc, i)
        core = cores[i % len(cores)]
        procs.append(subprocess.Popen(
            [exe, str(CPU_CONFIG["L"]), str(count), str(sweeps), str(CPU_CONFIG["mag_output_int"]),
             str(BETA), str(H), str(seed + i), str(CPU_MARK_INT)],
            stdout=subprocess.DEVNULL, stderr=subprocess.PIPE, text=True,
            preexec_fn=(lambda c=core: os.sched_setaffinity(0, {c}))))
    attempts, marks, cpu, walls = 0.0, [], [], []
    for p in procs:
        _, err = p.communicate()
        if p.returncode != 0:
            raise RuntimeError(f"ref_cpu_bench failed ({p.returncode}): {err[-300:]}")
        lines = err.strip().splitlines()
        a, w = lines[-3].split()
        attempts += float(a)
        walls.append(float(w))
        f = lines[-2].split()[1:]
        marks.append((float(f[0]), {int(f[i]): float(f[i + 1]) for i in range(1, len(f), 2)}))
        cpu.append(float(lines[-1].split()[1]))
    wall = time.perf_counter() - t0
    return {"attempts": attempts, "wall_s": wall, "cores": nproc, "marks": marks,
            "replicas": replicas, "sweeps": sweeps,
            # CPU time / wall time of the processes: below 1 when a core was shared
            "cpu_share": sum(cpu) / max(sum(walls), 1e-9),
            "loadavg_after": os.getloadavg()[0]}


def cpu_steps(run, steps):
    """Step times of one CPU run cut into `steps` equal sweep ranges: a step
    ends when every process has passed its last sweep (boundaries rounded to
    the callback interval)."""
    sweeps = run["sweeps"]
    bounds = [0] + [int(round(k * sweeps / steps / CPU_MARK_INT)) * CPU_MARK_INT
                    for k in range(1, steps)] + [None]

    def at(b):
        ts = []
        for t_start, m in run["marks"]:
            if b == 0:
                ts.append(t_start)
            elif b is None or b not in m:
                ts.append(max(m.values()))  # the end of that process's run
            else:
                ts.append(m[b])
        return max(ts)

    times = [at(bounds[k + 1]) - at(bounds[k]) for k in range(steps)]
    return [max(t, 0.0) for t in times]


def cpu_config_baseline():
    """cpu_baseline of the JSON line: the CPU configuration run once in full."""
    run = cpu_reference_run(CPU_CONFIG["replicas"], CPU_CONFIG["sweeps"])
    if run is None:
        return None
    return {"value": run["attempts"] / run["wall_s"], "unit": UNIT, "cores": run["cores"],
            "kind": "reference", "wall_s": run["wall_s"], "cpu_share": run["cpu_share"],
            "sample": (f"the CPU configuration: L=64, {run['replicas']} replicas, "
                       f"{run['sweeps']} sweeps, checks every {CPU_CONFIG['mag_output_int']}, "
                       f"beta={BETA}, h={H}, all-down; {run['cores']} processes (one per core, "
                       "pinned), mc_driver_cpu unmodified")}


def run_reference(args, rank, world):
    """The reference arm: the reference's own CPU path (mc_driver_cpu compiled
    unmodified) on all host cores.  The K timed steps are the CPU
    configuration (1248 replicas x 5000 sweeps) run once in full and cut into
    K equal sweep ranges; the W warm-up steps are short runs before it.  The
    line also reports the reference's GPU sweep kernels, compiled unmodified
    for sm_100a, timed on this GPU on the headline workload."""
    if rank != 0:
        return
    for _ in range(args.warmup):
        if cpu_reference_run(len(_cpu_cores()), 100) is None:
            break
    run = cpu_reference_run(CPU_CONFIG["replicas"], CPU_CONFIG["sweeps"])
    if run is None:
        print(json.dumps({"impl": "reference",
                          "unavailable": "oracle/_ref/ref_cpu_bench not built (make -C oracle ref)"}))
        return
    step_s = cpu_steps(run, args.steps)
    value = run["attempts"] / run["wall_s"]
    sample = (f"the CPU configuration (L=64, {run['replicas']} replicas, {run['sweeps']} "
              f"sweeps, checks every {CPU_CONFIG['mag_output_int']}) cut into {args.steps} "
              f"steps; {run['cores']} processes, one per core, mc_driver_cpu unmodified")
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * run["wall_s"] / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "i32",
        "data": "synthetic (all-down L=64 lattices, seeded MT19937 per process)",
        # the same workload as this script's own line (the same system: L=64,
        # beta=0.54, h=0.07, all-down), timed on a bounded sample of it -- the
        # CPU configuration, described by "cpu_config" and the sample text
        "config": CONFIG,
        "cpu_config": {"workload": f"plain reversal on the CPU: L=64, beta=0.54, h=0.07, "
                                   f"all-down, {run['replicas']} replicas, {run['sweeps']} "
                                   f"sweeps, magnetisation checked every "
                                   f"{CPU_CONFIG['mag_output_int']}", **CPU_CONFIG},
        "impl": "reference",
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": run["cores"], "kind": "reference",
                         "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "step_ms": [round(1e3 * t, 3) for t in step_s],
        "wall_s": run["wall_s"], "cpu_share": run["cpu_share"],
    }
    if not args.no_reference_gpu and _gpu_visible():
        line["reference_gpu_kernels"] = reference_gpu_kernels()
    print(json.dumps(line), flush=True)


def _gpu_visible():
    try:
        r = subprocess.run(["nvidia-smi", "-L"], capture_output=True, text=True, timeout=30)
        return r.returncode == 0 and "GPU" in r.stdout
    except (OSError, subprocess.TimeoutExpired):
        return False


def reference_gpu_kernels(calls=5):
    """The reference's own GPU sweep kernels (src/mc_gpu.cu mc_sweep_gpu_bitmap32,
    _bitrep, mc_sweep_gpu; compiled unmodified for sm_100a into
    oracle/_ref/libref_gpu.so) on the headline workload: L=64, 32768 all-down
    replicas, beta=0.54, h=0.07, 100 sweeps per launch, tpb 32 -- the
    reference driver's launch shape.  Device time per launch from CUDA events."""
    import ctypes as C
    path = os.path.join(REPO, "oracle", "_ref", "libref_gpu.so")
    if not os.path.exists(path):
        return {"unavailable": "oracle/_ref/libref_gpu.so not built"}
    try:
        lib = C.CDLL(path)
    except OSError as e:
        return {"unavailable": f"libref_gpu.so did not load: {e}"}
    lib.refgpu_time_kernels.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, C.c_ulonglong,
                                        C.c_double, C.c_double, C.c_int, C.c_int,
                                        C.POINTER(C.c_double)]
    out = {}
    with ClockSampler(int(os.environ.get("LOCAL_RANK", "0"))) as clk:
        for method in (2, 1, 0):
            ms = C.c_double(0.0)
            rc = lib.refgpu_time_kernels(L, R, 32, method, 2024, BETA, H, SWEEPS_PER_STEP, calls,
                                         C.byref(ms))
            if rc != 0:
                out[f"gpu_method_{method}"] = {"error": f"rc {rc}"}
                continue
            out[f"gpu_method_{method}"] = {
                "ms_per_launch": ms.value,
                "attempts_per_s": L * L * R * SWEEPS_PER_STEP / (ms.value / 1e3)}
    return {"what": "reference GPU sweep kernels, unmodified, sm_100a, this GPU",
            "workload": f"L=64, {R} all-down replicas, beta=0.54, h=0.07, {SWEEPS_PER_STEP} "
                        "sweeps per launch, tpb 32", "calls": calls, "methods": out,
            "clocks": clk.summary()}


def read_profile_traffic():
    """DRAM bytes per sweep launch from the committed ncu summary, if any."""
    p = os.path.join(REPO, "profiles", "sweep_exact_L64_R32768.txt")
    if not os.path.exists(p):
        return None
    for ln in open(p):
        if ln.startswith("dram_bytes_per_launch_full_size:"):
            try:
                return float(ln.split(":", 1)[1].split()[0])
            except ValueError:
                return None
    return None


def run_e2e(args, rank, world, dist, torch, engine):
    engine.set_stream(0)
    # the user's initial grids, in pinned host memory
    host = torch.full((R, L, L), -1, dtype=torch.int32).pin_memory().numpy()
    dumped = [0]

    def packed(L_, ng_, payload, isweep, m):
        dumped[0] += payload.size
        return 0

    torch.cuda.synchronize()
    if dist is not None:
        dist.barrier()
    t0 = time.perf_counter()
    dg2 = engine.DeviceGrids(L, R, host)
    t1 = time.perf_counter()
    rng2 = engine.RngStates(R, shards.rank_seed(SEED, rank) + 1, kind=args.rng)
    t2 = time.perf_counter()
    _, _, drv_s, attempts = engine.run_driver(dg2, rng2, BETA, H, SWEEPS_PER_STEP * args.steps,
                                          MAG_INT, GRID_INT, itask=0, dn_thr=-0.9, up_thr=0.9,
                                          packed_out=packed)
    t3 = time.perf_counter()
    torch.cuda.synchronize()
    e2e_s = time.perf_counter() - t0
    e2e_s = shards.max_over_ranks(e2e_s, dist, device="cuda")
    h2d = R * L * L * 4 + 20 * 4 + 20 * 8
    d2h = R * 4 * (SWEEPS_PER_STEP * args.steps // MAG_INT) + dumped[0]
    dg2.close()
    rng2.close()
    return {"value": attempts * world / e2e_s, "unit": UNIT,
            "h2d_bytes_per_step": h2d / args.steps, "d2h_bytes_per_step": d2h / args.steps,
            "wall_s": e2e_s, "upload_s": t1 - t0, "rng_init_s": t2 - t1, "driver_s": drv_s,
            "driver_call_s": t3 - t2,
            "scope": "gasp_init_grid (int32 host grids) + gasp_init_rand + "
                     "gasp_mc_driver_gpu over all steps (per-check magnetisation D2H, "
                     "packed dumps every 1000 sweeps)"}


def _init_dist(world, local_rank, backend):
    if world <= 1:
        return None
    import datetime
    import torch
    import torch.distributed as dist
    kw = {"timeout": datetime.timedelta(seconds=120)}
    if backend == "nccl":
        kw["device_id"] = torch.device("cuda", local_rank)
    dist.init_process_group(backend, **kw)
    return dist


def run_dry(args, rank, world, local_rank):
    """The rank plumbing of the default line without a GPU: each rank times a
    host stand-in step (a numpy bit-count over a seeded lattice stack), the
    step time is the max over ranks, rank 0 prints the line."""
    dist = _init_dist(world, local_rank, "gloo")
    rs = np.random.default_rng(shards.rank_seed(SEED, rank))
    lat = rs.integers(0, 2 ** 32, size=(64, 128), dtype=np.uint64)
    if dist is not None:
        dist.barrier()
    t0 = time.perf_counter()
    pc = 0
    for _ in range(args.steps):
        pc += int(np.unpackbits(lat.view(np.uint8)).sum())
    t = shards.max_over_ranks(time.perf_counter() - t0, dist)
    n = shards.sum_over_ranks(args.steps * lat.size, dist)
    if rank == 0:
        line = {"metric": "dry run: host stand-in words/s", "value": n / max(t, 1e-9),
                "unit": "words/s", "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * t / args.steps,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dry_run": True, "backend": "gloo" if dist is not None else None,
                "world_size": dist.get_world_size() if dist is not None else 1,
                "config": {"workload": "dry run: host stand-in step, no GPU"}}
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


def run_secondary_child(args):
    """The secondary figures, measured in a child process after the timed
    region (its own CUDA context: a failure there cannot take the headline
    line with it)."""
    cmd = [sys.executable, os.path.abspath(__file__), "--workload", "secondary",
           "--rng", "xorwow"]
    if args.secondary_quick:
        cmd.append("--secondary-quick")
    try:
        r = subprocess.run(cmd, capture_output=True, text=True, timeout=args.secondary_timeout)
    except subprocess.TimeoutExpired:
        return {"error": f"secondary measurements exceeded {args.secondary_timeout} s"}
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    if r.returncode != 0 or not lines:
        return {"error": f"rc {r.returncode}: {r.stderr.strip()[-400:]}"}
    return json.loads(lines[-1])


def run_ours(args, rank, world, local_rank):
    # The CPU baseline runs first, before this process starts CUDA and torch's
    # thread pools, so that nothing of ours shares the host cores with it.
    cpu_first = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu_first = cpu_config_baseline()
    import torch
    from gpu_2dising_b200 import engine

    torch.cuda.set_device(local_rank)
    dist = _init_dist(world, local_rank, "nccl")
    engine.init_device(local_rank)
    stream = torch.cuda.Stream()
    engine.set_stream(stream.cuda_stream)
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device="cuda")

    dg = engine.DeviceGrids(L, R, -np.ones((R, L, L), np.int32))
    dg.set_option(1, args.variant)  # GASP_OPT_SWEEP_VARIANT
    rng = engine.RngStates(R, shards.rank_seed(SEED, rank), kind=args.rng)

    def barrier():
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    with torch.cuda.stream(stream):
        for _ in range(args.warmup):
            dg.sweep(rng, BETA, H, SWEEPS_PER_STEP, gpu_method=2)
        barrier()
        evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
               for _ in range(args.steps)]
        with ClockSampler(local_rank) as clk:
            for e0, e1 in evs:
                flush.zero_()
                e0.record(stream)
                dg.sweep(rng, BETA, H, SWEEPS_PER_STEP, gpu_method=2)
                e1.record(stream)
            barrier()
        t_ms = sum(e0.elapsed_time(e1) for e0, e1 in evs)
    t_max = shards.max_over_ranks(t_ms, dist, device="cuda")
    attempts_step = float(R) * L * L * SWEEPS_PER_STEP
    value = attempts_step * args.steps * world / (t_max / 1e3)
    mag = dg.magnetisation()
    assert np.all(np.abs(mag) <= 1.0)
    dg.close()
    rng.close()
    del flush
    torch.cuda.empty_cache()

    # End to end through the public driver (gasp_mc_driver_gpu): host int32
    # grids in, RNG seeding, K check intervals with the per-check
    # magnetisation read back and packed grid dumps, results out.
    e2e = None
    if not args.no_e2e:
        e2e = run_e2e(args, rank, world, dist, torch, engine)
    line = None
    if rank == 0:
        sm_max_mhz, peak_kind = load_peaks()
        peak = 148 * 128 * sm_max_mhz * 1e6 / 1e12       # T lane-ops/s
        launch_s = t_max / 1e3 / args.steps
        achieved = OPS_PER_ATTEMPT * attempts_step / launch_s / 1e12
        traffic = read_profile_traffic()
        if args.rng != "xorwow":
            CONFIG["rng"] = "MWC64X production stream (statistically equivalent, not bit-exact)"
            CONFIG["workload"] = CONFIG["workload"].replace("gpu_method 2 exact", "production RNG")
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": t_max / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u32",
            "data": "synthetic (all-down L=64 lattices, seeded cuRAND streams)",
            "config": CONFIG,
            "roofline": {"bound": "int-issue", "achieved": achieved, "peak": peak,
                         "unit": "Tlane-op/s", "frac": achieved / peak, "traffic": traffic,
                         "ops_per_attempt": OPS_PER_ATTEMPT,
                         "peak_basis": f"148 SMs x 128 lanes x {sm_max_mhz:.0f} MHz "
                                       f"({peak_kind} sm_max_mhz)"},
            "cpu_baseline": None,
            "e2e": e2e,
            "gpu_launches": args.steps,
            "clocks": clk.summary(),
        }
        if dist is not None:
            line["nccl_world"] = dist.get_world_size()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        # after the timed region and after the other ranks are done
        line["cpu_baseline"] = cpu_first
        if world == 1 and not args.no_secondary:
            line["secondary"] = run_secondary_child(args)
        print(json.dumps(line), flush=True)


BATCH_GROUPS_L = (32, 48, 64, 96, 128)
BATCH_GROUPS_R = (16384, 8192, 4096, 2048, 512)


def batched_groups(seed=2024):
    """The uneven-batch workload: five groups, beta ~ U[0.45, 0.60] and
    h ~ U[0.03, 0.12] drawn per group from a seed."""
    rs = np.random.default_rng(seed)
    return [(L, R_, float(rs.uniform(0.45, 0.60)), float(rs.uniform(0.03, 0.12)))
            for L, R_ in zip(BATCH_GROUPS_L, BATCH_GROUPS_R)]


def batched_measure(args):
    """The uneven batched launch vs one plain launch per group, both counting
    only attempts of not-yet-nucleated replicas."""
    import ctypes as C
    from gpu_2dising_b200 import _native as nat, engine
    engine.init_device(0)
    groups = batched_groups()
    arr = (nat.GroupT * len(groups))(*[nat.GroupT(L, n, b, h) for L, n, b, h in groups])
    h = C.c_void_p()
    kind = nat.RNG_MWC64X if args.rng == "mwc64x" else nat.RNG_XORWOW
    nat.check(nat.lib().gasp_batch_create(arr, len(groups), SEED, kind, C.byref(h)))
    choice = np.zeros(2 * len(groups), np.int32)
    nat.check(nat.lib().gasp_batch_autotune(h, 2, choice))
    t_sep, t_one = C.c_float(), C.c_float()
    layout = nat.lib().gasp_batch_layout(h, C.byref(t_sep), C.byref(t_one))
    tot, chk, up = args.batched_sweeps, 50, 0.9
    res = {}
    for name, mode in (("plain", nat.BATCH_PLAIN), ("graph", nat.BATCH_GRAPH),
                       ("one_launch", nat.BATCH_MULTI)):
        counts = np.zeros((tot // chk) * len(groups), np.int32)
        att, el = C.c_longlong(), C.c_double()
        nat.check(nat.lib().gasp_batch_swarm(h, tot, chk, up, mode, counts, C.byref(att),
                                             C.byref(el)))
        res[name] = {"attempts": att.value, "seconds": el.value, "value": att.value / el.value,
                     "nucleated": counts.reshape(-1, len(groups))[-1].tolist()}
    nat.lib().gasp_batch_free(h)
    return {
        "metric": "spin-flip attempts/s, uneven batched launch vs plain per-group launches",
        "value": res["graph"]["value"], "unit": UNIT, "n_gpus": 1,
        "speedup_vs_plain": res["graph"]["value"] / res["plain"]["value"],
        "one_launch_speedup_vs_plain": res["one_launch"]["value"] / res["plain"]["value"],
        "plain": res["plain"], "graph": res["graph"], "one_launch": res["one_launch"],
        "layout": {"chosen": ["one kernel per group", "one persistent launch"][layout],
                   "autotune_ms_3_intervals": {"per_group_kernels": t_sep.value,
                                               "one_launch": t_one.value}},
        "config": {"workload": "5 groups L=32/48/64/96/128, replicas 16384/8192/4096/2048/512, "
                               "all-down, nucleated replicas (m > 0.9 at a check) finished",
                   "groups": [{"L": L, "replicas": n, "beta": b, "h": hh}
                              for L, n, b, hh in groups],
                   "sweeps": tot, "check_int": chk, "rng": args.rng,
                   "autotune": choice.reshape(-1, 2).tolist()},
    }


def run_batched(args):
    print(json.dumps(clocked(batched_measure, args)), flush=True)


def committor_inputs(n=64, L_=L, seed=7):
    """Seeded committor inputs: all -1, a centred +1 disc of radius
    r ~ U[4, 12] (dist <= r from (L/2, L/2)), then 2% of sites flipped."""
    rs = np.random.default_rng(seed)
    yy, xx = np.mgrid[0:L_, 0:L_]
    out, radii = [], []
    for _ in range(n):
        r = rs.uniform(4.0, 12.0)
        g = np.where((yy - L_ / 2) ** 2 + (xx - L_ / 2) ** 2 <= r * r, 1, -1).astype(np.int32)
        flip = rs.random((L_, L_)) < 0.02
        g[flip] *= -1
        out.append(g)
        radii.append(r)
    return np.stack(out), np.array(radii)


def committor_measure(args, rng_kind=None):
    """Committor shooting of 64 seeded droplet grids, 4096 replicas each,
    until every replica reaches A (m < -0.93) or B (m > 0.9), cap 20000 sweeps."""
    from gpu_2dising_b200 import analysis, engine
    engine.init_device(0)
    rng_kind = rng_kind or args.rng
    ngrid_in, shots = args.committor_inputs, args.committor_shots
    inputs, radii = committor_inputs(ngrid_in)
    n = ngrid_in * shots
    # untimed warm-up: a short shooting run on the same kernels (first launches
    # in a process load their modules), then the timed run
    wg = engine.DeviceGrids(L, 4 * 256)
    wg.upload_inputs(inputs[:4])
    wr = engine.RngStates(4 * 256, SEED + 1, kind=rng_kind)
    engine.run_driver(wg, wr, BETA, H, 500, args.committor_check, 500, itask=1, dn_thr=-0.93,
                      up_thr=0.90, ninputs=4, compact=True)
    wg.close()
    wr.close()
    t0 = time.perf_counter()
    dg = engine.DeviceGrids(L, n)
    dg.upload_inputs(inputs)
    if args.committor_tail >= 0:  # 3 = GASP_OPT_TAIL_REPLICAS
        dg.set_option(3, args.committor_tail)
    rng = engine.RngStates(n, SEED, kind=rng_kind)
    res, fates, drv_s, attempts = engine.run_driver(
        dg, rng, BETA, H, 20000, args.committor_check, 20000, itask=1, dn_thr=-0.93,
        up_thr=0.90, ninputs=ngrid_in, compact=True)
    wall = time.perf_counter() - t0
    dg.close()
    rng.close()
    errs = [analysis.committor_errbar(fates[i * shots:(i + 1) * shots]) for i in range(ngrid_in)]
    resolved = [int(np.count_nonzero(fates[i * shots:(i + 1) * shots] >= 0))
                for i in range(ngrid_in)]
    return {
        "metric": "committor evaluations/s (shooting)", "value": ngrid_in / wall,
        "unit": "grids/s", "n_gpus": 1, "attempts_per_s": attempts / drv_s,
        "wall_s": wall, "driver_s": drv_s, "attempts": attempts,
        "unresolved": int(np.count_nonzero(fates == -1)),
        "pB": [round(float(x), 5) for x in res], "pB_err": [round(e, 5) for e in errs],
        "resolved": resolved, "radii": [round(float(r), 3) for r in radii],
        "config": {"workload": f"{ngrid_in} droplet grids L=64 (r~U[4,12], 2% flips), "
                               f"{shots} shots each, beta=0.54, h=0.07, dn=-0.93, up=0.9, "
                               "cap 20000 sweeps, compaction on",
                   "check_int": args.committor_check, "rng": rng_kind,
                   "tail_replicas": (args.committor_tail if args.committor_tail >= 0
                                     else "default")},
    }


def compare_pb(a, b):
    """Per-grid pB of two independent shooting runs: z-scores of the
    differences under binomial errors."""
    pa, pb_ = np.asarray(a["pB"], np.float64), np.asarray(b["pB"], np.float64)
    na, nb = np.asarray(a["resolved"], np.float64), np.asarray(b["resolved"], np.float64)
    var = pa * (1 - pa) / np.maximum(na, 1) + pb_ * (1 - pb_) / np.maximum(nb, 1)
    diff = pa - pb_
    z = np.where(var > 0, diff / np.sqrt(np.where(var > 0, var, 1.0)), 0.0)
    return {"grids": int(pa.size), "max_abs_z": float(np.max(np.abs(z))),
            "n_abs_z_above_3": int(np.count_nonzero(np.abs(z) > 3)),
            "mean_abs_diff": float(np.mean(np.abs(diff))),
            "chi2_per_grid": float(np.mean(z ** 2))}


def run_committor(args):
    print(json.dumps(clocked(committor_measure, args)), flush=True)


def cnn_measure(args):
    """Surrogate CNN inference throughput: predict() on int8 L=64 grids from
    host memory (batches of 1024), timed on the host around synchronised
    calls, plus one timed Adam step on a 1024-grid batch."""
    from gpu_2dising_b200 import engine, surrogate
    engine.init_device(0)
    n = args.cnn_grids
    rs = np.random.default_rng(SEED)
    grids = np.where(rs.random((n, L, L)) < 0.1, 1, -1).astype(np.int8)
    labels = rs.random(1024).astype(np.float32)
    net = surrogate.CommittorCNN(L, 1024, surrogate.init_params(0))
    if args.cnn_fused:  # the whole-network kernel for prediction (L = 64)
        from gpu_2dising_b200._native import check, lib
        check(lib().gasp_cnn_set_fused(net._h, 1))
    for _ in range(args.warmup):
        net.predict(grids[:2048])
    t0 = time.perf_counter()
    for _ in range(args.steps):
        net.predict(grids)
    pred_s = (time.perf_counter() - t0) / args.steps
    for _ in range(args.warmup):
        net.train_step(grids[:1024], labels, 1e-3)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        net.train_step(grids[:1024], labels, 1e-3)
    step_s = (time.perf_counter() - t0) / args.steps
    flop = 2.0 * L * L * (32 * 9 + 3 * 32 * 288) + 2.0 * 32  # convolutions + head, per grid
    line = {"metric": "committor CNN inference (grids/s)", "value": n / pred_s, "unit": "grids/s",
            "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1e3 * pred_s, "higher_is_better": True, "dtype": "bf16",
            "effective_tflops": flop * n / pred_s / 1e12,
            "train_step_ms_batch1024": 1e3 * step_s,
            "config": {"workload": f"predict on {n} int8 L=64 grids (host memory, batches of "
                                   "1024); 4x conv3x3(32) tcgen05, pool, 32->1",
                       "prediction_kernels": "fused whole network" if args.cnn_fused
                       else "layer by layer"}}
    net.close()
    return line


def run_cnn(args):
    print(json.dumps(clocked(cnn_measure, args)), flush=True)


def cluster_measure(args):
    """Largest-cluster collective variable on the device: gasp_largest_cluster
    over 32768 L=64 grids, near the site-percolation threshold (p = 0.593,
    the largest and most tangled clusters) and sparse (2 % of sites up, like a
    metastable swarm)."""
    from gpu_2dising_b200 import engine
    engine.init_device(0)
    rs = np.random.default_rng(SEED)
    out = {}
    for name, grids in (("percolating p=0.593", np.where(rs.random((R, L, L)) < 0.593, 1, -1)),
                        ("all -1 with 2% flips", np.where(rs.random((R, L, L)) < 0.02, 1, -1))):
        dg = engine.DeviceGrids(L, R, grids.astype(np.int32))
        for _ in range(args.warmup):
            dg.largest_cluster(1)
        t0 = time.perf_counter()
        for _ in range(args.steps):
            dg.largest_cluster(1)
        dt = (time.perf_counter() - t0) / args.steps
        out[name] = {"grids_per_s": R / dt, "ms_per_call": 1e3 * dt}
        dg.close()
    line = {"metric": "largest-cluster evaluations (grids/s)",
            "value": out["percolating p=0.593"]["grids_per_s"], "unit": "grids/s", "n_gpus": 1,
            "steps": args.steps, "warmup": args.warmup, "higher_is_better": True,
            "cases": out,
            "config": {"workload": f"gasp_largest_cluster(spin=+1) on {R} L=64 grids, "
                                   "including the device->host copy of the sizes"}}
    return line


def run_cluster(args):
    print(json.dumps(clocked(cluster_measure, args)), flush=True)


def tail_measure(args):
    """The end of a committor run: few undecided L=64 replicas (production
    stream unless --tail-rng xorwow).  Per replica count, the time of one sweep with the row
    kernel (one lane per replica, variant 0) and with one warp per replica
    (variant 6), CUDA events on the library's stream, 10 sweeps per launch as
    in committor shooting."""
    import torch
    from gpu_2dising_b200 import _native as nat, engine
    engine.init_device(0)
    stream = torch.cuda.Stream()
    engine.set_stream(stream.cuda_stream)
    counts = [args.tail_replicas] if args.tail_replicas else [32, 148, 592, 2368, 4736, 9472,
                                                                18944]
    per_launch = 10
    out = {}
    with torch.cuda.stream(stream):
        for n in counts:
            row = {}
            for v in (0, 6):
                dg = engine.DeviceGrids(L, n, -np.ones((n, L, L), np.int32))
                dg.set_option(nat.OPT_SWEEP_VARIANT, v)
                rng = engine.RngStates(n, SEED + n, kind=args.tail_rng)
                for _ in range(args.warmup):
                    dg.sweep(rng, BETA, H, per_launch)
                torch.cuda.synchronize()
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                for _ in range(args.steps):
                    dg.sweep(rng, BETA, H, per_launch)
                e1.record(stream)
                torch.cuda.synchronize()
                ms = e0.elapsed_time(e1) / (args.steps * per_launch)
                row[f"variant{v}"] = {"ms_per_sweep": ms,
                                      "attempts_per_s": n * L * L / (ms / 1e3)}
                dg.close()
                rng.close()
            row["speedup"] = row["variant0"]["ms_per_sweep"] / row["variant6"]["ms_per_sweep"]
            out[str(n)] = row
    first = out[str(counts[0])]
    line = {"metric": "sweep time of few replicas, one warp per replica vs one lane per replica",
            "value": first["variant6"]["ms_per_sweep"], "unit": "ms/sweep", "n_gpus": 1,
            "steps": args.steps, "warmup": args.warmup, "higher_is_better": False,
            "speedup_vs_row_kernel": first["speedup"], "by_replicas": out,
            "config": {"workload": f"L=64 all-down replicas, beta=0.54, h=0.07, "
                                   f"{args.tail_rng} stream, "
                                   f"{per_launch} sweeps per launch; replica counts {counts}"}}
    return line


def run_tail(args):
    print(json.dumps(clocked(tail_measure, args)), flush=True)


def rate_measure(args):
    """The full production swarm of the headline workload (L=64, 32768
    replicas, beta=0.54, h=0.07, 50 000 sweeps, checks every 100, dumps every
    1000 not written): nucleated-fraction curve fitted to 1 - exp(-k (t - t0))
    as the reference's notebook does, bootstrap errors over replicas, for the
    reference stream and the production stream."""
    from gpu_2dising_b200 import analysis, engine
    engine.init_device(0)
    tot = args.rate_sweeps
    out = {}
    for kind in ("xorwow", "mwc64x"):
        dg = engine.DeviceGrids(L, R)
        rng = engine.RngStates(R, SEED, kind=kind)
        fu = np.full(R, -1, np.int32)
        t0 = time.perf_counter()
        res, _, drv_s, att = engine.run_driver(dg, rng, BETA, H, tot, MAG_INT, GRID_INT, itask=0,
                                               dn_thr=-0.9, up_thr=0.9, first_up=fu)
        wall = time.perf_counter() - t0
        k, t_ind, k_site = analysis.fit_nucleation_rate(res, MAG_INT, L=L)
        bs = analysis.bootstrap_rate(fu, tot, MAG_INT, nboot=100, L=L)
        out[kind] = {"k": k, "t0": t_ind, "k_per_site": k_site, "k_se": bs["k_se"],
                     "t0_se": bs["t0_se"], "final_fraction": float(res[-1]),
                     "never_crossed": int(np.count_nonzero(fu < 0)), "wall_s": wall,
                     "attempts_per_s": att / drv_s}
        dg.close()
        rng.close()
    a, b = out["xorwow"], out["mwc64x"]
    line = {"metric": "nucleation rate k (1/sweep), full production swarm", "value": a["k"],
            "unit": "1/sweep", "n_gpus": 1, "higher_is_better": None,
            "exact_stream": a, "production_stream": b,
            "k_diff_sigma": abs(a["k"] - b["k"]) / float(np.hypot(a["k_se"], b["k_se"])),
            "t0_diff_sigma": abs(a["t0"] - b["t0"]) / float(np.hypot(a["t0_se"], b["t0_se"])),
            "published_anchor": {"k": 1.5032e-4, "replicas": 1024,
                                 "source": "Jupyter/GASP_rates.ipynb:178 (single run, Quadro "
                                           "P2000)"},
            "config": {"workload": f"L=64, {R} replicas, beta=0.54, h=0.07, all-down, {tot} "
                                   "sweeps, magnetisation checked every 100 sweeps, up 0.9"}}
    return line


def run_rate(args):
    print(json.dumps(clocked(rate_measure, args)), flush=True)


def surrogate_measure(args):
    """The learned committor surrogate: snapshots from a swarm at beta=0.54,
    h=0.07, shooting labels, GPU training, held-out MAE against 1024-shot
    labels, and screening throughput vs shooting alone."""
    from gpu_2dising_b200 import engine, surrogate
    engine.init_device(0)
    res = surrogate.run_experiment(n_train=args.surrogate_train, n_test=args.surrogate_test,
                                   n_screen=args.surrogate_screen, epochs=args.surrogate_epochs,
                                   focus=args.surrogate_focus)
    hist = res.pop("history")
    line = {"metric": "committor evaluations/s, surrogate-screened vs shooting alone",
            "value": res["screen_grids_per_s"], "unit": "grids/s", "n_gpus": 1,
            "speedup_vs_shooting": res["speedup"], **res,
            "val_mae_by_epoch": [round(h["val_mae"], 4) for h in hist],
            "epochs": args.surrogate_epochs, "focus": args.surrogate_focus,
            "config": {"workload": f"{res['n_train']} L=64 swarm snapshots (beta=0.54, h=0.07, "
                                   "m in (-0.93,-0.65)) labelled by 256-shot pB, "
                                   f"{res['n_test']} held out with 1024-shot pB, "
                                   f"{res['n_screen']} screened; CNN 4x conv3x3(32)+ReLU, "
                                   "avg-pool, 32->1 sigmoid, batch 1024; fallback "
                                   "|pred-0.5|<0.1 shot with 64 trajectories"}}
    return line


def run_surrogate(args):
    print(json.dumps(clocked(surrogate_measure, args)), flush=True)


def secondary_measure(args):
    """The figures of the metric's second half and of the other
    configurations, each with its own clock record: committor shooting of
    the 64 droplet grids on both streams (pB compared), the uneven batch
    against plain per-group launches, the full production swarm's rate fit
    on both streams, and surrogate screening against shooting alone."""
    from gpu_2dising_b200 import engine
    engine.init_device(0)
    out = {}
    if args.secondary_quick:  # a short form for development runs
        args.committor_inputs, args.committor_shots = 16, 1024
        args.batched_sweeps = 200
        args.surrogate_train, args.surrogate_test, args.surrogate_screen = 2048, 512, 8192
        args.surrogate_epochs = 4
        args.rate_sweeps = 5000
    ex = clocked(committor_measure, args, "xorwow")
    pr = clocked(committor_measure, args, "mwc64x")
    keep = ("value", "unit", "attempts_per_s", "wall_s", "unresolved", "clocks")
    out["committor"] = {
        "metric": "committor evaluations/s (shooting)", "unit": "grids/s",
        "workload": ex["config"]["workload"],
        "exact_stream": {k: ex[k] for k in keep},
        "production_stream": {k: pr[k] for k in keep},
        "pB_exact_vs_production": compare_pb(ex, pr),
        "pB_exact": ex["pB"], "pB_production": pr["pB"]}
    bt = clocked(batched_measure, args)
    out["batched"] = {"metric": bt["metric"], "value": bt["value"], "unit": bt["unit"],
                      "speedup_vs_plain": bt["speedup_vs_plain"],
                      "one_launch_speedup_vs_plain": bt["one_launch_speedup_vs_plain"],
                      "layout": bt["layout"],
                      "plain": bt["plain"], "graph": bt["graph"], "one_launch": bt["one_launch"],
                      "autotune": bt["config"]["autotune"], "workload": bt["config"]["workload"],
                      "clocks": bt["clocks"]}
    # the full production swarm's own output (config 2): the nucleated fraction
    # over 50 000 sweeps fitted to 1 - exp(-k (t - t0)), both streams
    rt = clocked(rate_measure, args)
    keep_r = ("k", "k_se", "t0", "t0_se", "k_per_site", "final_fraction", "never_crossed",
              "wall_s", "attempts_per_s")
    out["rate"] = {"metric": rt["metric"], "unit": rt["unit"],
                   "exact_stream": {k: rt["exact_stream"][k] for k in keep_r},
                   "production_stream": {k: rt["production_stream"][k] for k in keep_r},
                   "k_diff_sigma": rt["k_diff_sigma"], "t0_diff_sigma": rt["t0_diff_sigma"],
                   "published_anchor": rt["published_anchor"],
                   "workload": rt["config"]["workload"], "clocks": rt["clocks"]}
    su = clocked(surrogate_measure, args)
    keys = ("value", "unit", "speedup_vs_shooting", "screen_grids_per_s", "shoot_grids_per_s",
            "cnn_only_grids_per_s", "mae_surrogate", "mae_screened", "mae_shooting_baseline",
            "fallback_fraction", "test_mid_0.1_0.9", "mae_shooting_by_shots", "n_train",
            "n_test", "n_screen", "times_s", "clocks")
    out["surrogate"] = {"metric": su["metric"], **{k: su[k] for k in keys if k in su},
                        "equal_mae": su.get("by_cap", {}).get("equal_mae"),
                        "bar_0.05": su.get("by_cap", {}).get("bar_0.05"),
                        "workload": su["config"]["workload"]}
    out["quick"] = bool(args.secondary_quick)
    return out


def run_secondary(args):
    print(json.dumps(secondary_measure(args)), flush=True)


def spawn_ranks(n, argv):
    """Runs this script on n ranks of this host (torch.distributed.run), each
    rank seeing WORLD_SIZE; returns the launcher's exit status."""
    import socket
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1",
           f"--nproc-per-node={n}", "--master-addr", "127.0.0.1", f"--master-port={port}",
           os.path.abspath(__file__), *argv]
    return subprocess.call(cmd)


def main(argv=None):
    global SWEEPS_PER_STEP
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--sweeps-per-step", type=int, default=SWEEPS_PER_STEP,
                    help="smaller values give a short launch for ncu captures")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--workload", default="swarm",
                    choices=["swarm", "batched", "committor", "surrogate", "cnn", "rate",
                             "cluster", "tail", "secondary"],
                    help="swarm: the headline single-group swarm; batched: uneven groups; "
                         "committor: seeded droplet shooting")
    ap.add_argument("--cnn-grids", type=int, default=100000)
    ap.add_argument("--cnn-fused", action="store_true",
                    help="cnn workload: predict through the fused whole-network kernel")
    ap.add_argument("--rate-sweeps", type=int, default=50000)
    ap.add_argument("--tail-replicas", type=int, default=0,
                    help="tail workload: one replica count (default: a range)")
    ap.add_argument("--committor-inputs", type=int, default=64)
    ap.add_argument("--committor-shots", type=int, default=4096)
    ap.add_argument("--committor-check", type=int, default=10)
    ap.add_argument("--committor-tail", type=int, default=-1,
                    help="live replicas at which shooting switches to one warp per "
                         "replica (-1: library default, 0: never)")
    ap.add_argument("--tail-rng", default="mwc64x", choices=["xorwow", "mwc64x"],
                    help="stream of the tail workload")
    ap.add_argument("--surrogate-train", type=int, default=20000)
    ap.add_argument("--surrogate-test", type=int, default=2000)
    ap.add_argument("--surrogate-screen", type=int, default=100000)
    ap.add_argument("--surrogate-epochs", type=int, default=120)
    ap.add_argument("--surrogate-focus", type=float, default=3.0,
                    help="training draws grids with weight 1 + focus*4y(1-y)")
    ap.add_argument("--batched-sweeps", type=int, default=1000)
    ap.add_argument("--rng", default="xorwow", choices=["xorwow", "mwc64x"],
                    help="xorwow: the reference stream (bit-exact); mwc64x: production stream")
    ap.add_argument("--variant", type=int, default=0,
                    help="sweep kernel variant (0 fastest for L, 1 generic) for comparisons")
    ap.add_argument("--no-secondary", action="store_true",
                    help="default line without the secondary block")
    ap.add_argument("--secondary-quick", action="store_true",
                    help="secondary block at reduced sizes (development runs)")
    ap.add_argument("--secondary-timeout", type=int, default=900)
    ap.add_argument("--no-reference-gpu", action="store_true",
                    help="reference arm without timing the reference's GPU kernels")
    ap.add_argument("--cpu-replicas", type=int, default=CPU_CONFIG["replicas"],
                    help="CPU runs: replicas (default: the CPU configuration's 1248)")
    ap.add_argument("--cpu-sweeps", type=int, default=CPU_CONFIG["sweeps"],
                    help="CPU runs: sweeps (default: the CPU configuration's 5000)")
    ap.add_argument("--dry-run", action="store_true",
                    help="rank plumbing with a host stand-in step (no GPU, gloo)")
    argv = sys.argv[1:] if argv is None else list(argv)
    args = ap.parse_args(argv)
    args.warmup = max(args.warmup, 3)
    CPU_CONFIG["replicas"], CPU_CONFIG["sweeps"] = args.cpu_replicas, args.cpu_sweeps
    SWEEPS_PER_STEP = args.sweeps_per_step
    CONFIG["sweeps_per_step"] = SWEEPS_PER_STEP
    if "WORLD_SIZE" not in os.environ and args.gpus > 1 and args.impl == "ours" \
            and args.workload == "swarm":
        return spawn_ranks(args.gpus, argv)
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", str(args.gpus if args.impl == "reference" else 1)))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank, world)
    elif args.dry_run:
        run_dry(args, rank, world, local_rank)
    elif args.workload == "secondary":
        run_secondary(args)
    elif args.workload == "batched":
        if rank == 0:
            run_batched(args)
    elif args.workload == "committor":
        if rank == 0:
            run_committor(args)
    elif args.workload == "surrogate":
        if rank == 0:
            run_surrogate(args)
    elif args.workload == "cnn":
        if rank == 0:
            run_cnn(args)
    elif args.workload == "rate":
        if rank == 0:
            run_rate(args)
    elif args.workload == "tail":
        run_tail(args)
    elif args.workload == "cluster":
        if rank == 0:
            run_cluster(args)
    else:
        run_ours(args, rank, world, local_rank)


if __name__ == "__main__":
    sys.exit(main() or 0)
