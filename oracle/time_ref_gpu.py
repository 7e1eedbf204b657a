"""Device time of the reference's own GPU sweep kernels (src/mc_gpu.cu
mc_sweep_gpu / _bitrep / _bitmap32, compiled unmodified for sm_100a into
oracle/_ref/libref_gpu.so) on the headline swarm workload: L=64, 32768
all-down replicas, beta=0.54, h=0.07, 100 sweeps per launch, the reference
driver's launch shape (tpb 32).  TEST INFRASTRUCTURE: it times the reference
beside bench.py's figures for this implementation on the same GPU; nothing in
the product calls it.

    python oracle/time_ref_gpu.py [--calls 5] [--replicas 32768]
"""
import argparse
import ctypes as C
import json
import os

HERE = os.path.dirname(os.path.abspath(__file__))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--calls", type=int, default=5)
    ap.add_argument("--replicas", type=int, default=32768)
    ap.add_argument("--sweeps", type=int, default=100)
    args = ap.parse_args()
    lib = C.CDLL(os.path.join(HERE, "_ref", "libref_gpu.so"))
    lib.refgpu_time_kernels.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, C.c_ulonglong,
                                        C.c_double, C.c_double, C.c_int, C.c_int,
                                        C.POINTER(C.c_double)]
    L, R = 64, args.replicas
    out = {}
    for method in (2, 0, 1):
        ms = C.c_double(0.0)
        rc = lib.refgpu_time_kernels(L, R, 32, method, 2024, 0.54, 0.07, args.sweeps, args.calls,
                                     C.byref(ms))
        if rc != 0:
            raise SystemExit(f"reference kernel method {method} failed ({rc})")
        out[f"gpu_method_{method}"] = {"ms_per_launch": ms.value,
                                       "attempts_per_s": L * L * R * args.sweeps / (ms.value / 1e3)}
    print(json.dumps({"what": "reference GPU sweep kernels, unmodified, sm_100a",
                      "workload": f"L=64, {R} all-down replicas, beta=0.54, h=0.07, "
                                  f"{args.sweeps} sweeps per launch, tpb 32",
                      "calls": args.calls, "methods": out}))


if __name__ == "__main__":
    main()
