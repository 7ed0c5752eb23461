"""Test infrastructure: time the CPU oracle (the restatement of SWALS's
OpenMP loops) on a bounded sample of a benchmark workload.

Used only by bench.py's cpu_baseline leg and its `--impl reference` arm.
Runs in its own process so the oracle's OpenMP runtime never shares a
process with the GPU runtime.  Prints one JSON line.
"""
from __future__ import annotations

import argparse
import json
import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
# Run as a script, sys.path[0] is oracle/ itself, where `import oracle` would
# find oracle/oracle.py instead of the package directory.
sys.path = [p for p in sys.path if os.path.abspath(p or ".") != HERE]
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", default="rk2_beach")
    ap.add_argument("--min-seconds", type=float, default=10.0)
    ap.add_argument("--max-steps", type=int, default=1000)
    ap.add_argument("--exact-steps", type=int, default=0)
    ap.add_argument("--samples", type=int, default=0, help="time this many samples of --exact-steps timesteps")
    ap.add_argument("--warmup-steps", type=int, default=1)
    ap.add_argument("--variant", default="fast", choices=["fast", "native", "strict"],
                    help="oracle build: fast = -O3 -ffast-math with libm pow (the reference's -Ofast), "
                         "native = the same with -march=native (built here on first use), strict = the "
                         "IEEE-strict parity checker")
    args = ap.parse_args()
    from ptha_b200 import workloads
    from tests.pairs import oracle_from_kw
    variant = args.variant
    if variant == "native" and not os.path.exists(os.path.join(HERE, "liboracle64_native.so")):
        import subprocess
        r = subprocess.run(["make", "-s", "-C", HERE, "native"], capture_output=True, text=True)
        if r.returncode != 0:
            variant = "fast"
    flags = {"fast": "-O3 -ffast-math, libm pow", "native": "-O3 -ffast-math -march=native, libm pow",
             "strict": "-O2 IEEE-strict, no FMA contraction"}[variant]
    if args.workload == "rk2_beach":
        kw, U, gauges, nsq = workloads.rk2_beach()
        o = oracle_from_kw(kw, variant=variant)
        o.U[:] = U
        o.manning_squared[:] = nsq
        dt = None
    elif args.workload == "linear_gaussian_basin":
        kw, U, gauges = workloads.linear_gaussian_basin()
        o = oracle_from_kw(kw, variant=variant)
        o.U[:] = U
        dt = o.linear_timestep_max()
    else:
        raise SystemExit(f"unknown workload {args.workload}")
    nx, ny = kw["nx"]
    for _ in range(max(1, args.warmup_steps)):
        o.evolve_one_step(dt)  # untimed (page-in, thread start)
    threads = int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))
    if args.samples:
        # `samples` timed samples of exact_steps timesteps each, in a row
        vals = []
        for _ in range(args.samples):
            t0 = time.perf_counter()
            for _ in range(args.exact_steps):
                o.evolve_one_step(dt)
            vals.append(nx * ny * args.exact_steps / (time.perf_counter() - t0))
        vals_sorted = sorted(vals)
        med = vals_sorted[len(vals) // 2] if len(vals) % 2 else 0.5 * (vals_sorted[len(vals) // 2 - 1] +
                                                                        vals_sorted[len(vals) // 2])
        print(json.dumps({"value": med, "values": vals, "unit": "cell-updates/s", "cores": threads,
                          "steps": args.exact_steps * args.samples, "cells": nx * ny, "variant": variant,
                          "flags": flags,
                          "sample": f"{args.workload} {nx}x{ny}: {args.samples} samples of {args.exact_steps} "
                                    f"timesteps after {args.warmup_steps} untimed ({flags})"}))
        return
    steps = 0
    t0 = time.perf_counter()
    while True:
        o.evolve_one_step(dt)
        steps += 1
        el = time.perf_counter() - t0
        if args.exact_steps:
            if steps >= args.exact_steps:
                break
        elif el >= args.min_seconds or steps >= args.max_steps:
            break
    el = time.perf_counter() - t0
    print(json.dumps({"value": nx * ny * steps / el, "unit": "cell-updates/s", "cores": threads,
                      "steps": steps, "seconds": el, "cells": nx * ny, "variant": variant, "flags": flags,
                      "sample": f"{args.workload} {nx}x{ny}: {steps} timesteps after {args.warmup_steps} untimed "
                                f"({flags})"}))


if __name__ == "__main__":
    main()
