#!/usr/bin/env python
"""Benchmark of the SWALS time-step hot path on B200.

Workload (one GPU): nonlinear finite-volume 'rk2' with wetting and drying on
a 2048 x 2048 Cartesian grid, dx = 10 m, planar beach from -50 m to +10 m
(slope 1/40) plus 30 seeded 0.5 m Gaussian bumps, Manning n = 0.025, a
solitary wave (H/d = 0.1) entering through the west boundary, walls
elsewhere, FP64, adaptive CFL timestep (cfl 0.99, theta 1.6).  One bench
step = 2000 model timesteps, so the default 10 timed steps are the
configuration's 20000 timesteps.  Synthetic seeded data.

metric: cell-updates/s = nx * ny * timesteps / device seconds (all GPUs).

  python bench.py [--gpus N --steps K --warmup W]   # our CUDA path
  python bench.py --impl reference ...              # CPU restatement of the
                                                    # reference's OpenMP loops
Under torchrun each rank advances its own replica of the domain (the path
does not shard: replicas only) and rank 0 prints one JSON line.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

METRIC = "cell-updates/s/GPU (fwd, batched, adjoint) at FP64-oracle tol; HBM % of peak"
UNIT = "cell-updates/s"
INNER = 2000          # model timesteps per bench step (default)
N = 2048              # grid cells per side (default)
WORKLOAD = "rk2_beach_2048x2048_fp64_adaptive"
# Algorithmic HBM bytes per cell for the fused FV stage kernel (FP64):
#   stage 1 reads STG,UH,VH,ELV,n^2 and writes STG,UH,VH            = 8 planes
#   stage 2 reads the same 5 + backup U0 (3), writes 3, max_stage r+w = 13 planes
BYTES_STAGE1 = 8 * 8
BYTES_STAGE2 = 13 * 8
BYTES_PER_CELL_UPDATE = BYTES_STAGE1 + BYTES_STAGE2   # 168 B (matches the rk2 + max_stage row)


def hbm_peak():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def profile_traffic(kernel_tag):
    """DRAM bytes per launch from a committed ncu summary, if present."""
    pdir = os.path.join(ROOT, "profiles")
    if not os.path.isdir(pdir):
        return None
    for fn in sorted(os.listdir(pdir)):
        if not fn.endswith((".md", ".txt")):
            continue
        for line in open(os.path.join(pdir, fn)):
            if line.startswith(f"traffic_per_launch_bytes[{kernel_tag}]"):
                try:
                    return float(line.split("=")[1].split()[0])
                except Exception:
                    return None
    return None


class ClockSampler:
    """nvidia-smi samples of SM clock and throttle reasons during a region."""
    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, pci_bus_id):
        self.pci = pci_bus_id
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.pci}", f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 8:
                continue
            try:
                sm.append(float(parts[0]))
                smax.append(float(parts[1]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[4:8]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        os.unlink(self.path)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def cpu_baseline(workload="rk2_beach", min_seconds=12.0, exact_steps=0):
    cmd = [sys.executable, os.path.join(ROOT, "oracle", "cpu_baseline.py"), "--workload", workload,
           "--min-seconds", str(min_seconds)]
    if exact_steps:
        cmd += ["--exact-steps", str(exact_steps)]
    env = dict(os.environ)
    env.setdefault("OMP_NUM_THREADS", str(os.cpu_count() or 1))
    env.setdefault("OMP_PROC_BIND", "true")
    out = subprocess.run(cmd, capture_output=True, text=True, env=env, check=True)
    r = json.loads(out.stdout.strip().splitlines()[-1])
    return {"value": r["value"], "unit": UNIT, "cores": r["cores"], "kind": "port",
            "sample": r["sample"] + " (C restatement of the reference's OpenMP loops; no Fortran compiler)"}


def dist_setup(ngpus):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def run_reference(args, world, rank):
    if rank != 0:
        return
    # Each step: a bounded sample (a few timesteps) of the same 2048^2 workload.
    steps_per = 3
    cpu_baseline("rk2_beach", exact_steps=steps_per * max(1, args.warmup))  # warm-up (page-in, threads)
    vals = []
    t0 = time.perf_counter()
    for _ in range(args.steps):
        r = cpu_baseline("rk2_beach", exact_steps=steps_per)
        vals.append(r["value"])
    wall = time.perf_counter() - t0
    value = statistics.median(vals)
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": N * N * steps_per / value * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": WORKLOAD, "nx": N, "ny": N, "timesteps_per_step": steps_per},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": r["cores"], "kind": "port",
                             "sample": f"{steps_per} rk2 timesteps of the 2048x2048 workload per step"},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "wall_s": wall}
    print(json.dumps(line), flush=True)


def run_ours(args, world, rank, local):
    import numpy as np
    import torch
    torch.cuda.set_device(local)
    torch.zeros(1, device=f"cuda:{local}")
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    from ptha_b200 import Domain, workloads

    global N, INNER
    N, INNER = args.n, args.inner
    kw, U, gauges, nsq = workloads.rk2_beach(n=N, dx=10.0 * 2048 / N, toe=17580.0 * N / 2048)
    if args.real32:
        kw["real_bytes"] = 4
    d = Domain(**kw, device=local)
    d.set_U(U)
    d.set_manning_squared(nsq)
    d.gauges_setup(gauges, capacity=INNER * (args.warmup + args.steps + 8) + 16)
    stream = torch.cuda.ExternalStream(d.stream(), device=f"cuda:{local}")
    cells = N * N

    def barrier():
        if dist is not None:
            dist.barrier()

    for _ in range(args.warmup):
        d.evolve_steps(INNER)
    d.synchronize()
    if args.profile:
        # Short untimed run for profilers: the warm-up above, then `steps`
        # bench steps, nothing else.
        for _ in range(args.steps):
            d.evolve_steps(INNER)
        d.synchronize()
        if rank == 0:
            print(json.dumps({"profile_run": True, "n": N, "inner": INNER, "launches": d.launch_count()}))
        d.close()
        return

    barrier()
    torch.cuda.synchronize()
    props = torch.cuda.get_device_properties(local)
    pci = f"{props.pci_domain_id:08x}:{props.pci_bus_id:02x}:{props.pci_device_id:02x}.0" \
        if hasattr(props, "pci_bus_id") else str(local)
    sampler = ClockSampler(pci)
    sampler.start()
    time.sleep(0.3)
    launches0 = d.launch_count()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        d.evolve_steps(INNER)
    e1.record(stream)
    e1.synchronize()
    launches = d.launch_count() - launches0
    clocks = sampler.stop()
    torch.cuda.synchronize()
    barrier()
    ms = e0.elapsed_time(e1)
    ms_t = torch.tensor([ms], dtype=torch.float64, device=f"cuda:{local}")
    if dist is not None:
        dist.all_reduce(ms_t, op=dist.ReduceOp.MAX)
    ms_max = float(ms_t.item())
    value = cells * INNER * args.steps * world / (ms_max / 1e3)
    st = d.state()
    ok = bool(np.isfinite(st.time))

    # Per-kernel timing pass (CUDA events around each launch) for the roofline.
    d.timers_enable(True)
    d.evolve_steps(200)
    tm = d.timers_read()
    d.timers_enable(False)
    t1_ms, n1 = tm["fv_stage1"]
    t2_ms, n2 = tm["fv_stage2"]
    es_scale = 0.5 if args.real32 else 1.0   # byte counts above are for 8-byte reals
    bytes_kernel = cells * (BYTES_STAGE1 * n1 + BYTES_STAGE2 * n2) * es_scale
    achieved = bytes_kernel / ((t1_ms + t2_ms) / 1e3) / 1e9
    peak, peak_kind = hbm_peak()
    per_step_ms = {k: (v[0] / v[1] if v[1] else 0.0) for k, v in tm.items()}

    # End to end through the C ABI with host buffers: pinned H2D of the state,
    # INNER timesteps, D2H of the state, every step.
    tdt = torch.float32 if args.real32 else torch.float64
    pin_in = torch.empty((4, N, N), dtype=tdt, pin_memory=True)
    pin_in.copy_(torch.from_numpy(d.get_U()))
    pin_out = torch.empty((4, N, N), dtype=tdt, pin_memory=True)
    h_in, h_out = pin_in.numpy(), pin_out.numpy()
    e2e_steps = 3
    barrier()
    torch.cuda.synchronize()
    e2 = torch.cuda.Event(enable_timing=True)
    e3 = torch.cuda.Event(enable_timing=True)
    e2.record(stream)
    for _ in range(e2e_steps):
        d.set_U(h_in)
        d.evolve_steps(INNER)
        d.get_U(out=h_out)
    e3.record(stream)
    e3.synchronize()
    e2e_ms = torch.tensor([e2.elapsed_time(e3)], dtype=torch.float64, device=f"cuda:{local}")
    if dist is not None:
        dist.all_reduce(e2e_ms, op=dist.ReduceOp.MAX)
    e2e_value = cells * INNER * e2e_steps * world / (float(e2e_ms.item()) / 1e3)
    h2d = int(h_in.nbytes)
    d2h = int(h_out.nbytes)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline and N == 2048:
        try:
            cpu = cpu_baseline("rk2_beach", min_seconds=12.0)
        except Exception as ex:  # the baseline is reported, never required
            cpu = {"value": None, "unit": UNIT, "cores": os.cpu_count(), "kind": "port", "sample": f"failed: {ex}"}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32" if args.real32 else "f64", "data": "synthetic",
            "config": {"workload": (f"rk2_beach_{N}x{N}_{'fp32' if args.real32 else 'fp64'}_adaptive"),
                       "nx": N, "ny": N, "timesteps_per_step": INNER,
                       "timestepping_method": "rk2", "dt": "adaptive (CFL, cfl=0.99)", "theta": 1.6,
                       "manning_n": 0.025, "boundary": "solitary wave H/d=0.1 west, walls elsewhere",
                       "l2": "inputs larger than L2 (state 4x32 MB + manning 32 MB + max_stage 32 MB + "
                             "stage copies; ~0.7 GB streamed per timestep)",
                       "parallelism": f"replicas x{world}", "gauges": 9},
            "roofline": {"bound": "hbm", "kernel": "rk2_stage_kernel (FV stage 1 + stage 2)",
                         "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                         "peak_source": peak_kind,
                         "bytes_per_cell": {"stage1": BYTES_STAGE1, "stage2": BYTES_STAGE2},
                         "traffic": profile_traffic("rk2_stage_kernel"),
                         "step_effective_GBps": cells * BYTES_PER_CELL_UPDATE * es_scale /
                                                (ms_max / args.steps / INNER / 1e3) / 1e9,
                         "per_launch_ms": per_step_ms},
            "cpu_baseline": cpu,
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                    "steps": e2e_steps, "timesteps_per_step": INNER},
            "gpu_launches": launches,
            "clocks": clocks,
            "state_ok": ok, "sim_time_s": st.time, "max_dt": st.max_dt,
        }
        print(json.dumps(line), flush=True)
    d.close()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--n", type=int, default=N, help="grid cells per side (default 2048)")
    ap.add_argument("--inner", type=int, default=INNER, help="timesteps per bench step (default 2000)")
    ap.add_argument("--real32", action="store_true", help="FP32 state (-DREALFLOAT analogue)")
    ap.add_argument("--profile", action="store_true", help="short untimed run for ncu")
    args = ap.parse_args()
    if args.warmup < 3 and not args.profile:
        args.warmup = 3
    world, rank, local = dist_setup(args.gpus)
    if args.impl == "reference":
        run_reference(args, world, rank)
        return
    run_ours(args, world, rank, local)


if __name__ == "__main__":
    main()
