#!/usr/bin/env python
"""Benchmark of the SWALS time-step hot path on B200.

Headline workload (one GPU): nonlinear finite-volume 'rk2' with wetting and
drying on a 2048 x 2048 Cartesian grid, dx = 10 m, planar beach from -50 m
to +10 m (slope 1/40) plus 30 seeded 0.5 m Gaussian bumps, Manning
n = 0.025, a solitary wave (H/d = 0.1) entering through the west boundary,
walls elsewhere, FP64, adaptive CFL timestep (cfl 0.99, theta 1.6).  One
bench step = 2000 model timesteps, so the default 10 timed steps are the
configuration's 20000 timesteps.  Synthetic seeded data.

metric: cell-updates/s = nx * ny * timesteps / device seconds (all GPUs).

The same JSON line carries, under "forms", the metric's other forms timed
on the same GPU right after the headline (N = 1 only): the headline with
FP32 state, the plain linear configuration at its own 400^2, the plain FP64
leapfrog at 4096^2 and 8192^2 against the HBM roofline, the batched FP32
leapfrog (3600 x 2400 x 256 instances) against the per-instance loop, the
adjoint misfit gradient (1200 x 800, K = 50) against one forward solve, and
the nested four-domain configuration (one source, and 16 sources as a
batch of nests).

  python bench.py [--gpus N --steps K --warmup W]   # our CUDA path
  python bench.py --impl reference ...              # CPU restatement of the
                                                    # reference's OpenMP loops
  python bench.py --workload linear|batched|adjoint|multidomain|nested16
                                                    # one form on its own line
Under torchrun each rank advances its own replica of the headline domain
(the path does not shard: replicas only) and rank 0 prints one JSON line.
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


def cpu_baseline(workload="rk2_beach", min_seconds=12.0, exact_steps=0, variant="native", samples=0,
                 warmup_steps=1):
    """The oracle on this machine's host cores, in its own process (its OpenMP
    runtime never shares a process with the GPU runtime)."""
    cmd = [sys.executable, os.path.join(ROOT, "oracle", "cpu_baseline.py"), "--workload", workload,
           "--min-seconds", str(min_seconds), "--variant", variant, "--warmup-steps", str(warmup_steps)]
    if exact_steps:
        cmd += ["--exact-steps", str(exact_steps)]
    if samples:
        cmd += ["--samples", str(samples)]
    env = dict(os.environ)
    env.setdefault("OMP_NUM_THREADS", str(os.cpu_count() or 1))
    env.setdefault("OMP_PROC_BIND", "true")
    out = subprocess.run(cmd, capture_output=True, text=True, env=env, check=True)
    r = json.loads(out.stdout.strip().splitlines()[-1])
    return {"value": r["value"], "unit": UNIT, "cores": r["cores"], "kind": "port", "variant": r["variant"],
            "values": r.get("values"),
            "sample": r["sample"] + "; C restatement of the reference's OpenMP loops (no Fortran compiler)"}


# CPU samples: timesteps per sample of the 2048^2 workload (about 1 s on 16
# cores), after CPU_WARMUP untimed timesteps; the same procedure in both arms.
CPU_STEPS_PER_SAMPLE = 12
CPU_WARMUP = 3


def headline_config(n, real32=False, world=1):
    """The workload, identical in both arms' lines."""
    return {"workload": f"rk2_beach_{n}x{n}_{'fp32' if real32 else 'fp64'}_adaptive", "nx": n, "ny": n,
            "parallelism": f"replicas x{world}",
            "timestepping_method": "rk2", "dt": "adaptive (CFL, cfl=0.99)", "theta": 1.6, "manning_n": 0.025,
            "boundary": "solitary wave H/d=0.1 west, walls elsewhere", "gauges": 9,
            "l2": "inputs larger than L2 (state 4x32 MB + manning 32 MB + max_stage 32 MB + stage copies; "
                  "~0.7 GB streamed per timestep)"}


def dist_setup(ngpus):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def run_reference(args, world, rank):
    """The reference's CPU path for this workload: the oracle built with the
    flags the reference ships (-O3 -ffast-math, libm pow) plus -march=native
    on this machine, all host threads; each bench step is one sample of
    CPU_STEPS_PER_SAMPLE timesteps of the same 2048^2 workload, the samples
    taken one after another in one process after W x CPU_WARMUP untimed
    timesteps.  The IEEE-strict build's rate is reported beside it."""
    if rank != 0:
        return
    t0 = time.perf_counter()
    r = cpu_baseline("rk2_beach", exact_steps=CPU_STEPS_PER_SAMPLE, samples=args.steps,
                     warmup_steps=CPU_WARMUP * max(1, args.warmup))
    wall = time.perf_counter() - t0
    value = r["value"]
    strict = cpu_baseline("rk2_beach", exact_steps=CPU_STEPS_PER_SAMPLE, samples=1, variant="strict",
                          warmup_steps=CPU_WARMUP)
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": N * N * CPU_STEPS_PER_SAMPLE / value * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": headline_config(N, world=world), "timesteps_per_step": CPU_STEPS_PER_SAMPLE,
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": r["cores"], "kind": "port",
                             "sample": r["sample"], "samples": r["values"],
                             "strict_build_value": strict["value"]},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "wall_s": wall}
    print(json.dumps(line), flush=True)


# Nominal FP64 peak of the FV kernels' pipe: 64 FP64 FMA lanes per SM
# (B200: 37 TFLOP/s FP64 at 1965 MHz over 148 SMs), 2 flops per FMA.
FP64_LANES_PER_SM = 64


def profile_value(tag):
    """A number committed in a profiles/ summary as `tag = value`."""
    pdir = os.path.join(ROOT, "profiles")
    if not os.path.isdir(pdir):
        return None
    for fn in sorted(os.listdir(pdir)):
        if not fn.endswith((".md", ".txt")):
            continue
        for line in open(os.path.join(pdir, fn)):
            if line.startswith(tag + " ="):
                try:
                    return float(line.split("=")[1].split()[0])
                except Exception:
                    return None
    return None


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
    d.gauges_setup(gauges, capacity=INNER * (args.warmup + 2 * args.steps + 8) + 16)
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
    # Dominant kernel: stage 2 (edges, update, rk2 average and max_stage of
    # every cell in one pass; 104 algorithmic bytes per cell in FP64).
    t2_ms, n2 = tm["fv_stage2"]
    es_scale = 0.5 if args.real32 else 1.0   # byte counts above are for 8-byte reals
    bytes_kernel = cells * BYTES_STAGE2 * n2 * es_scale
    achieved = bytes_kernel / (t2_ms / 1e3) / 1e9
    peak, peak_kind = hbm_peak()
    per_step_ms = {k: (v[0] / v[1] if v[1] else 0.0) for k, v in tm.items()}
    step_ms = sum(per_step_ms.values())
    stage2_share = per_step_ms["fv_stage2"] / step_ms if step_ms else None
    # FP64 work of the same launch: flops per cell from the committed ncu
    # count (dadd + dmul + 2 dfma thread instructions / cells).
    fpc = profile_value("fp64_flops_per_cell[rk2_stage2]") if not args.real32 else None
    pipe = profile_value("fp64_pipe_active_frac[rk2_stage2]") if not args.real32 else None
    fp64 = None
    if fpc:
        sm_mhz = clocks.get("sm_mhz") or 1965.0
        fp64_peak = 2.0 * FP64_LANES_PER_SM * props.multi_processor_count * sm_mhz * 1e6 / 1e12
        fp64_ach = fpc * cells / (per_step_ms["fv_stage2"] / 1e3) / 1e12
        fp64 = {"bound": "fp64", "achieved": fp64_ach, "peak": fp64_peak, "unit": "TFLOP/s",
                "frac": fp64_ach / fp64_peak, "flops_per_cell": fpc,
                "peak_source": f"nominal: {FP64_LANES_PER_SM} FP64 FMA lanes/SM x {props.multi_processor_count} "
                               f"SMs x {sm_mhz:.0f} MHz (median under load)",
                "pipe_active_frac_ncu": pipe}

    # End to end through the C ABI with host buffers: pinned H2D of the state,
    # INNER timesteps, D2H of the state, every step; as many steps as timed above.
    tdt = torch.float32 if args.real32 else torch.float64
    pin_in = torch.empty((4, N, N), dtype=tdt, pin_memory=True)
    pin_in.copy_(torch.from_numpy(d.get_U()))
    pin_out = torch.empty((4, N, N), dtype=tdt, pin_memory=True)
    h_in, h_out = pin_in.numpy(), pin_out.numpy()
    e2e_steps = args.steps
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
    d.close()

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline and N == 2048:
        try:
            cpu = cpu_baseline("rk2_beach", exact_steps=CPU_STEPS_PER_SAMPLE, samples=7, warmup_steps=CPU_WARMUP)
            cpu["strict_build_value"] = cpu_baseline("rk2_beach", exact_steps=CPU_STEPS_PER_SAMPLE, samples=1,
                                                     variant="strict", warmup_steps=CPU_WARMUP)["value"]
        except Exception as ex:  # the baseline is reported, never required
            cpu = {"value": None, "unit": UNIT, "cores": os.cpu_count(), "kind": "port", "sample": f"failed: {ex}"}

    forms = None
    if rank == 0 and world == 1 and not args.no_forms and N == 2048 and not args.real32:
        forms = {}
        for name, fn in (("rk2_fp32", form_rk2_fp32), ("linear_400", form_linear_400),
                         ("linear_fp64", form_linear_sweep), ("batched", form_batched), ("adjoint", form_adjoint),
                         ("multidomain", form_multidomain), ("nested16", form_nested16)):
            t0 = time.perf_counter()
            try:
                forms[name] = fn(local)
            except Exception as ex:   # a form that fails is reported, the headline stands
                forms[name] = {"error": f"{type(ex).__name__}: {ex}"}
            forms[name]["wall_s"] = round(time.perf_counter() - t0, 1)
            torch.cuda.empty_cache()

    if rank == 0:
        cfg = headline_config(N, args.real32, world)
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32" if args.real32 else "f64", "data": "synthetic",
            "config": cfg, "timesteps_per_step": INNER,
            "roofline": {"bound": "hbm",
                         "kernel": f"rk2 stage-2 kernel, rk2_srow_kernel (dominant: {100 * stage2_share:.0f}% of the step)",
                         "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                         "peak_source": peak_kind,
                         "bytes_per_cell": BYTES_STAGE2 * es_scale,
                         "algorithmic_bytes_per_launch": cells * BYTES_STAGE2 * es_scale,
                         "traffic": (profile_traffic("rk2_stage2") if N == 2048 and not args.real32
                                     else None),
                         "traffic_unit": "DRAM bytes of one stage-2 launch (ncu, 2048x2048 FP64)",
                         "fp64": fp64,
                         "step_effective_GBps": cells * BYTES_PER_CELL_UPDATE * es_scale /
                                                (ms_max / args.steps / INNER / 1e3) / 1e9,
                         "per_launch_ms": per_step_ms},
            "cpu_baseline": cpu,
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                    "steps": e2e_steps, "timesteps_per_step": INNER},
            "gpu_launches": launches,
            "clocks": clocks,
            "state_ok": ok, "sim_time_s": st.time, "max_dt": st.max_dt,
            "forms": forms,
        }
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


# ---------------------------------------------------------------------------
# The metric's other forms.  Each returns a dict of device-timed numbers
# (CUDA events on the stream the kernels run on); `--workload X` prints one
# of them as a line of its own.

def _event_ms(stream, fn):
    import torch
    a = torch.cuda.Event(enable_timing=True)
    b = torch.cuda.Event(enable_timing=True)
    a.record(stream)
    fn()
    b.record(stream)
    b.synchronize()
    return a.elapsed_time(b)


def form_linear(local, n, inner=200, reps=3, warmup=1):
    """The 400x400 Gaussian-basin configuration scaled up for the roofline
    (dx 1 km, flat 4000 m, walls, CFL 0.7, FP64, max_stage on): device
    throughput, and the step kernel's HBM fraction at 72 B per cell."""
    import torch
    from ptha_b200 import Domain, workloads
    peak, peak_kind = hbm_peak()
    kw, U, gauges = workloads.linear_gaussian_basin(n=n)
    d = Domain(**kw, device=local)
    d.set_U(U)
    del U
    dt = d.linear_timestep_max()
    stream = torch.cuda.ExternalStream(d.stream(), device=f"cuda:{local}")
    for _ in range(warmup):
        d.evolve_steps(inner, dt)
    d.synchronize()
    ms = _event_ms(stream, lambda: [d.evolve_steps(inner, dt) for _ in range(reps)])
    value = n * n * inner * reps / (ms / 1e3)
    d.timers_enable(True)
    d.evolve_steps(50, dt)
    tm = d.timers_read()
    d.timers_enable(False)
    t_ms, cnt = tm["leapfrog_step"]
    achieved = n * n * 72.0 * cnt / (t_ms / 1e3) / 1e9
    d.close()
    return {"workload": f"linear_gaussian_basin_{n}x{n}_fp64", "value": value, "unit": UNIT,
            "ms_per_timestep": ms / (reps * inner), "dt": dt,
            "roofline": {"bound": "hbm", "kernel": "linear leapfrog step kernel", "achieved": achieved,
                         "peak": peak, "unit": "GB/s", "frac": achieved / peak, "peak_source": peak_kind,
                         "bytes_per_cell": 72,
                         "per_launch_ms": {k: (v[0] / v[1] if v[1] else 0.0) for k, v in tm.items()}}}


def form_linear_sweep(local):
    return {f"n{n}": form_linear(local, n) for n in (4096, 8192)}


def form_linear_400(local, nsteps=2000, reps=3):
    """The plain linear configuration at its own size: 400x400, dx 1 km,
    flat 4000 m, walls, Gaussian hump, FP64, CFL 0.7, 2000 steps, 9 gauges
    sampled every step (L2-resident: latency and launch bound)."""
    import torch
    from ptha_b200 import Domain, workloads
    kw, U, gauges = workloads.linear_gaussian_basin(n=400)
    d = Domain(**kw, device=local)
    d.set_U(U)
    dt = d.linear_timestep_max()
    d.gauges_setup(gauges, capacity=nsteps * (reps + 1) + 8)
    stream = torch.cuda.ExternalStream(d.stream(), device=f"cuda:{local}")
    d.evolve_steps(nsteps, dt)
    d.synchronize()
    ms = _event_ms(stream, lambda: [d.evolve_steps(nsteps, dt) for _ in range(reps)])
    d.close()
    return {"workload": "linear_gaussian_basin_400x400_fp64_9_gauges", "value": 400 * 400 * nsteps * reps / (ms / 1e3),
            "unit": UNIT, "ms_per_timestep": ms / (reps * nsteps), "timesteps": nsteps, "dt": dt}


def form_rk2_fp32(local, nsteps=2000, reps=2):
    """The headline workload with FP32 state (the reference's -DREALFLOAT
    build; pressure/source terms stay FP64)."""
    import torch
    from ptha_b200 import Domain, workloads
    kw, U, gauges, nsq = workloads.rk2_beach()
    d = Domain(**kw, real_bytes=4, device=local)
    d.set_U(U)
    d.set_manning_squared(nsq)
    d.gauges_setup(gauges, capacity=nsteps * (reps + 1) + 8)
    stream = torch.cuda.ExternalStream(d.stream(), device=f"cuda:{local}")
    d.evolve_steps(nsteps)
    d.synchronize()
    ms = _event_ms(stream, lambda: [d.evolve_steps(nsteps) for _ in range(reps)])
    d.close()
    cells = kw["nx"][0] * kw["nx"][1]
    return {"workload": "rk2_beach_2048x2048_fp32_adaptive", "value": cells * nsteps * reps / (ms / 1e3), "unit": UNIT,
            "ms_per_timestep": ms / (reps * nsteps), "timesteps": nsteps * reps}


def form_batched(local, B=256, nx=3600, ny=2400, inner=50, reps=2, world=1, rank=0, dist=None):
    """Spherical 3600x2400 (1 arcmin) FP32, B dipole initial conditions,
    Coriolis on, fixed CFL-0.7 step, 200 gauges: one batched launch per step
    against one instance stepped as a plain domain (the per-instance loop)."""
    import numpy as np
    import torch
    from ptha_b200 import Domain, workloads
    from ptha_b200.batch import Batch
    from ptha_b200.sharding import gather_instance_series, instance_range
    peak, peak_kind = hbm_peak()
    first_inst, count = instance_range(B, world, rank)
    gkw, U0, lon, lat = workloads.batched_grid(nx, ny)
    grid = Domain(**gkw, device=local)
    grid.set_U(U0)
    dt = grid.linear_timestep_max()
    wet = U0[3] < 0
    b = Batch(grid, count)
    chunk = 8
    first_eta = None
    for q0 in range(0, count, chunk):
        cnt = min(chunk, count - q0)
        U3 = np.zeros((cnt, 3, ny, nx), np.float32)
        for t in range(cnt):
            U3[t, 0] = workloads.batched_instance_stage(lon, lat, wet, first_inst + q0 + t, B)
            if first_eta is None:
                first_eta = U3[t, 0].copy()
        b.set_U(U3, first=q0)
        del U3
    cfg, _ = b.tune()
    stream = torch.cuda.ExternalStream(grid.stream(), device=f"cuda:{local}")
    b.gauges_setup(workloads.batched_gauges(lon, lat, wet), capacity=inner * (reps + 1))
    b.evolve(inner, dt)
    torch.cuda.synchronize()
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()
    ms_b = _event_ms(stream, lambda: [b.evolve(inner, dt) for _ in range(reps)])
    if dist is not None:
        t = torch.tensor([ms_b], dtype=torch.float64, device=f"cuda:{local}")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms_b = float(t.item())
    v_batched = nx * ny * B * inner * reps / (ms_b / 1e3)
    series = gather_instance_series(b.gauges_read(), B, world, rank) if dist is not None else b.gauges_read()
    b.close()
    out = {"workload": f"batched_linear_spherical_{nx}x{ny}_B{B}_fp32", "value": v_batched, "unit": UNIT,
           "ms_per_timestep": ms_b / (reps * inner), "batch": B, "dt": dt, "tile_config": cfg, "gauges": 200,
           "gauge_series": list(series.shape)}
    if rank == 0:
        # The per-instance loop: one instance as its own domain step loop.
        single = Domain(**gkw, device=local)
        U = U0.astype(np.float32).copy()
        U[0] = first_eta
        single.set_U(U)
        single.evolve_steps(inner, dt)
        single.synchronize()
        s_stream = torch.cuda.ExternalStream(single.stream(), device=f"cuda:{local}")
        ms_s = _event_ms(s_stream, lambda: [single.evolve_steps(inner, dt) for _ in range(reps)])
        single.close()
        v_loop = nx * ny * inner * reps / (ms_s / 1e3)
        bytes_cell = 32.0 + 4.0 / B
        out.update({"per_instance_loop": {"value": v_loop, "ms_per_timestep": ms_s / (reps * inner)},
                    "speedup_vs_loop": v_batched / v_loop,
                    "roofline": {"bound": "hbm", "kernel": "batched linear leapfrog step kernel",
                                 "achieved": v_batched * bytes_cell / 1e9, "peak": peak, "unit": "GB/s",
                                 "frac": v_batched * bytes_cell / 1e9 / peak, "peak_source": peak_kind,
                                 "bytes_per_cell": bytes_cell,
                                 "loop_frac": v_loop * 36.0 / 1e9 / peak}})
    grid.close()
    return out


def form_adjoint(local, nx=1200, ny=800, reps=2):
    """Spherical 1200x800 (2 arcmin) FP64, 30 gauges, a hidden dipole's
    waveforms as the target, 2 h simulated, checkpoint every 50 steps: the
    misfit gradient's device time against one forward solve."""
    import numpy as np
    import torch
    from ptha_b200 import Domain, workloads
    gkw, U0, gauges, eta_t, _ = workloads.adjoint_case(nx, ny)
    d = Domain(**gkw, device=local)
    d.set_U(U0)
    dt = d.linear_timestep_max()
    nsteps = int(round(2 * 3600.0 / dt))
    Ut = U0.copy()
    Ut[0] = eta_t
    d.set_U(Ut)
    d.gauges_setup(gauges, capacity=nsteps + 8)
    stream = torch.cuda.ExternalStream(d.stream(), device=f"cuda:{local}")
    d.evolve_steps(nsteps, dt)
    target = d.gauges_read()[:nsteps, :, 0].copy()
    Ui = U0.copy()
    Ui[0] = 0.0
    times_f, times_a = [], []
    res = {}
    for _ in range(reps):
        d.set_U(Ui)
        d.gauges_reset()
        d.time = 0.0
        d.synchronize()
        times_f.append(_event_ms(stream, lambda: d.evolve_steps(nsteps, dt)))
        d.set_U(Ui)
        d.time = 0.0
        d.synchronize()

        def grad_call():
            res["lg"] = d.misfit_gradient(nsteps, dt, target, checkpoint_every=50)
        # Device time on the domain's stream, including the gradient's copy
        # back to the host (the forward solve has no copy).
        times_a.append(_event_ms(stream, grad_call))
    loss, grad = res["lg"]
    d.close()
    f_ms, a_ms = min(times_f), min(times_a)
    return {"workload": f"adjoint_linear_spherical_{nx}x{ny}_fp64", "value": nx * ny * nsteps / (a_ms / 1e3),
            "unit": UNIT, "nsteps": nsteps, "dt": dt, "gauges": 30, "checkpoint_every": 50,
            "forward_ms": f_ms, "gradient_ms": a_ms, "gradient_over_forward": a_ms / f_ms,
            "loss": loss, "grad_norm": float(np.linalg.norm(grad[0]))}


def _nested(local, nts, source_seed=11, elevations=None):
    from ptha_b200 import Multidomain, workloads
    specs, coasts = workloads.nested_specs(nts)
    kw = [dict(real_bytes=4, spherical=True), dict(spherical=True), dict(spherical=True), dict(spherical=True)]
    md = Multidomain(specs, domain_kwargs=kw, use_wetdry_limiting=True, flux_correction=True, device=local,
                     periodic_xs=(0.0, 360.0))
    for k, (s_, d) in enumerate(zip(specs, md.domains)):
        d.set_U(workloads.nested_initial_state(s_, k, coasts, source_seed=source_seed,
                                               elevation=None if elevations is None else elevations[k]))
        if d.timestepping_method == "rk2":
            d.set_manning_squared(0.025 ** 2)
    return specs, md


def _nested_refinement(local):
    import math
    specs, md = _nested(local, (1, 1, 1, 1))
    dt = md.domains[0].linear_timestep_max()
    lims = [d.stationary_timestep_max() if d.timestepping_method == "rk2" else dt for d in md.domains]
    md.close()
    return dt, [max(1, int(math.ceil(dt / lim))) for lim in lims]


def form_multidomain(local, reps=20, K=3):
    """The nested configuration with one source: a coarse 'linear' FP32 band
    (4 arcmin, 5400x1800, 60S-60N, periodic over 0-360), one ratio-3 'rk2'
    FP64 domain (900x900) and two ratio-9 'rk2' FP64 wet/dry domains
    (1197x801, 702x1098) on coastal ramps; fixed md step from the coarse
    CFL, refinement factors from each domain's stationary CFL; graph-captured
    md steps."""
    import numpy as np
    import torch
    dt, nts = _nested_refinement(local)
    specs, md = _nested(local, nts)
    cells = sum(s_.nx[0] * s_.nx[1] * nt for s_, nt in zip(specs, nts))
    stream = torch.cuda.ExternalStream(md.domains[0].stream(), device=f"cuda:{local}")
    md.evolve_one_step(dt)
    md.synchronize()
    ms_plain = _event_ms(stream, lambda: [md.evolve_one_step(dt) for _ in range(K * 2)]) / (K * 2)
    md.capture_graph(K, dt)
    md.replay(1)
    md.synchronize()
    ms = _event_ms(stream, lambda: md.replay(reps))
    ms_step = ms / (reps * K)
    vols = [d.volume_interior() for d in md.domains]
    out = {"workload": "nested_multidomain_4dom", "value": cells / (ms_step / 1e3), "unit": UNIT,
           "ms_per_md_step": ms_step, "dtype": "f32 coarse / f64 fine",
           "domains": [{"nx": list(s_.nx), "method": s_.timestepping_method, "nt": nt,
                        "nest_layer_width": s_.nest_layer_width} for s_, nt in zip(specs, nts)],
           "md_dt": dt, "exchanges": len(md.exchanges), "flux_correction": True, "graph_steps": K, "sources": 1,
           "cell_updates_per_md_step": cells, "ms_per_md_step_without_graph": ms_plain,
           "finite": bool(all(np.isfinite(v) for v in vols))}
    md.close()
    return out


def form_nested16(local, B=16, K=3, reps=6):
    """The nested configuration with B = 16 dipole sources (seeds 11..26):
    16 instances of the four-domain nest advanced together, K md steps of
    every instance captured into one CUDA graph (one branch per instance, the
    instances' kernels running concurrently), against the same instances
    replayed one after another (each instance's own K-step graph)."""
    import numpy as np
    import torch
    from ptha_b200 import MultidomainGroup, workloads
    dt, nts = _nested_refinement(local)
    specs0, coasts = workloads.nested_specs(nts)
    specs0, md0 = _nested(local, nts)
    elevations = [workloads.nested_elevation(s_, k, coasts) for k, s_ in enumerate(specs0)]
    mds = [md0] + [_nested(local, nts, source_seed=11 + q, elevations=elevations)[1] for q in range(1, B)]
    cells = sum(s_.nx[0] * s_.nx[1] * nt for s_, nt in zip(specs0, nts))
    for md in mds:
        md.capture_graph(K, dt)
        md.replay(1)
    torch.cuda.synchronize()
    # one after another: each instance's own graph, device time on its stream
    seq = 0.0
    for md in mds:
        st = torch.cuda.ExternalStream(md.domains[0].stream(), device=f"cuda:{local}")
        seq += _event_ms(st, lambda: md.replay(reps))
    group = MultidomainGroup(mds, K, dt)
    group.replay(1)
    torch.cuda.synchronize()
    gs = torch.cuda.ExternalStream(group.stream(), device=f"cuda:{local}")
    ms = _event_ms(gs, lambda: group.replay(reps))
    torch.cuda.synchronize()
    vols = [d.volume_interior() for md in mds for d in md.domains]
    group.close()
    for md in mds:
        md.close()
    ms_step = ms / (reps * K)
    return {"workload": "nested_multidomain_4dom_x16_sources", "value": B * cells / (ms_step / 1e3), "unit": UNIT,
            "sources": B, "ms_per_md_step_all_sources": ms_step, "md_dt": dt, "graph_steps": K,
            "cell_updates_per_md_step": B * cells,
            "one_after_another": {"value": B * cells / (seq / (reps * K) / 1e3),
                                  "ms_per_md_step_all_sources": seq / (reps * K)},
            "speedup_vs_one_after_another": seq / ms,
            "dtype": "f32 coarse / f64 fine", "finite": bool(all(np.isfinite(v) for v in vols))}


def run_form(args, local, world=1, rank=0):
    import torch
    torch.cuda.set_device(local)
    torch.zeros(1, device=f"cuda:{local}")
    line = {"metric": METRIC, "unit": UNIT, "n_gpus": 1, "higher_is_better": True, "data": "synthetic",
            "vs_baseline": None}
    if args.workload == "linear":
        r = form_linear(local, args.n if args.n != N else 8192,
                        inner=args.inner if args.inner != INNER else 200, reps=args.steps, warmup=args.warmup)
        line.update(r, dtype="f64", steps=args.steps, config={"workload": r["workload"], "max_stage": True})
    elif args.workload == "batched":
        dist = None
        if world > 1:
            import datetime
            import torch.distributed as dist
            dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
        nx, ny = (3600, 2400) if args.n == N else (args.n * 3 // 2, args.n)
        r = form_batched(local, B=args.batch, nx=nx, ny=ny, inner=args.inner if args.inner != INNER else 50,
                         reps=args.steps, world=world, rank=rank, dist=dist)
        if dist is not None:
            dist.barrier()
            dist.destroy_process_group()
        if rank != 0:
            return
        line.update(r, dtype="f32", steps=args.steps, n_gpus=world, scaling="strong",
                    config={"workload": r["workload"], "batch": args.batch,
                            "parallelism": f"instances sharded x{world}"})
    elif args.workload == "adjoint":
        nx, ny = (1200, 800) if args.n == N else (args.n * 3 // 2, args.n)
        r = form_adjoint(local, nx, ny, reps=max(1, args.steps))
        line.update(r, dtype="f64", steps=args.steps, config={"workload": r["workload"]})
    elif args.workload == "multidomain":
        r = form_multidomain(local)
        line.update(r, steps=r["graph_steps"], config={"workload": r["workload"]})
    elif args.workload == "nested16":
        r = form_nested16(local)
        line.update(r, config={"workload": "nested_multidomain_4dom_x16_sources"})
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-forms", action="store_true", help="headline only (no secondary forms)")
    ap.add_argument("--n", type=int, default=N, help="grid cells per side (default 2048)")
    ap.add_argument("--inner", type=int, default=INNER, help="timesteps per bench step (default 2000)")
    ap.add_argument("--real32", action="store_true", help="FP32 state (-DREALFLOAT analogue)")
    ap.add_argument("--profile", action="store_true", help="short untimed run for ncu")
    ap.add_argument("--workload", default="rk2",
                    choices=["rk2", "linear", "batched", "adjoint", "multidomain", "nested16"],
                    help="rk2 (default, the headline) or a secondary form")
    ap.add_argument("--batch", type=int, default=256, help="instances for --workload batched")
    args = ap.parse_args()
    if args.warmup < 3 and not args.profile:
        args.warmup = 3
    world, rank, local = dist_setup(args.gpus)
    if args.impl == "reference":
        run_reference(args, world, rank)
        return
    if args.workload == "batched" and world > 1:
        run_form(args, local, world, rank)   # instances sharded over the ranks
        return
    if args.workload != "rk2":
        if rank == 0:
            run_form(args, local)
        return
    run_ours(args, world, rank, local)


if __name__ == "__main__":
    main()
