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
    # Dominant kernel: stage 2 (edges, update, rk2 average and max_stage of
    # every cell in one pass; 104 algorithmic bytes per cell in FP64).
    t2_ms, n2 = tm["fv_stage2"]
    es_scale = 0.5 if args.real32 else 1.0   # byte counts above are for 8-byte reals
    bytes_kernel = cells * BYTES_STAGE2 * n2 * es_scale
    achieved = bytes_kernel / (t2_ms / 1e3) / 1e9
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
            "roofline": {"bound": "hbm", "kernel": "rk2_stream_kernel stage 2 (dominant: ~42% of the step)",
                         "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                         "peak_source": peak_kind,
                         "bytes_per_cell": BYTES_STAGE2 * es_scale,
                         "algorithmic_bytes_per_launch": cells * BYTES_STAGE2 * es_scale,
                         "traffic": (profile_traffic("rk2_stream_kernel_stage2") if N == 2048 and not args.real32
                                     else None),
                         "traffic_unit": "DRAM bytes of one stage-2 launch (ncu, 2048x2048 FP64)",
                         "bound_note": "FP64 issue/latency bound (DRAM ~10% busy); see profiles/",
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


# ---------------------------------------------------------------------------
# Secondary forms (`--workload linear|batched|adjoint`): one JSON line each,
# for the evidence of the plain leapfrog roofline, the batched form against a
# per-instance loop, and the adjoint's cost against a forward solve.

def _event_ms(stream, fn):
    import torch
    a = torch.cuda.Event(enable_timing=True)
    b = torch.cuda.Event(enable_timing=True)
    a.record(stream)
    fn()
    b.record(stream)
    b.synchronize()
    return a.elapsed_time(b)


def _dipoles(lon, lat, count, seed, band=((150.0, -40.0), (190.0, -10.0)), width_km=400.0):
    """Compact dipole uplift patches in a band: a random centre within
    width_km of the band's axis, extent L in U[50, 200] km, amplitude A in
    U[0.5, 3] m, eta = A [G(s - L/4, n) - G(s + L/4, n)] with Gaussians of
    sigma L/6 in band-aligned coordinates; evaluated within 3L of the centre
    (zero beyond)."""
    import numpy as np
    rng = np.random.default_rng(seed)
    (x0, y0), (x1, y1) = band
    km_deg = 111.19
    ang = np.arctan2(y1 - y0, x1 - x0)
    out = []
    for _ in range(count):
        t = rng.uniform(0.0, 1.0)
        off = rng.uniform(-0.5, 0.5) * width_km / km_deg
        cx = x0 + t * (x1 - x0) - off * np.sin(ang)
        cy = y0 + t * (y1 - y0) + off * np.cos(ang)
        L = rng.uniform(50.0, 200.0)
        A = rng.uniform(0.5, 3.0)
        eta = np.zeros((len(lat), len(lon)))
        r_deg = 3.0 * L / km_deg
        ii = np.flatnonzero(np.abs(lon - cx) <= r_deg / max(np.cos(np.deg2rad(cy)), 0.2))
        jj = np.flatnonzero(np.abs(lat - cy) <= r_deg)
        if len(ii) and len(jj):
            LON, LAT = np.meshgrid(lon[ii], lat[jj])
            dx = (LON - cx) * km_deg * np.cos(np.deg2rad(cy))
            dy = (LAT - cy) * km_deg
            s_ = dx * np.cos(ang) + dy * np.sin(ang)
            n_ = -dx * np.sin(ang) + dy * np.cos(ang)
            sg = L / 6.0
            eta[np.ix_(jj, ii)] = A * (np.exp(-((s_ - L / 4) ** 2 + n_ ** 2) / (2 * sg ** 2)) -
                                       np.exp(-((s_ + L / 4) ** 2 + n_ ** 2) / (2 * sg ** 2)))
        out.append(eta)
    return out


def run_form(args, local, world=1, rank=0):
    import numpy as np
    import torch
    torch.cuda.set_device(local)
    torch.zeros(1, device=f"cuda:{local}")
    from ptha_b200 import Domain, workloads
    peak, peak_kind = hbm_peak()
    line = {"metric": METRIC, "unit": UNIT, "n_gpus": 1, "higher_is_better": True, "data": "synthetic",
            "vs_baseline": None}
    if args.workload == "linear":
        # The 400x400 Gaussian-basin configuration scaled up for the roofline
        # sweep (dx 1 km, flat 4000 m, walls, CFL 0.7, FP64, max_stage on).
        n = args.n if args.n != N else 8192
        kw, U, gauges = workloads.linear_gaussian_basin(n=n)
        d = Domain(**kw, device=local)
        d.set_U(U)
        dt = d.linear_timestep_max()
        stream = torch.cuda.ExternalStream(d.stream(), device=f"cuda:{local}")
        inner = max(1, args.inner if args.inner != INNER else 200)
        for _ in range(args.warmup):
            d.evolve_steps(inner, dt)
        d.synchronize()
        ms = _event_ms(stream, lambda: [d.evolve_steps(inner, dt) for _ in range(args.steps)])
        value = n * n * inner * args.steps / (ms / 1e3)
        d.timers_enable(True)
        d.evolve_steps(50, dt)
        tm = d.timers_read()
        d.timers_enable(False)
        t_ms, cnt = tm["leapfrog_step"]
        achieved = n * n * 72.0 * cnt / (t_ms / 1e3) / 1e9
        line.update({"workload": f"linear_gaussian_basin_{n}x{n}_fp64", "value": value, "steps": args.steps,
                     "ms_per_step": ms / args.steps, "dtype": "f64",
                     "config": {"workload": f"linear_gaussian_basin_{n}x{n}_fp64", "timesteps_per_step": inner,
                                "dt": dt, "max_stage": True},
                     "roofline": {"bound": "hbm", "kernel": "linear_step_kernel", "achieved": achieved,
                                  "peak": peak, "unit": "GB/s", "frac": achieved / peak, "peak_source": peak_kind,
                                  "bytes_per_cell": 72,
                                  "per_launch_ms": {k: (v[0] / v[1] if v[1] else 0.0) for k, v in tm.items()}}})
        d.close()
    elif args.workload == "batched":
        # Spherical 3600x2400 (1 arcmin) FP32, B dipole initial conditions,
        # Coriolis on, fixed CFL-0.7 step: one batched launch per step
        # against the same instances stepped one domain at a time.
        from ptha_b200.batch import Batch
        from ptha_b200.sharding import gather_instance_series, instance_range
        dist = None
        if world > 1:
            import datetime
            import torch.distributed as dist
            dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
        nxg, nyg = (3600, 2400) if args.n == N else (args.n * 3 // 2, args.n)
        B = args.batch
        first_inst, count = instance_range(B, world, rank)
        dl = 1.0 / 60.0 * (3600 / nxg)
        gkw, U0 = workloads.spherical_patch(nx=nxg, ny=nyg, dlon=dl, ll=(140.0, -45.0), seed=3)
        grid = Domain(**gkw, timestepping_method="linear", real_bytes=4, device=local)
        grid.set_U(U0)
        dt = grid.linear_timestep_max()
        lon = gkw["lower_left"][0] + (np.arange(nxg) + 0.5) * dl
        lat = gkw["lower_left"][1] + (np.arange(nyg) + 0.5) * dl
        wet = U0[3] < 0
        b = Batch(grid, count)
        chunk = 8
        first_eta = None
        # instance q's initial condition depends on q only, not on the ranks
        rng_seeds = np.random.default_rng(4).integers(0, 2 ** 31, size=B)
        for q0 in range(0, count, chunk):
            cnt = min(chunk, count - q0)
            U3 = np.zeros((cnt, 3, nyg, nxg), np.float32)
            for t in range(cnt):
                eta = _dipoles(lon, lat, 1, seed=int(rng_seeds[first_inst + q0 + t]))[0]
                U3[t, 0] = np.where(wet, eta, 0.0)
                if first_eta is None:
                    first_eta = U3[t, 0].copy()
            b.set_U(U3, first=q0)
            del U3
        cfg, _ = b.tune()
        stream = torch.cuda.ExternalStream(grid.stream(), device=f"cuda:{local}")
        inner = args.inner if args.inner != INNER else 50
        # 200 gauges at random wet cells (seed 5), sampled every step
        gr = np.random.default_rng(5)
        wj, wi = np.nonzero(wet)
        pick = gr.choice(wj.size, size=200, replace=False)
        gxy = np.stack([lon[wi[pick]], lat[wj[pick]]], axis=1)
        b.gauges_setup(gxy, capacity=inner * (args.steps + 1))
        b.evolve(inner, dt)
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()
        ms_b = _event_ms(stream, lambda: [b.evolve(inner, dt) for _ in range(args.steps)])
        if dist is not None:
            t = torch.tensor([ms_b], dtype=torch.float64, device=f"cuda:{local}")
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            ms_b = float(t.item())
        v_batched = nxg * nyg * B * inner * args.steps / (ms_b / 1e3)
        series = gather_instance_series(b.gauges_read(), B, world, rank) if dist is not None else b.gauges_read()
        if dist is not None and rank != 0:
            b.close()
            grid.close()
            dist.barrier()
            dist.destroy_process_group()
            return
        # Per-instance loop: each instance as its own domain step loop.
        single = Domain(**gkw, timestepping_method="linear", real_bytes=4, device=local)
        U = U0.astype(np.float32).copy()
        U[0] = first_eta
        single.set_U(U)
        single.evolve_steps(inner, dt)
        single.synchronize()
        s_stream = torch.cuda.ExternalStream(single.stream(), device=f"cuda:{local}")
        ms_s = _event_ms(s_stream, lambda: [single.evolve_steps(inner, dt) for _ in range(args.steps)])
        v_loop = nxg * nyg * inner * args.steps / (ms_s / 1e3)
        bytes_cell = 32.0 + 4.0 / B
        line.update({"workload": f"batched_linear_spherical_{nxg}x{nyg}_B{B}_fp32", "value": v_batched,
                     "steps": args.steps, "ms_per_step": ms_b / args.steps, "dtype": "f32", "n_gpus": world,
                     "scaling": "strong",
                     "config": {"workload": f"batched_linear_spherical_{nxg}x{nyg}_B{B}_fp32", "batch": B,
                                "timesteps_per_step": inner, "dt": dt, "coriolis": True, "tile_config": cfg,
                                "gauges": 200, "parallelism": f"instances sharded x{world}"},
                     "gauge_series_gathered": list(series.shape),
                     "per_instance_loop": {"value": v_loop, "ms_per_step_one_instance": ms_s / args.steps},
                     "speedup_vs_loop": v_batched / v_loop,
                     "roofline": {"bound": "hbm", "kernel": "linear_step_kernel (batched)",
                                  "achieved": v_batched * bytes_cell / 1e9, "peak": peak, "unit": "GB/s",
                                  "frac": v_batched * bytes_cell / 1e9 / peak, "peak_source": peak_kind,
                                  "bytes_per_cell": bytes_cell}})
        b.close()
        single.close()
        grid.close()
        if dist is not None:
            dist.barrier()
            dist.destroy_process_group()
    elif args.workload == "adjoint":
        # Spherical 1200x800 (2 arcmin) FP64, 30 gauges, a hidden dipole's
        # waveforms as the target, 2 h simulated, checkpoint every 50 steps.
        nxg, nyg = (1200, 800) if args.n == N else (args.n * 3 // 2, args.n)
        dl = 2.0 / 60.0 * (1200 / nxg)
        gkw, U0 = workloads.spherical_patch(nx=nxg, ny=nyg, dlon=dl, ll=(150.0, -40.0), seed=6)
        d = Domain(**gkw, timestepping_method="linear", device=local)
        lon = gkw["lower_left"][0] + (np.arange(nxg) + 0.5) * dl
        lat = gkw["lower_left"][1] + (np.arange(nyg) + 0.5) * dl
        wet = U0[3] < 0
        rng = np.random.default_rng(7)
        wi = np.argwhere(wet)
        pick = wi[rng.choice(len(wi), 30, replace=False)]
        gauges = np.stack([lon[pick[:, 1]], lat[pick[:, 0]]], axis=1)
        d.set_U(U0)
        dt = d.linear_timestep_max()
        nsteps = int(round(2 * 3600.0 / dt))
        eta_t = _dipoles(lon, lat, 1, seed=8, band=((lon[0] + 5, lat[0] + 5), (lon[-1] - 5, lat[-1] - 5)))[0]
        Ut = U0.copy()
        Ut[0] = np.where(wet, eta_t, 0.0)
        d.set_U(Ut)
        d.gauges_setup(gauges, capacity=nsteps + 8)
        stream = torch.cuda.ExternalStream(d.stream(), device=f"cuda:{local}")
        d.evolve_steps(nsteps, dt)
        target = d.gauges_read()[:nsteps, :, 0].copy()
        Ui = U0.copy()
        Ui[0] = 0.0
        times_f, times_a = [], []
        for _ in range(max(1, args.steps)):
            d.set_U(Ui)
            d.gauges_reset()
            d.time = 0.0
            d.synchronize()
            times_f.append(_event_ms(stream, lambda: d.evolve_steps(nsteps, dt)))
            d.set_U(Ui)
            d.time = 0.0
            d.synchronize()
            res = {}

            def grad_call():
                res["lg"] = d.misfit_gradient(nsteps, dt, target, checkpoint_every=50)
            # Device time on the domain's stream, including the gradient's
            # copy back to the host (the forward solve above has no copy).
            times_a.append(_event_ms(stream, grad_call))
            loss, grad = res["lg"]
        f_ms, a_ms = min(times_f), min(times_a)
        line.update({"workload": f"adjoint_linear_spherical_{nxg}x{nyg}_fp64", "value": nxg * nyg * nsteps /
                     (a_ms / 1e3), "steps": args.steps, "ms_per_step": a_ms, "dtype": "f64",
                     "config": {"workload": f"adjoint_linear_spherical_{nxg}x{nyg}_fp64", "nsteps": nsteps,
                                "dt": dt, "gauges": 30, "checkpoint_every": 50},
                     "forward_ms": f_ms, "gradient_ms": a_ms, "gradient_over_forward": a_ms / f_ms,
                     "loss": loss, "grad_norm": float(np.linalg.norm(grad[0]))})
        d.close()
    elif args.workload == "multidomain":
        line.update(_run_multidomain(args, local, peak, peak_kind))
    print(json.dumps(line), flush=True)


def _coast_elevation(lon, lat, coasts):
    """Deep ocean (-4000 m) shoaling over a 60 km shelf slope to -50 m, then a
    1/40 coastal ramp to +10 m, for each straight coastline (lon0, lat0,
    bearing of the seaward normal, (lon_min, lon_max, lat_min, lat_max) of
    the region it shapes)."""
    import numpy as np
    km = 111.19
    elv = np.full(np.broadcast(lon, lat).shape, -4000.0)
    for (x0, y0, ang, box) in coasts:
        inside = (lon >= box[0]) & (lon <= box[1]) & (lat >= box[2]) & (lat <= box[3])
        # seaward distance (km) from the coastline
        d = ((lon - x0) * np.cos(np.deg2rad(y0)) * np.cos(ang) + (lat - y0) * np.sin(ang)) * km
        ramp = np.clip(-50.0 - (d * 1000.0) / 40.0, -50.0, 10.0)           # within ~2.4 km of the coast
        shelf = np.clip(-50.0 - (d - 0.0) * (3950.0 / 60.0), -4000.0, -50.0)  # 60 km shelf slope
        e = np.where(d <= 0.0, ramp, shelf)
        elv = np.where(inside, np.maximum(elv, e), elv)
    return elv


def _run_multidomain(args, local, peak, peak_kind):
    """Nested multidomain in the shape of the 5-domain configuration: a
    coarse 'linear' FP32 band (4 arcmin, 5400x1800, 60S-60N, periodic in
    longitude over 0-360 through periodic self-exchanges), one ratio-3
    'rk2' FP64 domain (900x900) and two ratio-9 'rk2' FP64 wet/dry domains
    (1197x801 and 702x1098, the nearest sizes that are whole parent cells)
    on synthetic coastal ramps; one dipole source; fixed md step from the
    coarse domain's CFL, refinement factors from each domain's stationary
    CFL; graph-captured md steps."""
    import math
    import numpy as np
    import torch
    from ptha_b200 import Multidomain, NestDomain
    c = 1.0 / 15.0                     # coarse cell (degrees)
    f3, f9 = c / 3.0, c / 9.0
    specs = [
        NestDomain((0.0, -60.0), (5400 * c, 1800 * c), (5400, 1800), "linear", 1),
        NestDomain((140.0, -40.0), (900 * f3, 900 * f3), (900, 900), "rk2", 1),
        NestDomain((141.0 + 2 * c, -39.0), (1197 * f9, 801 * f9), (1197, 801), "rk2", 1),
        NestDomain((152.0, -35.0), (702 * f9, 1098 * f9), (702, 1098), "rk2", 1),
    ]
    coasts = [(141.0 + 2 * c + 1197 * f9 * 0.75, -39.0 + 801 * f9 * 0.5, 0.0,
               (140.5, 151.0, -39.5, -32.5)),
              (152.0 + 702 * f9 * 0.5, -35.0 + 1098 * f9 * 0.8, math.pi / 2,
               (151.5, 157.7, -35.5, -26.3))]
    # Refinement factors from the stationary CFL limits need the domains;
    # set them up once with nt = 1, read the limits, then build the real nest.
    kw = [dict(real_bytes=4, spherical=True), dict(spherical=True), dict(spherical=True), dict(spherical=True)]

    def build(nts):
        sp = [NestDomain(s.lower_left, s.lw, s.nx, s.timestepping_method, nt) for s, nt in zip(specs, nts)]
        md = Multidomain(sp, domain_kwargs=kw, use_wetdry_limiting=True, flux_correction=True, device=local,
                         periodic_xs=(0.0, 360.0))
        for k, (s, d) in enumerate(zip(sp, md.domains)):
            lon, lat = s.x(), s.y()
            LON, LAT = np.meshgrid(lon, lat)
            elv = _coast_elevation(LON, LAT, coasts)
            if k == 0:   # walls north and south; periodic east-west
                elv[:2, :] = 100.0
                elv[-2:, :] = 100.0
            eta = _dipoles(lon, lat, 1, seed=11, band=((144.0, -37.0), (150.0, -30.0)))[0]
            U = np.zeros((4, s.nx[1], s.nx[0]))
            U[3] = elv
            U[0] = np.where(elv < 0, eta, elv)
            d.set_U(U)
            if d.timestepping_method == "rk2":
                d.set_manning_squared(0.025 ** 2)
        return sp, md

    sp, md = build([1, 1, 1, 1])
    dt = md.domains[0].linear_timestep_max()
    lims = [d.stationary_timestep_max() if d.timestepping_method == "rk2" else dt for d in md.domains]
    nts = [max(1, int(math.ceil(dt / l))) for l in lims]
    md.close()
    sp, md = build(nts)
    cells = sum(s.nx[0] * s.nx[1] * nt for s, nt in zip(sp, nts))
    stream = torch.cuda.ExternalStream(md.domains[0].stream(), device=f"cuda:{local}")
    K = 3
    for _ in range(args.warmup):
        md.evolve_one_step(dt)
    md.synchronize()
    ms_plain = _event_ms(stream, lambda: [md.evolve_one_step(dt) for _ in range(K * 4)]) / (K * 4)
    md.capture_graph(K, dt)
    md.replay(1)
    md.synchronize()
    reps = max(1, args.inner if args.inner != INNER else 100)
    l0 = md.launch_count()
    ms = _event_ms(stream, lambda: md.replay(reps))
    ms_step = ms / (reps * K)
    value = cells / (ms_step / 1e3)
    vols = [d.volume_interior() for d in md.domains]
    out = {"workload": "nested_multidomain_4dom", "value": value, "steps": reps * K, "ms_per_step": ms_step,
           "dtype": "f32 coarse / f64 fine",
           "config": {"workload": "nested_multidomain_4dom",
                      "domains": [{"nx": list(s.nx), "method": s.timestepping_method, "nt": nt,
                                   "nest_layer_width": s.nest_layer_width} for s, nt in zip(sp, nts)],
                      "md_dt": dt, "exchanges": len(md.exchanges), "flux_correction": True,
                      "graph_steps": K, "sources": 1, "periodic_xs": [0.0, 360.0]},
           "cell_updates_per_md_step": cells,
           "ms_per_md_step_without_graph": ms_plain,
           "graph_replay_speedup": ms_plain / ms_step,
           "gpu_launches_per_md_step_graph": 1.0 / K,
           "finite": bool(all(np.isfinite(v) for v in vols))}
    md.close()
    return out


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
    ap.add_argument("--workload", default="rk2", choices=["rk2", "linear", "batched", "adjoint", "multidomain"],
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
