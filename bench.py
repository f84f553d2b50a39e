#!/usr/bin/env python
"""Benchmark of the fused FP32 3D viscoelastic time step on B200.

Workload (the configuration the headline metric is quoted on): 3D
viscoelastic forward run, 1024 x 1024 x 512 cells, dx = dy = dz = 0.1 km,
dt = 0.005 s, nm = 3 Zener mechanisms fitted over 0.05-2 Hz, ADE-CFS PML of
32 cells, free surface at z = 0 (air layer of 3 cells above), the four-layer
background perturbed by a seeded von Karman medium (eps = 5 %, a = 5 km,
kappa = 0.5), 8 double couples at seeded depths 5-15 km, 1024 surface
stations.  All inputs are seeded synthetic data.

A step is one full time step (stress + velocity, interior + absorber,
sources, receivers) over every cell.  Metric: Gcell-updates/s.

Arms
  default            this library on the GPU (CUDA graphs of the C-ABI step)
  --impl reference   the CPU restatement of the reference's Fortran path
                     (the oracle; the Fortran reference cannot be compiled
                     here), all host threads, on a bounded sample of the same
                     workload.

Multi-GPU (torchrun): one independent replica per GPU (the hot path has no
inter-GPU exchange on one domain per GPU); value = cells x steps x N / max
time over ranks.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "Gcell-updates/s (3D visco, FP32)"
UNIT = "Gcell-updates/s"
# algorithmic bytes per cell-update (FP32 storage, nm = 3): each array read
# once per phase that needs it and written once
B_STRESS_INT, B_STRESS_PML = 58 * 4, 38 * 4
B_VEL_INT, B_VEL_PML = 15 * 4, 33 * 4
FALLBACK_HBM_GBS = 6650.0
# DRAM traffic of one launch measured by ncu (dram__bytes_read.sum + dram__bytes_write.sum) on the c1 mix scaled
# down by 4 per axis (256x256x128, na = 8: 1/64 of c1's interior and PML cells), divided by that launch's
# algorithmic bytes; profiles/stress3d_kernel_256x256x128_na8.md and profiles/vel3d_kernel_256x256x128_na8.md
TRAFFIC_PER_ALGORITHMIC = {"stress": 1.988e9 / 1.828028416e9, "vel": 0.652e9 / 0.609632256e9}


def make_params(name: str):
    """Parameters of the named workload (the synthetic inputs are seeded)."""
    from openswpc_b200.params import Layer, Params, Station, dc_source

    layers = [Layer(0.0, 2.7, 5.5, 3.2, 300, 150), Layer(5.0, 2.8, 6.0, 3.5, 500, 250),
              Layer(18.0, 2.9, 6.7, 3.9, 600, 300), Layer(30.0, 3.3, 7.8, 4.5, 1000, 500)]
    if name == "c1":
        nx, ny, nz, dx, dt, nt, na, nsrc, nst = 1024, 1024, 512, 0.1, 0.005, 4000, 32, 8, 1024
    elif name == "c4":
        nx, ny, nz, dx, dt, nt, na, nsrc, nst = 512, 512, 256, 0.2, 0.01, 3000, 32, 8, 256
    elif name == "c0":
        nx, ny, nz, dx, dt, nt, na, nsrc, nst = 192, 192, 96, 0.5, 0.02, 1000, 20, 1, 16
    else:
        raise ValueError(name)
    rng = np.random.default_rng(20241203)
    xb, yb = -nx // 2 * dx, -ny // 2 * dx
    srcs = []
    for s in range(nsrc):
        if nsrc == 1:
            x, y, z = 0.0, 0.0, 10.0
        else:
            x = float(rng.uniform(xb + (na + 10) * dx, xb + (nx - na - 10) * dx))
            y = float(rng.uniform(yb + (na + 10) * dx, yb + (ny - na - 10) * dx))
            z = float(rng.uniform(5.0, 15.0))
        srcs.append(dc_source(x, y, z, 0.0, 2.0, 1e16, 30, 60, 90))
    st = [Station(float(rng.uniform(xb + (na + 2) * dx, xb + (nx - na - 2) * dx)),
                  float(rng.uniform(yb + (na + 2) * dx, yb + (ny - na - 2) * dx)), 0.0, f"s{n:04d}", "fsb")
          for n in range(nst)]
    return Params(nx=nx, ny=ny, nz=nz, nt=nt, dx=dx, dy=dx, dz=dx, dt=dt, na=na, nm=3, xbeg=xb, ybeg=yb,
                  zbeg=-3 * dx, fq_min=0.05, fq_max=2.0, layers=layers, sources=srcs, stations=st, ntdec_w=1,
                  ntdec_r=50)


def cell_counts(p):
    ni, nj, nk = p.nx - 2 * p.na, p.ny - 2 * p.na, p.nz - p.na
    n_int = ni * nj * nk
    return n_int, p.nx * p.ny * p.nz - n_int


def rmed(p, seed=5, device=None):
    from openswpc_b200.media import vonkarman_3d

    return vonkarman_3d((p.ny + 6, p.nx + 6, p.nz + 6), p.dx, p.dy, p.dz, 0.05, 5.0, 0.5, seed, device)


def hbm_peak():
    f = ROOT / "MEASURED_PEAKS.json"
    if f.exists():
        try:
            return float(json.loads(f.read_text())["hbm_gbs"]), "measured"
        except Exception:
            pass
    return FALLBACK_HBM_GBS, "fallback"


class ClockSampler:
    """Samples SM clock and throttle reasons through NVML while running."""

    REASONS = {0x1: "gpu_idle", 0x2: "applications_clocks_setting", 0x4: "sw_power_cap", 0x8: "hw_slowdown",
               0x10: "sync_boost", 0x20: "sw_thermal_slowdown", 0x40: "hw_thermal_slowdown",
               0x80: "hw_power_brake_slowdown", 0x100: "display_clock_setting"}

    def __init__(self, device_index: int):
        self.samples = []
        self.reasons = 0
        self.ok = False
        self.max_mhz = None
        try:
            import pynvml

            pynvml.nvmlInit()
            vis = os.environ.get("CUDA_VISIBLE_DEVICES")
            idx = int(vis.split(",")[device_index]) if vis else device_index
            self.h = pynvml.nvmlDeviceGetHandleByIndex(idx)
            self.nv = pynvml
            self.max_mhz = pynvml.nvmlDeviceGetMaxClockInfo(self.h, pynvml.NVML_CLOCK_SM)
            self.ok = True
        except Exception:
            pass
        self._stop = threading.Event()

    def _loop(self):
        while not self._stop.is_set():
            try:
                self.samples.append(self.nv.nvmlDeviceGetClockInfo(self.h, self.nv.NVML_CLOCK_SM))
                self.reasons |= self.nv.nvmlDeviceGetCurrentClocksEventReasons(self.h)
            except Exception:
                pass
            time.sleep(0.05)

    def __enter__(self):
        if self.ok:
            self.t = threading.Thread(target=self._loop, daemon=True)
            self.t.start()
        return self

    def __exit__(self, *a):
        self._stop.set()
        if self.ok:
            self.t.join()

    def summary(self):
        if not self.ok or not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": self.max_mhz, "reasons": ["nvml unavailable"]}
        r = [name for bit, name in self.REASONS.items() if self.reasons & bit and name != "gpu_idle"]
        return {"sm_mhz": float(np.median(self.samples)), "sm_max_mhz": self.max_mhz, "reasons": r,
                "samples": len(self.samples)}


def cpu_reference(p, xi, steps: int, warmup: int, threads: int, budget_s: float | None = None):
    """Time the oracle on a bounded sample of the workload: the full-depth
    column block of nx_s x ny_s cells at the centre of the same medium."""
    from oracle.oracle import Oracle3D
    from openswpc_b200.params import Params

    ns = min(256, p.nx)
    i0 = (p.nx - ns) // 2
    j0 = (p.ny - ns) // 2
    q = Params(**{**p.__dict__})
    q.nx, q.ny = ns, ns
    q.xbeg = float(np.float32(p.xbeg) + np.float32(i0) * np.float32(p.dx))
    q.ybeg = float(np.float32(p.ybeg) + np.float32(j0) * np.float32(p.dy))
    q.stations = []
    q.sources = [s for s in p.sources][:1]
    xs = np.ascontiguousarray(xi[j0:j0 + ns + 6, i0:i0 + ns + 6, :]) if xi is not None else None
    o = Oracle3D(q, xs, variant="f32", threads=threads)
    for it in range(1, warmup + 1):
        o.step(it)
    t0 = time.perf_counter()
    n = 0
    for it in range(warmup + 1, warmup + 1 + steps):
        o.step(it)
        n += 1
        if budget_s and time.perf_counter() - t0 > budget_s and n >= 2:
            break
    dt = time.perf_counter() - t0
    cells = q.nx * q.ny * q.nz
    o.close()
    return cells * n / dt / 1e9, n, cells, dt


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=30)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--workload", default="c1", choices=["c1", "c0", "c4"])
    ap.add_argument("--grid", default=None, help="override the grid as NXxNYxNZ (profiling runs)")
    ap.add_argument("--na", type=int, default=None, help="override the PML width (profiling runs)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-budget", type=float, default=20.0, help="seconds of CPU work for cpu_baseline")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    p = make_params(args.workload)
    if args.grid:
        nx, ny, nz = (int(v) for v in args.grid.lower().split("x"))
        p.nx, p.ny, p.nz = nx, ny, nz
        p.xbeg, p.ybeg = -nx // 2 * p.dx, -ny // 2 * p.dy
        lim = lambda lo, hi: (lambda v: min(max(v, lo), hi))
        for s in p.sources:
            s.x = lim(p.xbeg + (p.na + 4) * p.dx, p.xbeg + (nx - p.na - 4) * p.dx)(s.x)
            s.y = lim(p.ybeg + (p.na + 4) * p.dy, p.ybeg + (ny - p.na - 4) * p.dy)(s.y)
            s.z = min(s.z, (nz - p.na - 4) * p.dz + p.zbeg)
        p.stations = [st for st in p.stations if p.xbeg + (p.na + 2) * p.dx < st.x < p.xbeg + (nx - p.na - 2) * p.dx
                      and p.ybeg + (p.na + 2) * p.dy < st.y < p.ybeg + (ny - p.na - 2) * p.dy]
    if args.na is not None:
        p.na = args.na
    n_int, n_pml = cell_counts(p)
    cells = p.nx * p.ny * p.nz
    wl = {"workload": f"3D viscoelastic forward {p.nx}x{p.ny}x{p.nz} (nm=3, PML {p.na}, von Karman medium, "
                      f"{len(p.sources)} double couples, {len(p.stations)} stations)",
          "nx": p.nx, "ny": p.ny, "nz": p.nz, "dx_km": p.dx, "dt_s": p.dt, "na": p.na, "nm": p.nm,
          "cells": cells, "interior_cells": n_int, "pml_cells": n_pml,
          "l2": "inputs larger than L2 (whole wavefield + medium resident, tens of GB)",
          "parallelism": f"replicas x{args.gpus}"}

    if args.impl == "reference":
        if rank != 0:
            return
        threads = os.cpu_count() or 1
        xi = rmed(p, device="cpu")
        # each step = one oracle step over the bounded sample (warm-up untimed)
        v, n, sample_cells, dt = cpu_reference(p, xi, args.steps, args.warmup, threads)
        line = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus,
                "steps": n, "warmup": args.warmup, "ms_per_step": dt / n * 1e3, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                "config": wl,
                "cpu_baseline": {"value": v, "unit": UNIT, "cores": threads, "kind": "port",
                                 "sample": f"oracle f32 (CPU restatement of the Fortran path; the Fortran "
                                           f"reference cannot be compiled here), one step per timed step over "
                                           f"the centre {256}x{256}x{p.nz} column block of the same medium"},
                "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line), flush=True)
        return

    import torch
    from openswpc_b200 import _lib
    from openswpc_b200.swpc3d import Medium, Swpc3D

    dist = None
    if world > 1:
        import torch.distributed as dist_mod
        from datetime import timedelta

        dist = dist_mod
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=timedelta(seconds=600), device_id=torch.device("cuda", local))

    def barrier():
        if dist is not None:
            dist.barrier()

    def max_over_ranks(x: float) -> float:
        if dist is None:
            return x
        t = torch.tensor([x], device=f"cuda:{local}", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    device = local
    xi = rmed(p, device=f"cuda:{device}")
    med = Medium(p, xi)
    torch.cuda.empty_cache()
    sim = Swpc3D(p, device=device, medium=med)
    lib = sim.lib
    ctx = sim.ctx

    # ---- device throughput: CUDA-graph replays of the whole step ----------
    sim.run(1, args.warmup)
    sim.sync()
    barrier()
    torch.cuda.synchronize(device)
    it0 = args.warmup + 1
    with ClockSampler(device) as clk:
        ms = C.c_float()
        _lib.check(ctx, lib.swpc_time_steps(ctx, it0, args.steps, C.byref(ms)))
        ms_total = ms.value
    torch.cuda.synchronize(device)
    barrier()
    ms_total = max_over_ranks(ms_total)
    ms_step = ms_total / args.steps
    value = cells * args.steps * world / (ms_total / 1e3) / 1e9

    # ---- per-kernel times for the roofline (CUDA events on the ctx stream) --
    stream = torch.cuda.ExternalStream(lib.swpc_stream(ctx), device=device)
    ev = [[torch.cuda.Event(enable_timing=True) for _ in range(4)] for _ in range(args.steps)]
    it = it0 + args.steps
    nk = min(args.steps, p.nt - it + 1)
    for n in range(nk):
        e = ev[n]
        _lib.check(ctx, lib.swpc_wav_store(ctx, it + n))
        e[0].record(stream)
        _lib.check(ctx, lib.swpc_update_stress(ctx))
        e[1].record(stream)
        _lib.check(ctx, lib.swpc_source_stressglut(ctx, it + n))
        e[2].record(stream)
        _lib.check(ctx, lib.swpc_update_vel(ctx))
        e[3].record(stream)
    stream.synchronize()
    t_stress = np.mean([ev[n][0].elapsed_time(ev[n][1]) for n in range(nk)])
    t_vel = np.mean([ev[n][2].elapsed_time(ev[n][3]) for n in range(nk)])
    b_stress = n_int * B_STRESS_INT + n_pml * B_STRESS_PML
    b_vel = n_int * B_VEL_INT + n_pml * B_VEL_PML
    peak, peak_kind = hbm_peak()
    ach_stress = b_stress / (t_stress / 1e3) / 1e9
    ach_vel = b_vel / (t_vel / 1e3) / 1e9
    ach_step = (b_stress + b_vel) / (ms_step / 1e3) / 1e9

    # ---- end to end through the C ABI with host buffers ---------------------
    # medium upload from pinned host memory + per-routine C-ABI calls per step
    # (vmax report every ntdec_r) + trace download, all inside the timed region
    pinned = {}
    for name in Medium.FIELDS[1:]:
        a = getattr(med, name)
        t = torch.empty(a.shape, dtype=torch.float32, pin_memory=True)
        t.numpy()[...] = a
        pinned[name] = t
        setattr(med, name, t.numpy())
    view = med.view()
    ntw, nst = C.c_int(), C.c_int()
    lib.swpc_wav_dims(ctx, C.byref(ntw), C.byref(nst))
    tr = torch.empty((nst.value, 3, ntw.value), dtype=torch.float32, pin_memory=True)
    vm = (C.c_float * 3)()
    barrier()
    torch.cuda.synchronize(device)
    t0 = time.perf_counter()
    _lib.check(ctx, lib.swpc_upload_medium(ctx, C.byref(view)))
    it = 1
    for n in range(args.steps):
        if it % p.ntdec_r == 0:
            _lib.check(ctx, lib.swpc_vmax(ctx, vm))
        _lib.check(ctx, lib.swpc_wav_store(ctx, it))
        _lib.check(ctx, lib.swpc_update_stress(ctx))
        _lib.check(ctx, lib.swpc_source_stressglut(ctx, it))
        _lib.check(ctx, lib.swpc_update_vel(ctx))
        it += 1
    _lib.check(ctx, lib.swpc_wav_fetch(ctx, _lib.WAV_V, tr.numpy().ctypes.data_as(C.POINTER(C.c_float))))
    _lib.check(ctx, lib.swpc_sync(ctx))
    t_e2e = max_over_ranks(time.perf_counter() - t0)
    e2e_val = cells * args.steps * world / t_e2e / 1e9
    med_bytes = sum(v.nbytes for v in pinned.values())
    h2d = med_bytes / args.steps
    d2h = (tr.numel() * 4 + 12 * (args.steps // p.ntdec_r)) / args.steps

    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded layered + von Karman medium)",
            "config": wl,
            "roofline": {"bound": "hbm", "kernel": "stress3d_kernel (fused interior + PML stress update)",
                         "achieved": ach_stress, "peak": peak, "unit": "GB/s", "frac": ach_stress / peak,
                         "peak_kind": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured"
                         else "fallback 6650 GB/s",
                         "traffic": b_stress * TRAFFIC_PER_ALGORITHMIC["stress"],
                         "traffic_source": "ncu DRAM bytes of the 1/64-scale case times 64 (same interior/PML mix)",
                         "algorithmic_bytes_per_launch": b_stress, "launch_ms": t_stress},
            "roofline_vel": {"kernel": "vel3d_kernel", "achieved": ach_vel, "frac": ach_vel / peak,
                             "traffic": b_vel * TRAFFIC_PER_ALGORITHMIC["vel"],
                             "algorithmic_bytes_per_launch": b_vel, "launch_ms": t_vel},
            "roofline_step": {"achieved": ach_step, "frac": ach_step / peak,
                              "algorithmic_bytes_per_step": b_stress + b_vel},
            "e2e": {"value": e2e_val, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                    "what": "medium upload from pinned host memory + per-routine C-ABI step calls + vmax "
                            "reports + trace download, wall clock, max over ranks"},
            "gpu_launches": args.steps * (3 + 1 + 1),
            "clocks": clk.summary()}
    sim.close()
    if rank == 0 and not args.no_cpu_baseline:
        v, n, sc, dt = cpu_reference(p, xi, 1000, 1, os.cpu_count() or 1, budget_s=args.cpu_budget)
        line["cpu_baseline"] = {"value": v, "unit": UNIT, "cores": os.cpu_count() or 1, "kind": "port",
                                "sample": f"oracle f32 on the centre 256x256x{p.nz} column block, {n} steps "
                                          f"after 1 warm-up ({dt:.1f} s)"}
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
