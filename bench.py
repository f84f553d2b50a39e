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

from openswpc_b200 import replicas  # noqa: E402  (rank logic; no CUDA at import)

METRIC = "Gcell-updates/s (3D visco, FP32)"
UNIT = "Gcell-updates/s"
# algorithmic bytes per cell-update (FP32 storage, nm = 3): each array read
# once per phase that needs it and written once
B_STRESS_INT, B_STRESS_PML = 58 * 4, 38 * 4
B_VEL_INT, B_VEL_PML = 15 * 4, 33 * 4
# the same per storage form of S and R: (stress int, stress PML, vel int, vel PML); BF16 R saves 36 x 2 B of the
# interior stress phase, FP16 S + R also 12 x 2 B of stress and 6 x 2 B of velocity accesses per cell
BYTES = {"f32": (232, 152, 60, 132), "bf16r": (160, 152, 60, 132), "f16r": (160, 152, 60, 132),
         "f16sr": (136, 128, 48, 120)}
FALLBACK_HBM_GBS = 6650.0
# DRAM traffic of one launch measured by ncu (dram__bytes_read.sum + dram__bytes_write.sum) on the c1 mix scaled
# down by 4 per axis (256x256x128, na = 8: 1/64 of c1's interior and PML cells), divided by that launch's
# algorithmic bytes, for the default (TMA-staged) kernels (the ncu summaries of stress3d_tma_kernel and
# vel3d_tma_kernel on that grid, under profiles/)
TRAFFIC_PER_ALGORITHMIC = {"stress": (1.261579e9 + 0.708133e9) / 1.828028416e9,
                           "vel": (0.510744e9 + 0.124089e9) / 0.609632256e9}


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


# 2D P-SV algorithmic bytes per cell-update (FP32, nm = 3): velocity phase 2 V read+write, 3 S, rho; stress
# phase 2 V, 3 S read+write, 9 R read+write, lam, mu, taup, taus (interior); PML: 34 floats
B_PSV_INT, B_PSV_PML = 38 * 4, 34 * 4
# DRAM traffic of the staged 2D kernels over their algorithmic bytes, measured by ncu on the first 16 c2A models
# (stress 0.941 + 0.546 GB, velocity 0.328 + 0.087 GB against 1.481 + 0.430 GB; the 2D batch summary under profiles/)
TRAFFIC_PER_ALGORITHMIC_2D = (0.941275 + 0.545625 + 0.328020 + 0.086632) / (1.4813472 + 0.429801472)
# one adjoint step per cell (FP32 state, FP32 segment sums of the gradients, nm = 3), interior / absorber:
# velocity weights (lV, b read, nine w40 + nine w41 written, the three stress divergences of the slot read, three b
# gradient sums read and written; absorber: nine PML auxiliaries read and written instead of the divergences and
# sums), velocity gather (18 weights read, six lS read and written), stress weights (lS, seven medium fields, 18 lR
# read and written, 18 weights written, V of the slot, five medium gradient sums read and written; absorber: lS,
# five medium fields, nine auxiliaries, 18 weights), stress gather (18 weights read, three lV read and written)
B_ADJ_INT = (12 + 12 + 72 + 12 + 24) + (72 + 48) + (24 + 28 + 144 + 72 + 12 + 40) + (72 + 24)
B_ADJ_PML = (12 + 12 + 72 + 72) + (72 + 48) + (24 + 20 + 72 + 72) + (72 + 24)
# inside a checkpoint segment the stress gather of each step forms the velocity weights of the next from the lV it
# has just summed, so every step but the first of a segment reads lV once instead of twice
B_ADJ_FUSED_SAVES = 12
# every forward step whose slot is kept or recomputed: V copied into the slot over the kernel region with a two-cell
# halo in i, j and k (read and written), and the three stress divergences of the interior cells formed from S (six
# read, three written)
B_SLOT = 3 * 4 * 2
B_SLOT_INT = 6 * 4 + 3 * 4
# V, S and R (27 fields) saved at each checkpoint and restored before the segment's recompute; at the end of each
# segment the eight FP32 gradient sums (read, zeroed) folded into the FP64 totals (read and written)
B_CKPT = 27 * 4 * 2 * 2 + 8 * (4 * 2 + 8 * 2)


def make_c2a_models(n: int = 64, seed: int = 20260203):
    """The batched-ensemble workload: n seeded P-SV models of uneven size
    (nx in [256, 2048], nz in [128, 1024]), dx = 0.1 km, dt = 0.005 s,
    nt = 3000, 3-6 layers with vs 1.5-4.5 km/s (increasing with depth),
    vp/vs 1.7-1.9, rho from Gardner's law (rho = 1.741 vp^0.25), Q = 50 vs
    (Qp = 2 Qs), nm = 3, one explosion (mxx = mzz = 1) with a Kupper wavelet
    of T = 0.5 s, 16 surface stations."""
    from openswpc_b200.params import Layer, Params, Source, Station

    rng = np.random.default_rng(seed)
    out = []
    for m in range(n):
        nx = int(rng.integers(256, 2049))
        nz = int(rng.integers(128, 1025))
        dx = 0.1
        nl = int(rng.integers(3, 7))
        tops = [0.0] + sorted(float(v) for v in rng.uniform(0.3, 0.8 * nz * dx, nl - 1))
        vs = np.sort(rng.uniform(1.5, 4.5, nl))
        vp = vs * rng.uniform(1.7, 1.9, nl)
        layers = [Layer(tops[l], float(1.741 * vp[l] ** 0.25), float(vp[l]), float(vs[l]), float(100 * vs[l]),
                        float(50 * vs[l])) for l in range(nl)]
        xb = -(nx // 2) * dx
        na = 20
        src = [Source(float(rng.uniform(xb + (na + 10) * dx, -xb - (na + 10) * dx)), 0.0,
                      float(rng.uniform(0.5, 0.5 * (nz - na) * dx)), 0.0, 0.5, mo=1e15, mxx=1.0, myy=1.0, mzz=1.0)]
        st = [Station(float(xb + (na + 2 + (nx - 2 * na - 4) * (q + 0.5) / 16) * dx), 0.0, 0.0, f"s{q:02d}", "fsb")
              for q in range(16)]
        out.append(Params(nx=nx, ny=1, nz=nz, nt=3000, dx=dx, dy=dx, dz=dx, dt=0.005, na=na, nm=3, xbeg=xb,
                          ybeg=0.0, zbeg=-3 * dx, fq_min=0.05, fq_max=4.0, layers=layers, sources=src, stations=st,
                          ntdec_w=5, ntdec_r=100))
    return out


def c2a_cells(ps):
    n_int = sum((p.nx - 2 * p.na) * (p.nz - p.na) for p in ps)
    return n_int, sum(p.nx * p.nz for p in ps) - n_int


def bench_c2a(args, world, rank, local):
    """Batched 2D P-SV ensemble (one persistent launch per half step, CUDA
    graph) against the plain per-model loop on the same GPU."""
    ps_all = make_c2a_models()
    ps_all = [ps_all[args.only_model]] if args.only_model is not None else ps_all[:args.models]
    ps = replicas.shard(ps_all, world, rank)   # members shard across GPUs
    wl = {"workload": f"batched ensemble of {len(ps_all)} uneven 2D P-SV models (nx 256-2048, nz 128-1024, nm=3, "
                      f"PML 20)",
          "models": len(ps_all), "cells": sum(p.nx * p.nz for p in ps_all),
          "l2": "inputs larger than L2 (all members resident, several GB)", "parallelism": f"members/{world} GPUs"}
    if args.impl == "reference":
        if rank != 0:
            return
        from oracle.oracle import Oracle2D

        p = ps_all[0]
        o = Oracle2D(p, "psv")
        for it in range(1, args.warmup + 1):
            o.step(it)
        t0 = time.perf_counter()
        n = 0
        for it in range(args.warmup + 1, args.warmup + 1 + args.steps):
            o.step(it)
            n += 1
            if time.perf_counter() - t0 > args.cpu_budget and n >= 2:
                break
        dt = time.perf_counter() - t0
        v = p.nx * p.nz * n / dt / 1e9
        line = {"impl": "reference", "metric": "Gcell-updates/s (2D P-SV visco, FP32, batched ensemble)", "value": v,
                "unit": UNIT, "n_gpus": args.gpus, "steps": n, "warmup": args.warmup,
                "ms_per_step": dt / n * 1e3, "higher_is_better": True, "scaling": "strong", "vs_baseline": None,
                "dtype": "f32", "data": "synthetic", "config": wl,
                "cpu_baseline": {"value": v, "unit": UNIT, "cores": 1, "kind": "port",
                                 "sample": f"2D oracle f32, one thread, model 0 ({p.nx}x{p.nz}), {n} steps"},
                "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line), flush=True)
        return

    import torch
    from openswpc_b200 import _lib
    from openswpc_b200.swpc2d import Batch2D, Swpc2D

    ranks = replicas.init("nccl") if world > 1 else replicas.Ranks(1, 0, local)
    dist = ranks.dist

    max_over_ranks = ranks.max

    runs = [Swpc2D(p, "psv", device=local) for p in ps]
    lib = _lib.load()
    batch = Batch2D(runs)
    used, ti, ri, bps = batch.autotune(1, reps=2)
    pick = batch.launch()
    kern = " + ".join([("stress2d_tma_kernel" if pick["stress_ti"] else "tile2d_kernel (stress)"),
                       ("vel2d_tma_kernel" if pick["vel_ti"] else "tile2d_kernel (velocity)")])
    it0 = 1 + used
    batch.run(it0, args.warmup)
    it0 += args.warmup
    if dist is not None:
        dist.barrier()
    with ClockSampler(local) as clk:
        ms_batch = batch.time_steps(it0, args.steps)
    it0 += args.steps
    ms_batch = max_over_ranks(ms_batch)
    # the plain per-model loop: each member alone, its own CUDA graph, one after another
    ms_loop = 0.0
    for r in runs:
        check = _lib.check
        check(r.ctx, lib.swpc_run(r.ctx, it0, args.warmup))
        ms = C.c_float()
        check(r.ctx, lib.swpc_time_steps(r.ctx, it0 + args.warmup, args.steps, C.byref(ms)))
        ms_loop += ms.value
    ms_loop = max_over_ranks(ms_loop)
    # the same loop through per-step C-ABI calls (no graph), as a driver calling swpc_step would
    ms_calls = 0.0
    it1 = it0 + args.warmup + args.steps
    for r in runs:
        st = torch.cuda.ExternalStream(lib.swpc_stream(r.ctx), device=local)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        _lib.check(r.ctx, lib.swpc_sync(r.ctx))
        e0.record(st)
        for n in range(args.steps):
            _lib.check(r.ctx, lib.swpc_step(r.ctx, it1 + n))
        e1.record(st)
        e1.synchronize()
        ms_calls += e0.elapsed_time(e1)
    ms_calls = max_over_ranks(ms_calls)
    cells = wl["cells"]
    n_int, n_pml = c2a_cells(ps_all)
    value = cells * args.steps / (ms_batch / 1e3) / 1e9
    loop_value = cells * args.steps / (ms_loop / 1e3) / 1e9
    peak, peak_kind = hbm_peak()
    bytes_step = n_int * B_PSV_INT + n_pml * B_PSV_PML
    ach = bytes_step * args.steps / (ms_batch / 1e3) / 1e9

    # end to end through the C ABI: media from pinned host memory, per-step batch calls, traces back
    pinned = []
    for r in runs:
        for name in r.medium.FIELDS:
            a = getattr(r.medium, name)
            t = torch.empty(a.shape, dtype=torch.float32, pin_memory=True)
            t.numpy()[...] = a
            pinned.append(t)
            setattr(r.medium, name, t.numpy())
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize(local)
    t0 = time.perf_counter()
    for r in runs:
        _lib.check(r.ctx, lib.swpc_upload_medium(r.ctx, C.byref(r.medium.view())))
    it = 1
    for n in range(args.steps):
        rc = lib.swpc_batch_step(batch.b, it)
        if rc:
            raise RuntimeError(lib.swpc_batch_last_error(batch.b).decode())
        it += 1
    lib.swpc_batch_sync(batch.b)
    h2d = 0
    d2h = 0
    for r in runs:
        w = r.waveforms()
        d2h += w.nbytes
        m = r.medium
        h2d += sum(getattr(m, f).nbytes for f in ("rho", "lam", "mu", "taup", "taus"))
    t_e2e = max_over_ranks(time.perf_counter() - t0)
    e2e_val = cells * args.steps / t_e2e / 1e9
    line = {"metric": "Gcell-updates/s (2D P-SV visco, FP32, batched ensemble)", "value": value, "unit": UNIT,
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_batch / args.steps,
            "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded layered models)", "config": wl,
            "plain_loop": {"value": loop_value, "unit": UNIT, "ms_per_step": ms_loop / args.steps,
                           "what": "each member alone, its own CUDA graph, members one after another"},
            "plain_loop_calls": {"value": cells * args.steps / (ms_calls / 1e3) / 1e9, "unit": UNIT,
                                 "ms_per_step": ms_calls / args.steps,
                                 "what": "each member alone through per-step swpc_step calls, one after another"},
            "batched_over_loop": ms_loop / ms_batch,
            "batched_over_loop_calls": ms_calls / ms_batch,
            "autotune": {**pick, "steps_used": used},
            "roofline": {"bound": "hbm", "kernel": f"{kern} (whole batched step)",
                         "achieved": ach, "peak": peak, "unit": "GB/s", "frac": ach / peak,
                         "peak_kind": peak_kind,
                         "traffic": bytes_step * TRAFFIC_PER_ALGORITHMIC_2D if pick["stress_ti"] and pick["vel_ti"]
                         else None,
                         "traffic_source": "ncu DRAM bytes of both staged kernels on the first 16 models, as a ratio "
                                           "to their algorithmic bytes, times this step's algorithmic bytes",
                         "algorithmic_bytes_per_step": bytes_step},
            "e2e": {"value": e2e_val, "unit": UNIT, "h2d_bytes_per_step": h2d / args.steps,
                    "d2h_bytes_per_step": d2h / args.steps,
                    "what": "media upload from pinned host memory + per-step batch calls + trace download, "
                            "wall clock"},
            "gpu_launches": args.steps * 4, "clocks": clk.summary()}
    batch.close()
    for r in runs:
        r.close()
    ranks.close()
    if rank == 0:
        print(json.dumps(line), flush=True)


def make_c2b(nmem: int = 32):
    """The reciprocity batch: 384 x 384 x 192 cells of the four-layer medium
    at dx = 0.5 km, dt = 0.02 s, nt = 1000, nm = 3, PML 20; 32 single forces
    (x, y, z in turn) at seeded surface stations, Kupper T = 2 s; the members
    record at 16 seeded surface stations."""
    from openswpc_b200.params import Layer, Params, Station

    layers = [Layer(0.0, 2.7, 5.5, 3.2, 300, 150), Layer(5.0, 2.8, 6.0, 3.5, 500, 250),
              Layer(18.0, 2.9, 6.7, 3.9, 600, 300), Layer(30.0, 3.3, 7.8, 4.5, 1000, 500)]
    nx, ny, nz, dx, na = 384, 384, 192, 0.5, 20
    rng = np.random.default_rng(20241204)
    xb, yb = -nx // 2 * dx, -ny // 2 * dx
    pick = lambda lo, hi: float(rng.uniform(lo + (na + 4) * dx, lo + (hi - na - 4) * dx))
    st = [Station(pick(xb, nx), pick(yb, ny), 0.0, f"r{n:02d}", "fsb") for n in range(16)]
    fst = [Station(pick(xb, nx), pick(yb, ny), 0.0, f"f{n:02d}", "fsb") for n in range(nmem)]
    p = Params(nx=nx, ny=ny, nz=nz, nt=1000, dx=dx, dy=dx, dz=dx, dt=0.02, na=na, nm=3, xbeg=xb, ybeg=yb,
               zbeg=-3 * dx, fq_min=0.05, fq_max=2.0, layers=layers, sources=[], stations=fst + st, ntdec_w=1,
               ntdec_r=100, green_mode=True, green_trise=2.0, green_station=0, green_cmp="z")
    forces = [(fst[m], "xyz"[m % 3]) for m in range(nmem)]
    return p, forces, st


def bench_c2b(args, world, rank, local):
    """32 single-force reciprocity sources over one shared 3D medium, batched
    in one launch per half step, against the plain per-source loop."""
    nmem = 32
    wl = {"workload": "reciprocity batch: 32 single forces over one shared 384x384x192 grid (four-layer medium, "
                      "nm=3, PML 20, 16 stations)", "nx": 384, "ny": 384, "nz": 192, "members": nmem,
          "l2": "inputs larger than L2 (32 wavefields resident, ~130 GB)", "parallelism": f"members/{world} GPUs"}
    metric = "Gcell-updates/s (3D visco, FP32, reciprocity batch)"
    p, forces, st = make_c2b(nmem)
    forces = replicas.shard(forces, world, rank)   # members shard across GPUs
    cells = p.nx * p.ny * p.nz
    if args.impl == "reference":
        if rank != 0:
            return
        threads = os.cpu_count() or 1
        q = Params_copy(p)
        q.green_mode = False
        from openswpc_b200.params import dc_source
        q.sources = [dc_source(0.0, 0.0, 10.0, 0.0, 2.0, 1e16, 30, 60, 90)]
        v, n, sample_cells, dt = cpu_reference(q, None, args.steps, args.warmup, threads, budget_s=args.cpu_budget)
        line = {"impl": "reference", "metric": metric, "value": v, "unit": UNIT, "n_gpus": args.gpus, "steps": n,
                "warmup": args.warmup, "ms_per_step": dt / n * 1e3, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f32", "data": "synthetic", "config": wl,
                "cpu_baseline": {"value": v, "unit": UNIT, "cores": threads, "kind": "port",
                                 "sample": f"oracle f32, one source per run as the reference runs it, one step per "
                                           f"timed step over the centre 256x256x{p.nz} column block"},
                "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line), flush=True)
        return
    import torch
    from openswpc_b200 import _lib
    from openswpc_b200.swpc3d import ForceBatch3D, Swpc3D

    ranks = replicas.init("nccl") if world > 1 else replicas.Ranks(1, 0, local)
    dist = ranks.dist

    max_over_ranks = ranks.max

    base = Swpc3D(p, device=local)
    base.record(st)
    lib = base.lib
    # the plain per-source loop: one green-mode run (its own CUDA graph) per source, one after another; every
    # source costs the same on this grid, so the loop time is nmem x one source's time
    _lib.check(base.ctx, lib.swpc_run(base.ctx, 1, args.warmup))
    ms1 = C.c_float()
    _lib.check(base.ctx, lib.swpc_time_steps(base.ctx, 1 + args.warmup, args.steps, C.byref(ms1)))
    ms_loop = max_over_ranks(ms1.value * len(forces))
    fb = ForceBatch3D(base, forces)
    used, strip = fb.autotune(1, reps=2)
    it0 = 1 + used
    fb.run(it0, args.warmup)
    it0 += args.warmup
    if dist is not None:
        dist.barrier()
    with ClockSampler(local) as clk:
        ms_batch = fb.time_steps(it0, args.steps)
    it0 += args.steps
    ms_batch = max_over_ranks(ms_batch)
    sweep = None
    if args.sweep:
        # launch order x j block x member groups per CTA, 3 timed steps each (profiling runs); then the tuned form again
        tuned = fb.launch()
        sweep = []
        for tiles_first in (1, 0):
            for jb in (1, 2, 4, 16):
                for bi, bj, mpc in ((4, 4, 1), (4, 2, 2), (2, 2, 2), (2, 2, 4), (4, 1, 4)):
                    if it0 + 4 > p.nt:
                        break
                    _lib.check(base.ctx, lib.swpc_set_launch(base.ctx, 7, 1, jb, 1))
                    fb.set_launch(5, mpc, bi, bj)
                    fb.set_launch(6, mpc, bi, bj)
                    fb.set_launch(7, tiles_first, 0, 0)
                    fb.run(it0, 1)
                    t = fb.time_steps(it0 + 1, 3) / 3
                    it0 += 4
                    sweep.append({"tiles_first": tiles_first, "jblock": jb, "tile": [bi, bj], "members_per_cta": mpc,
                                  "ms_per_step": t, "loop_over_batch": ms_loop / args.steps / t})
        _lib.check(base.ctx, lib.swpc_set_launch(base.ctx, 7, 1, 0, 1))
        fb.set_launch(5, tuned["stress"][2], tuned["stress"][0], tuned["stress"][1])
        fb.set_launch(6, tuned["velocity"][2], tuned["velocity"][0], tuned["velocity"][1])
        fb.set_launch(7, int(tuned["tiles_first"]), 0, 0)
    n_int, n_pml = cell_counts(p)
    # algorithmic bytes: per member the 3D step without its medium reads (292 - 40 interior, 284 - 32 PML),
    # plus the medium once per step for all members
    b_mem = n_int * (B_STRESS_INT + B_VEL_INT - 40) + n_pml * (B_STRESS_PML + B_VEL_PML - 32)
    b_step = len(forces) * b_mem + n_int * 40 + n_pml * 32
    peak, peak_kind = hbm_peak()
    ach = b_step / (ms_batch / args.steps / 1e3) / 1e9
    value = cells * nmem * args.steps / (ms_batch / 1e3) / 1e9
    # end to end through the public API: the shared medium from pinned host memory (the averaged arrays formed
    # on the device), per-step batch calls, every member's traces back to the host
    med = base.medium
    pinned = []
    for name in med.FIELDS[:5]:
        a = getattr(med, name)
        t = torch.empty(a.shape, dtype=torch.float32, pin_memory=True)
        t.numpy()[...] = a
        pinned.append(t)
        setattr(med, name, t.numpy())
    view = med.view(average_on_device=True)
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize(local)
    t0 = time.perf_counter()
    _lib.check(base.ctx, lib.swpc_upload_medium(base.ctx, C.byref(view)))
    for n in range(args.steps):
        fb.step(it0 + n)
    tr = [fb.waveforms(m) for m in range(len(forces))]
    t_e2e = max_over_ranks(time.perf_counter() - t0)
    d2h = sum(t.nbytes for t in tr)
    h2d = sum(t.numel() * 4 for t in pinned)
    line = {"metric": metric, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_batch / args.steps, "higher_is_better": True,
            "scaling": "strong", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded layered medium)",
            "config": wl,
            "what": "value counts cells x members per step",
            "plain_loop": {"value": cells * nmem * args.steps / (ms_loop / 1e3) / 1e9, "unit": UNIT,
                           "ms_per_step": ms_loop / args.steps,
                           "what": "one green-mode run per source, its own CUDA graph, sources one after another"},
            "batched_over_loop": ms_loop / ms_batch,
            "autotune": {"launch": fb.launch(), "steps_used": used},
            "roofline": {"bound": "hbm", "kernel": "stress3d_tma_kernel + vel3d_tma_kernel, members grouped per CTA "
                                                     "(whole batched step)",
                         "achieved": ach, "peak": peak, "unit": "GB/s", "frac": ach / peak, "peak_kind": peak_kind,
                         "traffic": None, "algorithmic_bytes_per_step": b_step},
            "e2e": {"value": cells * len(forces) * world * args.steps / t_e2e / 1e9, "unit": UNIT,
                    "h2d_bytes_per_step": h2d / args.steps, "d2h_bytes_per_step": d2h / args.steps,
                    "what": "shared medium from pinned host memory (5 arrays; the 6 averaged ones formed on the "
                            "device) + per-step batch calls + every member's traces downloaded, wall clock"},
            "gpu_launches": args.steps * 5, "clocks": clk.summary()}
    if sweep is not None:
        line["launch_sweep"] = sweep
    fb.close()
    base.close()
    ranks.close()
    if rank == 0:
        print(json.dumps(line), flush=True)


def bench_decomp(args, world, rank, local):
    """The c4 grid split into blocks as the reference's MPI split lays them
    out (m_global.f90:236-303, default 2 x 2), all blocks on one GPU, against
    the single-domain run of the same grid: the decomposed step's rate with
    the sleeve exchange after each half step, and the exchange's pack / unpack
    kernels against HBM."""
    px, py = (int(v) for v in args.split.lower().split("x"))
    p = make_params("c4")
    wl = {"workload": f"decomposed 3D forward: the 512x512x256 grid (nm=3, PML 32) split {px}x{py}, all blocks on one "
                      f"GPU, sleeves exchanged through device buffers", "nx": p.nx, "ny": p.ny, "nz": p.nz,
          "split": [px, py], "l2": "inputs larger than L2 (whole wavefield + medium resident)",
          "parallelism": f"{px * py} blocks on one GPU"}
    metric = "Gcell-updates/s (3D visco, FP32)"
    if args.impl == "reference":
        if rank == 0:
            print(json.dumps({"impl": "reference", "unavailable": "the reference splits a grid only through its MPI "
                                                                  "build, which cannot be built here"}), flush=True)
        return
    if rank != 0:
        return
    import torch
    from openswpc_b200 import _lib
    from openswpc_b200.decomp import SIDES, Decomposed3D
    from openswpc_b200.swpc3d import Medium, Swpc3D

    cells = p.nx * p.ny * p.nz
    xi = rmed(p, device=f"cuda:{local}")
    med = Medium(p, xi)
    torch.cuda.empty_cache()
    # the single-domain run: graph replays of the step
    g = Swpc3D(p, device=local, medium=med)
    g.run(1, args.warmup)
    ms1 = C.c_float()
    _lib.check(g.ctx, g.lib.swpc_time_steps(g.ctx, 1 + args.warmup, args.steps, C.byref(ms1)))
    ms_single = ms1.value / args.steps
    g.close()
    torch.cuda.empty_cache()
    # the decomposed run: per block and half step a launch, then the exchange
    d = Decomposed3D(p, px, py, medium=med, devices=[local] * (px * py))
    for it in range(1, args.warmup + 1):
        d.step(it)
    for b in d.blocks:
        b.sync()
    with ClockSampler(local) as clk:
        t0 = time.perf_counter()
        for n in range(args.steps):
            d.step(1 + args.warmup + n)
        for b in d.blocks:
            b.sync()
        ms_dec = (time.perf_counter() - t0) * 1e3 / args.steps
    # the exchange kernels of the block with the most neighbours, timed on its stream
    b = max(d.blocks, key=lambda q: sum(n is not None for n in q.neighbours))
    lib = b.lib
    stream = torch.cuda.ExternalStream(lib.swpc_stream(b.ctx), device=local)
    sides = [s for s in range(SIDES) if b.neighbours[s] is not None]
    bufs = {(h, s): torch.empty(max(b.halo_count[h][s], b.halo_count[h][s ^ 1]), dtype=torch.float32,
                                device=f"cuda:{local}") for h in (0, 1) for s in sides}
    reps = 20
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    b.sync()
    e0.record(stream)
    for _ in range(reps):
        for h in (0, 1):
            for s in sides:
                b.pack(h, s, bufs[h, s].data_ptr())
            for s in sides:
                b.unpack(h, s, bufs[h, s].data_ptr())
    e1.record(stream)
    e1.synchronize()
    ms_halo = e0.elapsed_time(e1) / reps
    # bytes of one step's exchange on this block: pack reads and writes its messages, unpack the same
    floats = sum(b.halo_count[h][s] + b.halo_count[h][s ^ 1] for h in (0, 1) for s in sides)
    halo_bytes = 2 * 4 * floats
    peak, peak_kind = hbm_peak()
    ach = halo_bytes / (ms_halo / 1e3) / 1e9
    d.close()
    line = {"metric": metric, "value": cells / (ms_dec / 1e3) / 1e9, "unit": UNIT, "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_dec, "higher_is_better": True, "scaling": "strong",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded layered + von Karman medium)",
            "config": wl,
            "single_domain": {"value": cells / (ms_single / 1e3) / 1e9, "ms_per_step": ms_single,
                              "what": "the same grid as one context, CUDA-graph replays"},
            "decomposed_over_single": ms_single / ms_dec,
            "exchange": {"block": [b.px, b.py], "sides": len(sides), "ms_per_step": ms_halo,
                         "bytes_per_step": halo_bytes, "message_bytes_per_step": 4 * floats,
                         "achieved_gbs": ach, "peak": peak, "peak_kind": peak_kind, "frac": ach / peak,
                         "what": "pack + unpack kernels of both half steps on one block, CUDA events on its stream"},
            "timing": "wall clock around the steps, the host waiting for the blocks only at the end (the exchange "
                      "orders the blocks' streams by events)",
            "clocks": clk.summary()}
    print(json.dumps(line), flush=True)


def Params_copy(p):
    from openswpc_b200.params import Params

    return Params(**{**p.__dict__})


def make_c3(grid=None, nt=2000):
    """The adjoint-gradient workload: 256 x 256 x 128 cells, dx = 0.25 km,
    dt = 0.01 s, nt = 2000, nm = 3, PML 20; the four-layer background, one
    double couple at 8 km depth, 64 seeded surface stations.  Returns the
    parameters, the starting model (vp, vs, rho, qp, qs) and the true vs:
    the background with a seeded Gaussian blob of -8 % (radius 3 km).
    `grid` (nx, ny, nz) and `nt` shrink the case for profiling runs (the
    source and the stations stay inside the smaller grid)."""
    from openswpc_b200.params import Layer, Params, Station, dc_source
    from openswpc_b200.swpc3d import lhm_model

    layers = [Layer(0.0, 2.7, 5.5, 3.2, 300, 150), Layer(5.0, 2.8, 6.0, 3.5, 500, 250),
              Layer(18.0, 2.9, 6.7, 3.9, 600, 300), Layer(30.0, 3.3, 7.8, 4.5, 1000, 500)]
    nx, ny, nz, dx, na = 256, 256, 128, 0.25, 20
    if grid is not None:
        nx, ny, nz = grid
    rng = np.random.default_rng(20241205)
    xb, yb = -nx // 2 * dx, -ny // 2 * dx
    st = [Station(float(rng.uniform(xb + (na + 2) * dx, xb + (nx - na - 2) * dx)),
                  float(rng.uniform(yb + (na + 2) * dx, yb + (ny - na - 2) * dx)), 0.0, f"s{n:02d}", "fsb")
          for n in range(64)]
    zsrc = min(8.0, 0.5 * (nz - na) * dx)
    p = Params(nx=nx, ny=ny, nz=nz, nt=nt, dx=dx, dy=dx, dz=dx, dt=0.01, na=na, nm=3, xbeg=xb, ybeg=yb,
               zbeg=-3 * dx, fq_min=0.05, fq_max=2.0, layers=layers,
               sources=[dc_source(0.0, 0.0, zsrc, 0.0, 2.0, 1e16, 30, 60, 90)], stations=st, ntdec_w=1,
               ntdec_r=100)
    vp, vs, rho, qp, qs = lhm_model(p)
    # blob centre: seeded in the middle third of the domain, 4-12 km deep
    cx, cy = (float(rng.uniform(-nx / 6, nx / 6) * dx) for _ in range(2))
    cz = float(rng.uniform(4.0, 12.0))
    z = p.zbeg + (np.arange(-2, nz + 4) - 0.5) * dx
    y = p.ybeg + (np.arange(-2, ny + 4) - 0.5) * dx
    x = p.xbeg + (np.arange(-2, nx + 4) - 0.5) * dx
    r2 = (y[:, None, None] - cy) ** 2 + (x[None, :, None] - cx) ** 2 + (z[None, None, :] - cz) ** 2
    vs_true = (vs * (1.0 - 0.08 * np.exp(-r2 / (2 * 3.0 ** 2)))).astype(np.float32)
    return p, (vp, vs, rho, qp, qs), vs_true


def bench_c3(args, world, rank, local):
    """Checkpointed adjoint gradient of the L2 velocity misfit with respect to
    per-cell vp, vs, rho, against one plain forward run of the same model."""
    grid = tuple(int(v) for v in args.grid.lower().split("x")) if args.grid else (256, 256, 128)
    nt = args.nt or 2000
    ckpt = min(50, nt)
    wl = {"workload": f"adjoint gradient {grid[0]}x{grid[1]}x{grid[2]}, nt={nt} (nm=3, PML 20, 1 double couple, "
                      f"64 stations, checkpoint every {ckpt} steps)", "nx": grid[0], "ny": grid[1], "nz": grid[2],
          "nt": nt, "ckpt": ckpt,
          "l2": "inputs larger than L2 (wavefield, checkpoints and adjoint state resident, tens of GB)",
          "parallelism": f"replicas x{world}"}
    metric = "Gcell-updates/s (3D visco adjoint gradient, FP32, imaging sums folded into FP64 per checkpoint segment)"
    if args.impl == "reference":
        if rank != 0:
            return
        print(json.dumps({"impl": "reference", "unavailable": "the reference has no adjoint or gradient path"}),
              flush=True)
        return
    import torch
    from openswpc_b200 import _lib
    from openswpc_b200.adjoint import Misfit3D, waveform_misfit
    from openswpc_b200.swpc3d import Medium, Swpc3D

    p, (vp, vs, rho, qp, qs), vs_true = make_c3(grid, nt)
    cells = p.nx * p.ny * p.nz
    true = Swpc3D(p, device=local, medium=Medium.from_model(p, vp, vs_true, rho, qp, qs))
    _lib.check(true.ctx, true.lib.swpc_run(true.ctx, 1, p.nt))
    obs = true.waveforms(_lib.WAV_V)
    true.close()
    prob = Misfit3D(p, vp, vs, rho, qp, qs, obs, device=local, ckpt=ckpt,
                    slot_memory=0 if args.recompute_all else "auto")
    kept = prob.kept_steps()
    s = prob.solver
    lib, ctx = s.lib, s.ctx
    stream = torch.cuda.ExternalStream(lib.swpc_stream(ctx), device=local)
    J = C.c_double()
    obsf = np.ascontiguousarray(obs, np.float32)

    def t_forward():
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        _lib.check(ctx, lib.swpc_reset_state(ctx))
        e0.record(stream)
        _lib.check(ctx, lib.swpc_run(ctx, 1, p.nt))
        e1.record(stream)
        e1.synchronize()
        return e0.elapsed_time(e1)

    def t_gradient():
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        _lib.check(ctx, lib.swpc_sync(ctx))
        e0.record(stream)
        _lib.check(ctx, lib.swpc_gradient(ctx, _lib.fptr(obsf), ckpt, C.byref(J)))
        e1.record(stream)
        e1.synchronize()
        return e0.elapsed_time(e1)

    for _ in range(args.warmup):
        t_gradient()
    t_forward()
    with ClockSampler(local) as clk:
        ms_fwd = [t_forward() for _ in range(args.steps)]
        ms_grad = [t_gradient() for _ in range(args.steps)]
    fwd, grad = float(np.mean(ms_fwd)), float(np.mean(ms_grad))
    # end to end through the public API: CPU tensors in, autograd gradient out
    tv = [torch.tensor(a, requires_grad=True) for a in (vp, vs, rho)]
    t0 = time.perf_counter()
    Jt = waveform_misfit(*tv, prob)
    Jt.backward()
    t_e2e = time.perf_counter() - t0
    h2d = sum(a.nbytes for a in (vp, vs, rho)) * 2 + obsf.nbytes
    d2h = sum(t.grad.numel() * 8 for t in tv) + obsf.nbytes
    # algorithmic bytes of one gradient: the forward and the recompute of the steps whose slots are not kept (the
    # 3D step each), slot copies, the adjoint step, checkpoint save and restore of the recomputed segments
    n_int, n_pml = cell_counts(p)
    nseg = -(-p.nt // ckpt)
    nrec = -(-(p.nt - kept) // ckpt)
    b_fwd = n_int * (B_STRESS_INT + B_VEL_INT) + n_pml * (B_STRESS_PML + B_VEL_PML)
    n_slot = (p.nx - 2 * p.na + 4) * (p.ny - 2 * p.na + 4) * (p.nz - p.na + 2)
    # a kept step saves V of the shell (the slot box less the interior: written, and read back when the segment's
    # V is rebuilt) and rebuilds the interior V from its divergences (12 B read, 12 B written)
    n_shell = n_slot - n_int
    b_grad = ((2 * p.nt - kept) * b_fwd
              + (p.nt - kept) * n_slot * B_SLOT + kept * (n_shell * B_SLOT + n_int * 24)
              # kept steps: the velocity update itself stores the divergences (12 B); recomputed: slot_div_kernel
              + ((p.nt - kept) * B_SLOT_INT + kept * 12) * n_int
              + p.nt * (n_int * B_ADJ_INT + n_pml * B_ADJ_PML)
              - (p.nt - nseg) * (n_int + n_pml) * B_ADJ_FUSED_SAVES
              + nrec * (n_int + n_pml) * B_CKPT)
    peak, peak_kind = hbm_peak()
    ach = b_grad / (grad / 1e3) / 1e9
    ach_fwd = p.nt * b_fwd / (fwd / 1e3) / 1e9
    line = {"metric": metric, "value": cells * p.nt / (grad / 1e3) / 1e9, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": grad, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded layered model + "
            "Gaussian vs blob)", "config": wl,
            "what": "one step = one gradient evaluation (forward, keeping the stress divergences and the shell V of "
                    "every step of the trailing segments that fit in free HBM, checkpoints and per-segment "
                    "recompute of the others, adjoint); value counts cells x nt per gradient",
            "misfit": J.value,
            "forward_ms": fwd, "forward_gcells": cells * p.nt / (fwd / 1e3) / 1e9,
            "gradient_over_forward": grad / fwd,
            "kept_steps": kept, "recomputed_steps": p.nt - kept, "slot_memory_bytes": prob.slot_memory,
            "algorithmic_gradient_over_forward": b_grad / (p.nt * b_fwd),
            "roofline": {"bound": "hbm", "kernel": "whole gradient: stress3d_tma_kernel + vel3d_tma_kernel (forward "
                                                     "and recompute), adj_*_kernel (adjoint step), slot and "
                                                     "checkpoint copies",
                         "achieved": ach, "peak": peak, "unit": "GB/s", "frac": ach / peak, "peak_kind": peak_kind,
                         "traffic": None, "algorithmic_bytes_per_step": b_grad},
            "roofline_forward": {"achieved": ach_fwd, "frac": ach_fwd / peak,
                                 "algorithmic_bytes_per_step": p.nt * b_fwd},
            "e2e": {"value": cells * p.nt / t_e2e / 1e9, "unit": UNIT, "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h,
                    "what": "waveform_misfit(vp, vs, rho) + backward from CPU tensors: medium setup on the host, "
                            "upload, gradient, chain rule, gradients back, wall clock"},
            # per gradient: forward and recompute steps (wav, stress, injection, velocity, step counter), the
            # adjoint steps (two weight and two gather kernels, residual injection), zeroing of 8 gradients
            "gpu_launches": args.steps * ((2 * p.nt - kept) * 5 + p.nt * (3 + 5) + nseg + 8),
            "clocks": clk.summary()}
    prob.close()
    if rank == 0 and not args.no_cpu_baseline:
        # the reference has no adjoint: its CPU cost of a gradient is at least its forward run, timed here
        v, n, sc, dt = cpu_reference(p, None, 1000, 1, os.cpu_count() or 1, budget_s=args.cpu_budget)
        line["cpu_baseline"] = {"value": v, "unit": UNIT, "cores": os.cpu_count() or 1, "kind": "port",
                                "sample": f"oracle f32 forward of the starting model on the centre "
                                          f"{min(256, p.nx)}x{min(256, p.ny)}x{p.nz} column block, {n} steps after "
                                          f"1 warm-up ({dt:.1f} s); the reference has no adjoint, so this is the "
                                          f"forward part of a gradient only"}
    if rank == 0:
        print(json.dumps(line), flush=True)


def cell_counts(p):
    ni, nj, nk = p.nx - 2 * p.na, p.ny - 2 * p.na, p.nz - p.na
    n_int = ni * nj * nk
    return n_int, p.nx * p.ny * p.nz - n_int


def rmed(p, seed=5, device=None):
    """The von Karman medium of a run (eps = 5 %, a = 5 km, kappa = 0.5), generated in HBM by the library."""
    from openswpc_b200.media import vonkarman_3d

    return vonkarman_3d((p.ny + 6, p.nx + 6, p.nz + 6), p.dx, p.dy, p.dz, 0.05, 5.0, 0.5, seed, device)


def rmed_sample(p, seed=5):
    """The same statistics over the CPU baseline's centre column block, from the oracle's restatement of the
    generator (the reference arm runs without the library)."""
    from oracle.rmedia import vonkarman_box

    ns = min(256, p.nx)
    return vonkarman_box((ns + 6, ns + 6, p.nz + 6), p.dx, p.dy, p.dz, 0.05, 5.0, 0.5, seed)


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
    # xi over the whole grid, or a medium of the sample block itself
    si, sj = (0, 0) if xi is not None and xi.shape[:2] == (ns + 6, ns + 6) else (i0, j0)
    q = Params(**{**p.__dict__})
    q.nx, q.ny = ns, ns
    q.xbeg = float(np.float32(p.xbeg) + np.float32(i0) * np.float32(p.dx))
    q.ybeg = float(np.float32(p.ybeg) + np.float32(j0) * np.float32(p.dy))
    q.stations = []
    q.sources = [s for s in p.sources][:1]
    xs = np.ascontiguousarray(xi[sj:sj + ns + 6, si:si + ns + 6, :]) if xi is not None else None
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


def sample_mix(p) -> str:
    """What the CPU sample of a 3D workload is, against the workload."""
    ns = min(256, p.nx), min(256, p.ny)
    n_int, n_pml = cell_counts(p)
    si = (ns[0] - 2 * p.na) * (ns[1] - 2 * p.na) * (p.nz - p.na)
    frac = 1 - si / (ns[0] * ns[1] * p.nz)
    return (f"a grid of its own with the workload's {p.na}-cell PML on every side ({100 * frac:.0f} % absorber "
            f"cells against the workload's {100 * n_pml / (n_int + n_pml):.0f} %), one double couple, no stations")


def accuracy_sample(p, precision: str, device: int, steps: int = 200):
    """rel-L2 error of one storage form against the all-double oracle on a
    128 x 128 x 64 sample of the workload (same spacing, medium statistics,
    one source, 16 surface stations), after `steps` steps."""
    from oracle.oracle import Oracle3D
    from openswpc_b200 import _lib
    from openswpc_b200.params import Params, Station
    from openswpc_b200.swpc3d import Swpc3D

    q = Params(**{**p.__dict__})
    q.nx, q.ny, q.nz, q.na = 128, 128, 64, 16
    q.nt = steps
    q.xbeg, q.ybeg = -64 * q.dx, -64 * q.dy
    src = q.sources[0]
    q.sources = [type(src)(**{**src.__dict__, "x": 0.0, "y": 0.0, "z": min(src.z, 0.35 * q.nz * q.dz)})]
    rng = np.random.default_rng(11)
    q.stations = [Station(float(rng.uniform(-40, 40) * q.dx), float(rng.uniform(-40, 40) * q.dy), 0.0, f"a{n}", "fsb")
                  for n in range(16)]
    q.ntdec_r = 25
    xi = rmed(q, seed=9, device=device)
    o = Oracle3D(q, xi, variant="f64", threads=os.cpu_count() or 1)
    o.run(1, steps)
    g = Swpc3D(q, xi, device=device, precision=precision)
    g.run(1, steps)

    def rel(a, b):
        a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
        return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))

    out = {"sample": f"128x128x64, {steps} steps, vs f64 oracle", "traces_v": rel(g.waveforms(_lib.WAV_V), o.waveforms("v"))}
    out["final_v"] = rel(np.stack([g.download(n) for n in range(3)]), np.stack([o.array(nm) for nm in ("Vx", "Vy", "Vz")]))
    g.close()
    o.close()
    return out


def accuracy_full_grid(p, xi, precision: str, device: int, steps: int = 1000):
    """rel-L2 distance of one storage form to the FP32 form on the workload's own grid after `steps` steps
    (traces and final velocity); with the FP32 form's own error against the all-double oracle (the sample
    above) this bounds the form's error against FP64 at full size."""
    from openswpc_b200 import _lib
    from openswpc_b200.swpc3d import Swpc3D

    def rel(a, b):
        a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
        return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))

    runs = {}
    for form in (precision, "f32"):
        g = Swpc3D(p, xi, device=device, precision=form)
        g.run(1, steps)   # reports (and FP16 rescales) every ntdec_r steps
        runs[form] = (g.waveforms(_lib.WAV_V), np.stack([g.download(n) for n in range(3)]))
        g.close()
    a, b = runs[precision], runs["f32"]
    return {"grid": f"{p.nx}x{p.ny}x{p.nz}", "steps": steps, "traces_v_vs_f32": rel(a[0], b[0]),
            "final_v_vs_f32": rel(a[1], b[1])}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=30)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--workload", default="c1", choices=["c1", "c0", "c4", "c2a", "c2b", "c3", "decomp"])
    ap.add_argument("--split", default="2x2", help="decomp: blocks along x and y (nproc_x x nproc_y)")
    ap.add_argument("--models", type=int, default=64, help="c2a: the first N of the 64 models (profiling runs)")
    ap.add_argument("--only-model", type=int, default=None, help="c2a: model I of the 64 alone (profiling runs)")
    ap.add_argument("--sweep", action="store_true",
                    help="c2b: also time every launch order x j block x members-per-CTA form (profiling runs)")
    ap.add_argument("--grid", default=None, help="override the grid as NXxNYxNZ (profiling runs)")
    ap.add_argument("--na", type=int, default=None, help="override the PML width (profiling runs)")
    ap.add_argument("--recompute-all", action="store_true",
                    help="c3: keep no forward slots, recompute every segment (the smallest-memory form)")
    ap.add_argument("--nt", type=int, default=None, help="override the number of time steps (c3 profiling runs)")
    ap.add_argument("--precision", default="f32", choices=["f32", "bf16r", "f16r", "f16sr"],
                    help="storage of stress and memory variables (arithmetic is FP32)")
    ap.add_argument("--accuracy", action="store_true",
                    help="add the rel-L2 error against the f64 oracle on a 128x128x64 sample of the workload")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-secondary", action="store_true",
                    help="c1 on one GPU: skip the batched-ensemble, reciprocity, gradient and storage-form lines "
                         "measured after the headline")
    ap.add_argument("--cpu-budget", type=float, default=20.0, help="seconds of CPU work for cpu_baseline")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.workload == "c2a":
        return bench_c2a(args, world, rank, local)
    if args.workload == "c3":
        return bench_c3(args, world, rank, local)
    if args.workload == "c2b":
        return bench_c2b(args, world, rank, local)
    if args.workload == "decomp":
        return bench_decomp(args, world, rank, local)
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
        xi = rmed_sample(p)
        # each step = one oracle step over the bounded sample (warm-up untimed)
        v, n, sample_cells, dt = cpu_reference(p, xi, args.steps, args.warmup, threads)
        line = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus,
                "steps": n, "warmup": args.warmup, "ms_per_step": dt / n * 1e3, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                "config": wl,
                "cpu_baseline": {"value": v, "unit": UNIT, "cores": threads, "kind": "port",
                                 "sample": f"oracle f32 (CPU restatement of the Fortran path; the Fortran "
                                           f"reference cannot be compiled here), one step per timed step over "
                                           f"the centre {256}x{256}x{p.nz} column block of the same medium as "
                                           f"{sample_mix(p)}"},
                "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line), flush=True)
        return

    import torch
    from openswpc_b200 import _lib
    from openswpc_b200.swpc3d import DeviceMedium, Medium, Swpc3D

    ranks = replicas.init("nccl") if world > 1 else replicas.Ranks(1, 0, local)
    dist = ranks.dist

    def barrier():
        if dist is not None:
            dist.barrier()

    max_over_ranks = ranks.max

    device = local
    xi = rmed(p, device=f"cuda:{device}")
    med = Medium(p, xi)
    torch.cuda.empty_cache()
    sim = Swpc3D(p, device=device, medium=med, precision=args.precision)
    lib = sim.lib
    ctx = sim.ctx

    # ---- device throughput: CUDA-graph replays of the whole step ----------
    sim.run(1, args.warmup)
    sim.rescale()   # FP16 storage: centre the array scales (no-op otherwise)
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
    value = replicas.throughput(cells, args.steps, world, ms_total)

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
    bsi, bsp, bvi, bvp = BYTES[args.precision]
    b_stress = n_int * bsi + n_pml * bsp
    b_vel = n_int * bvi + n_pml * bvp
    peak, peak_kind = hbm_peak()
    ach_stress = b_stress / (t_stress / 1e3) / 1e9
    ach_vel = b_vel / (t_vel / 1e3) / 1e9
    ach_step = (b_stress + b_vel) / (ms_step / 1e3) / 1e9

    # ---- end to end through the C ABI with host buffers ---------------------
    # the medium from host memory, the per-routine C-ABI calls of every step
    # (vmax report every ntdec_r) and the trace download, all inside the timed
    # region.  Headline: the layer table and the pinned perturbation xi, with
    # vmodel_lhm and medium__setup run on the device (DeviceMedium).  Beside
    # it: the host-built medium from pinned memory (rho, lam, mu, taup, taus;
    # the averaged fields formed on the device).
    xi_h = torch.empty(xi.shape, dtype=torch.float32, pin_memory=True)
    xi_h.numpy()[...] = xi
    pinned = {}
    for name in Medium.FIELDS[:5]:
        a = getattr(med, name)
        t = torch.empty(a.shape, dtype=torch.float32, pin_memory=True)
        t.numpy()[...] = a
        pinned[name] = t
        setattr(med, name, t.numpy())
    view = med.view(average_on_device=True)
    ntw, nst = C.c_int(), C.c_int()
    lib.swpc_wav_dims(ctx, C.byref(ntw), C.byref(nst))
    tr = torch.empty((nst.value, 3, ntw.value), dtype=torch.float32, pin_memory=True)
    vm = (C.c_float * 3)()

    def e2e_run(load_medium):
        barrier()
        torch.cuda.synchronize(device)
        t0 = time.perf_counter()
        load_medium()
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
        return cells * args.steps * world / max_over_ranks(time.perf_counter() - t0) / 1e9

    e2e_host_val = e2e_run(lambda: _lib.check(ctx, lib.swpc_upload_medium(ctx, C.byref(view))))
    e2e_val = e2e_run(lambda: DeviceMedium(lib, ctx, p, xi_h.numpy()))
    d2h = (tr.numel() * 4 + 12 * (args.steps // p.ntdec_r)) / args.steps
    h2d = (xi_h.numel() * 4 + 24 * len(p.layers)) / args.steps
    h2d_host = sum(v.nbytes for v in pinned.values()) / args.steps

    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32",
            "storage": {"f32": "S, R FP32", "bf16r": "R BF16", "f16r": "R FP16 (power-of-two scales)",
                        "f16sr": "S, R FP16 (power-of-two scales)"}[args.precision],
            "data": "synthetic (seeded layered + von Karman medium)",
            "config": wl,
            "roofline": {"bound": "hbm", "kernel": "stress3d_tma_kernel (TMA-staged fused interior + PML stress update"
                                                     + ("" if args.precision == "f32" else
                                                        f", {args.precision} storage tiles") + ")",
                         "achieved": ach_stress, "peak": peak, "unit": "GB/s", "frac": ach_stress / peak,
                         "peak_kind": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured"
                         else "fallback 6650 GB/s",
                         "traffic": b_stress * TRAFFIC_PER_ALGORITHMIC["stress"] if args.precision == "f32" else None,
                         "traffic_source": "ncu DRAM bytes of the 1/64-scale case times 64 (same interior/PML mix)",
                         "algorithmic_bytes_per_launch": b_stress, "launch_ms": t_stress},
            "roofline_vel": {"kernel": "vel3d_tma_kernel" + (" (FP16 stress tiles)" if args.precision == "f16sr" else ""),
                             "achieved": ach_vel, "frac": ach_vel / peak,
                             "traffic": b_vel * TRAFFIC_PER_ALGORITHMIC["vel"] if args.precision == "f32" else None,
                             "algorithmic_bytes_per_launch": b_vel, "launch_ms": t_vel},
            "roofline_step": {"achieved": ach_step, "frac": ach_step / peak,
                              "algorithmic_bytes_per_step": b_stress + b_vel},
            "e2e": {"value": e2e_val, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                    "what": "layer table + random perturbation xi from pinned host memory, vmodel_lhm and "
                            "medium__setup on the device, per-routine C-ABI step calls, vmax reports, trace "
                            "download; wall clock, max over ranks"},
            "e2e_host_medium": {"value": e2e_host_val, "unit": UNIT, "h2d_bytes_per_step": h2d_host,
                                "d2h_bytes_per_step": d2h,
                                "what": "the host-built medium from pinned memory (5 arrays; the 6 averaged ones "
                                        "formed on the device), then the same calls"},
            "gpu_launches": args.steps * (3 + 1 + 1),
            "clocks": clk.summary()}
    sim.close()
    if rank == 0 and args.accuracy:
        line["accuracy"] = accuracy_sample(p, args.precision, device)
        if args.precision != "f32":
            torch.cuda.empty_cache()
            line["accuracy_full_grid"] = accuracy_full_grid(p, xi, args.precision, device)
    if rank == 0 and not args.no_cpu_baseline:
        v, n, sc, dt = cpu_reference(p, xi, 1000, 1, os.cpu_count() or 1, budget_s=args.cpu_budget)
        line["cpu_baseline"] = {"value": v, "unit": UNIT, "cores": os.cpu_count() or 1, "kind": "port",
                                "sample": f"oracle f32 on the centre 256x256x{p.nz} column block of the same "
                                          f"medium as {sample_mix(p)}, {n} steps after 1 warm-up ({dt:.1f} s)"}
    ranks.close()
    if rank == 0 and world == 1 and args.workload == "c1" and args.precision == "f32" and not args.no_secondary:
        line["secondary"] = secondary_lines()
    if rank == 0:
        print(json.dumps(line), flush=True)


# the other workloads, measured after the headline in the default run (one GPU): each in its own process with a
# bounded number of steps, the whole set bounded in time; the summary keeps the figures each workload is judged on
SECONDARY = [
    ("c2a", ["--steps", "10", "--warmup", "3"], ("value", "ms_per_step", "batched_over_loop", "plain_loop",
                                                  "batched_over_loop_calls", "roofline", "e2e", "clocks")),
    ("c2b", ["--steps", "10", "--warmup", "3"], ("value", "ms_per_step", "batched_over_loop", "plain_loop",
                                                  "roofline", "e2e", "clocks")),
    ("c3", ["--steps", "1", "--warmup", "3", "--no-cpu-baseline"],
     ("value", "ms_per_step", "forward_ms", "gradient_over_forward", "algorithmic_gradient_over_forward",
      "kept_steps", "roofline", "roofline_forward", "e2e", "clocks")),
    ("c4", ["--steps", "10", "--warmup", "3", "--no-cpu-baseline", "--no-secondary", "--accuracy",
            "--precision", "bf16r"], ("value", "ms_per_step", "storage", "roofline", "accuracy",
                                      "accuracy_full_grid", "clocks")),
    ("c4", ["--steps", "10", "--warmup", "3", "--no-cpu-baseline", "--no-secondary", "--accuracy",
            "--precision", "f16r"], ("value", "ms_per_step", "storage", "roofline", "accuracy",
                                     "accuracy_full_grid", "clocks")),
    ("c4", ["--steps", "10", "--warmup", "3", "--no-cpu-baseline", "--no-secondary", "--accuracy",
            "--precision", "f32"], ("value", "ms_per_step", "storage", "roofline", "accuracy", "clocks")),
]


def secondary_lines(budget_s: float = 420.0) -> dict:
    import subprocess

    out = {}
    t0 = time.perf_counter()
    for wl, extra, keys in SECONDARY:
        name = wl if "--precision" not in extra else f"{wl}_{extra[extra.index('--precision') + 1]}"
        left = budget_s - (time.perf_counter() - t0)
        if left < 30:
            out[name] = {"skipped": "time budget of the secondary workloads spent"}
            continue
        cmd = [sys.executable, str(ROOT / "bench.py"), "--workload", wl] + extra
        try:
            r = subprocess.run(cmd, capture_output=True, text=True, timeout=left, cwd=ROOT)
            rows = [l for l in r.stdout.splitlines() if l.startswith("{")]
            if r.returncode != 0 or not rows:
                out[name] = {"failed": f"exit {r.returncode}: " + (r.stderr.strip().splitlines() or [""])[-1][:300]}
                continue
            full = json.loads(rows[-1])
            out[name] = {"workload": full["config"].get("workload"), "metric": full["metric"],
                         "command": " ".join(["python", "bench.py", "--workload", wl] + extra),
                         **{k: full[k] for k in keys if k in full}}
        except subprocess.TimeoutExpired:
            out[name] = {"skipped": "did not finish within the time budget"}
    return out


if __name__ == "__main__":
    main()
