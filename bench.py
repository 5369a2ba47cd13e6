#!/usr/bin/env python
"""Benchmark of the particle-mesh vortex step (M4' P2M -> unbounded FFT Poisson solve
with the 6th-order regularised Green's function and spectral curl -> M4' M2P).

Workload (default ``rings256``): 256^3 cells on [-1,1]^3, free on all axes, two
coaxial vortex rings + 1 % noise, 16.7 M particles (seeded synthetic data).  The
headline is the FP32 form's steps/s with inputs resident in HBM; beside it the FP64
plain path is timed on the same inputs and the FP32 velocities are compared with it.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

N > 1 runs one independent replica per GPU (a single grid does not shard: the path
has no exchange step), launched by torch.distributed.run; the value is the steps of
all ranks divided by the slowest rank's device time.  Rank 0 prints one JSON line.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "256^3 vortex steps/s (FP32 form; FP64 plain path and rel-L2 alongside; batched and served solves/s, p50/p99)"
L2_NOTE = "inputs and intermediates larger than the 126 MB L2 (no flush)"


def env_rank():
    return (int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)),
            int(os.environ.get("LOCAL_RANK", 0)))


# ------------------------------------------------------------------ clocks
class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms during a region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu: int):
        self.gpu = gpu
        self.proc = None
        self.file = None

    def start(self):
        try:
            self.file = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=self.file, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.file.flush()
        rows = []
        with open(self.file.name) as f:
            for line in f:
                parts = [p.strip() for p in line.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
        os.unlink(self.file.name)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower().startswith("active")})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def workload_desc(w):
    """The config.workload string of both arms (same workload, same words)."""
    return (f"{w.name}: {w.n}^3 cells, free-free-free, two coaxial rings + 1% noise, {w.npart} particles, "
            f"order 6 Green's function, eps = 2h, M4'")


# ------------------------------------------------------------------ CPU oracle (baseline / reference arm)
def oracle_setup(w, threads):
    from oracle import oracle as O
    O.set_threads(threads)
    O.set_sample(1.0)
    po = O.make_patch(w.xmin, w.xmax, w.dx, bound_cond=w.bound_cond, nghost=w.nghost)
    ierr, t = O.topology_cuboid(po, w.interp)
    t.npart = w.npart
    par = O.make_params(order=w.order, kernel=1, radius=w.radius, interp=w.interp)
    ierr, pk = O.poisson_setup(po, par)
    assert ierr == 0
    return O, po, t, par, pk


def oracle_step(O, po, t, par, pk, w):
    """One whole oracle step (P2M, solve, M2P) on the full workload; returns
    (seconds, particle velocities)."""
    mesh = np.zeros(O.topo_shape(t))
    t0 = time.perf_counter()
    O.interp_particle_mesh(t, w.interp, w.pos, w.vort, mesh)
    ierr, vel, _ = O.poisson_solve(po, t, par, pk, mesh)
    ierr, up = O.interp_mesh_particle(t, w.interp, vel, w.pos)
    dt = time.perf_counter() - t0
    return dt, up


def run_reference(args):
    """--impl reference: the reference's algorithm on the host cores.  The Fortran/MPI
    reference cannot be built on these machines (no gfortran, MPI or FFTW), so this
    times the C restatement of its plain path (oracle/), with all host threads, over
    whole steps of the full-size workload (no sampling)."""
    rank, world, _ = env_rank()
    if rank != 0:
        return 0
    from pmlib3d_b200 import workloads as Wl
    w = Wl.make(args.config)
    threads = os.cpu_count() or 1
    O, po, t, par, pk = oracle_setup(w, threads)
    for _ in range(args.warmup):
        oracle_step(O, po, t, par, pk, w)
    tot = 0.0
    for _ in range(args.steps):
        tot += oracle_step(O, po, t, par, pk, w)[0]
    value = args.steps / tot
    sample = (f"whole steps: oracle P2M + solve + M2P over all {w.npart} particles of the full {w.n}^3 workload "
              f"({tot / args.steps:.2f} s a step on {threads} threads)")
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "steps/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 / value,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded Philox)",
            "config": {"workload": workload_desc(w), "parallelism": "host threads"},
            "cpu_baseline": {"value": value, "unit": "steps/s", "cores": threads, "kind": "port", "sample": sample},
            "e2e": {"value": value, "unit": "steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


# ------------------------------------------------------------------ batched and served solves
def run_batched(P, Wl, torch, steps, warmup, count=96, rank=0, world=1, fused=True):
    """96 patches of uneven sizes and boundary types (FP32 form), one batch solve per
    step replayed from a CUDA graph; solves/s and the 5-pass model bytes per second.
    fused: each pass family of all patches in one persistent launch (else every patch's
    passes on internal streams).  With several ranks the patches are shared out by
    bytes (each rank solves its part)."""
    from pmlib3d_b200 import shard
    specs_all = Wl.batch_specs(count)
    owner = shard.assign([float(np.prod([c + 8 for c in s["ncell"]])) for s in specs_all], world)
    specs = [s for i, s in enumerate(specs_all) if owner[i] == rank]
    par = P.make_params(order=6, kernel=1, radius=2.0, interp=3)
    patches, topos, vort, nbytes = [], [], [], 0
    for s in specs:
        pa = P.make_patch(s["xmin"], s["xmax"], s["dx"], bound_cond=s["bound_cond"], nghost=4)
        assert P.pmlib_patch_adjust(pa) == 0
        ierr, t = P.pmlib_topology_cuboid(pa, 3)
        patches.append(pa)
        topos.append(t)
        vort.append(Wl.blob_field(t, s["axis"], xp=torch).float().contiguous())
        per = [t.bound_cond[2 * d] != 0 for d in range(3)]
        Pp = [t.ncell[d] if per[d] else t.ncell[d] + t.nghost[2 * d] + t.nghost[2 * d + 1] for d in range(3)]
        M = [Pp[d] if per[d] else 2 * Pp[d] for d in range(3)]
        nbytes += Wl.solve_bytes(M, Pp, 4)
    t0 = time.perf_counter()
    old_mode = P.batch_mode(fused)
    try:
        b = P.Batch(patches, topos, par, P.FP32)
    finally:
        P.batch_mode(old_mode)
    setup_s = time.perf_counter() - t0
    mode = ("persistent launch per pass family (x fwd, y fwd, z, y inv, x inv, ghost fill) over a work list of "
            "(patch, tile) items" if b.fused else "every patch's own passes on 8 internal streams")
    vel = [torch.empty_like(w) for w in vort]
    wp, up = [w.data_ptr() for w in vort], [u.data_ptr() for u in vel]
    st = torch.cuda.Stream()
    with torch.cuda.stream(st):
        for _ in range(max(2, warmup)):
            assert b.solve(wp, up, st.cuda_stream) == 0, P.last_error()
        st.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        for _ in range(steps):
            b.solve(wp, up, st.cuda_stream)
        e1.record(st)
        st.synchronize()
    ms = shard.max_over_ranks(e0.elapsed_time(e1) / steps)
    cells = sum(int(np.prod(s["ncell"])) for s in specs_all)
    b.close()
    return {"workload": f"batched{count}: {count} patches, cells per axis log-uniform in [32,192] before "
                        f"pmlib_patch_adjust, bc from {{fff, ppf, pff}}, Gaussian blob along a random axis, "
                        f"h = 1/64, FP32 form, FP64 Green's set-up",
            "solves_per_s": count / (ms / 1e3), "ms_per_batch": ms, "cells": cells,
            "model_bytes_per_rank": nbytes, "achieved_gbs_per_rank": nbytes / (ms / 1e3) / 1e9,
            "setup_s": setup_s, "graph": "captured CUDA graph", "mode": mode,
            "scaling": "strong: patches shared out over the ranks by bytes" if world > 1 else "single GPU"}


def run_ppf512(P, Wl, torch, steps, warmup, stream, max_over_ranks, barrier):
    """The 512 x 512 x 256 periodic-periodic-free step (67.1 M particles): FP32 form and
    FP64 plain path on the same inputs, inputs resident in HBM, CUDA events on the
    launching stream; FP32 against FP64 on the last step."""
    w = Wl.make("ppf512")
    n = w.npart
    P.fft_tune(True)
    patch = P.make_patch(w.xmin, w.xmax, w.dx, bound_cond=w.bound_cond, nghost=w.nghost)
    ierr, topo = P.pmlib_topology_cuboid(patch, w.interp)
    params = P.make_params(order=w.order, kernel=1, radius=w.radius, interp=w.interp)
    ierr32, plan32 = P.pmlib_poisson_setup(patch, topo, params, P.FP32)
    ierr64, plan64 = P.pmlib_poisson_setup(patch, topo, params, P.FP64)
    P.fft_tune(False)
    assert ierr32 == 0 and ierr64 == 0, P.last_error()
    dev = torch.device("cuda", torch.cuda.current_device())
    pos64 = torch.from_numpy(w.pos).to(dev)
    vort64 = torch.from_numpy(w.vort).to(dev)
    del w.pos, w.vort
    pos32, vort32 = pos64.float().contiguous(), vort64.float().contiguous()
    vel32, vel64 = torch.empty_like(pos32), torch.empty_like(pos64)
    sptr = stream.cuda_stream

    def run(plan, pos, vort, vel, k):
        for i in range(warmup + k):
            if i == warmup:
                torch.cuda.synchronize()
                barrier()
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(stream)
            if P.step_dev(plan, pos.data_ptr(), vort.data_ptr(), n, vel.data_ptr(), sptr) != 0:
                raise RuntimeError(P.last_error())
        e1.record(stream)
        torch.cuda.synchronize()
        return max_over_ranks(e0.elapsed_time(e1)) / k

    ms32 = run(plan32, pos32, vort32, vel32, steps)
    k64 = max(3, steps // 2)
    ms64 = run(plan64, pos64, vort64, vel64, k64)
    d = vel32.double() - vel64
    rel_l2 = float(torch.sqrt((d * d).sum() / (vel64 * vel64).sum()).item())
    max_err = float((d.abs().max() / vel64.abs().max()).item())
    pen = (512, 512, 264)  # transform input extents: periodic axes N, free axis N + 2 nghost
    V = pen[0] * pen[1] * pen[2]
    step_bytes = Wl.solve_bytes((512, 512, 528), pen, 4) + 2 * (24 * n + 12 * V)
    for p in (plan32, plan64):
        p.close()
    return {"value": 1000.0 / ms32, "unit": "steps/s", "ms_per_step": ms32, "steps": steps,
            "fp64_plain": {"value": 1000.0 / ms64, "unit": "steps/s", "ms_per_step": ms64, "steps": k64},
            "fp32_speedup_vs_fp64": ms64 / ms32, "particles_per_s": n * 1000.0 / ms32,
            "accuracy": {"rel_l2_fp32_vs_fp64": rel_l2, "max_rel_err": max_err},
            "model_bytes_per_step_fp32": step_bytes, "achieved_gbs_fp32": step_bytes / (ms32 / 1e3) / 1e9,
            "workload": "ppf512: 512 x 512 x 256 cells, h = 1/256 on [-1,1]^2 x [-0.5,0.5], periodic x, y, free z, "
                        f"two coaxial rings about z (R 0.5, sigma 0.08, z = -+0.15) + 1% noise, {n} particles, "
                        "order 6 Green's function with periodic images, eps = 2h, M4'; FFT 512 x 512 x 528",
            "api": "pmgpu_step_dev (device arrays, P2M + solve + M2P)"}


def run_penal512(P, torch, stream, max_over_ranks, steps=10):
    """The penalised sphere at 512^3 as the penalisation client runs it: an
    impulsively started sphere (no vorticity, uniform inflow U = (1, 0, 0)) for
    `steps` time steps of low-storage RK3 at CFL 0.5 (dt = h/2), FP32 form against the
    FP64 plain path, each through pmgpu_penalisation_stage_dev.  Sphere D = 0.25 at the
    centre of [-1,1]^3 (free), mask chi = (1 - tanh((r - r0) / h)) / 2 (a 2h-wide
    transition) with the Brinkman parameter lambda = 1e4 as the implicit factor
    lambda dt chi / (1 + lambda dt chi); the client's settings otherwise (remeshing
    every step with truncation 1e-3, reprojection and vorticity regularisation,
    penalisation tolerance 0.01 and relaxation 1 on a box with a 5-cell buffer, FD 4,
    Re = 1000).  The drag is the penalisation force along x at the first stage."""
    n, h = 512, 2.0 / 512
    r0, nbuff, lam, U = 0.125, 5, 1.0e4, 1.0
    dt = 0.5 * h / U
    dev = torch.device("cuda", torch.cuda.current_device())
    patch = P.make_patch((-1.0,) * 3, (1.0,) * 3, (h,) * 3, bound_cond=(0, 0, 0), nghost=4)
    ierr, topo = P.pmlib_topology_cuboid(patch, 3)
    params = P.make_params(order=6, kernel=1, radius=2.0, interp=3)
    lo = [round((-r0 + 1.0) / h - nbuff) * h - 1.0 for _ in range(3)]
    hi = [round((r0 + 1.0) / h + nbuff) * h - 1.0 for _ in range(3)]
    bpatch = P.make_patch(lo, hi, (h,) * 3, bound_cond=(0, 0, 0), nghost=4)
    ierr, btopo = P.pmlib_topology_cuboid(bpatch, 3)
    bx = []
    for d in range(3):
        i = torch.arange(1 - btopo.nghost[2 * d], btopo.ncell[d] + btopo.nghost[2 * d + 1] + 1,
                         dtype=torch.float64, device=dev)
        bx.append(btopo.xmin[d] + (i - 0.5) * btopo.dx[d])
    bz, by, bxx = torch.meshgrid(bx[2], bx[1], bx[0], indexing="ij")
    r = torch.sqrt(bxx ** 2 + by ** 2 + bz ** 2)
    chi = 0.5 * (1.0 - torch.tanh((r - r0) / h))
    chi = (lam * dt * chi / (1.0 + lam * dt * chi)).unsqueeze(-1).contiguous()
    del bz, by, bxx, r
    sptr = stream.cuda_stream
    max_part = 16 << 20
    out = {}
    for name, prec, dtype in (("fp32", P.FP32, torch.float32), ("fp64", P.FP64, torch.float64)):
        P.fft_tune(True)
        ierr, plan = P.pmlib_poisson_setup(patch, topo, params, prec)
        ierr2, bplan = P.pmlib_poisson_setup(bpatch, btopo, params, prec)
        P.fft_tune(False)
        assert ierr == 0 and ierr2 == 0, P.last_error()
        solid = chi.to(dtype).contiguous()
        svel = torch.zeros(solid.shape[:3] + (3,), dtype=dtype, device=dev)
        arr = [torch.zeros((max_part, 3), dtype=dtype, device=dev) for _ in range(6)]
        npart, drag, counts, passes = 0, [], [], []
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for step in range(steps):
            for stage in (1, 2, 3):
                a = P.penal_stage_args(time_order=3, itimestage=stage, dtime=dt, fd_order=4, visc=1.0e-3,
                                       reproject=True, regularise_vort=True, first_step=step == 0, remesh=True,
                                       remesh_trunc=1.0e-3, relaxation=1.0, tolerance=0.01, max_iter=1000,
                                       vel_inf=(U, 0.0, 0.0))
                npart, force, it, res = P.penalisation_stage_dev(plan, bplan, solid.data_ptr(), svel.data_ptr(), a,
                                                                 *[t.data_ptr() for t in arr[:4]], npart, max_part,
                                                                 arr[4].data_ptr(), arr[5].data_ptr(), stream=sptr)
                if stage == 1:
                    drag.append(force[0])
                    passes.append(it)
            counts.append(npart)
        e1.record(stream)
        torch.cuda.synchronize()
        ms = max_over_ranks(e0.elapsed_time(e1))
        out[name] = {"ms_per_step": ms / steps, "drag": drag, "particles": counts, "penalisation_passes": passes}
        plan.close()
        bplan.close()
        del arr, solid, svel
        torch.cuda.empty_cache()
    d32, d64 = out["fp32"]["drag"], out["fp64"]["drag"]
    out["drag_max_rel_diff_fp32_vs_fp64"] = max(abs(a - b) / max(abs(b), 1e-300) for a, b in zip(d32, d64))
    out["fp32_speedup_vs_fp64"] = out["fp64"]["ms_per_step"] / out["fp32"]["ms_per_step"]
    out["box_cells"] = list(btopo.ncell)
    out["workload"] = ("penal512: 512^3 cells on [-1,1]^3 (free), impulsively started sphere D = 0.25 at the centre "
                       "in U = (1,0,0), tanh mask (2h transition), lambda = 1e4 at CFL 0.5 (dt = h/2) as the implicit "
                       f"Brinkman factor; {steps} steps of RK3, remesh every step (truncation 1e-3), reprojection, "
                       "regularised vorticity, penalisation tolerance 0.01, FD 4, Re 1000, order 6 kernel, eps = 2h, "
                       "M4'; the particles are those the remeshing keeps (the mesh holds 134 M cells)")
    out["api"] = "pmgpu_penalisation_stage_dev (device arrays; one call per RK stage, particle counts to the host)"
    return out


def run_served(P, torch, rates=(100.0, 300.0, 1000.0), count=60, budget_gb=24.0):
    """Served stream at swept Poisson arrival rates (FP32 form): solves/s, p50/p99."""
    from pmlib3d_b200 import serve as S
    par = P.make_params(order=6, kernel=1, radius=2.0, interp=3)
    # warm-up: one stream of large requests (its own seed) through a server of its own,
    # so that the first measured rate does not pay the first use of kernels and tables
    # or the growth of the device's memory pool
    warm = S.request_stream(48, rate=1000.0, seed=9, nmin=128, nmax=256)
    srv = S.Server(par, precision=P.FP32, slots=8, budget=int(budget_gb * 1e9))
    srv.run(warm)
    srv.close()
    del warm
    torch.cuda.synchronize()
    out = []
    for k, rate in enumerate(rates):
        reqs = S.request_stream(count, rate=rate, seed=10 + k)
        torch.cuda.synchronize()
        srv = S.Server(par, precision=P.FP32, slots=8, budget=int(budget_gb * 1e9))
        rep = srv.run(reqs)
        srv.close()
        rep["rate_per_s"] = rate
        out.append(rep)
        del reqs
        torch.cuda.empty_cache()
    return {"workload": f"served: Poisson arrivals, cells per axis log-uniform 32-256, bc from {{fff, ppf, pff}}, "
                        f"Gaussian blob or ring along a random axis, FP32 form, {count} requests per rate "
                        f"after a warm-up stream of 48 (128-256 cells a side), HBM budget {budget_gb:g} GB, 8 slots, Green's spectra "
                        f"cached per grid",
            "sweep": out}


# ------------------------------------------------------------------ GPU arm
def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default="rings256")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--mode", default="full", choices=["full", "profile"],
                    help="profile: only the FP32 warm-up and timed steps (for ncu captures)")
    ap.add_argument("--precision", default="fp32", choices=["fp32", "fp64"],
                    help="precision of --mode profile")
    ap.add_argument("--no-tune", action="store_true",
                    help="the model's radix schedules instead of the autotuner's (profiling)")
    ap.add_argument("--no-specialised", action="store_true",
                    help="line passes on the run-time register engine only (no compile-time-plan kernels)")
    ap.add_argument("--no-batched", action="store_true", help="skip the batched and served measurements")
    ap.add_argument("--no-stage", action="store_true", help="skip the full vortex-stage measurement")
    ap.add_argument("--no-penal", action="store_true", help="skip the penalisation measurement")
    ap.add_argument("--no-ppf512", action="store_true", help="skip the 512 x 512 x 256 ppf step")
    ap.add_argument("--no-penal512", action="store_true", help="skip the 512^3 penalised sphere")
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference(args)

    import torch
    import torch.distributed as dist
    from pmlib3d_b200 import pmlib as P
    from pmlib3d_b200 import workloads as Wl

    rank, world, local = env_rank()
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))

    def barrier():
        if world > 1:
            dist.barrier()

    def max_over_ranks(x):
        if world == 1:
            return x
        t = torch.tensor([x], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    w = Wl.make(args.config)
    n = w.npart
    P.fft_specialised(not args.no_specialised)
    P.fft_tune(not args.no_tune)  # schedules (radix sequence, kx tile) measured when the plans are made
    patch = P.make_patch(w.xmin, w.xmax, w.dx, bound_cond=w.bound_cond, nghost=w.nghost)
    ierr, topo = P.pmlib_topology_cuboid(patch, w.interp)
    params = P.make_params(order=w.order, kernel=1, radius=w.radius, interp=w.interp)
    ierr32, plan32 = P.pmlib_poisson_setup(patch, topo, params, P.FP32)
    ierr64, plan64 = P.pmlib_poisson_setup(patch, topo, params, P.FP64)
    assert ierr32 == 0 and ierr64 == 0, P.last_error()
    P.fft_tune(False)  # batched and served plans: many short-lived lengths, no tuning

    dev = torch.device("cuda", local)
    pos64 = torch.from_numpy(w.pos).to(dev)
    vort64 = torch.from_numpy(w.vort).to(dev)
    pos32, vort32 = pos64.float().contiguous(), vort64.float().contiguous()
    vel32 = torch.empty_like(pos32)
    vel64 = torch.empty_like(pos64)
    stream = torch.cuda.current_stream()
    sptr = stream.cuda_stream

    def step(plan, pos, vort, vel):
        rc = P.step_dev(plan, pos.data_ptr(), vort.data_ptr(), n, vel.data_ptr(), sptr)
        if rc != 0:
            raise RuntimeError(P.last_error())

    def timed(plan, pos, vort, vel, steps, warmup, sample_clocks=False):
        for _ in range(warmup):
            step(plan, pos, vort, vel)
        torch.cuda.synchronize()
        barrier()
        torch.cuda.synchronize()
        clk = ClockSampler(local) if sample_clocks else None
        if clk:
            clk.start()
        P.launch_count(reset=True)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.nvtx.range_push("timed")  # lets a profiler capture the timed steps only
        e0.record(stream)
        for _ in range(steps):
            step(plan, pos, vort, vel)
        e1.record(stream)
        torch.cuda.nvtx.range_pop()
        torch.cuda.synchronize()
        launches = P.launch_count()
        barrier()
        torch.cuda.synchronize()
        clocks = clk.stop() if clk else None
        ms = e0.elapsed_time(e1)
        return max_over_ranks(ms), launches, clocks

    if args.mode == "profile":
        if args.precision == "fp32":
            ms, launches, _ = timed(plan32, pos32, vort32, vel32, args.steps, args.warmup)
        else:
            ms, launches, _ = timed(plan64, pos64, vort64, vel64, args.steps, args.warmup)
        if rank == 0:
            print(json.dumps({"mode": "profile", "precision": args.precision, "config": args.config,
                              "ms_per_step": ms / args.steps, "gpu_launches": launches}), flush=True)
        for p in (plan32, plan64):
            p.close()
        if world > 1:
            dist.destroy_process_group()
        return 0

    # ---- headline: FP32 form, inputs resident in HBM
    ms32, launches32, clocks = timed(plan32, pos32, vort32, vel32, args.steps, args.warmup, sample_clocks=True)
    value = world * args.steps / (ms32 / 1000.0)
    # ---- FP64 plain path on the same inputs
    k64 = max(3, args.steps // 2)
    ms64, _, _ = timed(plan64, pos64, vort64, vel64, k64, args.warmup)
    value64 = world * k64 / (ms64 / 1000.0)
    # ---- FP32 against FP64 on the last step
    d = (vel32.double() - vel64)
    rel_l2 = float(torch.sqrt((d * d).sum() / (vel64 * vel64).sum()).item())
    max_err = float((d.abs().max() / vel64.abs().max()).item())

    # ---- per-kernel device times (events around every launch) for the roofline
    P.timing_reset()
    P.timing_enable(True)
    nprof = 3
    for _ in range(nprof):
        step(plan32, pos32, vort32, vel32)
    torch.cuda.synchronize()
    P.timing_enable(False)
    kt = P.timing_read()
    mb = Wl.model_bytes(w.n, w.nghost, 4, n)
    kernels = {}
    for k, (kms, cnt) in kt.items():
        if cnt == 0:
            continue
        kernels[k] = {"ms_per_step": kms / nprof, "launches_per_step": cnt / nprof}
        if k in mb:
            # the model's bytes are those of the whole step's work of this kernel class
            # (M2P: the tiled launch and the launch for particles outside every bin)
            kernels[k]["model_bytes_per_step"] = mb[k]
            kernels[k]["achieved_gbs"] = mb[k] / (kms / nprof / 1e3) / 1e9
    modeled = {k: v for k, v in kernels.items() if "model_bytes_per_step" in v}
    dom = max(modeled, key=lambda k: modeled[k]["ms_per_step"])
    peaks = {}
    pk_path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(pk_path):
        peaks = json.load(open(pk_path))
    peak = peaks.get("hbm_gbs")
    peak_src = "measured (MEASURED_PEAKS.json hbm_gbs)" if peak else "fallback 6650 GB/s"
    peak = peak or 6650.0
    traffic = None
    tr_path = os.path.join(ROOT, "profiles", "dram_traffic.json")
    if os.path.exists(tr_path):
        traffic = json.load(open(tr_path)).get(args.config, {}).get(dom)
    achieved = kernels[dom]["achieved_gbs"]
    roofline = {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "peak_source": peak_src, "traffic": traffic,
                "algorithmic_bytes_per_launch": mb[dom] / kernels[dom]["launches_per_step"],
                "launches_per_step": kernels[dom]["launches_per_step"]}

    # ---- end to end through the C ABI with host buffers (H2D + step + D2H per step)
    e2e = None
    if not args.no_e2e:
        # two pinned input sets and two output sets, used in turn by the steps
        hp = [torch.from_numpy(w.pos.astype(np.float32)).pin_memory() for _ in range(2)]
        hv = [torch.from_numpy(w.vort.astype(np.float32)).pin_memory() for _ in range(2)]
        hu = [torch.empty_like(hp[0]).pin_memory() for _ in range(2)]
        pn, vn, un = [t.numpy() for t in hp], [t.numpy() for t in hv], [t.numpy() for t in hu]
        ke = max(4, args.steps)
        lists = ([pn[i % 2] for i in range(ke)], [vn[i % 2] for i in range(ke)], [un[i % 2] for i in range(ke)])
        # single steps: copies and GPU work in sequence
        for _ in range(args.warmup):
            P.step(plan32, pn[0], vn[0], un[0])
        torch.cuda.synchronize()
        barrier()
        t0 = time.perf_counter()
        for i in range(ke):
            if P.step(plan32, pn[i % 2], vn[i % 2], un[i % 2]) != 0:
                raise RuntimeError(P.last_error())
        torch.cuda.synchronize()
        dt1 = max_over_ranks(time.perf_counter() - t0)
        # independent steps in one call: step i+1's inputs and step i-1's velocities
        # cross PCIe while step i runs
        if P.step_many(plan32, *[l[:args.warmup] for l in lists]) != 0:
            raise RuntimeError(P.last_error())
        torch.cuda.synchronize()
        barrier()
        t0 = time.perf_counter()
        if P.step_many(plan32, *lists) != 0:
            raise RuntimeError(P.last_error())
        torch.cuda.synchronize()
        dt = max_over_ranks(time.perf_counter() - t0)
        # the copies alone (same bytes, same pinned buffers, uploads on one stream and
        # the download on another, no step): the PCIe ceiling of the pipelined rate
        dpos, dvort, dvel = (torch.empty_like(pos32) for _ in range(3))
        cu, cd = torch.cuda.Stream(), torch.cuda.Stream()

        def copies_only():
            with torch.cuda.stream(cu):
                dpos.copy_(hp[0], non_blocking=True)
                dvort.copy_(hv[0], non_blocking=True)
            with torch.cuda.stream(cd):
                hu[0].copy_(dvel, non_blocking=True)

        copies_only()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(ke):
            copies_only()
        torch.cuda.synchronize()
        dtc = max_over_ranks(time.perf_counter() - t0)
        del dpos, dvort, dvel
        e2e = {"value": world * ke / dt, "unit": "steps/s", "h2d_bytes_per_step": 24 * n,
               "d2h_bytes_per_step": 12 * n, "steps": ke,
               "api": "pmgpu_step_many (host pointers, pinned; copies of neighbouring steps overlap each step)",
               "single_step": {"value": world * ke / dt1, "unit": "steps/s",
                               "api": "pmgpu_step (one call per step, copies and GPU work in sequence)"},
               "copy_bound": {"value": world * ke / dtc, "unit": "steps/s",
                              "h2d_gbs": 24 * n * ke / dtc / 1e9,
                              "what": "the same H2D and D2H bytes per step with no step, uploads and download "
                                      "on two streams: the rate the pipelined path cannot exceed"}}

    # ---- one full stage of the vortex client's RK3 step (P2M, solve, right-hand side,
    # M2P of velocity and right-hand side, stage update with the particle map)
    stage = None
    if not args.no_stage:
        sp, sv = pos32.clone(), vort32.clone()
        srk, sdrk = torch.zeros_like(sp), torch.zeros_like(sp)
        su, sdw = torch.empty_like(sp), torch.empty_like(sp)
        h = float(w.dx[0])
        dt_stage = 0.05 * h / max(float(vel32.abs().max().item()), 1e-30)  # CFL 0.05 on the last velocity
        live = [n]

        def one_stage(i):
            rc, m = P.vortex_stage_dev(plan32, 3, 1 + i % 3, dt_stage, 4, 1e-4, sp.data_ptr(), sv.data_ptr(),
                                       srk.data_ptr(), sdrk.data_ptr(), live[0], su.data_ptr(), sdw.data_ptr(),
                                       stream=sptr)
            if rc != 0:
                raise RuntimeError(P.last_error())
            live[0] = m

        for i in range(args.warmup):
            one_stage(i)
        torch.cuda.synchronize()
        barrier()
        ks = 3 * max(1, args.steps // 6)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for i in range(ks):
            one_stage(i)
        e1.record(stream)
        torch.cuda.synchronize()
        sms = max_over_ranks(e0.elapsed_time(e1)) / ks
        stage = {"value": world * 1000.0 / sms, "unit": "stages/s", "ms_per_stage": sms, "stages": ks,
                 "particles_after": live[0],
                 "scheme": "low-storage RK3 (stages 1-3 in turn), fd_order 4, visc 1e-4, CFL 0.05",
                 "api": "pmgpu_vortex_stage_dev (device arrays; the map's particle count comes back to the host)"}

    # ---- Brinkman penalisation of a sphere (radius 1/8 at the centre) on a box of the
    # grid with a 5-cell buffer: 10 passes (tolerance 0), then the main solve
    penal = None
    if not args.no_penal:
        h = float(w.dx[0])
        r0, nbuff = 0.125, 5
        lo = [round((-r0 - w.xmin[d]) / h - nbuff) * h + w.xmin[d] for d in range(3)]
        hi = [round((r0 - w.xmin[d]) / h + nbuff) * h + w.xmin[d] for d in range(3)]
        bpatch = P.make_patch(lo, hi, w.dx, bound_cond=(0, 0, 0), nghost=4)
        ierr, btopo = P.pmlib_topology_cuboid(bpatch, w.interp)
        ierr, bplan = P.pmlib_poisson_setup(bpatch, btopo, params, P.FP32)
        assert ierr == 0, P.last_error()
        bx = []
        for d in range(3):
            i = torch.arange(1 - btopo.nghost[2 * d], btopo.ncell[d] + btopo.nghost[2 * d + 1] + 1, dtype=torch.float64,
                             device=dev)
            bx.append(btopo.xmin[d] + (i - 0.5) * btopo.dx[d])
        bz, by, bxx = torch.meshgrid(bx[2], bx[1], bx[0], indexing="ij")
        solid = ((bxx ** 2 + by ** 2 + bz ** 2) <= r0 * r0).float().unsqueeze(-1).contiguous()
        svel = torch.zeros(solid.shape[:3] + (3,), dtype=torch.float32, device=dev)
        pw = Wl.blob_field(topo, 0, xp=torch).float().contiguous()
        pu = torch.empty_like(pw)
        if P.pmlib_poisson_solve_dev(plan32, pw.data_ptr(), pu.data_ptr(), stream=sptr) != 0:
            raise RuntimeError(P.last_error())
        pu[..., 0] += 1.0
        w0, u0 = pw.clone(), pu.clone()

        def penal_once():
            pw.copy_(w0)
            pu.copy_(u0)
            return P.penalisation_solve_dev(plan32, bplan, solid.data_ptr(), svel.data_ptr(), pw.data_ptr(),
                                            pu.data_ptr(), relaxation=1.0, tolerance=0.0, max_iter=10, dtime=0.01,
                                            fd_order=4, vel_inf=(1.0, 0.0, 0.0), stream=sptr)

        penal_once()
        torch.cuda.synchronize()
        kp = 3
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(kp):
            force, npass, res = penal_once()
        e1.record(stream)
        torch.cuda.synchronize()
        pms = max_over_ranks(e0.elapsed_time(e1)) / kp
        penal = {"ms_per_solve": pms, "passes": npass, "force": force, "residuals": list(res),
                 "box_cells": list(btopo.ncell),
                 "workload": f"sphere r = {r0} at the centre, box with a {nbuff}-cell buffer, relaxation 1, "
                             f"FD 4, 10 passes (tolerance 0) + the main {w.n}^3 solve, FP32",
                 "api": "pmgpu_penalisation_solve_dev (the host tests the residual after every pass)"}
        bplan.close()

    # ---- the 512 x 512 x 256 periodic-periodic-free step and the penalised sphere at
    # 512^3, FP32 against FP64 (one GPU only: at N > 1 every rank would build the
    # 67 M-particle inputs on the host at once, and these rows do not scale)
    ppf = penal512 = None
    if not args.no_ppf512 and world == 1:
        ppf = run_ppf512(P, Wl, torch, max(4, args.steps // 2), args.warmup, stream, max_over_ranks, barrier)
        torch.cuda.empty_cache()
    if not args.no_penal512 and world == 1:
        penal512 = run_penal512(P, torch, stream, max_over_ranks)

    # ---- batched uneven patches (every rank: replicas) and the served stream (rank 0)
    batched = served = None
    if not args.no_batched:
        batched = run_batched(P, Wl, torch, max(3, args.steps // 2), args.warmup, rank=rank, world=world)
        streams = run_batched(P, Wl, torch, max(3, args.steps // 2), args.warmup, rank=rank, world=world,
                              fused=False)
        batched["per_patch_streams"] = {k: streams[k] for k in ("solves_per_s", "ms_per_batch", "mode")}
        if rank == 0:
            served = run_served(P, torch)
        barrier()

    # ---- CPU baseline: the oracle on this box's host cores (rank 0, one GPU only), one
    # whole step on the same inputs; its velocities pin the FP64 and FP32 GPU steps
    cpu = oracle_acc = None
    if not args.no_cpu_baseline and world == 1 and rank == 0:
        threads = os.cpu_count() or 1
        O, po, t, par, pk = oracle_setup(w, threads)
        dt, up = oracle_step(O, po, t, par, pk, w)
        cpu = {"value": 1.0 / dt, "unit": "steps/s", "cores": threads, "kind": "port",
               "sample": f"one whole step: oracle (C restatement of the reference's plain FP64 path) P2M + solve + "
                         f"M2P over all {n} particles of the full workload, {dt:.2f} s"}
        ref = torch.from_numpy(up).to(dev)
        oracle_acc = {}
        for name, v in (("fp64", vel64), ("fp32", vel32)):
            d = v.double() - ref
            oracle_acc[f"rel_l2_{name}_vs_oracle"] = float(torch.sqrt((d * d).sum() / (ref * ref).sum()).item())
            oracle_acc[f"max_rel_err_{name}_vs_oracle"] = float((d.abs().max() / ref.abs().max()).item())
        del ref, d

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "steps/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms32 / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded Philox)",
            "config": {"workload": workload_desc(w),
                       "grid": f"N={w.n}, nghost={w.nghost}, FFT M={2 * (w.n + 2 * w.nghost)}",
                       "parallelism": f"replicas x{world}", "l2": L2_NOTE},
            "fft_schedules": [e for e in P.fft_tuned() if e["length"] in (2 * (w.n + 2 * w.nghost),)],
            "fp64_plain": {"value": value64, "unit": "steps/s", "ms_per_step": ms64 / k64},
            "particles_per_s": value * n, "fp32_speedup_vs_fp64": value / value64,
            "accuracy": {"rel_l2_fp32_vs_fp64": rel_l2, "max_rel_err": max_err, **(oracle_acc or {})},
            "roofline": roofline, "kernels": kernels, "gpu_launches": launches32,
            "clocks": clocks, "e2e": e2e, "cpu_baseline": cpu, "batched": batched, "served": served,
            "vortex_stage": stage, "penalisation": penal, "ppf512": ppf,
            "penal512": penal512,
        }
        print(json.dumps(line), flush=True)
    for p in (plan32, plan64):
        p.close()
    if world > 1:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
