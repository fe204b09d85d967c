#!/usr/bin/env python
"""Benchmark of the RHybrid hot path on B200.

Workload (default): the plain FP64 Mars-like obstacle run, 120x160x160 cells of
300 km, absorbing sphere r=3390 km, solar-wind H+ (n=2e6 m^-3, 30 ppc) and He++
(4 %, 1.5 ppc), V=-450 km/s, T=1e5 K, IMF (0,3,0) nT, dt=0.05 s; about 9.7e7
ions. Inputs are synthetic (seeded uniform-in-cell Maxwellian fill, the
reference's InjectorUniform), generated on the host. --workload c3 (the FP32
form's Mars-like run at 256^3 cells, 100 ppc, 1.72e9 ions) and --workload
mercury (320^3 cells, 40 ppc, 1.28e9 ions) are filled on the GPU
(rhgpu_fill_uniform); --form learned runs the learned form's closed-loop
evaluation instead of the plain step.

A step is one propagate(): push + migration + deposit + particle boundary
conditions + field update, for all populations.

  value   particle-steps/s over all GPUs, state resident in HBM (> L2, no flush needed)
  e2e     the same metric through the C ABI with the state in pinned host memory
          each step: upload of all particles, one step, download of the
          particles and of rhoq, Ji, faceB (the round trip of a host that keeps
          ownership of the particle lists, as Corsair/ParGrid does);
          e2e.output_step_host is the host that keeps the state on the device
          and reads back each step's diagnostic sums, with the particles and
          the grid arrays downloaded at the output step closing the sample
  cpu_baseline  the reference's hot-path sources (oracle/_ref) on every host
          core, one process per core on a slab of the workload; one warm-up
          step, then the median of 5 timed steps

--impl reference times the reference's own hot-path sources (oracle/_ref,
compiled from the reference tree) on the host cores, as independent
processes on sub-boxes of the same workload.

Multi-GPU: replicas only (one independent run per GPU, no collective on the
data path); timing is the maximum over ranks.
"""
import argparse
import json
import math
import os
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

PEAKS_FILE = os.path.join(ROOT, "MEASURED_PEAKS.json")
FALLBACK_HBM_GBS = 6650.0


def hbm_peak():
    try:
        with open(PEAKS_FILE) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


def workload(name, scale=1.0):
    from rhybrid_b200 import config as cf
    if name == "mars":
        if scale == 1.0:
            return cf.config_mars(exosphere=True)
        f = scale ** (1.0 / 3.0)
        return cf.config_mars(nx=max(8, int(round(120 * f))), ny=max(8, int(round(160 * f))),
                              nz=max(8, int(round(160 * f))), exosphere=True)
    if name == "empty_box":
        return cf.config_empty_box(32, 32, 32, ppc=20.0)
    f = scale ** (1.0 / 3.0)
    if name == "c3":
        # the FP32 precision form's workload: the Mars-like run at 256^3 cells of
        # 300 km, 100 ppc (H+ 100, He++ 5; about 1.76e9 ions) with its O+ exosphere
        n = max(8, int(round(256 * f)))
        return cf.config_mars(nx=n, ny=n, nz=n, ppc=100.0, exosphere=True)
    if name == "mercury":
        n = max(8, int(round(320 * f)))
        return cf.config_mercury(nx=n, ny=n, nz=n)
    raise ValueError(name)


# workloads too large for host-side particle records: filled on the GPU
GPU_FILL = ("c3", "mercury")


# ---------------------------------------------------------------------------
# clocks during the timed region

class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            p = [x.strip() for x in ln.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                smax = float(p[2])
            except ValueError:
                continue
            for nm, v in zip(names, p[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------------------
# CPU: the reference's own sources (oracle/_ref), one process per core

def _cpu_worker(args):
    """Runs `steps` steps of a sub-box of the workload in the reference build
    (or the oracle port) and returns (particle_steps, seconds)."""
    kind, wl, nz_sub, steps, warm = args
    sys.path.insert(0, ROOT)
    from oracle import oracle
    from rhybrid_b200 import abi
    from rhybrid_b200 import config as cf
    lib = oracle.reference() if kind == "reference" else oracle.port()
    full = workload(wl)
    # a slab through the middle of the box, periodic across its thickness so
    # that its cells do the same work per ion as interior cells of the full run
    cfg = full.replace(nz=nz_sub, z_min=-0.5 * nz_sub * full.dx,
                       periodic=(full.periodic[0], full.periodic[1], 1))
    grid, pops = cf.initial_state(cfg)
    ctx = abi.Context(lib, cf.params(cfg), cf.species(cfg))
    try:
        ctx.upload_array("faceB", grid["faceB"])
        ctx.upload_array("cellB", grid["cellB"])
        ctx.upload_array("nodeEta", grid["nodeEta"])
        ctx.upload_cell_flags(grid["flags"])
        for s, (c, p) in enumerate(pops):
            ctx.upload_particles(s, c, p)
        for _ in range(warm):
            ctx.step(1)
        times, psteps = [], []
        for _ in range(steps):
            n = sum(ctx.num_particles(s) for s in range(len(pops)))
            t0 = time.perf_counter()
            ctx.step(1)
            times.append(time.perf_counter() - t0)
            psteps.append(n)
        return psteps, times
    finally:
        ctx.close()


def cpu_measure(wl, steps, warm, budget_cores=None, nz_sub=None):
    """All host cores, one reference process per core, each on a slab of the
    workload (nz_sub cells thick). Returns per-step aggregate rates."""
    import multiprocessing as mp
    from oracle import oracle
    kind = "reference" if oracle.reference() is not None else "port"
    try:
        cores = len(os.sched_getaffinity(0))
    except Exception:
        cores = os.cpu_count() or 1
    if budget_cores:
        cores = min(cores, budget_cores)
    full = workload(wl)
    if nz_sub is None:
        nz_sub = max(3, min(full.nz, 4))
    ctx = mp.get_context("spawn")
    with ctx.Pool(cores) as pool:
        res = pool.map(_cpu_worker, [(kind, wl, nz_sub, steps, warm)] * cores)
    rates = []
    for st in range(steps):
        tot = sum(r[0][st] for r in res)
        wall = max(r[1][st] for r in res)
        rates.append(tot / wall)
    return {"kind": kind, "cores": cores, "rates": rates, "nz_sub": nz_sub,
            "particles_per_core": res[0][0][0] if res and res[0][0] else 0}


# ---------------------------------------------------------------------------

def algorithmic_bytes(cfg, n_particles):
    """Bytes the plain FP64 step must move (per step): 56 B read + 48 B
    written per particle, and per cell 7 doubles read (faceB, rhoq, Ji) and
    10 written (faceB, cellUe, rhoq, Ji), plus 6 for cellEp with electron
    pressure on."""
    per_cell = 136 + (48 if cfg.use_electron_pressure else 0)
    return 104 * n_particles + per_cell * cfg.ncells


KERNEL_BYTES = {
    # algorithmic bytes per launch of the dominant kernels (units: particles p
    # in one launch, cells c), and whether the kernel is launched per species.
    # exact path
    "push": (lambda p, c: 96 * p + 72 * c, True),
    "mig_scatter": (lambda p, c: 112 * p, True),
    "deposit_cell": (lambda p, c: 56 * p + 32 * c, True),
    "deposit_gather": (lambda p, c: 32 * c, False),
    # fast path: one launch pushes, migrates in-row and deposits every
    # species (56 B read + 48 B written per particle; faceB, cellUe, cellEp
    # read and 4 moment partials per cell written)
    "fast_push_deposit": (lambda p, c: 104 * p + 104 * c, False),
    "fast_gather": (lambda p, c: 32 * c, False),
    # FP32 form: 28 B read + 28 B written per particle (cell, 3 offsets, 3 velocities)
    "f32_push_deposit": (lambda p, c: 56 * p + 104 * c, False),
    "f32_gather": (lambda p, c: 32 * c, False),
}

# DRAM traffic (dram__bytes_read.sum + dram__bytes_write.sum) of one launch
# from an ncu --set full capture at 5 % of the cells (44x59x59, 4.080e6 ions):
#   ncu --set full --clock-control none -k regex:<kernel> -s 3 -c 1 -o prof \
#       python bench.py --scale 0.05 --steps 2 --warmup 3 --no-e2e --no-cpu-baseline [--path fp32]
# The full workload is too large to capture with ~40 replay passes, so the
# traffic of a full launch is this capture's traffic scaled by the units
# processed (its algorithmic bytes), as particle and cell traffic grow in
# proportion with the number of particles and cells.
KERNEL_TRAFFIC = {
    # kernel: (traffic bytes, particles, cells) of the captured launch
    "fast_push_deposit": (263.379712e6 + 216.007168e6, 4110000, 44 * 59 * 59),
    "f32_push_deposit": (144.102912e6 + 89.603840e6, 4110000, 44 * 59 * 59),
}


def scaled_traffic(kernel: str, alg_bytes: float):
    if kernel not in KERNEL_TRAFFIC:
        return None
    t, p, c = KERNEL_TRAFFIC[kernel]
    return t * alg_bytes / KERNEL_BYTES[kernel][0](p, c)


def reduce_over_ranks(dist, seconds: float, work: float, device: str):
    """Whole-job figures of a replica run: the slowest rank's time and the
    total work of all ranks (one collective each; every rank calls it)."""
    if dist is None:
        return seconds, work
    import torch
    tmax = torch.tensor([seconds], dtype=torch.float64, device=device)
    tsum = torch.tensor([work], dtype=torch.float64, device=device)
    dist.all_reduce(tmax, op=dist.ReduceOp.MAX)
    dist.all_reduce(tsum, op=dist.ReduceOp.SUM)
    return float(tmax.item()), float(tsum.item())


def run_gpu(args, rank, world, local_rank):
    import torch
    from rhybrid_b200 import abi
    from rhybrid_b200 import config as cf

    torch.cuda.set_device(local_rank)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    cfg = workload(args.workload, args.scale)
    gpu_fill = args.fill == "gpu" or (args.fill == "auto" and args.workload in GPU_FILL)
    if gpu_fill and args.path == "exact":
        raise SystemExit("the exact path takes host records: --fill host")
    t0 = time.time()
    lib = abi.gpu_library()
    if gpu_fill:
        grid, pops = cf.init_grid(cfg), None
        ctx = abi.Context(lib, cf.params(cfg), cf.species(cfg), device=local_rank)
    else:
        grid, pops = cf.initial_state(cfg)
        nps = [p[1].shape[0] for p in pops]
        ctx = abi.Context(lib, cf.params(cfg), cf.species(cfg), capacity=[n + n // 20 + (1 << 20) for n in nps],
                          device=local_rank)
    ctx.set_path({"fast": abi.PATH_FAST, "exact": abi.PATH_EXACT, "fp32": abi.PATH_FP32}[args.path])
    ctx.upload_array("faceB", grid["faceB"])
    ctx.upload_array("cellB", grid["cellB"])
    ctx.upload_array("nodeEta", grid["nodeEta"])
    ctx.upload_cell_flags(grid["flags"])
    nspec = len(cfg.populations)
    if gpu_fill:
        for s, pop in enumerate(cfg.populations):
            if pop.fill and pop.ppc > 0 and pop.density > 0:
                ctx.fill_uniform(s, pop.density, pop.temperature, pop.velocity, pop.ppc, seed=cfg.seed + 101 * s)
            else:
                ctx.upload_particles(s, np.zeros(cfg.ncells, dtype=np.uint32), np.zeros((0, 7)))
    else:
        for s, (c, p) in enumerate(pops):
            ctx.upload_particles(s, c, p)
    torch.cuda.synchronize()
    gen_s = time.time() - t0
    # the configuration's particle sources (solar wind inflow, O+ exosphere) on
    # the GPU; the exact path (the reference's particle order) takes none
    sources = cf.source_injectors(cfg, seed=cfg.seed) if args.path != "exact" else []
    ctx.set_injectors(sources)
    stream = torch.cuda.ExternalStream(ctx.stream(), device=local_rank)
    for _ in range(args.warmup):
        ctx.step(1)
    n0 = sum(ctx.num_particles(s) for s in range(nspec))
    ctx.set_timing(True)
    clocks = ClockSampler(local_rank)
    clocks.start()
    time.sleep(0.3)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    ctx.step(args.steps)
    ev1.record(stream)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    ms = ev0.elapsed_time(ev1)
    clk = clocks.stop()
    free_b, total_b = torch.cuda.mem_get_info(local_rank)
    mem_used_gb = (total_b - free_b) / 1e9
    launches = ctx.last_launch_count()
    ktimes = ctx.timing()
    ctx.set_timing(False)
    n1 = sum(ctx.num_particles(s) for s in range(nspec))
    psteps = 0.5 * (n0 + n1) * args.steps
    ms_all, psteps_all = reduce_over_ranks(dist, ms, psteps, "cuda")
    value = psteps_all / (ms_all / 1e3)

    # roofline of the dominant kernel class
    peak, peak_kind = hbm_peak()
    top = max(ktimes.items(), key=lambda kv: kv[1]) if ktimes else ("none", 0.0)
    per_species = KERNEL_BYTES.get(top[0], (None, False))[1]
    nlaunch_top = args.steps * (nspec if per_species else 1)
    per_launch_ms = top[1] / max(nlaunch_top, 1)
    roof = None
    if top[0] in KERNEL_BYTES and per_launch_ms > 0:
        # particles of one launch (per-species kernels: the mean over species)
        pcount = 0.5 * (n0 + n1) / (nspec if per_species else 1)
        alg = KERNEL_BYTES[top[0]][0](pcount, cfg.ncells)
        ach = alg / (per_launch_ms / 1e3) / 1e9
        roof = {"kernel": top[0], "bound": "hbm", "achieved": round(ach, 1), "peak": peak, "unit": "GB/s",
                "frac": round(ach / peak, 4), "traffic": None, "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)",
                "ms_per_launch": round(per_launch_ms, 4)}
        tr = scaled_traffic(top[0], alg)
        if tr is not None:
            roof["traffic"] = int(tr)
            roof["algorithmic_bytes"] = int(alg)
            roof["traffic_source"] = ("ncu dram__bytes_read.sum + dram__bytes_write.sum of one launch at 5 % of "
                                      "the cells, scaled by the units processed")
    step_alg = algorithmic_bytes(cfg, 0.5 * (n0 + n1))
    step_ach = step_alg / ((ms / args.steps) / 1e3) / 1e9

    # end to end through the C ABI with host-resident state (rank-local)
    e2e = None
    if not args.no_e2e and not gpu_fill:
        # the FP32 form moves its own 6-float records (rhgpu_*_particles_f32), the
        # FP64 paths 7 doubles per particle
        f32rec = args.path == "fp32"
        rw, rdt, rct = (6, torch.float32, abi.C.c_float) if f32rec else (7, torch.float64, abi.C.c_double)
        cnts, parts, weights = [], [], []
        for s in range(len(pops)):
            if f32rec:
                c, p, w = ctx.download_particles_f32(s)
            else:
                (c, p), w = ctx.download_particles(s), None
            pin = torch.empty((max(p.shape[0], 1), rw), dtype=rdt, pin_memory=True).numpy()[: p.shape[0]]
            pin[:] = p
            cnts.append(c)
            parts.append(pin)
            weights.append(w)
        out_pin = [torch.empty((max(p.shape[0], 1), rw), dtype=rdt, pin_memory=True).numpy() for p in parts]
        ke = max(1, min(8, args.steps))
        h2d = sum(p.nbytes + c.nbytes for p, c in zip(parts, cnts))
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        t1 = time.perf_counter()
        e2e_ps = 0
        for _ in range(ke):
            for s in range(nspec):
                if f32rec:
                    ctx.upload_particles_f32(s, cnts[s], parts[s], weights[s])
                else:
                    ctx.upload_particles(s, cnts[s], parts[s])
                e2e_ps += parts[s].shape[0]
            ctx.step(1)
            d2h = 0
            for s in range(nspec):
                n = ctx.num_particles(s)
                if n > out_pin[s].shape[0]:
                    out_pin[s] = np.empty((n, rw), dtype=parts[s].dtype)
                cnt = np.empty(cfg.ncells, dtype=np.uint32)
                nout = abi.C.c_int64()
                if f32rec:
                    wout = np.zeros(1)
                    lib.call("download_particles_f32", ctx.h, s, abi._ptr(cnt, abi.C.c_uint32),
                             abi._ptr(out_pin[s], rct), out_pin[s].shape[0], abi.C.byref(nout),
                             abi._ptr(wout, abi.C.c_double))
                else:
                    lib.call("download_particles", ctx.h, s, abi._ptr(cnt, abi.C.c_uint32),
                             abi._ptr(out_pin[s], rct), out_pin[s].shape[0], abi.C.byref(nout))
                d2h += nout.value * out_pin[s].itemsize * rw + cnt.nbytes
            for name in ("cellRhoQi", "cellJi", "faceB"):
                d2h += ctx.download_array(name).nbytes
        torch.cuda.synchronize()
        e2e_s = time.perf_counter() - t1
        e2e_s, e2e_ps = reduce_over_ranks(dist, e2e_s, float(e2e_ps), "cuda")
        e2e = {"value": e2e_ps / e2e_s, "unit": "particle-steps/s", "h2d_bytes_per_step": int(h2d),
               "d2h_bytes_per_step": int(d2h), "steps": ke,
               "host": "every step: all particles uploaded from pinned host memory, one step, particles and "
                       "rhoq, Ji, faceB downloaded (a host that owns the particle lists)" +
                       ("; the FP32 form's own 24-byte records (rhgpu_upload/download_particles_f32)" if f32rec
                        else "; 56-byte double records")}
    if not args.no_e2e:
        # a host that keeps the state on the device (Corsair with the GPU plugin):
        # per step it reads back the step's diagnostics (population and field log
        # sums) and nothing else; the particles and the grid come back at the output
        # step that closes the sample
        ko = max(1, args.steps)
        ndiag = 8 * nspec + 30
        diag = torch.empty(ndiag, dtype=torch.float64, pin_memory=True).numpy()
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        t1 = time.perf_counter()
        out_ps = 0
        for _ in range(ko):
            out_ps += sum(ctx.num_particles(s) for s in range(nspec))
            ctx.step(1)
            lib.call("reduce_diagnostics", ctx.h, abi._ptr(diag, abi.C.c_double), ndiag)
        d2h_out = 0
        if not gpu_fill:
            # into pinned buffers, as the per-step round trip above
            for s in range(nspec):
                n = ctx.num_particles(s)
                if n > out_pin[s].shape[0]:
                    out_pin[s] = torch.empty((n, rw), dtype=rdt, pin_memory=True).numpy()
                cnt = np.empty(cfg.ncells, dtype=np.uint32)
                nout = abi.C.c_int64()
                if f32rec:
                    wout = np.zeros(1)
                    lib.call("download_particles_f32", ctx.h, s, abi._ptr(cnt, abi.C.c_uint32),
                             abi._ptr(out_pin[s], rct), out_pin[s].shape[0], abi.C.byref(nout),
                             abi._ptr(wout, abi.C.c_double))
                else:
                    lib.call("download_particles", ctx.h, s, abi._ptr(cnt, abi.C.c_uint32),
                             abi._ptr(out_pin[s], rct), out_pin[s].shape[0], abi.C.byref(nout))
                d2h_out += nout.value * out_pin[s].itemsize * rw + cnt.nbytes
        for name in ("cellRhoQi", "cellJi", "faceB"):
            d2h_out += ctx.download_array(name).nbytes
        torch.cuda.synchronize()
        out_s = time.perf_counter() - t1
        out_s, out_ps = reduce_over_ranks(dist, out_s, float(out_ps), "cuda")
        out = {"value": out_ps / out_s, "unit": "particle-steps/s", "steps": ko,
                                   "h2d_bytes_per_step": 0, "d2h_bytes_per_step": int(diag.nbytes + d2h_out / ko),
                                   "host": f"state resident on the device; each step reads back its {ndiag} "
                                           "diagnostic sums, and " + ("" if gpu_fill else "the particles and ")
                                           + f"rhoq, Ji, faceB come back once at the output step closing the "
                                           f"{ko}-step sample" + (" (the particles, filled on the GPU, stay there: "
                                           "the run's output saves grid arrays only, save_particles = 0 as in "
                                           "the reference's examples)" if gpu_fill else "")}
        if e2e is None:
            e2e = dict(out, note="particles filled on the GPU: no host-owned particle lists for a per-step "
                                 "round trip; this is the device-resident host")
        else:
            e2e["output_step_host"] = out

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline and args.workload == "mars":
        m = cpu_measure(args.workload, steps=5, warm=1)
        cpu = {"value": round(float(np.median(m["rates"])), 1), "unit": "particle-steps/s", "cores": m["cores"],
               "kind": m["kind"],
               "sample": f"{m['cores']} processes, each on a 120x160x{m['nz_sub']} slab of the workload "
                         f"({m['particles_per_core']} ions per process): one warm-up step, then the median of 5 "
                         f"timed steps; reference hot-path sources built with g++ -O2 -ffp-contract=off"}
    ctx.close()
    if rank == 0:
        line = {
            "metric": "particle-steps/s", "value": round(value, 1), "unit": "particle-steps/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms_all / args.steps, 4),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32" if args.path == "fp32" else "f64",
            "data": "synthetic (seeded uniform-in-cell Maxwellian fill, InjectorUniform" +
                    (", generated on the GPU" if gpu_fill else "") + "; sources on the GPU)",
            "config": {"workload": cfg.name, "cells": [cfg.nx, cfg.ny, cfg.nz], "dx_m": cfg.dx, "dt_s": cfg.dt,
                       "ions": int(0.5 * (n0 + n1)), "species": [p.name for p in cfg.populations],
                       "sources": [("exosphere " if j.type == abi.INJECT_EXOSPHERE else "solar wind ")
                                   + cfg.populations[j.species].name for j in sources],
                       "parallelism": f"replicas x{world}", "particle_path": args.path, "l2": "state 10+ GB > 126 MB L2, no flush needed",
                       "device_mem_gb": round(mem_used_gb, 1),
                       "sim_s_per_wall_s": round(args.steps * cfg.dt / (ms_all / 1e3), 4),
                       "step_roofline": {"achieved_gbs": round(step_ach, 1), "alg_bytes_per_step": int(step_alg),
                                         "frac": round(step_ach / peak, 4)},
                       "kernel_ms": {k: round(v / args.steps, 4) for k, v in sorted(ktimes.items(), key=lambda kv: -kv[1])},
                       "init_gen_s": round(gen_s, 1)},
            "roofline": roof, "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": int(launches),
            "clocks": clk,
        }
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


def run_learned(args, rank, world, local_rank):
    """The learned form in closed loop (rhybrid_b200.learned.closed_loop): one
    line with the learned form's simulated seconds per wall second, its error
    against the check run, and its speed-up over the plain FP64 path at matched
    error (measured plain points only). Replicas only: every rank runs it, rank
    0 prints. --workload mercury takes the Mercury-like geometry (at --scale of its
    cells: its 256-ppc check run fits one GPU up to about 0.064), --path fp32 runs
    the learned form on the FP32 precision form, --velocity denoises rho and the
    bulk velocity J / rho in place of rho and J."""
    import torch
    from rhybrid_b200 import abi, learned
    torch.cuda.set_device(local_rank)
    workload = "mercury" if args.workload == "mercury" else "mars"
    low_path = abi.PATH_FP32 if args.path == "fp32" else abi.PATH_FAST
    out = learned.closed_loop(scale=args.scale, workload=workload, low_path=low_path, velocity=args.velocity,
                              keep_radius=args.keep_radius, log=lambda m: print(m, file=sys.stderr, flush=True))
    lr = out["learned"]
    if rank == 0:
        form = "FP32 form" if low_path == abi.PATH_FP32 else "FP64 fast path"
        line = {
            "metric": f"sim-s per wall-s (learned 8 ppc {form} + denoiser; plain FP64 at matched error)",
            "value": round(lr["sim_s_per_wall_s"], 4), "unit": "sim-s/wall-s", "n_gpus": world,
            "steps": out["window"]["last_step"], "warmup": 0, "ms_per_step": round(lr["ms_per_step"], 4),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": ("f32" if low_path == abi.PATH_FP32 else "f64") + " (network bf16, fp32 accum)",
            "data": "synthetic (uniform fill generated on the GPU, solar wind sources)",
            "config": {"workload": f"{workload}_{out['geometry'][0]}x{out['geometry'][1]}x{out['geometry'][2]}_learned",
                       "denoised": out["denoised"], "keep_radius": out["keep_radius"],
                       "check_run": out["check_run"], "training": out["training"], "window": out["window"],
                       "threshold": out["threshold"],
                       "learned": {k: v for k, v in lr.items() if k != "samples"},
                       "plain": [{k: v for k, v in p.items() if k != "samples"} for p in out["plain"]],
                       "matched_error": out["matched_error"], "seconds": out["seconds"]},
            "samples": {"learned": lr["samples"], **{f"plain_{p['ppc']}": p["samples"] for p in out["plain"]}},
        }
        print(json.dumps(line), flush=True)


def run_reference(args, rank, world):
    if rank != 0:
        return
    m = cpu_measure(args.workload, steps=args.steps, warm=args.warmup)
    rates = m["rates"]
    value = float(np.median(rates))
    line = {
        "impl": "reference", "metric": "particle-steps/s", "value": round(value, 1), "unit": "particle-steps/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded uniform-in-cell Maxwellian fill)",
        "config": {"workload": workload(args.workload).name, "sample": f"slabs 120x160x{m['nz_sub']}",
                   "sources": "none: the reference's injectors are not part of its built hot path"},
        "cpu_baseline": {"value": round(value, 1), "unit": "particle-steps/s", "cores": m["cores"], "kind": m["kind"],
                         "sample": f"{m['cores']} processes of the reference hot path, each on a 120x160x{m['nz_sub']} "
                                   f"slab ({m['particles_per_core']} ions), median of {len(rates)} steps"},
        "e2e": {"value": round(value, 1), "unit": "particle-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="gpu", choices=["gpu", "reference"])
    ap.add_argument("--workload", default="mars", choices=["mars", "empty_box", "c3", "mercury"],
                    help="mars: plain FP64 Mars-like run (default); c3: the FP32 form's 256^3 100-ppc Mars-like run; "
                         "mercury: the Mercury-like dipole 320^3 40 ppc")
    ap.add_argument("--form", default="plain", choices=["plain", "learned"],
                    help="plain: the hot path (default); learned: the learned form's closed-loop evaluation at the "
                         "Mars-like geometry (8 ppc + denoiser against a 256-ppc FP64 check run, plain FP64 at "
                         "8-128 ppc)")
    ap.add_argument("--fill", default="auto", choices=["auto", "host", "gpu"],
                    help="initial particles from host records (host) or generated on the GPU (gpu); auto: gpu for "
                         "c3 and mercury")
    ap.add_argument("--scale", type=float, default=1.0, help="fraction of the workload's cells (testing only)")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--velocity", action="store_true",
                    help="--form learned: the denoiser sees rho and J / rho (rhgpu_dn_set_velocity_form)")
    ap.add_argument("--keep-radius", type=float, default=0.0,
                    help="--form learned: moments within this many obstacle radii stay as deposited")
    ap.add_argument("--path", default="fast", choices=["fast", "exact", "fp32"],
                    help="fast: FP64, segment storage and deposit order (default); exact: the reference's order; "
                         "fp32: the FP32 precision form")
    args = ap.parse_args()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank, world)
    elif args.form == "learned":
        run_learned(args, rank, world, local_rank)
    else:
        run_gpu(args, rank, world, local_rank)


if __name__ == "__main__":
    main()
