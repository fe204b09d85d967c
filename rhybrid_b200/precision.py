"""Error of the FP32 precision form against the FP64 path on the same run.

    python -m rhybrid_b200.precision [--workload c3|mercury] [--scale 0.125] [--steps 40] [--json out.json]

Both paths start from the same particles: the uniform fill generated on the
GPU (rhgpu_fill_uniform) draws every particle from a stream keyed by (seed,
cell, index), so the FP64 fast path and the FP32 form hold the same particle
set (positions and velocities rounded to FP32 in the latter), with the same
fields and particle sources. After each of the sampled steps the moments and
fields of both are compared: relative L2 error over the grid,
||a32 - a64|| / ||a64||, of rhoq, Ji, faceB, nodeE and cellUe, and the
relative difference of the total charge. Step times of both are reported.

The full FP32 workloads (1.3e9 - 1.8e9 ions) do not fit one GPU in FP64
(56 bytes per particle and buffer), so the comparison runs the same setup
scaled down in cells (same cell size, ppc and sources).
"""
from __future__ import annotations

import argparse
import json
import sys
import time

import numpy as np

from . import abi
from . import config as cf

ARRAYS = ("cellRhoQi", "cellJi", "faceB", "nodeE", "cellUe")


def workload(name: str, scale: float) -> cf.Config:
    f = scale ** (1.0 / 3.0)
    if name == "c3":
        n = max(12, int(round(256 * f)))
        return cf.config_mars(nx=n, ny=n, nz=n, ppc=100.0, exosphere=True)
    if name == "mercury":
        n = max(12, int(round(320 * f)))
        return cf.config_mercury(nx=n, ny=n, nz=n)
    raise ValueError(name)


def start(lib, cfg: cf.Config, path: int, seed: int):
    grid = cf.init_grid(cfg)
    ctx = abi.Context(lib, cf.params(cfg), cf.species(cfg))
    ctx.set_path(path)
    for k in ("faceB", "cellB", "nodeEta"):
        ctx.upload_array(k, grid[k])
    ctx.upload_cell_flags(grid["flags"])
    for s, pop in enumerate(cfg.populations):
        if pop.fill and pop.ppc > 0 and pop.density > 0:
            ctx.fill_uniform(s, pop.density, pop.temperature, pop.velocity, pop.ppc, seed=seed + 101 * s)
        else:
            ctx.upload_particles(s, np.zeros(cfg.ncells, dtype=np.uint32), np.zeros((0, 7)))
    ctx.set_injectors(cf.source_injectors(cfg, seed=seed))
    return ctx


def rel_l2(a, b) -> float:
    d = float(np.linalg.norm((a - b).ravel()))
    n = float(np.linalg.norm(b.ravel()))
    return d / n if n > 0 else d


def compare(lib, cfg: cf.Config, steps: int, sample_every: int, seed: int) -> dict:
    ctxs = {"fp64": start(lib, cfg, abi.PATH_FAST, seed), "fp32": start(lib, cfg, abi.PATH_FP32, seed)}
    out = {"workload": cfg.name, "cells": [cfg.nx, cfg.ny, cfg.nz], "steps": steps, "samples": [],
           "ms_per_step": {}}
    try:
        n0 = {k: sum(c.num_particles(s) for s in range(len(cfg.populations))) for k, c in ctxs.items()}
        out["ions"] = n0
        done = 0
        times = {k: 0.0 for k in ctxs}
        while done < steps:
            k = min(sample_every, steps - done)
            for name, c in ctxs.items():
                import torch
                torch.cuda.synchronize()
                t0 = time.perf_counter()
                c.step(k)
                torch.cuda.synchronize()
                times[name] += time.perf_counter() - t0
            done += k
            a = {name: {n: c.download_array(n) for n in ARRAYS} for name, c in ctxs.items()}
            row = {"step": done}
            for n in ARRAYS:
                row[n] = rel_l2(a["fp32"][n], a["fp64"][n])
            q = {name: float(a[name]["cellRhoQi"].sum()) for name in a}
            row["total_charge_rel_diff"] = abs(q["fp32"] - q["fp64"]) / abs(q["fp64"])
            out["samples"].append(row)
            print(json.dumps(row), flush=True)
        out["ms_per_step"] = {k: 1e3 * v / steps for k, v in times.items()}
        out["max_error"] = {n: max(r[n] for r in out["samples"]) for n in ARRAYS}
    finally:
        for c in ctxs.values():
            c.close()
    return out


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", default="c3", choices=["c3", "mercury"])
    ap.add_argument("--scale", type=float, default=0.125, help="fraction of the workload's cells")
    ap.add_argument("--steps", type=int, default=40)
    ap.add_argument("--every", type=int, default=10)
    ap.add_argument("--seed", type=int, default=6461674)
    ap.add_argument("--json", default=None)
    args = ap.parse_args(argv)
    lib = abi.gpu_library()
    cfg = workload(args.workload, args.scale)
    out = compare(lib, cfg, args.steps, args.every, args.seed)
    out["command"] = "python -m rhybrid_b200.precision " + " ".join(sys.argv[1:] if argv is None else argv)
    print(json.dumps(out))
    if args.json:
        with open(args.json, "w") as f:
            json.dump(out, f, indent=1)


if __name__ == "__main__":
    main()
