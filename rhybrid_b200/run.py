"""Run a simulation from a RHybrid .cfg file on the GPU, as Corsair's time
loop drives the reference (src/user.cpp:49-158): particle sources every step,
the population and field logs every log_interval steps (before the step, with
the max-B stop), and at every data save step the variables of
Hybrid.output_parameters (the arrays the reference's output operator hands to
its VLSV writer, output.cell_variables) and, with Hybrid.save_particles, the
particle points (output.particle_points), written as the reference's VLSV
state file (state_<timestep>.vlsv, rhybrid_b200.vlsv); with
Hybrid.save_reduced_state_interval, the reduced state every that many steps
(reduced<timestep>.vlsv: cellB of every Nstride-th cell, optionally those
cells' particles).

    python -m rhybrid_b200.run mars.cfg --steps 1000 --out run1

The state is device-resident: particles cross PCIe only when uploaded at the
start.
"""
import argparse
import os
import sys
from typing import Optional

import numpy as np

from . import abi
from . import cfg as C
from . import config as cf
from . import output as O
from . import vlsv as V


def run(cfg_path: str, steps: Optional[int] = None, out_dir: str = ".", path: str = "fast", device: int = 0,
        lib: Optional[abi.Library] = None, quiet: bool = False) -> dict:
    """Runs `steps` time steps (the file's maximum_timesteps by default).
    Returns {"steps": steps run, "stopped": max-B stop, "saved": [state files],
    "reduced": [reduced state files]}."""
    config, rs = C.load(cfg_path)
    os.makedirs(out_dir, exist_ok=True)
    nsteps = rs.maximum_timesteps if steps is None else steps
    lib = lib or abi.gpu_library()
    grid, pops = cf.initial_state(config)
    sources = cf.source_injectors(config, seed=config.seed)
    if sources and not lib.has("set_injectors"):
        raise RuntimeError(f"{lib.path}: this library has no particle sources")
    cap = [p[1].shape[0] + p[1].shape[0] // 4 + (1 << 16) for p in pops]
    ctx = abi.Context(lib, cf.params(config), cf.species(config), capacity=cap, device=device)
    saved, reduced, stopped, done = [], [], False, 0
    try:
        if lib.has("set_path"):
            ctx.set_path({"fast": abi.PATH_FAST, "fp32": abi.PATH_FP32, "exact": abi.PATH_EXACT}[path])
        ctx.upload_array("faceB", grid["faceB"])
        ctx.upload_array("cellB", grid["cellB"])
        ctx.upload_array("nodeEta", grid["nodeEta"])
        ctx.upload_cell_flags(grid["flags"])
        for s, (cnt, p) in enumerate(pops):
            ctx.upload_particles(s, cnt, p)
        if sources:
            ctx.set_injectors(sources)
        # the population averages run on the fast and exact paths (the FP32 form has none)
        averages = (any(g >= 0 for g in rs.output_groups) and lib.has("set_population_averages")
                    and not (path == "fp32" and lib.has("set_path")))
        if averages:
            ctx.set_population_averages(rs.output_groups)
        logging = rs.log_interval > 0 and lib.has("log_open")
        if logging:
            ctx.log_open(out_dir, rs.species_names, precision=rs.log_precision,
                         include_inner_cells=rs.include_inner_cells_in_field_log,
                         max_B_stop_run=rs.max_magnetic_field_stop_run)
        for _ in range(nsteps):
            ts = ctx.time()[1]
            if logging and ts % rs.log_interval == 0:
                main = rs.main_log_diagnostics_interval > 0 and ts % rs.main_log_diagnostics_interval == 0
                stopped, msg = ctx.log_write(main_log_diagnostics=main)
                if msg and not quiet:
                    sys.stdout.write(msg)
                if stopped:
                    break
            # inside the window of Hybrid.data_save_all_timesteps_t_*, a state at
            # every step (user.cpp:66-71, decided on the time before the step)
            interval = rs.data_save_interval
            t0 = ctx.time()[0]
            if rs.data_save_all_timesteps_t_start >= 0 and \
                    rs.data_save_all_timesteps_t_start <= t0 <= rs.data_save_all_timesteps_t_end:
                interval = 1
            ctx.step(1)
            done += 1
            ts = ctx.time()[1]
            # the reduced state, written at the end of propagate() (user.cpp:150-155)
            if rs.save_reduced_state_interval > 0 and ts % rs.save_reduced_state_interval == 0:
                red = O.reduced_state(ctx, rs.species_names, rs.save_reduced_state_nstride,
                                      rs.save_reduced_state_particles)
                fn = os.path.join(out_dir, f"reduced{ts:08d}.vlsv")
                V.write_reduced_state(fn, ctx.time()[0], ts, rs.save_reduced_state_nstride, red, rs.species_names)
                reduced.append(fn)
            if interval > 0 and ts % interval == 0:
                out = O.cell_variables(ctx, rs.output_parameters, rs.output_groups, rs.output_group_names)
                parts = O.particle_points(ctx, rs.species_names, rs.save_particles_nstride) if rs.save_particles else None
                fn = os.path.join(out_dir, f"state_{ts:07d}.vlsv")
                V.write_state(fn, V.grid_of(ctx), ctx.time()[0], ts, out, parts)
                saved.append(fn)
        if logging:
            ctx.log_close()
    finally:
        ctx.close()
    return {"steps": done, "stopped": stopped, "saved": saved, "reduced": reduced}


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("cfg")
    ap.add_argument("--steps", type=int, default=None, help="time steps (default: the file's maximum_timesteps)")
    ap.add_argument("--out", default=".", help="directory of the log files and saved states")
    ap.add_argument("--path", default="fast", choices=["fast", "fp32", "exact"])
    ap.add_argument("--device", type=int, default=0)
    a = ap.parse_args(argv)
    r = run(a.cfg, a.steps, a.out, a.path, a.device)
    print(f"{r['steps']} steps{' (stopped: max |B|)' if r['stopped'] else ''}, {len(r['saved'])} states saved")


if __name__ == "__main__":
    main()
