"""Matched-error evaluation of the learned form against the plain FP64 path.

    python -m rhybrid_b200.evaluate [--scale 0.05] [--json out.json]

A high-ppc (256) run of the Mars-like geometry (scaled) is the judge. Its
state is sampled by the method itself: depositing one in k of its particles
with weights times k gives exactly what a plain run at 256/k ppc would deposit
from that state, so the plain method's moment error at P ppc is the error of
that subsample against the full 256-ppc deposit. The denoiser is trained on
8-ppc pairs from earlier states and judged on a later, held-out state.

Reported: the relative L2 error (rho, J) of the plain deposit at 8, 16, 32,
64, 128 ppc and of the denoised 8-ppc deposit; the step time of the plain
fast path at those ppc and of the learned form at 8 ppc (FP64 fast path and
FP32 form); the plain ppc whose error equals the learned form's (from the fit
e(P) = k sqrt(1/P - 1/256) of the measured errors) with its step time
interpolated in P, and the simulated time per wall second of the learned form
over that of the plain path at that matched error; as a lower bound, the same
ratio against the measured plain point just below the matched ppc.
"""
from __future__ import annotations

import argparse
import dataclasses
import json
import sys
import time

import numpy as np

from . import abi
from . import config as cf
from . import learned


def mars_at(ppc: float, scale: float) -> cf.Config:
    f = scale ** (1.0 / 3.0)
    cfg = cf.config_mars(nx=max(12, int(round(120 * f))), ny=max(12, int(round(160 * f))),
                         nz=max(12, int(round(160 * f))), ppc=ppc)
    # the judge and the low-ppc runs carry the solar-wind protons only
    return cfg.replace(populations=[dataclasses.replace(cfg.populations[0], ppc=ppc)])


def step_time(lib, cfg: cf.Config, steps: int, dn=None, path: int = abi.PATH_FAST) -> float:
    grid, pops = cf.initial_state(cfg)
    ctx = abi.Context(lib, cf.params(cfg), cf.species(cfg), capacity=[int(1.3 * p[1].shape[0]) + 1024 for p in pops])
    try:
        ctx.set_path(path)
        learned.load_state(ctx, cfg, grid, pops)
        if dn is not None:
            ctx.set_denoiser(dn, True)
        ctx.step(2)
        import torch
        st = torch.cuda.ExternalStream(ctx.stream())
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(st)
        ctx.step(steps)
        e1.record(st)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / steps
    finally:
        ctx.close()


def run(scale: float = 0.05, train_steps: int = 8, iters: int = 80, lr: float = 2e-3, timed_steps: int = 5):
    lib = abi.gpu_library()
    judge = mars_at(256.0, scale)
    low_ppc, factor = 8, 32
    dn = learned.new_denoiser(lib, judge, pair_capacity=64)
    t0 = time.time()
    losses, ctx = learned.train_on_run(lib, judge, dn, factor=factor, steps=train_steps, pairs_per_step=8,
                                       iters_per_step=iters, lr=lr)
    train_s = time.time() - t0
    try:
        ctx.step(3)   # a later, held-out state
        errors = {}
        for k in (32, 16, 8, 4, 2):
            dn.add_pair(ctx, k, 1)
            _, newest = dn.num_pairs()
            e = dn.pair_error(newest)
            errors[256 // k] = {"rho": e["raw_rho"], "J": e["raw_J"]}
            if k == factor:
                denoised = {"rho": e["dn_rho"], "J": e["dn_J"]}
    finally:
        ctx.close()
    times = {p: step_time(lib, mars_at(float(p), scale), timed_steps) for p in sorted(errors)}
    t_learned = step_time(lib, mars_at(float(low_ppc), scale), timed_steps, dn=dn)
    t_learned32 = step_time(lib, mars_at(float(low_ppc), scale), timed_steps, dn=dn, path=abi.PATH_FP32)
    dn.close()
    worst = max(denoised.values())
    # the plain error follows e(P) = k sqrt(1/P - 1/256) (sampling noise against the
    # 256-ppc judge): fit k on the measured points, solve e(P) = worst, and
    # interpolate the plain step time linearly in P
    ps = np.array(sorted(errors), float)
    es = np.array([max(errors[int(p)].values()) for p in ps])
    k = float(np.mean(es / np.sqrt(1.0 / ps - 1.0 / 256.0)))
    p_equiv = 1.0 / ((worst / k) ** 2 + 1.0 / 256.0)
    t_equiv = float(np.interp(p_equiv, ps, [times[int(p)] for p in ps]))
    below = [p for p in sorted(errors) if p <= p_equiv]
    p_low = below[-1] if below else None
    out = {
        "geometry": [judge.nx, judge.ny, judge.nz], "judge_ppc": 256, "low_ppc": low_ppc,
        "train": {"pairs": train_steps * 8, "adam_steps": train_steps * iters, "seconds": round(train_s, 1),
                  "losses": [round(x, 6) for x in losses]},
        "plain_error": {str(p): {k: round(v, 4) for k, v in e.items()} for p, e in errors.items()},
        "learned_error": {k: round(v, 4) for k, v in denoised.items()},
        "plain_ms_per_step": {str(p): round(t, 4) for p, t in times.items()},
        "learned_ms_per_step": round(t_learned, 4),
        "learned_fp32_ms_per_step": round(t_learned32, 4),
        "plain_ppc_at_matched_error": round(p_equiv, 1),
        "plain_ms_at_matched_error": round(t_equiv, 4),
        "speedup_at_matched_error": round(t_equiv / t_learned, 2),
        "speedup_at_matched_error_fp32": round(t_equiv / t_learned32, 2),
        "speedup_lower_bound": round(times[p_low] / t_learned, 2) if p_low else None,
        "lower_bound_plain_ppc": p_low,
    }
    return out


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--scale", type=float, default=0.05)
    ap.add_argument("--json", default=None)
    a = ap.parse_args(argv)
    out = run(scale=a.scale)
    print(json.dumps(out))
    if a.json:
        with open(a.json, "w") as f:
            json.dump(out, f, indent=1)


if __name__ == "__main__":
    sys.exit(main())
