"""Matched-error evaluation of the learned form against the plain FP64 path.

    python -m rhybrid_b200.evaluate [--scale 0.05] [--judge-ppc 256] [--json out.json]

A high-ppc run (J ppc) of the Mars-like geometry (scaled) is the judge. Its
state is sampled by the method itself: depositing one in k of its particles
with weights times k gives exactly what a plain run at J/k ppc would deposit
from that state, so the plain method's moment error at P ppc is the error of
that subsample against the full J-ppc deposit. The denoiser is trained on
8-ppc pairs (factor J/8) from earlier states and judged on a later, held-out
state.

Reported: the relative L2 error (rho, J) of the plain deposit at 8 .. J/2 ppc
and of the denoised 8-ppc deposit; the step time of the plain fast path at
those ppc and of the learned form at 8 ppc (FP64 fast path and FP32 form).

Matched error against the judge (conservative): the plain ppc whose error
equals the learned form's, from the fit e(P) = k sqrt(1/P - 1/J) of the
measured errors, its step time interpolated in P, and the simulated time per
wall second of the learned form over that of the plain path there; as a lower
bound, the same ratio against the measured plain point just below.

Matched error against the truth (estimate): the judge has its own sampling
error k / sqrt(J); a plain subsample's error is nested in it (hence the fit),
while the denoised output's error against the judge is about
sqrt(e_D^2 + k^2 / J) with e_D its error against the truth. So e_D =
sqrt(e^2 - k^2 / J), the plain ppc with the same error against the truth is
(k / e_D)^2, and its step time is interpolated (or extrapolated linearly
beyond the largest measured ppc). The estimate assumes the denoised output's
error independent of the judge's; the larger J, the smaller the correction.
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


def run(scale: float = 0.05, train_steps: int = 8, iters: int = 160, lr: float = 2e-3, timed_steps: int = 5,
        judge_ppc: int = 256):
    lib = abi.gpu_library()
    judge = mars_at(float(judge_ppc), scale)
    low_ppc = 8
    factor = judge_ppc // low_ppc
    dn = learned.new_denoiser(lib, judge, pair_capacity=64)
    t0 = time.time()
    losses, ctx = learned.train_on_run(lib, judge, dn, factor=factor, steps=train_steps, pairs_per_step=8,
                                       iters_per_step=iters, lr=lr)
    train_s = time.time() - t0
    try:
        ctx.step(3)   # a later, held-out state
        errors = {}
        k = factor
        while k >= 2:
            dn.add_pair(ctx, k, 1)
            _, newest = dn.num_pairs()
            e = dn.pair_error(newest)
            errors[judge_ppc // k] = {"rho": e["raw_rho"], "J": e["raw_J"]}
            if k == factor:
                denoised = {"rho": e["dn_rho"], "J": e["dn_J"]}
            k //= 2
    finally:
        ctx.close()
    times = {p: step_time(lib, mars_at(float(p), scale), timed_steps) for p in sorted(errors)}
    t_learned = step_time(lib, mars_at(float(low_ppc), scale), timed_steps, dn=dn)
    t_learned32 = step_time(lib, mars_at(float(low_ppc), scale), timed_steps, dn=dn, path=abi.PATH_FP32)
    dn.close()
    worst = max(denoised.values())
    # the plain error follows e(P) = k sqrt(1/P - 1/J) (sampling noise against the
    # J-ppc judge): fit k on the measured points, solve e(P) = worst, and
    # interpolate the plain step time linearly in P
    J = float(judge_ppc)
    ps = np.array(sorted(errors), float)
    es = np.array([max(errors[int(p)].values()) for p in ps])
    k = float(np.mean(es / np.sqrt(1.0 / ps - 1.0 / J)))
    p_equiv = 1.0 / ((worst / k) ** 2 + 1.0 / J)
    tp = [times[int(p)] for p in ps]
    t_equiv = float(np.interp(p_equiv, ps, tp))
    below = [p for p in sorted(errors) if p <= p_equiv]
    p_low = below[-1] if below else None
    # against the truth: remove the judge's own sampling error from the denoised error
    e_judge = k / np.sqrt(J)
    e_dn_truth = float(np.sqrt(max(worst ** 2 - e_judge ** 2, 1e-30)))
    p_truth = (k / e_dn_truth) ** 2
    if p_truth <= ps[-1]:
        t_truth = float(np.interp(p_truth, ps, tp))
    else:   # linear in P beyond the largest measured ppc, from the last two points
        slope = (tp[-1] - tp[-2]) / (ps[-1] - ps[-2])
        t_truth = float(tp[-1] + slope * (p_truth - ps[-1]))
    out = {
        "geometry": [judge.nx, judge.ny, judge.nz], "judge_ppc": judge_ppc, "low_ppc": low_ppc,
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
        "vs_truth": {
            "judge_error": round(float(e_judge), 4),
            "learned_error": round(e_dn_truth, 4),
            "plain_ppc_at_matched_error": round(float(p_truth), 1),
            "plain_ms_at_matched_error": round(t_truth, 4),
            "extrapolated": bool(p_truth > ps[-1]),
            "speedup_at_matched_error": round(t_truth / t_learned, 2),
            "speedup_at_matched_error_fp32": round(t_truth / t_learned32, 2),
        },
    }
    return out


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--scale", type=float, default=0.05)
    ap.add_argument("--judge-ppc", type=int, default=256)
    ap.add_argument("--iters", type=int, default=160, help="Adam steps per training step")
    ap.add_argument("--json", default=None)
    a = ap.parse_args(argv)
    out = run(scale=a.scale, judge_ppc=a.judge_ppc, iters=a.iters)
    print(json.dumps(out))
    if a.json:
        with open(a.json, "w") as f:
            json.dump(out, f, indent=1)


if __name__ == "__main__":
    sys.exit(main())
