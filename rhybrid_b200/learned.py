"""The learned form: a low particles-per-cell run whose deposited moments pass
through the learned denoiser (rhgpu_dn, BF16 tensor-core network) before the
field update, trained on pairs the method itself generates, and judged
against a high-ppc plain run.

Training pairs (train_on_run): a high-ppc fast-path context is stepped; after
each step, rhgpu_dn_add_pair deposits one in `factor` of its particles with
the weights multiplied by `factor` (a low-ppc sample of the same state) and
stores it next to the deposit of all its particles. Adam steps on random stored
pairs follow (rhgpu_dn_train).

The gate (LearnedForm.judge): at each output step the denoised moments of the
low-ppc run are compared with those of the high-ppc check run; when the
relative L2 error of rho or J exceeds the threshold (2 % by default), the
denoiser is switched off and the run continues with the plain deposit.

The network can denoise rho and J, or rho and the bulk velocity J / rho (the
velocity form, velocity_scales; J is handed back as rho' u'), and can leave
the cells near the planet as deposited (keep_mask). closed_loop measures the
whole scheme against plain runs at matched error.
"""
from __future__ import annotations

import time

import numpy as np

from . import abi
from . import config as cf

C, TAPS = 16, 27
LAYER = TAPS * C * C + C


def init_params(seed: int = 0) -> np.ndarray:
    """Signed pass-through start: layer 0 maps each input channel c to
    lrelu(x_c) and lrelu(-x_c) (channels c and c+4) at the centre tap, layer 1
    carries channels 0-7 through unchanged, channels 8-15 of both are
    He-normal random features, and the last layer is zero, so the untrained
    network is the identity (residual) and any linear filter of the input is
    one layer of training away."""
    rng = np.random.default_rng(seed)
    p = np.zeros(abi.DN_PARAMS, dtype=np.float32)
    W0 = p[0:TAPS * C * C].reshape(TAPS, C, C)
    W1 = p[LAYER:LAYER + TAPS * C * C].reshape(TAPS, C, C)
    for c in range(4):
        W0[13, c, c] = 1.0
        W0[13, c, c + 4] = -1.0
    W0[:, :4, 8:] = rng.normal(0.0, np.sqrt(2.0 / (TAPS * 4)), (TAPS, 4, 8))
    for c in range(8):
        W1[13, c, c] = 1.0
    W1[:, :, 8:] = rng.normal(0.0, np.sqrt(2.0 / (TAPS * C)), (TAPS, C, 8))
    return p


def moment_scales(cfg: cf.Config):
    """Normalization of the network input: the upstream charge density and
    that density times the upstream speed."""
    rho = sum(p.q * p.density for p in cfg.populations if p.upstream) or 1.0
    speed = max((float(np.linalg.norm(p.velocity)) for p in cfg.populations if p.upstream), default=1.0) or 1.0
    return abs(rho), abs(rho) * speed


def velocity_scales(cfg: cf.Config):
    """Normalization of the velocity form: the upstream charge density and the
    upstream speed."""
    rho, j = moment_scales(cfg)
    return rho, j / rho


def keep_mask(cfg: cf.Config, radius: float) -> np.ndarray:
    """Cells whose centre lies within `radius` field-obstacle radii of the
    origin (the planet's centre): the denoiser leaves their moments as
    deposited (rhgpu_dn_set_keep_mask)."""
    k, j, i = np.meshgrid(np.arange(cfg.nz), np.arange(cfg.ny), np.arange(cfg.nx), indexing="ij")
    x = cfg.x_min + (i + 0.5) * cfg.dx
    y = cfg.y_min + (j + 0.5) * cfg.dx
    z = cfg.z_min + (k + 0.5) * cfg.dx
    R = radius * max(cfg.R_fieldObstacle, 0.0)
    return ((x * x + y * y + z * z) < R * R).astype(np.uint8).reshape(-1)


def relative_l2(a: np.ndarray, b: np.ndarray) -> float:
    a, b = np.asarray(a, float).reshape(-1), np.asarray(b, float).reshape(-1)
    d = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / d) if d > 0 else float(np.linalg.norm(a - b))


def load_state(ctx: abi.Context, cfg: cf.Config, grid, pops):
    ctx.upload_array("faceB", grid["faceB"])
    ctx.upload_array("cellB", grid["cellB"])
    ctx.upload_array("nodeEta", grid["nodeEta"])
    ctx.upload_cell_flags(grid["flags"])
    for s, (cnt, p) in enumerate(pops):
        ctx.upload_particles(s, cnt, p)


def new_denoiser(lib: abi.Library, cfg: cf.Config, pair_capacity: int = 64, seed: int = 0) -> abi.Denoiser:
    dn = abi.Denoiser(lib, cfg.nx, cfg.ny, cfg.nz, cfg.periodic, pair_capacity=pair_capacity)
    dn.set_scales(*moment_scales(cfg))
    dn.set_params(init_params(seed))
    return dn


def train_on_run(lib: abi.Library, cfg_high: cf.Config, dn: abi.Denoiser, factor: int, steps: int,
                 pairs_per_step: int, iters_per_step: int, lr: float = 1e-3, grid=None, pops=None):
    """Steps a high-ppc fast-path run; after each step stores `pairs_per_step`
    (low-ppc subsample, full) pairs and trains. Returns the mean losses and the
    context (still open, for held-out pairs)."""
    if grid is None:
        grid, pops = cf.initial_state(cfg_high)
    ctx = abi.Context(lib, cf.params(cfg_high), cf.species(cfg_high),
                      capacity=[int(1.3 * p[1].shape[0]) + 1024 for p in pops])
    ctx.set_path(abi.PATH_FAST)
    load_state(ctx, cfg_high, grid, pops)
    losses = []
    for st in range(steps):
        ctx.step(1)
        for k in range(pairs_per_step):
            dn.add_pair(ctx, factor, (st * pairs_per_step + k) % factor)
        losses.append(dn.train(iters_per_step, lr))
    return losses, ctx


class LearnedForm:
    """A low-ppc run with the denoiser applied before the field update, and a
    high-ppc plain check run advanced in lockstep that judges it."""

    def __init__(self, lib: abi.Library, cfg_low: cf.Config, cfg_check: cf.Config, dn: abi.Denoiser,
                 threshold: float = 0.02):
        self.threshold = threshold
        self.dn = dn
        self.enabled = True
        self.history = []
        gl, pl = cf.initial_state(cfg_low)
        gc, pc = cf.initial_state(cfg_check)
        self.low = abi.Context(lib, cf.params(cfg_low), cf.species(cfg_low),
                               capacity=[int(1.3 * p[1].shape[0]) + 1024 for p in pl])
        self.check = abi.Context(lib, cf.params(cfg_check), cf.species(cfg_check),
                                 capacity=[int(1.3 * p[1].shape[0]) + 1024 for p in pc])
        for ctx, cfg, g, p in ((self.low, cfg_low, gl, pl), (self.check, cfg_check, gc, pc)):
            ctx.set_path(abi.PATH_FAST)
            load_state(ctx, cfg, g, p)
        self.low.set_denoiser(dn, True)

    def step(self, n: int = 1):
        self.low.step(n)
        self.check.step(n)

    def judge(self):
        """Relative L2 error of the low-ppc run's moments against the check run;
        switches the denoiser off when either exceeds the threshold."""
        e_rho = relative_l2(self.low.download_array("cellRhoQi"), self.check.download_array("cellRhoQi"))
        e_j = relative_l2(self.low.download_array("cellJi"), self.check.download_array("cellJi"))
        if self.enabled and max(e_rho, e_j) > self.threshold:
            self.low.set_denoiser(self.dn, False)
            self.enabled = False
        self.history.append((e_rho, e_j, self.enabled))
        return e_rho, e_j, self.enabled

    def close(self):
        self.low.close()
        self.check.close()


# ---------------------------------------------------------------------------
# closed-loop evaluation at the full Mars-like geometry

def c4_config(ppc: float, scale: float = 1.0) -> cf.Config:
    """The learned form's workload: the Mars-like geometry (120x160x160 cells of
    300 km, absorbing sphere, closed walls with the IMF on the +x wall) with its
    solar wind H+ at `ppc` and He++ at ppc/20 and their inflow sources."""
    f = scale ** (1.0 / 3.0)
    return cf.config_mars(nx=max(16, int(round(120 * f))), ny=max(16, int(round(160 * f))),
                          nz=max(16, int(round(160 * f))), ppc=ppc)


def c5_config(ppc: float, scale: float = 1.0) -> cf.Config:
    """The Mercury-like dipole geometry (320^3 cells of 100 km at scale 1) with
    its solar wind H+ at `ppc` and its inflow source; `scale` is the fraction
    of the cells, at the same cell size."""
    n = max(16, int(round(320 * scale ** (1.0 / 3.0))))
    return cf.config_mercury(nx=n, ny=n, nz=n, ppc=ppc)


GEOMETRIES = {"mars": c4_config, "mercury": c5_config}


def filled_context(lib: abi.Library, cfg: cf.Config, seed: int, path: int = abi.PATH_FAST) -> abi.Context:
    """A context of cfg with its populations filled on the GPU and its sources set."""
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


def _timed_steps(ctx: abi.Context, n: int) -> float:
    import torch
    st = torch.cuda.ExternalStream(ctx.stream())
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(st)
    ctx.step(n)
    e1.record(st)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1)


def closed_loop(scale: float = 1.0, judge_ppc: int = 256, low_ppc: int = 8, plain_ppcs=(8, 16, 32, 64, 128),
                train_steps: int = 100, crops_per_step: int = 20, crop: int = 64, adam_steps: int = 4000,
                lr: float = 1e-3, eval_steps: int = 100, every: int = 10, threshold: float = 0.02,
                enforce_gate: bool = False, seed: int = 6461674, workload: str = "mars",
                low_path: int = abi.PATH_FAST, rho_only: bool = False, velocity: bool = False,
                keep_radius: float = 0.0, log=print) -> dict:
    """The learned form in closed loop against a high-ppc plain check run.

    workload: "mars" (c4_config) or "mercury" (c5_config), at `scale` of the
    cells. low_path: the particle path of the learned run (PATH_FAST, FP64, or
    PATH_FP32, the FP32 precision form); the check run and the plain runs are
    always the FP64 fast path. rho_only: after training, the last layer's
    current outputs are zeroed, so the learned run denoises the charge density
    and keeps its deposited current. velocity: the network denoises rho and
    the bulk velocity J / rho (rhgpu_dn_set_velocity_form) instead of rho and J.
    keep_radius: in the learned run, the moments of cells within that many
    field-obstacle radii of the planet's centre stay as deposited (keep_mask).

    1. Check run (judge_ppc, FP64 fast path, filled on the GPU) steps
       train_steps + eval_steps. During the first train_steps it yields the
       training pairs: after each step, crops_per_step random crop^3 crops of
       (one in judge_ppc/low_ppc of its particles, weights scaled; all of
       them) (rhgpu_dn_add_crops). During the last eval_steps its moments are
       stored at every `every` steps, together with its own sampling error
       (split-half: half of its particles against all, rhgpu_dn_add_pair with
       factor 2).
    2. The network is trained on the crop pairs (Adam, adam_steps), with the
       3-voxel crop border left out of the loss.
    3. Each low-ppc run starts from its own fill of the same initial state and
       steps train_steps + eval_steps with the same sources: the learned form
       (low_ppc, the denoiser between deposit and field update, the gate on)
       and the plain FP64 path at each of plain_ppcs. At every stored step its
       rho and J are compared with the check run's (relative L2 over the
       grid). The gate compares the error against the truth estimate,
       sqrt(e^2 - e_check^2), with `threshold` (against the raw error a check
       run of J ppc fails every run once its own sampling error k/sqrt(J)
       approaches the threshold). With enforce_gate it switches the denoiser
       off as LearnedForm does; otherwise (the evaluation) the denoiser stays
       on and the first step where the gate would have switched it off is
       recorded.
    4. Simulated seconds per wall second of each run over the evaluation
       window (CUDA events, state resident), and the speed-up of the learned
       form over the measured plain run with the smallest ppc whose error is
       at most the learned form's (no interpolation).
    """
    lib = abi.gpu_library()
    t_start = time.time()
    geom = GEOMETRIES[workload]
    judge_cfg = geom(float(judge_ppc), scale)
    factor = judge_ppc // low_ppc
    dn = abi.Denoiser(lib, crop, crop, crop, (0, 0, 0), pair_capacity=train_steps * crops_per_step)
    if velocity:
        dn.set_velocity_form(True)
        dn.set_scales(*velocity_scales(judge_cfg))
    else:
        dn.set_scales(*moment_scales(judge_cfg))
    dn.set_params(init_params(seed % 1000))
    dn.set_loss_border(3)
    half = abi.Denoiser(lib, judge_cfg.nx, judge_cfg.ny, judge_cfg.nz, judge_cfg.periodic, pair_capacity=1)
    half.set_scales(*moment_scales(judge_cfg))
    rng = np.random.default_rng(seed)
    judge = filled_context(lib, judge_cfg, seed)
    n_judge = sum(judge.num_particles(s) for s in range(len(judge_cfg.populations)))
    ref = {}
    judge_noise = {}
    try:
        for st in range(train_steps):
            judge.step(1)
            org = np.stack([rng.integers(0, n - crop + 1, crops_per_step)
                            for n in (judge_cfg.nx, judge_cfg.ny, judge_cfg.nz)], axis=1)
            dn.add_crops(judge, factor, st % factor, org)
        t_judge = 0.0
        for st in range(eval_steps // every):
            t_judge += _timed_steps(judge, every)
            k = train_steps + (st + 1) * every
            ref[k] = (judge.download_array("cellRhoQi"), judge.download_array("cellJi"))
            half.add_pair(judge, 2, 0)
            e = half.pair_error(0)
            judge_noise[k] = (e["raw_rho"], e["raw_J"])
        judge_ms = t_judge / eval_steps
    finally:
        judge.close()
        half.close()
    log(f"check run: {n_judge} ions, {judge_ms:.2f} ms/step, split-half noise {judge_noise}")
    t0 = time.time()
    losses = [dn.train(adam_steps // 20, lr) for _ in range(20)]
    train_s = time.time() - t0
    params = dn.params()
    if rho_only:
        last = params[2 * LAYER:3 * LAYER]
        last[:TAPS * C * C].reshape(TAPS, C, C)[:, :, 1:4] = 0.0
        last[TAPS * C * C + 1:TAPS * C * C + 4] = 0.0
    dn.close()
    log(f"training: {adam_steps} Adam steps on {train_steps * crops_per_step} crop pairs, {train_s:.1f} s, "
        f"losses {losses[0]:.4g} -> {losses[-1]:.4g}")

    def run_low(ppc: int, learned: bool) -> dict:
        cfg = geom(float(ppc), scale)
        ctx = filled_context(lib, cfg, seed + 7, path=low_path if learned else abi.PATH_FAST)
        net = None
        try:
            if learned:
                net = abi.Denoiser(lib, cfg.nx, cfg.ny, cfg.nz, cfg.periodic)
                if velocity:
                    net.set_velocity_form(True)
                    net.set_scales(*velocity_scales(cfg))
                else:
                    net.set_scales(*moment_scales(cfg))
                net.set_params(params)
                if keep_radius > 0:
                    net.set_keep_mask(keep_mask(cfg, keep_radius))
                ctx.set_denoiser(net, True)
            ctx.step(train_steps)
            n_ions = sum(ctx.num_particles(s) for s in range(len(cfg.populations)))
            on = learned
            gate_step = None
            rows, t = [], 0.0
            for st in range(eval_steps // every):
                t += _timed_steps(ctx, every)
                k = train_steps + (st + 1) * every
                r, j = ctx.download_array("cellRhoQi"), ctx.download_array("cellJi")
                e_r, e_j = relative_l2(r, ref[k][0]), relative_l2(j, ref[k][1])
                n_r, n_j = judge_noise[k]
                t_r = float(np.sqrt(max(e_r * e_r - n_r * n_r, 0.0)))
                t_j = float(np.sqrt(max(e_j * e_j - n_j * n_j, 0.0)))
                if learned and gate_step is None and max(t_r, t_j) > threshold:
                    gate_step = k
                    if enforce_gate:
                        ctx.set_denoiser(net, False)
                        on = False
                rows.append({"step": k, "rho": e_r, "J": e_j, "rho_vs_truth": t_r, "J_vs_truth": t_j,
                             "denoiser_on": on if learned else None})
            ms = t / eval_steps
            out = {"ppc": ppc, "learned": learned, "ions": int(n_ions), "ms_per_step": ms,
                   "sim_s_per_wall_s": cfg.dt / (ms / 1e3), "samples": rows,
                   "max_error": max(max(x["rho"], x["J"]) for x in rows),
                   "max_error_vs_truth": max(max(x["rho_vs_truth"], x["J_vs_truth"]) for x in rows),
                   "gate_would_switch_off_at": gate_step if learned else None,
                   "gate_enforced": enforce_gate if learned else None}
            log(f"{'learned' if learned else 'plain'} {ppc} ppc: {ms:.3f} ms/step, max error "
                f"{out['max_error']:.4f} (vs truth {out['max_error_vs_truth']:.4f})")
            return out
        finally:
            ctx.close()
            if net is not None:
                net.close()

    learned_run = run_low(low_ppc, True)
    plain = [run_low(p, False) for p in plain_ppcs]
    e_l = learned_run["max_error"]
    match = [p for p in plain if p["max_error"] <= e_l]
    above = [p for p in plain if p["max_error"] > e_l]
    res = {
        "workload": workload, "geometry": [judge_cfg.nx, judge_cfg.ny, judge_cfg.nz], "dx_m": judge_cfg.dx,
        "dt_s": judge_cfg.dt, "learned_path": "fp32" if low_path == abi.PATH_FP32 else "fast",
        "denoised": "rho" if rho_only else ("rho, J/rho" if velocity else "rho, J"),
        "keep_radius": keep_radius,
        "check_run": {"ppc": judge_ppc, "ions": int(n_judge), "ms_per_step": judge_ms,
                      "split_half_noise": {str(k): {"rho": v[0], "J": v[1]} for k, v in judge_noise.items()}},
        "training": {"pairs": train_steps * crops_per_step, "crop": crop, "factor": factor, "adam_steps": adam_steps,
                     "lr": lr, "seconds": round(train_s, 1), "losses": [round(x, 6) for x in losses]},
        "window": {"first_step": train_steps + 1, "last_step": train_steps + eval_steps, "every": every},
        "threshold": threshold, "learned": learned_run, "plain": plain,
        "matched_error": None,
        "seconds": round(time.time() - t_start, 1),
    }
    # plain runs at least as accurate as the learned form bound its matched-error
    # speed-up from above (the matching ppc is at most theirs), less accurate
    # ones from below (the learned form is both more accurate and faster)
    res["matched_error"] = {"learned_max_error": e_l}
    if above:
        a = max(above, key=lambda p: p["ppc"])
        res["matched_error"].update({
            "speedup_lower_bound": a["ms_per_step"] / learned_run["ms_per_step"],
            "lower_bound_plain_ppc": a["ppc"], "lower_bound_plain_error": a["max_error"]})
    if match:
        m = min(match, key=lambda p: p["ppc"])
        res["matched_error"].update({
            "speedup_upper_bound": m["ms_per_step"] / learned_run["ms_per_step"],
            "upper_bound_plain_ppc": m["ppc"], "upper_bound_plain_error": m["max_error"]})
    res["matched_error"]["note"] = ("measured plain runs only: the plain ppc matching the learned form's error "
                                    "lies between the two bounds' ppc")
    return res


def apply_timing(scale: float = 1.0, ppc: float = 8.0, warmup: int = 3, steps: int = 10, seed: int = 5) -> dict:
    """Cost of the denoiser inside the step: a C4 context at `ppc` with the
    network applied between deposit and field update (untrained weights
    slightly perturbed, so every layer computes), `warmup` untimed steps, then
    `steps` steps with the library's per-kernel CUDA-event timer. The
    convolutions execute 3 x 27 x 16 x 16 x 2 flop per voxel on the tensor
    cores (layer 0 has 4 input and layer 2 4 output channels, padded to 16)."""
    lib = abi.gpu_library()
    cfg = c4_config(ppc, scale)
    ctx = filled_context(lib, cfg, seed)
    net = abi.Denoiser(lib, cfg.nx, cfg.ny, cfg.nz, cfg.periodic)
    try:
        net.set_scales(*moment_scales(cfg))
        net.set_params(init_params(0) * 1.01)
        ctx.set_denoiser(net, True)
        ctx.step(warmup)
        ctx.set_timing(True)
        ctx.step(steps)
        t = {k: v / steps for k, v in ctx.timing().items()}
        ctx.set_timing(False)
    finally:
        ctx.close()
        net.close()
    voxels = cfg.nx * cfg.ny * cfg.nz
    flop = 3 * TAPS * C * C * 2 * voxels
    ms = t.get("dn_apply", 0.0)
    return {"geometry": [cfg.nx, cfg.ny, cfg.nz], "ppc": ppc, "steps": steps, "dn_apply_ms_per_step": ms,
            "step_ms": sum(t.values()), "executed_tflops": flop / (ms * 1e-3) / 1e12 if ms > 0 else None,
            "kernel_ms": t}


def main(argv=None):
    import argparse
    import json
    ap = argparse.ArgumentParser(description="the learned form in closed loop against a high-ppc check run")
    ap.add_argument("--apply-only", action="store_true",
                    help="only time the denoiser applied inside the step (apply_timing) at --scale")
    ap.add_argument("--scale", type=float, default=1.0)
    ap.add_argument("--judge-ppc", type=int, default=256)
    ap.add_argument("--train-steps", type=int, default=100)
    ap.add_argument("--eval-steps", type=int, default=100)
    ap.add_argument("--adam-steps", type=int, default=4000)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--rho-only", action="store_true", help="denoise the charge density only (keep the current)")
    ap.add_argument("--velocity", action="store_true", help="denoise rho and the bulk velocity J/rho")
    ap.add_argument("--keep-radius", type=float, default=0.0,
                    help="leave the moments within this many obstacle radii of the planet as deposited")
    ap.add_argument("--plain", default="8,16,32,64,128")
    ap.add_argument("--workload", default="mars", choices=sorted(GEOMETRIES))
    ap.add_argument("--learned-path", default="fast", choices=["fast", "fp32"],
                    help="particle path of the learned run (the check and plain runs are FP64)")
    ap.add_argument("--json", default=None)
    a = ap.parse_args(argv)
    if a.apply_only:
        out = apply_timing(scale=a.scale)
        print(json.dumps(out))
        return
    out = closed_loop(scale=a.scale, judge_ppc=a.judge_ppc, train_steps=a.train_steps, eval_steps=a.eval_steps,
                      adam_steps=a.adam_steps, lr=a.lr, plain_ppcs=tuple(int(x) for x in a.plain.split(",")),
                      workload=a.workload, rho_only=a.rho_only, velocity=a.velocity,
                      keep_radius=a.keep_radius,
                      low_path=abi.PATH_FP32 if a.learned_path == "fp32" else abi.PATH_FAST)
    print(json.dumps(out))
    if a.json:
        with open(a.json, "w") as f:
            json.dump(out, f, indent=1)


if __name__ == "__main__":
    main()
