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
"""
from __future__ import annotations

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
