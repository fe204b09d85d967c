"""rhgpu_reduce_diagnostics against the population and field logs of the
reference (logCalcParticle / logCalcField, diagnostics.h:187-404) computed in
numpy from the downloaded state: sums to 1e-12 relative of their magnitude,
maxima and counts exact."""
import numpy as np
import pytest

from rhybrid_b200 import abi
from rhybrid_b200 import config as cf

from harness import closed_box_config, load

pytestmark = pytest.mark.gpu


def expected(ctx, cfg):
    pops = []
    for s in range(ctx.nspecies):
        _, p = ctx.download_particles(s)
        w, v = p[:, 6], p[:, 3:6]
        v2 = (v ** 2).sum(axis=1)
        vt = np.sqrt(v2)
        pops.append({"N_macroParticles": float(p.shape[0]), "N_realParticles": w.sum(), "sumVx": (w * v[:, 0]).sum(),
                     "sumVy": (w * v[:, 1]).sum(), "sumVz": (w * v[:, 2]).sum(), "sumV": (w * vt).sum(),
                     "sumWV2": (w * v2).sum(), "maxVi": vt.max() if vt.size else 0.0})
    nx, ny, nz = cfg.nx, cfg.ny, cfg.nz
    grid = lambda name: ctx.download_array(name).reshape(nz, ny, nx, -1)   # noqa: E731
    fb, ji, ep, ne, ue = grid("faceB"), grid("cellJi"), grid("cellEp"), grid("nodeE"), grid("cellUe")
    rho = ctx.download_array("cellRhoQi").reshape(nz, ny, nx)
    flags = cf.init_grid(cfg)["flags"].reshape(nz, ny, nx)
    per = cfg.periodic
    ok = np.ones((nz, ny, nx), bool)
    if not per[0]: ok[:, :, 0] = ok[:, :, -1] = False
    if not per[1]: ok[:, 0, :] = ok[:, -1, :] = False
    if not per[2]: ok[0, :, :] = ok[-1, :, :] = False
    ok &= (flags & abi.FLAG_INNER_FIELD) == 0
    bx0 = np.roll(fb[..., 0], 1, axis=2)
    by0 = np.roll(fb[..., 1], 1, axis=1)
    bz0 = np.roll(fb[..., 2], 1, axis=0)
    divB = np.abs(((fb[..., 0] - bx0) + (fb[..., 1] - by0) + (fb[..., 2] - bz0)) / cfg.dx)
    B = np.stack([0.5 * (fb[..., 0] + bx0), 0.5 * (fb[..., 1] + by0), 0.5 * (fb[..., 2] + bz0)], -1)
    B2 = (B ** 2).sum(-1)
    Bt = np.sqrt(B2)
    dpb = np.where(Bt > 0, divB / np.where(Bt > 0, Bt, 1.0), 0.0)
    cellE = -np.cross(ue, B)
    norm = lambda a: np.sqrt((a ** 2).sum(-1))   # noqa: E731
    m = ok
    f = {"N_cells": float(m.sum()), "sumBx": B[..., 0][m].sum(), "sumBy": B[..., 1][m].sum(),
         "sumBz": B[..., 2][m].sum(), "sumB": Bt[m].sum(), "maxB": Bt[m].max(), "sumDivB": divB[m].sum(),
         "maxDivB": divB[m].max(), "maxDivBPerB": dpb[m].max(), "sumB2": B2[m].sum(),
         "sumCellJix": ji[..., 0][m].sum(), "sumCellJiy": ji[..., 1][m].sum(), "sumCellJiz": ji[..., 2][m].sum(),
         "sumCellJi": norm(ji)[m].sum(), "maxCellJi": norm(ji)[m].max(),
         "sumCellEpx": ep[..., 0][m].sum(), "sumCellEpy": ep[..., 1][m].sum(), "sumCellEpz": ep[..., 2][m].sum(),
         "sumCellEp": norm(ep)[m].sum(), "maxCellEp": norm(ep)[m].max(), "sumCellEp2": (ep ** 2).sum(-1)[m].sum(),
         "sumNodeEx": ne[..., 0][m].sum(), "sumNodeEy": ne[..., 1][m].sum(), "sumNodeEz": ne[..., 2][m].sum(),
         "sumNodeE": norm(ne)[m].sum(), "maxNodeE": norm(ne)[m].max(), "sumNodeE2": (ne ** 2).sum(-1)[m].sum(),
         "sumCellE2": (cellE ** 2).sum(-1)[m].sum(), "maxUe": norm(ue)[m].max(), "sumCellRhoQi": rho[m].sum()}
    return pops, f


def check(got, want, what, scale_of):
    for k, w in want.items():
        v = got[k]
        if k.startswith("max") or k in ("N_macroParticles", "N_cells"):
            assert v == pytest.approx(w, rel=1e-15, abs=0.0), f"{what} {k}: {v} vs {w}"
        else:
            assert abs(v - w) <= 1e-12 * scale_of(k), f"{what} {k}: {v} vs {w}"


@pytest.mark.parametrize("fast", [False, True], ids=["exact", "fast"])
def test_diagnostics_match_numpy(fast):
    cfg = closed_box_config()
    grid, pops = cf.initial_state(cfg)
    ctx = abi.Context(abi.gpu_library(), cf.params(cfg), cf.species(cfg), capacity=[p[1].shape[0] + 256 for p in pops])
    try:
        ctx.select_path(fast)
        load(ctx, cfg, grid, pops)
        ctx.step(3)
        d = ctx.reduce_diagnostics()
        wp, wf = expected(ctx, cfg)
        for s, (g, w) in enumerate(zip(d["populations"], wp)):
            mag = {"sumVx": "sumV", "sumVy": "sumV", "sumVz": "sumV"}
            check(g, w, f"species {s}", lambda k: abs(w[mag.get(k, k)]) + 1e-300)
        mag = {"sumBx": "sumB", "sumBy": "sumB", "sumBz": "sumB", "sumCellJix": "sumCellJi", "sumCellJiy": "sumCellJi",
               "sumCellJiz": "sumCellJi", "sumCellEpx": "sumCellEp", "sumCellEpy": "sumCellEp",
               "sumCellEpz": "sumCellEp", "sumNodeEx": "sumNodeE", "sumNodeEy": "sumNodeE", "sumNodeEz": "sumNodeE"}
        check(d["field"], wf, "field", lambda k: abs(wf[mag.get(k, k)]) + 1e-300)
        assert d["field"]["N_cells"] > 0 and d["populations"][0]["N_macroParticles"] > 0
    finally:
        ctx.close()
