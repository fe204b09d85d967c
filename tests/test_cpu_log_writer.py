"""The library's log writer (rhybrid_b200/csrc/rh_logs.h, host code) against
the reference's own writer (diagnostics::logWriteParticleField, built from
its sources in oracle/_ref) on CPU: the reference writes its files from its
state; the library's writer, compiled into tests/log_writer_harness.cpp, gets
the same log steps' sums (formed here in numpy from that state, as
logCalcParticle / logCalcField define them) and counters. Same files, columns
and blanks, values to the printed precision."""
import os
import shutil
import subprocess

import numpy as np
import pytest

from rhybrid_b200 import abi
from rhybrid_b200 import config as cf

from harness import closed_box_config, load
from test_gpu_logs import NAMES, compare

HERE = os.path.dirname(os.path.abspath(__file__))
BIG = np.finfo(np.float64).max


@pytest.fixture(scope="module")
def writer(tmp_path_factory):
    if shutil.which("g++") is None:
        pytest.skip("g++ not available")
    exe = str(tmp_path_factory.mktemp("lw") / "log_writer_harness")
    subprocess.run(["g++", "-std=c++17", "-O1", "-o", exe, os.path.join(HERE, "log_writer_harness.cpp")], check=True)
    return exe


def log_step_values(ctx, cfg, t_start):
    """One log step's inputs of the library's writer: population sums,
    counters, field sums and scales, field counters."""
    sp = cf.species(cfg)
    N = cfg.ncells
    dV = cfg.dx ** 3
    c = ctx.counters()
    out = []
    rhom = np.zeros(N)
    for s in range(ctx.nspecies):
        cnt, p = ctx.download_particles(s)
        w, v = p[:, 6], p[:, 3:6]
        v2 = (v ** 2).sum(axis=1)
        vt = np.sqrt(v2)
        out += [float(p.shape[0]), w.sum(), (w * v[:, 0]).sum(), (w * v[:, 1]).sum(), (w * v[:, 2]).sum(),
                (w * vt).sum(), (w * v2).sum(), vt.max() if vt.size else 0.0]
        # escape, impact, inject, inject macro, escape KE, impact KE, inject KE, maxVi
        out += [c[f"particleEscape[{s}]"], c[f"particleImpact[{s}]"], 0.0, 0.0, c[f"particleEscapeKineticEnergy[{s}]"],
                c[f"particleImpactKineticEnergy[{s}]"], 0.0, c[f"particleMaxVi[{s}]"]]
        np.add.at(rhom, np.repeat(np.arange(N), cnt.astype(np.int64)), w * sp[s].m)
    rhom = np.maximum(rhom / dV, cf.params(cfg).min_ion_charge_density * abi.MASS_PROTON / abi.CHARGE_ELEMENTARY)
    grid = lambda name: ctx.download_array(name).reshape(cfg.nz, cfg.ny, cfg.nx, -1)   # noqa: E731
    fb, ji, ep, ne, ue = grid("faceB"), grid("cellJi"), grid("cellEp"), grid("nodeE"), grid("cellUe")
    rho = ctx.download_array("cellRhoQi").reshape(cfg.nz, cfg.ny, cfg.nx)
    flags = cf.init_grid(cfg)["flags"].reshape(cfg.nz, cfg.ny, cfg.nx)
    m = np.ones((cfg.nz, cfg.ny, cfg.nx), bool)
    m[:, :, 0] = m[:, :, -1] = m[:, 0, :] = m[:, -1, :] = m[0] = m[-1] = False
    m &= (flags & abi.FLAG_INNER_FIELD) == 0
    bx0, by0, bz0 = np.roll(fb[..., 0], 1, 2), np.roll(fb[..., 1], 1, 1), np.roll(fb[..., 2], 1, 0)
    divB = np.abs(((fb[..., 0] - bx0) + (fb[..., 1] - by0) + (fb[..., 2] - bz0)) / cfg.dx)
    B = np.stack([0.5 * (fb[..., 0] + bx0), 0.5 * (fb[..., 1] + by0), 0.5 * (fb[..., 2] + bz0)], -1)
    B2 = (B ** 2).sum(-1)
    Bt = np.sqrt(B2)
    nrm = lambda a: np.sqrt((a ** 2).sum(-1))   # noqa: E731
    cellE = -np.cross(ue, B)
    mu0, e, me, mp = abi.PERMEABILITY, abi.CHARGE_ELEMENTARY, abi.MASS_ELECTRON, abi.MASS_PROTON
    rq = rho[m][rho[m] > 0]
    rm = rhom.reshape(cfg.nz, cfg.ny, cfg.nx)[m]
    de = lambda r: np.sqrt(me / (mu0 * e * r))                   # noqa: E731
    di = lambda r: np.sqrt(mp * mp / (mu0 * (e * e) * r))         # noqa: E731
    bt = Bt[m][Bt[m] > 0]
    f = [float(m.sum()), B[..., 0][m].sum(), B[..., 1][m].sum(), B[..., 2][m].sum(), Bt[m].sum(), Bt[m].max(),
         divB[m].sum(), divB[m].max(), np.where(Bt > 0, divB / np.where(Bt > 0, Bt, 1), 0)[m].max(), B2[m].sum(),
         ji[..., 0][m].sum(), ji[..., 1][m].sum(), ji[..., 2][m].sum(), nrm(ji)[m].sum(), nrm(ji)[m].max(),
         ep[..., 0][m].sum(), ep[..., 1][m].sum(), ep[..., 2][m].sum(), nrm(ep)[m].sum(), nrm(ep)[m].max(),
         (ep ** 2).sum(-1)[m].sum(), ne[..., 0][m].sum(), ne[..., 1][m].sum(), ne[..., 2][m].sum(), nrm(ne)[m].sum(),
         nrm(ne)[m].max(), (ne ** 2).sum(-1)[m].sum(), (cellE ** 2).sum(-1)[m].sum(),
         de(rq.max()) if rq.size else BIG, de(rq.min()) if rq.size else -BIG,
         di(rm.max()) if rm.size else BIG, di(rm.min()) if rm.size else -BIG,
         2.0 * np.pi * mp / (e * bt.max()) if bt.size else BIG, (Bt[m] / np.sqrt(mu0 * rm)).max(), nrm(ue)[m].max()]
    # maxCellUe, maxNodeUe, the maxVw column (which carries the node Ue counter), maxE, min rho cell, min rho node
    fc = [c["fieldMaxCellUe"], c["fieldMaxNodeUe"], c["fieldMaxNodeUe"], c["fieldMaxE"], c["fieldMinCellRhoQi"],
          c["fieldMinNodeRhoQi"]]
    t, ts = ctx.time()
    head = [t, cfg.dt, cfg.dx, dV, t_start, ts, abi.PERMEABILITY, abi.PERMITTIVITY]
    return head, out, f, fc


def test_log_writer_matches_reference_writer(tmp_path, ref_lib, writer):
    cfg = closed_box_config()
    gdir, rdir = tmp_path / "lib", tmp_path / "ref"
    gdir.mkdir()
    rdir.mkdir()
    grid, pops = cf.initial_state(cfg)
    ctx = abi.Context(ref_lib, cf.params(cfg), cf.species(cfg), capacity=[p[1].shape[0] + 256 for p in pops])
    steps, stops = [], []
    try:
        load(ctx, cfg, grid, pops)
        ctx.log_open(str(rdir), NAMES)
        t_start = ctx.time()[0]
        for n in (0, 3, 3):
            if n:
                ctx.step(n)
            steps.append(log_step_values(ctx, cfg, t_start))
            stops.append(ctx.log_write()[0])
            t_start = ctx.time()[0]
        ctx.log_close()
    finally:
        ctx.close()
    sp = cf.species(cfg)
    lines = [f"{gdir} {len(sp)} 10 1e300 0 {len(steps)}"]
    lines += [f"{NAMES[s]} {sp[s].m!r} {sp[s].q!r}" for s in range(len(sp))]
    for head, pop, f, fc in steps:
        lines.append(" ".join(repr(float(x)) for x in head[:5]) + f" {int(head[5])} {head[6]!r} {head[7]!r}")
        lines.append(" ".join(repr(float(x)) for x in pop))
        lines.append(" ".join(repr(float(x)) for x in f + fc))
    inp = tmp_path / "steps.txt"
    inp.write_text("\n".join(lines) + "\n")
    res = subprocess.run([writer, str(inp)], check=True, capture_output=True, text=True)
    assert res.stdout.split() == ["ok"] * 3 and stops == [False] * 3
    compare(gdir, rdir, 2e-9, cfg.dx)
