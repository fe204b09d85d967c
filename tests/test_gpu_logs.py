"""Population and field log files (rhgpu_log_open / rhgpu_log_write) against
the reference's own log writer (diagnostics::logWriteParticleField,
src/diagnostics.h:405-818, built from the reference's sources in
oracle/_ref) run on the same state: same files, same columns and blanks,
values to the printed precision (the sums are formed in another order), the
counter rates exact, and the max-B stop."""
import math

import numpy as np
import pytest

from rhybrid_b200 import abi
from rhybrid_b200 import config as cf

from harness import closed_box_config, load

pytestmark = pytest.mark.gpu

NAMES = ["H+sw", "O+"]
POP_HEADER = ["% columns = 17", "% 01. Time [s]", "% 02. Particles [#]", "% 03. Macroparticles [#]",
              "% 04. avg(Vx) [m/s]", "% 05. avg(Vy) [m/s]", "% 06. avg(Vz) [m/s]", "% 07. avg(|V|) [m/s]",
              "% 08. Kinetic energy [J]", "% 09. max(|V|) [m/s]", "% 10. Escape rate [#/s]",
              "% 11. Impact rate [#/s]", "% 12. Inject rate [#/s]", "% 13. Macroparticle inject rate [#/dt]",
              "% 14. Kinetic energy escape rate [J/s]", "% 15. Kinetic energy impact rate [J/s]",
              "% 16. Kinetic energy inject rate [J/s]", "% 17. Constraint maxVi rate [#/dt]"]


def run_logs(lib, cfg, path, outdir, steps=(0, 3, 3), stop_B=math.inf):
    grid, pops = cf.initial_state(cfg)
    ctx = abi.Context(lib, cf.params(cfg), cf.species(cfg), capacity=[p[1].shape[0] + 512 for p in pops])
    stops = []
    try:
        if path is not None:
            ctx.set_path(path)
        load(ctx, cfg, grid, pops)
        ctx.log_open(str(outdir), NAMES[:ctx.nspecies], precision=10, max_B_stop_run=stop_B)
        for n in steps:
            if n:
                ctx.step(n)
            stops.append(ctx.log_write())
        ctx.log_close()
    finally:
        ctx.close()
    return stops


def data_lines(path):
    return [ln.rstrip("\n") for ln in open(path) if not ln.startswith("%")]


# signed averages are compared on the scale of their magnitude's average
# (1-based column -> column of the |.| average)
POP_SCALE = {4: 7, 5: 7, 6: 7}
FIELD_SCALE = {2: 5, 3: 5, 4: 5, 11: 14, 12: 14, 13: 14, 16: 19, 17: 19, 18: 19, 22: 25, 23: 25, 24: 25}


def compare(gpu_dir, ref_dir, rel, dx):
    files = [f"pop00{s + 1}_{n}.log" for s, n in enumerate(NAMES)] + ["field.log"]
    bad = []
    for f in files:
        g, r = data_lines(gpu_dir / f), data_lines(ref_dir / f)
        assert len(g) == len(r) > 0, f
        scale_of = FIELD_SCALE if f == "field.log" else POP_SCALE
        for lg, lr in zip(g, r):
            tg, tr = lg.split(" "), lr.split(" ")
            # same columns, the same empty fields (double blanks), trailing blank
            assert [t == "" for t in tg] == [t == "" for t in tr], f"{f}: layout\n{lg}\n{lr}"
            xg = [float(t) for t in tg if t]
            xr = [float(t) for t in tr if t]
            for k, (x, y) in enumerate(zip(xg, xr)):
                if x == y:
                    continue
                c = scale_of.get(k + 1)
                scale = max(abs(x), abs(y), abs(xr[c - 1]) if c else 0.0)
                if f == "field.log" and k + 1 in (7, 8):
                    # div B is round-off of |B|/dx: its own scale
                    scale = max(scale, xr[4] / dx)
                if f == "field.log" and k + 1 == 9:
                    scale = max(scale, 1.0)
                if not abs(x - y) <= rel * scale:
                    bad.append(f"{f} column {k + 1}: {x!r} vs {y!r}")
    assert not bad, "\n".join(bad)


@pytest.mark.parametrize("path,rel", [(abi.PATH_EXACT, 2e-9), (abi.PATH_FAST, 1e-8), (abi.PATH_FP32, 1e-4)],
                         ids=["exact", "fast", "fp32"])
def test_logs_match_reference_writer(tmp_path, ref_lib, path, rel):
    cfg = closed_box_config()
    gdir, rdir = tmp_path / "gpu", tmp_path / "ref"
    gdir.mkdir()
    rdir.mkdir()
    sg = run_logs(abi.gpu_library(), cfg, path, gdir)
    sr = run_logs(ref_lib, cfg, None, rdir)
    assert [s for s, _ in sg] == [s for s, _ in sr] == [False, False, False]
    compare(gdir, rdir, rel, cfg.dx)
    # the headers of src/user.cpp:2158-2229
    pop = [ln.rstrip("\n") for ln in open(gdir / "pop001_H+sw.log") if ln.startswith("%")]
    assert pop[0] == "% H+sw" and pop[1].startswith("% m [kg] = +1.67") and pop[2].startswith("% q [C] = +1.60")
    assert pop[3:] == POP_HEADER
    fld = [ln.rstrip("\n") for ln in open(gdir / "field.log") if ln.startswith("%")]
    assert fld[:3] == ["% field", "% columns = 41", "% 01. Time [s]"] and len(fld) == 43
    assert fld[-1] == "% 41. Maximum electron fluid speed [m/s]"
    assert all(len([t for t in ln.split(" ") if t]) == 41 for ln in data_lines(gdir / "field.log"))
    assert all(len([t for t in ln.split(" ") if t]) == 17 for ln in data_lines(gdir / "pop001_H+sw.log"))


def test_log_stop_on_max_B(tmp_path, ref_lib):
    cfg = closed_box_config()
    gdir, rdir = tmp_path / "gpu", tmp_path / "ref"
    gdir.mkdir()
    rdir.mkdir()
    sg = run_logs(abi.gpu_library(), cfg, abi.PATH_FAST, gdir, steps=(0, 2), stop_B=1e-12)
    sr = run_logs(ref_lib, cfg, None, rdir, steps=(0, 2), stop_B=1e-12)
    assert [s for s, _ in sg] == [s for s, _ in sr] == [True, True]
    assert "CONSTRAINT: maximum B reached" in sg[1][1]


def test_log_counters_zeroed_after_write(tmp_path):
    cfg = closed_box_config()
    grid, pops = cf.initial_state(cfg)
    ctx = abi.Context(abi.gpu_library(), cf.params(cfg), cf.species(cfg), capacity=[p[1].shape[0] + 512 for p in pops])
    try:
        load(ctx, cfg, grid, pops)
        ctx.log_open(str(tmp_path), NAMES)
        ctx.step(4)
        before = ctx.counters()
        assert any(v > 0 for k, v in before.items() if k != "gridTemporalAverageCounter")
        stop, msg = ctx.log_write(main_log_diagnostics=True)
        assert not stop and "Diagnostics (time step = 4" in msg and "Nmacroparticles(O+)" in msg
        after = ctx.counters()
        assert all(v == 0 for k, v in after.items() if k != "gridTemporalAverageCounter")
        assert after["gridTemporalAverageCounter"] == before["gridTemporalAverageCounter"]
    finally:
        ctx.close()


@pytest.mark.parametrize("path", [abi.PATH_EXACT, abi.PATH_FAST, abi.PATH_FP32], ids=["exact", "fast", "fp32"])
def test_scales_match_numpy(path):
    """The six field-log scales of rhgpu_reduce_diagnostics against numpy from
    the downloaded state (diagnostics.h:223-238, 375-395)."""
    cfg = closed_box_config()
    grid, pops = cf.initial_state(cfg)
    ctx = abi.Context(abi.gpu_library(), cf.params(cfg), cf.species(cfg), capacity=[p[1].shape[0] + 512 for p in pops])
    try:
        ctx.set_path(path)
        load(ctx, cfg, grid, pops)
        ctx.step(3)
        d = ctx.reduce_diagnostics(scales=True)["field"]
        N = cfg.nx * cfg.ny * cfg.nz
        rhom = np.zeros(N)
        sp = cf.species(cfg)
        for s in range(ctx.nspecies):
            counts, p = ctx.download_particles(s)
            cell = np.repeat(np.arange(N), counts.astype(np.int64))
            np.add.at(rhom, cell, p[:, 6] * sp[s].m)
        rhom /= cfg.dx ** 3
        rhom = np.maximum(rhom, cf.params(cfg).min_ion_charge_density * abi.MASS_PROTON / abi.CHARGE_ELEMENTARY)
        rho = ctx.download_array("cellRhoQi")
        fb = ctx.download_array("faceB").reshape(cfg.nz, cfg.ny, cfg.nx, 3)
        B = np.stack([0.5 * (fb[..., 0] + np.roll(fb[..., 0], 1, 2)), 0.5 * (fb[..., 1] + np.roll(fb[..., 1], 1, 1)),
                      0.5 * (fb[..., 2] + np.roll(fb[..., 2], 1, 0))], -1).reshape(N, 3)
        Bt = np.sqrt((B ** 2).sum(-1))
        flags = cf.init_grid(cfg)["flags"].reshape(cfg.nz, cfg.ny, cfg.nx)
        ok = np.ones((cfg.nz, cfg.ny, cfg.nx), bool)
        per = cfg.periodic
        if not per[0]: ok[:, :, 0] = ok[:, :, -1] = False
        if not per[1]: ok[:, 0, :] = ok[:, -1, :] = False
        if not per[2]: ok[0, :, :] = ok[-1, :, :] = False
        ok = (ok & ((flags & abi.FLAG_INNER_FIELD) == 0)).reshape(N)
        mu0, e, me, mp = abi.PERMEABILITY, abi.CHARGE_ELEMENTARY, abi.MASS_ELECTRON, abi.MASS_PROTON
        rq = rho[ok][rho[ok] > 0]
        de = np.sqrt(me / (mu0 * e * rq))
        rm = rhom[ok]
        di = np.sqrt(mp * mp / (mu0 * (e * e) * rm))
        va = Bt[ok] / np.sqrt(mu0 * rm)
        tl = 2.0 * np.pi * mp / (e * Bt[ok][Bt[ok] > 0])
        want = {"minInerLengthElectron": de.min(), "maxInerLengthElectron": de.max(),
                "minInerLengthProton": di.min(), "maxInerLengthProton": di.max(), "minTLarmor": tl.min(),
                "maxVAlfven": va.max()}
        for k, w in want.items():
            assert d[k] == pytest.approx(w, rel=1e-13), f"{k}: {d[k]} vs {w}"
    finally:
        ctx.close()
