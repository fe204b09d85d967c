"""Shared test helpers: run any implementation of the rhgpu C ABI on a
configuration and collect its whole state."""
import numpy as np

from rhybrid_b200 import abi
from rhybrid_b200 import config as cf

STATE_ARRAYS = ["faceB", "cellB", "cellUe", "cellEp", "cellRhoQi", "cellJi", "cellJ", "nodeRhoQi",
                "nodeJi", "nodeJ", "nodeUe", "nodeB", "nodeE", "nodeEta", "cellAverageB"]


def load(ctx, cfg, grid, pops):
    ctx.upload_array("faceB", grid["faceB"])
    ctx.upload_array("cellB", grid["cellB"])
    ctx.upload_array("nodeEta", grid["nodeEta"])
    ctx.upload_cell_flags(grid["flags"])
    for s, (cnt, p) in enumerate(pops):
        ctx.upload_particles(s, cnt, p)


def snapshot(ctx):
    st = {"arrays": {n: ctx.download_array(n).copy() for n in STATE_ARRAYS}, "particles": []}
    for s in range(ctx.nspecies):
        st["particles"].append(ctx.download_particles(s))
    st["counters"] = ctx.counters()
    st["time"] = ctx.time()
    return st


def run(lib, cfg, nsteps, grid=None, pops=None, capacity=None, setup=None, per_step=False, fast=False):
    """fast=False: the reference's order (the GPU's bit-exact path, the
    oracle's RHO_DEPOSIT_REFERENCE); fast=True: the GPU's fast path and the
    oracle's restatement of its order."""
    if grid is None:
        grid, pops = cf.initial_state(cfg)
    cap = capacity or [int(1.5 * p[1].shape[0]) + 1024 for p in pops]
    ctx = abi.Context(lib, cf.params(cfg), cf.species(cfg), capacity=cap)
    try:
        ctx.select_path(fast)
        if setup:
            setup(ctx)
        load(ctx, cfg, grid, pops)
        snaps = []
        for _ in range(nsteps if per_step else 1):
            ctx.step(1 if per_step else nsteps)
            if per_step:
                snaps.append(snapshot(ctx))
        return snaps if per_step else snapshot(ctx)
    finally:
        ctx.close()


def assert_bitwise(a, b, what=""):
    for n in STATE_ARRAYS:
        x, y = a["arrays"][n], b["arrays"][n]
        if not np.array_equal(x.view(np.uint64), y.view(np.uint64)):
            bad = np.argwhere(x.view(np.uint64) != y.view(np.uint64))
            raise AssertionError(f"{what}: array {n} differs at {bad[:5].tolist()} "
                                 f"({x.reshape(-1)[:0]}) max abs diff {np.max(np.abs(x - y))}")
    for s, ((ca, pa), (cb, pb)) in enumerate(zip(a["particles"], b["particles"])):
        assert np.array_equal(ca, cb), f"{what}: species {s} counts differ"
        assert np.array_equal(pa.view(np.uint64), pb.view(np.uint64)), \
            f"{what}: species {s} particles differ, max abs diff {np.max(np.abs(pa - pb))}"
    for k, v in a["counters"].items():
        assert v == b["counters"][k], f"{what}: counter {k}: {v} != {b['counters'][k]}"
    assert a["time"] == b["time"]


def rel_err(x, y):
    x = np.asarray(x, dtype=np.float64)
    y = np.asarray(y, dtype=np.float64)
    scale = np.max(np.abs(y)) if y.size else 0.0
    if scale == 0.0:
        return float(np.max(np.abs(x - y))) if x.size else 0.0
    return float(np.max(np.abs(x - y)) / scale)


def closed_box_config(nx=12, ny=10, nz=9, ppc=4.0, two_species=True, **kw):
    """Non-periodic box with an absorbing sphere and every field option the
    hot path has switched on: IMF walls, electron pressure, superconducting
    sphere resistivity with outer-boundary coefficients, E smoothing."""
    dx = 100e3
    R = 2.2 * dx
    pops = [cf.Population(name="H+", obstacle=R, density=2e6, velocity=(-450e3, 20e3, -10e3),
                          temperature=1e5, ppc=ppc)]
    if two_species:
        pops.append(cf.Population(name="He++", mass=3.9737, charge=2.0, obstacle=R, density=0.08e6,
                                  velocity=(-450e3, 0, 0), temperature=1e5, ppc=max(ppc / 4, 1.0)))
    c = cf.Config(nx=nx, ny=ny, nz=nz, x_min=-0.5 * nx * dx + 0.3 * dx, y_min=-0.5 * ny * dx,
                  z_min=-0.5 * nz * dx - 0.2 * dx, dx=dx, periodic=(0, 0, 0), dt=0.05,
                  R_fieldObstacle=R, R_particleObstacle=R, fieldObstacleUe=(1e3, -2e3, 0.5e3),
                  imf=(1e-9, 3e-9, -0.5e-9), imf_boundary_cellB=(1, 0, 1, 0, 0, 1),
                  imf_boundary_faceB=(1, 0, 0, 1, 1, 0), use_electron_pressure=True,
                  electron_temperature=2e5, electron_gamma=2, R_zeroElectronPressure=1.5 * dx,
                  resistivity_profile="resistivitySuperConductingSphere", resistivity_unit="Rm",
                  resistivity_value=6.0, resistivity_R=1.5 * dx,
                  resistivity_outer_cells=(2, 1, 0, 1, 1, 0), resistivity_outer_coeffs=(3, 2, 1, 4, 5, 1),
                  max_ion_velocity=1500e3, max_electron_velocity=800e3,
                  min_ion_charge_density_relative=0.3, max_electric_field=2e-3,
                  max_whistler_velocity=1500e3, electric_field_linear_smoothing_number=1,
                  electric_field_smoothing_gauss_sigma=0.8, populations=pops, name="closed_box")
    return c.replace(**kw) if kw else c


SUM_COUNTERS = ("particleEscape", "particleEscapeKineticEnergy", "particleImpact", "particleImpactKineticEnergy")


def assert_state_equal(a, b, what="", bitwise=True, rtol=0.0, sum_rtol=1e-12):
    """GPU-vs-oracle comparison: arrays and particles bitwise (or within rtol
    relative to each array's max), integer counters exact, FP-sum counters
    (escape/impact, accumulated with atomics on the GPU) within sum_rtol."""
    for n in STATE_ARRAYS:
        x, y = a["arrays"][n], b["arrays"][n]
        if bitwise:
            if not np.array_equal(x.view(np.uint64), y.view(np.uint64)):
                bad = np.argwhere(x.view(np.uint64) != y.view(np.uint64))
                raise AssertionError(f"{what}: {n} differs at {bad[:4].tolist()}, rel {rel_err(x, y):.3e}")
        else:
            e = rel_err(x, y)
            assert e <= rtol, f"{what}: {n} rel err {e:.3e} > {rtol}"
    for s, ((ca, pa), (cb, pb)) in enumerate(zip(a["particles"], b["particles"])):
        assert np.array_equal(ca, cb), f"{what}: species {s} counts differ ({ca.sum()} vs {cb.sum()})"
        if bitwise:
            assert np.array_equal(pa.view(np.uint64), pb.view(np.uint64)), \
                f"{what}: species {s} particles differ, rel {rel_err(pa, pb):.3e}"
        else:
            for col in range(7):
                e = rel_err(pa[:, col], pb[:, col])
                assert e <= rtol, f"{what}: species {s} column {col} rel err {e:.3e}"
    for k, v in a["counters"].items():
        w = b["counters"][k]
        if k.split("[")[0] in SUM_COUNTERS:
            assert abs(v - w) <= sum_rtol * max(abs(w), 1e-300), f"{what}: counter {k}: {v} vs {w}"
        else:
            assert v == w, f"{what}: counter {k}: {v} != {w}"
    assert a["time"][1] == b["time"][1] and abs(a["time"][0] - b["time"][0]) <= 1e-12 * max(1.0, abs(b["time"][0]))


def canonical_order(st):
    """The same state with each cell's particles sorted by position: the fast
    path stores a cell's particles grouped by CIC dual cell, so its per-cell
    order differs from the reference's while the set is the same."""
    out = {k: v for k, v in st.items() if k != "particles"}
    out["particles"] = []
    for cnt, p in st["particles"]:
        cell = np.repeat(np.arange(cnt.size), cnt.astype(np.int64))
        o = np.lexsort((p[:, 2], p[:, 1], p[:, 0], cell))
        out["particles"].append((cnt, p[o]))
    return out
