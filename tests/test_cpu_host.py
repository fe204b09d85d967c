"""CPU tests of the host-side logic: the C ABI library loads and exports every
entry point its header declares (no GPU call is made), parameter derivation,
initial state, and known answers of the oracle itself."""
import math
import os
import re

import numpy as np
import pytest

from rhybrid_b200 import abi
from rhybrid_b200 import config as cf

from harness import load, run

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_functions():
    txt = open(os.path.join(ROOT, "include", "rhgpu.h")).read()
    return sorted(set(re.findall(r"\b(rhgpu_[a-z_]+)\s*\(", txt)))


def test_library_exports_every_declared_symbol():
    path = abi.gpu_library_path()
    if not os.path.exists(path):
        pytest.skip("librhgpu.so not built")
    import ctypes
    dll = ctypes.CDLL(path)
    missing = [f for f in header_functions() if not hasattr(dll, f)]
    assert not missing, missing
    lib = abi.gpu_library()
    assert "sm_100a" in lib.fn["version"]().decode()


def test_entry_points_refuse_null_handles():
    """Entry points given a null context or denoiser return RHGPU_ERR_ARG
    before any CUDA call, so this runs without a GPU."""
    path = abi.gpu_library_path()
    if not os.path.exists(path):
        pytest.skip("librhgpu.so not built")
    import ctypes
    dll = ctypes.CDLL(path)
    dll.rhgpu_last_error.restype = ctypes.c_char_p
    for name, args in [("rhgpu_dn_set_velocity_form", (None, 1)), ("rhgpu_dn_set_keep_mask", (None, None)),
                       ("rhgpu_dn_set_scales", (None, ctypes.c_double(1.0), ctypes.c_double(1.0))),
                       ("rhgpu_set_path", (None, 0)), ("rhgpu_step", (None, 1)),
                       ("rhgpu_accumulate_noalloc", (None,))]:
        assert getattr(dll, name)(*args) == abi.ERR_ARG, name
        assert dll.rhgpu_last_error(), name


def test_resistivity_units():
    cfg = cf.config_empty_box()
    # Rm: eta = mu0*dx*U/Rm (resistivity.h:86-93)
    assert math.isclose(cf.resistivity_eta(cfg), abi.PERMEABILITY * cfg.dx * 400e3 / 6.0, rel_tol=1e-15)
    for unit, val, expect in [("SI", 3.0, 3.0), ("grid", 2.0, 2.0 * abi.PERMEABILITY * cfg.dx ** 2 / cfg.dt),
                              ("td", 4.0, 0.25 * abi.PERMEABILITY * cfg.dx ** 2 / cfg.dt),
                              ("URm", 1e3, 1e3 * abi.PERMEABILITY * cfg.dx)]:
        c = cfg.replace(resistivity_unit=unit, resistivity_value=val)
        assert math.isclose(cf.resistivity_eta(c), expect, rel_tol=1e-15)


def test_params_derivation():
    cfg = cf.config_mars(nx=12, ny=16, nz=16, ppc=4)
    P = cf.params(cfg)
    rhoq = 2e6 * abi.CHARGE_ELEMENTARY + 0.08e6 * 2 * abi.CHARGE_ELEMENTARY
    assert math.isclose(P.min_ion_charge_density, 0.05 * rhoq, rel_tol=1e-15)
    assert P.max_ion_speed2 == (1500e3) ** 2
    assert P.use_electron_pressure == 1 and P.isothermal_electrons == 0
    ne = rhoq / abi.CHARGE_ELEMENTARY
    assert math.isclose(P.electron_pressure_coeff, 2 * abi.BOLTZMANN * 1e5 / (ne * abi.CHARGE_ELEMENTARY ** 2), rel_tol=1e-15)
    # maximum ion speed capped at 0.9 dx/dt (user.cpp:1774-1777)
    P2 = cf.params(cfg.replace(max_ion_velocity=1e7))
    assert math.isclose(P2.max_ion_speed2, (0.9 * cfg.dx / cfg.dt) ** 2, rel_tol=1e-15)


def test_obstacle_flags():
    cfg = cf.config_mars(nx=24, ny=24, nz=24, ppc=1, dx=600e3)
    g = cf.init_grid(cfg)
    fl = g["flags"].reshape(cfg.nz, cfg.ny, cfg.nx)
    inner = (fl & abi.FLAG_INNER_FIELD) != 0
    part = (fl & abi.FLAG_INNER_PARTICLE) != 0
    assert inner.sum() > 0 and part.sum() >= inner.sum()
    # symmetric about the box centre
    assert np.array_equal(inner, inner[::-1, ::-1, ::-1])
    # superconducting sphere: no resistivity inside R
    assert (g["nodeEta"][(fl.reshape(-1) & abi.FLAG_INNER_NODE) != 0] == 0).all()


def test_uniform_population_statistics():
    cfg = cf.config_empty_box(16, 16, 16, ppc=20.0)
    cnt, p = cf.uniform_population(cfg, 0)
    assert (cnt == 20).all() and p.shape == (20 * 16 ** 3, 7)
    assert (p[:, :3] >= 0).all() and (p[:, :3] < cfg.dx).all()
    vth = math.sqrt(abi.BOLTZMANN * 1e5 / abi.MASS_PROTON)
    n = p.shape[0]
    assert abs(p[:, 3].mean() + 400e3) < 5 * vth / math.sqrt(n)
    assert abs(p[:, 4].std() / vth - 1) < 0.02
    assert np.allclose(p[:, 6], 5e6 * cfg.dx ** 3 / 20)
    # fractional ppc: probabilistic rounding keeps the mean
    cnt2, _ = cf.uniform_population(cfg.replace(populations=[cf.Population(ppc=1.5)]), 0)
    assert abs(cnt2.mean() - 1.5) < 0.05


def test_oracle_charge_conservation(port_lib):
    """examples/test_accumulation_sum_grid.py: sum(rho)*dV equals the total
    macroparticle charge on a periodic grid (checked on the oracle)."""
    cfg = cf.config_empty_box(10, 9, 8, ppc=5.0).replace(min_ion_charge_density_relative=0.0)
    grid, pops = cf.initial_state(cfg)
    ctx = abi.Context(port_lib, cf.params(cfg), cf.species(cfg))
    try:
        load(ctx, cfg, grid, pops)
        ctx.push()
        ctx.accumulate()
        rho = ctx.download_array("cellRhoQi")
        total = pops[0][1][:, 6].sum() * cfg.populations[0].q
        assert abs(rho.sum() * cfg.dx ** 3 - total) <= 1e-13 * total
    finally:
        ctx.close()


def test_oracle_gyration_preserves_speed(port_lib):
    """Boris rotation with E = 0 (first step: cellUe = 0) keeps |v| to round-off."""
    cfg = cf.config_empty_box(6, 6, 6, ppc=3.0)
    grid, pops = cf.initial_state(cfg)
    ctx = abi.Context(port_lib, cf.params(cfg), cf.species(cfg))
    try:
        load(ctx, cfg, grid, pops)
        ctx.push()
        _, p = ctx.download_particles(0)
        v0 = np.sort(np.linalg.norm(pops[0][1][:, 3:6], axis=1))
        v1 = np.sort(np.linalg.norm(p[:, 3:6], axis=1))
        assert np.max(np.abs(v1 - v0) / v0) < 1e-14
    finally:
        ctx.close()


def test_mars_sources():
    """The Mars workload's particle sources: solar wind inflow of both upstream
    populations and the O+ exosphere of examples/mars.cfg, its macroparticle
    count tied to the solar wind's (upstreamMacroPleRatio,
    particle_injector.cpp:690-712: |U| dt / dx times the upstream wall cells)."""
    cfg = cf.config_mars(exosphere=True)
    assert cf.upstream_macro_ratio(cfg) == pytest.approx(450e3 * 0.05 / 300e3 * 158 * 158)
    src = cf.source_injectors(cfg, seed=7)
    assert [j.type for j in src] == [abi.INJECT_SOLARWIND, abi.INJECT_SOLARWIND, abi.INJECT_EXOSPHERE]
    exo = src[2]
    assert exo.species == 2 and exo.n_components == 3 and exo.total_production_rate == 0.156e24
    assert list(exo.H0)[:3] == [626.2e3, 2790e3, 88.47e3] and exo.temperature == 6500.0
    grid, pops = cf.initial_state(cfg.replace(nx=12, ny=16, nz=16))
    assert pops[2][1].shape[0] == 0 and pops[0][1].shape[0] > 0
