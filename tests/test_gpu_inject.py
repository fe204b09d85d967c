"""Particle sources on the GPU (the reference's InjectorSolarWind and
InjectorFlow, src/particle_injector.cpp): counts, placement and velocity
statistics of the injected macroparticles. The reference draws from one
sequential random stream, so the comparison is statistical, as its own
tests/run_tests.py checks populations; the counter-based stream makes every
run reproducible."""
import dataclasses
import math

import numpy as np
import pytest

from rhybrid_b200 import abi
from rhybrid_b200 import config as cf

pytestmark = pytest.mark.gpu

U, T, N0, PPC = 400e3, 1e5, 5e6, 50.0


def box(periodic=(0, 1, 1), accelerate=False, nx=12, ny=8, nz=8):
    pop = cf.Population(name="H+", density=N0, velocity=(-U, 0.0, 0.0), temperature=T, ppc=PPC,
                        accelerate=accelerate)
    return cf.Config(nx=nx, ny=ny, nz=nz, x_min=-0.5 * nx * 100e3, y_min=-0.5 * ny * 100e3,
                     z_min=-0.5 * nz * 100e3, dx=100e3, periodic=periodic, dt=0.05, populations=[pop],
                     name="inject_box")


def empty_context(lib, cfg, path=abi.PATH_FAST, seed=1, cap=400000):
    grid, _ = cf.initial_state(cfg.replace(populations=[dataclasses.replace(cfg.populations[0], ppc=1.0)]))
    ctx = abi.Context(lib, cf.params(cfg), cf.species(cfg), capacity=[cap])
    ctx.set_path(path)
    ctx.upload_array("faceB", grid["faceB"])
    ctx.upload_array("cellB", grid["cellB"])
    ctx.upload_array("nodeEta", grid["nodeEta"])
    ctx.upload_cell_flags(grid["flags"])
    ctx.upload_particles(0, np.zeros(cfg.ncells, dtype=np.uint32), np.zeros((0, 7)))
    ctx.set_injectors(cf.solar_wind_injectors(cfg, seed=seed))
    return ctx


@pytest.fixture(scope="module")
def lib():
    return abi.gpu_library()


def test_solar_wind_one_step(lib):
    """ppc U dt / dx = 10 macroparticles per wall cell per step (an integer, so
    probRound is exact), at the +x wall face, moving inward."""
    cfg = box()
    ctx = empty_context(lib, cfg)
    try:
        ctx.step(1)
        cnt, p = ctx.download_particles(0)
        ncell_wall = cfg.ny * cfg.nz
        assert p.shape[0] == 10 * ncell_wall
        cell = np.repeat(np.arange(cfg.ncells), cnt.astype(np.int64))
        assert np.all(cell % cfg.nx == cfg.nx - 1)
        assert np.all(p[:, 0] == 0.0) and np.all((p[:, 1] >= 0) & (p[:, 1] < cfg.dx))
        assert np.all(p[:, 3] < 0)
        w = N0 * cfg.dx ** 3 / PPC
        assert np.allclose(p[:, 6], w, rtol=1e-12)
        ic = ctx.injection_counters()[0]
        assert ic["macroparticles"] == p.shape[0]
        assert math.isclose(ic["weight"], p.shape[0] * w, rel_tol=1e-12)
        assert math.isclose(ic["weight_v2"], float(np.sum(w * np.sum(p[:, 3:6] ** 2, axis=1))), rel_tol=1e-9)
    finally:
        ctx.close()


def test_solar_wind_fills_box_at_density(lib):
    """Drift only, 30 steps: the injected plasma fills the box behind its front
    with the upstream density (ppc per cell), bulk velocity -U and thermal
    spread sqrt(kT/m) across the flow."""
    cfg = box()
    ctx = empty_context(lib, cfg)
    try:
        ctx.step(30)
        cnt, p = ctx.download_particles(0)
    finally:
        ctx.close()
    per_cell = cnt.reshape(cfg.nz, cfg.ny, cfg.nx).mean(axis=(0, 1))
    # each step's 10 particles per wall cell enter at the wall face (x = 11 cells)
    # and drift 0.2 cells per step: the front is at 11 - 29 * 0.2 = 5.2 cells,
    # cells 6..9 hold 5 injection groups each (ppc), cell 10 holds 4.5 (the last
    # group is still on the face, in the injection layer 11)
    filled = per_cell[6:10]
    assert np.all(np.abs(filled / PPC - 1.0) < 0.05), filled
    assert abs(per_cell[10] / (0.9 * PPC) - 1.0) < 0.05, per_cell[10]
    vth = math.sqrt(abi.BOLTZMANN * T / abi.MASS_PROTON)
    assert abs(p[:, 3].mean() / -U - 1.0) < 0.02
    for a in (4, 5):
        assert abs(p[:, a].std() / vth - 1.0) < 0.05
        assert abs(p[:, a].mean()) < 0.05 * vth


def test_reproducible_by_seed(lib):
    cfg = box()
    out = []
    for seed in (1, 1, 2):
        ctx = empty_context(lib, cfg, seed=seed)
        try:
            ctx.step(3)
            out.append(ctx.download_particles(0)[1])
        finally:
            ctx.close()
    assert np.array_equal(out[0].view(np.uint64), out[1].view(np.uint64))
    assert out[0].shape != out[2].shape or not np.array_equal(out[0], out[2])


def test_fp32_form_injects_the_same_count(lib):
    cfg = box()
    ctx = empty_context(lib, cfg, path=abi.PATH_FP32)
    try:
        ctx.step(1)
        assert ctx.num_particles(0) == 10 * cfg.ny * cfg.nz
    finally:
        ctx.close()


def test_exact_path_refuses_sources(lib):
    cfg = box()
    ctx = empty_context(lib, cfg, path=abi.PATH_EXACT)
    try:
        with pytest.raises(abi.RhError):
            ctx.step(1)
    finally:
        ctx.close()


def exo_box():
    """A planet of 500 km radius at the centre of a closed box of 24^3 cells of
    100 km, an O+ species, an exponential neutral profile from 600 km."""
    pop = cf.Population(name="O+", mass=16.0, charge=1.0, density=0.0, velocity=(0.0, 0.0, 0.0),
                        temperature=1e3, ppc=1.0, accelerate=False, upstream=False)
    return cf.Config(nx=24, ny=24, nz=24, x_min=-1.2e6, y_min=-1.2e6, z_min=-1.2e6, dx=100e3,
                     periodic=(0, 0, 0), dt=0.05, populations=[pop], name="exo_box")


def test_rejected_source_set_keeps_the_previous_one(lib):
    """rhgpu_set_injectors replaces the whole source set only when every
    source is accepted: a set whose second source names no species is
    refused, and the solar wind set before it keeps injecting the same
    particles as an untouched context."""
    cfg = box()
    counts = []
    for bad_call in (False, True):
        ctx = empty_context(lib, cfg)
        try:
            if bad_call:
                good = cf.solar_wind_injectors(cfg, seed=1)[0]
                bad = abi.Injector(species=7, type=abi.INJECT_SOLARWIND, density=N0, temperature=T,
                                   macroparticles_per_cell=PPC, seed=2)
                with pytest.raises(abi.RhError):
                    ctx.set_injectors([good, bad])
            ctx.step(2)
            cnt, p = ctx.download_particles(0)
            counts.append((cnt, p))
        finally:
            ctx.close()
    assert counts[0][1].shape[0] > 0
    assert np.array_equal(counts[0][0], counts[1][0])
    assert np.array_equal(counts[0][1], counts[1][1])


def exo_injector(shadow=1.0, seed=5):
    j = abi.Injector(species=0, type=abi.INJECT_EXOSPHERE, temperature=1e3, seed=seed,
                     profile=abi.NEUTRAL_PROFILES["Exponential"], n_components=1, r0=600e3,
                     exobase_radius=600e3, shadow_radius=600e3, ionization_rate=1e-6,
                     ionization_factor_shadow=shadow, total_production_rate=-1.0,
                     macroparticles_per_cell_relative=1.0, upstream_macro_ratio=400.0)
    j.n0[0] = 1e12
    j.H0[0] = 200e3
    return j


def test_exosphere_source(lib):
    """InjectorExosphere: about macroparticles_per_cell_relative *
    upstream_macro_ratio = 400 new ions per step (fewer: those drawn below the
    exobase in cells that straddle it are dropped, as in the reference), all
    above the exobase, concentrated within a few scale heights, none in
    the shadow when its factor is zero, weight total rate * dt / 400."""
    cfg = exo_box()
    grid, _ = cf.initial_state(cfg)
    for shadow in (1.0, 0.0):
        ctx = abi.Context(lib, cf.params(cfg), cf.species(cfg), capacity=[100000])
        try:
            ctx.set_path(abi.PATH_FAST)
            ctx.upload_array("faceB", grid["faceB"])
            ctx.upload_array("cellB", grid["cellB"])
            ctx.upload_array("nodeEta", grid["nodeEta"])
            ctx.upload_cell_flags(grid["flags"])
            ctx.upload_particles(0, np.zeros(cfg.ncells, dtype=np.uint32), np.zeros((0, 7)))
            ctx.set_injectors([exo_injector(shadow)])
            ctx.step(1)
            cnt, p = ctx.download_particles(0)
            ic = ctx.injection_counters()[0]
        finally:
            ctx.close()
        cell = np.repeat(np.arange(cfg.ncells), cnt.astype(np.int64))
        i, j, k = cell % 24, (cell // 24) % 24, cell // 576
        xg = -1.2e6 + i * 100e3 + p[:, 0]
        yg = -1.2e6 + j * 100e3 + p[:, 1]
        zg = -1.2e6 + k * 100e3 + p[:, 2]
        r = np.sqrt(xg ** 2 + yg ** 2 + zg ** 2)
        assert np.all(r >= 600e3)
        assert ic["macroparticles"] == p.shape[0]
        if shadow == 1.0:
            assert 300 <= p.shape[0] <= 440, p.shape[0]
            assert np.mean(r < 1.2e6) > 0.8
            w = p[0, 6]
            assert math.isclose(ic["weight"], p.shape[0] * w, rel_tol=1e-12)
            vth = math.sqrt(abi.BOLTZMANN * 1e3 / (16 * abi.MASS_PROTON))
            assert abs(p[:, 3:6].std() / vth - 1.0) < 0.15
        else:
            xc = -1.2e6 + (i + 0.5) * 100e3
            rc2 = (-1.2e6 + (j + 0.5) * 100e3) ** 2 + (-1.2e6 + (k + 0.5) * 100e3) ** 2
            assert not np.any((xc < 0) & (rc2 < 600e3 ** 2))
            assert p.shape[0] > 0


# the planetary neutral models of neutral_profiles.h:79-214 restated in numpy
# (constants as the library states them: IAU radii and masses, 15.999 u oxygen)
VENUS_R, VENUS_M, M_O, MERCURY_R = 6051.8e3, 4.8675e24, 15.999 * 1.66053906660e-27, 2439.7e3


def np_venus_h(x, y, z):
    r = np.sqrt(x * x + y * y + z * z)
    chi = np.arccos(x / r)
    exoR = VENUS_R + 170e3
    GM = abi.GRAVITY * VENUS_M
    bd, bn = GM * abi.MASS_PROTON / (abi.BOLTZMANN * 285), GM * abi.MASS_PROTON / (abi.BOLTZMANN * 110)
    th = (1 - chi / np.pi) * 1.32e11 * np.exp(-bd * (1 / exoR - 1 / r)) + (chi / np.pi) * 2.59e12 * np.exp(-bn * (1 / exoR - 1 / r))
    h = [np.exp(a1 * r + a2 + a3 / r) for a1, a2, a3 in ((-6.2625e-5 / 1e3, 15.4817, 3.6414e7),
                                                         (-8.4607e-5 / 1e3, 15.9944, 2.9743e7),
                                                         (-6.2309e-5 / 1e3, 15.2723, 4.3781e7))]
    u = chi / (np.pi / 2)
    hot = np.where(chi <= np.pi / 2, (1 - u) * h[0] + u * h[1], (2 - u) * h[1] + (u - 1) * h[2])
    return th + hot


def np_venus_o(x, y, z):
    r = np.sqrt(x * x + y * y + z * z)
    chi = np.arccos(x / r)
    GMm = abi.GRAVITY * VENUS_M * M_O
    r0d, r0n = VENUS_R + 200e3, VENUS_R + 300e3
    nd = np.where(r < r0d, 0.0, 7.5e10 * np.exp(-GMm / (abi.BOLTZMANN * 6400) * (1 / r0d - 1 / r)))
    nn = np.where(r < r0n, 0.0, 2e9 * np.exp(-GMm / (abi.BOLTZMANN * 4847) * (1 / r0n - 1 / r)))
    return (1 - chi / np.pi) * nd + (chi / np.pi) * nn


def np_mercury_na(x, y, z):
    r = np.sqrt(x * x + y * y + z * z)
    d = np.pi / 180
    lat, lon = np.arctan2(z, np.sqrt(x * x + y * y)), np.arctan2(y, x)

    def lobe(n0, hr, ht, la, lo):
        dth = np.arccos(np.sin(lat) * np.sin(la) + np.cos(lat) * np.cos(la) * np.cos(lo - lon))
        return n0 * np.exp(-(r - MERCURY_R) / hr) * np.exp(-(dth / ht) ** 2)
    s = 7.84e6 * np.exp(-(r - MERCURY_R) / 431e3)
    for args in ((8.86e9, 100e3, 15 * d, 0, 0), (5.67e6, 748e3, 15 * d, 80 * d, 0), (5.67e6, 748e3, 15 * d, -80 * d, 0),
                 (5.67e6, 748e3, 10 * d, 15 * d, np.pi), (5.67e6, 748e3, 10 * d, -15 * d, np.pi),
                 (4.06e10, 232e3, 20 * d, 50 * d, 0), (4.06e10, 232e3, 20 * d, -50 * d, 0)):
        s = s + lobe(*args)
    return (MERCURY_R / r) ** 2 * s


@pytest.mark.parametrize("name,fn,R", [("VenusHydrogen", np_venus_h, VENUS_R), ("VenusOxygen", np_venus_o, VENUS_R),
                                       ("MercurySodiumExner20", np_mercury_na, MERCURY_R)])
def test_planetary_neutral_models(lib, name, fn, R):
    """getNeutralDensity's planetary models (neutral_profiles.h:79-214) on the
    GPU against numpy at points from the surface to 5 planet radii, all
    directions."""
    rng = np.random.default_rng(11)
    n = 20000
    u = rng.normal(size=(n, 3))
    u /= np.linalg.norm(u, axis=1, keepdims=True)
    xyz = u * rng.uniform(1.0, 5.0, size=(n, 1)) * R
    j = abi.Injector(type=abi.INJECT_EXOSPHERE, profile=abi.NEUTRAL_PROFILES[name])
    got = abi.neutral_density(lib, j, 16 * abi.MASS_PROTON, xyz)
    want = fn(xyz[:, 0], xyz[:, 1], xyz[:, 2])
    assert np.all(want >= 0) and want.max() > 0
    np.testing.assert_allclose(got, want, rtol=1e-10, atol=1e-10 * want.max())


def iono_injector(profile, noon=1.0, night=0.1, seed=9):
    return abi.Injector(species=0, type=abi.INJECT_IONOSPHERE, temperature=1e3, seed=seed,
                        emission_radius=650e3, noon_factor=noon, night_factor=night,
                        iono_profile=abi.IONO_PROFILES[profile], total_production_rate=1e24,
                        macroparticles_per_cell_relative=1.0, upstream_macro_ratio=400.0)


@pytest.mark.parametrize("profile", ["ionoCosSzaDayConstantNight", "ionoConstant"])
def test_ionosphere_source(lib, profile):
    """InjectorIonosphere: about macroparticles_per_cell_relative *
    upstream_macro_ratio = 400 new ions per step, in the cells the emission
    shell r = 650 km crosses, moving outward, weight total rate * dt / 400; the
    cos(SZA)-day / constant-night profile (noon 1, night 0.1) puts most of them
    on the dayside, the constant one about half."""
    cfg = exo_box()
    grid, _ = cf.initial_state(cfg)
    ctx = abi.Context(lib, cf.params(cfg), cf.species(cfg), capacity=[100000])
    try:
        ctx.set_path(abi.PATH_FAST)
        ctx.upload_array("faceB", grid["faceB"])
        ctx.upload_array("cellB", grid["cellB"])
        ctx.upload_array("nodeEta", grid["nodeEta"])
        ctx.upload_cell_flags(grid["flags"])
        ctx.upload_particles(0, np.zeros(cfg.ncells, dtype=np.uint32), np.zeros((0, 7)))
        ctx.set_injectors([iono_injector(profile)])
        ctx.step(1)
        cnt, p = ctx.download_particles(0)
        ic = ctx.injection_counters()[0]
    finally:
        ctx.close()
    cell = np.repeat(np.arange(cfg.ncells), cnt.astype(np.int64))
    i, j, k = cell % 24, (cell // 24) % 24, cell // 576
    xg = -1.2e6 + i * 100e3 + p[:, 0]
    yg = -1.2e6 + j * 100e3 + p[:, 1]
    zg = -1.2e6 + k * 100e3 + p[:, 2]
    r = np.sqrt(xg ** 2 + yg ** 2 + zg ** 2)
    assert 320 <= p.shape[0] <= 480, p.shape[0]
    assert ic["macroparticles"] == p.shape[0]
    assert np.all(np.abs(r - 650e3) < math.sqrt(3) * 100e3 + 0.05 * 3.0 * 900e3 * 0.05)
    # outward at injection; one push of 0.05 s at thermal speeds keeps it so for nearly all
    assert np.mean(p[:, 3] * xg + p[:, 4] * yg + p[:, 5] * zg > 0) > 0.95
    assert math.isclose(p[0, 6], 1e24 * cfg.dt / 400.0, rel_tol=1e-12)
    day = np.mean(xg > 0)
    if profile == "ionoConstant":
        assert 0.4 < day < 0.6
    else:
        assert day > 0.75


def test_chapman_ionosphere_source(lib):
    """InjectorChapmanIonosphere: about 400 new ions per step in a thin
    Chapman layer around the emission radius (scale height k_B T / (m g_Mars),
    here about 21 km for O+ at 150 K), moving outward, mostly on the dayside
    (noon 1, night 0.1), weight total rate * dt / 400, and no device error
    from the position redraws."""
    cfg = exo_box()
    grid, _ = cf.initial_state(cfg)
    j = abi.Injector(species=0, type=abi.INJECT_CHAPMAN_IONOSPHERE, temperature=150.0, seed=13,
                     emission_radius=650e3, noon_factor=1.0, night_factor=0.1, total_production_rate=1e24,
                     macroparticles_per_cell_relative=1.0, upstream_macro_ratio=400.0)
    ctx = abi.Context(lib, cf.params(cfg), cf.species(cfg), capacity=[100000])
    try:
        ctx.set_path(abi.PATH_FAST)
        ctx.upload_array("faceB", grid["faceB"])
        ctx.upload_array("cellB", grid["cellB"])
        ctx.upload_array("nodeEta", grid["nodeEta"])
        ctx.upload_cell_flags(grid["flags"])
        ctx.upload_particles(0, np.zeros(cfg.ncells, dtype=np.uint32), np.zeros((0, 7)))
        ctx.set_injectors([j])
        ctx.step(1)
        assert ctx.device_errors() == 0
        cnt, p = ctx.download_particles(0)
        ic = ctx.injection_counters()[0]
    finally:
        ctx.close()
    cell = np.repeat(np.arange(cfg.ncells), cnt.astype(np.int64))
    i, jj, k = cell % 24, (cell // 24) % 24, cell // 576
    xg = -1.2e6 + i * 100e3 + p[:, 0]
    yg = -1.2e6 + jj * 100e3 + p[:, 1]
    zg = -1.2e6 + k * 100e3 + p[:, 2]
    r = np.sqrt(xg ** 2 + yg ** 2 + zg ** 2)
    assert 320 <= p.shape[0] <= 480, p.shape[0]
    assert ic["macroparticles"] == p.shape[0]
    assert np.all(np.abs(r - 650e3) < 250e3), (r.min(), r.max())
    assert np.mean(np.abs(r - 650e3) < 120e3) > 0.9
    assert np.all(p[:, 3] * xg + p[:, 4] * yg + p[:, 5] * zg >= 0)
    assert math.isclose(p[0, 6], 1e24 * cfg.dt / 400.0, rel_tol=1e-12)
    assert np.mean(xg > 0) > 0.8
