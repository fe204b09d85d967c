"""Run configuration and initial state (host side).

Restates the parts of RHybrid's initialisation that feed the hot path:
  * parameter derivation of userLateInitialization (src/user.cpp:356-1807):
    squared radii and speeds, resistivity unit conversion, minimum charge
    density relative to the upstream one, electron-pressure coefficient,
    Gaussian smoothing coefficients;
  * per-cell flags and the node resistivity table (src/user.cpp:1883-1941,
    src/resistivity.h:29-215);
  * the initial magnetic field on faces and cells (src/user.cpp:2107-2144,
    src/magnetic_field.h);
  * uniform particle populations (InjectorUniform, src/particle_injector.cpp:177-260)
    from a seeded SplitMix64 stream (Corsair's RNG is not vendored).

A `Config` mirrors the .cfg sections the hot path reads: [LogicallyCartesian],
[Simulation] dt, [Hybrid], [IMF], [IntrinsicB], [ElectronPressure],
[Resistivity], [Constraints] and one section per population.
"""
from __future__ import annotations

import dataclasses
import math
from dataclasses import dataclass, field
from typing import List, Optional, Sequence

import numpy as np

from . import abi


@dataclass
class Population:
    """A [population] section plus its UniformInjector parameters."""
    name: str = "H+"
    mass: float = 1.0            # mass_unit = MASS_PROTON
    charge: float = 1.0          # charge_unit = CHARGE_ELEMENTARY
    obstacle: float = -100.0     # particle obstacle radius [m]
    accumulate: bool = True
    accelerate: bool = True
    density: float = 5e6         # [m^-3]
    velocity: Sequence[float] = (-400e3, 0.0, 0.0)
    temperature: float = 1e5     # [K]
    ppc: float = 20.0            # macroparticles_per_cell
    upstream: bool = True        # counts towards the upstream plasma parameters
    exosphere: Optional[dict] = None   # ExosphereInjector parameters of a planetary source
    ionosphere: Optional[dict] = None  # IonosphereInjector parameters of a planetary source
    flow_walls: Sequence[str] = ()     # FlowInjector inflow walls ("+x", "-x", ...)
    fill: bool = True                  # filled uniformly at the start (UniformInjector); sources fill the rest

    @property
    def q(self) -> float:
        return self.charge * abi.CHARGE_ELEMENTARY

    @property
    def m(self) -> float:
        return self.mass * abi.MASS_PROTON


@dataclass
class Config:
    # [LogicallyCartesian]
    nx: int = 32
    ny: int = 32
    nz: int = 32
    x_min: float = -1600e3
    y_min: float = -1600e3
    z_min: float = -1600e3
    dx: float = 100e3
    periodic: Sequence[int] = (1, 1, 1)
    # [Simulation]
    dt: float = 0.01
    t_initial: float = 0.0
    # [Hybrid]
    R_fieldObstacle: float = -100.0
    R_particleObstacle: float = -100.0
    fieldObstacleUe: Sequence[float] = (0.0, 0.0, 0.0)
    use_gravity: bool = False
    M_object: float = 0.0
    use_hall_term: bool = True
    # [IMF]
    imf: Sequence[float] = (0.0, 5e-9, 0.0)
    imf_boundary_cellB: Sequence[int] = (0, 0, 0, 0, 0, 0)
    imf_boundary_faceB: Sequence[int] = (0, 0, 0, 0, 0, 0)
    # [IntrinsicB]
    b_profile: str = "constantB"
    dipole_surface_B: float = 0.0
    dipole_surface_R: float = 0.0
    dipole_min_R: float = 0.0
    dipole_origin: Sequence[float] = (0.0, 0.0, 0.0)
    laminar_R: float = 0.0
    # [ElectronPressure]
    use_electron_pressure: bool = False
    electron_temperature: float = 0.0
    electron_gamma: int = 2
    R_zeroElectronPressure: float = -100.0
    # [Resistivity]
    resistivity_profile: str = "resistivityConstant"
    resistivity_unit: str = "Rm"
    resistivity_value: float = 6.0
    resistivity_R: float = 0.0
    resistivity_outer_cells: Sequence[int] = (0, 0, 0, 0, 0, 0)
    resistivity_outer_coeffs: Sequence[float] = (1, 1, 1, 1, 1, 1)
    # [Constraints]
    max_ion_velocity: float = 1500e3
    max_electron_velocity: float = 1500e3
    min_ion_charge_density_relative: float = 0.05
    max_electric_field: float = -100.0
    max_whistler_velocity: float = 1500e3
    initial_flow_throughs: float = -1.0
    electric_field_linear_smoothing_number: int = 0
    electric_field_smoothing_gauss_sigma: float = 0.0
    populations: List[Population] = field(default_factory=lambda: [Population()])
    seed: int = 6461674
    name: str = "custom"

    @property
    def ncells(self) -> int:
        return self.nx * self.ny * self.nz

    def replace(self, **kw) -> "Config":
        return dataclasses.replace(self, **kw)


# ---------------------------------------------------------------------------
# named configurations (workloads)

C_DOUBLE3 = abi.C.c_double * 3


def solar_wind_injectors(cfg: "Config", seed: int = 1) -> list:
    """One InjectorSolarWind per upstream population with a velocity along one
    axis, as the reference's .cfg files set the solar wind sources: density,
    temperature and macroparticles per cell of the population (weight
    n dx^3 / ppc, the uniform fill's weight)."""
    out = []
    for s, p in enumerate(cfg.populations):
        v = tuple(float(x) for x in p.velocity)
        if not p.upstream or sum(1 for x in v if x != 0.0) != 1 or p.temperature <= 0 or p.ppc <= 0:
            continue
        out.append(abi.Injector(species=s, type=abi.INJECT_SOLARWIND, velocity=(C_DOUBLE3)(*v), density=p.density,
                                temperature=p.temperature, macroparticles_per_cell=p.ppc, inflow_walls=0,
                                reserved=0, seed=seed * 1000003 + s))
    return out


def upstream_macro_ratio(cfg: "Config") -> float:
    """Hybrid::upstreamMacroPleRatio: the solar wind macroparticles injected per
    step over the macroparticles per cell, of the first solar wind population
    (particle_injector.cpp:690-712): |U| dt / dx times the wall cells."""
    for p in cfg.populations:
        v = [float(x) for x in p.velocity]
        if not p.upstream or sum(1 for x in v if x != 0.0) != 1 or p.ppc <= 0:
            continue
        ax = next(a for a in range(3) if v[a] != 0.0)
        dims, per = (cfg.nx, cfg.ny, cfg.nz), cfg.periodic
        wall = 1
        for a in range(3):
            if a != ax:
                wall *= dims[a] if per[a] else dims[a] - 2
        return abs(v[ax]) * cfg.dt / cfg.dx * wall
    return 0.0


def source_injectors(cfg: "Config", seed: int = 1) -> list:
    """Every particle source of the configuration: the solar wind injectors,
    one InjectorExosphere per population with exosphere parameters, one
    InjectorFlow per population with inflow walls and one InjectorIonosphere
    (or InjectorChapmanIonosphere) per population with ionosphere parameters."""
    out = solar_wind_injectors(cfg, seed)
    ratio = upstream_macro_ratio(cfg)
    for s, p in enumerate(cfg.populations):
        e = p.exosphere
        if not e:
            continue
        j = abi.Injector(species=s, type=abi.INJECT_EXOSPHERE, temperature=p.temperature, seed=seed * 1000003 + s,
                         profile=abi.NEUTRAL_PROFILES[e["profile"]], n_components=len(e["n0"]), r0=e["r0"],
                         exobase_radius=e["exobase_radius"], shadow_radius=e["shadow_radius"],
                         ionization_rate=e.get("ionization_rate", -1.0),
                         ionization_factor_shadow=e.get("ionization_factor_shadow", 1.0),
                         total_production_rate=e.get("total_production_rate", -1.0),
                         macroparticles_per_cell_relative=e.get("macroparticles_per_cell_relative", 1.0),
                         upstream_macro_ratio=ratio)
        j.gm_object = abi.GRAVITY * cfg.M_object
        for k, n0 in enumerate(e["n0"]):
            j.n0[k] = n0
            for key in ("H0", "T0", "k0"):
                vals = e.get(key) or []
                if k < len(vals):
                    getattr(j, key)[k] = vals[k]
        out.append(j)
    for s, p in enumerate(cfg.populations):
        if not p.flow_walls or p.ppc <= 0 or p.density <= 0:
            continue
        mask = sum(abi.WALLS[w] for w in p.flow_walls)
        out.append(abi.Injector(species=s, type=abi.INJECT_FLOW, velocity=(C_DOUBLE3)(*[float(x) for x in p.velocity]),
                                density=p.density, temperature=p.temperature, macroparticles_per_cell=p.ppc,
                                inflow_walls=mask, reserved=0, seed=seed * 1000003 + 700 + s))
    for s, p in enumerate(cfg.populations):
        o = p.ionosphere
        if not o:
            continue
        chapman = o["profile"] == "Chapman"
        out.append(abi.Injector(species=s, type=abi.INJECT_CHAPMAN_IONOSPHERE if chapman else abi.INJECT_IONOSPHERE,
                                temperature=p.temperature,
                                seed=seed * 1000003 + 500 + s, emission_radius=o["emission_radius"],
                                noon_factor=o["noon"], night_factor=o["night"],
                                iono_profile=0 if chapman else abi.IONO_PROFILES[o["profile"]],
                                total_production_rate=o["total_production_rate"],
                                macroparticles_per_cell_relative=o.get("macroparticles_per_cell_relative", 1.0),
                                upstream_macro_ratio=ratio))
    return out


def config_empty_box(nx=32, ny=32, nz=32, ppc=20.0) -> Config:
    """Plain FP64 periodic empty box: cell 100 km, one H+ species, n=5e6 m^-3,
    drift Vx=-400 km/s, Maxwellian T=1e5 K, B=(0,5,0) nT uniform, 20
    particles/cell, dt=0.01 s. Constraints and resistivity as in
    examples/empty_box_periodic.cfg."""
    half = 0.5 * nx * 100e3
    return Config(nx=nx, ny=ny, nz=nz, x_min=-half, y_min=-0.5 * ny * 100e3, z_min=-0.5 * nz * 100e3,
                  dx=100e3, periodic=(1, 1, 1), dt=0.01,
                  populations=[Population(name="H+", density=5e6, velocity=(-400e3, 0, 0),
                                          temperature=1e5, ppc=ppc)],
                  name=f"empty_box_{nx}x{ny}x{nz}_ppc{ppc:g}")


def config_mars(nx=120, ny=160, nz=160, ppc=30.0, dx=300e3, exosphere=False) -> Config:
    """Plain FP64 Mars-like obstacle: cell 300 km, absorbing sphere r=3390 km,
    solar wind H+ (n=2e6 m^-3, 30 ppc) + He++ (4% of n, 1.5 ppc), V=-450 km/s,
    T=1e5 K, IMF (0,3,0) nT, closed walls with IMF on the +x wall, dt=0.05 s,
    superconducting-sphere resistivity, electron pressure on. With exosphere,
    a third population exoO+ starts empty and is fed by the exponential O+
    exosphere source of examples/mars.cfg ([exoO+], [injector_exoO+]);
    `source_injectors` gives it and the solar wind inflow."""
    R = 3390e3
    Lx, Ly, Lz = nx * dx, ny * dx, nz * dx
    pops = [
        Population(name="swH+", mass=1.0, charge=1.0, obstacle=R, density=2e6,
                   velocity=(-450e3, 0, 0), temperature=1e5, ppc=ppc),
        Population(name="swHe++", mass=3.9737, charge=2.0, obstacle=R, density=0.04 * 2e6,
                   velocity=(-450e3, 0, 0), temperature=1e5, ppc=ppc / 20.0),
    ]
    if exosphere:
        pops.append(Population(name="exoO+", mass=15.883821896403, charge=1.0, obstacle=3590e3, density=0.0,
                               velocity=(0.0, 0.0, 0.0), temperature=6500.0, ppc=0.0, upstream=False,
                               exosphere={"profile": "Exponential", "r0": 3393.5e3,
                                          "n0": [5.23e9, 9.76e8, 3.71e10], "H0": [626.2e3, 2790e3, 88.47e3],
                                          "exobase_radius": 3790e3, "shadow_radius": 3390e3,
                                          "ionization_factor_shadow": 0.0, "total_production_rate": 0.156e24,
                                          "macroparticles_per_cell_relative": 1.0}))
    return Config(nx=nx, ny=ny, nz=nz, x_min=-0.5 * Lx, y_min=-0.5 * Ly, z_min=-0.5 * Lz, dx=dx,
                  periodic=(0, 0, 0), dt=0.05, R_fieldObstacle=R, R_particleObstacle=R,
                  imf=(0.0, 3e-9, 0.0), imf_boundary_cellB=(1, 0, 0, 0, 0, 0),
                  imf_boundary_faceB=(1, 0, 0, 0, 0, 0),
                  use_electron_pressure=True, electron_temperature=1e5, electron_gamma=2,
                  R_zeroElectronPressure=R,
                  resistivity_profile="resistivitySuperConductingSphere", resistivity_unit="Rm",
                  resistivity_value=6.0, resistivity_R=R,
                  max_ion_velocity=1500e3, max_electron_velocity=1500e3,
                  min_ion_charge_density_relative=0.05, max_whistler_velocity=1500e3,
                  populations=pops, name=f"mars_{nx}x{ny}x{nz}_ppc{ppc:g}" + ("_exoO+" if exosphere else ""))


def config_mercury(nx=320, ny=320, nz=320, ppc=40.0, dx=100e3) -> Config:
    """Mercury-like dipole: cell 100 km, a dipole of 190 nT at r = 2440 km
    (surface field, southward as in examples/mercury.cfg) plus the IMF Bx
    draped around a 1800 km sphere (translateDipoleBAndLaminarFlowAroundSphereBx,
    src/magnetic_field.h:182-185), absorbing sphere r = 2439.7 km, solar wind
    H+ n = 3e7 m^-3 at 40 ppc, V = -400 km/s. The box puts the planet at 5/8 of
    x (more room downstream), as the example does. The rest follows
    examples/mercury.cfg: T = 1.7e5 K, IMF (2, 0, -10) nT on the +x wall,
    electron pressure 2.26e5 K (gamma 2), superconducting-core resistivity
    (Rm 6 within 1800 km, 10x on the +y outer cells), constraints 4000 km/s
    and E 0.0906 V/m, dt = 0.02 s, no gravity."""
    R = 2439.7e3
    Lx, Ly, Lz = nx * dx, ny * dx, nz * dx
    pops = [Population(name="swH+", mass=1.0, charge=1.0, obstacle=R, density=3e7,
                       velocity=(-400e3, 0, 0), temperature=1.7e5, ppc=ppc)]
    return Config(nx=nx, ny=ny, nz=nz, x_min=-0.625 * Lx, y_min=-0.5 * Ly, z_min=-0.5 * Lz, dx=dx,
                  periodic=(0, 0, 0), dt=0.02, R_fieldObstacle=R, R_particleObstacle=R,
                  imf=(2e-9, 0.0, -10e-9), imf_boundary_cellB=(1, 0, 0, 0, 0, 0),
                  imf_boundary_faceB=(1, 0, 0, 0, 0, 0),
                  b_profile="translateDipoleBAndLaminarFlowAroundSphereBx", laminar_R=1800e3,
                  dipole_surface_B=-190e-9, dipole_surface_R=2440e3, dipole_min_R=1000e3,
                  dipole_origin=(0.0, 0.0, 0.0),
                  use_electron_pressure=True, electron_temperature=2.26e5, electron_gamma=2,
                  R_zeroElectronPressure=-100.0,
                  resistivity_profile="resistivitySuperConductingSphere", resistivity_unit="Rm",
                  resistivity_value=6.0, resistivity_R=1800e3,
                  resistivity_outer_cells=(0, 4, 0, 0, 0, 0), resistivity_outer_coeffs=(1, 10, 1, 1, 1, 1),
                  max_ion_velocity=4000e3, max_electron_velocity=4000e3,
                  min_ion_charge_density_relative=0.05, max_electric_field=0.0906,
                  max_whistler_velocity=4000e3, populations=pops,
                  name=f"mercury_{nx}x{ny}x{nz}_ppc{ppc:g}")


# ---------------------------------------------------------------------------
# parameter derivation (src/user.cpp:356-1807)

def upstream(cfg: Config):
    """Upstream ion charge density, electron density and bulk speed from the
    upstream populations (diagnostics.h:80-96: rhoq = sum n*q, ne = rhoq/e)."""
    rhoq = 0.0
    U = 0.0
    for p in cfg.populations:
        if not p.upstream:
            continue
        rhoq += p.density * p.q
        if U == 0.0:
            U = math.sqrt(sum(v * v for v in p.velocity))
    return rhoq, rhoq / abi.CHARGE_ELEMENTARY, U


def resistivity_eta(cfg: Config) -> float:
    """setResistivityProfile unit conversion (src/resistivity.h:63-99)."""
    _, _, U = upstream(cfg)
    grid_unit = abi.PERMEABILITY * cfg.dx * cfg.dx / cfg.dt
    v, u = cfg.resistivity_value, cfg.resistivity_unit
    if u == "SI":
        return v
    if u == "grid":
        return v * grid_unit
    if u == "td":
        return (1.0 / v) * grid_unit
    if u == "Rm":
        return (1.0 / v) * abi.PERMEABILITY * cfg.dx * U
    if u == "URm":
        return v * abi.PERMEABILITY * cfg.dx
    raise ValueError(f"unknown resistivity unit {u}")


def _gaussian(x: float, sigma: float) -> float:
    return math.exp(-0.5 * (x / sigma) ** 2) / (sigma * math.sqrt(2.0 * math.pi))


def params(cfg: Config) -> abi.Params:
    """Fills struct rhgpu_params as userLateInitialization leaves Hybrid::."""
    P = abi.Params()
    P.nx, P.ny, P.nz = cfg.nx, cfg.ny, cfg.nz
    for a in range(3):
        P.periodic[a] = int(cfg.periodic[a])
    P.x_min, P.y_min, P.z_min = cfg.x_min, cfg.y_min, cfg.z_min
    P.dx, P.dt, P.t_initial = cfg.dx, cfg.dt, cfg.t_initial
    rhoq, ne, U = upstream(cfg)
    P.use_hall = int(cfg.use_hall_term)
    P.use_gravity = int(cfg.use_gravity)
    P.GMdt = abi.GRAVITY * cfg.M_object * cfg.dt
    # electron pressure (user.cpp:1565-1601)
    if cfg.use_electron_pressure:
        Te = max(cfg.electron_temperature, 0.0)
        if cfg.electron_gamma == 1:
            P.isothermal_electrons = 1
            P.electron_pressure_coeff = abi.BOLTZMANN * Te / abi.CHARGE_ELEMENTARY
        elif cfg.electron_gamma == 2:
            P.isothermal_electrons = 0
            P.electron_pressure_coeff = (2.0 * abi.BOLTZMANN * Te / (ne * abi.CHARGE_ELEMENTARY ** 2)
                                         if ne > 0 else 0.0)
        else:
            raise ValueError("ElectronPressure.closure_gamma must be 1 or 2")
        P.use_electron_pressure = 1
    for l in range(3):
        P.field_obstacle_Ue[l] = cfg.fieldObstacleUe[l]
    # constraints (user.cpp:1737-1807)
    vmax_e = cfg.max_electron_velocity if cfg.max_electron_velocity >= 0 else 1e10
    P.max_electron_speed2 = vmax_e * vmax_e
    vmax_i = cfg.max_ion_velocity if cfg.max_ion_velocity >= 0 else 1e10
    if vmax_i > cfg.dx / cfg.dt:
        vmax_i = 0.9 * cfg.dx / cfg.dt
    P.max_ion_speed2 = vmax_i * vmax_i
    rmin = cfg.min_ion_charge_density_relative
    P.min_ion_charge_density = 0.0 if rmin < 0 else rmin * rhoq
    P.max_electric_field2 = cfg.max_electric_field ** 2 if cfg.max_electric_field > 0 else 0.0
    P.max_whistler_speed = cfg.max_whistler_velocity
    if U > 0 and cfg.initial_flow_throughs > 0:
        P.initial_flow_through_period = cfg.initial_flow_throughs * (cfg.nx * cfg.dx) / U
        P.use_initial_flow_through = 1
    else:
        P.initial_flow_through_period = -100.0
        P.use_initial_flow_through = 0
    P.n_linear_smoothings_nodeE = max(int(cfg.electric_field_linear_smoothing_number), 0)
    sig = cfg.electric_field_smoothing_gauss_sigma
    if sig > 0:
        C1, C2 = _gaussian(0.0, sig), _gaussian(1.0, sig)
        C3, C4 = _gaussian(math.sqrt(2.0), sig), _gaussian(math.sqrt(3.0), sig)
        Cs = 1.0 * C1 + 6.0 * C2 + 12.0 * C3 + 8.0 * C4
        P.use_gaussian_smoothing_nodeE = 1
        for i, v in enumerate((C1, C2, C3, C4)):
            P.gaussian_coeffs[i] = v / Cs
    for l in range(3):
        P.imf_B[l] = cfg.imf[l]
    for w in range(6):
        P.imf_boundary_cellB[w] = int(cfg.imf_boundary_cellB[w])
        P.imf_boundary_faceB[w] = int(cfg.imf_boundary_faceB[w])
    return P


def species(cfg: Config) -> List[abi.Species]:
    """struct Species per population (src/particle_species.cpp:38-107)."""
    out = []
    for p in cfg.populations:
        s = abi.Species()
        s.q, s.m = p.q, p.m
        s.R2_obstacle = p.obstacle * p.obstacle if p.obstacle > 0 else -1.0
        s.accumulate, s.accelerate = int(p.accumulate), int(p.accelerate)
        out.append(s)
    return out


# ---------------------------------------------------------------------------
# grid initial state

def cell_ijk(cfg: Config):
    n = np.arange(cfg.ncells, dtype=np.int64)
    return n % cfg.nx, (n // cfg.nx) % cfg.ny, n // (cfg.nx * cfg.ny)


def block_origin(cfg: Config):
    """Minimum corner of every cell: x_min + i*dx."""
    i, j, k = cell_ijk(cfg)
    return (cfg.x_min + i.astype(np.float64) * cfg.dx,
            cfg.y_min + j.astype(np.float64) * cfg.dx,
            cfg.z_min + k.astype(np.float64) * cfg.dx)


def _eta_at(cfg: Config, x, y, z):
    """getResistivity (src/resistivity.h:29-62,212) for the constant and
    superconducting-sphere profiles."""
    eta = resistivity_eta(cfg)
    if cfg.resistivity_profile == "resistivityConstant":
        return np.full_like(x, eta)
    if cfg.resistivity_profile == "resistivitySuperConductingSphere":
        r2 = x * x + y * y + z * z
        R2 = cfg.resistivity_R * cfg.resistivity_R
        return np.where(r2 < R2, 0.0, eta)
    raise ValueError(f"resistivity profile {cfg.resistivity_profile} not supported")


def _initial_B(cfg: Config, x, y, z):
    """setInitialB (src/magnetic_field.h:257-260) for constantB, constantBx,
    translateDipoleB (:98-111), laminarFlowAroundSphereBx (:44-54) and their
    sum translateDipoleBAndLaminarFlowAroundSphereBx (:182-185)."""
    Bx = np.zeros_like(x)
    By = np.zeros_like(x)
    Bz = np.zeros_like(x)
    prof = cfg.b_profile
    known = ("constantB", "constantBx", "translateDipoleB", "laminarFlowAroundSphereBx",
             "translateDipoleBAndLaminarFlowAroundSphereBx")
    if prof not in known:
        raise ValueError(f"IntrinsicB profile {prof} not supported")
    if prof in ("constantB", "constantBx"):
        Bx = Bx + cfg.imf[0]
        if prof == "constantB":
            By = By + cfg.imf[1]
            Bz = Bz + cfg.imf[2]
    if prof in ("translateDipoleB", "translateDipoleBAndLaminarFlowAroundSphereBx"):
        x1, y1, z1 = x - cfg.dipole_origin[0], y - cfg.dipole_origin[1], z - cfg.dipole_origin[2]
        r2 = x1 * x1 + y1 * y1 + z1 * z1
        rr = np.sqrt(r2)
        r5 = (r2 * r2) * rr
        mom = 3.0 * cfg.dipole_surface_B * cfg.dipole_surface_R ** 3
        with np.errstate(divide="ignore", invalid="ignore"):
            coeff = mom / r5
            ok = r2 >= cfg.dipole_min_R ** 2
            Bx = np.where(ok, Bx + coeff * x1 * z1, Bx)
            By = np.where(ok, By + coeff * y1 * z1, By)
            Bz = np.where(ok, Bz + coeff * (z1 * z1 - r2 / 3.0), Bz)
    if prof in ("laminarFlowAroundSphereBx", "translateDipoleBAndLaminarFlowAroundSphereBx"):
        # IMF Bx draped around a sphere, nothing added inside it (magnetic_field.h:44-54)
        r2 = x * x + y * y + z * z
        R3 = cfg.laminar_R ** 3
        with np.errstate(divide="ignore", invalid="ignore"):
            r = np.sqrt(r2)
            coeff = -1.5 * cfg.imf[0] * R3 * x / r ** 5
            ok = r2 >= cfg.laminar_R ** 2
            Bx = np.where(ok, Bx + (coeff * x + cfg.imf[0] * (1 + 0.5 * (R3 / r ** 3))), Bx)
            By = np.where(ok, By + coeff * y, By)
            Bz = np.where(ok, Bz + coeff * z, Bz)
    return Bx, By, Bz


def init_grid(cfg: Config):
    """Returns the arrays userLateInitialization fills before the first step:
    faceB, cellB (initial field), nodeEta, and the cell flag bytes."""
    dx = cfg.dx
    xb, yb, zb = block_origin(cfg)
    xc, yc, zc = xb + 0.5 * dx, yb + 0.5 * dx, zb + 0.5 * dx
    xn, yn, zn = xb + 1.0 * dx, yb + 1.0 * dx, zb + 1.0 * dx
    R2f = cfg.R_fieldObstacle ** 2 if cfg.R_fieldObstacle > 0 else -1.0
    # Hybrid::R2_particleObstacle (user.cpp:1925-1926)
    R2p = cfg.R_particleObstacle ** 2 if cfg.R_particleObstacle > 0 else -1.0
    R2z = cfg.R_zeroElectronPressure ** 2 if cfg.R_zeroElectronPressure > 0 else 0.0
    r2 = xc * xc + yc * yc + zc * zc
    flags = np.zeros(cfg.ncells, dtype=np.uint8)
    flags |= np.where(r2 < R2f, abi.FLAG_INNER_FIELD, 0).astype(np.uint8)
    rp2 = (np.sqrt(r2) - 0.5 * math.sqrt(3) * dx) ** 2
    flags |= np.where(rp2 < R2p, abi.FLAG_INNER_PARTICLE, 0).astype(np.uint8)
    flags |= np.where(rp2 < R2z, abi.FLAG_INNER_CELLEP, 0).astype(np.uint8)
    rn2 = xn * xn + yn * yn + zn * zn
    flags |= np.where(rn2 < R2f, abi.FLAG_INNER_NODE, 0).astype(np.uint8)
    eta = _eta_at(cfg, xn, yn, zn)
    x_max = cfg.x_min + cfg.nx * dx
    y_max = cfg.y_min + cfg.ny * dx
    z_max = cfg.z_min + cfg.nz * dx
    oc, co = cfg.resistivity_outer_cells, cfg.resistivity_outer_coeffs
    base = _eta_at(cfg, xn, yn, zn)
    for cond, c in (
        ((oc[0] > 0) & (xn > (x_max - dx * oc[0] * 0.99)), co[0]),
        ((oc[1] > 0) & (xn < (cfg.x_min + dx * oc[1] * 1.01)), co[1]),
        ((oc[2] > 0) & (yn > (y_max - dx * oc[2] * 0.99)), co[2]),
        ((oc[3] > 0) & (yn < (cfg.y_min + dx * oc[3] * 1.01)), co[3]),
        ((oc[4] > 0) & (zn > (z_max - dx * oc[4] * 0.99)), co[4]),
        ((oc[5] > 0) & (zn < (cfg.z_min + dx * oc[5] * 1.01)), co[5]),
    ):
        eta = np.where(cond, base * c, eta)
    faceB = np.zeros((cfg.ncells, 3))
    faceB[:, 0] = _initial_B(cfg, xb + 1.0 * dx, yb + 0.5 * dx, zb + 0.5 * dx)[0]
    faceB[:, 1] = _initial_B(cfg, xb + 0.5 * dx, yb + 1.0 * dx, zb + 0.5 * dx)[1]
    faceB[:, 2] = _initial_B(cfg, xb + 0.5 * dx, yb + 0.5 * dx, zb + 1.0 * dx)[2]
    cellB = np.stack(_initial_B(cfg, xc, yc, zc), axis=1)
    return {"faceB": faceB, "cellB": cellB, "nodeEta": eta, "flags": flags}


# ---------------------------------------------------------------------------
# uniform populations (InjectorUniform, src/particle_injector.cpp:177-260)

EPS_CELL = 1.0e-4   # particle_injector.cpp:31
_GOLDEN = np.uint64(0x9E3779B97F4A7C15)


def splitmix64(seed: int, count: int, stream: int = 0) -> np.ndarray:
    """`count` outputs of SplitMix64 started at seed + stream*2^40 (own
    seeded generator; counter-based so it vectorises)."""
    with np.errstate(over="ignore"):
        s = (np.uint64(seed) + np.uint64(stream) * np.uint64(1 << 40)
             + (np.arange(1, count + 1, dtype=np.uint64) * _GOLDEN))
        z = s
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        z = z ^ (z >> np.uint64(31))
    return z


def uniform01(seed: int, count: int, stream: int) -> np.ndarray:
    """Uniform doubles in [0,1) with 53 random bits."""
    return (splitmix64(seed, count, stream) >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)


def uniform_population(cfg: Config, s: int, seed: Optional[int] = None, cell_mask=None):
    """Particles of population s filling every cell (or the cells where
    cell_mask is true): positions uniform in the central (1-1e-4) of the cell,
    velocity U + vth*N(0,1) per component (Box-Muller), weight n*dV/ppc.
    Returns (counts[ncells] uint32, particles[n,7] float64) grouped by cell."""
    p = cfg.populations[s]
    seed = cfg.seed if seed is None else seed
    N = cfg.ncells
    if not p.fill:
        return np.zeros(N, dtype=np.uint32), np.zeros((0, 7), dtype=np.float64)
    dx = cfg.dx
    dV = dx * dx * dx
    ppc = p.ppc
    w = p.density * dV / ppc if (ppc > 0 and p.density > 0) else 0.0
    vth = math.sqrt(abi.BOLTZMANN * p.temperature / p.m) if p.temperature > 0 else 0.0
    f = math.floor(ppc)
    # probRound (particle_injector.cpp:41-48)
    r = uniform01(seed, N, 16 * s + 0)
    counts = np.where(r < (ppc - f), f + 1, f).astype(np.uint32)
    if cell_mask is not None:
        counts = np.where(cell_mask, counts, 0).astype(np.uint32)
    n = int(counts.sum())
    u = [uniform01(seed, n, 16 * s + 1 + a) for a in range(9)]
    xc = 0.5 * dx
    parts = np.empty((n, 7), dtype=np.float64)
    for a in range(3):
        parts[:, a] = xc + (1.0 - EPS_CELL) * dx * (u[a] - 0.5)
    for a in range(3):
        u1 = 1.0 - u[3 + 2 * a]          # (0,1]
        u2 = u[4 + 2 * a]
        g = np.sqrt(-2.0 * np.log(u1)) * np.cos(2.0 * math.pi * u2)
        parts[:, 3 + a] = p.velocity[a] + vth * g
    parts[:, 6] = w
    return counts, parts


def initial_state(cfg: Config, cell_masks=None):
    """Grid arrays plus all populations for a fresh run."""
    g = init_grid(cfg)
    pops = []
    for s in range(len(cfg.populations)):
        m = None if cell_masks is None else cell_masks[s]
        pops.append(uniform_population(cfg, s, cell_mask=m))
    return g, pops
