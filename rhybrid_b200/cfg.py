"""Reader of RHybrid run configuration files (.cfg, Corsair's ConfigReader
format: `[section]` headers, `key = value` lines, `#` comments, repeated keys
for vector items such as neutral_profile.n0).

`load(path)` returns the `Config` the library runs (grid, physics switches,
limits, populations with their particle sources) and the `RunSettings` of the
output side (log files, averages, run length). The keys read are those that
userLateInitialization and the plugins take (src/user.cpp:356-1807,
src/particle_injector.cpp, src/particle_species.cpp); keys of the parts this
library does not run (load balancing, restarts, detectors, VLSV output
selection) are kept in RunSettings.extra or ignored.
"""
from dataclasses import dataclass, field
from typing import Dict, List, Optional, Tuple

from . import config as cf


@dataclass
class RunSettings:
    """The output-side settings of a .cfg."""
    maximum_timesteps: int = 0
    data_save_interval: int = 0
    log_interval: int = 50                  # Hybrid.log_interval (default 50, user.cpp:412)
    log_precision: int = 10
    include_inner_cells_in_field_log: bool = False
    main_log_diagnostics_interval: int = 100
    max_magnetic_field_stop_run: float = float("inf")
    output_parameters: List[str] = field(default_factory=list)
    output_groups: List[int] = field(default_factory=list)   # output population of each species (-1: none)
    output_group_names: List[str] = field(default_factory=list)   # output_str of each output population
    save_particles: bool = False            # Hybrid.save_particles (user.cpp:396)
    save_particles_nstride: int = 10        # Hybrid.save_particles_Nstride (user.cpp:397)
    data_save_all_timesteps_t_start: float = -1.0   # Hybrid.data_save_all_timesteps_t_start (user.cpp:418)
    data_save_all_timesteps_t_end: float = -1.0     # Hybrid.data_save_all_timesteps_t_end (user.cpp:419)
    save_reduced_state_interval: int = 0    # Hybrid.save_reduced_state_interval (user.cpp:420)
    save_reduced_state_nstride: int = 10    # Hybrid.save_reduced_state_Nstride (user.cpp:421; <= 0 gives 10, :2452-2455)
    save_reduced_state_particles: bool = False   # Hybrid.save_reduced_state_include_particles (user.cpp:422)
    species_names: List[str] = field(default_factory=list)
    extra: Dict[str, Dict[str, List[str]]] = field(default_factory=dict)


def parse(text: str) -> Dict[str, Dict[str, List[str]]]:
    """Sections -> key -> every value given (in file order). Keys before the
    first section are in section ""."""
    out: Dict[str, Dict[str, List[str]]] = {"": {}}
    sec = ""
    for raw in text.splitlines():
        line = raw.split("#", 1)[0].strip()
        if not line:
            continue
        if line.startswith("[") and line.endswith("]"):
            sec = line[1:-1].strip()
            out.setdefault(sec, {})
            continue
        if "=" not in line:
            raise ValueError(f"cfg: cannot read line {raw!r}")
        k, v = line.split("=", 1)
        out[sec].setdefault(k.strip(), []).append(v.strip())
    return out


class _Section:
    def __init__(self, name: str, items: Dict[str, List[str]]):
        self.name, self.items = name, items

    def has(self, key: str) -> bool:
        return key in self.items and self.items[key][-1] != ""

    def str(self, key: str, default: Optional[str] = None) -> Optional[str]:
        return self.items[key][-1] if self.has(key) else default

    def float(self, key: str, default: float = 0.0) -> float:
        return float(self.items[key][-1]) if self.has(key) else default

    def int(self, key: str, default: int = 0) -> int:
        return int(float(self.items[key][-1])) if self.has(key) else default

    def bool(self, key: str, default: bool = False) -> bool:
        if not self.has(key):
            return default
        v = self.items[key][-1].lower()
        if v in ("yes", "true", "1", "on"):
            return True
        if v in ("no", "false", "0", "off"):
            return False
        return float(v) != 0.0

    def floats(self, key: str) -> List[float]:
        """All values of a repeated key, or the items of one space-separated value."""
        vals = self.items.get(key, [])
        if len(vals) == 1:
            return [float(x) for x in vals[0].replace(",", " ").split()]
        return [float(x) for x in vals if x != ""]

    def vector(self, key: str, default=(0.0, 0.0, 0.0)) -> Tuple[float, float, float]:
        if not self.has(key):
            return tuple(default)
        v = self.items[key][-1].strip().strip("()")
        a = [float(x) for x in v.replace(",", " ").split()]
        if len(a) != 3:
            raise ValueError(f"cfg [{self.name}] {key}: expected three components, got {v!r}")
        return tuple(a)


def _sec(parsed, name) -> _Section:
    return _Section(name, parsed.get(name, {}))


_UNITS = {"MASS_PROTON": 1.0, "CHARGE_ELEMENTARY": 1.0}
_WALLS = ("+x", "-x", "+y", "-y", "+z", "-z")


def _population(parsed, name: str, R_particle: float) -> Tuple[cf.Population, str]:
    s = _sec(parsed, name)
    if not s.items:
        raise ValueError(f"cfg: population section [{name}] is missing")
    for unitkey in ("mass_unit", "charge_unit"):
        u = s.str(unitkey, None)
        if u not in (None,) + tuple(_UNITS):
            raise ValueError(f"cfg [{name}] {unitkey} = {u}: only MASS_PROTON / CHARGE_ELEMENTARY units are read")
    inj_name = s.str("injector.name", "")
    inj = _sec(parsed, s.str("injector.parameters", "") or "")
    pop = cf.Population(name=name, mass=s.float("mass", 1.0), charge=s.float("charge", 1.0),
                        obstacle=s.float("obstacle", R_particle), accumulate=s.bool("accumulate", True),
                        accelerate=s.bool("accelerate", True), density=0.0, velocity=(0.0, 0.0, 0.0),
                        temperature=0.0, ppc=0.0, upstream=False, fill=False)
    if inj_name in ("UniformInjector", "SolarWindInjector", "FlowInjector"):
        pop.density = inj.float("density")
        pop.velocity = inj.vector("velocity")
        pop.temperature = inj.float("temperature")
        pop.ppc = inj.float("macroparticles_per_cell")
        pop.upstream = inj_name == "SolarWindInjector"
        # only the uniform injector fills the box at the start; the others inject from step 1
        pop.fill = inj_name == "UniformInjector"
        if inj_name == "FlowInjector":
            walls = (inj.str("inflow_boundaries", "") or "").replace(",", " ").split()
            bad = [w for w in walls if w not in _WALLS]
            if bad:
                raise ValueError(f"cfg [{name}]: unknown inflow boundaries {bad}")
            pop.flow_walls = walls
    elif inj_name == "ExosphereInjector":
        pop.temperature = inj.float("temperature")
        prof = inj.str("neutral_profile", "")
        e = {"profile": prof, "r0": inj.float("neutral_profile.r0", -1.0),
             "n0": inj.floats("neutral_profile.n0"), "H0": inj.floats("neutral_profile.H0"),
             "T0": inj.floats("neutral_profile.T0"), "k0": inj.floats("neutral_profile.k0"),
             "exobase_radius": inj.float("exobase_radius"), "shadow_radius": inj.float("shadow_radius"),
             "ionization_factor_shadow": inj.float("ionization_factor_shadow", 1.0),
             "macroparticles_per_cell_relative": inj.float("macroparticles_per_cell_relative", 1.0)}
        if inj.has("ionization_rate"):
            e["ionization_rate"] = inj.float("ionization_rate")
        if inj.has("total_production_rate"):
            e["total_production_rate"] = inj.float("total_production_rate")
        if not e["n0"] and prof in ("ChamberlainH", "ChamberlainT", "Exponential", "PowerLaw"):
            raise ValueError(f"cfg [{name}]: neutral profile {prof} needs neutral_profile.n0")
        pop.exosphere = e
    elif inj_name in ("IonosphereInjector", "ChapmanIonosphereInjector"):
        pop.temperature = inj.float("temperature")
        pop.ionosphere = {"profile": "Chapman" if inj_name.startswith("Chapman") else inj.str("profile_name", ""),
                          "emission_radius": inj.float("emission_radius"), "noon": inj.float("noon"),
                          "night": inj.float("night"), "total_production_rate": inj.float("total_production_rate"),
                          "macroparticles_per_cell_relative": inj.float("macroparticles_per_cell_relative", 1.0)}
    elif inj_name:
        raise ValueError(f"cfg [{name}]: injector {inj_name} is not supported")
    return pop, s.str("output_str", "-") or "-"


def load_text(text: str) -> Tuple[cf.Config, RunSettings]:
    """A .cfg's content as (Config, RunSettings)."""
    P = parse(text)
    sim, lc, hy = _sec(P, "Simulation"), _sec(P, "LogicallyCartesian"), _sec(P, "Hybrid")
    n = [lc.int(f"{a}_size") for a in "xyz"]
    lo = [lc.float(f"{a}_min") for a in "xyz"]
    hi = [lc.float(f"{a}_max") for a in "xyz"]
    d = [(hi[i] - lo[i]) / n[i] for i in range(3)]
    if min(n) < 1 or any(abs(d[i] - d[0]) > 1e-9 * abs(d[0]) for i in range(3)):
        raise ValueError(f"cfg [LogicallyCartesian]: cells must be cubes (dx, dy, dz = {d})")
    per = tuple(1 if lc.bool(f"{a}_periodic") else 0 for a in "xyz")
    # the populations, in the order the [Hybrid] particle.population.* lines list them
    names: List[str] = []
    for k, vals in P.get("Hybrid", {}).items():
        if k.startswith("particle.population"):
            names += [v for v in vals if v]
    R_particle = hy.float("R_particleObstacle", -100.0)
    pops, outs = [], []
    for nm in names:
        p, o = _population(P, nm, R_particle)
        pops.append(p)
        outs.append(o)
    groups, seen = [], []
    for o in outs:
        if o == "-":
            groups.append(-1)
        else:
            if o not in seen:
                seen.append(o)
            groups.append(seen.index(o))
    ep, res, con, imf, ib = (_sec(P, x) for x in ("ElectronPressure", "Resistivity", "Constraints", "IMF", "IntrinsicB"))
    cfgobj = cf.Config(
        nx=n[0], ny=n[1], nz=n[2], x_min=lo[0], y_min=lo[1], z_min=lo[2], dx=d[0], periodic=per,
        dt=sim.float("dt"), t_initial=sim.float("time_initial"),
        R_fieldObstacle=hy.float("R_fieldObstacle", -100.0), R_particleObstacle=R_particle,
        fieldObstacleUe=hy.vector("fieldObstacleUe"), use_gravity=hy.bool("use_gravity"),
        M_object=hy.float("M_object"), use_hall_term=hy.bool("use_hall_term", True),
        imf=(imf.float("Bx"), imf.float("By"), imf.float("Bz")),
        imf_boundary_cellB=tuple(int(x) for x in (imf.floats("BoundaryCellB") or [0] * 6)),
        imf_boundary_faceB=tuple(int(x) for x in (imf.floats("BoundaryFaceB") or [0] * 6)),
        b_profile=ib.str("profile_name", "constantB") or "constantB",
        dipole_surface_B=ib.float("dipoleSurfaceB"), dipole_surface_R=ib.float("dipoleSurfaceR"),
        dipole_min_R=ib.float("minimumR"), dipole_origin=(ib.float("x"), ib.float("y"), ib.float("z")),
        laminar_R=ib.float("laminarR"),
        use_electron_pressure=ep.bool("use_electron_pressure"), electron_temperature=ep.float("temperature"),
        electron_gamma=ep.int("closure_gamma", 2), R_zeroElectronPressure=ep.float("R_zero", -100.0),
        resistivity_profile=res.str("profile_name", "resistivityConstant") or "resistivityConstant",
        resistivity_unit=res.str("value_unit", "Rm") or "Rm", resistivity_value=res.float("value"),
        resistivity_R=res.float("R"),
        resistivity_outer_cells=tuple(int(x) for x in (res.floats("outer_boundary_cells") or [0] * 6)),
        resistivity_outer_coeffs=tuple(res.floats("outer_boundary_coeffs") or [1.0] * 6),
        max_ion_velocity=con.float("max_ion_velocity", 1500e3),
        max_electron_velocity=con.float("max_electron_velocity", 1500e3),
        min_ion_charge_density_relative=con.float("min_ion_charge_density_relative", 0.05),
        max_electric_field=con.float("max_electric_field", -100.0),
        max_whistler_velocity=con.float("max_whistler_velocity", 1500e3),
        initial_flow_throughs=con.float("initial_flow_throughs", -1.0),
        electric_field_linear_smoothing_number=con.int("electric_field_linear_smoothing_number"),
        electric_field_smoothing_gauss_sigma=con.float("electric_field_smoothing_gauss_sigma"),
        populations=pops, seed=sim.int("random_number_generator.seed", 6461674), name="cfg")
    rs = RunSettings(
        maximum_timesteps=sim.int("maximum_timesteps"), data_save_interval=sim.int("data_save_interval"),
        log_interval=hy.int("log_interval", 50), log_precision=hy.int("log_precision", 10),
        include_inner_cells_in_field_log=hy.bool("includeInnerCellsInFieldLog"),
        main_log_diagnostics_interval=hy.int("main_log_diagnostics_interval", 100),
        max_magnetic_field_stop_run=con.float("max_magnetic_field_stop_run", float("inf")),
        output_parameters=(hy.str("output_parameters", "") or "").split(), output_groups=groups,
        output_group_names=seen, save_particles=hy.bool("save_particles"),
        save_particles_nstride=hy.int("save_particles_Nstride", 10), species_names=names,
        data_save_all_timesteps_t_start=hy.float("data_save_all_timesteps_t_start", -1.0),
        data_save_all_timesteps_t_end=hy.float("data_save_all_timesteps_t_end", -1.0),
        save_reduced_state_interval=hy.int("save_reduced_state_interval", 0),
        save_reduced_state_nstride=(hy.int("save_reduced_state_Nstride", 10)
                                    if hy.int("save_reduced_state_Nstride", 10) > 0 else 10),
        save_reduced_state_particles=hy.bool("save_reduced_state_include_particles"),
        extra={k: v for k, v in P.items() if k in ("Restart", "LoadBalance", "DetectorParticle",
                                                    "DetectorBulkParameter", "DataOperatorExcludes")})
    # the window of saving at every step (user.cpp:2381-2388): start > end is an
    # error, a negative start or a non-positive end switches it off
    if rs.data_save_all_timesteps_t_start > rs.data_save_all_timesteps_t_end:
        raise ValueError("Hybrid.data_save_all_timesteps_t_start must be below Hybrid.data_save_all_timesteps_t_end")
    if rs.data_save_all_timesteps_t_start < 0 or rs.data_save_all_timesteps_t_end <= 0:
        rs.data_save_all_timesteps_t_start = rs.data_save_all_timesteps_t_end = -1.0
    return cfgobj, rs


def load(path: str) -> Tuple[cf.Config, RunSettings]:
    """Reads a .cfg file (see load_text)."""
    with open(path) as f:
        return load_text(f.read())
