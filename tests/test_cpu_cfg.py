"""Reader of RHybrid .cfg files (rhybrid_b200/cfg.py): the ConfigReader format
(sections, repeated keys, comments), the grid, switches, limits, populations
with their sources and the output settings; every example of the reference
that has cube cells loads, and a loaded configuration steps on the oracle."""
import glob
import os

import numpy as np
import pytest

from rhybrid_b200 import abi
from rhybrid_b200 import cfg as C
from rhybrid_b200 import config as cf
from rhybrid_b200 import output as O

TEXT = """
gridbuilder = LogicallyCartesian
[Simulation]
time_initial = 0.0
maximum_timesteps = 200
dt = 0.04                      # seconds
random_number_generator.seed = 99
[LogicallyCartesian]
x_periodic = no
y_periodic = yes
z_periodic = no
x_min = -1200e3
x_max = +1200e3
y_min = -800e3
y_max = +800e3
z_min = -600e3
z_max = +600e3
x_size = 24
y_size = 16
z_size = 12
[Hybrid]
log_interval = 5
log_precision = 8
output_parameters = cellB n_ave v_ave
R_fieldObstacle = 300e3
R_particleObstacle = 250e3
fieldObstacleUe = (1e3,0,-2e3)
use_hall_term = 1
particle.population.solarwind = swH+
particle.population.exosphere = exoO+
particle.population.ionosphere = ionoO+
[Constraints]
max_ion_velocity = 1200e3
max_magnetic_field_stop_run = 500e-9
[IMF]
Bx = 1e-9
By = 2e-9
Bz = -1e-9
BoundaryCellB = 1 0 0 0 0 0
BoundaryFaceB = 1 0 0 0 0 0
[Resistivity]
profile_name = resistivityConstant
value_unit = Rm
value = 5
[swH+]
mass_unit = MASS_PROTON
charge_unit = CHARGE_ELEMENTARY
mass = 1.0
charge = +1.0
output_str = H+
injector.name = SolarWindInjector
injector.parameters = inj_sw
[inj_sw]
velocity = (-400e3,0,0)
density = 4e6
temperature = 1e5
macroparticles_per_cell = 12
[exoO+]
mass = 16.0
charge = 1.0
output_str = O+
injector.name = ExosphereInjector
injector.parameters = inj_exo
[inj_exo]
neutral_profile = Exponential
neutral_profile.r0 = 300e3
neutral_profile.n0 = 1e10
neutral_profile.n0 = 2e9
neutral_profile.H0 = 100e3
neutral_profile.H0 = 400e3
temperature = 2000
exobase_radius = 320e3
shadow_radius = 300e3
total_production_rate = 1e23
[ionoO+]
mass = 16.0
charge = 1.0
output_str = O+
injector.name = IonosphereInjector
injector.parameters = inj_iono
[inj_iono]
profile_name = ionoCosSzaDayConstantNight
emission_radius = 350e3
noon = 1.0
night = 0.2
temperature = 1000
total_production_rate = 5e22
"""


def test_cfg_reader():
    c, rs = C.load_text(TEXT)
    assert (c.nx, c.ny, c.nz) == (24, 16, 12) and c.dx == 100e3 and c.periodic == (0, 1, 0)
    assert (c.x_min, c.dt, c.seed) == (-1200e3, 0.04, 99)
    assert c.fieldObstacleUe == (1e3, 0.0, -2e3) and c.R_particleObstacle == 250e3
    assert c.imf == (1e-9, 2e-9, -1e-9) and c.imf_boundary_cellB == (1, 0, 0, 0, 0, 0)
    assert c.max_ion_velocity == 1200e3 and c.resistivity_value == 5.0
    assert [p.name for p in c.populations] == ["swH+", "exoO+", "ionoO+"]
    sw, exo, iono = c.populations
    assert sw.upstream and not sw.fill and sw.ppc == 12 and sw.velocity == (-400e3, 0.0, 0.0)
    assert exo.exosphere["n0"] == [1e10, 2e9] and exo.exosphere["H0"] == [100e3, 400e3]
    assert iono.ionosphere["profile"] == "ionoCosSzaDayConstantNight" and iono.ionosphere["night"] == 0.2
    assert rs.log_interval == 5 and rs.log_precision == 8 and rs.max_magnetic_field_stop_run == 500e-9
    assert rs.output_groups == [0, 1, 1] and rs.output_parameters == ["cellB", "n_ave", "v_ave"]
    assert rs.output_group_names == ["H+", "O+"] and not rs.save_particles and rs.save_particles_nstride == 10
    src = cf.source_injectors(c)
    assert [(j.species, j.type) for j in src] == [(0, abi.INJECT_SOLARWIND), (1, abi.INJECT_EXOSPHERE),
                                                 (2, abi.INJECT_IONOSPHERE)]
    assert src[1].n_components == 2 and src[1].upstream_macro_ratio == pytest.approx(400e3 * 0.04 / 100e3 * 16 * 10)
    # sources fill the box from step 1: nothing at the start
    grid, pops = cf.initial_state(c)
    assert all(p[1].shape[0] == 0 for p in pops)


def test_cfg_rejects_non_cubic_cells():
    with pytest.raises(ValueError):
        C.load_text(TEXT.replace("z_size = 12", "z_size = 10"))


def test_loaded_cfg_steps_on_oracle(port_lib):
    """A configuration read from a .cfg with a uniform population runs on the
    C restatement (the library's ABI without a GPU)."""
    text = TEXT.replace("injector.name = SolarWindInjector", "injector.name = UniformInjector")
    c, _ = C.load_text(text)
    c.populations = c.populations[:1]
    grid, pops = cf.initial_state(c)
    assert pops[0][1].shape[0] > 0
    ctx = abi.Context(port_lib, cf.params(c), cf.species(c), capacity=[pops[0][1].shape[0] + 256])
    try:
        ctx.upload_array("faceB", grid["faceB"])
        ctx.upload_array("cellB", grid["cellB"])
        ctx.upload_array("nodeEta", grid["nodeEta"])
        ctx.upload_cell_flags(grid["flags"])
        ctx.upload_particles(0, *pops[0])
        ctx.step(2)
        assert np.all(np.isfinite(ctx.download_array("faceB")))
    finally:
        ctx.close()


def test_reference_examples_load():
    from oracle import oracle
    files = sorted(glob.glob(os.path.join(oracle.REF_DIR, "examples", "*.cfg")))
    if not files:
        pytest.skip("the reference's examples are not present")
    loaded = 0
    for f in files:
        try:
            c, rs = C.load(f)
        except ValueError as e:
            assert "cube" in str(e), (f, e)   # the 2-D example with a flat cell
            continue
        cf.source_injectors(c)
        assert len(rs.output_groups) == len(c.populations)
        assert len(rs.output_group_names) == max(rs.output_groups, default=-1) + 1
        # every output parameter an example asks for is one the output step knows
        assert set(rs.output_parameters) <= set(O.PARAMETERS), (f, set(rs.output_parameters) - set(O.PARAMETERS))
        loaded += 1
    assert loaded >= 10
