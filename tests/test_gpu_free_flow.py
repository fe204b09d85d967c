"""The reference's own acceptance test of the free flow, run through this
build's time loop: tests/run_tests.py:333-404 with the configuration of
tests/test_empty_1d.cfg (restated below with the same keys and values). A box
of 40 cells of 100 km along the flow and 3 x 3 across, periodic (the
reference's box is one cell across; this library's grids have at least 3
cells per axis, and a uniform free flow is the same at any width), 1000
macroparticles per cell of solar wind protons (not accelerated by the fields)
injected at the upstream wall for three flow-throughs at 400 km/s, a state
saved every tenth of the run. In the second-to-last saved state the domain
means of n, T, U and B (the layers along the flow that the reference's slice
[Nbc : -1 - Nbc] keeps, Nbc a tenth of them, over the whole cross-section)
must equal the nonzero inputs within a factor 1 +- 1 / sqrt(ppc). The
injection, the push, the deposit, the bulk parameters and the VLSV state
files (rhybrid_b200.vlsv) are all on the path."""
import math
import os

import numpy as np
import pytest

from rhybrid_b200 import run as R
from rhybrid_b200 import vlsv as V

pytestmark = pytest.mark.gpu

NCELLS, WIDTH, DX, PPC, FLOW_THROUGHS, SAVES = 40, 3, 100e3, 1000, 3, 10
MAX_USW = 400e3
DT = 0.025                                  # dx / (10 max Usw), two significant digits
STEPS = math.ceil(FLOW_THROUGHS * NCELLS * DX / MAX_USW / DT)
SAVE_INTERVAL = STEPS // SAVES
A_VAR = 1.0 / math.sqrt(PPC)

CFG = """
[Simulation]
time_initial = 0.0
maximum_timesteps = {steps}
dt = {dt}
data_save_interval = {save}
data_save_interval_unit = timestep
random_number_generator.seed = 6461674
save_particles = 0
[LogicallyCartesian]
geometry = cartesian
x_periodic = {per[0]}
y_periodic = {per[1]}
z_periodic = {per[2]}
x_min = {lo[0]}
y_min = {lo[1]}
z_min = {lo[2]}
x_max = {hi[0]}
y_max = {hi[1]}
z_max = {hi[2]}
x_size = {size[0]}
y_size = {size[1]}
z_size = {size[2]}
[Hybrid]
log_interval = 0
output_parameters = cellB n v T
R_fieldObstacle = -100
R_particleObstacle = -100
hall_term = 1
particle.population.solarwind = sw_protons
[Resistivity]
profile_name = resistivityConstant
value_unit = grid
value = 0.005465166666667
outer_boundary_cells = 0 0 0 0 0 0
outer_boundary_coeffs = 1 1 1 1 1 1
[IMF]
Bx = 0.0
By = 0.0
Bz = 0.0
BoundaryCellB = 0 0 0 0 0 0
BoundaryFaceB = 0 0 0 0 0 0
[IntrinsicB]
profile_name = constantB
[sw_protons]
mass_unit = MASS_PROTON
charge_unit = CHARGE_ELEMENTARY
mass = 1.0
charge = +1.0
obstacle = -100.0
accumulate = 1
accelerate = 0
output_str = H+
output_plasma = 1
injector.name = SolarWindInjector
injector.parameters = inj_sw_protons
[inj_sw_protons]
velocity = {u[0]} {u[1]} {u[2]}
density = {n}
temperature = {T}
macroparticles_per_cell = {ppc}
"""


def config_text(axis: int, usw: float, n: float, T: float) -> str:
    """The reference's test configuration for a flow of speed usw (signed)
    along `axis`: that axis 40 cells and closed, the others WIDTH cells and
    periodic."""
    half = NCELLS * DX / 2.0
    per = ["yes"] * 3
    lo, hi, size, u = [-WIDTH * DX / 2.0] * 3, [WIDTH * DX / 2.0] * 3, [WIDTH] * 3, [0.0] * 3
    per[axis], lo[axis], hi[axis], size[axis], u[axis] = "no", -half, half, NCELLS, usw
    return CFG.format(steps=STEPS, dt=DT, save=SAVE_INTERVAL, per=per, lo=lo, hi=hi, size=size, u=u, n=n, T=T, ppc=PPC)


def check_flow_conditions(state: dict, axis: int, n: float, T: float, u) -> list:
    """checkFlowConditions / doComparison (run_tests.py:333-404): the failed
    comparisons of the domain means with the inputs."""
    order = np.argsort(state["CellID"])
    nbc = int(math.floor(NCELLS / 10))
    layers = np.arange(NCELLS)[nbc:-1 - nbc]   # the layers along the flow the reference's slice keeps
    shape = [WIDTH, WIDTH, WIDTH]
    shape[2 - axis] = NCELLS                   # cells in linear order: x fastest, (z, y, x)

    def cells(a):
        a = np.asarray(a)[order]
        a = a.reshape(tuple(shape) + a.shape[1:])
        return np.take(a, layers, axis=2 - axis).reshape((-1,) + a.shape[3:])

    means = {"n": cells(state["n_H+"]).mean(), "T": cells(state["T_H+"]).mean()}
    U = cells(state["v_H+"])
    B = cells(state["cellB"])
    failed = []
    for name, model, want in [("n", means["n"], n), ("T", means["T"], T)] + \
            [(f"U{c}", U[:, k].mean(), u[k]) for k, c in enumerate("xyz")] + \
            [(f"B{c}", B[:, k].mean(), 0.0) for k, c in enumerate("xyz")]:
        if abs(want) > 0:
            rel = abs(model / want)
            if rel < 1.0 - A_VAR or rel > 1.0 + A_VAR:
                failed.append(f"{name}: input {want}, modeled {model}, |modeled/input| {rel:.4f}")
    return failed


CASES = [(axis, sign * 400e3, 1e6, 1e5) for axis in range(3) for sign in (-1, 1)] + [(0, -300e3, 10e6, 1e4)]


@pytest.mark.parametrize("axis,usw,n,T", CASES)
def test_free_flow_conditions(tmp_path, axis, usw, n, T):
    f = tmp_path / "test_empty_1d.cfg"
    f.write_text(config_text(axis, usw, n, T))
    r = R.run(str(f), out_dir=str(tmp_path), quiet=True)
    assert r["steps"] == STEPS and len(r["saved"]) == SAVES
    state = V.load_state(sorted(r["saved"])[-2])
    assert os.path.basename(sorted(r["saved"])[-2]) == f"state_{STEPS - SAVE_INTERVAL:07d}.vlsv"
    u = [0.0, 0.0, 0.0]
    u[axis] = usw
    failed = check_flow_conditions(state, axis, n, T, u)
    assert not failed, failed
