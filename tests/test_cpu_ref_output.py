"""The output step's cell variables and particle points
(rhybrid_b200/output.py) against the reference's own output operator,
UserDataOP::writeData (src/operator_userdata.cpp:55-312), compiled from its
sources in oracle/_ref with a VLSV writer stand-in that keeps the arrays it is
given. Both run on the same state of the reference build (through the
library's ABI): same names, same write order, values equal bit for bit."""
import numpy as np
import pytest

from rhybrid_b200 import abi
from rhybrid_b200 import config as cf
from rhybrid_b200 import output as O

from harness import closed_box_config, load

WRITTEN = [p for p in O.PARAMETERS if p not in ("prod_rate_iono", "prod_rate_exo", "cellB0", "MPI_rank", "Load")]
GROUPS, NAMES = [0, 1, 1], ["H+", "heavy"]


def three_species_config():
    c = closed_box_config(periodic=(0, 1, 0))
    R = c.R_particleObstacle
    pops = c.populations + [cf.Population(name="O+", mass=16.0, charge=1.0, obstacle=R, density=0.05e6,
                                          velocity=(-300e3, 10e3, 0), temperature=3e4, ppc=1.0)]
    return c.replace(populations=pops)


def run_state(lib, steps=3, counters=False):
    cfg = three_species_config()
    grid, pops = cf.initial_state(cfg)
    ctx = abi.Context(lib, cf.params(cfg), cf.species(cfg), capacity=[p[1].shape[0] + 256 for p in pops])
    load(ctx, cfg, grid, pops)
    ctx.set_population_averages(GROUPS)
    if counters:
        ctx.set_grid_counters(True)
    ctx.step(steps)
    return ctx


def compare(mine, ref):
    assert list(mine) == list(ref)
    for k in ref:
        assert mine[k].shape == ref[k].shape, k
        assert np.array_equal(mine[k], ref[k]), (k, float(np.abs(mine[k] - ref[k]).max()))


@pytest.mark.parametrize("params", [WRITTEN, ["cellB", "n", "T", "v"], ["faceB", "n_ave", "cellDivB"],
                                    ["v_ave", "cellNPles", "ne", "innerFlagParticle"], ["cellBAverage"]],
                         ids=["all", "moments", "averages", "ne_gate", "cellBAverage"])
def test_cell_variables_match_reference_writer(ref_lib, params):
    from oracle import oracle
    with run_state(ref_lib) as ctx:
        mine = O.cell_variables(ctx, params, GROUPS, NAMES)
    with run_state(ref_lib) as ctx:
        ref = oracle.reference_write_data(ctx, params, NAMES)
    compare(mine, ref)
    if "n" in params:
        assert np.any(mine["n_heavy"] > 0) and np.any(mine["T_H+"] > 0)


def test_second_output_restarts_the_averages(ref_lib):
    """Two output steps in a row: the second one's averages cover only the
    steps after the first (both sides restart their sums and counter)."""
    from oracle import oracle
    params = ["cellBAverage", "n_ave", "v_ave"]
    with run_state(ref_lib, steps=2) as ctx:
        O.cell_variables(ctx, params, GROUPS, NAMES)
        ctx.step(2)
        mine = O.cell_variables(ctx, params, GROUPS, NAMES)
    with run_state(ref_lib, steps=2) as ctx:
        oracle.reference_write_data(ctx, params, NAMES)
        ctx.step(2)
        ref = oracle.reference_write_data(ctx, params, NAMES)
    compare(mine, ref)


def test_grid_counter_variables_match_reference_writer(ref_gc_lib):
    from oracle import oracle
    params = ["gridCounterCellMaxUe", "gridCounterCellMaxVi", "gridCounterCellMinRhoQi", "gridCounterNodeMaxE",
              "gridCounterNodeMaxVw", "cellRhoQi"]
    with run_state(ref_gc_lib, counters=True) as ctx:
        mine = O.cell_variables(ctx, params, GROUPS, NAMES, grid_counters=True)
    with run_state(ref_gc_lib, counters=True) as ctx:
        ref = oracle.reference_write_data(ctx, params, NAMES)
    compare(mine, ref)


def test_particle_points(ref_lib):
    """writeParticles' cell selection (every Nstride'th cell id, in the
    planes and rows the id rule keeps), global coordinates inside their cell,
    velocities and cell ids of the same particles."""
    with run_state(ref_lib, steps=1) as ctx:
        p = ctx.params
        out = O.particle_points(ctx, ["swH+", "swHe++", "ionoO+"], nstride=3)
        cnt0, q0 = ctx.download_particles(0)
    nx, ny = p.nx, p.ny
    cid = out["CellID_swH+"].astype(np.int64)
    assert cid.size > 0 and np.all(cid % 3 == 0) and np.all(cid % (3 * nx) < nx) and np.all(cid % (3 * nx * ny) < nx * ny)
    sel = [c for c in range(p.nx * p.ny * p.nz) if c % 3 == 0 and c % (3 * nx) < nx and c % (3 * nx * ny) < nx * ny]
    assert cid.size == int(cnt0[sel].sum())
    i, j, k = cid % nx, (cid // nx) % ny, cid // (nx * ny)
    xyz = out["ParticlePointMesh_swH+"]
    lo = np.stack([p.x_min + i * p.dx, p.y_min + j * p.dx, p.z_min + k * p.dx], axis=1)
    assert np.all(xyz >= lo) and np.all(xyz < lo + p.dx)
    assert out["v_swH+"].shape == (cid.size, 3) and set(out) == {f"{a}_{n}" for n in ("swH+", "swHe++", "ionoO+")
                                                                for a in ("ParticlePointMesh", "v", "CellID")}


def test_unknown_parameter_and_group_checks(ref_lib):
    """An unknown name is skipped with a warning (user.cpp:2405-2410); output
    population names must match the groups."""
    with run_state(ref_lib, steps=0) as ctx:
        with pytest.warns(UserWarning, match="notAVariable"):
            out = O.cell_variables(ctx, ["cellB", "notAVariable"], GROUPS, NAMES)
        assert list(out) == ["cellB"]
        with pytest.raises(ValueError):
            O.cell_variables(ctx, ["n"], GROUPS, ["H+"])


class _SourcesOnly:
    """Stand-in context with sources only: source_rates(q) is q+1 everywhere."""
    ncells = 5

    def __init__(self, injectors):
        self.injectors = injectors

    def source_rates(self, q):
        return np.full(self.ncells, q + 1.0)


def test_production_rate_slots():
    """prod_rate_iono<k>: one counter per ionosphere injector class, both
    writing cellIonosphere (particle_injector.cpp:1112-1114, :1415-1417), the
    later source in species order staying; prod_rate_exo<k> in species order."""
    J = lambda t, s: abi.Injector(type=t, species=s)   # noqa: E731
    srcs = [J(abi.INJECT_IONOSPHERE, 1), J(abi.INJECT_CHAPMAN_IONOSPHERE, 2), J(abi.INJECT_IONOSPHERE, 3),
            J(abi.INJECT_EXOSPHERE, 4), J(abi.INJECT_EXOSPHERE, 0), J(abi.INJECT_SOLARWIND, 5)]
    out = O.production_rates(_SourcesOnly(srcs))
    assert list(out) == ["prod_rate_iono0", "prod_rate_iono1", "prod_rate_iono2", "prod_rate_exo0", "prod_rate_exo1"]
    assert out["prod_rate_iono0"][0] == 2.0     # the Chapman source (species 2) after species 1
    assert out["prod_rate_iono1"][0] == 3.0     # the second IonosphereInjector (species 3)
    assert not out["prod_rate_iono2"].any()     # no third writer
    assert out["prod_rate_exo0"][0] == 5.0 and out["prod_rate_exo1"][0] == 4.0
    assert O.production_rates(_SourcesOnly([])) == {}
