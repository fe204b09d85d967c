"""The reference built with USE_GRID_CONSTRAINT_COUNTERS (oracle/_ref) as the
oracle of the per-cell constraint counters: each plane sums to the matching
global log counter of the same run (hybrid_propagator.cpp:1382, 1440, 1513,
1579, boris.h:153-155, particle_accumulator.cpp:327)."""
from rhybrid_b200 import abi
from rhybrid_b200 import config as cf

from harness import closed_box_config, load


def check_planes_against_log_counters(ctx, nspecies):
    gc = ctx.grid_counters()
    c = ctx.counters()
    assert gc["cellMaxUe"].sum() == c["fieldMaxCellUe"] + c["fieldMaxNodeUe"]
    assert gc["cellMaxVi"].sum() == sum(c[f"particleMaxVi[{s}]"] for s in range(nspecies))
    assert gc["cellMinRhoQi"].sum() == c["fieldMinCellRhoQi"]
    assert gc["nodeMaxE"].sum() == c["fieldMaxE"]
    assert gc["nodeMaxVw"].sum() == c["fieldMaxVw"]
    return gc


# tight limits so that every counter fires in a few steps
TIGHT = dict(max_ion_velocity=430e3, max_electron_velocity=430e3, max_electric_field=1.5e-3)


def test_reference_grid_counters(ref_gc_lib):
    cfg = closed_box_config(**TIGHT)
    grid, pops = cf.initial_state(cfg)
    ctx = abi.Context(ref_gc_lib, cf.params(cfg), cf.species(cfg), capacity=[p[1].shape[0] + 256 for p in pops])
    try:
        load(ctx, cfg, grid, pops)
        ctx.set_grid_counters(True)
        ctx.step(4)
        gc = check_planes_against_log_counters(ctx, ctx.nspecies)
        assert all(v.sum() > 0 for v in gc.values())
        ctx.set_grid_counters(True)   # zeroes them again
        assert all(v.sum() == 0 for v in ctx.grid_counters().values())
    finally:
        ctx.close()
