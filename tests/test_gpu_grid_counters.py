"""Per-cell grid constraint counters (rhgpu_set_grid_counters,
rhgpu_download_grid_counters) against the reference built with
USE_GRID_CONSTRAINT_COUNTERS (oracle/_ref): every plane equal on the exact
path (counts of the same events in the same cells); on the fast and FP32
paths each plane sums to the path's own global log counter."""
import numpy as np
import pytest

from rhybrid_b200 import abi
from rhybrid_b200 import config as cf

from harness import closed_box_config, load
from test_cpu_ref_grid_counters import TIGHT, check_planes_against_log_counters

pytestmark = pytest.mark.gpu


def run(lib, cfg, path=None, steps=4):
    grid, pops = cf.initial_state(cfg)
    ctx = abi.Context(lib, cf.params(cfg), cf.species(cfg), capacity=[p[1].shape[0] + 512 for p in pops])
    try:
        if path is not None:
            ctx.set_path(path)
        load(ctx, cfg, grid, pops)
        ctx.set_grid_counters(True)
        ctx.step(steps)
        return check_planes_against_log_counters(ctx, ctx.nspecies)
    finally:
        ctx.close()


def test_grid_counters_exact_path_equal_reference(ref_gc_lib):
    cfg = closed_box_config(**TIGHT)
    g = run(abi.gpu_library(), cfg, abi.PATH_EXACT)
    r = run(ref_gc_lib, cfg)
    for k in abi.GRID_COUNTERS:
        assert np.array_equal(g[k], r[k]), (k, g[k].sum(), r[k].sum())
        assert r[k].sum() > 0, k


@pytest.mark.parametrize("path", [abi.PATH_FAST, abi.PATH_FP32], ids=["fast", "fp32"])
def test_grid_counters_fast_paths(path):
    cfg = closed_box_config(**TIGHT)
    g = run(abi.gpu_library(), cfg, path)
    assert all(g[k].sum() > 0 for k in abi.GRID_COUNTERS)


def test_grid_counters_off_by_default():
    cfg = closed_box_config()
    grid, pops = cf.initial_state(cfg)
    ctx = abi.Context(abi.gpu_library(), cf.params(cfg), cf.species(cfg), capacity=[p[1].shape[0] + 512 for p in pops])
    try:
        load(ctx, cfg, grid, pops)
        ctx.step(1)
        with pytest.raises(abi.RhError):
            ctx.grid_counters()
    finally:
        ctx.close()
