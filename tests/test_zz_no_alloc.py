"""rhgpu_accumulate_noalloc (the exact-path deposit with its scratch in static
device memory) against rhgpu_accumulate, through the C ABI."""
import numpy as np
import pytest

from rhybrid_b200 import abi
from rhybrid_b200 import config as cf

from harness import SUM_COUNTERS, closed_box_config, load

pytestmark = pytest.mark.gpu

MAX_CELLS = 16384   # RHGPU_NOALLOC_MAX_CELLS in include/rhgpu.h


def exact_context(lib, cfg, grid, pops):
    ctx = abi.Context(lib, cf.params(cfg), cf.species(cfg), capacity=[p[1].shape[0] + 256 for p in pops])
    ctx.set_path(abi.PATH_EXACT)
    load(ctx, cfg, grid, pops)
    return ctx


def test_noalloc_matches_accumulate_on_two_calls_in_a_row():
    cfg = closed_box_config()
    grid, pops = cf.initial_state(cfg)
    lib = abi.gpu_library()
    a = exact_context(lib, cfg, grid, pops)
    b = exact_context(lib, cfg, grid, pops)
    try:
        for call in range(2):
            a.push()
            b.push()
            a.accumulate()
            b.accumulate_noalloc()
            for name in ("cellRhoQi", "cellJi"):
                x, y = a.download_array(name), b.download_array(name)
                assert np.array_equal(x.view(np.uint64), y.view(np.uint64)), f"call {call + 1}: {name} differs"
            ca, cb = a.counters(), b.counters()
            for k, v in ca.items():
                if k.split("[")[0] in SUM_COUNTERS:   # FP64 sums of the push, accumulated with atomics
                    assert abs(v - cb[k]) <= 1e-12 * max(abs(v), 1e-300), k
                else:
                    assert v == cb[k], k
            assert b.device_errors() == 0
    finally:
        a.close()
        b.close()


def test_noalloc_rejects_a_grid_above_the_limit():
    cfg = cf.config_empty_box(32, 32, MAX_CELLS // (32 * 32) + 1, ppc=1.0)
    grid, pops = cf.initial_state(cfg)
    ctx = exact_context(abi.gpu_library(), cfg, grid, pops)
    try:
        with pytest.raises(abi.RhError) as ei:
            ctx.accumulate_noalloc()
        assert ei.value.code == abi.ERR_ARG
        assert "RHGPU_NOALLOC_MAX_CELLS" in str(ei.value)
    finally:
        ctx.close()


def test_noalloc_needs_the_exact_path():
    cfg = cf.config_empty_box(6, 6, 6, ppc=2.0)
    grid, pops = cf.initial_state(cfg)
    ctx = abi.Context(abi.gpu_library(), cf.params(cfg), cf.species(cfg), capacity=[pops[0][1].shape[0] + 64])
    try:
        load(ctx, cfg, grid, pops)
        with pytest.raises(abi.RhError) as ei:
            ctx.accumulate_noalloc()
        assert ei.value.code == abi.ERR_STATE
    finally:
        ctx.close()
