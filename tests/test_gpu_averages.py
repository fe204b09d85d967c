"""Temporal averages of the output populations (rhgpu_set_population_averages,
rhgpu_output_averages) against the reference's own sums (accumulateCell,
particle_accumulator.cpp:148-150, built in oracle/_ref) and its output step
(operator_userdata.cpp:155-223): bit for bit on the exact path, to round-off
on the fast path; the sums and the counter restart after an output."""
import numpy as np
import pytest

from rhybrid_b200 import abi
from rhybrid_b200 import config as cf

from harness import closed_box_config, load

pytestmark = pytest.mark.gpu


def run(lib, cfg, groups, path=None, steps=(3, 2)):
    grid, pops = cf.initial_state(cfg)
    ctx = abi.Context(lib, cf.params(cfg), cf.species(cfg), capacity=[p[1].shape[0] + 512 for p in pops])
    outs = []
    try:
        if path is not None:
            ctx.set_path(path)
        load(ctx, cfg, grid, pops)
        ctx.set_population_averages(groups)
        for n in steps:
            ctx.step(n)
            outs.append(ctx.output_averages())
    finally:
        ctx.close()
    return outs


@pytest.mark.parametrize("groups", [[0, 1], [0, 0], [-1, 0]], ids=["two", "shared", "one"])
def test_averages_exact_path_bitwise(ref_lib, groups):
    cfg = closed_box_config()
    g = run(abi.gpu_library(), cfg, groups, abi.PATH_EXACT)
    r = run(ref_lib, cfg, groups)
    for og, orr in zip(g, r):
        for k in ("cellBAverage", "n_ave", "v_ave"):
            assert np.array_equal(og[k].view(np.uint64), orr[k].view(np.uint64)), k
    assert np.any(g[0]["n_ave"]) and np.any(g[1]["v_ave"])


def test_averages_fast_path(ref_lib):
    cfg = closed_box_config()
    g = run(abi.gpu_library(), cfg, [0, 1], abi.PATH_FAST)
    r = run(ref_lib, cfg, [0, 1])
    for og, orr in zip(g, r):
        assert np.allclose(og["cellBAverage"], orr["cellBAverage"], rtol=1e-11, atol=1e-11 * np.abs(orr["cellBAverage"]).max())
        for grp in range(2):
            n, m = og["n_ave"][grp], orr["n_ave"][grp]
            scale = np.abs(m).max()
            assert scale > 0 and np.abs(n - m).max() <= 1e-11 * scale
            dense = np.abs(m) > 1e-3 * scale
            v, w = og["v_ave"][grp][dense], orr["v_ave"][grp][dense]
            assert np.abs(v - w).max() <= 1e-9 * np.abs(w).max()


def test_averages_refused_on_fp32():
    cfg = closed_box_config()
    grid, pops = cf.initial_state(cfg)
    ctx = abi.Context(abi.gpu_library(), cf.params(cfg), cf.species(cfg), capacity=[p[1].shape[0] + 512 for p in pops])
    try:
        ctx.set_path(abi.PATH_FP32)
        with pytest.raises(abi.RhError):
            ctx.set_population_averages([0, 0])
    finally:
        ctx.close()
