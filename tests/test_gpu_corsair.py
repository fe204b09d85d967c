"""The Corsair-side adaptor (rhybrid_b200/corsair/rhgpu_corsair.h), compiled
against the oracle's Corsair/ParGrid shim into oracle/_ref/librhref_corsair.so.

Its plugins are made through Corsair's object factories by the names a run's
.cfg uses (BorisBuneman, HybridAccumulator, HybridBoundaryCond), called the
way RHybrid's propagate() calls them, and its propagate() hook steps the GPU
library; the state comes back into the reference's ParGrid containers. On the
closed box (walls, an absorbing sphere, two species, every field option) it
must equal the GPU library driven directly through its C ABI, bit for bit,
on both particle paths."""
import numpy as np
import pytest

from oracle import oracle
from rhybrid_b200 import abi
from rhybrid_b200 import config as cf

from harness import STATE_ARRAYS, closed_box_config, load, run

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def corsair_lib():
    lib = oracle.reference_corsair()
    if lib is None:
        pytest.skip("oracle/_ref/librhref_corsair.so not built")
    return lib


@pytest.mark.parametrize("path", [abi.PATH_FAST, abi.PATH_EXACT])
def test_adaptor_matches_the_c_abi(corsair_lib, path):
    cfg = closed_box_config(nx=14, ny=12, nz=10, ppc=6.0)
    grid, pops = cf.initial_state(cfg)
    steps = 6
    direct = run(abi.gpu_library(), cfg, steps, grid=grid, pops=pops, fast=path == abi.PATH_FAST)
    ctx = abi.Context(corsair_lib, cf.params(cfg), cf.species(cfg))
    try:
        load(ctx, cfg, grid, pops)
        oracle.corsair_run(ctx, steps, path)
        for n in STATE_ARRAYS:
            a, b = ctx.download_array(n), direct["arrays"][n]
            assert np.array_equal(a.view(np.uint64), b.view(np.uint64)), f"{n} differs"
        for s in range(len(pops)):
            (ca, pa), (cb, pb) = ctx.download_particles(s), direct["particles"][s]
            assert np.array_equal(ca, cb), f"species {s} counts differ"
            assert np.array_equal(pa.view(np.uint64), pb.view(np.uint64)), f"species {s} particles differ"
        t, ts = ctx.time()
        assert ts == steps and abs(t - direct["time"][0]) <= 1e-12 * max(1.0, abs(t))
    finally:
        ctx.close()
