"""The reference's temporal averages of the output populations as the
oracle: its own accumulateCell adds each step's charge and current sums
(particle_accumulator.cpp:148-150); the output step (restated in the oracle
driver from operator_userdata.cpp:155-223) divides by q dV and the step count.
With every species in one population, n_ave * q is the time mean of the
unclamped cellRhoQi (in the interior cells), and cellBAverage the time mean
of cellB."""
import numpy as np

from rhybrid_b200 import config as cf
from rhybrid_b200 import abi

from harness import closed_box_config, load


def test_reference_population_averages(ref_lib):
    cfg = closed_box_config()
    grid, pops = cf.initial_state(cfg)
    sp = cf.species(cfg)
    ctx = abi.Context(ref_lib, cf.params(cfg), sp, capacity=[p[1].shape[0] + 256 for p in pops])
    try:
        load(ctx, cfg, grid, pops)
        ctx.set_population_averages([0] * ctx.nspecies)
        rho, B = [], []
        for _ in range(4):
            ctx.step(1)
            rho.append(ctx.download_array("cellRhoQi").copy())
            B.append(ctx.download_array("cellB").copy())
        out = ctx.output_averages()
        assert ctx.counters()["gridTemporalAverageCounter"] == 0
        again = ctx.output_averages()
    finally:
        ctx.close()
    mean_rho = np.mean(rho, axis=0)
    minrho = cf.params(cfg).min_ion_charge_density
    # interior cells: the field update rewrites cellRhoQi in the exterior cells
    inner = np.zeros((cfg.nz, cfg.ny, cfg.nx), bool)
    inner[1:-1, 1:-1, 1:-1] = True
    free = np.all(np.array(rho) > minrho, axis=0) & inner.reshape(-1)
    assert free.sum() > 100
    got = out["n_ave"][0] * sp[0].q
    assert np.allclose(got[free], mean_rho[free], rtol=1e-12, atol=0)
    assert np.allclose(out["cellBAverage"], np.mean(B, axis=0), rtol=1e-12, atol=1e-25)
    # the sums and the counter restarted
    assert not np.any(again["n_ave"]) and not np.any(again["cellBAverage"])
