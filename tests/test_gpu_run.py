"""The .cfg-driven time loop (rhybrid_b200/run.py) on the GPU with solar wind,
exosphere and ionosphere sources, log files, and saved states holding the
temporal averages and the sources' production rates."""
import numpy as np
import pytest

from rhybrid_b200 import abi
from rhybrid_b200 import cfg as C
from rhybrid_b200 import config as cf
from rhybrid_b200 import run as R
from rhybrid_b200 import vlsv as V

from test_cpu_cfg import TEXT

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("path", ["fast", "fp32"])
def test_run_loop_gpu(tmp_path, path):
    text = TEXT.replace("log_interval = 5", "log_interval = 2").replace(
        "maximum_timesteps = 200", "maximum_timesteps = 6\ndata_save_interval = 3").replace(
        "output_parameters = cellB n_ave v_ave", "output_parameters = cellB n_ave v_ave prod_rate_exo prod_rate_iono")
    f = tmp_path / "run.cfg"
    f.write_text(text)
    out = tmp_path / "out"
    r = R.run(str(f), out_dir=str(out), path=path, quiet=True)
    assert r["steps"] == 6 and not r["stopped"] and len(r["saved"]) == 2
    assert len([ln for ln in open(out / "field.log") if not ln.startswith("%")]) == 3
    pop = [ln.split() for ln in open(out / "pop001_swH+.log") if not ln.startswith("%")]
    assert float(pop[-1][2]) > 0 and float(pop[-1][11]) > 0   # macroparticles, inject rate
    st = V.load_state(r["saved"][-1])
    assert np.all(np.isfinite(st["cellB"])) and np.all(np.isfinite(st["ne"]))
    # the sources' expected macroparticles per step: the ionosphere's add up to its
    # macroparticles per step, the exosphere's to at most that (shadow factor)
    c, _ = C.load(str(f))
    J = {j.type: j for j in cf.source_injectors(c, seed=c.seed)}
    for t, key, exact in ((abi.INJECT_IONOSPHERE, "prod_rate_iono0", True), (abi.INJECT_EXOSPHERE, "prod_rate_exo0", False)):
        j = J[t]
        per_dt = (j.macroparticles_per_cell_relative if j.macroparticles_per_cell_relative >= 0 else 1.0) * (
            j.upstream_macro_ratio if j.upstream_macro_ratio > 0 else 100.0)
        rate = st[key]
        assert rate.shape == (24 * 16 * 12,) and np.all(rate >= 0) and rate.sum() > 0
        assert abs(rate.sum() - per_dt) <= 1e-9 * per_dt if exact else rate.sum() <= per_dt * (1 + 1e-9)
    if path == "fast":   # the FP32 form keeps no population averages
        assert np.any(st["n_H+_ave"] > 0) and st["v_O+_ave"].shape == (24 * 16 * 12, 3)
