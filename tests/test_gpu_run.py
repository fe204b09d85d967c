"""The .cfg-driven time loop (rhybrid_b200/run.py) on the GPU with solar wind,
exosphere and ionosphere sources, log files and the temporal averages."""
import numpy as np
import pytest

from rhybrid_b200 import run as R

from test_cpu_cfg import TEXT

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("path", ["fast", "fp32"])
def test_run_loop_gpu(tmp_path, path):
    text = TEXT.replace("log_interval = 5", "log_interval = 2").replace(
        "maximum_timesteps = 200", "maximum_timesteps = 6\ndata_save_interval = 3")
    f = tmp_path / "run.cfg"
    f.write_text(text)
    out = tmp_path / "out"
    r = R.run(str(f), out_dir=str(out), path=path, quiet=True)
    assert r["steps"] == 6 and not r["stopped"] and len(r["saved"]) == 2
    assert len([ln for ln in open(out / "field.log") if not ln.startswith("%")]) == 3
    pop = [ln.split() for ln in open(out / "pop001_swH+.log") if not ln.startswith("%")]
    assert float(pop[-1][2]) > 0 and float(pop[-1][11]) > 0   # macroparticles, inject rate
    st = np.load(r["saved"][-1])
    assert np.all(np.isfinite(st["cellB"])) and np.all(np.isfinite(st["ne"]))
    if path == "fast":   # the FP32 form keeps no population averages
        assert np.any(st["n_H+_ave"] > 0) and st["v_O+_ave"].shape == (24 * 16 * 12, 3)
