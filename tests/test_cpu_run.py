"""The .cfg-driven time loop (rhybrid_b200/run.py) on the reference build
(the library's ABI without a GPU): logs every log_interval steps before the
step, states with the temporal averages at every data save step."""
import numpy as np

from rhybrid_b200 import run as R
from rhybrid_b200 import vlsv as V

from test_cpu_cfg import TEXT


def test_run_loop(tmp_path, ref_lib):
    text = TEXT.replace("injector.name = SolarWindInjector", "injector.name = UniformInjector")
    text = text.replace("particle.population.exosphere = exoO+\n", "").replace("particle.population.ionosphere = ionoO+\n", "")
    text = text.replace("log_interval = 5", "log_interval = 2").replace("maximum_timesteps = 200",
                                                                        "maximum_timesteps = 6\ndata_save_interval = 3")
    f = tmp_path / "run.cfg"
    f.write_text(text)
    out = tmp_path / "out"
    r = R.run(str(f), out_dir=str(out), lib=ref_lib, quiet=True)
    assert r["steps"] == 6 and not r["stopped"] and len(r["saved"]) == 2
    field = [ln for ln in open(out / "field.log") if not ln.startswith("%")]
    assert len(field) == 3   # time steps 0, 2, 4
    st = V.load_state(r["saved"][1])
    assert r["saved"][1].endswith("state_0000006.vlsv")
    assert int(st["timestep"]) == 6 and st["cellB"].shape == (24 * 16 * 12, 3)
    assert np.array_equal(st["CellID"], np.arange(24 * 16 * 12))
    # Hybrid.output_parameters = cellB n_ave v_ave: ne comes with the averages (operator_userdata.cpp:104-116)
    assert sorted(st) == sorted(["CellID", "cellB", "ne", "n_H+_ave", "v_H+_ave", "time", "timestep"])
    assert st["n_H+_ave"].shape == (24 * 16 * 12,) and np.any(st["n_H+_ave"] > 0)
