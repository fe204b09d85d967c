"""The .cfg-driven time loop (rhybrid_b200/run.py) on the reference build
(the library's ABI without a GPU): logs every log_interval steps before the
step, states with the temporal averages at every data save step."""
import os

import numpy as np
import pytest

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


def test_run_reduced_state(tmp_path, ref_lib):
    """Hybrid.save_reduced_state_*: reduced<timestep>.vlsv every interval
    steps with cellB of every Nstride-th cell and, with particles, those
    cells' particles (diagnostics.h:819-960), equal to the full state's."""
    text = TEXT.replace("injector.name = SolarWindInjector", "injector.name = UniformInjector")
    text = text.replace("particle.population.exosphere = exoO+\n", "").replace("particle.population.ionosphere = ionoO+\n", "")
    text = text.replace("maximum_timesteps = 200", "maximum_timesteps = 3\ndata_save_interval = 3")
    text = text.replace("[Hybrid]", "[Hybrid]\nsave_reduced_state_interval = 3\nsave_reduced_state_Nstride = 4\n"
                        "save_reduced_state_include_particles = 1\nsave_particles = 1\nsave_particles_Nstride = 4")
    f = tmp_path / "run.cfg"
    f.write_text(text)
    r = R.run(str(f), out_dir=str(tmp_path), lib=ref_lib, quiet=True)
    assert [os.path.basename(p) for p in r["reduced"]] == ["reduced00000003.vlsv"]
    st = V.load_state(r["saved"][0])
    raw = V.read(r["reduced"][0])
    par = {n: a for (tag, n, m), a in raw.items() if tag == "PARAMETER"}
    assert int(par["timestep"][0]) == 3 and int(par["Nstride"][0]) == 4 and par["time"][0] == st["time"]
    nx, ny, nz = 24, 16, 12
    cid = np.arange(nx * ny * nz)
    keep = (cid % 4 == 0) & (cid % (4 * nx) < nx) & (cid % (4 * nx * ny) < nx * ny)
    ids = raw[("VARIABLE", "CellID", "ReducedPointMesh")]
    assert np.array_equal(ids, cid[keep]) and ids.dtype == np.uint32
    assert np.array_equal(raw[("VARIABLE", "cellB", "ReducedPointMesh")], st["cellB"][keep])
    names = [k.split("ParticlePointMesh_", 1)[1] for k in st if k.startswith("ParticlePointMesh_") and "/" not in k]
    assert names
    for name in names:
        mesh = f"ReducedParticlePointMesh_{name}"
        assert np.array_equal(raw[("VARIABLE", f"CellID_{name}", mesh)], st[f"ParticlePointMesh_{name}/CellID_{name}"])
        assert np.array_equal(raw[("VARIABLE", f"v_{name}", mesh)], st[f"ParticlePointMesh_{name}/v_{name}"])


def test_run_save_window(tmp_path, ref_lib):
    """Hybrid.data_save_all_timesteps_t_start/end: a state after every step
    that starts inside the window (user.cpp:66-71), the regular interval
    elsewhere; a window ending before it starts is refused (user.cpp:2381)."""
    from rhybrid_b200 import cfg as C
    text = TEXT.replace("injector.name = SolarWindInjector", "injector.name = UniformInjector")
    text = text.replace("particle.population.exosphere = exoO+\n", "").replace("particle.population.ionosphere = ionoO+\n", "")
    text = text.replace("maximum_timesteps = 200", "maximum_timesteps = 8\ndata_save_interval = 4")
    win = text.replace("[Hybrid]", "[Hybrid]\ndata_save_all_timesteps_t_start = 0.09\ndata_save_all_timesteps_t_end = 0.17")
    f = tmp_path / "run.cfg"
    f.write_text(win)
    r = R.run(str(f), out_dir=str(tmp_path), lib=ref_lib, quiet=True)
    assert [os.path.basename(p) for p in r["saved"]] == ["state_0000004.vlsv", "state_0000005.vlsv",
                                                         "state_0000008.vlsv"]
    bad = text.replace("[Hybrid]", "[Hybrid]\ndata_save_all_timesteps_t_start = 0.2\ndata_save_all_timesteps_t_end = 0.1")
    with pytest.raises(ValueError):
        C.load_text(bad)
    _, rs = C.load_text(text.replace("[Hybrid]", "[Hybrid]\ndata_save_all_timesteps_t_start = -1\ndata_save_all_timesteps_t_end = 0.3"))
    assert rs.data_save_all_timesteps_t_start == -1.0 and rs.data_save_all_timesteps_t_end == -1.0
