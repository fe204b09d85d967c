"""The reference's own log writer (diagnostics::logWriteParticleField, built
from the reference's sources in oracle/_ref) as the oracle of the log files:
it runs on the oracle's state, writes 17 particle-log and 41 field-log
columns per line, starts the scales at their sentinels, stops on max |B| and
zeroes its counters after each line."""
import pytest

from rhybrid_b200 import abi
from rhybrid_b200 import config as cf

from harness import closed_box_config, load


def lines(path):
    return [ln.rstrip("\n").split(" ") for ln in open(path) if not ln.startswith("%")]


def test_reference_log_writer(tmp_path, ref_lib):
    cfg = closed_box_config()
    grid, pops = cf.initial_state(cfg)
    ctx = abi.Context(ref_lib, cf.params(cfg), cf.species(cfg), capacity=[p[1].shape[0] + 256 for p in pops])
    try:
        load(ctx, cfg, grid, pops)
        ctx.log_open(str(tmp_path), ["H+sw", "O+"], max_B_stop_run=1.0)
        assert ctx.log_write() == (False, "")
        ctx.step(3)
        assert any(v > 0 for k, v in ctx.counters().items() if k != "gridTemporalAverageCounter")
        assert ctx.log_write() == (False, "")
        assert all(v == 0 for k, v in ctx.counters().items() if k != "gridTemporalAverageCounter")
        ctx.log_close()
        stop_dir = tmp_path / "stop"
        stop_dir.mkdir()
        ctx.log_open(str(stop_dir), ["H+sw", "O+"], max_B_stop_run=1e-12)
        assert ctx.log_write()[0] is True
        ctx.log_close()
    finally:
        ctx.close()
    fld = lines(tmp_path / "field.log")
    pop = lines(tmp_path / "pop001_H+sw.log")
    assert len(fld) == len(pop) == 2
    for ln in fld:
        assert len([t for t in ln if t]) == 41 and ln[-1] == "" and ln.index("") == 25
    for ln in pop:
        assert len([t for t in ln if t]) == 17 and ln[-1] == ""
    # at t = 0 no charge is deposited yet: the electron inertial lengths keep their start values
    assert fld[0][35] == "+1.7976931349e+308" and fld[0][36] == "-1.7976931349e+308"
    assert float(fld[1][35]) > 0 and float(fld[1][0]) == pytest.approx(3 * cfg.dt)
