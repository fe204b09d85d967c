"""Pins the C restatement (oracle/rh_oracle.c) bit for bit against RHybrid's
own hot-path sources compiled through oracle/shim (the reference itself, run
here). The reference publishes no golden vectors (its tests are statistical,
tests/run_tests.py); these runs are the known answers, and
tests/golden/make_golden.py freezes some of them as fixtures."""
import pytest

from rhybrid_b200 import config as cf

from harness import assert_bitwise, closed_box_config, run


def test_periodic_box_matches_reference(port_lib, ref_lib):
    cfg = cf.config_empty_box(8, 8, 8, ppc=4.0)
    a = run(port_lib, cfg, 25)
    b = run(ref_lib, cfg, 25)
    assert_bitwise(a, b, "periodic box")


def test_closed_box_all_options_matches_reference(port_lib, ref_lib):
    cfg = closed_box_config()
    a = run(port_lib, cfg, 8, per_step=True)
    b = run(ref_lib, cfg, 8, per_step=True)
    for n, (x, y) in enumerate(zip(a, b)):
        assert_bitwise(x, y, f"closed box step {n + 1}")


@pytest.mark.parametrize("variant", ["isothermal_no_hall", "gravity_flowthrough"])
def test_option_variants_match_reference(port_lib, ref_lib, variant):
    if variant == "isothermal_no_hall":
        cfg = closed_box_config(electron_gamma=1, use_hall_term=False, electric_field_linear_smoothing_number=2,
                                electric_field_smoothing_gauss_sigma=0.0, periodic=(1, 0, 1))
    else:
        cfg = closed_box_config(use_gravity=True, M_object=6.4e23 * 1e5, initial_flow_throughs=0.02,
                                periodic=(0, 1, 0), max_electric_field=-1)
    a = run(port_lib, cfg, 6)
    b = run(ref_lib, cfg, 6)
    assert_bitwise(a, b, variant)
