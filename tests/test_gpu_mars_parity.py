"""Parity at the geometry of the Mars-like workload, reduced in size.

The benchmark workload (120x160x160 cells of 300 km) is too large for the
reference's CPU sources in a test, so this runs the same setup on 30x40x40
cells of 1200 km (1.5 million ions): a resolved absorbing sphere, solar wind
H+ at 30 ppc with He++ at 1.5 ppc, closed walls with the IMF on the +x wall,
and the hot-path settings of examples/mars.cfg on top of the workload's
(field and particle obstacle radii, gravity, the laminar-flow IMF draping,
the IMF and its wall flags, electron pressure, the grid-unit
superconducting-sphere resistivity, the constraints and linear E
smoothing). Twenty steps.

The escape and impact counters are FP64 sums that the GPU forms with atomics,
in no fixed order. Here about 4e5 particle weights leave the box in 20 steps,
so two orders of the same sum may differ by up to n eps = 4e5 x 1.1e-16 =
4.4e-11 relative: those counters are compared at 1e-10.

  exact path  bit for bit against the reference's own sources built here
              (oracle/_ref/librhref.so): particles, every grid array, the
              integer counters
  fast path   bit for bit against the oracle's restatement of its order, and
              within 1e-12 relative of the reference build, particles compared
              per cell in canonical order
"""
import dataclasses

import pytest

from rhybrid_b200 import abi
from rhybrid_b200 import config as cf

from harness import assert_state_equal, canonical_order, run

pytestmark = pytest.mark.gpu

STEPS = 20
SUM_RTOL = 1e-10   # the atomically summed escape/impact counters (see above)


def mars_reduced():
    cfg = cf.config_mars(nx=30, ny=40, nz=40, dx=1200e3)
    pops = [dataclasses.replace(p, obstacle=3590e3) for p in cfg.populations]
    return cfg.replace(populations=pops, R_fieldObstacle=3690e3, R_particleObstacle=3590e3,
                       use_gravity=True, M_object=0.64169e24,
                       b_profile="laminarFlowAroundSphereBx", laminar_R=3690e3,
                       imf=(-1.82e-9, 2.79e-9, 0.0), imf_boundary_cellB=(1, 0, 0, 0, 0, 0),
                       imf_boundary_faceB=(1, 0, 0, 0, 0, 0),
                       electron_temperature=1e4, electron_gamma=2, R_zeroElectronPressure=-100.0,
                       resistivity_profile="resistivitySuperConductingSphere", resistivity_unit="grid",
                       resistivity_value=0.02, resistivity_R=3690e3,
                       max_ion_velocity=5000e3, max_electron_velocity=5000e3, max_whistler_velocity=5000e3,
                       min_ion_charge_density_relative=0.05, max_electric_field=-100.0,
                       electric_field_linear_smoothing_number=1, name="mars_reduced_30x40x40")


@pytest.fixture(scope="module")
def gpu_lib():
    return abi.gpu_library()


@pytest.fixture(scope="module")
def reference_state(ref_lib):
    if ref_lib is None:
        pytest.skip("reference build (oracle/_ref/librhref.so) not present")
    return run(ref_lib, mars_reduced(), STEPS)


def test_mars_geometry_exact_path_bitwise_vs_reference_build(gpu_lib, reference_state):
    cfg = mars_reduced()
    st = run(gpu_lib, cfg, STEPS)
    assert sum(int(c.sum()) for c, _ in st["particles"]) > 1_000_000
    assert st["counters"]["particleImpact[0]"] > 0, "the sphere must absorb particles in 20 steps"
    assert_state_equal(st, reference_state, "Mars geometry, exact path vs reference build", sum_rtol=SUM_RTOL)


def test_mars_geometry_fast_path(gpu_lib, port_lib, reference_state):
    cfg = mars_reduced()
    fast = run(gpu_lib, cfg, STEPS, fast=True)
    assert_state_equal(fast, run(port_lib, cfg, STEPS, fast=True), "Mars geometry, fast path vs oracle fast order",
                       sum_rtol=SUM_RTOL)
    assert_state_equal(canonical_order(fast), canonical_order(reference_state),
                       "Mars geometry, fast path vs reference build", bitwise=False, rtol=1e-12, sum_rtol=SUM_RTOL)
