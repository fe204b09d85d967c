"""Parity at the geometry of the Mercury-like workload, reduced in size.

The workload of the FP32 form (320^3 cells of 100 km, 1.3e9 ions) is far too
large for the reference's CPU sources in a test, so this runs its setup on
32^3 cells of 400 km (1.3 million ions): the dipole of 190 nT at 2440 km
with the IMF Bx draped around an 1800 km sphere
(translateDipoleBAndLaminarFlowAroundSphereBx), the absorbing planet, solar
wind H+ at 40 ppc, the IMF (2, 0, -10) nT on the +x wall, electron pressure
with gamma 2, the superconducting-core resistivity in units of Rm with the
10x coefficient on the +y outer cells, and the workload's constraints (ion,
electron and whistler speeds, E). Twenty steps.

The escape and impact counters are FP64 sums that the GPU forms with atomics
in no fixed order; they are compared at n eps (1e-10 relative), as in the
Mars-geometry test.

  exact path  bit for bit against the reference's own sources built here
              (oracle/_ref/librhref.so): particles, every grid array, the
              integer counters
  fast path   bit for bit against the oracle's restatement of its order, and
              within 1e-12 relative of the reference build, particles compared
              per cell in canonical order
"""
import pytest

from rhybrid_b200 import abi
from rhybrid_b200 import config as cf

from harness import assert_state_equal, canonical_order, run

pytestmark = pytest.mark.gpu

STEPS = 20
SUM_RTOL = 1e-10   # the atomically summed escape/impact counters


def mercury_reduced():
    cfg = cf.config_mercury(nx=32, ny=32, nz=32, ppc=40.0, dx=400e3)
    return cfg.replace(name="mercury_reduced_32cubed")


@pytest.fixture(scope="module")
def gpu_lib():
    return abi.gpu_library()


@pytest.fixture(scope="module")
def reference_state(ref_lib):
    if ref_lib is None:
        pytest.skip("reference build (oracle/_ref/librhref.so) not present")
    return run(ref_lib, mercury_reduced(), STEPS)


def test_mercury_geometry_exact_path_bitwise_vs_reference_build(gpu_lib, reference_state):
    st = run(gpu_lib, mercury_reduced(), STEPS)
    assert sum(int(c.sum()) for c, _ in st["particles"]) > 1_000_000
    assert st["counters"]["particleImpact[0]"] > 0, "the planet must absorb particles in 20 steps"
    assert_state_equal(st, reference_state, "Mercury geometry, exact path vs reference build", sum_rtol=SUM_RTOL)


def test_mercury_geometry_fast_path(gpu_lib, port_lib, reference_state):
    cfg = mercury_reduced()
    fast = run(gpu_lib, cfg, STEPS, fast=True)
    assert_state_equal(fast, run(port_lib, cfg, STEPS, fast=True),
                       "Mercury geometry, fast path vs oracle fast order", sum_rtol=SUM_RTOL)
    assert_state_equal(canonical_order(fast), canonical_order(reference_state),
                       "Mercury geometry, fast path vs reference build", bitwise=False, rtol=1e-12, sum_rtol=SUM_RTOL)
