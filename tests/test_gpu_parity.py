"""GPU parity: the B200 library (through its C ABI) against the oracle
restatement, which tests/test_oracle_pin.py pins bit for bit to the
reference's own sources.

Exact path (RHGPU_PATH_EXACT): the reference's particle order and summation
order; particle state, every grid array and the integer counters are
compared bitwise with the oracle in reference order.
Fast path (RHGPU_PATH_FAST, the default): particles stored by CIC dual cell,
its own deterministic deposit order; bitwise against the oracle's
restatement of that order, and within 1e-12 relative of the reference order.
Both: the FP64 escape/impact sums, accumulated with atomics on the GPU,
to 1e-12 relative."""
import dataclasses

import numpy as np
import pytest

from rhybrid_b200 import abi
from rhybrid_b200 import config as cf

from harness import (assert_state_equal, canonical_order, closed_box_config, load, rel_err, run,
                     snapshot)

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def gpu_lib():
    return abi.gpu_library()


def test_periodic_box_bitwise(gpu_lib, port_lib):
    cfg = cf.config_empty_box(8, 8, 8, ppc=4.0)
    assert_state_equal(run(gpu_lib, cfg, 25), run(port_lib, cfg, 25), "periodic 8^3")


def test_closed_box_bitwise_every_step(gpu_lib, port_lib):
    cfg = closed_box_config()
    a = run(gpu_lib, cfg, 8, per_step=True)
    b = run(port_lib, cfg, 8, per_step=True)
    for n, (x, y) in enumerate(zip(a, b)):
        assert_state_equal(x, y, f"closed box step {n + 1}")


@pytest.mark.parametrize("variant", ["isothermal_no_hall", "gravity_flowthrough", "mixed_periodic"])
def test_option_variants_bitwise(gpu_lib, port_lib, variant):
    if variant == "isothermal_no_hall":
        cfg = closed_box_config(electron_gamma=1, use_hall_term=False, electric_field_linear_smoothing_number=2,
                                electric_field_smoothing_gauss_sigma=0.0, periodic=(1, 0, 1))
    elif variant == "gravity_flowthrough":
        cfg = closed_box_config(use_gravity=True, M_object=6.4e28, initial_flow_throughs=0.02,
                                periodic=(0, 1, 0), max_electric_field=-1)
    else:
        cfg = closed_box_config(nx=9, ny=7, nz=11, periodic=(0, 0, 1), ppc=6.0)
    assert_state_equal(run(gpu_lib, cfg, 6), run(port_lib, cfg, 6), variant)


def test_empty_box_32cubed_100_steps(gpu_lib, port_lib):
    """The plain FP64 periodic empty box (32^3 cells, 20 ppc, 655,360 ions,
    100 steps of dt=0.01 s): identical particle state and moments."""
    cfg = cf.config_empty_box(32, 32, 32, ppc=20.0)
    assert_state_equal(run(gpu_lib, cfg, 100), run(port_lib, cfg, 100), "empty box 32^3")


@pytest.mark.parametrize("fast", [False, True], ids=["exact", "fast"])
def test_split_entry_points_match_step(gpu_lib, port_lib, fast):
    """push / accumulate / apply_boundaries / propagate_fields one at a time."""
    cfg = closed_box_config()
    grid, pops = cf.initial_state(cfg)
    cap = [int(1.5 * p[1].shape[0]) + 64 for p in pops]
    ctxs = [abi.Context(lib, cf.params(cfg), cf.species(cfg), capacity=cap) for lib in (gpu_lib, port_lib)]
    try:
        for c in ctxs:
            c.select_path(fast)
            load(c, cfg, grid, pops)
        for phase in ["push", "accumulate", "apply_boundaries", "propagate_fields"] * 3:
            for c in ctxs:
                getattr(c, phase)()
            assert_state_equal(snapshot(ctxs[0]), snapshot(ctxs[1]), phase)
    finally:
        for c in ctxs:
            c.close()


def test_field_update_alone_random_moments(gpu_lib, port_lib):
    """propagateB on random moments and fields, closed box with obstacle and
    every option: all grid arrays bitwise."""
    cfg = closed_box_config(nx=10, ny=9, nz=8)
    grid, pops = cf.initial_state(cfg)
    rng = np.random.default_rng(7)
    N = cfg.ncells
    arrays = {
        "faceB": rng.normal(0, 5e-9, (N, 3)), "cellB": rng.normal(0, 5e-9, (N, 3)),
        "cellRhoQi": rng.uniform(0.2, 2.0, N) * 2e6 * abi.CHARGE_ELEMENTARY,
        "cellJi": rng.normal(0, 1e-7, (N, 3)), "cellUe": rng.normal(0, 1e5, (N, 3)),
        "nodeEta": grid["nodeEta"], "cellAverageB": rng.normal(0, 1e-9, (N, 3)),
    }
    ctxs = [abi.Context(lib, cf.params(cfg), cf.species(cfg), capacity=[1, 1]) for lib in (gpu_lib, port_lib)]
    try:
        for c in ctxs:
            for name, a in arrays.items():
                c.upload_array(name, a)
            c.upload_cell_flags(grid["flags"])
            for _ in range(3):
                c.propagate_fields()
        assert_state_equal(snapshot(ctxs[0]), snapshot(ctxs[1]), "propagate_fields")
    finally:
        for c in ctxs:
            c.close()


@pytest.mark.parametrize("fast", [False, True], ids=["exact", "fast"])
def test_deterministic(gpu_lib, fast):
    cfg = closed_box_config()
    a = run(gpu_lib, cfg, 5, fast=fast)
    b = run(gpu_lib, cfg, 5, fast=fast)
    assert_state_equal(a, b, "two GPU runs", sum_rtol=1e-12)


@pytest.mark.parametrize("fast", [False, True], ids=["exact", "fast"])
def test_charge_conservation_known_answer(gpu_lib, fast):
    """The reference's accumulation test (examples/test_accumulation_sum_grid.py):
    the deposited charge summed over the periodic grid equals the total
    macroparticle charge, sum(rho)*dV == sum(w)*q."""
    cfg = cf.config_empty_box(12, 10, 8, ppc=7.0).replace(min_ion_charge_density_relative=0.0)
    grid, pops = cf.initial_state(cfg)
    ctx = abi.Context(gpu_lib, cf.params(cfg), cf.species(cfg), capacity=[pops[0][1].shape[0] + 64])
    try:
        ctx.select_path(fast)
        load(ctx, cfg, grid, pops)
        ctx.push()
        ctx.accumulate()
        rho = ctx.download_array("cellRhoQi")
        _, p = ctx.download_particles(0)
        total = p[:, 6].sum() * cfg.populations[0].q
        assert abs(rho.sum() * cfg.dx ** 3 - total) <= 1e-13 * total
    finally:
        ctx.close()


@pytest.mark.parametrize("fast", [False, True], ids=["exact", "fast"])
def test_particle_upload_download_roundtrip(gpu_lib, fast):
    """Exact path: the same particles in the same order. Fast path: the same
    particles per cell (stored by dual cell, so the per-cell order may change)."""
    cfg = closed_box_config()
    grid, pops = cf.initial_state(cfg)
    ctx = abi.Context(gpu_lib, cf.params(cfg), cf.species(cfg), capacity=[p[1].shape[0] for p in pops])
    try:
        ctx.select_path(fast)
        load(ctx, cfg, grid, pops)
        for s, (cnt, p) in enumerate(pops):
            c2, p2 = ctx.download_particles(s)
            assert np.array_equal(cnt, c2)
            if fast:
                a = canonical_order({"particles": [(cnt, p)]})["particles"][0][1]
                b = canonical_order({"particles": [(c2, p2)]})["particles"][0][1]
                assert np.array_equal(a.view(np.uint64), b.view(np.uint64))
            else:
                assert np.array_equal(p.view(np.uint64), p2.view(np.uint64))
        for name in ("faceB", "cellB", "nodeEta"):
            assert np.array_equal(ctx.download_array(name).reshape(-1), np.asarray(grid[name]).reshape(-1))
    finally:
        ctx.close()


@pytest.mark.parametrize("fast", [False, True], ids=["exact", "fast"])
def test_nonfinite_particle_raises_device_error(gpu_lib, fast):
    """Failure detection without a GPU fault: a corrupted particle (NaN
    velocity) is uploaded from the host; the push raises the device error word
    and rhgpu_step returns RHGPU_ERR_DEVICE; the context stays usable."""
    cfg = cf.config_empty_box(6, 6, 6, ppc=2.0)
    grid, pops = cf.initial_state(cfg)
    cnt, p = pops[0]
    p = p.copy()
    p[5, 3] = np.nan
    ctx = abi.Context(gpu_lib, cf.params(cfg), cf.species(cfg), capacity=[p.shape[0] + 8])
    try:
        ctx.select_path(fast)
        load(ctx, cfg, grid, [(cnt, p)])
        with pytest.raises(abi.RhError) as ei:
            ctx.step(1)
        assert ei.value.code == abi.ERR_DEVICE
        assert ctx.device_errors() & abi.DEVERR_NAN_PARTICLE
        c2, p2 = ctx.download_particles(0)
        assert c2.sum() == cnt.sum()
    finally:
        ctx.close()


@pytest.mark.parametrize("fast", [False, True], ids=["exact", "fast"])
def test_capacity_is_enforced(gpu_lib, fast):
    cfg = cf.config_empty_box(6, 6, 6, ppc=2.0)
    grid, pops = cf.initial_state(cfg)
    ctx = abi.Context(gpu_lib, cf.params(cfg), cf.species(cfg), capacity=[10])
    try:
        ctx.select_path(fast)
        with pytest.raises(abi.RhError) as ei:
            ctx.upload_particles(0, *pops[0])
        assert ei.value.code == abi.ERR_CAPACITY
    finally:
        ctx.close()


# ---- fast path ------------------------------------------------------------

def test_fast_periodic_box_bitwise(gpu_lib, port_lib):
    cfg = cf.config_empty_box(8, 8, 8, ppc=4.0)
    assert_state_equal(run(gpu_lib, cfg, 25, fast=True), run(port_lib, cfg, 25, fast=True), "fast periodic 8^3")


def test_fast_closed_box_bitwise_every_step(gpu_lib, port_lib):
    cfg = closed_box_config()
    a = run(gpu_lib, cfg, 8, per_step=True, fast=True)
    b = run(port_lib, cfg, 8, per_step=True, fast=True)
    for n, (x, y) in enumerate(zip(a, b)):
        assert_state_equal(x, y, f"fast closed box step {n + 1}")


@pytest.mark.parametrize("variant", ["isothermal_no_hall", "gravity_flowthrough", "mixed_periodic", "odd_sizes",
                                     "segments_walls", "segments_periodic"])
def test_fast_option_variants_bitwise(gpu_lib, port_lib, variant):
    """Option variants; the last two have rows of 3 storage segments (71 and
    70 dual cells), so particles cross segment boundaries."""
    if variant == "isothermal_no_hall":
        cfg = closed_box_config(electron_gamma=1, use_hall_term=False, electric_field_linear_smoothing_number=2,
                                electric_field_smoothing_gauss_sigma=0.0, periodic=(1, 0, 1))
    elif variant == "gravity_flowthrough":
        cfg = closed_box_config(use_gravity=True, M_object=6.4e28, initial_flow_throughs=0.02,
                                periodic=(0, 1, 0), max_electric_field=-1)
    elif variant == "mixed_periodic":
        cfg = closed_box_config(nx=9, ny=7, nz=11, periodic=(0, 0, 1), ppc=6.0)
    elif variant == "odd_sizes":
        cfg = closed_box_config(nx=37, ny=5, nz=3, periodic=(1, 1, 0), ppc=9.0)
    elif variant == "segments_walls":
        cfg = closed_box_config(nx=70, ny=5, nz=4, ppc=5.0)
    else:
        cfg = closed_box_config(nx=70, ny=4, nz=5, periodic=(1, 0, 1), ppc=5.0)
    assert_state_equal(run(gpu_lib, cfg, 6, fast=True), run(port_lib, cfg, 6, fast=True), "fast " + variant)


def test_fast_empty_box_32cubed_100_steps(gpu_lib, port_lib):
    """The fast path on the periodic 32^3 box (655,360 ions, 100 steps):
    bitwise against the oracle's restatement of the fast order, and within
    1e-12 relative of the reference order (particles compared per cell)."""
    cfg = cf.config_empty_box(32, 32, 32, ppc=20.0)
    fast = run(gpu_lib, cfg, 100, fast=True)
    assert_state_equal(fast, run(port_lib, cfg, 100, fast=True), "fast 32^3 vs oracle fast order")
    ref = run(port_lib, cfg, 100, fast=False)
    assert_state_equal(canonical_order(fast), canonical_order(ref), "fast 32^3 vs reference order",
                       bitwise=False, rtol=1e-12)


def test_fast_closed_box_vs_reference_order(gpu_lib, port_lib):
    """Walls, an absorbing sphere and two species for 20 steps: the fast path
    stays within 1e-12 relative of the reference order."""
    cfg = closed_box_config(nx=16, ny=14, nz=12, ppc=8.0)
    fast = run(gpu_lib, cfg, 20, fast=True)
    ref = run(port_lib, cfg, 20, fast=False)
    assert_state_equal(canonical_order(fast), canonical_order(ref), "fast closed box vs reference order",
                       bitwise=False, rtol=1e-12, sum_rtol=1e-12)


def test_fast_large_arrival_buckets_bitwise(gpu_lib, port_lib):
    """300 ppc of a hot plasma (1e7 K, 40 % of a cell per step) in a small
    periodic box: hundreds of particles arrive in each destination segment per
    step, more than one thread orders, so each destination's movers are ordered
    by one block in shared memory; bitwise with the oracle."""
    cfg = cf.config_empty_box(8, 6, 5, ppc=300.0).replace(dt=0.1)
    cfg = cfg.replace(populations=[dataclasses.replace(cfg.populations[0], temperature=1e7)])
    assert_state_equal(run(gpu_lib, cfg, 4, fast=True), run(port_lib, cfg, 4, fast=True), "fast 300 ppc hot")


def test_fast_huge_arrival_buckets_bitwise(gpu_lib, port_lib):
    """3000 ppc of the same plasma: thousands of arrivals per destination
    segment, more than one block orders, so the movers are placed through the
    two radix sorts over all of them; bitwise with the oracle."""
    cfg = cf.config_empty_box(8, 6, 5, ppc=3000.0).replace(dt=0.1)
    cfg = cfg.replace(populations=[dataclasses.replace(cfg.populations[0], temperature=1e7)])
    assert_state_equal(run(gpu_lib, cfg, 3, fast=True), run(port_lib, cfg, 3, fast=True), "fast 3000 ppc hot")


def test_fast_segment_overflow_relayout(gpu_lib, port_lib):
    """Two cold beams converging in y pile up more particles in the middle
    dual rows than their segments' slack holds: the mover placement overflows,
    the storage is relaid out, and the result stays bitwise with the oracle."""
    cfg = cf.config_empty_box(16, 16, 4, ppc=12.0).replace(dt=0.06)
    cfg = cfg.replace(populations=[dataclasses.replace(cfg.populations[0], temperature=1e2)])
    grid, pops = cf.initial_state(cfg)
    cnt, p = pops[0]
    p = p.copy()
    j = (np.repeat(np.arange(cnt.size), cnt.astype(np.int64)) // cfg.nx) % cfg.ny
    p[:, 4] = np.where(j < cfg.ny // 2, 1.2e6, -1.2e6)
    pops = [(cnt, p)]
    a = run(gpu_lib, cfg, 12, grid=grid, pops=pops, fast=True)
    b = run(port_lib, cfg, 12, grid=grid, pops=pops, fast=True)
    assert_state_equal(a, b, "fast converging beams")
    assert a["particles"][0][0].max() > 1.5 * cnt.max()


def test_fast_relayout_of_one_species(gpu_lib, port_lib):
    """Only the species whose arrivals overflow their segments is relaid out:
    converging cold beams of one species beside a second, slow population whose
    segments keep their layout; bitwise with the oracle (which has no layout)."""
    cfg = cf.config_empty_box(16, 16, 4, ppc=12.0).replace(dt=0.06)
    beam = dataclasses.replace(cfg.populations[0], temperature=1e2)
    slow = dataclasses.replace(cfg.populations[0], name="slow", ppc=4.0, temperature=1e3, velocity=(0.0, 0.0, 0.0))
    cfg = cfg.replace(populations=[beam, slow])
    grid, pops = cf.initial_state(cfg)
    cnt, p = pops[0]
    p = p.copy()
    j = (np.repeat(np.arange(cnt.size), cnt.astype(np.int64)) // cfg.nx) % cfg.ny
    p[:, 4] = np.where(j < cfg.ny // 2, 1.2e6, -1.2e6)
    pops = [(cnt, p), pops[1]]
    a = run(gpu_lib, cfg, 12, grid=grid, pops=pops, fast=True)
    b = run(port_lib, cfg, 12, grid=grid, pops=pops, fast=True)
    assert_state_equal(a, b, "fast converging beams beside a slow population")
    assert a["particles"][0][0].max() > 1.5 * cnt.max()
