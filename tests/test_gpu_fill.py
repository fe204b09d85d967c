"""The uniform fill generated on the GPU (rhgpu_fill_uniform, the reference's
InjectorUniform::injectParticles, src/particle_injector.cpp:188-255) for the
fast path and the FP32 form: counts per cell, positions, weights and velocity
statistics, reproducibility, the region, and the same particle set in both
storages. The random stream is the library's own (Philox keyed by seed, cell
and particle index), so the checks are the injector's properties, as the
reference's own tests check populations statistically."""
import math

import numpy as np
import pytest

from rhybrid_b200 import abi
from rhybrid_b200 import config as cf

pytestmark = pytest.mark.gpu

N0, T, U, PPC = 4e6, 2e5, (-400e3, 30e3, 0.0), 24.0


def box(periodic=(0, 1, 0), nx=40, ny=7, nz=6):
    pop = cf.Population(name="H+", density=N0, velocity=U, temperature=T, ppc=PPC)
    return cf.Config(nx=nx, ny=ny, nz=nz, x_min=-0.5 * nx * 100e3, y_min=-0.5 * ny * 100e3,
                     z_min=-0.5 * nz * 100e3, dx=100e3, periodic=periodic, dt=0.02, populations=[pop],
                     name="fill_box")


def filled(lib, cfg, path, ppc=PPC, seed=3, region=None):
    grid, _ = cf.initial_state(cfg)
    ctx = abi.Context(lib, cf.params(cfg), cf.species(cfg))
    ctx.set_path(path)
    ctx.upload_array("faceB", grid["faceB"])
    ctx.upload_array("cellB", grid["cellB"])
    ctx.upload_array("nodeEta", grid["nodeEta"])
    ctx.upload_cell_flags(grid["flags"])
    ctx.fill_uniform(0, N0, T, U, ppc, seed=seed, region=region)
    return ctx


@pytest.fixture(scope="module")
def lib():
    return abi.gpu_library()


@pytest.mark.parametrize("periodic", [(0, 1, 0), (1, 1, 1)])
def test_fill_counts_positions_weights_velocities(lib, periodic):
    cfg = box(periodic)
    ctx = filled(lib, cfg, abi.PATH_FAST)
    try:
        cnt, p = ctx.download_particles(0)
    finally:
        ctx.close()
    assert np.all(cnt == PPC)   # an integer ppc: probRound is exact
    eps = 1e-4 * cfg.dx
    assert np.all(p[:, :3] >= 0.5 * eps * 0.999) and np.all(p[:, :3] <= cfg.dx - 0.5 * eps * 0.999)
    assert np.all(p[:, 6] == N0 * cfg.dx ** 3 / PPC)
    vth = math.sqrt(abi.BOLTZMANN * T / cfg.populations[0].m)
    n = p.shape[0]
    for a in range(3):
        m, sd = p[:, 3 + a].mean(), p[:, 3 + a].std()
        assert abs(m - U[a]) < 5 * vth / math.sqrt(n)
        assert abs(sd / vth - 1) < 5 / math.sqrt(2 * n)
    # positions uniform in the cell: each half of every axis holds half of them
    for a in range(3):
        f = np.mean(p[:, a] < 0.5 * cfg.dx)
        assert abs(f - 0.5) < 5 * 0.5 / math.sqrt(n)


def test_fill_fractional_ppc_reproducible_and_region(lib):
    cfg = box()
    runs = []
    for seed in (7, 7, 8):
        ctx = filled(lib, cfg, abi.PATH_FAST, ppc=2.5, seed=seed)
        try:
            runs.append(ctx.download_particles(0))
        finally:
            ctx.close()
    (c1, p1), (c2, p2), (c3, p3) = runs
    assert np.array_equal(c1, c2) and np.array_equal(p1.view(np.uint64), p2.view(np.uint64))
    assert not np.array_equal(c1, c3)
    assert set(np.unique(c1)) <= {2, 3}
    assert abs(c1.mean() - 2.5) < 5 * 0.5 / math.sqrt(c1.size)
    # cell centres with x in [0, 1 Mm] only
    ctx = filled(lib, cfg, abi.PATH_FAST, region=(0.0, 1e6, -1e9, 1e9, -1e9, 1e9))
    try:
        cnt, _ = ctx.download_particles(0)
    finally:
        ctx.close()
    xc = cfg.x_min + (np.arange(cfg.nx) + 0.5) * cfg.dx
    inside = np.repeat(((xc >= 0) & (xc <= 1e6))[None, :], cfg.ny * cfg.nz, axis=0).reshape(-1)
    assert np.all(cnt[inside] == PPC) and np.all(cnt[~inside] == 0)


def test_fill_same_set_in_fp32_form_and_steps(lib):
    """The FP32 form holds the same particles (positions to FP32 offsets,
    velocities to FP32), and both storages step after the fill."""
    cfg = box()
    got = {}
    for name, path in (("fast", abi.PATH_FAST), ("fp32", abi.PATH_FP32)):
        ctx = filled(lib, cfg, path)
        try:
            got[name] = ctx.download_particles(0)
            ctx.step(3)
            # the particles of the cells at the non-periodic walls leave at the first step
            assert ctx.num_particles(0) > 0.4 * got[name][1].shape[0]
        finally:
            ctx.close()
    (ca, pa), (cb, pb) = got["fast"], got["fp32"]
    assert np.array_equal(ca, cb)

    def canon(c, p):
        cell = np.repeat(np.arange(c.size), c.astype(np.int64))
        o = np.lexsort((p[:, 2], p[:, 1], p[:, 0], cell))
        return p[o]
    qa, qb = canon(ca, pa), canon(cb, pb)
    assert np.max(np.abs(qa[:, :3] - qb[:, :3])) <= 1e-6 * cfg.dx
    assert np.max(np.abs(qa[:, 3:6] - qb[:, 3:6]) / np.abs(qa[:, 3:6]).max()) <= 1e-6
