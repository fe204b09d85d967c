"""The FP32 precision form (RHGPU_PATH_FP32): particles as int32 cell + FP32
offsets + FP32 velocities, FP32 push and deposit with FP32 accumulation, FP64
field update. Its results are compared with the FP64 fast path (itself bitwise
against the oracle) and the measured relative L2 errors are checked against
stated bounds."""
import numpy as np
import pytest

from rhybrid_b200 import abi
from rhybrid_b200 import config as cf

from harness import closed_box_config, load, snapshot

pytestmark = pytest.mark.gpu

EPS32 = 2.0 ** -24


def run_path(cfg, nsteps, path, grid=None, pops=None):
    if grid is None:
        grid, pops = cf.initial_state(cfg)
    ctx = abi.Context(abi.gpu_library(), cf.params(cfg), cf.species(cfg),
                      capacity=[int(1.5 * p[1].shape[0]) + 1024 for p in pops])
    try:
        ctx.set_path(path)
        load(ctx, cfg, grid, pops)
        ctx.step(nsteps)
        return snapshot(ctx)
    finally:
        ctx.close()


def rel_l2(a, b):
    a, b = np.asarray(a, float).reshape(-1), np.asarray(b, float).reshape(-1)
    d = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / d) if d > 0 else float(np.linalg.norm(a - b))


def test_fp32_upload_download_roundtrip():
    cfg = closed_box_config()
    grid, pops = cf.initial_state(cfg)
    ctx = abi.Context(abi.gpu_library(), cf.params(cfg), cf.species(cfg), capacity=[p[1].shape[0] for p in pops])
    try:
        ctx.set_path(abi.PATH_FP32)
        load(ctx, cfg, grid, pops)
        for s, (cnt, p) in enumerate(pops):
            c2, p2 = ctx.download_particles(s)
            assert np.array_equal(cnt, c2)
            key = lambda q: np.lexsort((q[:, 2], q[:, 1], q[:, 0], np.repeat(np.arange(cnt.size), cnt)))  # noqa: E731
            a, b = p[key(p)], p2[key(p2)]
            assert np.all(np.abs(a[:, :3] - b[:, :3]) <= cfg.dx * EPS32)
            assert np.all(np.abs(a[:, 3:6] - b[:, 3:6]) <= np.abs(a[:, 3:6]) * EPS32)
            assert np.array_equal(a[:, 6], b[:, 6])
    finally:
        ctx.close()


def test_fp32_rejects_per_particle_weights():
    cfg = cf.config_empty_box(6, 6, 6, ppc=2.0)
    grid, pops = cf.initial_state(cfg)
    cnt, p = pops[0]
    p = p.copy()
    p[3, 6] *= 1.5
    ctx = abi.Context(abi.gpu_library(), cf.params(cfg), cf.species(cfg), capacity=[p.shape[0] + 8])
    try:
        ctx.set_path(abi.PATH_FP32)
        with pytest.raises(abi.RhError) as ei:
            ctx.upload_particles(0, cnt, p)
        assert ei.value.code == abi.ERR_ARG
    finally:
        ctx.close()


def test_fp32_charge_conservation():
    """Sum(rho) dV == sum(w) q to FP32 accumulation accuracy (periodic box)."""
    cfg = cf.config_empty_box(12, 10, 8, ppc=7.0).replace(min_ion_charge_density_relative=0.0)
    grid, pops = cf.initial_state(cfg)
    ctx = abi.Context(abi.gpu_library(), cf.params(cfg), cf.species(cfg), capacity=[pops[0][1].shape[0] + 64])
    try:
        ctx.set_path(abi.PATH_FP32)
        load(ctx, cfg, grid, pops)
        ctx.push()
        ctx.accumulate()
        rho = ctx.download_array("cellRhoQi")
        _, p = ctx.download_particles(0)
        total = p[:, 6].sum() * cfg.populations[0].q
        err = abs(rho.sum() * cfg.dx ** 3 - total) / total
        print(f"FP32 charge conservation error {err:.2e}")
        assert err <= 1e-6
    finally:
        ctx.close()


def test_fp32_deterministic():
    cfg = closed_box_config()
    a = run_path(cfg, 5, abi.PATH_FP32)
    b = run_path(cfg, 5, abi.PATH_FP32)
    for n in ("faceB", "cellRhoQi", "cellJi"):
        assert np.array_equal(a["arrays"][n].view(np.uint64), b["arrays"][n].view(np.uint64)), n
    for (ca, pa), (cb, pb) in zip(a["particles"], b["particles"]):
        assert np.array_equal(ca, cb) and np.array_equal(pa.view(np.uint64), pb.view(np.uint64))


@pytest.mark.parametrize("case", ["closed_box_10", "empty_box_32cubed_100"])
def test_fp32_error_against_fp64(case):
    """Relative L2 error of the moments and fields of the FP32 form against the
    FP64 fast path after N steps; the bounds are the stated error of the form."""
    if case == "closed_box_10":
        cfg, n, bound = closed_box_config(nx=16, ny=14, nz=12, ppc=8.0), 10, 1e-4
    else:
        cfg, n, bound = cf.config_empty_box(32, 32, 32, ppc=20.0), 100, 1e-4
    a = run_path(cfg, n, abi.PATH_FP32)
    b = run_path(cfg, n, abi.PATH_FAST)
    errs = {k: rel_l2(a["arrays"][k], b["arrays"][k]) for k in ("cellRhoQi", "cellJi", "faceB", "nodeE", "cellUe")}
    print(f"FP32 vs FP64 after {n} steps ({case}): " + ", ".join(f"{k} {v:.2e}" for k, v in errs.items()))
    for k, v in errs.items():
        assert v <= bound, f"{k}: {v:.3e} > {bound}"
    na = sum(int(c.sum()) for c, _ in a["particles"])
    nb = sum(int(c.sum()) for c, _ in b["particles"])
    assert abs(na - nb) <= 1e-4 * nb


def test_fp32_nonfinite_particle_raises_device_error():
    cfg = cf.config_empty_box(6, 6, 6, ppc=2.0)
    grid, pops = cf.initial_state(cfg)
    cnt, p = pops[0]
    p = p.copy()
    p[5, 3] = np.nan
    ctx = abi.Context(abi.gpu_library(), cf.params(cfg), cf.species(cfg), capacity=[p.shape[0] + 8])
    try:
        ctx.set_path(abi.PATH_FP32)
        load(ctx, cfg, grid, [(cnt, p)])
        with pytest.raises(abi.RhError) as ei:
            ctx.step(1)
        assert ei.value.code == abi.ERR_DEVICE
        assert ctx.device_errors() & abi.DEVERR_NAN_PARTICLE
    finally:
        ctx.close()


def test_fp32_diagnostics_in_fp64():
    cfg = closed_box_config()
    grid, pops = cf.initial_state(cfg)
    ctx = abi.Context(abi.gpu_library(), cf.params(cfg), cf.species(cfg), capacity=[p[1].shape[0] + 256 for p in pops])
    try:
        ctx.set_path(abi.PATH_FP32)
        load(ctx, cfg, grid, pops)
        ctx.step(2)
        d = ctx.reduce_diagnostics()
        for s in range(len(pops)):
            _, p = ctx.download_particles(s)
            got = d["populations"][s]
            assert got["N_macroParticles"] == p.shape[0]
            assert abs(got["N_realParticles"] - p[:, 6].sum()) <= 1e-12 * p[:, 6].sum()
            e = (p[:, 6] * (p[:, 3:6] ** 2).sum(1)).sum()
            assert abs(got["sumWV2"] - e) <= 1e-12 * e
    finally:
        ctx.close()


def test_fp32_own_records_roundtrip_and_same_run():
    """rhgpu_upload_particles_f32 / rhgpu_download_particles_f32: the form's own
    6-float records (offsets in cell units, velocities) with the weight apart.
    Records come back exactly as stored, and a context loaded from them steps
    bit for bit like the context they were downloaded from."""
    cfg = closed_box_config()
    grid, pops = cf.initial_state(cfg)
    lib = abi.gpu_library()
    cap = [int(1.5 * p[1].shape[0]) + 1024 for p in pops]
    a = abi.Context(lib, cf.params(cfg), cf.species(cfg), capacity=cap)
    b = abi.Context(lib, cf.params(cfg), cf.species(cfg), capacity=cap)
    try:
        a.set_path(abi.PATH_FP32)
        b.set_path(abi.PATH_FP32)
        load(a, cfg, grid, pops)
        for k in ("faceB", "cellB", "nodeEta"):
            b.upload_array(k, grid[k])
        b.upload_cell_flags(grid["flags"])
        for s, (cnt, p) in enumerate(pops):
            c32, r32, w = a.download_particles_f32(s)
            assert np.array_equal(c32, cnt) and r32.dtype == np.float32 and r32.shape == (p.shape[0], 6)
            assert w == p[0, 6]
            assert np.all((r32[:, :3] >= 0) & (r32[:, :3] < 1))
            # the double records of the same particles: positions = offsets x dx
            c64, p64 = a.download_particles(s)
            assert np.array_equal(c64, c32)
            assert np.array_equal(p64[:, :3], r32[:, :3].astype(np.float64) * cfg.dx)
            assert np.array_equal(p64[:, 3:6], r32[:, 3:6].astype(np.float64))
            b.upload_particles_f32(s, c32, r32, w)
            c2, r2, w2 = b.download_particles_f32(s)
            assert np.array_equal(c2, c32) and np.array_equal(r2.view(np.uint32), r32.view(np.uint32)) and w2 == w
        a.step(5)
        b.step(5)
        sa, sb = snapshot(a), snapshot(b)
        for n in sa["arrays"]:
            assert np.array_equal(sa["arrays"][n].view(np.uint64), sb["arrays"][n].view(np.uint64)), n
        for (ca, pa), (cb, pb) in zip(sa["particles"], sb["particles"]):
            assert np.array_equal(ca, cb) and np.array_equal(pa.view(np.uint64), pb.view(np.uint64))
    finally:
        a.close()
        b.close()


def test_fp32_own_records_need_the_fp32_form():
    cfg = closed_box_config()
    ctx = abi.Context(abi.gpu_library(), cf.params(cfg), cf.species(cfg))
    try:
        ctx.set_path(abi.PATH_FAST)
        with pytest.raises(abi.RhError):
            ctx.upload_particles_f32(0, np.zeros(cfg.ncells, dtype=np.uint32), np.zeros((0, 6), np.float32), 1.0)
    finally:
        ctx.close()
