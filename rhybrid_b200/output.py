"""Output step: the arrays RHybrid hands to its VLSV writer at a data save
step, assembled from a context's state under the reference's names, in its
write order and with its arithmetic.

  cell_variables   UserDataOP::writeData (src/operator_userdata.cpp:55-312):
                   the grid arrays selected by Hybrid.output_parameters, ne,
                   the temporal averages, cellDivB (calcCellDiv :342-356),
                   cellNPles (calcCellNPles :359-380) and the bulk n, T, v of
                   each output population (calcCellParticleBulkParameters
                   :383-457)
  particle_points  ParticleListHybrid::writeParticles
                   (src/particle_list_hybrid.h:41-159): coordinates,
                   velocities and cell ids of the particles of every
                   Nstride'th cell

Arrays come back as a dict in write order: (N,) for scalars, (N, 3) for
vectors, N cells in linear order n = i + nx*(j + ny*k). The grid arrays,
particles and averages are read from the device through the context; the
per-cell moments are then summed on the host in the reference's order (per
cell: output populations in species order, particles in list order), so the
values are the reference's bit for bit on the same state. rhybrid_b200.vlsv
writes them as the reference's VLSV state file (run.py).

prod_rate_iono<k> / prod_rate_exo<k> are the rate-based sources' expected
macroparticles per step in each cell (rhgpu_source_rates). Not written: cellB0
(USE_B_CONSTANT is off in the reference's default build). faceJ is written as zeros: in the default build
(USE_EDGE_J) the reference computes J on edges and faceJ keeps its initial
zeros (user.cpp:1855).
"""
import warnings
from typing import Dict, Iterable, Optional, Sequence

import numpy as np

from . import abi

# grid arrays in writeData's order (operator_userdata.cpp:79-102) with their vector sizes
GRID_ARRAYS = [("faceB", 3), ("faceJ", 3), ("cellRhoQi", 1), ("cellB", 3), ("cellJ", 3), ("cellUe", 3),
               ("cellJi", 3), ("cellEp", 3), ("nodeRhoQi", 1), ("nodeE", 3), ("nodeB", 3), ("nodeJ", 3),
               ("nodeUe", 3), ("nodeJi", 3), ("nodeEta", 1)]
GRID_COUNTER_ARRAYS = [("gridCounterCellMaxUe", "cellMaxUe"), ("gridCounterCellMaxVi", "cellMaxVi"),
                       ("gridCounterCellMinRhoQi", "cellMinRhoQi"), ("gridCounterNodeMaxE", "nodeMaxE"),
                       ("gridCounterNodeMaxVw", "nodeMaxVw")]
INNER_FLAGS = [("innerFlagField", abi.FLAG_INNER_FIELD), ("innerFlagNode", abi.FLAG_INNER_NODE),
               ("innerFlagParticle", abi.FLAG_INNER_PARTICLE), ("innerFlagCellEp", abi.FLAG_INNER_CELLEP)]
# every name Hybrid.output_parameters accepts (user.cpp:2302-2343)
PARAMETERS = ([n for n, _ in GRID_ARRAYS] + [n for n, _ in GRID_COUNTER_ARRAYS] + [n for n, _ in INNER_FLAGS]
              + ["prod_rate_iono", "prod_rate_exo", "cellBAverage", "n_ave", "v_ave", "cellDivB", "cellNPles",
                 "cellB0", "ne", "n", "T", "v", "MPI_rank", "Load"])


def _grid(ctx):
    p = ctx.params
    return p.nx, p.ny, p.nz


def _cell_index(cnt: np.ndarray) -> np.ndarray:
    return np.repeat(np.arange(cnt.size, dtype=np.int64), cnt.astype(np.int64))


def cell_div(ctx, faceB: np.ndarray) -> np.ndarray:
    """calcCellDiv (operator_userdata.cpp:342-356): the face divergence of
    faceB in every cell whose 26 neighbours exist (non-periodic walls have
    none outside), 0 elsewhere."""
    nx, ny, nz = _grid(ctx)
    per = tuple(ctx.params.periodic)
    fb = faceB.reshape(nz, ny, nx, 3)
    d = ((fb[..., 0] - np.roll(fb[..., 0], 1, 2)) + (fb[..., 1] - np.roll(fb[..., 1], 1, 1))) \
        + (fb[..., 2] - np.roll(fb[..., 2], 1, 0))
    d = d / ctx.params.dx
    ok = np.ones((nz, ny, nx), bool)
    for axis, n, p in ((2, nx, per[0]), (1, ny, per[1]), (0, nz, per[2])):
        if not p:
            sl = [slice(None)] * 3
            sl[axis] = 0
            ok[tuple(sl)] = False
            sl[axis] = n - 1
            ok[tuple(sl)] = False
    return np.where(ok, d, 0.0).reshape(-1)


def bulk_parameters(ctx, species: Sequence[int], particles: Optional[dict] = None):
    """calcCellParticleBulkParameters (operator_userdata.cpp:383-457) of the
    species set `species`: number density n = sum(w)/dV, bulk velocity
    U = sum(w v)/sum(w) and kinetic temperature
    T = m sum(w |v - U|^2) / (3 sum(w) kB), m of the set's first species;
    all 0 in empty cells. Returns (n (N,), T (N,), U (N, 3))."""
    N = ctx.ncells
    parts = particles or {}
    cells, P = [], []
    for s in species:
        cnt, p = parts[s] if s in parts else ctx.download_particles(s)
        cells.append(_cell_index(cnt))
        P.append(p)
    cell = np.concatenate(cells) if cells else np.zeros(0, np.int64)
    p = np.concatenate(P) if P else np.zeros((0, 7))
    w = p[:, 6]
    # np.bincount adds its weights in array order: per cell, the species in
    # set order and each one's particles in list order, as the reference
    dens = np.bincount(cell, weights=w, minlength=N)
    U = np.stack([np.bincount(cell, weights=p[:, 3 + l] * w, minlength=N) for l in range(3)], axis=1)
    pos = dens > 0
    U = np.where(pos[:, None], U / np.where(pos, dens, 1.0)[:, None], 0.0)
    dv = p[:, 3:6] - U[cell]
    T = np.bincount(cell, weights=w * ((dv[:, 0] * dv[:, 0] + dv[:, 1] * dv[:, 1]) + dv[:, 2] * dv[:, 2]),
                    minlength=N)
    m = ctx.species[species[0]].m if len(species) else 0.0
    T = np.where(pos, T * (m / ((3 * np.where(pos, dens, 1.0)) * abi.BOLTZMANN)), 0.0)
    dx = ctx.params.dx
    return dens / (dx * dx * dx), T, U


def production_rates(ctx, iono: bool = True, exo: bool = True) -> Dict[str, np.ndarray]:
    """prod_rate_iono<k> and prod_rate_exo<k> (operator_userdata.cpp:123-154)
    from the context's sources, in species order. The reference numbers its
    ionosphere slots with one counter per injector class
    (particle_injector.cpp:1112-1114 for IonosphereInjector, :1415-1417 for
    ChapmanIonosphereInjector), and both classes write cellIonosphere. So the
    k-th source of each class fills slot k, and the later one in species
    order is the one that stays. There is one slot per ionosphere population;
    a slot no source writes is zeros."""
    srcs = list(getattr(ctx, "injectors", []))
    out: Dict[str, np.ndarray] = {}
    if iono:
        kinds = (abi.INJECT_IONOSPHERE, abi.INJECT_CHAPMAN_IONOSPHERE)
        members = [q for q, j in enumerate(srcs) if j.type in kinds]
        slots = [np.zeros(ctx.ncells) for _ in members]
        seen = {t: 0 for t in kinds}
        for q in sorted(members, key=lambda q: srcs[q].species):
            t = srcs[q].type
            slots[seen[t]] = ctx.source_rates(q)
            seen[t] += 1
        for k, a in enumerate(slots):
            out[f"prod_rate_iono{k}"] = a
    if exo:
        members = sorted((q for q, j in enumerate(srcs) if j.type == abi.INJECT_EXOSPHERE), key=lambda q: srcs[q].species)
        for k, q in enumerate(members):
            out[f"prod_rate_exo{k}"] = ctx.source_rates(q)
    return out


def cell_variables(ctx, params: Iterable[str], groups: Sequence[int] = (), group_names: Sequence[str] = (),
                   grid_counters: bool = False) -> Dict[str, np.ndarray]:
    """The cell variables UserDataOP::writeData writes for the output
    parameters `params`, by name in its write order. `groups`: the output
    population of each species (-1: none), `group_names` their names
    (output_str), as set_population_averages takes them; n_ave and v_ave
    are written when the context keeps those averages (not on the FP32
    form). `grid_counters`: the per-cell constraint counters are on
    (set_grid_counters). Reading the temporal averages restarts them, as the
    reference's output step does."""
    want = set(params)
    # an unknown name is skipped with a warning, as the reference's
    # configuration step does (user.cpp:2405-2410)
    for name in sorted(want - set(PARAMETERS)):
        warnings.warn(f"parameter requested for output does not exist: {name}")
    N = ctx.ncells
    out: Dict[str, np.ndarray] = {}
    for name, dim in GRID_ARRAYS:
        if name not in want or (name == "cellEp" and not ctx.params.use_electron_pressure):
            continue
        out[name] = np.zeros((N, 3)) if name == "faceJ" else ctx.download_array(name)
    if grid_counters and any(n in want for n, _ in GRID_COUNTER_ARRAYS):
        gc = ctx.grid_counters()
        for name, plane in GRID_COUNTER_ARRAYS:
            if name in want:
                out[name] = gc[plane].copy()
    for name, bit in INNER_FLAGS:
        if name in want:
            if ctx.cell_flags is None:
                raise RuntimeError(f"{name}: no cell flags were uploaded")
            out[name] = ((ctx.cell_flags & bit) != 0).astype(np.float64)
    if "n_ave" in want or "v_ave" in want:
        out["ne"] = ctx.download_array("cellRhoQi") / abi.CHARGE_ELEMENTARY
    if "prod_rate_iono" in want or "prod_rate_exo" in want:
        out.update(production_rates(ctx, "prod_rate_iono" in want, "prod_rate_exo" in want))
    ngroups = max(groups, default=-1) + 1
    if len(group_names) != ngroups or (len(groups) and len(groups) != ctx.nspecies):
        raise ValueError(f"{len(groups)} groups and {len(group_names)} names for {ctx.nspecies} species")
    avg = getattr(ctx, "_avg_groups", 0)
    if avg and avg != ngroups:
        raise ValueError(f"the context averages {avg} output populations, not {ngroups}")
    if ctx.lib.has("output_averages"):
        av = ctx.output_averages(cellB=True, populations=avg > 0)
        if "cellBAverage" in want:
            out["cellBAverage"] = av["cellBAverage"]
        if avg and ("n_ave" in want or "v_ave" in want):
            for m, g in enumerate(group_names):
                if "n_ave" in want:
                    out[f"n_{g}_ave"] = av["n_ave"][m]
                if "v_ave" in want:
                    out[f"v_{g}_ave"] = av["v_ave"][m]
    parts = None
    if "cellNPles" in want or ({"n", "T", "v"} & want and ngroups):
        parts = {s: ctx.download_particles(s) for s in range(ctx.nspecies)}
    if "cellDivB" in want:
        out["cellDivB"] = cell_div(ctx, ctx.download_array("faceB"))
    if "cellNPles" in want:
        out["cellNPles"] = sum((parts[s][0].astype(np.float64) for s in range(ctx.nspecies)), np.zeros(N))
    if {"n", "T", "v"} & want and ngroups:
        members = [[s for s in range(ctx.nspecies) if groups[s] == m] for m in range(ngroups)]
        for m, g in enumerate(group_names):
            n, T, U = bulk_parameters(ctx, members[m], parts)
            if "n" in want:
                out[f"n_{g}"] = n
            if "T" in want:
                out[f"T_{g}"] = T
            if "v" in want:
                out[f"v_{g}"] = U
    return out


def _strided_cells(nx: int, ny: int, n: int, nstride: int) -> np.ndarray:
    """The cells an Nstride output keeps: id c with c % Nstride == 0,
    c % (Nstride nx) < nx and c % (Nstride nx ny) < nx ny (ids are the linear
    cell index)."""
    cid = np.arange(n, dtype=np.int64)
    return (cid % nstride == 0) & (cid % (nstride * nx) < nx) & (cid % (nstride * nx * ny) < nx * ny)


def reduced_state(ctx, species_names: Sequence[str], nstride: int = 10, particles: bool = False) -> Dict[str, np.ndarray]:
    """diagnostics::saveStateReduced (diagnostics.h:819-960): cellB and the
    cell id of every cell an Nstride output keeps, and with `particles` each
    species' particles in those cells as CellID_<name> and v_<name>."""
    nx, ny, nz = _grid(ctx)
    sel = _strided_cells(nx, ny, ctx.ncells, nstride)
    out = {"CellID": np.flatnonzero(sel).astype(np.uint32), "cellB": ctx.download_array("cellB")[sel]}
    if particles:
        for s, name in enumerate(species_names):
            cnt, q = ctx.download_particles(s)
            cell = _cell_index(cnt)
            keep = sel[cell]
            out[f"CellID_{name}"] = cell[keep].astype(np.uint32)
            out[f"v_{name}"] = q[keep, 3:6].copy()
    return out


def particle_points(ctx, species_names: Sequence[str], nstride: int = 10) -> Dict[str, np.ndarray]:
    """ParticleListHybrid::writeParticles (particle_list_hybrid.h:41-159) for
    every species: the particles of the cells whose id c satisfies
    c % Nstride == 0, c % (Nstride nx) < nx and c % (Nstride nx ny) < nx ny,
    as ParticlePointMesh_<name> (global coordinates: local + cell corner),
    v_<name> and CellID_<name>. Cell ids are the linear cell index
    i + nx*(j + ny*k)."""
    if nstride <= 0:
        nstride = 10   # the reference's fallback for save_particles_Nstride <= 0 (user.cpp:2373-2376)
    nx, ny, nz = _grid(ctx)
    p = ctx.params
    cid = np.arange(ctx.ncells, dtype=np.int64)
    sel = _strided_cells(nx, ny, ctx.ncells, nstride)
    i, j, k = cid % nx, (cid // nx) % ny, cid // (nx * ny)
    corner = np.stack([p.x_min + i.astype(np.float64) * p.dx, p.y_min + j.astype(np.float64) * p.dx,
                       p.z_min + k.astype(np.float64) * p.dx], axis=1)
    out = {}
    for s, name in enumerate(species_names):
        cnt, q = ctx.download_particles(s)
        cell = _cell_index(cnt)
        keep = sel[cell]
        out[f"ParticlePointMesh_{name}"] = q[keep, 0:3] + corner[cell[keep]]
        out[f"v_{name}"] = q[keep, 3:6].copy()
        out[f"CellID_{name}"] = cell[keep].astype(np.uint32)   # pargrid::CellID, unsigned int
    return out
