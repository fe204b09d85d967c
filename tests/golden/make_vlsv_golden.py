"""Pins the VLSV container of the saved states (rhybrid_b200/vlsv.py) on the
reference's own reader: writes a small state with the library's writer, reads
it back with the reference's VlsvReader / VlsvParticles (tools/rhybridpy.py of
the reference tree) and freezes what they return, with the written file.

    python tests/golden/make_vlsv_golden.py

The reference tree is RH_REFERENCE_DIR, else the checkout next to this
repository. Writes vlsv_state_5x4x3.vlsv and vlsv_state_5x4x3.npz (the inputs
under in_*, the reader's answers under ref_*), and the reduced state of the
same cells (every REDUCED_NSTRIDE-th) as vlsv_reduced_5x4x3.vlsv, its reader
answers under red_*.
"""
import hashlib
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from rhybrid_b200 import vlsv as V  # noqa: E402

REF_DIR = os.environ.get("RH_REFERENCE_DIR") or os.path.normpath(
    os.path.join(HERE, "..", "..", "..", "reference"))
NAME = "vlsv_state_5x4x3"
REDUCED = "vlsv_reduced_5x4x3"
REDUCED_NSTRIDE = 2
GRID = {"nx": 5, "ny": 4, "nz": 3, "x_min": -750e3, "y_min": -600e3, "z_min": -450e3, "dx": 300e3,
        "periodic": (False, True, False)}
TIME, TIMESTEP = 12.5, 250
# cells looked up by id, and points (inside cells) looked up by coordinates
QUERY_IDS = np.array([5, 0, 59, 17, 33])
QUERY_POINTS = np.array([[-700e3, -550e3, -400e3], [10e3, 20e3, 30e3], [740e3, 590e3, 440e3],
                         [-100e3, 250e3, -300e3]])


def inputs():
    """The state written: cell variables as the output operator names them,
    two particle populations whose points lie in the cells their ids name."""
    rng = np.random.default_rng(20261204)
    n = GRID["nx"] * GRID["ny"] * GRID["nz"]
    cells = {
        "cellB": rng.normal(0, 5e-9, (n, 3)),
        "n_H+": rng.uniform(1e6, 3e6, n),
        "v_H+": rng.normal(0, 4e5, (n, 3)),
        "T_H+": rng.uniform(5e4, 2e5, n),
        "cellNPles": rng.integers(0, 40, n).astype(np.float64),
    }
    parts = {}
    for pop, m in (("H+", 17), ("O+", 5)):
        cid = rng.integers(0, n, m).astype(np.uint32)
        i, j, k = cid % GRID["nx"], (cid // GRID["nx"]) % GRID["ny"], cid // (GRID["nx"] * GRID["ny"])
        corner = np.stack([GRID["x_min"] + i * GRID["dx"], GRID["y_min"] + j * GRID["dx"],
                           GRID["z_min"] + k * GRID["dx"]], axis=1)
        parts[f"ParticlePointMesh_{pop}"] = corner + rng.uniform(0, GRID["dx"], (m, 3))
        parts[f"v_{pop}"] = rng.normal(0, 4e5, (m, 3))
        parts[f"CellID_{pop}"] = cid
    return cells, parts


def reduced_inputs(cells, parts):
    """The reduced state of the same cells: every REDUCED_NSTRIDE-th cell's
    id and cellB, and those cells' particles."""
    nx, ny, n = GRID["nx"], GRID["ny"], GRID["nx"] * GRID["ny"] * GRID["nz"]
    cid = np.arange(n)
    s = REDUCED_NSTRIDE
    keep = (cid % s == 0) & (cid % (s * nx) < nx) & (cid % (s * nx * ny) < nx * ny)
    red = {"CellID": cid[keep].astype(np.uint32), "cellB": cells["cellB"][keep]}
    for pop in ("H+", "O+"):
        k = keep[parts[f"CellID_{pop}"]]
        red[f"CellID_{pop}"] = parts[f"CellID_{pop}"][k]
        red[f"v_{pop}"] = parts[f"v_{pop}"][k]
    return red


def main():
    sys.path.insert(0, os.path.join(REF_DIR, "tools"))
    import rhybridpy as rhb   # the reference's reader

    cells, parts = inputs()
    path = os.path.join(HERE, NAME + ".vlsv")
    V.write_state(path, GRID, TIME, TIMESTEP, cells, parts)
    vr = rhb.vlsvfile.VlsvReader(path)
    vp = rhb.vlsvfile.VlsvParticles(path)
    out = {f"in_{k}": np.asarray(v) for k, v in cells.items()}
    out.update({f"inp_{k}": np.asarray(v) for k, v in parts.items()})
    out["ref_extent"] = vr.get_spatial_mesh_extent()
    out["ref_mesh_size"] = vr.get_spatial_mesh_size()
    out["ref_block_size"] = vr.get_spatial_block_size()
    out["ref_variables"] = np.array(vr.get_all_variables())
    out["ref_time"] = np.array(vr.read_parameter("time"))
    out["ref_t"] = np.array(vr.read_parameter("t"))
    out["ref_timestep"] = np.array(vr.read_parameter("timestep"))
    for name in list(cells) + ["CellID"]:
        out[f"ref_var_{name}"] = np.asarray(vr.read_variable(name))
        out[f"ref_vsize_{name}"] = np.array(vr.read_variable_vectorsize(name))
        out[f"ref_byid_{name}"] = np.asarray(vr.read_variable(name, cellids=QUERY_IDS))
    out["ref_cellid_of_points"] = np.asarray(vr.get_cellid(QUERY_POINTS))
    out["ref_cell_coordinates"] = np.asarray(vr.get_cell_coordinates(QUERY_IDS + 1))
    _, ids, values, _ = rhb.calculations.vlsv_intpol_points(vr, QUERY_POINTS, ["n_H+"], "pass", 0)
    out["ref_intpol0_ids"], out["ref_intpol0_n"] = np.asarray(ids), np.asarray(values)
    out["ref_point_meshes"] = np.array(vp.get_all_point_meshes())
    out["ref_point_variables"] = np.array(vp.get_all_point_variables())
    for pop in ("H+", "O+"):
        out[f"ref_mesh_{pop}"] = vp.read_particle_mesh(f"ParticlePointMesh_{pop}")
        out[f"ref_pv_{pop}"] = vp.read_particle_variable(f"v_{pop}")
        out[f"ref_pcid_{pop}"] = vp.read_particle_variable(f"CellID_{pop}")
    out["sha256"] = np.array(hashlib.sha256(open(path, "rb").read()).hexdigest())
    red = reduced_inputs(cells, parts)
    rpath = os.path.join(HERE, REDUCED + ".vlsv")
    V.write_reduced_state(rpath, TIME, TIMESTEP, REDUCED_NSTRIDE, red, ("H+", "O+"))
    rr = rhb.vlsvfile.VlsvReader(rpath)
    rp = rhb.vlsvfile.VlsvParticles(rpath)
    out.update({f"red_in_{k}": np.asarray(v) for k, v in red.items()})
    for par in ("time", "timestep", "Nstride"):
        out[f"red_par_{par}"] = np.array(rr.read_parameter(par))
    out["red_point_variables"] = np.array(rp.get_all_point_variables())
    for name in ("CellID", "cellB", "CellID_H+", "v_H+", "CellID_O+", "v_O+"):
        out[f"red_var_{name}"] = rp.read_particle_variable(name)
    out["red_sha256"] = np.array(hashlib.sha256(open(rpath, "rb").read()).hexdigest())
    np.savez_compressed(os.path.join(HERE, NAME + ".npz"), **out)
    print(f"wrote {path} ({os.path.getsize(path)} bytes) and {NAME}.npz")


if __name__ == "__main__":
    main()
