"""The VLSV container of a saved state: the file the reference's output step
writes (Corsair's VLSV writer fed by UserDataOP::writeData,
src/operator_userdata.cpp:55-312, ParticleListHybrid::writeParticles,
src/particle_list_hybrid.h:41-159, and the time parameters,
src/diagnostics.h:834-839).

Layout, as the reference's own reader takes it (tools/rhybridpy.py:113-123,
219-280):

    bytes 0-7    endianness word (0: little-endian)
    bytes 8-15   byte offset of the XML footer (uint64, little-endian)
    ...          the arrays, raw little-endian, one after the other
    footer       <VLSV> with one element per array: the tag is the array's
                 kind (PARAMETER, MESH, MESH_BBOX, MESH_NODE_CRDS_X/Y/Z,
                 MESH_DOMAIN_SIZES, MESH_GHOST_DOMAINS, MESH_GHOST_LOCALIDS,
                 VARIABLE), the attributes are name, mesh, type, arraysize,
                 vectorsize, datatype (float, int, uint) and datasize (bytes
                 per element), and the text is the array's byte offset.

The spatial grid is the mesh SpatialGrid, one block per cell: MESH_BBOX holds
the cells per axis and the block size (1 1 1), MESH_NODE_CRDS_X/Y/Z the node
coordinates of each axis, and the CellID variable the cells' ids, the linear
index i + nx (j + ny k), which is the id the reference's particle output
selects cells by (particle_list_hybrid.h:86-90). The cell variables are
VARIABLE celldata on SpatialGrid, in the order given; each particle
population is the point mesh ParticlePointMesh_<name> (MESH type point) with
v_<name> and CellID_<name> as pointdata on it. The time and the time step are
PARAMETERs.
"""
import os
import struct
import xml.etree.ElementTree as ET
from typing import Dict, Mapping, Optional
from xml.sax.saxutils import quoteattr

import numpy as np

SPATIAL_MESH = "SpatialGrid"
_KIND = {"f": "float", "i": "int", "u": "uint"}


class Writer:
    """Arrays appended to one VLSV file; close() writes the footer."""

    def __init__(self, path: str):
        self.path = os.fspath(path)
        self._f = open(self.path, "wb")
        self._f.write(struct.pack("<QQ", 0, 0))
        self._entries = []

    def write(self, tag: str, data, name: Optional[str] = None, mesh: Optional[str] = None,
              type: Optional[str] = None, **extra) -> None:
        """One array: rows are the array entries, columns the vector components
        (a 1-D array has vector size 1; a scalar is one entry)."""
        a = np.asarray(data)
        if a.dtype.kind not in _KIND:
            raise TypeError(f"VLSV arrays are float, int or uint, not {a.dtype}")
        if a.dtype.itemsize not in (4, 8):
            a = a.astype(a.dtype.kind + "8")
        if a.ndim > 2:
            raise ValueError("VLSV arrays are one- or two-dimensional")
        a = np.ascontiguousarray(a, dtype=a.dtype.newbyteorder("<"))
        arraysize = 1 if a.ndim == 0 else a.shape[0]
        vectorsize = a.shape[1] if a.ndim == 2 else 1
        attrs = []
        for key, value in (("name", name), ("mesh", mesh), ("type", type)):
            if value is not None:
                attrs.append((key, str(value)))
        attrs += [("arraysize", str(arraysize)), ("vectorsize", str(vectorsize)),
                  ("datatype", _KIND[a.dtype.kind]), ("datasize", str(a.dtype.itemsize))]
        attrs += [(str(k), str(v)) for k, v in extra.items()]
        offset = self._f.tell()
        self._f.write(a.tobytes())
        self._entries.append((tag, attrs, offset))

    def close(self) -> None:
        if self._f is None:
            return
        footer = self._f.tell()
        lines = ["<VLSV>"]
        for tag, attrs, offset in self._entries:
            a = " ".join(f"{k}={quoteattr(v)}" for k, v in attrs)
            lines.append(f"   <{tag} {a}>{offset}</{tag}>")
        lines.append("</VLSV>\n")
        self._f.write("\n".join(lines).encode("utf-8"))
        self._f.seek(8)
        self._f.write(struct.pack("<Q", footer))
        self._f.close()
        self._f = None

    def __enter__(self) -> "Writer":
        return self

    def __exit__(self, *_) -> None:
        self.close()


def write_spatial_grid(w: Writer, nx: int, ny: int, nz: int, x_min: float, y_min: float, z_min: float,
                       dx: float, periodic=(False, False, False)) -> np.ndarray:
    """The mesh SpatialGrid of an nx x ny x nz grid of cells of size dx from
    (x_min, y_min, z_min), one domain, every cell stored in linear order;
    returns the cell ids."""
    n = nx * ny * nz
    cid = np.arange(n, dtype=np.uint32)
    per = {f"{a}periodic": "yes" if p else "no" for a, p in zip("xyz", periodic)}
    w.write("MESH", cid, name=SPATIAL_MESH, type="multi_ucd", **per)
    w.write("MESH_BBOX", np.array([nx, ny, nz, 1, 1, 1], dtype=np.uint64), mesh=SPATIAL_MESH)
    for axis, m, lo in (("X", nx, x_min), ("Y", ny, y_min), ("Z", nz, z_min)):
        w.write(f"MESH_NODE_CRDS_{axis}", lo + np.arange(m + 1, dtype=np.float64) * dx, mesh=SPATIAL_MESH)
    w.write("MESH_DOMAIN_SIZES", np.array([[n, 0]], dtype=np.uint64), mesh=SPATIAL_MESH)
    w.write("MESH_GHOST_DOMAINS", np.zeros(0, dtype=np.uint64), mesh=SPATIAL_MESH)
    w.write("MESH_GHOST_LOCALIDS", np.zeros(0, dtype=np.uint64), mesh=SPATIAL_MESH)
    w.write("VARIABLE", cid, name="CellID", mesh=SPATIAL_MESH, type="celldata")
    return cid


def write_state(path: str, grid: Mapping, time: float, timestep: int, cell_variables: Mapping[str, np.ndarray],
                particles: Optional[Mapping[str, np.ndarray]] = None) -> str:
    """One saved state: the time parameters, the spatial grid (`grid`: nx, ny,
    nz, x_min, y_min, z_min, dx and optionally periodic), the cell variables
    (name -> N or N x 3 array, cells in linear order) and the particle points
    (output.particle_points: ParticlePointMesh_<name>, v_<name>, CellID_<name>)."""
    with Writer(path) as w:
        w.write("PARAMETER", np.float64(time), name="time")
        w.write("PARAMETER", np.uint32(timestep), name="timestep")
        nx, ny, nz = int(grid["nx"]), int(grid["ny"]), int(grid["nz"])
        write_spatial_grid(w, nx, ny, nz, float(grid["x_min"]), float(grid["y_min"]), float(grid["z_min"]),
                           float(grid["dx"]), grid.get("periodic", (False, False, False)))
        n = nx * ny * nz
        for name, a in cell_variables.items():
            a = np.asarray(a)
            if a.shape[0] != n:
                raise ValueError(f"cell variable {name}: {a.shape[0]} rows for {n} cells")
            w.write("VARIABLE", a, name=name, mesh=SPATIAL_MESH, type="celldata")
        for mesh, crd in (particles or {}).items():
            if not mesh.startswith("ParticlePointMesh_"):
                continue
            pop = mesh[len("ParticlePointMesh_"):]
            w.write("MESH", np.asarray(crd, dtype=np.float64).reshape(-1, 3), name=mesh, type="point")
            w.write("VARIABLE", np.asarray(particles[f"v_{pop}"], dtype=np.float64).reshape(-1, 3), name=f"v_{pop}",
                    mesh=mesh, type="pointdata")
            w.write("VARIABLE", np.asarray(particles[f"CellID_{pop}"], dtype=np.uint32), name=f"CellID_{pop}",
                    mesh=mesh, type="pointdata")
    return path


def write_reduced_state(path: str, time: float, timestep: int, nstride: int, reduced: Mapping[str, np.ndarray],
                        species_names=()) -> str:
    """The reduced state file (diagnostics::saveStateReduced,
    diagnostics.h:819-960): the time, time step and Nstride parameters, then
    CellID and cellB of the kept cells as pointdata on ReducedPointMesh, and
    for each species in `reduced` (output.reduced_state with particles) its
    CellID_<name> and v_<name> as pointdata on ReducedParticlePointMesh_<name>.
    No mesh element is written for these point meshes, as in the reference."""
    with Writer(path) as w:
        w.write("PARAMETER", np.float64(time), name="time")
        w.write("PARAMETER", np.uint32(timestep), name="timestep")
        w.write("PARAMETER", np.uint32(nstride), name="Nstride")
        w.write("VARIABLE", np.asarray(reduced["CellID"], dtype=np.uint32), name="CellID", mesh="ReducedPointMesh",
                type="pointdata")
        w.write("VARIABLE", np.asarray(reduced["cellB"], dtype=np.float64).reshape(-1, 3), name="cellB",
                mesh="ReducedPointMesh", type="pointdata")
        for name in species_names:
            if f"v_{name}" not in reduced:
                continue
            mesh = f"ReducedParticlePointMesh_{name}"
            w.write("VARIABLE", np.asarray(reduced[f"CellID_{name}"], dtype=np.uint32), name=f"CellID_{name}",
                    mesh=mesh, type="pointdata")
            w.write("VARIABLE", np.asarray(reduced[f"v_{name}"], dtype=np.float64).reshape(-1, 3), name=f"v_{name}",
                    mesh=mesh, type="pointdata")
    return path


def grid_of(ctx) -> dict:
    """The spatial grid of a context (abi.Context) as write_state takes it."""
    p = ctx.params
    return {"nx": p.nx, "ny": p.ny, "nz": p.nz, "x_min": p.x_min, "y_min": p.y_min, "z_min": p.z_min, "dx": p.dx,
            "periodic": tuple(bool(x) for x in p.periodic)}


def load_state(path: str) -> Dict[str, np.ndarray]:
    """A saved state by name: the PARAMETERs, the SpatialGrid variables
    (CellID included), and each particle population's point mesh
    (ParticlePointMesh_<name>) with its pointdata variables as
    ParticlePointMesh_<name>/<variable> (a population's v_<name> and a cell
    variable v_<name> differ only by their mesh)."""
    out = {}
    for (tag, name, mesh), a in read(path).items():
        if tag == "PARAMETER":
            out[name] = a[0] if a.shape == (1,) else a
        elif tag == "VARIABLE" and mesh == SPATIAL_MESH:
            out[name] = a
        elif tag == "VARIABLE" and mesh:
            out[f"{mesh}/{name}"] = a
        elif tag == "MESH" and name and name.startswith("ParticlePointMesh_"):
            out[name] = a
    return out


def read(path: str) -> Dict[tuple, np.ndarray]:
    """Every array of a VLSV file, keyed by (tag, name, mesh): the container's
    own reading, for tests and tools."""
    out = {}
    with open(path, "rb") as f:
        raw = f.read()
    (footer,) = struct.unpack_from("<Q", raw, 8)
    root = ET.fromstring(raw[footer:])
    for el in root:
        a = el.attrib
        dt = np.dtype({"float": "f", "int": "i", "uint": "u"}[a["datatype"]] + a["datasize"]).newbyteorder("<")
        n, v = int(a["arraysize"]), int(a["vectorsize"])
        data = np.frombuffer(raw, dtype=dt, count=n * v, offset=int(el.text))
        out[(el.tag, a.get("name"), a.get("mesh"))] = (data.reshape(n, v) if v > 1 else data).copy()
    return out
