"""The VLSV container of the saved states (rhybrid_b200/vlsv.py), pinned on
the reference's own reader: tests/golden/make_vlsv_golden.py wrote a small
state with this writer and froze what the reference's VlsvReader and
VlsvParticles (tools/rhybridpy.py) read from it. The writer must reproduce
that file byte for byte, and what the reference's reader returned must be the
state that was written."""
import hashlib
import os

import numpy as np
import pytest

from rhybrid_b200 import vlsv as V

from golden import make_vlsv_golden as G

HERE = os.path.dirname(os.path.abspath(__file__))
FILE = os.path.join(HERE, "golden", G.NAME + ".vlsv")


@pytest.fixture(scope="module")
def gold():
    return np.load(os.path.join(HERE, "golden", G.NAME + ".npz"))


def state(gold):
    cells = {k[3:]: gold[k] for k in gold.files if k.startswith("in_")}
    parts = {k[4:]: gold[k] for k in gold.files if k.startswith("inp_")}
    order = ["cellB", "n_H+", "v_H+", "T_H+", "cellNPles"]
    return {k: cells[k] for k in order}, parts


def test_writer_reproduces_the_pinned_file(tmp_path, gold):
    cells, parts = state(gold)
    path = str(tmp_path / "s.vlsv")
    V.write_state(path, G.GRID, G.TIME, G.TIMESTEP, cells, parts)
    data = open(path, "rb").read()
    assert hashlib.sha256(data).hexdigest() == str(gold["sha256"])
    assert data == open(FILE, "rb").read()


def test_reference_reader_read_the_state(gold):
    cells, parts = state(gold)
    g = G.GRID
    ext = [g["x_min"], g["y_min"], g["z_min"], g["x_min"] + g["nx"] * g["dx"], g["y_min"] + g["ny"] * g["dx"],
           g["z_min"] + g["nz"] * g["dx"]]
    assert np.allclose(gold["ref_extent"], ext, rtol=0, atol=1e-6)
    assert list(gold["ref_mesh_size"]) == [g["nx"], g["ny"], g["nz"]]
    assert list(gold["ref_block_size"]) == [1, 1, 1]
    assert float(gold["ref_time"]) == G.TIME and float(gold["ref_t"]) == G.TIME
    assert int(gold["ref_timestep"]) == G.TIMESTEP
    n = g["nx"] * g["ny"] * g["nz"]
    assert np.array_equal(gold["ref_var_CellID"], np.arange(n))
    for name, a in cells.items():
        assert np.array_equal(gold[f"ref_var_{name}"], a), name
        assert int(gold[f"ref_vsize_{name}"]) == (3 if a.ndim == 2 else 1)
        assert np.array_equal(gold[f"ref_byid_{name}"], a[G.QUERY_IDS]), name
    assert list(gold["ref_point_meshes"]) == ["ParticlePointMesh_H+", "ParticlePointMesh_O+"]
    assert list(gold["ref_point_variables"]) == ["v_H+", "CellID_H+", "v_O+", "CellID_O+"]
    for pop in ("H+", "O+"):
        assert np.array_equal(gold[f"ref_mesh_{pop}"], parts[f"ParticlePointMesh_{pop}"])
        assert np.array_equal(gold[f"ref_pv_{pop}"], parts[f"v_{pop}"])
        assert np.array_equal(gold[f"ref_pcid_{pop}"].reshape(-1), parts[f"CellID_{pop}"])


def test_reference_reader_point_lookup_convention(gold):
    """The reference's reader maps a point to the 1-based geometric id of its
    cell and looks that id up among the stored ids, which are the 0-based
    linear indices RHybrid's output holds (the reader documents both); a point
    in the last cell has no stored partner (0)."""
    cells, _ = state(gold)
    g = G.GRID
    p = G.QUERY_POINTS
    idx = np.floor((p - np.array([g["x_min"], g["y_min"], g["z_min"]])) / g["dx"]).astype(np.int64)
    lin = idx[:, 0] + g["nx"] * (idx[:, 1] + g["ny"] * idx[:, 2])
    n = g["nx"] * g["ny"] * g["nz"]
    want = np.where(lin + 1 < n, lin + 1, 0)
    assert np.array_equal(gold["ref_cellid_of_points"], want)
    got = gold["ref_intpol0_n"].reshape(-1)
    ok = want > 0
    assert np.array_equal(got[ok], cells["n_H+"][want[ok]]) and np.all(np.isnan(got[~ok]))


def test_own_reader(gold):
    cells, parts = state(gold)
    st = V.load_state(FILE)
    assert float(st["time"]) == G.TIME and int(st["timestep"]) == G.TIMESTEP
    for name, a in cells.items():
        assert np.array_equal(st[name], a)
    for pop in ("H+", "O+"):
        mesh = f"ParticlePointMesh_{pop}"
        assert np.array_equal(st[mesh], parts[mesh])
        assert np.array_equal(st[f"{mesh}/v_{pop}"], parts[f"v_{pop}"])
        assert np.array_equal(st[f"{mesh}/CellID_{pop}"], parts[f"CellID_{pop}"])
    raw = V.read(FILE)
    assert list(raw[("MESH_BBOX", None, "SpatialGrid")]) == [5, 4, 3, 1, 1, 1]


def test_writer_rejects_bad_arrays(tmp_path):
    with V.Writer(str(tmp_path / "x.vlsv")) as w:
        with pytest.raises(TypeError):
            w.write("VARIABLE", np.array(["a"]), name="s")
        with pytest.raises(ValueError):
            w.write("VARIABLE", np.zeros((2, 2, 2)), name="cube")
    with pytest.raises(ValueError):
        V.write_state(str(tmp_path / "y.vlsv"), G.GRID, 0.0, 0, {"short": np.zeros(3)})


def test_reduced_state_pinned(tmp_path, gold):
    """The reduced state file: reproduced byte for byte, and the reference's
    reader read its parameters and point data back as written."""
    red = {k[len("red_in_"):]: gold[k] for k in gold.files if k.startswith("red_in_")}
    path = str(tmp_path / "r.vlsv")
    V.write_reduced_state(path, G.TIME, G.TIMESTEP, G.REDUCED_NSTRIDE, red, ("H+", "O+"))
    assert hashlib.sha256(open(path, "rb").read()).hexdigest() == str(gold["red_sha256"])
    assert open(path, "rb").read() == open(os.path.join(HERE, "golden", G.REDUCED + ".vlsv"), "rb").read()
    assert float(gold["red_par_time"]) == G.TIME and int(gold["red_par_timestep"]) == G.TIMESTEP
    assert int(gold["red_par_Nstride"]) == G.REDUCED_NSTRIDE
    assert list(gold["red_point_variables"]) == ["CellID", "cellB", "CellID_H+", "v_H+", "CellID_O+", "v_O+"]
    cells, parts = state(gold)
    want = G.reduced_inputs(cells, parts)
    for name, a in want.items():
        assert np.array_equal(gold[f"red_var_{name}"].reshape(a.shape), a), name
