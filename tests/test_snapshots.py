"""ParaView snapshots (hirensi_b200.snapshots): the reference's XDMF grids with raw
binary data files; checked by reading the files back (no GPU)."""
import os
import xml.etree.ElementTree as ET

import numpy as np

from hirensi_b200 import snapshots as P
from hirensi_b200.mesh import box_mesh


def test_connectivity_reorders_edge_nodes_like_the_reference():
    inod = np.arange(27)[None, :] + 100
    c = P.connectivity_mixed(inod)
    assert c.shape == (21,)
    assert c[0] == 48
    # local nodes 1-12, then 17-20, then 13-16 (1-based)
    assert list(c[1:13]) == list(range(100, 112))
    assert list(c[13:17]) == [116, 117, 118, 119]
    assert list(c[17:21]) == [112, 113, 114, 115]


def test_nodal_vectors_fill_constrained_dofs_with_zero():
    ID = np.array([[-1, 0, 1, 5, 6, 7, 8, 9, 10], [2, 3, 4, -1, -1, -1, -1, -1, -1]])
    v = np.arange(11, dtype=float) + 0.5
    out = P.nodal_vectors(ID, v)
    assert out.dtype == np.float32
    assert out.tolist() == [[0.0, 0.5, 1.5], [2.5, 3.5, 4.5]]


def test_step_files_read_back(tmp_path):
    m = box_mesh(2, 2, 1, 2.5, 1)
    rng = np.random.default_rng(0)
    u, v = rng.standard_normal(m.neq), rng.standard_normal(m.neq)
    xmf = P.write_step(str(tmp_path), "box", 40, 0.004, m, u, v)
    grid = ET.parse(tmp_path / xmf).getroot().find("Grid")
    assert float(grid.find("Time").get("Value")) == 0.004
    topo = grid.find("Topology")
    assert topo.get("NumberOfElements") == str(m.nel)
    items = {a.get("Name"): a.find("DataItem") for a in grid.findall("Attribute")}
    assert set(items) == {"Displacement", "Velocity"}
    d = np.fromfile(tmp_path / items["Displacement"].text, dtype="<f4").reshape(m.nj, 3)
    assert np.array_equal(d, P.nodal_vectors(m.ID, u))
    cnn = np.fromfile(tmp_path / topo.find("DataItem").text, dtype="<i4")
    assert cnn.size == 21 * m.nel and np.all(cnn[::21] == 48)
    xyz = np.fromfile(tmp_path / grid.find("Geometry").find("DataItem").text, dtype="<f8").reshape(m.nj, 3)
    assert np.array_equal(xyz, m.xyz)
    coll = P.write_collection(str(tmp_path), "box", [xmf])
    assert os.path.basename(coll) == "box_All.xmf"
    assert xmf in open(coll).read()
