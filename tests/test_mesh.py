"""Integer layout of the generated meshes (bit-exact numbering rules, CPU)."""
import numpy as np
import pytest

from hirensi_b200.mesh import GLL_TO_LOCAL, LOCAL_IJK, box_mesh, element_colors, surface_grid


def test_config1_sizes():
    m = box_mesh(16, 16, 8, 2.5, 3)
    assert m.nel == 5324 and m.nj == 46575
    assert m.rd_dof == 55539          # 3 x (RD + interface nodes)
    assert int((m.mtel == 1).sum()) == 16 * 16 * 8


@pytest.mark.parametrize("nx,ny,nz,npml,nel,nj,dof,neq", [
    (40, 40, 20, 3, 48668, 406503, 807003, 2083956),        # training meshes
    (80, 80, 40, 4, 340736, 2788281, 6298803, 12679806),    # batched uneven shots
])
def test_larger_config_sizes(nx, ny, nz, npml, nel, nj, dof, neq):
    """Element, node and regular-domain DOF counts of the larger box meshes, and the
    equation count (PML nodes carry 9 equations, the outer faces fix u)."""
    m = box_mesh(nx, ny, nz, 2.5, npml)
    assert m.nel == nel and m.nj == nj
    assert m.rd_dof == dof
    assert m.neq == neq
    assert int((m.mtel == 1).sum()) == nx * ny * nz


def test_constraint_and_numbering_rules():
    m = box_mesh(4, 3, 2, 2.5, 2)
    NX, NY, NZ = m.lattice
    ID = m.ID
    in_pml = np.zeros(m.nj, bool)
    in_pml[m.inod[m.mtel == 2].ravel()] = True
    # stress DOFs exist exactly on nodes of PML elements (interface included)
    assert np.all((ID[:, 3:] >= 0).all(axis=1) == in_pml)
    assert np.all((ID[:, 3:] < 0).all(axis=1) == ~in_pml)
    # outer faces (not the free surface) have fixed displacements
    i = np.arange(m.nj) % NX
    j = (np.arange(m.nj) // NX) % NY
    k = np.arange(m.nj) // (NX * NY)
    outer = (i == 0) | (i == NX - 1) | (j == 0) | (j == NY - 1) | (k == 0)
    assert np.all((ID[:, :3] < 0).all(axis=1) == outer)
    # equations are numbered node by node, DOF 1..9, free ones only, from 0
    flat = ID.ravel()
    free = flat[flat >= 0]
    assert np.array_equal(free, np.arange(m.neq))
    # history equations: x, y, z displacement of RD + interface nodes in node order
    nodes = np.nonzero(m.node_mat_id <= 1)[0]
    assert np.array_equal(m.store_eq, ID[nodes, :3].ravel())
    assert np.all(np.diff(m.store_eq) > 0)


def test_element_local_order_and_geometry():
    m = box_mesh(2, 2, 1, 2.0, 1)
    for e in (0, m.nel - 1):
        x = m.xyz[m.inod[e]]
        lo = x.min(axis=0)
        for n, (a, b, c) in enumerate(LOCAL_IJK):
            assert np.allclose(x[n], lo + 1.0 * np.array([a, b, c]))
    for q in range(27):
        a, b, c = LOCAL_IJK[GLL_TO_LOCAL[q]]
        assert q == 9 * c + 3 * b + a


def test_material_extension_map_targets_interface_nodes():
    m = box_mesh(4, 4, 2, 2.5, 2)
    pml_only = np.nonzero(m.node_mat_id == 2)[0]
    tgt = m.extend_to[pml_only]
    assert np.all(m.node_mat_id[tgt] == 1)
    keep = np.nonzero(m.node_mat_id <= 1)[0]
    assert np.array_equal(m.extend_to[keep], keep)
    # the target is the perpendicular projection onto the RD box
    (x0, x1), (y0, y1), (z0, _) = m.rd_box
    proj = np.clip(m.xyz[pml_only], [x0, y0, z0], [x1, y1, 0.0])
    assert np.allclose(m.xyz[tgt], proj)


def test_colouring_separates_elements_sharing_nodes():
    m = box_mesh(3, 3, 2, 1.0, 1)
    col = element_colors(m)
    for c in range(8):
        nodes = m.inod[col == c].ravel()
        assert np.unique(nodes).size == nodes.size


def test_receivers_and_store_positions():
    m = box_mesh(16, 16, 8, 2.5, 3)
    rec = surface_grid(m, [-15, -7.5, 0, 7.5, 15])
    assert rec.size == 25 and np.all(m.xyz[rec, 2] == 0.0)
    eq = m.equations(rec)
    pos = m.store_position(eq)
    assert np.array_equal(m.store_eq[pos], eq)
