"""Restated step-3 partitioner against the box-mesh generator: equation numbering,
material extension map and history equations must agree bit for bit at one part;
several parts keep the reference's numbering invariants; the .Inv_DS and step-3
input files round-trip."""
import os
import tempfile

import numpy as np
import pytest

from hirensi_b200 import pic
from hirensi_b200.mesh import box_mesh


@pytest.fixture(scope="module")
def mesh():
    return box_mesh(4, 3, 2, 2.5, 2)


def _flags(m):
    return (m.ID < 0).astype(np.int64)


def test_one_part_numbering_equals_mesh_ids(mesh):
    num = pic.numbering(mesh.inod, _flags(mesh), np.ones(mesh.nel, dtype=np.int64), 1)
    assert np.array_equal(num.global_petsc_num, np.arange(1, mesh.nj + 1))
    assert np.array_equal(num.equation_ids(), mesh.ID)
    assert num.neq_total == mesh.neq
    assert np.array_equal(num.id_application, num.id_petsc)


def test_material_map_equals_mesh_extension(mesh):
    s3 = pic.from_mesh(mesh)
    mat = pic.het_mat_numbering(mesh.xyz, mesh.inod, s3.pml_dim[0])
    assert np.array_equal(mat.node_mat_id, mesh.node_mat_id)
    assert np.array_equal(mat.node_mat_mapping - 1, mesh.extend_to)
    # regions: every PML element is one of the 17 PML regions, RD elements are 18
    assert np.array_equal(mat.element_region == 18, mesh.mtel == 1)


def test_one_part_inversion_sets_equal_mesh_history(mesh):
    s3 = pic.from_mesh(mesh)
    num = pic.numbering(mesh.inod, s3.flags, np.ones(mesh.nel, dtype=np.int64), 1)
    mat = pic.het_mat_numbering(mesh.xyz, mesh.inod, s3.pml_dim[0])
    (ds,) = pic.inversion_ds(num, mat, s3.flags)
    assert np.array_equal(ds.u_store_numbers_global, mesh.store_eq)
    assert np.array_equal(ds.idx_u_from, mesh.store_eq) and np.array_equal(ds.idx_u_to, mesh.store_eq)
    assert np.array_equal(ds.idx_mat_extend_to, np.arange(mesh.nj))
    assert np.array_equal(ds.idx_mat_extend_from, mesh.extend_to)
    assert ds.nstore_mapping == mesh.nstore == ds.nstore_rank


@pytest.mark.parametrize("nparts", [2, 3])
def test_several_parts_keep_numbering_invariants(mesh, nparts):
    flags = _flags(mesh)
    epart = (mesh.eid[:, 0] * nparts) // (mesh.eid[:, 0].max() + 1) + 1    # slabs along x
    num = pic.numbering(mesh.inod, flags, epart, nparts)
    # PETSc node numbers are a permutation; a node is owned by the lowest part holding it
    assert np.array_equal(np.sort(num.global_petsc_num), np.arange(1, mesh.nj + 1))
    lowest = np.argmax(num.member, axis=1) + 1
    assert np.array_equal(num.npart, lowest)
    # parts number their nodes in blocks, in node order inside each block
    for p in range(nparts):
        own = np.nonzero(num.npart == p + 1)[0]
        g = num.global_petsc_num[own]
        assert np.array_equal(g, np.arange(g[0], g[0] + own.size))
    # equations: same count, a permutation of the one-part numbering's free DOFs
    ids = num.equation_ids()
    assert np.array_equal(ids >= 0, mesh.ID >= 0)
    assert np.array_equal(np.sort(ids[ids >= 0]), np.arange(mesh.neq))
    assert num.neq_rank[-1] == mesh.neq
    # equations follow PETSc node order: node-major over free DOFs
    order = np.argsort(num.global_petsc_num)
    seq = ids[order].ravel()
    assert np.array_equal(seq[seq >= 0], np.arange(mesh.neq))
    # index sets of each part are consistent with its nodes
    mat = pic.het_mat_numbering(mesh.xyz, mesh.inod, pic.from_mesh(mesh).pml_dim[0])
    dss = pic.inversion_ds(num, mat, flags)
    assert sum(d.nj_mapping for d in dss) == mesh.nj
    assert sum(d.nstore_mapping for d in dss) == mesh.nstore
    allstore = np.concatenate([d.u_store_numbers_global for d in dss])
    assert np.array_equal(np.sort(allstore), np.sort(ids[mesh.store_nodes][:, :3].ravel()))


def test_small_two_part_example_by_hand():
    # two 27-node elements sharing a face: 45 nodes, the shared face nodes are ghosts of part 1
    m = box_mesh(1, 1, 1, 2.0, 1)
    e0, e1 = 0, 1                      # neighbours along x
    inod = m.inod[[e0, e1]]
    used = np.unique(inod)
    remap = np.full(m.nj, -1)
    remap[used] = np.arange(used.size)
    inod = remap[inod]
    flags = np.zeros((used.size, 9), dtype=np.int64)
    num = pic.numbering(inod, flags, np.array([1, 2]), 2)
    shared = np.intersect1d(inod[0], inod[1])
    assert shared.size == 9
    assert np.all(num.npart[shared] == 1)
    assert num.nnode_rank.tolist() == [27, 45]
    assert num.neq_rank.tolist() == [27 * 9, 45 * 9]
    assert num.nj_rank.tolist() == [27, 27]


def test_inv_ds_file_round_trip(mesh):
    s3 = pic.from_mesh(mesh)
    num = pic.numbering(mesh.inod, s3.flags, np.ones(mesh.nel, dtype=np.int64), 1)
    mat = pic.het_mat_numbering(mesh.xyz, mesh.inod, s3.pml_dim[0])
    (ds,) = pic.inversion_ds(num, mat, s3.flags)
    with tempfile.TemporaryDirectory() as d:
        path = os.path.join(d, "Mesh_1_0.Inv_DS")
        pic.write_inv_ds(path, ds)
        first = open(path).readline()
        assert first.endswith("NJ_Rank(IParts) | NJ_Mapping | NStore_Mapping | NStore_Rank\n")
        assert first[:44] == "".join(f"{v:10d} " for v in (ds.nj_rank, ds.nj_mapping, ds.nstore_mapping, ds.nstore_rank))
        back = pic.read_inv_ds(path)
    for f in ("idx_mat_from", "idx_mat_extend_from", "idx_mat_extend_to", "u_store_numbers_global", "idx_u_from", "idx_u_to"):
        assert np.array_equal(getattr(back, f), getattr(ds, f)), f


def test_step3_input_round_trip(mesh):
    hist = mesh.store_nodes[:5]
    s3 = pic.from_mesh(mesh, pmat=np.arange(16.0).reshape(2, 8), history_nodes=hist)
    with tempfile.TemporaryDirectory() as d:
        pic.write_step3(s3, d, "Mesh")
        back = pic.read_step3(d, "Mesh")
    assert np.array_equal(back.xyz, s3.xyz)
    assert np.array_equal(back.inod, s3.inod)
    for f in ("mtel", "elt", "elgr", "flags", "ndan"):
        assert np.array_equal(getattr(back, f), getattr(s3, f)), f
    assert np.array_equal(back.pmat, s3.pmat)
    assert np.array_equal(back.pml_dim, s3.pml_dim)
    # the mesh read back numbers to the same equations
    num = pic.numbering(back.inod, back.flags, np.ones(back.inod.shape[0], dtype=np.int64), 1)
    assert np.array_equal(num.equation_ids(), mesh.ID)


def test_configuration_mesh_is_bit_exact():
    m = box_mesh(16, 16, 8, 2.5, 3)
    s3 = pic.from_mesh(m)
    num = pic.numbering(m.inod, s3.flags, np.ones(m.nel, dtype=np.int64), 1)
    mat = pic.het_mat_numbering(m.xyz, m.inod, s3.pml_dim[0])
    (ds,) = pic.inversion_ds(num, mat, s3.flags)
    assert np.array_equal(num.equation_ids(), m.ID)
    assert np.array_equal(mat.node_mat_mapping - 1, m.extend_to)
    assert np.array_equal(ds.u_store_numbers_global, m.store_eq)
