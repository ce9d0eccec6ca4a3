"""Face-traction loading on the device (hrn_assemble_face_force,
hrn_set_shots_face_force) against the oracle's ASSEM_FORCE_PETSC_3D / ELEMENT_FS_3D
(S4/Assemble_PETSc_3D.F90:444-548, S4/Element_Matrices_3D.F90:890-1096): the
force vector B of a unit vertical traction on the loaded faces (ID_BC(:, 1)), the
face-6-as-5 adjustment, the stop on a loaded face off the surface, and a forward
solve loaded by the device B against the oracle's forward with its own B."""
import numpy as np
import pytest

import oracle as O
from problems import RHO, rel_l2, tiny

pytestmark = pytest.mark.gpu


def _surface_load(mesh, face=5):
    """nface per element: `face` on the regular-domain elements touching z = 0."""
    top = mesh.xyz[mesh.inod, 2].max(axis=1)
    nface = np.zeros(mesh.nel, np.int32)
    nface[(mesh.mtel == 1) & (np.abs(top) < 1e-9)] = face
    return nface


def _solver(p):
    from hirensi_b200.solver import Solver
    s = Solver("fp64")
    s.set_mesh(p["mesh"], RHO)
    s.assemble(p["lam"], p["mu"])
    s.set_history(p["mesh"].store_eq)
    return s


@pytest.mark.parametrize("mesh_size", [(4, 4, 2, 1), (16, 16, 8, 3)])
def test_face_force_vector_matches_oracle(gpu_lib, mesh_size):
    from hirensi_b200.mesh import box_mesh
    from problems import layered
    nx, ny, nz, npml = mesh_size
    m = box_mesh(nx, ny, nz, 2.5, npml)
    lam, mu = layered(m)
    nface = _surface_load(m)
    assert np.count_nonzero(nface) == nx * ny
    om = O.OracleMesh(m, RHO)
    _, b_ref = O.OracleSystem.assemble(om, lam, mu, id_bc=nface).vectors()
    p = dict(mesh=m, lam=lam, mu=mu)
    with _solver(p) as s:
        b = s.assemble_face_force(nface)
        b6 = s.assemble_face_force(np.where(nface == 5, 6, 0).astype(np.int32))
    assert np.count_nonzero(b_ref) > 0
    assert rel_l2(b, b_ref) <= 1e-13
    assert np.array_equal(np.nonzero(b)[0], np.nonzero(b_ref)[0])
    # only vertical entries, and the total force is the loaded area (unit traction)
    zeq = m.ID[:, 2]
    assert np.all(b[np.setdiff1d(np.arange(m.neq), zeq[zeq >= 0])] == 0.0)
    (x0, x1), (y0, y1), _ = m.rd_box
    assert abs(b.sum() - (x1 - x0) * (y1 - y0)) <= 1e-12 * (x1 - x0) * (y1 - y0)
    assert np.array_equal(b6, b)


def test_face_off_the_surface_is_refused(gpu_lib):
    p = tiny(nshot=1, nstep=10)
    m = p["mesh"]
    nface = _surface_load(m)
    bottom = m.xyz[m.inod, 2].min(axis=1)
    deep = np.nonzero((m.mtel == 1) & (bottom < -2.0))[0][0]
    nface[deep] = 5
    from hirensi_b200.capi import HrnError
    with _solver(p) as s:
        with pytest.raises(HrnError) as ei:
            s.assemble_face_force(nface)
        assert ei.value.code == 6           # HRN_EMESH


def test_forward_loaded_by_the_device_face_force(gpu_lib):
    p = tiny(nshot=2, nstep=150)
    m = p["mesh"]
    nface = _surface_load(m)
    om = O.OracleMesh(m, RHO)
    S = O.OracleSystem.assemble(om, p["lam"], p["mu"], id_bc=nface)
    _, b_ref = S.vectors()
    with _solver(p) as s:
        s.assemble_face_force(nface)
        s.set_shots_face_force(p["nstep"], p["dt"], p["ftab"])
        s.set_receivers(p["eqdis"], p["eqdis_map"])
        s.forward()
        for k in range(2):
            u_ref = S.forward(b_ref, p["ftab"][k], p["nstep"], p["dt"], m.store_eq)
            assert np.abs(u_ref).max() > 0
            assert rel_l2(s.history(k), u_ref) < 1e-10
