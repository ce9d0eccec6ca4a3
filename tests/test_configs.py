"""Host-side inputs of the workloads against the oracle (CPU)."""
import numpy as np
import pytest

import oracle as O
from hirensi_b200 import configs


@pytest.mark.parametrize("lcase,fr", [(2, 15.0), (2, 5.0), (2, 60.0), (3, 15.0)])
def test_time_table_matches_the_oracle(lcase, fr):
    """TIME_FUNCTION samples of the workloads (T, T + dt, T + dt/2 per step) equal
    the oracle's to the last bits of libm."""
    dt = 1e-4 if lcase == 2 else 1e-3
    a = configs.time_table(400, dt, lcase, fr)
    b = O.time_table(400, dt, lcase, fr)
    assert a.shape == b.shape == (401, 3)
    assert np.abs(a - b).max() <= 2e-16 * max(np.abs(b).max(), 1.0)


def test_inversion_config_inputs():
    """The bench's inversion workload: 4 shots on the 16 x 16 x 8 + PML 3 mesh, each
    loading one vertical equation with the 15 Hz Ricker table, and the 5 x 5 surface
    receiver grid."""
    p = configs.inversion_config(nstep=50)
    assert p.nshot == 4 and p.mesh.nel == 5324 and p.dof == 55539
    assert p.ftab.shape == (4, 51, 3)
    assert np.array_equal(p.ftab[0], O.time_table(50, p.dt, 2, 15.0)) or \
        np.abs(p.ftab[0] - O.time_table(50, p.dt, 2, 15.0)).max() <= 2e-16
    assert np.array_equal(p.src_b, np.eye(4))
    for e in p.src_eq:                       # the z equation of a surface node
        node, dof = np.argwhere(p.mesh.ID == e)[0]
        assert dof == 2 and p.mesh.xyz[node, 2] == 0.0
    assert len(p.eqdis) == 3 * 25
    assert np.all(p.mesh.xyz[np.unique(np.nonzero(np.isin(p.mesh.ID[:, :3], p.eqdis))[0]), 2] == 0.0)


def test_training_config_sizes():
    """The learned preconditioner's training mesh: 40 x 40 x 20 + PML 3 with the sizes
    of the configuration table (48,668 elements, 406,503 nodes, 807,003 displacement
    DOF), 8 surface shots and the 7 x 7 receiver grid."""
    p = configs.training_config(nstep=20)
    m = p.mesh
    assert m.nel == 48668 and m.nj == 406503 and p.dof == 807003
    assert p.nshot == 8 and len(p.eqdis) == 3 * 49
    assert p.name == "inversion_40x40x20_pml3"
    assert np.all(m.xyz[np.unique(np.nonzero(np.isin(m.ID[:, 2], p.src_eq))[0]), 2] == 0.0)
