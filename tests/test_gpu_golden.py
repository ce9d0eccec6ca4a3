"""The CUDA path (FP64, through the C ABI) against the committed golden fixtures of the
oracle (tests/golden/tiny_inversion.npz): seismograms, misfit and gradient within the
FP64 bar 1e-10, without running the oracle."""
import os

import numpy as np
import pytest

from problems import RHO, rel_l2, tiny

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "tiny_inversion.npz")


@pytest.mark.parametrize("variant", [0, 41, 45, 92])
def test_cuda_path_matches_golden_fixtures(gpu_lib, variant):
    from hirensi_b200.solver import Solver
    with np.load(GOLDEN) as d:
        g = {k: d[k] for k in d.files}
    p = tiny(nshot=2, nstep=200, seed=0)
    assert np.array_equal(np.asarray(p["mesh"].ID, dtype=np.int32), g["ID"])
    with Solver("fp64") as s:
        s.set_mesh(p["mesh"], RHO)
        s.assemble(p["lam"], p["mu"])
        s.set_history(p["mesh"].store_eq)
        s.set_shots(p["nstep"], p["dt"], p["src_eq"], p["src_b"], p["ftab"])
        s.set_receivers(p["eqdis"], p["eqdis_map"])
        if variant:
            s.set_variant(variant, variant)
        s.forward()
        assert rel_l2(s.traces(), g["traces0"]) < 1e-10
        J = s.misfit(g["dis"])
        gl, gm = s.adjoint_gradient(g["dis"])
    assert abs(J - float(g["misfit"])) <= 1e-10 * float(g["misfit"])
    assert rel_l2(gl, g["g_lambda"]) < 1e-10
    assert rel_l2(gm, g["g_mu"]) < 1e-10
