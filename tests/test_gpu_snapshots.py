"""Checkpointed forward states (hrn_get_state) and the snapshots written from them."""
import os

import numpy as np
import pytest

from problems import RHO, tiny

pytestmark = pytest.mark.gpu


def _solver(p, ckpt):
    from hirensi_b200.solver import Solver
    s = Solver("fp64")
    s.set_mesh(p["mesh"], RHO)
    s.assemble(p["lam"], p["mu"])
    s.set_history(p["mesh"].store_eq)
    s.set_shots(p["nstep"], p["dt"], p["src_eq"], p["src_b"], p["ftab"])
    s.set_receivers(p["eqdis"], p["eqdis_map"])
    s.set_variant(41, 41)
    if ckpt:
        s.set_checkpointing(ckpt)
    return s


def test_states_equal_the_history_rows(gpu_lib, tmp_path):
    from hirensi_b200 import snapshots as P
    from hirensi_b200.capi import HrnError
    p = tiny(nshot=2, nstep=90)
    with _solver(p, 0) as s0:
        s0.forward()
        hist = [s0.history(k) for k in range(2)]
    se = p["mesh"].store_eq
    with _solver(p, 30) as s:
        s.forward()
        for k in range(2):
            for step in (0, 30, 60, 90):
                x1, x2, x3 = s.state(step, k)
                assert np.array_equal(x2[se], hist[k][step])
                if step == 0:
                    assert not x1.any() and not x2.any() and not x3.any()
        with pytest.raises(HrnError):
            s.state(31, 0)
        coll = P.write_forward(str(tmp_path), "tiny", s, p["mesh"], p["dt"], shot=1)
        text = open(coll).read()
        for step in (0, 30, 60, 90):
            assert f"tiny_{step}.xmf" in text
            d = np.fromfile(os.path.join(tmp_path, f"Data_tiny_{step}_Dis.bin"), dtype="<f4").reshape(-1, 3)
            assert np.array_equal(d, P.nodal_vectors(p["mesh"].ID, s.state(step, 1)[1]))
