"""Diagonal pseudo-Hessian (hrn_pseudo_hessian): the gradient's zero-lag correlation
with the forward wavefield in both slots, against the oracle's control restatement
fed the forward history twice (FP64 bar 1e-10)."""
import numpy as np
import pytest

import oracle as O
from problems import RHO, oracle_forward, rel_l2, tiny

pytestmark = pytest.mark.gpu


def test_pseudo_hessian_matches_oracle(gpu_lib):
    import torch
    from hirensi_b200.inversion import DeviceBackend
    from hirensi_b200.solver import Solver
    p = tiny(nshot=2, nstep=120)
    om, S, hist = oracle_forward(p, p["lam"], p["mu"])
    ref_l, ref_m = 0.0, 0.0
    for k in range(2):
        a, b = O.control(om, p["nstep"], p["dt"], p["mesh"].store_eq, hist[k], hist[k])
        ref_l, ref_m = ref_l + a, ref_m + b
    with Solver("fp64") as s:
        s.set_mesh(p["mesh"], RHO)
        s.assemble(p["lam"], p["mu"])
        s.set_history(p["mesh"].store_eq)
        s.set_shots(p["nstep"], p["dt"], p["src_eq"], p["src_b"], p["ftab"])
        s.set_receivers(p["eqdis"], p["eqdis_map"])
        s.forward()
        be = DeviceBackend(s, p["mesh"])
        h_l, h_m = be.pseudo_hessian()
        torch.cuda.synchronize()
    assert np.abs(ref_m).max() > 0
    assert rel_l2(h_l, ref_l) < 1e-10
    assert rel_l2(h_m, ref_m) < 1e-10
    # a diagonal of squares: never negative where the oracle is clearly positive
    assert np.all(h_m[ref_m > 1e-6 * ref_m.max()] > 0)
