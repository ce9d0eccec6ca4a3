"""Forward-wavefield checkpointing: with the history recomputed segment by
segment from stored forward states, the misfit, receiver traces and adjoint
history equal those of the full-history run exactly (the same kernels run on the
same values in the same order), and so does the gradient, whose element-point
contributions are summed per node in a fixed order."""
import numpy as np
import pytest

from problems import RHO, oracle_forward, tiny, traces_from_history

pytestmark = pytest.mark.gpu


def _run(p, dis, precision, variant, interval):
    from hirensi_b200.solver import Solver
    with Solver(precision) as s:
        s.set_mesh(p["mesh"], RHO)
        s.assemble(p["lam"], p["mu"])
        s.set_history(p["mesh"].store_eq)
        s.set_shots(p["nstep"], p["dt"], p["src_eq"], p["src_b"], p["ftab"])
        s.set_receivers(p["eqdis"], p["eqdis_map"])
        s.set_variant(variant, variant)
        s.set_checkpointing(interval)
        s.forward()
        J = s.misfit(dis)
        tr = s.traces()
        gl, gm = s.adjoint_gradient(dis, keep_p=True)
        ph = [s.adjoint_history(k) for k in range(p["nshot"])]
    return J, tr, gl, gm, ph


@pytest.mark.parametrize("precision,variant,interval", [("fp64", 41, 1), ("fp64", 41, 7), ("fp64", 41, 60),
                                                        ("fp64", 90, 13), ("fp32", 41, 9), ("fp64", 45, 7)])
def test_checkpointed_adjoint_equals_full_history(gpu_lib, precision, variant, interval):
    p = tiny(nshot=2, nstep=60)
    _, _, hist_t = oracle_forward(p, p["lam_t"], p["mu_t"])
    dis = np.stack([traces_from_history(p, h) for h in hist_t])
    full = _run(p, dis, precision, variant, 0)
    ck = _run(p, dis, precision, variant, interval)
    assert full[0] > 0 and full[0] == ck[0]
    assert np.array_equal(full[1], ck[1])
    assert np.abs(full[3]).max() > 0
    assert np.array_equal(full[2], ck[2])
    assert np.array_equal(full[3], ck[3])
    for a, b in zip(full[4], ck[4]):
        assert np.array_equal(a, b)


def test_history_is_not_kept_with_checkpointing(gpu_lib):
    from hirensi_b200.solver import HrnError, Solver
    p = tiny(nshot=1, nstep=20)
    with Solver("fp64") as s:
        s.set_mesh(p["mesh"], RHO)
        s.assemble(p["lam"], p["mu"])
        s.set_history(p["mesh"].store_eq)
        s.set_shots(p["nstep"], p["dt"], p["src_eq"], p["src_b"], p["ftab"])
        s.set_receivers(p["eqdis"], p["eqdis_map"])
        s.set_checkpointing(5)
        s.forward()
        with pytest.raises(HrnError):
            s.history(0)
        assert np.abs(s.traces()).max() > 0
        with pytest.raises(HrnError):
            s.set_checkpointing(-1)
