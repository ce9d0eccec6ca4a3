"""The FWI driver (S4/Program_Main.F90:379-921 control flow) on the oracle backend (CPU)."""
import numpy as np
import pytest

from fwi_oracle import OracleBackend
from hirensi_b200.inversion import FWI, InversionConfig
from problems import oracle_forward, tiny, traces_from_history


def setup(nstep=160):
    p = tiny(nshot=2, nstep=nstep)
    _, _, hist_t = oracle_forward(p, p["lam_t"], p["mu_t"])
    dis = [traces_from_history(p, h) for h in hist_t]
    shots = []
    for s in range(p["nshot"]):
        b = np.zeros(p["mesh"].neq)
        b[p["src_eq"][s]] = 1.0
        shots.append((b, p["ftab"][s]))
    be = OracleBackend(p["mesh"], shots, p["nstep"], p["dt"], p["eqdis"], p["eqdis_map"], dis)
    return p, be


@pytest.mark.parametrize("reg", [None, "TV"])
def test_lbfgs_iterations_reduce_the_misfit(reg):
    p, be = setup()
    cfg = InversionConfig(m_lbfgs=5, bounds_lambda=(10.0, 1000.0), bounds_mu=(10.0, 1000.0), regularization=reg)
    hist = FWI(be, cfg).run(p["lam"], p["mu"], n_iter=3)
    J = [h["misfit"] for h in hist]
    assert J[0] > 0 and all(np.isfinite(J))
    assert all(J[i + 1] <= J[i] for i in range(len(J) - 1))   # Armijo accepted every step
    assert J[-1] < J[0]
    assert all(h["armijo"] < 10 for h in hist[1:])
