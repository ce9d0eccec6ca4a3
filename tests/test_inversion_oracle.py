"""The FWI driver (S4/Program_Main.F90:379-921 control flow) on the oracle backend (CPU)."""
import numpy as np
import pytest

import oracle as O
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


@pytest.mark.parametrize("reg", [None, "TV"])
def test_driver_on_the_oracle_follows_the_oracle_loop(reg):
    """hirensi_b200.inversion.FWI on the oracle backend and oracle.inversion_loop (the
    oracle's own restatement of the step and line-search rules) on the same forward
    problem: the same misfits, step sizes, Armijo trials and models."""
    from fwi_oracle import loop_primitives
    p, be = setup()
    cfg = InversionConfig(m_lbfgs=5, bounds_lambda=(10.0, 1000.0), bounds_mu=(10.0, 1000.0), regularization=reg)
    fwi = FWI(be, cfg)
    hist = fwi.run(p["lam"], p["mu"], n_iter=2)
    _, be2 = setup()
    evaluate, gradient, tv, img, restriction, extend_to = loop_primitives(be2)
    ref = O.inversion_loop(evaluate, gradient, p["lam"], p["mu"], 2, img, restriction, extend_to, cfg.bounds_lambda,
                           cfg.bounds_mu, m_lbfgs=5, tv=tv if reg else None)
    assert [h["armijo"] for h in hist] == [h["armijo"] for h in ref]
    for a, b in zip(hist, ref):
        assert abs(a["misfit"] - b["misfit"]) <= 1e-12 * b["misfit"]
    assert np.allclose(fwi.lam, ref[-1]["lam"], rtol=1e-12, atol=0)
    assert np.allclose(fwi.mu, ref[-1]["mu"], rtol=1e-12, atol=0)


@pytest.mark.parametrize("memory", [1, 2, 10])
def test_coupled_lbfgs_terminates_on_a_quadratic_with_exact_steps(memory):
    """Known answer of the two-loop recursion: on a strictly convex quadratic in the
    coupled (lambda, mu) vector, with exact line searches, L-BFGS with H0 = (y's)/(y'y)
    of the newest pair makes the conjugate-gradient directions (scaled), so it reaches
    the minimum in at most dim steps for any memory >= 1 (the ring buffer wraps for
    memory < dim)."""
    rng = np.random.default_rng(3)
    nj = 4
    Q = rng.standard_normal((2 * nj, 2 * nj))
    A = Q @ Q.T + 0.5 * np.eye(2 * nj)
    b = rng.standard_normal(2 * nj)
    lb = O.LBFGSCoupled(nj, memory, np.ones(nj))
    x = np.zeros(2 * nj)
    g = A @ x - b
    g0 = np.linalg.norm(g)
    x_pre = g_pre = None
    for it in range(1, 2 * nj + 1):
        if it == 1:
            p_l, p_m = lb.direction(it, 1, g[:nj], g[nj:], None, None, x[:nj], x[nj:], None, None)
        else:
            p_l, p_m = lb.direction(it, 1, g[:nj], g[nj:], g_pre[:nj], g_pre[nj:], x[:nj], x[nj:],
                                    x_pre[:nj], x_pre[nj:])
        p = np.concatenate([p_l, p_m])
        assert g @ p < 0                       # a descent direction every time
        alpha = -(g @ p) / (p @ A @ p)         # exact line search
        x_pre, g_pre = x.copy(), g.copy()
        x = x + alpha * p
        g = A @ x - b
    assert np.linalg.norm(g) < 1e-9 * g0
