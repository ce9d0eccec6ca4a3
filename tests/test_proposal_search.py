"""The line search of a preconditioner's proposal in hirensi_b200.inversion.FWI (no
reference counterpart): Armijo on the true misfit plus the weak curvature condition,
doubling a step that stops short, falling back to the reference's L-BFGS path when
the first trial fails, and handing the trial point's gradient to the next iteration.

The misfit is the quadratic stand-in of test_inversion_rules; a proposal pointing
at the true model m* gives J(m + t (m* - m)) = (1 - t)^2 J(m) and a directional
derivative (1 - t) g.q, so the curvature condition with c2 = 0.9 holds from
t = 0.1 on."""
import numpy as np
import pytest

from hirensi_b200.inversion import FWI, InversionConfig
from test_inversion_rules import EXTEND, PML, NumpyBackend, Synthetic


class Toward:
    """Proposes the step to the true model."""

    def __init__(self, prob):
        self.P = prob
        self.calls = 0

    def direction(self, backend, g_l, g_m, lam, mu):
        self.calls += 1
        return self.P.lt - lam, self.P.mt - mu


class CountingBackend(NumpyBackend):
    def __init__(self, prob):
        super().__init__(prob)
        self.forwards = 0
        self.gradients = 0

    def forward(self, lam, mu):
        self.forwards += 1
        return super().forward(lam, mu)

    def gradient(self, g_l, g_m):
        self.gradients += 1
        super().gradient(g_l, g_m)


class Walled(Synthetic):
    """The quadratic plus a steep wall once lambda has moved by more than `thr` at
    some node from the start (its gradient is only asked for inside the wall)."""

    def __init__(self, thr, **kw):
        super().__init__(**kw)
        self.thr = thr

    def J(self, lam, mu):
        d = float(np.abs(lam - self.start[0]).max())
        return super().J(lam, mu) + 1e9 * max(0.0, d - self.thr) ** 2


def _cfg(prob, t0, search="wolfe"):
    """Caps chosen so that the first trial is t0 of the way to the true model."""
    ql = prob.lt - prob.start[0]
    qm = prob.mt - prob.start[1]
    return InversionConfig(m_lbfgs=3, bounds_lambda=(1.0, 1e5), bounds_mu=(1.0, 1e5), regularization=None,
                           fac_max_update_lambda=t0 * float(np.abs(ql).max()),
                           fac_max_update_mu=t0 * float(np.abs(qm).max()), proposal_search=search)


def _img():
    img = np.ones(len(EXTEND))
    img[PML] = 0.0
    return img


def test_short_proposal_doubles_until_the_curvature_condition_holds():
    p = Synthetic()
    b = CountingBackend(p)
    J0 = p.J(*p.start)
    fwi = FWI(b, _cfg(p, 0.04), preconditioner=Toward(p))
    h = fwi.run(*p.start, n_iter=1)
    s = h[1]["search"]
    # t = 0.04 and 0.08 stop short of the curvature (t < 0.1); t = 0.16 meets it
    assert h[1]["learned"] and s == {"trials": 3, "scale": 4.0, "curvature": True}
    assert h[1]["misfit"] == pytest.approx((1 - 0.16) ** 2 * J0, rel=1e-12)
    assert np.allclose(fwi.lam, p.start[0] + 0.16 * (p.lt - p.start[0]), rtol=1e-13, atol=0)
    # one forward for J0 and one per trial; one gradient for iteration 1, one per trial
    assert b.forwards == 1 + 3 and b.gradients == 1 + 3
    assert (h[-1]["forward_solves"], h[-1]["adjoint_solves"]) == (b.forwards, b.gradients)


def test_accepted_proposal_hands_its_gradient_to_the_next_iteration():
    p = Synthetic()
    b = CountingBackend(p)
    fwi = FWI(b, _cfg(p, 0.3), preconditioner=Toward(p))
    h = fwi.run(*p.start, n_iter=2)
    assert h[1]["search"] == {"trials": 1, "scale": 1.0, "curvature": True}
    assert h[2]["search"]["trials"] == 1
    # iteration 2 took the gradient of iteration 1's trial instead of computing it again
    assert b.gradients == 1 + h[1]["search"]["trials"] + h[2]["search"]["trials"]
    lam1 = p.start[0] + 0.3 * (p.lt - p.start[0])
    mu1 = p.start[1] + 0.3 * (p.mt - p.start[1])
    p.J(lam1, mu1)
    gl, _ = p.raw_gradient()
    assert h[2]["g_lambda"] == pytest.approx(np.linalg.norm(-gl * _img()), rel=1e-12)


def test_overshooting_first_trial_falls_back_to_lbfgs():
    p = Synthetic()
    b = CountingBackend(p)
    J0 = p.J(*p.start)
    fwi = FWI(b, _cfg(p, 2.5), preconditioner=Toward(p))
    h = fwi.run(*p.start, n_iter=1)
    assert not h[1]["learned"] and h[1]["search"] == {"trials": 1}
    assert h[1]["misfit"] < J0
    # the same iteration without a proposal (its L-BFGS path is the reference's)
    p2 = Synthetic()
    h2 = FWI(NumpyBackend(p2), _cfg(p2, 2.5)).run(*p2.start, n_iter=1)
    assert h[1]["misfit"] == h2[1]["misfit"] and h[1]["armijo"] == h2[1]["armijo"]
    assert np.array_equal(fwi.lam, p2.last[0])


def test_doubled_step_that_fails_armijo_returns_to_the_last_good_trial():
    p0 = Synthetic()
    q_max = float(np.abs(p0.lt - p0.start[0]).max())
    lam1 = p0.start[0] + 0.04 * (p0.lt - p0.start[0])
    mu1 = p0.start[1] + 0.04 * (p0.mt - p0.start[1])

    p = Walled(thr=0.06 * q_max)                     # t = 0.04 inside the wall, 0.08 beyond it
    b = CountingBackend(p)
    J0 = p.J(*p.start)
    fwi = FWI(b, _cfg(p, 0.04), preconditioner=Toward(p))
    h = fwi.run(*p.start, n_iter=1)
    assert h[1]["learned"] and h[1]["search"] == {"trials": 2, "scale": 1.0, "curvature": False}
    assert h[1]["misfit"] == pytest.approx((1 - 0.04) ** 2 * J0, rel=1e-12)
    assert np.allclose(fwi.lam, lam1, rtol=1e-13, atol=0)
    # the accepted model's forward runs again, so the resident state is its own
    assert b.forwards == 1 + 2 + 1 and np.array_equal(p.last[0], fwi.lam)

    # the next iteration uses the gradient of the accepted trial, not of the rejected one
    p = Walled(thr=0.06 * q_max)
    h = FWI(CountingBackend(p), _cfg(p, 0.04), preconditioner=Toward(p)).run(*p.start, n_iter=2)
    q = Synthetic()
    q.J(lam1, mu1)
    gl, _ = q.raw_gradient()
    assert h[2]["g_lambda"] == pytest.approx(np.linalg.norm(-gl * _img()), rel=1e-12)


def test_armijo_only_search_takes_the_first_trial():
    p = Synthetic()
    b = CountingBackend(p)
    J0 = p.J(*p.start)
    fwi = FWI(b, _cfg(p, 0.04, search="armijo"), preconditioner=Toward(p))
    h = fwi.run(*p.start, n_iter=1)
    assert h[1]["learned"] and h[1]["search"] == {"trials": 1, "scale": 1.0}
    assert h[1]["misfit"] == pytest.approx((1 - 0.04) ** 2 * J0, rel=1e-12)
    assert b.gradients == 1
