"""The product's inversion driver (hirensi_b200.inversion.FWI) against the oracle's
independent restatement of the reference's step and line-search rules
(oracle.inversion_loop, S4/Program_Main.F90:379-896), on synthetic misfits that
drive every branch: the step cap of the first iteration and of L-BFGS steps, the
lambda-bias rule, the descent check, Fac_Max_Update / 6 at the third Armijo trial,
the sign flip at the ninth and the stop at the tenth.  The misfit here is a cheap
quadratic stand-in for the forward solve, so these tests run on the CPU; the GPU
test in test_gpu_inversion.py compares the device driver with the same oracle on a
real forward problem."""
import numpy as np
import pytest

import oracle as O
from hirensi_b200.inversion import FWI, ArmijoFailure, InversionConfig

N = 40
PML = np.arange(32, 40)            # the last 8 nodes play the PML
EXTEND = np.arange(N)
EXTEND[PML] = PML - 8              # each takes its interface node's material


class Synthetic:
    """J = 1/2 |A (lam - lam_t)|^2 + 1/2 |B (mu - mu_t)|^2 + coupling; the raw
    gradient follows the reference's sign (g = -raw is dJ/dm) unless `wrong_sign`."""

    def __init__(self, seed=0, wrong_sign=False, at_minimum=False):
        rng = np.random.default_rng(seed)
        self.A = np.eye(N) + 0.1 * rng.standard_normal((N, N))
        self.B = np.eye(N) + 0.1 * rng.standard_normal((N, N))
        self.lt = (100.0 + 20.0 * rng.random(N))[EXTEND]    # PML nodes hold their interface values
        self.mt = (60.0 + 10.0 * rng.random(N))[EXTEND]
        self.wrong = wrong_sign
        self.at_min = at_minimum
        self.rg = rng.standard_normal(N)
        self.start = (self.lt * 0.8, self.mt * 1.15)
        self.last = None
        self.calls = 0

    def J(self, lam, mu):
        self.calls += 1
        self.last = (lam.copy(), mu.copy())
        rl, rm = self.A @ (lam - self.lt), self.B @ (mu - self.mt)
        return 0.5 * float(rl @ rl) + 0.5 * float(rm @ rm) + 0.01 * float((lam - self.lt) @ (mu - self.mt))

    def raw_gradient(self):
        lam, mu = self.last
        if self.at_min:
            return 1e-3 * self.rg, -1e-3 * self.rg          # nonzero, but J rises in every direction
        gl = self.A.T @ (self.A @ (lam - self.lt)) + 0.01 * (mu - self.mt)
        gm = self.B.T @ (self.B @ (mu - self.mt)) + 0.01 * (lam - self.lt)
        return (gl, gm) if self.wrong else (-gl, -gm)

    @staticmethod
    def tv(lam, mu):
        d = np.gradient(lam), np.gradient(mu)
        return d[0] - d[0].mean(), d[1] - d[1].mean(), float(np.abs(d[0]).sum()), float(np.abs(d[1]).sum())


class NumpyBackend:
    """The FWI backend interface over numpy vectors and a Synthetic problem."""

    def __init__(self, prob):
        self.P = prob
        self.n = N

    def zeros(self):
        return np.zeros(N)

    def vec(self, host):
        return np.array(host, dtype=np.float64)

    def host(self, v):
        return v

    def copy(self, src, dst):
        dst[:] = src

    def axpby(self, a, x, b, y, z):
        z[:] = a * x + b * y if y is not None else a * x

    def mul(self, x, y, z):
        z[:] = x * y

    def dot(self, x, y):
        return float(x @ y)

    def norm2(self, x):
        return float(np.sqrt(x @ x))

    def norminf(self, x):
        return float(np.abs(x).max())

    def clip(self, x, lo, hi):
        np.clip(x, lo, hi, out=x)

    def extend(self, x):
        x[:] = x[EXTEND]

    def gradient_mass_inverse(self):
        img = np.ones(N)
        img[PML] = 0.0
        return img, (img > 0).astype(np.float64)

    def tv(self, lam, mu, reg_l, reg_m):
        rl, rm, cl, cm = self.P.tv(lam, mu)
        reg_l[:] = rl
        reg_m[:] = rm
        return cl, cm

    def lbfgs_setup(self, m, restriction):
        self.lb = O.LBFGSCoupled(N, m, restriction)

    def lbfgs_direction(self, it, it0, g_l, g_m, g_l_pre, g_m_pre, lam, mu, lam_pre, mu_pre, p_l, p_m):
        a, b = self.lb.direction(it, it0, g_l, g_m, g_l_pre, g_m_pre, lam, mu, lam_pre, mu_pre)
        p_l[:] = a
        p_m[:] = b

    def forward(self, lam, mu):
        return self.P.J(lam, mu)

    def gradient(self, g_l, g_m):
        a, b = self.P.raw_gradient()
        g_l[:] = a
        g_m[:] = b


def _start(prob):
    return prob.start


def _run_both(cfg, n_iter, make=Synthetic, **kw):
    pa, pb = make(**kw), make(**kw)
    lam0, mu0 = _start(pa)
    fwi = FWI(NumpyBackend(pa), cfg)
    img = np.ones(N)
    img[PML] = 0.0
    restriction = (img > 0).astype(np.float64)

    def run_product():
        return fwi.run(lam0, mu0, n_iter=n_iter)

    def run_oracle():
        def grad():
            return pb.raw_gradient()
        return O.inversion_loop(pb.J, grad, lam0, mu0, n_iter, img, restriction, EXTEND, cfg.bounds_lambda,
                                cfg.bounds_mu, m_lbfgs=cfg.m_lbfgs,
                                fac_max_update=(cfg.fac_max_update_lambda, cfg.fac_max_update_mu),
                                tv=pb.tv if cfg.regularization == "TV" else None, reg_factor=cfg.reg_factor,
                                bias_lambda=cfg.bias_lambda, n_iter_bias=cfg.n_iter_bias, iter_begin=cfg.iter_begin)
    return fwi, run_product, run_oracle, pa, pb


def _compare(h, r, fwi):
    assert len(h) == len(r)
    for a, b in zip(h, r):
        assert a["armijo"] == b["armijo"]
        assert abs(a["misfit"] - b["misfit"]) <= 1e-12 * abs(b["misfit"])
        if b["iter"] > 0:
            assert abs(a["alpha_lambda"] - b["alpha_lambda"]) <= 1e-13 * abs(b["alpha_lambda"])
            assert abs(a["alpha_mu"] - b["alpha_mu"]) <= 1e-13 * abs(b["alpha_mu"])
    assert np.allclose(fwi.lam, r[-1]["lam"], rtol=1e-12, atol=0)
    assert np.allclose(fwi.mu, r[-1]["mu"], rtol=1e-12, atol=0)


@pytest.mark.parametrize("tv", [None, "TV"])
@pytest.mark.parametrize("bias", [True, False])
def test_lbfgs_iterations_follow_the_reference_rules(tv, bias):
    cfg = InversionConfig(m_lbfgs=3, bounds_lambda=(10.0, 1000.0), bounds_mu=(10.0, 1000.0), regularization=tv,
                          bias_lambda=bias)
    fwi, run_p, run_o, _, _ = _run_both(cfg, 6)
    h, r = run_p(), run_o()
    _compare(h, r, fwi)
    assert h[-1]["misfit"] < h[0]["misfit"]


def test_bias_weight_uses_integer_division():
    """Iter < NIterBias: W = 1 - DBLE(Iter/NIterBias) = 1, so lambda moves along p_mu."""
    cfg = InversionConfig(m_lbfgs=3, bounds_lambda=(10.0, 1000.0), bounds_mu=(10.0, 1000.0), regularization=None,
                          n_iter_bias=2, iter_begin=1)
    fwi, run_p, run_o, _, _ = _run_both(cfg, 4)
    _compare(run_p(), run_o(), fwi)


def test_overshooting_steps_backtrack_and_shrink_the_cap():
    """A cap far too large: several Armijo trials per iteration, and from the third
    trial on Fac_Max_Update is divided by 6 for the later iterations."""
    cfg = InversionConfig(m_lbfgs=3, bounds_lambda=(1.0, 1e5), bounds_mu=(1.0, 1e5), regularization="TV",
                          fac_max_update_lambda=400.0, fac_max_update_mu=300.0)
    fwi, run_p, run_o, _, _ = _run_both(cfg, 4)
    h, r = run_p(), run_o()
    assert max(x["armijo"] for x in r) >= 3
    _compare(h, r, fwi)


def test_wrong_gradient_sign_flips_the_step_at_the_ninth_trial():
    # no lambda bias: it would move lambda along the mu direction, which need not ascend
    cfg = InversionConfig(m_lbfgs=3, bounds_lambda=(1.0, 1e5), bounds_mu=(1.0, 1e5), regularization=None,
                          fac_max_update_lambda=0.5, fac_max_update_mu=0.5, bias_lambda=False)
    fwi, run_p, run_o, _, _ = _run_both(cfg, 1, wrong_sign=True)
    h, r = run_p(), run_o()
    assert r[1]["armijo"] == 9 and r[1]["alpha_mu"] < 0 and r[1]["misfit"] < r[0]["misfit"]
    _compare(h, r, fwi)


def test_armijo_stops_after_the_tenth_trial():
    cfg = InversionConfig(m_lbfgs=3, bounds_lambda=(1.0, 1e5), bounds_mu=(1.0, 1e5), regularization=None)

    class AtMinimum(Synthetic):
        def __init__(self, **kw):
            super().__init__(at_minimum=True, **kw)
            self.start = (self.lt.copy(), self.mt.copy())        # the start model is the minimum

    fwi, run_p, run_o, pa, pb = _run_both(cfg, 2, make=AtMinimum)
    with pytest.raises(ArmijoFailure):
        run_p()
    with pytest.raises(O.ArmijoStop):
        run_o()
    assert pa.calls == pb.calls == 1 + 1 + 10     # initial model, first trial, ten backtracking trials
