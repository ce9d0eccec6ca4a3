"""Device model update (vector kernels, TV, gradient mass, coupled L-BFGS) and the
FWI driver on the device against the oracle's restatement of the inversion loop."""
import numpy as np
import pytest

import oracle as O
from fwi_oracle import OracleBackend
from hirensi_b200.inversion import FWI, DeviceBackend, InversionConfig
from problems import RHO, oracle_forward, rel_l2, tiny, traces_from_history

pytestmark = pytest.mark.gpu


def _device(p, dis):
    from hirensi_b200.solver import Solver
    s = Solver("fp64")
    s.set_mesh(p["mesh"], RHO)
    s.assemble(p["lam"], p["mu"])
    s.set_history(p["mesh"].store_eq)
    s.set_shots(p["nstep"], p["dt"], p["src_eq"], p["src_b"], p["ftab"])
    s.set_receivers(p["eqdis"], p["eqdis_map"])
    s.set_data(np.stack(dis))
    return s


def test_vector_kernels_tv_mass_and_lbfgs(gpu_lib):
    p = tiny(nshot=1, nstep=20)
    rng = np.random.default_rng(1)
    s = _device(p, [np.zeros((p["eqdis"].size, p["nstep"] + 1))])
    dev = DeviceBackend(s, p["mesh"])
    n = p["mesh"].nj
    x, y = rng.standard_normal(n), rng.standard_normal(n)
    X, Y, Z = dev.vec(x), dev.vec(y), dev.zeros()
    assert abs(dev.dot(X, Y) - x @ y) < 1e-12 * np.abs(x) @ np.abs(y)
    assert abs(dev.norm2(X) - np.linalg.norm(x)) < 1e-13 * np.linalg.norm(x)
    assert dev.norminf(X) == np.abs(x).max()
    dev.axpby(2.0, X, -3.0, Y, Z)
    assert np.array_equal(dev.host(Z), 2.0 * x + -3.0 * y)
    dev.clip(Z, -1.0, 1.0)
    assert np.array_equal(dev.host(Z), np.clip(2.0 * x - 3.0 * y, -1.0, 1.0))
    dev.extend(X)
    assert np.array_equal(dev.host(X), x[p["mesh"].extend_to])
    # TV regularization and gradient mass
    om = O.OracleMesh(p["mesh"], RHO)
    rl, rm, cl, cm = O.tv_reg(om, p["lam_t"], p["mu_t"])
    RL, RM = dev.zeros(), dev.zeros()
    dcl, dcm = dev.tv(dev.vec(p["lam_t"]), dev.vec(p["mu_t"]), RL, RM)
    assert rel_l2(dev.host(RL), rl) < 1e-12 and rel_l2(dev.host(RM), rm) < 1e-12
    assert abs(dcl - cl) < 1e-12 * abs(cl) and abs(dcm - cm) < 1e-12 * abs(cm)
    img, restr = dev.gradient_mass_inverse()
    img_r, restr_r = O.inverse_gradient_mass(O.rmg(om))
    assert rel_l2(dev.host(img), img_r) < 1e-14 and np.array_equal(dev.host(restr), restr_r)
    # L-BFGS over a few synthetic pairs
    M = 3
    dev.lbfgs_setup(M, restr)
    ref = O.LBFGSCoupled(n, M, restr_r)
    g_pre = [np.zeros(n), np.zeros(n)]
    m_pre = [np.zeros(n), np.zeros(n)]
    for it in range(1, 7):
        g = [rng.standard_normal(n) * restr_r for _ in range(2)]
        m = [m_pre[0] + 0.1 * rng.standard_normal(n), m_pre[1] + 0.1 * rng.standard_normal(n)]
        pl_r, pm_r = ref.direction(it, 1, g[0], g[1], g_pre[0], g_pre[1], m[0], m[1], m_pre[0], m_pre[1])
        PL, PM = dev.zeros(), dev.zeros()
        dev.lbfgs_direction(it, 1, *[dev.vec(v) for v in (g[0], g[1], g_pre[0], g_pre[1], m[0], m[1], m_pre[0], m_pre[1])],
                            PL, PM)
        assert rel_l2(dev.host(PL), pl_r) < 1e-11 and rel_l2(dev.host(PM), pm_r) < 1e-11, it
        g_pre, m_pre = g, m
    s.close()


@pytest.mark.parametrize("tv", ["TV", None])
def test_fwi_iterations_match_the_reference_rules(gpu_lib, tv):
    """The device driver (device forward, misfit, adjoint gradient, TV, gradient mass,
    L-BFGS and vector kernels, with hirensi_b200.inversion's control flow) against
    oracle.inversion_loop, the oracle's own restatement of S4/Program_Main.F90:379-896
    driven by the CPU forward, adjoint and control: per iteration the step sizes, the
    Armijo trials, the misfit and the model."""
    from fwi_oracle import loop_primitives
    p = tiny(nshot=2, nstep=160)
    _, _, hist_t = oracle_forward(p, p["lam_t"], p["mu_t"])
    dis = [traces_from_history(p, h) for h in hist_t]
    shots = []
    for k in range(2):
        b = np.zeros(p["mesh"].neq)
        b[p["src_eq"][k]] = 1.0
        shots.append((b, p["ftab"][k]))
    cfg = InversionConfig(m_lbfgs=5, bounds_lambda=(10.0, 1000.0), bounds_mu=(10.0, 1000.0), regularization=tv)
    be = OracleBackend(p["mesh"], shots, p["nstep"], p["dt"], p["eqdis"], p["eqdis_map"], dis)
    evaluate, gradient, tvf, img, restriction, extend_to = loop_primitives(be)
    ref = O.inversion_loop(evaluate, gradient, p["lam"], p["mu"], 3, img, restriction, extend_to, cfg.bounds_lambda,
                           cfg.bounds_mu, m_lbfgs=cfg.m_lbfgs,
                           fac_max_update=(cfg.fac_max_update_lambda, cfg.fac_max_update_mu),
                           tv=tvf if tv else None, reg_factor=cfg.reg_factor, bias_lambda=cfg.bias_lambda,
                           n_iter_bias=cfg.n_iter_bias, iter_begin=cfg.iter_begin)
    s = _device(p, dis)
    fwi = FWI(DeviceBackend(s, p["mesh"]), cfg)
    h_dev = fwi.run(p["lam"], p["mu"], n_iter=3)
    assert [h["armijo"] for h in h_dev] == [h["armijo"] for h in ref]
    for a, b in zip(h_dev, ref):
        assert abs(a["misfit"] - b["misfit"]) <= 1e-8 * b["misfit"]
        if b["iter"] > 0:
            assert abs(a["alpha_lambda"] - b["alpha_lambda"]) <= 1e-8 * abs(b["alpha_lambda"])
            assert abs(a["alpha_mu"] - b["alpha_mu"]) <= 1e-8 * abs(b["alpha_mu"])
    assert ref[-1]["misfit"] < ref[0]["misfit"]
    assert rel_l2(fwi.lam.cpu().numpy(), ref[-1]["lam"]) < 1e-9
    assert rel_l2(fwi.mu.cpu().numpy(), ref[-1]["mu"]) < 1e-9
    s.close()


def test_batched_backend_equals_one_batch(gpu_lib):
    """FWI over shots advanced in two batches (hirensi_b200.inversion.BatchedBackend) equals
    FWI with all shots in one batch: the misfit and the gradient are sums over shots, only
    the order of the gradient sum changes."""
    from hirensi_b200 import batching as B
    from hirensi_b200.inversion import BatchedBackend
    from hirensi_b200.solver import Solver
    p = tiny(nshot=4, nstep=120)
    _, _, hist_t = oracle_forward(p, p["lam_t"], p["mu_t"])
    dis = [traces_from_history(p, h) for h in hist_t]
    cfg = InversionConfig(m_lbfgs=5, bounds_lambda=(10.0, 1000.0), bounds_mu=(10.0, 1000.0), regularization=None)
    s = _device(p, dis)
    one = FWI(DeviceBackend(s, p["mesh"]), cfg)
    h1 = one.run(p["lam"], p["mu"], n_iter=3)
    lam1, mu1 = one.lam.cpu().numpy(), one.mu.cpu().numpy()
    s.close()
    shots = [B.Shot(np.array([p["src_eq"][k]], np.int32), np.ones(1), p["ftab"][k], p["eqdis"], dis[k]) for k in range(4)]
    batches = [B.pack(shots, ids) for ids in ([0, 1], [2, 3])]
    for b in batches:
        assert b.dis is not None and b.dis.shape[0] == 2
    sb = Solver("fp64")
    sb.set_mesh(p["mesh"], RHO)
    sb.assemble(p["lam"], p["mu"])
    sb.set_history(p["mesh"].store_eq)
    two = FWI(BatchedBackend(sb, p["mesh"], batches, p["dt"], p["mesh"].store_position), cfg)
    h2 = two.run(p["lam"], p["mu"], n_iter=3)
    assert [h["armijo"] for h in h1] == [h["armijo"] for h in h2]
    for a, b in zip(h1, h2):
        assert abs(a["misfit"] - b["misfit"]) <= 1e-10 * b["misfit"]
    assert h2[-1]["misfit"] < h2[0]["misfit"]
    assert rel_l2(two.lam.cpu().numpy(), lam1) < 1e-9 and rel_l2(two.mu.cpu().numpy(), mu1) < 1e-9
    sb.close()
