"""CUDA graphs of the time loops (hrn_set_graphs): a replayed call gives what the
same call gives launched directly, bit for bit (histories, traces, misfit and
gradient), except with the atomic matrix-free variants, whose sums run in varying
order."""
import numpy as np
import pytest

from problems import RHO, oracle_forward, rel_l2, tiny, traces_from_history

pytestmark = pytest.mark.gpu


def _solver(p, lam, mu, graphs, variant=41, ckpt=0, precision="fp64"):
    from hirensi_b200.solver import Solver
    s = Solver(precision)
    s.set_graphs(graphs)
    s.set_mesh(p["mesh"], RHO)
    s.assemble(lam, mu)
    s.set_history(p["mesh"].store_eq)
    s.set_shots(p["nstep"], p["dt"], p["src_eq"], p["src_b"], p["ftab"])
    s.set_receivers(p["eqdis"], p["eqdis_map"])
    if variant:
        s.set_variant(variant, variant)
    if ckpt:
        s.set_checkpointing(ckpt)
    return s


def _evaluate(s, dis, keep_p=False):
    s.forward()
    J = s.misfit(dis)
    gl, gm = s.adjoint_gradient(dis, keep_p=keep_p)
    return J, gl, gm, s.traces()


def _data(p):
    _, _, hist_t = oracle_forward(p, p["lam_t"], p["mu_t"])
    return np.stack([traces_from_history(p, h) for h in hist_t])


@pytest.mark.parametrize("variant,ckpt", [(41, 0), (45, 0), (41, 11), (92, 0), (0, 0)])
def test_replayed_calls_equal_direct_launches(gpu_lib, variant, ckpt):
    """variant 0: tuned on first use (that call runs directly), then captured; the
    direct reference runs the variants the tuner chose."""
    p = tiny(nshot=2, nstep=90)
    dis = _data(p)
    outs = []
    with _solver(p, p["lam"], p["mu"], True, variant, ckpt) as s1:
        for _ in range(3):   # (tune,) capture, then replays
            outs.append(_evaluate(s1, dis))
        vf, va = s1.variant()
    with _solver(p, p["lam"], p["mu"], False, 0, ckpt) as s0:
        s0.set_variant(vf, va)
        ref = _evaluate(s0, dis)
    # the atomic matrix-free variants (odd 91-105) add in varying order
    atomic = any(90 <= v <= 105 and v % 2 == 1 for v in (vf, va))
    for out in outs:
        if atomic:
            assert abs(out[0] - ref[0]) <= 1e-12 * ref[0]
            assert rel_l2(out[3], ref[3]) < 1e-12
            assert rel_l2(out[1], ref[1]) < 1e-12
            assert rel_l2(out[2], ref[2]) < 1e-12
        else:
            assert out[0] == ref[0]
            assert np.array_equal(out[3], ref[3])
            assert np.array_equal(out[1], ref[1])
            assert np.array_equal(out[2], ref[2])


def test_replay_follows_reassembly_and_new_data(gpu_lib):
    """Values change between replays (a new model, new data); the graph is kept.
    (Variant 92 and the CSR kernels sum in a fixed order; the atomic variants do not.)"""
    p = tiny(nshot=2, nstep=80)
    dis = _data(p)
    with _solver(p, p["lam"], p["mu"], True) as s:
        s.set_data(dis)
        _evaluate(s, None)
        _evaluate(s, None)   # the first adjoint allocates its gradient tables once
        n0 = s.launch_count()
        c0, r0 = s.graph_stats()
        s.assemble(p["lam_t"], p["mu_t"])
        s.set_data(0.5 * dis)
        got = _evaluate(s, None, keep_p=False)
        assert s.launch_count() > n0
        # no new capture: both loops replayed
        assert s.graph_stats() == (c0, r0 + 2)
    with _solver(p, p["lam_t"], p["mu_t"], False) as s0:
        ref = _evaluate(s0, 0.5 * dis)
    assert got[0] == ref[0]
    assert np.array_equal(got[3], ref[3])
    assert np.array_equal(got[1], ref[1])


def test_new_settings_capture_again(gpu_lib):
    p = tiny(nshot=2, nstep=60)
    q = tiny(nshot=2, nstep=110)
    with _solver(p, p["lam"], p["mu"], True) as s:
        s.forward()
        s.set_shots(q["nstep"], q["dt"], q["src_eq"], q["src_b"], q["ftab"])
        s.forward()
        h = [s.history(k) for k in range(2)]
        s.set_timing(True)            # timing runs the launches directly
        s.forward()
        ht = [s.history(k) for k in range(2)]
    with _solver(q, q["lam"], q["mu"], False) as s0:
        s0.forward()
        ref = [s0.history(k) for k in range(2)]
    for k in range(2):
        assert np.array_equal(h[k], ref[k])
        assert np.array_equal(ht[k], ref[k])


def test_graphs_with_uneven_shots_and_fp32(gpu_lib):
    p = tiny(nshot=3, nstep=100)
    dis = _data(p)
    lens = [100, 55, 80]
    mask = np.ones((3, len(p["eqdis"])), np.uint8)
    mask[1, ::2] = 0
    out = []
    for graphs in (False, True):
        with _solver(p, p["lam"], p["mu"], graphs, 41, 13, "fp32") as s:
            s.set_shot_records(lens, mask)
            for _ in range(2):
                r = _evaluate(s, dis)
            out.append(r)
    assert out[0][0] == out[1][0]
    assert np.array_equal(out[0][3], out[1][3])
    assert rel_l2(out[1][1], out[0][1]) < 1e-6
