"""Shots of uneven record length and receiver count in one batch (hrn_set_shot_records).

Each shot of the batch must give what the same shot gives solved alone with its
own NSTEP and receiver list, as the reference solves it: the batch misfit is the
sum of the shots' misfits and the batch gradient the sum of their gradients
(FP64 bar 1e-10 against the oracle; 1e-12 against single-shot GPU runs, whose
gradients are added over the shots in another order)."""
import numpy as np
import pytest

import oracle as O
from problems import RHO, oracle_forward, rel_l2, tiny, traces_from_history

pytestmark = pytest.mark.gpu

LENS = [120, 70, 95]


def _masks(p):
    nrec = len(p["eqdis"]) // 3
    node_mask = np.zeros((3, nrec), bool)
    node_mask[0] = True                       # every receiver
    node_mask[1, : nrec // 2] = True          # the first half
    node_mask[2, ::2] = True                  # every other one
    return np.repeat(node_mask, 3, axis=1)    # x, y, z of each receiver node


def _data(p):
    """Measured data of the true model, [nshot, nrec3, nstep + 1]."""
    _, _, hist_t = oracle_forward(p, p["lam_t"], p["mu_t"])
    return np.stack([traces_from_history(p, h) for h in hist_t])


def _batch(p, dis, mask, precision="fp64", variant=41, ckpt=0):
    from hirensi_b200.solver import Solver
    with Solver(precision) as s:
        s.set_mesh(p["mesh"], RHO)
        s.assemble(p["lam"], p["mu"])
        s.set_history(p["mesh"].store_eq)
        s.set_shots(p["nstep"], p["dt"], p["src_eq"], p["src_b"], p["ftab"])
        s.set_receivers(p["eqdis"], p["eqdis_map"])
        s.set_shot_records(LENS, mask)
        s.set_variant(variant, variant)
        if ckpt:
            s.set_checkpointing(ckpt)
        s.forward()
        J = s.misfit(dis)
        gl, gm = s.adjoint_gradient(dis)
        tr = s.traces()
    return J, gl, gm, tr


def _single(p, dis, mask, k, variant=41):
    from hirensi_b200.solver import Solver
    n = LENS[k]
    m = mask[k]
    with Solver("fp64") as s:
        s.set_mesh(p["mesh"], RHO)
        s.assemble(p["lam"], p["mu"])
        s.set_history(p["mesh"].store_eq)
        s.set_shots(n, p["dt"], p["src_eq"], p["src_b"][:, k:k + 1], p["ftab"][k:k + 1, : n + 1])
        s.set_receivers(p["eqdis"][m], p["eqdis_map"][m])
        s.set_variant(variant, variant)
        s.forward()
        d = np.ascontiguousarray(dis[k][m][:, : n + 1])[None]
        J = s.misfit(d)
        gl, gm = s.adjoint_gradient(d)
        tr = s.traces()
    return J, gl, gm, tr


def test_uneven_batch_equals_shots_solved_alone(gpu_lib):
    p = tiny(nshot=3, nstep=max(LENS))
    dis = _data(p)
    mask = _masks(p)
    J, gl, gm, tr = _batch(p, dis, mask)
    Js, gls, gms = 0.0, 0.0, 0.0
    for k in range(3):
        j1, gl1, gm1, tr1 = _single(p, dis, mask, k)
        Js, gls, gms = Js + j1, gls + gl1, gms + gm1
        # the shot's traces up to its own length, at its own receivers
        assert np.array_equal(tr[k][mask[k]][:, : LENS[k] + 1], tr1[0])
    assert J > 0
    assert abs(J - Js) <= 1e-12 * Js
    assert rel_l2(gl, gls) < 1e-12
    assert rel_l2(gm, gms) < 1e-12


def test_uneven_batch_matches_oracle(gpu_lib):
    p = tiny(nshot=3, nstep=max(LENS))
    dis = _data(p)
    mask = _masks(p)
    J, gl, gm, _ = _batch(p, dis, mask)
    om = O.OracleMesh(p["mesh"], RHO)
    S = O.OracleSystem.assemble(om, p["lam"], p["mu"])
    se = p["mesh"].store_eq
    Jr, glr, gmr = 0.0, 0.0, 0.0
    for k in range(3):
        n, m = LENS[k], mask[k]
        b = np.zeros(p["mesh"].neq)
        for i, e in enumerate(p["src_eq"]):
            b[e] += p["src_b"][i, k]
        u = S.forward(b, p["ftab"][k][: n + 1], n, p["dt"], se)
        d = np.ascontiguousarray(dis[k][m][:, : n + 1])
        Jr += O.misfit(n, p["dt"], p["eqdis"][m], p["eqdis_map"][m], u, d)
        pk = S.adjoint(n, p["dt"], se, u, p["eqdis"][m], p["eqdis_map"][m], d)
        a, c = O.control(om, n, p["dt"], se, u, pk)
        glr, gmr = glr + a, gmr + c
    assert abs(J - Jr) <= 1e-10 * Jr
    assert rel_l2(gl, glr) < 1e-10
    assert rel_l2(gm, gmr) < 1e-10


@pytest.mark.parametrize("variant,ckpt", [(41, 17), (45, 9)])
def test_uneven_batch_with_checkpointing(gpu_lib, variant, ckpt):
    p = tiny(nshot=3, nstep=max(LENS))
    dis = _data(p)
    mask = _masks(p)
    J0, gl0, gm0, _ = _batch(p, dis, mask, variant=variant)
    J1, gl1, gm1, _ = _batch(p, dis, mask, variant=variant, ckpt=ckpt)
    assert J1 == J0
    assert np.array_equal(gl1, gl0)
    assert np.array_equal(gm1, gm0)


def test_uneven_fp32_within_bars(gpu_lib):
    p = tiny(nshot=3, nstep=max(LENS))
    dis = _data(p)
    mask = _masks(p)
    J64, gl64, gm64, _ = _batch(p, dis, mask)
    J32, gl32, gm32, _ = _batch(p, dis, mask, precision="fp32")
    assert abs(J32 - J64) <= 1e-3 * J64
    assert rel_l2(gl32, gl64) < 1e-3
    assert rel_l2(gm32, gm64) < 1e-3


def test_shot_records_are_checked(gpu_lib):
    from hirensi_b200.capi import HrnError
    from hirensi_b200.solver import Solver
    p = tiny(nshot=2, nstep=50)
    with Solver("fp64") as s:
        s.set_mesh(p["mesh"], RHO)
        s.assemble(p["lam"], p["mu"])
        s.set_history(p["mesh"].store_eq)
        s.set_shots(p["nstep"], p["dt"], p["src_eq"], p["src_b"], p["ftab"])
        s.set_receivers(p["eqdis"], p["eqdis_map"])
        with pytest.raises(HrnError):
            s.set_shot_records([50, 51])
        with pytest.raises(HrnError):
            s.set_shot_records([0, 50])
        with pytest.raises(ValueError):
            s.set_shot_records(None, np.ones((3, len(p["eqdis"]))))
        s.set_shot_records([50, 20], None)


def test_planned_batches_equal_single_shots(gpu_lib):
    """Four shots of different lengths and receiver sets, planned into batches of at
    most three by hirensi_b200.batching, give each shot's own traces and misfit."""
    from hirensi_b200 import batching as B
    from hirensi_b200.solver import Solver
    lens = [120, 60, 95, 80]
    p = tiny(nshot=4, nstep=max(lens))
    dis = _data(p)
    nrec = len(p["eqdis"]) // 3
    keep = [np.arange(nrec), np.arange(0, nrec, 2), np.arange(nrec // 2, nrec), np.arange(1, nrec, 3)]
    shots = []
    for k in range(4):
        q = (3 * keep[k][:, None] + np.arange(3)).reshape(-1)
        shots.append(B.Shot(p["src_eq"][k:k + 1], np.ones(1), p["ftab"][k][: lens[k] + 1], p["eqdis"][q],
                            np.ascontiguousarray(dis[k][q][:, : lens[k] + 1])))
    batches = B.plan(lens, max_shots=3)
    assert batches == [[0, 2, 3], [1]]
    traces, J = {}, 0.0
    for ids in batches:
        b = B.pack(shots, ids)
        with Solver("fp64") as s:
            s.set_mesh(p["mesh"], RHO)
            s.assemble(p["lam"], p["mu"])
            s.set_history(p["mesh"].store_eq)
            B.configure(s, b, p["dt"], p["mesh"].store_position)
            s.set_variant(41, 41)
            s.forward()
            J += s.misfit(b.dis)
            for i, t in zip(ids, B.unpack_traces(b, s.traces())):
                traces[i] = t
    J1 = 0.0
    for k in range(4):
        sh = shots[k]
        with Solver("fp64") as s:
            s.set_mesh(p["mesh"], RHO)
            s.assemble(p["lam"], p["mu"])
            s.set_history(p["mesh"].store_eq)
            s.set_shots(sh.nstep, p["dt"], sh.src_eq, sh.src_b[:, None], sh.ftab[None])
            s.set_receivers(sh.eqdis, p["mesh"].store_position(sh.eqdis))
            s.set_variant(41, 41)
            s.forward()
            J1 += s.misfit(sh.dis[None])
            assert np.array_equal(traces[k], s.traces()[0])
    assert abs(J - J1) <= 1e-12 * J1
