"""Shot-parallel FWI on two gloo ranks (CPU, oracle backend) against the same
inversion in one process: the all-reduced misfit and gradient, and the replicated
L-BFGS update, must give every rank the single-process model."""
import os
import socket
import tempfile

import numpy as np
import pytest

from hirensi_b200.distributed import shard


def test_shard_covers_items_once_and_balances():
    for n in range(0, 12):
        for world in range(1, 5):
            blocks = [shard(n, world, r) for r in range(world)]
            flat = [i for b in blocks for i in b]
            assert flat == list(range(n))
            sizes = [len(b) for b in blocks]
            assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        shard(4, 2, 2)


def _problem(nshot=4, nstep=80):
    from problems import oracle_forward, tiny, traces_from_history
    p = tiny(nshot=nshot, nstep=nstep, seed=2)
    _, _, hist_t = oracle_forward(p, p["lam_t"], p["mu_t"])
    dis = [traces_from_history(p, h) for h in hist_t]
    shots = []
    for k in range(nshot):
        b = np.zeros(p["mesh"].neq)
        b[p["src_eq"][k]] = 1.0
        shots.append((b, p["ftab"][k]))
    return p, shots, dis


def _run_fwi(backend, p, n_iter):
    from hirensi_b200.inversion import FWI, InversionConfig
    cfg = InversionConfig(m_lbfgs=3, bounds_lambda=(10.0, 1000.0), bounds_mu=(10.0, 1000.0))
    fwi = FWI(backend, cfg)
    hist = fwi.run(p["lam"], p["mu"], n_iter=n_iter)
    return np.asarray(fwi.lam), np.asarray(fwi.mu), [h["misfit"] for h in hist]


def _rank_main(rank, world, port, out_dir, n_iter):
    import torch.distributed as dist
    from fwi_oracle import OracleBackend
    from hirensi_b200.distributed import ShotParallelBackend, shard as shard_
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    try:
        p, shots, dis = _problem()
        mine = shard_(len(shots), world, rank)
        local = OracleBackend(p["mesh"], [shots[k] for k in mine], p["nstep"], p["dt"], p["eqdis"], p["eqdis_map"],
                              [dis[k] for k in mine])
        lam, mu, misfits = _run_fwi(ShotParallelBackend(local), p, n_iter)
        np.savez(os.path.join(out_dir, f"rank{rank}.npz"), lam=lam, mu=mu, misfit=np.array(misfits))
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_rank_shot_parallel_fwi_matches_one_process():
    import torch.multiprocessing as mp
    from fwi_oracle import OracleBackend
    n_iter = 2
    with tempfile.TemporaryDirectory() as out:
        mp.start_processes(_rank_main, args=(2, _free_port(), out, n_iter), nprocs=2, join=True, start_method="spawn")
        r0 = np.load(os.path.join(out, "rank0.npz"))
        r1 = np.load(os.path.join(out, "rank1.npz"))
    # replicated update: both ranks hold the same model
    assert np.array_equal(r0["lam"], r1["lam"]) and np.array_equal(r0["mu"], r1["mu"])
    p, shots, dis = _problem()
    ref = OracleBackend(p["mesh"], shots, p["nstep"], p["dt"], p["eqdis"], p["eqdis_map"], dis)
    lam, mu, misfits = _run_fwi(ref, p, n_iter)
    # sums over shots differ from the one-process order only in rounding
    assert np.allclose(r0["misfit"], misfits, rtol=1e-12, atol=0.0)
    assert np.linalg.norm(r0["lam"] - lam) <= 1e-10 * np.linalg.norm(lam)
    assert np.linalg.norm(r0["mu"] - mu) <= 1e-10 * np.linalg.norm(mu)
    assert misfits[-1] < misfits[0]
