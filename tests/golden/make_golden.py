"""Writes tests/golden/tiny_inversion.npz: outputs of the oracle (the C restatement of
the reference's forward, adjoint, control and misfit) on a small seeded problem,
committed so that the parity tests check the CUDA path against fixed vectors and the
oracle against regressions.  No reference outputs exist to pin against (the reference
needs Fortran, PETSc and MPI); these fixtures are the oracle's.

Problem: tests/problems.py tiny(nshot=2, nstep=200, seed=0) -- 4 x 4 x 2 27-node
elements with a 1-element PML, two vertical Ricker sources, 3 x 3 surface receivers.

Contents:
* dis [2, nrec3, nstep+1]: traces of the true model (the measured data);
* traces0 [2, nrec3, nstep+1]: traces of the initial model;
* misfit: sum over shots of Compute_Misfit at the initial model;
* g_lambda, g_mu [nj]: the accumulated control-problem gradient (before the sign flip
  and the gradient mass), summed over shots;
* fd_nodes, fd_mu, fd_lambda, adj_mu, adj_lambda: the finite-difference check of
  S4/Gradient_check.F90 (relative step 1e-4 of one nodal mu or lambda) at 6 regular-domain
  nodes, with the sign-flipped adjoint gradient there;
* ID, store_eq: the integer inputs (equation numbers, U_Store equations).

Run from the repository root: python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
for p in (ROOT, os.path.join(ROOT, "oracle"), os.path.join(ROOT, "tests")):
    if p not in sys.path:
        sys.path.insert(0, p)

import oracle as O  # noqa: E402
from problems import RHO, oracle_forward, tiny, traces_from_history  # noqa: E402

OUT = os.path.join(HERE, "tiny_inversion.npz")


def compute():
    p = tiny(nshot=2, nstep=200, seed=0)
    m = p["mesh"]
    _, _, ht = oracle_forward(p, p["lam_t"], p["mu_t"])
    dis = np.stack([traces_from_history(p, h) for h in ht])
    om, S, h0 = oracle_forward(p, p["lam"], p["mu"])
    traces0 = np.stack([traces_from_history(p, h) for h in h0])
    J, gl, gm = 0.0, 0.0, 0.0
    for k in range(2):
        J += O.misfit(p["nstep"], p["dt"], p["eqdis"], p["eqdis_map"], h0[k], dis[k])
        pk = S.adjoint(p["nstep"], p["dt"], m.store_eq, h0[k], p["eqdis"], p["eqdis_map"], dis[k])
        a, b = O.control(om, p["nstep"], p["dt"], m.store_eq, h0[k], pk)
        gl, gm = gl + a, gm + b

    def misfit(lam, mu):
        _, _, h = oracle_forward(p, lam, mu)
        return sum(O.misfit(p["nstep"], p["dt"], p["eqdis"], p["eqdis_map"], h[k], dis[k]) for k in range(2))

    rd = np.nonzero(m.node_mat_id == 0)[0]
    nodes = np.random.default_rng(0).choice(rd, 6, replace=False)
    eps = 1.0e-4
    fd_mu, fd_lam = [], []
    for k in nodes:
        for name, out in (("mu", fd_mu), ("lam", fd_lam)):
            lam, mu = p["lam"].copy(), p["mu"].copy()
            arr = mu if name == "mu" else lam
            base = arr[k]
            arr[k] = base * (1.0 + eps)
            out.append((misfit(lam, mu) - J) / (base * eps))
    return dict(dis=dis, traces0=traces0, misfit=np.float64(J), g_lambda=gl, g_mu=gm,
                fd_nodes=nodes.astype(np.int32), fd_mu=np.array(fd_mu), fd_lambda=np.array(fd_lam),
                adj_mu=-gm[nodes], adj_lambda=-gl[nodes],
                ID=np.asarray(m.ID, dtype=np.int32), store_eq=np.asarray(m.store_eq, dtype=np.int32))


if __name__ == "__main__":
    np.savez_compressed(OUT, **compute())
    print(OUT, os.path.getsize(OUT), "bytes")
