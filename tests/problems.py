"""Small seeded test problems shared by the oracle and GPU tests."""
from __future__ import annotations

import numpy as np

import oracle as O
from hirensi_b200.mesh import box_mesh, surface_grid

RHO = 2.0e-3


def layered(mesh, vs=(200.0, 300.0, 400.0), bounds=(-7.5, -15.0), anomaly=None):
    """Nodal lambda, mu for horizontal layers (nu = 1/3, lambda = 2 mu), optionally
    scaled by a Gaussian Vs anomaly (centre, radius, amplitude)."""
    z = mesh.xyz[:, 2]
    v = np.where(z >= bounds[0], vs[0], np.where(z >= bounds[1], vs[1], vs[2])).astype(np.float64)
    if anomaly is not None:
        c, r, amp = anomaly
        d2 = ((mesh.xyz - np.asarray(c)) ** 2).sum(axis=1)
        v = v * (1.0 + amp * np.exp(-d2 / (r * r)))
    mu = RHO * v * v
    return 2.0 * mu, mu


def tiny(nshot=1, nstep=300, nx=4, ny=4, nz=2, npml=1, h=2.5, fr=60.0, seed=0, anomaly=True):
    """Mesh, model, sources, receivers and an oracle system for a few hundred steps."""
    rng = np.random.default_rng(seed)
    mesh = box_mesh(nx, ny, nz, h, npml)
    lam, mu = layered(mesh, bounds=(-0.25 * nz * h, -0.6 * nz * h))
    lam_t, mu_t = layered(mesh, bounds=(-0.25 * nz * h, -0.6 * nz * h),
                          anomaly=((0.0, 0.0, -0.5 * nz * h), 0.6 * h, -0.3) if anomaly else None)
    half = 0.5 * nx * h
    step = 0.5 * h
    cand = [(x, y) for x in np.arange(-half + step, half, step) for y in np.arange(-half + step, half, step)]
    pick = rng.choice(len(cand), size=nshot, replace=False)
    src_nodes = [mesh.node_at(cand[i][0], cand[i][1], 0.0) for i in pick]
    src_eq = mesh.equations(src_nodes, comps=(2,))
    src_b = np.eye(nshot)   # shot s loads only its own equation
    dt = 1.0e-4
    ft1 = O.time_table(nstep, dt, 2, fr)
    ftab = np.stack([ft1] * nshot)
    rec_nodes = surface_grid(mesh, [-0.5 * half, 0.0, 0.5 * half])
    eqdis = mesh.equations(rec_nodes)
    eqdis_map = mesh.store_position(eqdis)
    return dict(mesh=mesh, lam=lam, mu=mu, lam_t=lam_t, mu_t=mu_t, src_eq=src_eq, src_b=src_b, ftab=ftab,
                nstep=nstep, dt=dt, eqdis=eqdis, eqdis_map=eqdis_map, nshot=nshot)


def oracle_forward(p, lam, mu, nthreads=1):
    om = O.OracleMesh(p["mesh"], RHO)
    S = O.OracleSystem.assemble(om, lam, mu)
    hist = []
    for s in range(p["nshot"]):
        b = np.zeros(p["mesh"].neq)
        for k, e in enumerate(p["src_eq"]):
            b[e] += p["src_b"][k, s]
        hist.append(S.forward(b, p["ftab"][s], p["nstep"], p["dt"], p["mesh"].store_eq, nthreads))
    return om, S, hist


def traces_from_history(p, hist):
    """Dis_meas layout [nrec3, nstep+1] from a history [nstep+1, nstore]."""
    return np.ascontiguousarray(hist[:, p["eqdis_map"]].T)


def rel_l2(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    den = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (den if den > 0 else 1.0))
