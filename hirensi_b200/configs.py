"""Seeded synthetic workloads of the benchmark configurations.

No public dataset is involved: meshes, models, sources and receivers are
generated here.  Units follow the reference (stresses and moduli in 1e-6 units,
rho = 2e-3 for 2000 kg/m^3, S4/Adjustments.F90:20-27), so Vs = sqrt(mu / rho).
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np

from .mesh import Mesh, box_mesh, surface_grid

RHO = 2.0e-3


def time_function(t: float, lcase: int = 2, fr: float = 15.0) -> float:
    """TIME_FUNCTION (S4/IO.F90:541-728): 2 = Ricker pulse of central frequency fr
    (zero after 6 sqrt(6) / (2 pi fr)), 3 = the active Gaussian pulse (mean 0.06,
    variance parameter 0.0004), 8 = constant 1."""
    pi = 3.14159265358979323846264338327950288419716939937510
    if lcase == 2:
        wr = 2.0 * pi * fr
        t_max = 6.0 * math.sqrt(6.0) / wr
        u = wr * t - 3.0 * math.sqrt(6.0)
        if t < t_max:
            f1 = (0.25 * (u * u) - 0.5) * math.exp(-0.25 * (u * u)) - 13.0 * math.exp(-13.5)
            f2 = 0.50 + 13.0 * math.exp(-13.5)
            return f1 / f2
        return 0.0
    if lcase == 3:
        return math.exp(-(t - 0.06) * (t - 0.06) / 0.00040)
    if lcase == 8:
        return 1.0
    raise ValueError(f"unsupported time function case {lcase}")


def time_table(nstep: int, dt: float, lcase: int = 2, fr: float = 15.0) -> np.ndarray:
    """[nstep+1, 3]: the function at T, T+dt, T+dt/2 for T = ISTEP*dt
    (the three calls of S4/Solver_PETSc_Explicit.F90:983-995)."""
    tab = np.zeros((nstep + 1, 3))
    for i in range(nstep + 1):
        T = float(i) * dt
        tab[i] = (time_function(T, lcase, fr), time_function(T + dt, lcase, fr), time_function(T + 0.5 * dt, lcase, fr))
    return tab


def vs_to_lame(vs: np.ndarray, nu: float = 1.0 / 3.0, rho: float = RHO):
    """Nodal (lambda, mu) for a shear-wave speed and a Poisson ratio."""
    mu = rho * vs * vs
    lam = 2.0 * mu * nu / (1.0 - 2.0 * nu)
    return lam, mu


def layered_vs(mesh: Mesh, vs=(200.0, 300.0, 400.0), bounds=(-7.5, -15.0)) -> np.ndarray:
    """Horizontal layers; a node on an interface belongs to the upper layer."""
    z = mesh.xyz[:, 2]
    return np.where(z >= bounds[0], vs[0], np.where(z >= bounds[1], vs[1], vs[2])).astype(np.float64)


def extend_into_pml(mesh: Mesh, field: np.ndarray) -> np.ndarray:
    """Copy interface values into the PML along the material extension map."""
    return field[mesh.extend_to]


@dataclasses.dataclass
class Problem:
    name: str
    mesh: Mesh
    lam_true: np.ndarray
    mu_true: np.ndarray
    lam0: np.ndarray
    mu0: np.ndarray
    nstep: int
    dt: float
    src_eq: np.ndarray        # [nshot] vertical-force equations
    src_b: np.ndarray         # [nshot, nshot] unit load of shot s at its own equation
    ftab: np.ndarray          # [nshot, nstep+1, 3]
    eqdis: np.ndarray         # [nrec3]
    eqdis_map: np.ndarray     # [nrec3]

    @property
    def nshot(self) -> int:
        return int(self.src_eq.size)

    @property
    def dof(self) -> int:
        """The configuration's DOF: displacement DOF of the regular domain."""
        return self.mesh.rd_dof


def inversion_config(nstep: int = 2000, dt: float = 1.0e-4, fr: float = 15.0, nx: int = 16, ny: int = 16,
                     nz: int = 8, h: float = 2.5, npml: int = 3,
                     shots=((-10.0, -10.0), (10.0, -10.0), (-10.0, 10.0), (10.0, 10.0)),
                     receivers=(-15.0, -7.5, 0.0, 7.5, 15.0)) -> Problem:
    """The plain inversion workload: 40 x 40 x 20 m half-space of 16 x 16 x 8
    27-node hexahedra (2.5 m) with a 3-element PML on the sides and the bottom;
    true model = 3 layers (Vs 200/300/400, nu = 1/3, rho 2000) with a Gaussian
    Vs anomaly of -30 % (radius 5 m, depth 8 m); initial model = linear Vs
    200 -> 400 m/s over the 20 m depth; vertical Ricker point forces (15 Hz) at
    the surface, 5 x 5 surface receivers, dt = 1e-4 s, 2000 steps."""
    mesh = box_mesh(nx, ny, nz, h, npml)
    depth = nz * h
    vs_t = layered_vs(mesh)
    d2 = ((mesh.xyz - np.array([0.0, 0.0, -8.0])) ** 2).sum(axis=1)
    vs_t = vs_t * (1.0 - 0.3 * np.exp(-d2 / 25.0))
    vs_t = extend_into_pml(mesh, vs_t)
    z = np.clip(mesh.xyz[:, 2], -depth, 0.0)
    vs_0 = extend_into_pml(mesh, 200.0 + 200.0 * (-z / depth))
    lam_t, mu_t = vs_to_lame(vs_t)
    lam0, mu0 = vs_to_lame(vs_0)
    src_nodes = [mesh.node_at(x, y, 0.0) for x, y in shots]
    src_eq = mesh.equations(src_nodes, comps=(2,))
    ft = time_table(nstep, dt, 2, fr)
    rec = surface_grid(mesh, list(receivers))
    eqdis = mesh.equations(rec)
    return Problem(f"inversion_{nx}x{ny}x{nz}_pml{npml}", mesh, lam_t, mu_t, lam0, mu0, nstep, dt, src_eq,
                   np.eye(len(src_eq)), np.stack([ft] * len(src_eq)), eqdis, mesh.store_position(eqdis))


def training_config(nstep: int = 2000) -> Problem:
    """The learned preconditioner's training-mesh workload: the inversion
    configuration's model distribution on 40 x 40 x 20 hexahedra (100 x 100 x 50 m)
    plus a 3-element PML (2.08 M equations), 8 vertical Ricker forces on a 3 x 3
    surface grid without its centre (25 m apart), 7 x 7 surface receivers 12.5 m
    apart; 15 Hz, dt = 1e-4 s."""
    g = (-25.0, 0.0, 25.0)
    shots = tuple((x, y) for y in g for x in g if (x, y) != (0.0, 0.0))
    return inversion_config(nstep=nstep, nx=40, ny=40, nz=20, shots=shots,
                            receivers=(-37.5, -25.0, -12.5, 0.0, 12.5, 25.0, 37.5))


def forward_config(nstep: int = 2000) -> Problem:
    """The forward-only workload: same mesh, layered model, one vertical Ricker
    force at the surface centre."""
    p = inversion_config(nstep=nstep, shots=((0.0, 0.0),))
    lam, mu = vs_to_lame(extend_into_pml(p.mesh, layered_vs(p.mesh)))
    p.lam_true, p.mu_true, p.lam0, p.mu0 = lam, mu, lam, mu
    p.name = "forward_16x16x8_pml3"
    return p


@dataclasses.dataclass
class UnevenProblem:
    """Batched uneven shots on a large mesh: nodal lambda, mu, element density and
    one ``batching.Shot`` per source (no data)."""
    name: str
    mesh: Mesh
    lam: np.ndarray
    mu: np.ndarray
    rho_el: np.ndarray
    dt: float
    shots: list
    freqs: np.ndarray

    @property
    def dof(self) -> int:
        return self.mesh.rd_dof


def uneven_config(seed: int = 0, nx: int = 80, ny: int = 80, nz: int = 40, h: float = 2.5, npml: int = 4,
                  nshot: int = 64, dt: float = 1.0e-4, lengths=(1500, 4000), receivers=(100, 900),
                  length_scale: float = 1.0) -> UnevenProblem:
    """The batched uneven-shot workload: nx x ny x nz 27-node hexahedra (h) plus an
    npml-element PML; a seeded model of 3-6 horizontal layers (Vs 150-600 m/s,
    Poisson ratio 0.25-0.40, density 1800-2200 kg/m^3) with 1-3 ellipsoidal Vs
    inclusions of +-20-40 %; nshot vertical Ricker forces at random surface nodes
    (5-25 Hz), each with its own record length and 100-900 random surface receivers.
    length_scale < 1 shortens every record (a bounded sample of the workload)."""
    from .batching import Shot
    rng = np.random.default_rng(seed)
    mesh = box_mesh(nx, ny, nz, h, npml)
    depth = nz * h
    nlay = int(rng.integers(3, 7))
    tops = np.sort(rng.uniform(0.05, 0.9, nlay - 1) * depth)          # interface depths, ascending
    vs_l = np.sort(rng.uniform(150.0, 600.0, nlay))                    # stiffer with depth
    nu_l = rng.uniform(0.25, 0.40, nlay)
    rho_l = rng.uniform(1800.0, 2200.0, nlay) * 1.0e-6

    def layer_of(z):
        """Layer index of a point: the number of interfaces above it."""
        return (-np.asarray(z)[..., None] > tops[None, :]).sum(-1)

    lay = layer_of(mesh.xyz[:, 2])
    vs = vs_l[lay].copy()
    (x0, x1), (y0, y1), (z0, _) = mesh.rd_box
    for _ in range(int(rng.integers(1, 4))):
        c = np.array([rng.uniform(x0, x1), rng.uniform(y0, y1), rng.uniform(z0 * 0.8, z0 * 0.1)])
        ax = rng.uniform(0.05, 0.2, 3) * np.array([x1 - x0, y1 - y0, -z0])
        amp = rng.uniform(0.2, 0.4) * rng.choice([-1.0, 1.0])
        r2 = (((mesh.xyz - c) / ax) ** 2).sum(axis=1)
        vs = np.where(r2 <= 1.0, vs * (1.0 + amp), vs)
    vs = extend_into_pml(mesh, vs)
    lay = extend_into_pml(mesh, lay)
    nu = nu_l[lay]
    mu = rho_l[lay] * vs * vs
    lam = 2.0 * mu * nu / (1.0 - 2.0 * nu)
    cz = mesh.xyz[mesh.inod, 2].mean(axis=1)
    rho_el = rho_l[np.clip(layer_of(np.minimum(cz, 0.0)), 0, nlay - 1)]
    # surface nodes of the regular domain
    sx, sy, sz = mesh.xyz[:, 0], mesh.xyz[:, 1], mesh.xyz[:, 2]
    surf = np.nonzero((np.abs(sz) < 1e-9) & (sx >= x0 - 1e-9) & (sx <= x1 + 1e-9) & (sy >= y0 - 1e-9) & (sy <= y1 + 1e-9))[0]
    shots = []
    freqs = rng.uniform(5.0, 25.0, nshot)
    for k in range(nshot):
        n = int(rng.integers(lengths[0], lengths[1] + 1))
        n = max(2, int(round(n * length_scale)))
        src = int(rng.choice(surf))
        nrec = int(rng.integers(receivers[0], receivers[1] + 1))
        rec = np.sort(rng.choice(surf, size=nrec, replace=False))
        shots.append(Shot(mesh.equations([src], comps=(2,)), np.ones(1), time_table(n, dt, 2, float(freqs[k])),
                          mesh.equations(rec)))
    return UnevenProblem(f"uneven_{nx}x{ny}x{nz}_pml{npml}_{nshot}shots", mesh, lam, mu, rho_el, dt, shots, freqs)
