"""Structured 27-node hexahedral meshes with a PML on the four sides and the bottom.

Produces the integer and geometric inputs the HiReNSI solver consumes, following
the reference's conventions:

* element-local node order of ``SHAPE_3_27`` (S4/Shape_Functions.F90:124-274):
  8 corners, 12 edge mid-nodes (9-20), 6 face centres (21-26), centre (27);
* ``MTEL`` = 1 for regular-domain (RD) elements, 2 for PML elements;
* constraint rules of the 20->27 converter (S2/Main.F90:448-520): nodes of RD
  elements carry the 3 displacement DOFs only, nodes of PML elements (the RD/PML
  interface included) carry all 9, and the displacement DOFs of the outer box
  faces (x min/max, y min/max, z min) are fixed;
* equation numbering of the partitioner at one part (S3/PIC_ReNumbering.F90:
  244-283): node order, DOF order 1..9, free DOFs only, 0-based here;
* stored history equations ``U_Store_Numbers_Global``: the three displacement
  equations of every RD or interface node, in node order
  (S3/PIC_Inversion_Data_Structure.F90:255-300);
* ``PML_PARAM(6,4)`` = [alpha0, beta0, L, x0] for x+, x-, y+, y-, z+, z-
  (S4/Adjustments.F90:62-77).

Nodes are numbered lexicographically (x fastest, then y, then z), which keeps
the bandwidth of the assembled operators small.
"""
from __future__ import annotations

import dataclasses

import numpy as np

# (xi, eta, zeta) index in {0,1,2} (GLL points -1, 0, +1) of each local node of
# SHAPE_3_27, found by where each shape function equals one.
LOCAL_IJK = np.array([
    (2, 0, 0), (2, 2, 0), (0, 2, 0), (0, 0, 0), (2, 0, 2), (2, 2, 2), (0, 2, 2), (0, 0, 2),
    (2, 1, 0), (1, 2, 0), (0, 1, 0), (1, 0, 0), (2, 0, 1), (2, 2, 1), (0, 2, 1), (0, 0, 1),
    (2, 1, 2), (1, 2, 2), (0, 1, 2), (1, 0, 2), (1, 1, 0), (2, 1, 1), (1, 2, 1), (0, 1, 1),
    (1, 0, 1), (1, 1, 2), (1, 1, 1)], dtype=np.int64)

# local node index at GLL point q, with q = 9*c + 3*b + a (the reference's
# LZ/LY/LX quadrature loop order: x fastest)
GLL_TO_LOCAL = np.empty(27, dtype=np.int64)
for _i, (_a, _b, _c) in enumerate(LOCAL_IJK):
    GLL_TO_LOCAL[9 * _c + 3 * _b + _a] = _i
del _i, _a, _b, _c


@dataclasses.dataclass
class Mesh:
    nx: int
    ny: int
    nz: int
    npml: int
    h: float
    xyz: np.ndarray          # [nj, 3] float64
    inod: np.ndarray         # [nel, 27] int32, 0-based
    mtel: np.ndarray         # [nel] int32 (1 RD, 2 PML)
    eid: np.ndarray          # [nel, 3] int32 element lattice index
    ID: np.ndarray           # [nj, 9] int32 0-based equation numbers, -1 = constrained
    neq: int
    node_mat_id: np.ndarray  # [nj] int8: 0 RD only, 1 interface, 2 PML only
    store_nodes: np.ndarray  # [nstore/3] int32 node ids stored for the gradient
    store_eq: np.ndarray     # [nstore] int32 equations (node-major, x y z)
    extend_to: np.ndarray    # [nj] int32: node whose material a node takes (itself for RD/interface)
    pml_param: np.ndarray    # [6, 4] float64
    rd_box: tuple            # ((xmin, xmax), (ymin, ymax), (zmin, zmax)) of the regular domain
    lattice: tuple           # (NX, NY, NZ) node counts per axis

    @property
    def nj(self) -> int:
        return self.xyz.shape[0]

    @property
    def nel(self) -> int:
        return self.inod.shape[0]

    @property
    def nstore(self) -> int:
        return int(self.store_eq.shape[0])

    @property
    def rd_dof(self) -> int:
        """Displacement DOF of the regular domain (RD + interface nodes)."""
        return self.nstore

    def node_index(self, i: int, j: int, k: int) -> int:
        NX, NY, _ = self.lattice
        return int(i + NX * (j + NY * k))

    def node_at(self, x: float, y: float, z: float) -> int:
        """Node id at a coordinate that lies on the node lattice."""
        NX, NY, NZ = self.lattice
        x0, y0, z0 = self.xyz[0]
        s = 0.5 * self.h
        i, j, k = (round((x - x0) / s), round((y - y0) / s), round((z - z0) / s))
        if not (0 <= i < NX and 0 <= j < NY and 0 <= k < NZ):
            raise ValueError(f"point ({x}, {y}, {z}) is outside the mesh")
        n = self.node_index(i, j, k)
        if np.max(np.abs(self.xyz[n] - (x, y, z))) > 1e-9 * max(1.0, self.h):
            raise ValueError(f"point ({x}, {y}, {z}) is not a mesh node")
        return n

    def equations(self, nodes, comps=(0, 1, 2)) -> np.ndarray:
        """Equation numbers of ``nodes`` x ``comps`` in node-major order."""
        nodes = np.asarray(nodes, dtype=np.int64)
        eq = self.ID[nodes][:, list(comps)].reshape(-1)
        if np.any(eq < 0):
            raise ValueError("requested a constrained degree of freedom")
        return eq.astype(np.int32)

    def store_position(self, eqs) -> np.ndarray:
        """Map equations to their index in ``store_eq`` (EqDis_MAP_U_Store_Numbers_Global)."""
        inv = np.full(self.neq, -1, dtype=np.int64)
        inv[self.store_eq] = np.arange(self.nstore)
        pos = inv[np.asarray(eqs, dtype=np.int64)]
        if np.any(pos < 0):
            raise ValueError("equation is not a stored history equation")
        return pos.astype(np.int32)


def default_pml_param(rd_box, thickness, alpha0=5.0, beta0=400.0) -> np.ndarray:
    """PML_PARAM with the reference defaults alpha0 = 5, beta0 = 400 (S4/Adjustments.F90:76-77).

    The top face is traction free: its start coordinate is placed above the
    mesh so the top zone of PML_FINDER_3D is never entered.
    """
    (x0, x1), (y0, y1), (z0, _z1) = rd_box
    p = np.zeros((6, 4))
    p[:, 0] = alpha0
    p[:, 1] = beta0
    p[:, 2] = thickness
    p[0, 3], p[1, 3] = x1, x0
    p[2, 3], p[3, 3] = y1, y0
    p[4, 3], p[5, 3] = 1.0e30, z0
    return p


def box_mesh(nx: int, ny: int, nz: int, h: float, npml: int,
             alpha0: float = 5.0, beta0: float = 400.0) -> Mesh:
    """Regular domain of nx*ny*nz elements of edge ``h`` centred at x = y = 0 with
    its top face at z = 0, wrapped by ``npml`` PML elements on x+-, y+- and z-."""
    if min(nx, ny, nz) < 1 or npml < 1:
        raise ValueError("need at least one RD element per axis and one PML layer")
    EX, EY, EZ = nx + 2 * npml, ny + 2 * npml, nz + npml
    NX, NY, NZ = 2 * EX + 1, 2 * EY + 1, 2 * EZ + 1
    s = 0.5 * h
    xs = -0.5 * nx * h - npml * h + s * np.arange(NX)
    ys = -0.5 * ny * h - npml * h + s * np.arange(NY)
    zs = -(nz + npml) * h + s * np.arange(NZ)
    zz, yy, xx = np.meshgrid(zs, ys, xs, indexing="ij")
    xyz = np.stack([xx.ravel(), yy.ravel(), zz.ravel()], axis=1)

    ek, ej, ei = np.meshgrid(np.arange(EZ), np.arange(EY), np.arange(EX), indexing="ij")
    ei, ej, ek = ei.ravel(), ej.ravel(), ek.ravel()
    a, b, c = LOCAL_IJK[:, 0], LOCAL_IJK[:, 1], LOCAL_IJK[:, 2]
    gi = 2 * ei[:, None] + a[None, :]
    gj = 2 * ej[:, None] + b[None, :]
    gk = 2 * ek[:, None] + c[None, :]
    inod = (gi + NX * (gj + NY * gk)).astype(np.int32)
    in_rd = ((ei >= npml) & (ei < npml + nx) & (ej >= npml) & (ej < npml + ny) & (ek >= npml))
    mtel = np.where(in_rd, 1, 2).astype(np.int32)
    eid = np.stack([ei, ej, ek], axis=1).astype(np.int32)

    nj = NX * NY * NZ
    in_rd_el = np.zeros(nj, dtype=bool)
    in_pml_el = np.zeros(nj, dtype=bool)
    in_rd_el[inod[mtel == 1].ravel()] = True
    in_pml_el[inod[mtel == 2].ravel()] = True
    node_mat_id = np.where(in_rd_el & ~in_pml_el, 0, np.where(in_rd_el & in_pml_el, 1, 2)).astype(np.int8)

    # constraints (1 = fixed), S2/Main.F90:448-520
    cons = np.zeros((nj, 9), dtype=np.int8)
    cons[~in_pml_el, 3:9] = 1
    ii = np.arange(nj) % NX
    jj = (np.arange(nj) // NX) % NY
    kk = np.arange(nj) // (NX * NY)
    outer = (ii == 0) | (ii == NX - 1) | (jj == 0) | (jj == NY - 1) | (kk == 0)
    cons[outer, 0:3] = 1
    free = cons.ravel() == 0
    ID = np.full(nj * 9, -1, dtype=np.int64)
    ID[free] = np.arange(int(free.sum()))
    ID = ID.reshape(nj, 9).astype(np.int32)
    neq = int(free.sum())

    store_nodes = np.nonzero(node_mat_id <= 1)[0].astype(np.int32)
    store_eq = ID[store_nodes][:, 0:3].reshape(-1).astype(np.int32)

    rd_box = ((-0.5 * nx * h, 0.5 * nx * h), (-0.5 * ny * h, 0.5 * ny * h), (-nz * h, 0.0))
    # material extension: PML node -> the interface node reached by clamping its
    # lattice index into the RD lattice (perpendicular projection onto the RD box)
    ci = np.clip(ii, 2 * npml, 2 * (npml + nx))
    cj = np.clip(jj, 2 * npml, 2 * (npml + ny))
    ck = np.clip(kk, 2 * npml, NZ - 1)
    extend_to = (ci + NX * (cj + NY * ck)).astype(np.int32)
    pml_param = default_pml_param(rd_box, npml * h, alpha0, beta0)
    return Mesh(nx=nx, ny=ny, nz=nz, npml=npml, h=h, xyz=xyz, inod=inod, mtel=mtel, eid=eid,
                ID=ID, neq=neq, node_mat_id=node_mat_id, store_nodes=store_nodes, store_eq=store_eq,
                extend_to=extend_to, pml_param=pml_param, rd_box=rd_box, lattice=(NX, NY, NZ))


def surface_grid(mesh: Mesh, coords) -> np.ndarray:
    """Node ids of a surface (z = 0) receiver grid, x varying fastest."""
    nodes = [mesh.node_at(x, y, 0.0) for y in coords for x in coords]
    return np.asarray(nodes, dtype=np.int32)


def element_colors(mesh: Mesh) -> np.ndarray:
    """8-colouring of the structured element lattice: elements of one colour share no node."""
    e = mesh.eid.astype(np.int64)
    return ((e[:, 0] & 1) + 2 * (e[:, 1] & 1) + 4 * (e[:, 2] & 1)).astype(np.int32)
