"""Restatement of the step-3 partitioner (PIC) steps that produce the solver's
integer inputs, and of the files it reads and writes.

* ``numbering``: rank locations of nodes, global and per-rank PETSc node numbers,
  application and PETSc equation numbers (S3/PIC_ReNumbering.F90:34-319).
* ``het_mat_numbering``: element and node PML regions, node material ids
  (regular domain / interface / PML) and the map of PML nodes onto the interface
  node whose material they take (S3/PIC_Heterogeneous_Material.F90:551-1000, 3D).
* ``inversion_ds``: per-rank index sets idx_Mat_from, idx_Mat_Extend_from/to,
  U_Store_Numbers_Global and idx_u_from/to (S3/PIC_Inversion_Data_Structure.F90:143-369).
* The ``.Inv_DS`` file those sets are written to, which S4/IO_Parallel_Inversion.F90 reads.
* The step-3 input files ``<name>.txt``, ``.XYZ``, ``.Cnn``, ``.Cnt`` in the layout the
  partitioner's reader expects (S3/PIC_Input.F90), with the column layout of the
  step-2 writer (S2/Main.F90:741-760).

The element partition, computed by METIS in the reference, is an input here.  Array
values follow the reference: 1-based node and equation numbers where it uses them,
and 0-based where it subtracts one before writing.
"""
from __future__ import annotations

import dataclasses
import os

import numpy as np

NDOF = 9
TOL = 1.0e-6            # S3/PIC_Heterogeneous_Material.F90:165
CENTRE = 26             # local node 27 of SHAPE_3_27: the element centre


# ---------------------------------------------------------------------------
# Numbering (S3/PIC_ReNumbering.F90:34-319)

@dataclasses.dataclass
class Numbering:
    member: np.ndarray            # [nj, nparts] bool: the node belongs to an element of the part
    global_petsc_num: np.ndarray  # [nj] 1-based PETSc node number
    npart: np.ndarray             # [nj] 1-based part that numbers the node (owner)
    neq_rank: np.ndarray          # [nparts] highest equation number held by each part
    nnode_rank: np.ndarray        # [nparts] highest PETSc node number held by each part
    local_petsc_num: np.ndarray   # [nj, nparts] 1-based local node number, 0 if absent
    id_application: np.ndarray    # [nj, 9] 1-based equation in application order, 0 fixed
    id_petsc: np.ndarray          # [nj, 9] row = PETSc node number - 1; 1-based equation, 0 fixed
    neq_total: int

    @property
    def nj_rank(self) -> np.ndarray:
        return self.local_petsc_num.max(axis=0)

    def equation_ids(self) -> np.ndarray:
        """0-based PETSc equation of every (node, DOF) in application node order, -1 if
        fixed: the ID array of the C ABI."""
        eq = self.id_petsc[self.global_petsc_num - 1]
        return (eq - 1).astype(np.int32)


def numbering(inod: np.ndarray, flags: np.ndarray, epart: np.ndarray, nparts: int) -> Numbering:
    """inod [nel, nnode] 0-based node ids; flags [nj, 9] constraints (0 free, 1 fixed);
    epart [nel] 1-based part of each element."""
    inod = np.asarray(inod)
    flags = np.asarray(flags)
    epart = np.asarray(epart)
    nj = flags.shape[0]
    if np.any((flags != 0) & (flags != 1)):
        raise ValueError("constraint flags must be 0 or 1")
    member = np.zeros((nj, nparts), dtype=bool)
    for p in range(nparts):
        member[inod[epart == p + 1].ravel(), p] = True
    if not member.any(axis=1).all():
        raise ValueError("a node belongs to no element")
    # a node is numbered by the lowest part that holds it (interior nodes of a part
    # and the ghost nodes not numbered by a lower part), in node order per part
    glob = np.zeros(nj, dtype=np.int64)
    npart = np.zeros(nj, dtype=np.int64)
    neq_rank = np.zeros(nparts, dtype=np.int64)
    nnode_rank = np.zeros(nparts, dtype=np.int64)
    free_per_node = (flags == 0).sum(axis=1)
    count = 0
    for p in range(nparts):
        nodes = np.nonzero(member[:, p] & (glob == 0))[0]
        glob[nodes] = count + 1 + np.arange(nodes.size)
        npart[nodes] = p + 1
        count += nodes.size
        neq_rank[p] = free_per_node[nodes].sum()
        nnode_rank[p] = count
    neq_rank = np.cumsum(neq_rank)
    local = np.where(member, np.cumsum(member, axis=0), 0).astype(np.int64)

    def number(f):
        out = np.zeros(f.shape, dtype=np.int64)
        free = f.ravel() == 0
        out.ravel()[free] = np.arange(1, int(free.sum()) + 1)
        return out

    id_app = number(flags)
    perm = np.empty_like(flags)
    perm[glob - 1] = flags
    id_petsc = number(perm)
    return Numbering(member, glob, npart, neq_rank, nnode_rank, local, id_app, id_petsc, int(id_app.max(initial=0)))


# ---------------------------------------------------------------------------
# PML regions and the material extension map (S3/PIC_Heterogeneous_Material.F90:551-1000)

# (LOCx, LOCy, LOCz) -> region number of the reference (18 = regular domain)
_REGION = {(1, 1, 0): 1, (1, 0, 0): 2, (1, -1, 0): 3, (1, 1, -1): 4, (1, 0, -1): 5, (1, -1, -1): 6,
           (0, 1, 0): 7, (0, -1, 0): 8, (0, 1, -1): 9, (0, 0, -1): 10, (0, -1, -1): 11,
           (-1, 1, 0): 12, (-1, 0, 0): 13, (-1, -1, 0): 14, (-1, 1, -1): 15, (-1, 0, -1): 16,
           (-1, -1, -1): 17, (0, 0, 0): 18}
_SLABS = (2, 7, 8, 10, 13)
_TUBES = (1, 3, 5, 9, 11, 12, 14, 16)
_BOXES = (4, 6, 15, 17)


@dataclasses.dataclass
class MaterialMap:
    element_region: np.ndarray    # [nel] 1..18
    node_region: np.ndarray       # [nj] 1..18
    node_mat_id: np.ndarray       # [nj] 0 regular domain, 1 interface, 2 PML
    mat_indep_num: np.ndarray     # [nj] 1-based number of nodes with their own material, 0 for PML nodes
    node_mat_mapping: np.ndarray  # [nj] 1-based node whose material the node takes (itself if independent)


def _last_wins(target: np.ndarray, idx: np.ndarray, vals: np.ndarray) -> None:
    """target[idx[k]] = vals[k] for k in order, so the last write to an index wins."""
    if idx.size == 0:
        return
    u, first_rev = np.unique(idx[::-1], return_index=True)
    target[u] = vals[::-1][first_rev]


def het_mat_numbering(xyz: np.ndarray, inod: np.ndarray, pml_start: np.ndarray) -> MaterialMap:
    """xyz [nj, 3]; inod [nel, 27] 0-based (SHAPE_3_27 order); pml_start = PML_DIM(1:6, 1)
    = (x-, x+, y-, y+, z-, z+) planes where the PML starts."""
    xyz = np.asarray(xyz, dtype=np.float64)
    inod = np.asarray(inod)
    x02, x01, x04, x03, x06, x05 = (float(v) for v in pml_start)
    if x02 > x01 or x04 > x03 or x06 > x05:
        raise ValueError("PML starting planes out of order")
    c = xyz[inod[:, CENTRE]]
    locx = np.where(c[:, 0] >= x01, 1, np.where(c[:, 0] <= x02, -1, 0))
    locy = np.where(c[:, 1] >= x03, 1, np.where(c[:, 1] <= x04, -1, 0))
    if np.any(c[:, 2] > x05):
        raise ValueError("element in the top PML zone (the reference stops here)")
    locz = np.where(c[:, 2] <= x06, -1, 0)
    er = np.array([_REGION[(a, b, d)] for a, b, d in zip(locx, locy, locz)], dtype=np.int64)
    nel, nn = inod.shape
    nj = xyz.shape[0]
    # node regions: slabs, then tubes, then boxes; within a pass the last element wins
    nr = np.full(nj, 18, dtype=np.int64)
    for group in (_SLABS, _TUBES, _BOXES):
        sel = np.nonzero(np.isin(er, group))[0]
        _last_wins(nr, inod[sel].ravel(), np.repeat(er[sel], nn))
    # node material ids
    mid = np.zeros(nj, dtype=np.int64)
    mid[inod[er != 18].ravel()] = 2
    planes = {2: (0, x01), 13: (0, x02), 7: (1, x03), 8: (1, x04), 10: (2, x06)}
    for reg, (ax, x0) in planes.items():
        nodes = np.unique(inod[er == reg].ravel())
        mid[nodes[np.abs(xyz[nodes, ax] - x0) < TOL]] = 1
    indep = np.zeros(nj, dtype=np.int64)
    keep = mid != 2
    indep[keep] = np.arange(1, int(keep.sum()) + 1)
    mapping = np.where(indep != 0, np.arange(1, nj + 1), 0).astype(np.int64)
    # interface nodes in node order; a later interface node overwrites an earlier match
    match_axes = {1: (2,), 3: (2,), 12: (2,), 14: (2,), 4: (), 6: (), 15: (), 17: (),
                  2: (1, 2), 13: (1, 2), 7: (0, 2), 8: (0, 2), 5: (1,), 16: (1,), 9: (0,), 11: (0,), 10: (0, 1)}
    region_nodes = {r: np.nonzero(nr == r)[0] for r in match_axes}
    for ij in np.nonzero(mid == 1)[0]:
        r = int(nr[ij])
        if r not in match_axes:
            continue
        cand = region_nodes[r]
        axes = match_axes[r]
        if not axes:
            mapping[cand] = ij + 1
            continue
        diff = np.zeros(cand.size)
        for ax in axes:
            diff = diff + np.abs(xyz[ij, ax] - xyz[cand, ax])
        mapping[cand[diff < TOL]] = ij + 1
    return MaterialMap(er, nr, mid, indep, mapping)


# ---------------------------------------------------------------------------
# Inversion index sets (S3/PIC_Inversion_Data_Structure.F90:143-369), 0-based as written

@dataclasses.dataclass
class InvDS:
    nj_rank: int
    nj_mapping: int
    nstore_mapping: int
    nstore_rank: int
    idx_mat_from: np.ndarray
    idx_mat_extend_from: np.ndarray
    idx_mat_extend_to: np.ndarray
    u_store_numbers_global: np.ndarray
    idx_u_from: np.ndarray
    idx_u_to: np.ndarray


def inversion_ds(num: Numbering, mat: MaterialMap, flags: np.ndarray, ndim: int = 3) -> list[InvDS]:
    flags = np.asarray(flags)
    nparts = num.member.shape[1]
    nj = flags.shape[0]
    stored = mat.node_mat_id <= 1
    out = []
    for p in range(nparts):
        loc = num.local_petsc_num[:, p]
        nj_rank = int(loc.max())
        idx_mat_from = np.zeros(nj_rank, dtype=np.int64)
        has = np.nonzero(loc)[0]
        idx_mat_from[loc[has] - 1] = num.global_petsc_num[has]
        nj_mapping = int(num.nnode_rank[p] - (num.nnode_rank[p - 1] if p else 0))
        own = np.nonzero(num.npart == p + 1)[0]
        if np.any(mat.node_mat_mapping[own] == 0):
            raise ValueError("a node has no material mapping")
        ext_from = num.global_petsc_num[mat.node_mat_mapping[own] - 1]
        ext_to = num.global_petsc_num[own]
        own_st = own[stored[own]]
        if np.any(num.id_application[own_st, :ndim] == 0):
            raise ValueError("a stored node has a fixed displacement DOF")
        u_store = num.id_petsc[num.global_petsc_num[own_st] - 1, :ndim].ravel()
        rank_st = has[stored[has]]
        u_from = num.id_petsc[num.global_petsc_num[rank_st] - 1, :ndim].ravel()
        # local equation numbers of the part's nodes in local node order
        id_local = np.zeros((nj_rank, NDOF), dtype=np.int64)
        id_local[loc[has] - 1] = flags[has]
        free = id_local.ravel() == 0
        numbered = np.zeros(id_local.size, dtype=np.int64)
        numbered[free] = np.arange(1, int(free.sum()) + 1)
        id_local = numbered.reshape(nj_rank, NDOF)
        u_to = id_local[loc[rank_st] - 1, :ndim].ravel()
        if np.any(u_to == 0):
            raise ValueError("a stored node has a fixed local displacement DOF")
        out.append(InvDS(nj_rank, nj_mapping, int(u_store.size), int(u_from.size), idx_mat_from - 1, ext_from - 1,
                         ext_to - 1, u_store - 1, u_from - 1, u_to - 1))
    return out


def _fmt_ints(vals) -> str:
    return "".join(f"{int(v):10d} " for v in vals)


def write_inv_ds(path: str, ds: InvDS) -> None:
    """One rank's ``<model>_<nparts>_<rank>.Inv_DS`` file: every line is a run of
    (I10,1X) integers followed by its label (S3/PIC_Inversion_Data_Structure.F90:385-398)."""
    lines = [_fmt_ints([ds.nj_rank, ds.nj_mapping, ds.nstore_mapping, ds.nstore_rank])
             + "NJ_Rank(IParts) | NJ_Mapping | NStore_Mapping | NStore_Rank",
             _fmt_ints(ds.idx_mat_from) + "idx_Mat_from",
             _fmt_ints(ds.idx_mat_extend_from) + "idx_Mat_Extend_from",
             _fmt_ints(ds.idx_mat_extend_to) + "idx_Mat_Extend_to",
             _fmt_ints(ds.u_store_numbers_global) + "U_Store_Numbers_Global",
             _fmt_ints(ds.idx_u_from) + "idx_u_from",
             _fmt_ints(ds.idx_u_to) + "idx_u_to"]
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")


def read_inv_ds(path: str) -> InvDS:
    """Read a ``.Inv_DS`` file as the list-directed reads of S4 do: the integers of
    each line, the trailing label ignored."""
    def ints(line, n):
        tok = line.split()
        return np.array([int(t) for t in tok[:n]], dtype=np.int64)

    with open(path) as f:
        lines = f.read().splitlines()
    nj_rank, nj_mapping, nstore_mapping, nstore_rank = (int(v) for v in ints(lines[0], 4))
    return InvDS(nj_rank, nj_mapping, nstore_mapping, nstore_rank, ints(lines[1], nj_rank), ints(lines[2], nj_mapping),
                 ints(lines[3], nj_mapping), ints(lines[4], nstore_mapping), ints(lines[5], nstore_rank),
                 ints(lines[6], nstore_rank))


# ---------------------------------------------------------------------------
# Step-3 input files (S3/PIC_Input.F90), written with the step-2 formats (S2/Main.F90:741-760)

@dataclasses.dataclass
class Step3Model:
    xyz: np.ndarray            # [nj, 3]
    inod: np.ndarray           # [nel, 27] 0-based
    mtel: np.ndarray           # [nel] 1 regular domain, 2 PML
    elt: np.ndarray            # [nel] element type (34 regular-domain, 35 PML 27-node hexahedra)
    elgr: np.ndarray           # [nel] element group
    flags: np.ndarray          # [nj, 9] 0 free, 1 fixed
    pmat: np.ndarray           # [nmat, 8] material properties
    pml_dim: np.ndarray        # [2, 6] PML_DIM(1:6, 1:2): starting planes (x-, x+, y-, y+, z-, z+), outer planes
    ndan: np.ndarray           # [nndh] 1-based nodes with displacement history
    nparts: int = 1


def from_mesh(mesh, pmat=None, history_nodes=None) -> Step3Model:
    """The step-3 model of a ``hirensi_b200.mesh`` box mesh."""
    nj = mesh.nj
    flags = (mesh.ID < 0).astype(np.int64)
    (x0, x1), (y0, y1), (z0, _z1) = mesh.rd_box
    lo = mesh.xyz.min(axis=0)
    hi = mesh.xyz.max(axis=0)
    pml_dim = np.array([[x0, x1, y0, y1, z0, hi[2] + 1.0e30],
                        [lo[0], hi[0], lo[1], hi[1], lo[2], hi[2]]], dtype=np.float64)
    if pmat is None:
        pmat = np.zeros((1, 8))
    nd = np.zeros(0, dtype=np.int64) if history_nodes is None else np.asarray(history_nodes, dtype=np.int64) + 1
    return Step3Model(mesh.xyz.copy(), mesh.inod.astype(np.int64), mesh.mtel.astype(np.int64),
                      np.where(mesh.mtel == 1, 34, 35).astype(np.int64), np.ones(mesh.nel, dtype=np.int64), flags,
                      np.asarray(pmat, dtype=np.float64), pml_dim, nd, 1)


def write_step3(model: Step3Model, directory: str, name: str) -> None:
    """<name>.txt (basic data, dynamic-analysis block, materials, PML planes,
    displacement-history nodes), <name>.XYZ, <name>.Cnn and <name>.Cnt."""
    os.makedirs(directory, exist_ok=True)
    nel, nn = model.inod.shape
    nj = model.xyz.shape[0]
    nmat = model.pmat.shape[0]
    L = []
    L += [f"! step-3 input of {name}", "!", "!", "!", "!", "!", "! NEl NJ NGroup MaxNNode NDOF NDim"]
    L.append(f"{nel} {nj} {nmat} {nn} {NDOF} 3")
    L += ["!", "! load cases: body force, pressure, concentrated, supports, dynamic", "!", "0 0 0 0 1", "!"]
    # dynamic analysis: load type 1 (dynamic pressure), PML present
    L += ["! LoadType PML", "1 1", "!"]
    L += ["! NNDH NNVH NNAH NDamp NEnergy PARAM_Type", f"{model.ndan.size} 0 0 0 0 0", "!"]
    L += ["! NIDBC", "0", "!"]
    L += ["!", "! NParts NumFlag Matrix_Type MetisType KWay", f"{model.nparts} 1 1 0 {model.nparts}", "!"]
    # arrays
    L += ["!", "!", "! materials", "!", "!"]
    for k in range(nmat):
        L.append(f"{k + 1} " + " ".join(f"{v:.17g}" for v in model.pmat[k]))
    L.append("!")
    L += ["! PML dimensions", "! starting planes x- x+ y- y+ z- z+", " ".join(f"{v:.17g}" for v in model.pml_dim[0]),
          "! outer planes", " ".join(f"{v:.17g}" for v in model.pml_dim[1]), "!"]
    L += ["! dynamic pressure elements", "!"]
    L += ["! NDAN", " ".join(str(int(v)) for v in model.ndan), "!"]
    L += ["! NVAN", "", "!", "! NAAN", "", "!"]
    with open(os.path.join(directory, name + ".txt"), "w") as f:
        f.write("\n".join(L) + "\n")
    with open(os.path.join(directory, name + ".XYZ"), "w") as f:
        for i in range(nj):
            # full precision (the step-2 writer's E18.10 would round off-lattice coordinates)
            f.write(f"{i + 1:19d}  " + "".join(f"{v:25.17E}  " for v in model.xyz[i]) + "\n")
    with open(os.path.join(directory, name + ".Cnn"), "w") as f:
        for e in range(nel):
            f.write(f"{e + 1:19d}  " + "".join(f"{int(v) + 1:19d}  " for v in model.inod[e])
                    + f"{int(model.mtel[e]):5d}  {int(model.elt[e]):5d}  {int(model.elgr[e]):5d}\n")
    with open(os.path.join(directory, name + ".Cnt"), "w") as f:
        for j in range(nj):
            f.write(f"{j + 1:19d}  " + "".join(f"{int(v):1d} " for v in model.flags[j]) + "\n")


def read_step3(directory: str, name: str) -> Step3Model:
    """Read the step-3 input with the reference reader's line sequence
    (Input_BASIC and Input_Arrays, S3/PIC_Input.F90) for a model with the dynamic
    load case only."""
    with open(os.path.join(directory, name + ".txt")) as f:
        lines = f.read().splitlines()
    pos = 7
    nel, nj, ngroup, nnode, ndof, ndim = (int(v) for v in lines[pos].split()[:6])
    pos += 2                                # line 8 read, line 9 skipped
    pos += 2                                # two comment lines
    loadc = [int(v) for v in lines[pos].split()[:5]]
    pos += 2
    if any(loadc[:4]):
        raise ValueError("only the dynamic load case is read")
    pos += 1
    ltype, pml_flag = (int(v) for v in lines[pos].split()[:2])
    pos += 2
    pos += 1
    nndh = int(lines[pos].split()[0])
    pos += 2
    if ltype == 1:
        pos += 1
        nidbc = int(lines[pos].split()[0])
        pos += 2
    else:
        nidbc = 0
    pos += 2
    nparts = int(lines[pos].split()[0])
    pos += 2
    # Input_Arrays
    pos += 2 + 3
    pmat = np.zeros((ngroup, 8))
    for _ in range(ngroup):
        tok = lines[pos].split()
        pmat[int(tok[0]) - 1] = [float(v) for v in tok[1:9]]
        pos += 1
    pos += 1
    pml_dim = np.zeros((2, 2 * ndim))
    if pml_flag == 1:
        pos += 1
        for j in range(2):
            pos += 1
            pml_dim[j] = [float(v) for v in lines[pos].split()[:2 * ndim]]
            pos += 1
        pos += 1
    if ltype == 1:
        pos += 1 + nidbc + 1
    pos += 1
    ndan = np.array([int(v) for v in lines[pos].split()[:nndh]], dtype=np.int64)
    xyz = np.zeros((nj, ndim))
    with open(os.path.join(directory, name + ".XYZ")) as f:
        for line in f:
            tok = line.split()
            if tok:
                xyz[int(tok[0]) - 1] = [float(v) for v in tok[1:1 + ndim]]
    inod = np.zeros((nel, nnode), dtype=np.int64)
    mtel = np.zeros(nel, dtype=np.int64)
    elt = np.zeros(nel, dtype=np.int64)
    elgr = np.zeros(nel, dtype=np.int64)
    with open(os.path.join(directory, name + ".Cnn")) as f:
        for line in f:
            tok = line.split()
            if tok:
                e = int(tok[0]) - 1
                inod[e] = [int(v) - 1 for v in tok[1:1 + nnode]]
                mtel[e], elt[e], elgr[e] = (int(v) for v in tok[1 + nnode:4 + nnode])
    flags = np.zeros((nj, ndof), dtype=np.int64)
    with open(os.path.join(directory, name + ".Cnt")) as f:
        for line in f:
            tok = line.split()
            if tok:
                flags[int(tok[0]) - 1] = [int(v) for v in tok[1:1 + ndof]]
    return Step3Model(xyz, inod, mtel, elt, elgr, flags, pmat, pml_dim, ndan, nparts)
