"""Wavefield snapshots for ParaView, as the reference writes them, with raw binary
data files in place of HDF5 (no HDF5 library is available to this package).

The reference (S4/Solver_PETSc_Explicit.F90:936-975 -> Paraview_HDF5,
S4/ParaView.F90:1206-1440; geometry from S3/PIC_Output_HDF5.F90:675-800) writes
every NSParaview-th step:

* a data file with Dis, Vel, Acc as float32 [NJ][3] nodal vectors, built from the
  equation vector by walking the nodes and their x, y, z DOFs and writing 0 for a
  constrained DOF;
* one XDMF grid: time, a Mixed topology whose 27-node hexahedra are drawn as
  20-node hexahedra (XDMF cell type 48, serendipity node order: local nodes 1-12,
  then 17-20, then 13-16), the XYZ geometry and the three nodal attributes;
* a temporal collection that includes the step grids.

Here the same grids reference raw little-endian binary files through
``Format="Binary"`` data items, which ParaView's XDMF reader reads directly.  The
nodal data come from ``Solver.state`` (the checkpointed forward states).  As in
the reference, where the velocity and acceleration scatters are disabled, only
the displacement is required; velocity and acceleration are written when given.
"""
from __future__ import annotations

import os

import numpy as np

HEX20 = 48   # XDMF mixed-topology code of a 20-node hexahedron


def connectivity_mixed(inod: np.ndarray) -> np.ndarray:
    """Mixed-topology connectivity: per element the cell type then 20 node ids,
    with the reference's reordering of the 27-node hexahedron's edge nodes."""
    inod = np.asarray(inod, dtype=np.int64)
    order = np.concatenate([np.arange(12), np.arange(16, 20), np.arange(12, 16)])
    cells = np.empty((inod.shape[0], 21), dtype=np.int32)
    cells[:, 0] = HEX20
    cells[:, 1:] = inod[:, order]
    return cells.reshape(-1)


def nodal_vectors(ID: np.ndarray, eqvec: np.ndarray) -> np.ndarray:
    """float32 [NJ][3]: the x, y, z equation values of every node, 0 where constrained."""
    ID = np.asarray(ID)
    eq = ID[:, :3]
    out = np.zeros(eq.shape, dtype=np.float32)
    ok = eq >= 0
    out[ok] = np.asarray(eqvec, dtype=np.float64)[eq[ok]].astype(np.float32)
    return out


def _item(dims, number_type, precision, path):
    return (f'<DataItem Dimensions="{dims}" NumberType="{number_type}" Precision="{precision}" '
            f'Format="Binary" Endian="Little">{path}</DataItem>')


def write_geometry(out_dir: str, name: str, mesh) -> tuple[str, str]:
    """XYZ (float64 [NJ][3]) and the mixed connectivity (int32), written once."""
    os.makedirs(out_dir, exist_ok=True)
    xyz = os.path.join(out_dir, f"{name}_Geometry_XYZ.bin")
    cnn = os.path.join(out_dir, f"{name}_Geometry_Connectivity.bin")
    np.ascontiguousarray(mesh.xyz, dtype="<f8").tofile(xyz)
    connectivity_mixed(mesh.inod).astype("<i4").tofile(cnn)
    return os.path.basename(xyz), os.path.basename(cnn)


def write_step(out_dir: str, name: str, step: int, time: float, mesh, u, v=None, a=None) -> str:
    """One snapshot: the data files and the step's XDMF grid; returns the .xmf name."""
    nj, nel = mesh.xyz.shape[0], mesh.inod.shape[0]
    xyz, cnn = f"{name}_Geometry_XYZ.bin", f"{name}_Geometry_Connectivity.bin"
    if not os.path.exists(os.path.join(out_dir, xyz)):
        write_geometry(out_dir, name, mesh)
    attrs = []
    for label, field, vec in (("Displacement", "Dis", u), ("Velocity", "Vel", v), ("Acceleration", "Acc", a)):
        if vec is None:
            continue
        fn = f"Data_{name}_{step}_{field}.bin"
        nodal_vectors(mesh.ID, vec).astype("<f4").tofile(os.path.join(out_dir, fn))
        attrs.append(f'    <Attribute Name="{label}" AttributeType="Vector" Center="Node">\n'
                     f'      {_item(f"{nj} 3", "Float", 4, fn)}\n'
                     f'    </Attribute>')
    xmf = f"{name}_{step}.xmf"
    text = "\n".join([
        "<Grid GridType='Collection' CollectionType='Temporal'>",
        '  <Grid GridType="Uniform">',
        f'    <Time Value="{time:.10f}" />',
        f'    <Topology TopologyType="Mixed" NumberOfElements="{nel}" >',
        f'    {_item(nel * 21, "Int", 4, cnn)}',
        "    </Topology>",
        '    <Geometry GeometryType="XYZ">',
        f'      {_item(f"{nj} 3", "Float", 8, xyz)}',
        "    </Geometry>",
        *attrs,
        "  </Grid>",
        "</Grid>",
    ])
    with open(os.path.join(out_dir, xmf), "w") as f:
        f.write(text + "\n")
    return xmf


def write_collection(out_dir: str, name: str, step_files: list[str]) -> str:
    """The temporal collection that includes every step grid (the reference's wrapper file)."""
    path = os.path.join(out_dir, f"{name}_All.xmf")
    with open(path, "w") as f:
        f.write('<?xml version="1.0" ?>\n<!DOCTYPE Xdmf SYSTEM "Xdmf.dtd" []>\n')
        f.write('<Xdmf xmlns:xi="http://www.w3.org/2003/XInclude" Version="2.2">\n  <Domain>\n')
        f.write("   <Grid GridType='Collection' CollectionType='Temporal'>\n")
        for fn in step_files:
            f.write(f"     <xi:include href='{fn}'/>\n")
        f.write("   </Grid>\n  </Domain>\n</Xdmf>\n")
    return path


def write_forward(out_dir: str, name: str, solver, mesh, dt: float, shot: int = 0) -> str:
    """Every checkpointed state of a shot's last forward run as snapshots: needs
    ``solver.set_checkpointing(K)``; writes the steps 0, K, 2K, ... <= NSTEP."""
    K = solver.ckpt_interval
    if K <= 0:
        raise ValueError("snapshots need checkpointing: the states are the checkpoints")
    files = []
    for step in range(0, solver.nstep + 1, K):
        _, x2, x3 = solver.state(step, shot)
        files.append(write_step(out_dir, name, step, step * dt, mesh, x2, x3))
    return write_collection(out_dir, name, files)
