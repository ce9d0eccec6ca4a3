"""On-disk formats the HiReNSI driver reads and writes around the time loop.

* ``<model>.HisD.txt``: receiver displacement histories.  Two header lines, then for
  each step 0..NSTEP the time (E14.6E3) and, per receiver node, the NDim components
  (E18.10E3, 2x) followed by 3x (writer S4/PTC_Results.F90:99-101, 218-227).  The
  measured data Dis_meas(0:NSTEP, NNDH*NDim) is read back with the same format
  (S4/PTC_Input.F90:1015-1021), i.e. with 10 significant digits.
* ``<model>_<nparts>_<rank>.Lambda`` / ``.Mu``: the nodal material of an inversion
  iterate, one E31.23E3 value per line (writer S4/Material_Save_Disk.F90:29-44,
  reader S4/PTC_Input.F90:1172-1273).  With the lambda + 2 mu variable the file holds
  lambda.

Numbers are written with Fortran E editing: sign, ``0.``, d digits, ``E``, signed
exponent of e digits, right-justified in w columns.
"""
from __future__ import annotations

import numpy as np


def fortran_e(v: float, w: int, d: int, e: int = 3) -> str:
    """Fortran Ew.dEe edit of v (round to nearest, mantissa in [0.1, 1))."""
    v = float(v)
    if not np.isfinite(v):
        raise ValueError("non-finite value")
    if v == 0.0:
        body = "0." + "0" * d + "E+" + "0" * e
        sign = ""
    else:
        s = f"{abs(v):.{d - 1}e}"          # d significant digits, correctly rounded
        mant, ex = s.split("e")
        digits = mant.replace(".", "")
        x = int(ex) + 1
        if abs(x) >= 10 ** e:
            raise ValueError("exponent does not fit")
        body = "0." + digits + "E" + ("+" if x >= 0 else "-") + f"{abs(x):0{e}d}"
        sign = "-" if v < 0 else ""
    out = sign + body
    if len(out) > w:
        out = out.replace("0.", ".", 1)   # the optional leading zero goes first
    if len(out) > w:
        return "*" * w
    return out.rjust(w)


# ---------------------------------------------------------------------------
# displacement histories

def write_hisd(path: str, time: np.ndarray, dis: np.ndarray, app_nodes, petsc_nodes) -> None:
    """time [nstep+1]; dis [nstep+1, nndh*3] (node-major, components x, y, z);
    app_nodes / petsc_nodes: 1-based node numbers of the NNDH receivers."""
    app_nodes = [int(v) for v in app_nodes]
    petsc_nodes = [int(v) for v in petsc_nodes]
    nndh = len(app_nodes)
    dis = np.asarray(dis, dtype=np.float64).reshape(len(time), nndh * 3)
    with open(path, "w") as f:
        f.write("History of Displacements and stresses \n")
        f.write("Time     " + "".join(f"App#{a:19d} PETSc#{p:19d} " for a, p in zip(app_nodes, petsc_nodes)) + "\n")
        for n, t in enumerate(time):
            row = [fortran_e(t, 14, 6), "  "]
            for k in range(nndh):
                for c in range(3):
                    row += [fortran_e(dis[n, 3 * k + c], 18, 10), "  "]
                row.append("   ")
            f.write("".join(row) + "\n")


def read_hisd(path: str, nndh: int, nstep: int) -> tuple[np.ndarray, np.ndarray]:
    """(time [nstep+1], Dis_meas [nstep+1, nndh*3]) read by fixed columns, as the
    formatted read of the reference does."""
    with open(path) as f:
        lines = f.read().splitlines()
    time = np.zeros(nstep + 1)
    dis = np.zeros((nstep + 1, nndh * 3))
    for n in range(nstep + 1):
        line = lines[2 + n]
        time[n] = float(line[0:14])
        pos = 16
        for k in range(nndh):
            for c in range(3):
                dis[n, 3 * k + c] = float(line[pos:pos + 18])
                pos += 20
            pos += 3
    return time, dis


def traces_to_dis_meas(traces: np.ndarray) -> np.ndarray:
    """One shot's receiver traces [nrec3][nstep+1] (the C ABI layout) as Dis_meas
    [nstep+1][nrec3]."""
    return np.ascontiguousarray(np.asarray(traces).T)


def dis_meas_to_traces(dis: np.ndarray) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(dis).T)


# ---------------------------------------------------------------------------
# material resume files

def write_material(path_lambda: str, path_mu: str, lam: np.ndarray, mu: np.ndarray, lambda_2mu: bool = False) -> None:
    """lam holds lambda, or lambda + 2 mu when lambda_2mu (then lambda is written)."""
    lam = np.asarray(lam, dtype=np.float64)
    mu = np.asarray(mu, dtype=np.float64)
    out_l = lam - 2.0 * mu if lambda_2mu else lam
    with open(path_lambda, "w") as f:
        f.write("".join(fortran_e(v, 31, 23) + "  \n" for v in out_l))
    with open(path_mu, "w") as f:
        f.write("".join(fortran_e(v, 31, 23) + "  \n" for v in mu))


def read_material(path_lambda: str, path_mu: str, nj: int) -> tuple[np.ndarray, np.ndarray]:
    def read(path):
        with open(path) as f:
            vals = [float(line[:31]) for line in f.read().splitlines()[:nj]]
        if len(vals) != nj:
            raise ValueError(f"{path}: expected {nj} values")
        return np.array(vals)

    return read(path_lambda), read(path_mu)
