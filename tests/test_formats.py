"""Fortran E editing and the history / material files of the driver."""
import os
import tempfile

import numpy as np
import pytest

from hirensi_b200 import formats as F


@pytest.mark.parametrize("v,w,d,text", [
    (1.0, 18, 10, " 0.1000000000E+001"),
    (-2.5e-5, 18, 10, "-0.2500000000E-004"),
    (0.0, 18, 10, " 0.0000000000E+000"),
    (1.0e-4, 14, 6, " 0.100000E-003"),
    (123.456, 14, 6, " 0.123456E+003"),
    (-9.9999999999e-3, 18, 10, "-0.1000000000E-001"),   # rounds up into the next decade
    (2.0 / 3.0, 31, 23, " 0.66666666666666662965923E+000"),
])
def test_fortran_e_edit(v, w, d, text):
    out = F.fortran_e(v, w, d)
    assert out == text and len(out) == w


def test_hisd_round_trip_keeps_ten_digits():
    rng = np.random.default_rng(0)
    nstep, nndh = 12, 4
    time = np.arange(nstep + 1) * 1.0e-4
    dis = rng.standard_normal((nstep + 1, nndh * 3)) * 10.0 ** rng.integers(-12, 2, size=(nstep + 1, nndh * 3))
    with tempfile.TemporaryDirectory() as d:
        path = os.path.join(d, "Mesh.HisD.txt")
        F.write_hisd(path, time, dis, [5, 9, 11, 40], [5, 9, 11, 40])
        lines = open(path).read().splitlines()
        assert lines[0].startswith("History of Displacements")
        assert lines[1].startswith("Time     App#")
        assert len(lines[2]) == 14 + 2 + nndh * (3 * 20 + 3)
        t2, d2 = F.read_hisd(path, nndh, nstep)
    assert np.array_equal(t2, np.array([float(f"{v:.5e}") for v in time]))   # E14.6: 6 digits
    ten = np.array([[float(f"{v:.9e}") for v in row] for row in dis])
    assert np.array_equal(d2, ten)


def test_material_files_round_trip_exactly():
    rng = np.random.default_rng(1)
    lam = rng.uniform(50, 400, 37)
    mu = rng.uniform(20, 200, 37)
    with tempfile.TemporaryDirectory() as d:
        pl, pm = os.path.join(d, "Mesh_1_0.Lambda"), os.path.join(d, "Mesh_1_0.Mu")
        F.write_material(pl, pm, lam, mu)
        l2, m2 = F.read_material(pl, pm, 37)
        assert np.array_equal(l2, lam) and np.array_equal(m2, mu)
        F.write_material(pl, pm, lam + 2 * mu, mu, lambda_2mu=True)
        l3, _ = F.read_material(pl, pm, 37)
        assert np.allclose(l3, lam, rtol=1e-15, atol=0)


def test_traces_layout_conversion():
    tr = np.arange(15.0).reshape(3, 5)       # [nrec3][nstep+1]
    dm = F.traces_to_dis_meas(tr)
    assert dm.shape == (5, 3) and dm[2, 1] == tr[1, 2]
    assert np.array_equal(F.dis_meas_to_traces(dm), tr)
