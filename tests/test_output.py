"""Output formats on the host (no GPU): the VTK writer, the .dat field files, the step
histories and the state-file layout, through the library's host-only entry points."""
from __future__ import annotations

import ctypes as C

import numpy as np

import imex_b200 as ix
from imex_b200.problems import read_state_file, vortex, write_state_file


def _dp(a):
    return np.ascontiguousarray(a, dtype=np.float64).ctypes.data_as(C.POINTER(C.c_double))


def _parse_vtk(path):
    tok = open(path).read().split("\n")
    return tok


def test_vtk_writer_declares_what_it_writes(tmp_path):
    lib = ix.load_library()
    nx, ny = 6, 4
    rng = np.random.default_rng(0)
    cons = rng.standard_normal((8, ny, nx))
    prim = rng.standard_normal((8, ny, nx))
    path = tmp_path / "a.vtk"
    assert lib.imex_vtk_write_host(str(path).encode(), nx, ny, -1.0, 2.0, 0.5, 0.25, 0.125, 7, _dp(cons), _dp(prim)) == 0
    lines = open(path).read().splitlines()
    assert lines[0] == "# vtk DataFile Version 3.0" and lines[3] == "DATASET RECTILINEAR_GRID"
    assert lines[6] == "7" and float(lines[8]) == 0.125
    assert lines[9] == f"DIMENSIONS {nx + 1} {ny + 1} 1"
    assert lines[10] == f"X_COORDINATES {nx + 1} double"
    xs = np.array(lines[11].split(), dtype=float)
    np.testing.assert_array_equal(xs, -1.0 + 0.5 * np.arange(nx + 1))
    assert lines[12] == f"Y_COORDINATES {ny + 1} double"
    np.testing.assert_array_equal(np.array(lines[13].split(), dtype=float), 2.0 + 0.25 * np.arange(ny + 1))
    assert lines[16] == f"CELL_DATA {nx * ny}" and lines[17] == "FIELD FieldData 13"
    names = ["rho", "mom_X", "mom_Y", "mom_Z", "U", "B_X", "B_Y", "B_Z", "velX", "velY", "velZ", "p", "B"]
    row = 18
    for v, name in enumerate(names):
        assert lines[row] == f"{name} 1 {nx * ny} double"
        vals = np.array(" ".join(lines[row + 1:row + 1 + ny]).split(), dtype=float).reshape(ny, nx)
        if v < 8:
            want = cons[v]
        elif v < 12:
            want = prim[v - 7]
        else:
            want = np.sqrt(cons[5] ** 2 + cons[6] ** 2 + cons[7] ** 2)
        np.testing.assert_array_equal(vals, want, err_msg=name)  # 17 significant digits round-trip
        row += 1 + ny
    assert row == len(lines)


def test_dat_and_history_writers(tmp_path):
    lib = ix.load_library()
    nx, ny = 5, 3
    plane = np.arange(nx * ny, dtype=float).reshape(ny, nx) / 7.0
    path = tmp_path / "RK_rho.dat"
    assert lib.imex_dat_write_host(str(path).encode(), nx, ny, 0.0, -1.0, 0.2, 0.5, _dp(plane)) == 0
    d = np.loadtxt(path)
    assert d.shape == (nx * ny, 3)
    i, j = np.meshgrid(np.arange(nx), np.arange(ny), indexing="ij")  # x outer, y inner
    np.testing.assert_allclose(d[:, 0], 0.2 * (i.ravel() + 0.5), rtol=0, atol=1e-15)
    np.testing.assert_allclose(d[:, 1], -1.0 + 0.5 * (j.ravel() + 0.5), rtol=0, atol=1e-15)
    np.testing.assert_array_equal(d[:, 2], plane[j.ravel(), i.ravel()])
    steps = (C.c_int * 3)(1, 2, 3)
    vals = np.array([1e-16, 2.5e-15, 3.0])
    hp = tmp_path / "RK_div_error.dat"
    assert lib.imex_history_write_host(str(hp).encode(), 3, steps, _dp(vals)) == 0
    h = np.loadtxt(hp)
    np.testing.assert_array_equal(h[:, 0], [1, 2, 3])
    np.testing.assert_array_equal(h[:, 1], vals)


def test_state_file_round_trip(tmp_path):
    p = vortex(12, 10)
    path = tmp_path / "s.bin"
    write_state_file(p, str(path), t=0.5, timestep=3, prev_dt=0.01)
    h, prim, bx, by, A = read_state_file(str(path))
    assert h["nx"] == 12 and h["ny"] == 10 and h["timestep"] == 3 and h["t"] == 0.5 and h["prev_dt"] == 0.01
    np.testing.assert_array_equal(prim, p.prim)
    np.testing.assert_array_equal(bx, p.bx)
    np.testing.assert_array_equal(by, p.by)
    np.testing.assert_array_equal(A, p.A)
