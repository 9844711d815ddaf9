"""Output formats and the time-marching driver on the GPU: the per-step diagnostics, the VTK
and field files of a device state, bit-exact restart from a state file, and the imex_run
executable (the reference's main() over the C ABI) against the same run through the binding."""
from __future__ import annotations

import os
import subprocess

import numpy as np
import pytest

import imex_b200 as ix
from imex_b200.problems import read_state_file, vortex, write_state_file
from oracle.bindings import make_solver

pytestmark = pytest.mark.gpu

CFG = dict(recon="VanLeer", magfield="StaggerCT", GMREStol=1e-12)
HERE = os.path.dirname(os.path.abspath(__file__))
DRIVER = os.path.join(os.path.dirname(HERE), "imex_b200", "imex_run")


def test_diagnostics_match_the_state_and_the_oracle():
    p = vortex(32)
    sv = ix.Solver.for_problem(p, 2, CFG)
    cpu = make_solver("port", p, 2, CFG)
    for _ in range(3):
        sv.step()
        cpu.step()
    d = sv.diagnostics()
    u = cpu.cons()
    k = 0.5 * (u[1] ** 2 + u[2] ** 2 + u[3] ** 2) / u[0]
    m = 0.5 * (u[5] ** 2 + u[6] ** 2 + u[7] ** 2)
    e = u[4] - k - m
    assert d["timestep"] == 3 and d["t"] == pytest.approx(cpu.scalars()["t"], rel=1e-13)
    assert d["mass"] == pytest.approx(u[0].sum() * p.dx * p.dy, rel=1e-12)
    assert d["intE"] == pytest.approx(e.sum() * p.dx * p.dy, rel=1e-10)
    assert d["emin"] == pytest.approx(e.min(), rel=1e-10)
    assert d["magE_max"] == pytest.approx(m.max(), rel=1e-10)
    j, i = np.unravel_index(np.argmin(e), e.shape)
    assert d["emin_x"] == pytest.approx(p.x0 + (i + 0.5) * p.dx) and d["emin_y"] == pytest.approx(p.y0 + (j + 0.5) * p.dy)
    div = sv.divergence()
    assert d["div_error"] == div["face_l2"] and d["B_inf"] == div["cell_inf"]
    assert d["div_error"] == pytest.approx(cpu.div_error(), rel=1e-6, abs=1e-14)
    sc = sv.scalars()
    assert d["dt_comp"] == pytest.approx(sc["ch"] / sc["v_max"], rel=1e-12)
    sv.close()


def test_vtk_and_field_files_hold_the_device_state(tmp_path):
    p = vortex(24, 20)
    sv = ix.Solver.for_problem(p, 2, CFG)
    sv.step()
    cons, prim = sv.cons(), sv.prim()
    sv.write_vtk(str(tmp_path / "s.vtk"), cycle=1)
    lines = open(tmp_path / "s.vtk").read().splitlines()
    assert lines[9] == "DIMENSIONS 25 21 1" and lines[16] == f"CELL_DATA {24 * 20}"
    rho = np.array(" ".join(lines[19:39]).split(), dtype=float).reshape(20, 24)
    np.testing.assert_array_equal(rho, cons[0])
    sv.write_fields_dat(str(tmp_path))
    for name, want in (("RK_rho", cons[0]), ("RK_E", cons[4]), ("RK_p", prim[4]), ("RK_vx", prim[1]),
                       ("RK_Bz", prim[7]), ("RK_v_mag", np.sqrt(prim[1] ** 2 + prim[2] ** 2))):
        d = np.loadtxt(tmp_path / f"{name}.dat")
        np.testing.assert_array_equal(d[:, 2], want.T.ravel(), err_msg=name)
    sv.close()


def test_restart_from_a_state_file_continues_bit_for_bit(tmp_path):
    p = vortex(32)
    a = ix.Solver.for_problem(p, 2, CFG)
    for _ in range(6):
        a.step()
    b = ix.Solver.for_problem(p, 2, CFG)
    for _ in range(3):
        b.step()
    path = str(tmp_path / "mid.bin")
    b.save_state_file(path)
    b.close()
    c = ix.Solver(p.nx, p.ny, dict(p.settings, **CFG), (p.x0, p.x1, p.y0, p.y1), 2)
    c.load_state_file(path)
    assert c.scalars()["timestep"] == 3
    for _ in range(3):
        c.step()
    np.testing.assert_array_equal(c.cons(), a.cons())
    for x, y in zip(c.faces(), a.faces()):
        np.testing.assert_array_equal(x, y)
    assert c.scalars()["t"] == a.scalars()["t"]
    a.close()
    c.close()


def test_imex_run_driver_matches_the_binding(tmp_path):
    assert os.path.exists(DRIVER), "imex_b200/imex_run not built"
    p = vortex(32)
    init = str(tmp_path / "init.bin")
    write_state_file(p, init)
    cfg = tmp_path / "run.cfg"
    cfg.write_text("\n".join([
        "# the vortex on [-5, 5]^2", "nx = 32", "ny = 32", "RKs = 2", "recon = VanLeer", "magfield = StaggerCT",
        "GMREStol = 1e-12", "caltimestep = IMEXdt", "CFL = 0.8", "gamma_plasma = 1.6666666666666667",
        "vortex_test = 1", f"x_0 = {p.x0}", f"x_1 = {p.x1}", f"y_0 = {p.y0}", f"y_1 = {p.y1}",
        "time_stop = 0.5", "plot_interval = 4", "name = vortex"]) + "\n")
    out = tmp_path / "out"
    out.mkdir()
    r = subprocess.run([DRIVER, str(cfg), init, str(out)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    step_lines = [l for l in r.stdout.splitlines() if l.startswith("[timestep, dt, time]")]
    diag_lines = [l for l in r.stdout.splitlines() if l.startswith("DIAG ts=")]
    n = len(step_lines)
    assert n >= 2 and len(diag_lines) == n
    assert len([l for l in r.stdout.splitlines() if l.startswith("[CT-DIAG] ")]) == 4 * n
    # the same run through the binding
    sv = ix.Solver.for_problem(p, 2, dict(CFG, time_stop=0.5))
    for _ in range(n):
        sv.step()
    assert sv.scalars()["t"] == pytest.approx(0.5, abs=1e-14)
    h, prim, bx, by, _ = read_state_file(str(out / "final_state.bin"))
    assert h["timestep"] == n
    np.testing.assert_array_equal(prim, sv.prim())
    np.testing.assert_array_equal(bx, sv.faces()[0])
    hist = np.loadtxt(out / "RK_div_error.dat")
    assert hist.shape == (n, 2) and hist[-1, 1] == sv.divergence()["face_l2"]
    assert np.loadtxt(out / "RK_B_inf.dat").shape == (n, 2) and np.loadtxt(out / "RK_dt_comp.dat").shape == (n, 2)
    vtks = sorted(f for f in os.listdir(out) if f.endswith(".vtk"))
    want = {0} | {s for s in range(1, n + 1) if s % 4 == 0} | {n}
    assert vtks == sorted(f"plt_vortex_{s}.vtk" for s in want)
    assert np.loadtxt(out / "RK_rho.dat").shape == (32 * 32, 3)
    sv.close()


@pytest.mark.parametrize("kind", ["vortex", "open_blast", "sheet_primstate"])
def test_ct_emf_diagnostics_match_the_oracle(kind):
    """The reference driver's per-step [CT-DIAG] figures (Diagnose_CT_EMF) on the device against
    the oracle's restatement, which prints exactly the reference's lines."""
    from imex_b200.problems import open_blast, vortex_sheet
    if kind == "vortex":
        prob, st = vortex(24, 20), dict(recon="VanLeer", magfield="StaggerCT")
    elif kind == "open_blast":
        prob, st = open_blast(40, 36), dict(recon="WENO5", magfield="StaggerCT", p_floor=1e-8)
    else:
        prob, st = vortex_sheet(48), dict(recon="WENO5", magfield="PotentialA", p_floor=1e-8, theta=0.5,
                                          reconstate="PrimState")
    sv = ix.Solver.for_problem(prob, 2, st)
    cpu = make_solver("port", prob, 2, st)
    for _ in range(2):
        sv.step()
        cpu.step()
    g, c = sv.ct_emf_diagnostics(), cpu.ct_diag()
    for name in c:
        np.testing.assert_allclose(g[name], c[name], rtol=1e-9, atol=1e-14, err_msg=name)
    sv.close()
