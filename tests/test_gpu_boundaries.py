"""Transmissive boundaries (x_Transmissive / y_Transmissive) on the GPU, through the C ABI.

The reference fills the ghost cells of a transmissive direction with the nearest interior
cell (bound_cond_u, bound_cond_array, M_P / M_B), keeps the boundary normal faces Bx(x_0)
and By(y_0) as degrees of freedom that CT evolves, and clamps the averaged part of the
corner EMF on x_0 / y_0 (constrained_transport.cpp:5-30,147-164).  The checks here:

* every sub-step of every stage on the oracle's inputs of that sub-step: the explicit ones
  and CT (boundary faces included) bit-identical, the solves to 1e-12;
* full steps against the reference's golden steps are covered with the periodic ones in
  test_gpu_parity.py (the open-blast fixtures), boundary faces included;
* at 256^2: face div B at round-off, p > 0, bit-identical repeat runs;
* restart files carry the boundary faces (version 2) and continue bit for bit;
* mixed precision against FP64 at the north-star tolerance;
* ensembles of transmissive members match their single runs;
* the legacy CT variants (Staggered_CT, Unstaggered_CT) bit-identical on open boundaries;
* what is not built for these boundaries is refused, not run.
"""
from __future__ import annotations

import numpy as np
import pytest

import imex_b200 as ix
from conftest import rel
from imex_b200.problems import open_blast, read_state_file
from oracle.bindings import make_solver

pytestmark = pytest.mark.gpu

SUB_CASES = [
    (2, dict(recon="VanLeer", magfield="StaggerCT")),
    (3, dict(recon="WENO5", magfield="StaggerCT", p_floor=1e-8, y_bc="y_Periodic")),
    (2, dict(recon="Minmod", magfield="StaggerCT", x_bc="x_Periodic", formula="EnergyFormula", GMREStol=1e-12)),
    (2, dict(recon="ENO3", magfield="NoDivFree", reconstate="PrimState")),
    (3, dict(recon="WENO5", magfield="PotentialA", p_floor=1e-8, theta=0.5)),
    (2, dict(recon="Minmod", magfield="UnStaggerCT")),
    (2, dict(recon="VanLeer", magfield="StaggerCT", GLF=0, add_pvisc="AlfvenSpeedp")),
    (3, dict(recon="WENO5", magfield="PotentialA", p_floor=1e-8, theta=0.5, GLF=0)),
]


@pytest.mark.parametrize("rks,settings", SUB_CASES, ids=["vanleer_ct", "weno5_ct_yper", "energy_xper", "eno3_nodiv",
                                                        "weno5_potentialA", "minmod_unstag", "vanleer_ct_local",
                                                        "weno5_potentialA_local"])
def test_gpu_substeps_match_oracle_transmissive(rks, settings):
    prob = open_blast(40, 36)
    o = make_solver("port", prob, rks, settings)
    o.step()  # a non-trivial state at the boundaries
    o.step(snapshots=True)
    sc = o.scalars()
    ae, ai = o.tableau()
    exact = lambda a, b, msg: np.testing.assert_array_equal(a, b, err_msg=msg)
    g = ix.Solver.for_problem(prob, rks, dict(settings, arith="exact"))
    energy = settings.get("formula") == "EnergyFormula"
    for k in range(rks):
        S = lambda sub, w: o.snapshot(k, sub, w)
        SB = lambda sub, w: o.snapshot_boundary(k, sub, w)
        adt = ai[k, k] * sc["dt"]
        g.set_scalars(dt=sc["dt"], adt=adt, B_max_x=sc["B_max_x"], B_max_y=sc["B_max_y"],
                      vx_max=sc["vx_max"], vy_max=sc["vy_max"], a_max=sc["a_max"], v_max=sc["v_max"])
        g.set_buffer("Qe", S("combine", "Qe"))
        g.set_buffer("Qs", S("combine", "Qs"))
        g.TVDReconstruction()
        g.set_buffer("cons", S("combine", "u_con"))
        g.RusanovC_Update(adt, k)
        exact(g.get_buffer("cons")[:5], S("convective", "u_con")[:5], f"RusanovC stage {k}")
        g.set_buffer("cons", S("convective", "u_con"))
        if settings["magfield"] == "PotentialA":
            g.set_buffer("A", S("convective", "A"))
            g.set_buffer("A_s", S("combine", "A_s"))
            g.MagSubsystem_UpdateA(adt, k)
            assert rel(g.get_buffer("A"), S("magnetic", "A")) < 1e-12
        else:
            g.MagSubsystem_UpdateB(adt, k)
            assert rel(g.get_buffer("Fx"), S("magnetic", "Fx")) < 1e-12
            assert rel(g.get_buffer("Fy"), S("magnetic", "Fy")) < 1e-12
        assert rel(g.get_buffer("cons")[5:], S("magnetic", "u_con")[5:]) < 1e-12
        g.set_buffer("cons", S("magnetic", "u_con"))
        (g.Energy_flux_Update if energy else g.Pressure_flux_Update)(adt, k)
        exact(g.get_buffer("cons")[:5], S("pflux", "u_con")[:5], f"second flux stage {k}")
        g.set_buffer("cons", S("pflux", "u_con"))
        (g.PreSubsystem_Energy if energy else g.PreSubsystem_Pressure)(adt, k)
        out = g.get_buffer("cons")
        for q in (1, 2, 4):
            assert rel(out[q], S("pressure", "u_con")[q]) < 1e-12, (k, q)
        if settings["magfield"] == "StaggerCT":
            g.set_buffer("cons", S("pressure", "u_con"))
            g.set_buffer("Fx", S("magnetic", "Fx"))
            g.set_buffer("Fy", S("magnetic", "Fy"))
            g.set_buffer("bxQs", S("combine", "bxQs"))
            g.set_buffer("byQs", S("combine", "byQs"))
            g.set_buffer("bxQs_x0", SB("combine", "bxQs"))
            g.set_buffer("byQs_y0", SB("combine", "byQs"))
            g.Staggered_CT_Consistent(adt, k)
            exact(g.get_buffer("bx"), S("ct", "bx"), "CT bx")
            exact(g.get_buffer("by"), S("ct", "by"), "CT by")
            if settings.get("x_bc", "x_Transmissive") == "x_Transmissive":
                exact(g.get_buffer("bx_x0"), SB("ct", "bx"), "CT Bx on x_0")
            if settings.get("y_bc", "y_Transmissive") == "y_Transmissive":
                exact(g.get_buffer("by_y0"), SB("ct", "by"), "CT By on y_0")
            exact(g.get_buffer("cons"), S("ct", "u_con"), f"CT stage {k}")
        if settings["magfield"] == "UnStaggerCT":
            g.set_buffer("cons", S("pressure", "u_con"))
            g.set_buffer("Fx", S("magnetic", "Fx"))
            g.set_buffer("Fy", S("magnetic", "Fy"))
            g.set_buffer("A", S("pressure", "A"))
            g.set_buffer("A_s", S("combine", "A_s"))
            g.Unstaggered_CT_Consistent(adt, k)
            exact(g.get_buffer("A"), S("ct", "A"), "CT A")
            exact(g.get_buffer("cons"), S("ct", "u_con"), f"CT stage {k}")
    g.close()


def test_gpu_full_steps_match_oracle_transmissive():
    """Several whole steps against the oracle on a grid that is not a multiple of any tile."""
    prob = open_blast(70, 45)
    settings = dict(recon="WENO5", magfield="StaggerCT", p_floor=1e-8)
    cpu = make_solver("port", prob, 3, settings)
    gpu = ix.Solver.for_problem(prob, 3, settings)
    for _ in range(4):
        assert gpu.step() == pytest.approx(cpu.step(), rel=1e-13)
    a, b = gpu.cons(), cpu.cons()
    for k in range(8):
        assert rel(a[k], b[k]) <= 1e-12, k
    for u, v in zip(gpu.boundary_faces(), cpu.boundary_faces()):
        assert rel(u, v) <= 1e-12
    assert gpu.divergence()["face_l2"] == pytest.approx(cpu.div_error(), rel=1e-6, abs=1e-14)
    gpu.close()


@pytest.mark.parametrize("magfield,div", [("StaggerCT", "face_l2"), ("PotentialA", "cell_ref_l2")])
def test_gpu_transmissive_properties_256(magfield, div):
    """div B at round-off in each form's own measure (cal_divergence_error, imex_subsystems.cpp:630-660)."""
    prob = open_blast(256)
    settings = dict(recon="WENO5", magfield=magfield, p_floor=1e-8)
    runs = []
    for _ in range(2):
        gpu = ix.Solver.for_problem(prob, 3, settings)
        for _ in range(12):
            gpu.step()
            assert gpu.divergence()[div] <= 1e-12
            assert gpu.min_pressure() > 0.0
        c = gpu.cons()
        assert np.isfinite(c).all()
        runs.append((c, gpu.boundary_faces()))
        gpu.close()
    np.testing.assert_array_equal(runs[0][0], runs[1][0])
    for u, v in zip(runs[0][1], runs[1][1]):
        np.testing.assert_array_equal(u, v)


def test_gpu_restart_file_carries_the_boundary_faces(tmp_path):
    prob = open_blast(48, 40)
    settings = dict(recon="VanLeer", magfield="StaggerCT")
    a = ix.Solver.for_problem(prob, 2, settings)
    for _ in range(5):
        a.step()
    b = ix.Solver.for_problem(prob, 2, settings)
    for _ in range(2):
        b.step()
    path = tmp_path / "open.state"
    b.save_state_file(path)
    b.close()
    header, *_ = read_state_file(str(path))
    assert header["version"] == 2 and header["bx_x0"].shape == (40,) and header["by_y0"].shape == (48,)
    c = ix.Solver(prob.nx, prob.ny, dict(prob.settings, **settings), (prob.x0, prob.x1, prob.y0, prob.y1), 2)
    c.load_state_file(path)
    for _ in range(3):
        c.step()
    np.testing.assert_array_equal(c.cons(), a.cons())
    for u, v in zip(c.boundary_faces(), a.boundary_faces()):
        np.testing.assert_array_equal(u, v)
    a.close()
    c.close()


@pytest.mark.parametrize("magfield", ["StaggerCT", "PotentialA"])
def test_gpu_mixed_precision_transmissive(magfield):
    prob = open_blast(128)
    settings = dict(recon="WENO5", magfield=magfield, p_floor=1e-8, mixed_solves=3)
    f = ix.Solver.for_problem(prob, 3, settings)
    m = ix.Solver.for_problem(prob, 3, dict(settings, precision="mixed"))
    for _ in range(3):
        assert m.step() == pytest.approx(f.step(), rel=1e-12)
    a, b = m.cons(), f.cons()
    for k in range(8):
        assert rel(a[k], b[k]) <= 1e-8, k
    f.close()
    m.close()


@pytest.mark.parametrize("magfield,bc", [
    ("StaggerCT", ("x_Transmissive", "y_Transmissive")),
    ("StaggerCT", ("x_Periodic", "y_Transmissive")),
    ("UnStaggerCT", ("x_Transmissive", "y_Transmissive")),
    ("UnStaggerCT", ("x_Transmissive", "y_Periodic")),
], ids=["stag_open", "stag_y_open", "unstag_open", "unstag_x_open"])
def test_gpu_legacy_ct_transmissive_bit_exact(magfield, bc):
    """Staggered_CT / Unstaggered_CT (constrained_transport.cpp:66-143, 436-498) on open
    boundaries against the oracle: face EMFs from the reconstructed u_con clamped at the
    boundary, the boundary corners and faces of the consistent form, and A_s read with the
    extrapolated ghosts of bound_cond_A."""
    prob = open_blast(40, 36)
    settings = dict(recon="VanLeer", magfield=magfield, x_bc=bc[0], y_bc=bc[1])
    o = make_solver("port", prob, 2, settings)
    o.step()
    o.step(snapshots=True)
    k = 1  # the oracle's own bxQs / byQs boundary lines are the last stage's
    S = lambda sub, w: o.snapshot(k, sub, w)
    SB = lambda sub, w: o.snapshot_boundary(k, sub, w)
    u, Q, Qs = S("pressure", "u_con"), S("combine", "Qe"), S("combine", "Qs")
    bxq, byq = S("combine", "bxQs"), S("combine", "byQs")
    A, As = S("pressure", "A"), S("combine", "A_s")
    bx, by = S("pressure", "bx"), S("pressure", "by")
    h = 0.01
    ref = o.substep(6, h, k, u, Q, Qs, bx, by, bxq, byq, A, As)
    bx0, by0 = o.boundary_faces()
    g = ix.Solver.for_problem(prob, 2, dict(settings, arith="exact"))
    for name, val in (("cons", u), ("Qe", Q), ("Qs", Qs), ("bx", bx), ("by", by), ("bxQs", bxq),
                      ("byQs", byq), ("A", A), ("A_s", As)):
        g.set_buffer(name, val)
    if bc[0] == "x_Transmissive":
        g.set_buffer("bxQs_x0", SB("combine", "bxQs"))
    if bc[1] == "y_Transmissive":
        g.set_buffer("byQs_y0", SB("combine", "byQs"))
    (g.Staggered_CT if magfield == "StaggerCT" else g.Unstaggered_CT)(h, k)
    exact = lambda a, b, msg: np.testing.assert_array_equal(a, b, err_msg=msg)
    exact(g.get_buffer("cons"), ref["u_con"], "u_con")
    if magfield == "StaggerCT":
        exact(g.get_buffer("bx"), ref["bx"], "bx")
        exact(g.get_buffer("by"), ref["by"], "by")
        if bc[0] == "x_Transmissive":
            exact(g.get_buffer("bx_x0"), bx0, "Bx on x_0")
        if bc[1] == "y_Transmissive":
            exact(g.get_buffer("by_y0"), by0, "By on y_0")
    else:
        exact(g.get_buffer("A")[2], ref["A"][2], "A_z")
    g.close()


def test_gpu_unbuilt_boundary_paths_are_refused():
    prob = open_blast(16)
    sv = ix.Solver.for_problem(prob, 2, dict(magfield="StaggerCT", fixed_dt=0.01))
    with pytest.raises(ix.ImexError) as err:
        sv.adjoint_run(1, prob.prim[0], prob.prim[5:8])
    assert err.value.status == 2
    sv.close()


@pytest.mark.parametrize("rks,settings", [
    (2, dict(recon="VanLeer", magfield="StaggerCT")),
    (3, dict(recon="WENO5", magfield="PotentialA", p_floor=1e-8, theta=0.5, GMREStol=1e-12)),
], ids=["staggered", "potentialA"])
def test_gpu_batch_of_open_members_matches_single_runs(rks, settings):
    """An ensemble of transmissive members on uneven grids: each member's batched solves (its
    own CTA range, tiles clamped at its own boundaries) against the same run alone."""
    probs = [open_blast(40, 32), open_blast(64), open_blast(24, 48)]
    batch = ix.Batch(probs, rks, settings)
    batch.step(3)
    for m, p in enumerate(probs):
        single = ix.Solver.for_problem(p, rks, settings)
        for _ in range(3):
            single.step()
        a, b = batch.members[m].cons(), single.cons()
        for k in range(8):
            assert rel(a[k], b[k]) <= 1e-11, (m, k, rel(a[k], b[k]))
        for u, v in zip(batch.members[m].boundary_faces(), single.boundary_faces()):
            assert rel(u, v) <= 1e-11
        single.close()
    batch.close()


def test_imex_run_driver_transmissive_matches_the_binding(tmp_path):
    """The driver takes x_bc / y_bc by name and reads and writes the version-2 state files."""
    import os
    import subprocess

    from imex_b200.problems import write_state_file
    driver = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "imex_b200", "imex_run")
    assert os.path.exists(driver), "imex_b200/imex_run not built"
    p = open_blast(40, 32)
    init = str(tmp_path / "init.bin")
    write_state_file(p, init)
    cfg = tmp_path / "open.cfg"
    cfg.write_text("\n".join([
        "nx = 40", "ny = 32", "RKs = 2", "recon = VanLeer", "magfield = StaggerCT", "x_bc = x_Transmissive",
        "y_bc = y_Transmissive", "vortex_test = 0", "gamma_plasma = 1.6666666666666667", f"x_0 = {p.x0}",
        f"x_1 = {p.x1}", f"y_0 = {p.y0}", f"y_1 = {p.y1}", "time_stop = 0.05", "plot_interval = 0",
        "name = open"]) + "\n")
    out = tmp_path / "out"
    out.mkdir()
    r = subprocess.run([driver, str(cfg), init, str(out)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    n = len([l for l in r.stdout.splitlines() if l.startswith("[timestep, dt, time]")])
    assert n >= 2
    sv = ix.Solver.for_problem(p, 2, dict(recon="VanLeer", magfield="StaggerCT", time_stop=0.05))
    for _ in range(n):
        sv.step()
    h, prim, bx, by, _ = read_state_file(str(out / "final_state.bin"))
    assert h["timestep"] == n and h["version"] == 2
    np.testing.assert_array_equal(prim, sv.prim())
    np.testing.assert_array_equal(bx, sv.faces()[0])
    bxb, byb = sv.boundary_faces()
    np.testing.assert_array_equal(h["bx_x0"], bxb)
    np.testing.assert_array_equal(h["by_y0"], byb)
    sv.close()


def test_gpu_boundary_face_lines_follow_each_directions_kind():
    """A transmissive direction stores the line it is given; a periodic direction ignores it and
    reports the faces it identifies with x_0 / y_0, those at x_1 / y_1."""
    prob = open_blast(20, 16)
    sv = ix.Solver.for_problem(prob, 2, dict(magfield="StaggerCT", x_bc="x_Periodic"))
    bxb, byb = sv.boundary_faces()
    bx, by = sv.faces()
    np.testing.assert_array_equal(bxb, bx[:, -1])       # periodic x: Bx at x_1 of each row
    np.testing.assert_array_equal(byb, prob.by_y0)      # transmissive y: the line that was set
    sv.set_boundary_faces(np.full(16, 7.0), np.full(20, 3.0))
    bxb2, byb2 = sv.boundary_faces()
    np.testing.assert_array_equal(bxb2, bx[:, -1])
    np.testing.assert_array_equal(byb2, np.full(20, 3.0))
    sv.close()
    # without set_boundary_faces, the line defaults to the first interior face of its row / column
    q = open_blast(20, 16)
    q.bx_x0 = q.by_y0 = None
    sv = ix.Solver.for_problem(q, 2, dict(magfield="StaggerCT"))
    bxb, byb = sv.boundary_faces()
    np.testing.assert_array_equal(bxb, q.bx[:, 0])
    np.testing.assert_array_equal(byb, q.by[0, :])
    sv.close()


@pytest.mark.parametrize("shape,settings", [
    ((6, 5), dict(recon="WENO5", magfield="PotentialA", p_floor=1e-8, theta=0.5, GMREStol=1e-12)),
    ((5, 7), dict(recon="VanLeer", magfield="StaggerCT", GMREStol=1e-12)),
    ((4, 4), dict(recon="Minmod", magfield="UnStaggerCT", GMREStol=1e-12)),
    ((33, 17), dict(recon="ENO3", magfield="StaggerCT", y_bc="y_Periodic", GMREStol=1e-12)),
], ids=["6x5_potentialA", "5x7_staggered", "4x4_unstaggered", "33x17_yperiodic"])
def test_gpu_tiny_and_odd_open_grids_match_oracle(shape, settings):
    """Grids smaller than one solver tile (32 x 16), so a tile holds both boundaries of a
    direction and the halo extrapolates past both ends; and a grid one cell past a tile."""
    prob = open_blast(*shape)
    cpu = make_solver("port", prob, 2, settings)
    gpu = ix.Solver.for_problem(prob, 2, settings)
    for _ in range(3):
        assert gpu.step() == pytest.approx(cpu.step(), rel=1e-12)
    a, b = gpu.cons(), cpu.cons()
    for k in range(8):
        assert rel(a[k], b[k]) <= 1e-11, (k, rel(a[k], b[k]))
    for u, v in zip(gpu.boundary_faces(), cpu.boundary_faces()):
        assert rel(u, v) <= 1e-11
    gpu.close()
