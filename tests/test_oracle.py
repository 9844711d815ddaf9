"""The oracle is pinned: the C restatement reproduces the reference's own code.

* against the committed golden fixtures (outputs of the reference's own code,
  tests/golden/make_golden.py) - runs anywhere;
* against the live reference library oracle/_ref when it is present.
Arithmetic is restated operand for operand, so ideal-gas results are required
to be bit-identical; the Redlich-Kwong EOS calls libm log/sqrt, which may
differ by an ulp between hosts, hence 1e-13.
"""
from __future__ import annotations

import numpy as np
import pytest

from conftest import golden_problem, golden_step_cases, load_golden, rel
from oracle.bindings import PortSolver, RefSolver, make_solver
from imex_b200.problems import vortex, vortex_sheet


@pytest.mark.parametrize("case", golden_step_cases())
def test_port_reproduces_reference_golden_steps(case):
    g = load_golden(f"step_{case}.npz")
    prob, rks, settings = golden_problem(g)
    port = make_solver("port", prob, rks, settings)
    exact = settings.get("eos_type", "IDEAL_GAS") == "IDEAL_GAS"
    for s in range(len(g["dt"])):
        dt = port.step()
        assert dt == g["dt"][s]
        cons = port.cons()
        bx, by = port.faces()
        if exact:
            np.testing.assert_array_equal(cons, g["cons"][s])
            np.testing.assert_array_equal(bx, g["bx"][s])
            np.testing.assert_array_equal(by, g["by"][s])
            np.testing.assert_array_equal(port.vector_potential(), g["A"][s])
        else:
            assert rel(cons, g["cons"][s]) < 1e-13
        if "bx_x0" in g.files:  # boundary normal faces of the transmissive directions
            bxb, byb = port.boundary_faces()
            np.testing.assert_allclose(bxb, g["bx_x0"][s], rtol=0 if exact else 1e-13, atol=0)
            np.testing.assert_allclose(byb, g["by_y0"][s], rtol=0 if exact else 1e-13, atol=0)
    assert port.div_error() == pytest.approx(float(g["div"]), rel=1e-10, abs=1e-14)


def test_port_reproduces_reference_golden_functions():
    g = load_golden("fn_vortex16x12.npz")
    from imex_b200.problems import vortex
    prob = vortex(16, 12)
    for scheme in ("NoRecon", "Minmod", "VanLeer", "ENO3", "WENO5"):
        s = make_solver("port", prob, 2, dict(recon=scheme, magfield="StaggerCT"))
        np.testing.assert_array_equal(s.reconstruct(g["Q"]), g[f"recon_{scheme}"])
    s = make_solver("port", prob, 2, dict(recon="Minmod", reconstate="PrimState", magfield="StaggerCT"))
    np.testing.assert_array_equal(s.reconstruct(g["Q"]), g["recon_Minmod_prim"])
    s = make_solver("port", prob, 2, dict(recon="VanLeer", magfield="StaggerCT", GMREStol=1e-12))
    np.testing.assert_array_equal(s.shock(g["Q"]), g["shock"])
    s.set_scalars(*g["scalars"])
    h = float(g["h"])
    np.testing.assert_array_equal(s.operator(0, g["ucon"], g["Q"], g["Qs"], h, g["x1"]), g["op_pressure_L"])
    np.testing.assert_array_equal(
        s.operator(1, g["ucon"], g["Q"], g["Qs"], h, g["x1"], pfreeze=g["pfreeze"], mbig=float(g["mbig"])),
        g["op_pressure_J"])
    np.testing.assert_array_equal(s.operator(2, g["ucon"], g["Q"], g["Qs"], h, g["x3"]), g["op_magnetic_B"])
    np.testing.assert_array_equal(s.operator(4, g["ucon"], g["Q"], g["Qs"], h, g["x1"]), g["op_energy"])
    np.testing.assert_array_equal(s.operator(3, g["ucon"], g["Q"], g["Qs"], h, g["x3"]), g["op_magnetic_A"])


def test_port_reproduces_reference_local_dissipation_operators():
    """The four operators with GLF = false on the inputs of the function fixture."""
    g = load_golden("fn_vortex16x12.npz")
    loc = load_golden("fn_local_vortex16x12.npz")
    from imex_b200.problems import vortex
    prob = vortex(16, 12)
    args = (g["ucon"], g["Q"], g["Qs"], float(g["h"]))
    for name, extra in (("", {}), ("_alfven", dict(add_pvisc="AlfvenSpeedp"))):
        s = make_solver("port", prob, 2, dict(recon="VanLeer", magfield="StaggerCT", GMREStol=1e-12, GLF=0, **extra))
        s.set_scalars(*g["scalars"])
        np.testing.assert_array_equal(s.operator(0, *args, g["x1"]), loc[f"op_pressure_L{name}"])
        np.testing.assert_array_equal(s.operator(1, *args, g["x1"], pfreeze=g["pfreeze"], mbig=float(g["mbig"])),
                                      loc[f"op_pressure_J{name}"])
    np.testing.assert_array_equal(s.operator(2, *args, g["x3"]), loc["op_magnetic_B"])
    sa = make_solver("port", prob, 2, dict(recon="WENO5", magfield="PotentialA", p_floor=1e-8, theta=0.5,
                                           GMREStol=1e-12, GLF=0))
    sa.set_scalars(*g["scalars"])
    np.testing.assert_array_equal(sa.operator(3, *args, g["x3"]), loc["op_magnetic_A"])


LIVE_CASES = [
    ("vortex", 20, 2, dict(recon="VanLeer", magfield="StaggerCT", GMREStol=1e-12), 2),
    ("vortex", 20, 2, dict(recon="Minmod", magfield="UnStaggerCT"), 2),
    ("vortex", 20, 3, dict(recon="ENO3", magfield="StaggerCT", PressureSolver="once_correction"), 1),
    ("sheet", 18, 3, dict(recon="WENO5", magfield="PotentialA", p_floor=1e-8, theta=0.5), 2),
    ("sheet", 18, 2, dict(recon="WENO5", magfield="PotentialA", add_bvisc=0, PressureSolver="no_correction"), 1),
    ("vortex", 20, 2, dict(recon="VanLeer", magfield="StaggerCT", caltimestep="Fullydt"), 2),
    ("vortex", 20, 2, dict(recon="VanLeer", magfield="StaggerCT", add_pvisc="AlfvenSpeedp"), 1),
    ("vortex", 20, 2, dict(recon="VanLeer", magfield="StaggerCT", formula="EnergyFormula"), 2),
    ("sheet", 18, 3, dict(recon="WENO5", magfield="PotentialA", p_floor=1e-8, formula="EnergyFormula"), 1),
    ("vortex", 20, 2, dict(recon="VanLeer", magfield="StaggerCT", GLF=0), 2),
    ("vortex", 20, 2, dict(recon="WENO5", magfield="StaggerCT", GLF=0, add_pvisc="AlfvenSpeedp"), 1),
    ("sheet", 18, 3, dict(recon="WENO5", magfield="PotentialA", p_floor=1e-8, theta=0.5, GLF=0), 2),
]


@pytest.mark.skipif(not RefSolver.available(), reason="oracle/_ref not built (no reference sources)")
@pytest.mark.parametrize("kind,n,rks,settings,steps", LIVE_CASES)
def test_port_matches_live_reference(kind, n, rks, settings, steps):
    prob = vortex(n) if kind == "vortex" else vortex_sheet(n)
    ref = make_solver("ref", prob, rks, settings)
    port = make_solver("port", prob, rks, settings)
    for _ in range(steps):
        assert ref.step(snapshots=True) == port.step(snapshots=True)
        for k in range(rks):
            for sub in ("combine", "convective", "magnetic", "pflux", "pressure", "ct"):
                a, b = ref.snapshot(k, sub, "u_con"), port.snapshot(k, sub, "u_con")
                assert (a is None) == (b is None)
                if a is not None:
                    np.testing.assert_array_equal(b, a, err_msg=f"stage {k} after {sub}")
    np.testing.assert_array_equal(port.cons(), ref.cons())


@pytest.mark.skipif(not RefSolver.available(), reason="oracle/_ref not built")
@pytest.mark.parametrize("rks,settings", [
    (2, dict(recon="VanLeer", magfield="StaggerCT")),
    (3, dict(recon="WENO5", magfield="StaggerCT", p_floor=1e-8, y_bc="y_Periodic")),
    (2, dict(recon="Minmod", magfield="NoDivFree", formula="EnergyFormula", GMREStol=1e-12)),
    (3, dict(recon="WENO5", magfield="PotentialA", p_floor=1e-8, theta=0.5)),
    (2, dict(recon="VanLeer", magfield="UnStaggerCT", x_bc="x_Periodic")),
    (2, dict(recon="VanLeer", magfield="StaggerCT", GLF=0)),
    (2, dict(recon="WENO5", magfield="PotentialA", p_floor=1e-8, theta=0.5, GLF=0)),
], ids=["vanleer_ct", "weno5_ct_yperiodic", "minmod_nodivfree_energy", "weno5_potentialA", "unstag_xperiodic",
        "vanleer_ct_local_lf", "weno5_potentialA_local_lf"])
def test_port_matches_live_reference_transmissive(rks, settings):
    """Transmissive boundaries: every sub-step of every stage, boundary faces included."""
    from imex_b200.problems import open_blast
    prob = open_blast(18, 14)
    ref = make_solver("ref", prob, rks, settings)
    port = make_solver("port", prob, rks, settings)
    for _ in range(2):
        assert ref.step(snapshots=True) == port.step(snapshots=True)
        for k in range(rks):
            for sub in ("combine", "convective", "magnetic", "pflux", "pressure", "ct"):
                a, b = ref.snapshot(k, sub, "u_con"), port.snapshot(k, sub, "u_con")
                assert (a is None) == (b is None)
                if a is None:
                    continue
                np.testing.assert_array_equal(b, a, err_msg=f"stage {k} after {sub}")
                np.testing.assert_array_equal(port.snapshot(k, sub, "A"), ref.snapshot(k, sub, "A"))
                for w in ("bx", "by", "bxQs", "byQs"):
                    np.testing.assert_array_equal(port.snapshot(k, sub, w), ref.snapshot(k, sub, w))
                    np.testing.assert_array_equal(port.snapshot_boundary(k, sub, w),
                                                  ref.snapshot_boundary(k, sub, w), err_msg=f"{w} line")
    np.testing.assert_array_equal(port.cons(), ref.cons())
    assert port.div_error() == ref.div_error()


def test_port_refuses_unsupported_boundaries():
    from imex_b200.problems import open_blast
    prob = open_blast(12)
    for bc, magfield in ((("x_Reflective", "y_Periodic"), "StaggerCT"), (("x_Dirichlet", "y_Periodic"), "StaggerCT"),
                         (("x_Periodic", "y_JetInflow"), "StaggerCT"), (("x_Transmissive", "y_Reflective"), "PotentialA")):
        with pytest.raises(RuntimeError):
            make_solver("port", prob, 2, dict(magfield=magfield, x_bc=bc[0], y_bc=bc[1]))


@pytest.mark.skipif(not RefSolver.available(), reason="oracle/_ref not built")
@pytest.mark.parametrize("bc", [None, ("x_Transmissive", "y_Transmissive"), ("x_Periodic", "y_Transmissive"),
                                ("x_Transmissive", "y_Periodic")], ids=["periodic", "open", "y_open", "x_open"])
def test_port_matches_live_reference_legacy_ct(bc):
    """Staggered_CT / Unstaggered_CT (reachable only via commented call sites main.cpp:500,504),
    on periodic and transmissive boundaries (the boundary lines of the faces come from each
    solver's own state, so both solvers take the same step first)."""
    from imex_b200.problems import open_blast
    for magfield in ("StaggerCT", "UnStaggerCT"):
        prob = vortex(16) if bc is None else open_blast(16, 12)
        settings = dict(recon="VanLeer", magfield=magfield)
        if bc is not None:
            settings.update(x_bc=bc[0], y_bc=bc[1])
        ref = make_solver("ref", prob, 2, settings)
        port = make_solver("port", prob, 2, settings)
        ref.step(snapshots=True)
        port.step(snapshots=True)
        Q = ref.snapshot(0, "combine", "Qe")
        Qs = ref.snapshot(0, "combine", "Qs")
        u = ref.snapshot(0, "pressure", "u_con")
        bxq, byq = ref.snapshot(0, "combine", "bxQs"), ref.snapshot(0, "combine", "byQs")
        A, As = ref.snapshot(0, "pressure", "A"), ref.snapshot(0, "combine", "A_s")
        bx, by = ref.snapshot(0, "pressure", "bx"), ref.snapshot(0, "pressure", "by")
        h = 0.01
        r = ref.substep(6, h, 0, u, Q, Qs, bx, by, bxq, byq, A, As)
        p = port.substep(6, h, 0, u, Q, Qs, bx, by, bxq, byq, A, As)
        for key in ("u_con", "bx", "by", "A"):
            np.testing.assert_array_equal(p[key], r[key], err_msg=f"{magfield} {key}")
        if bc is not None:  # the boundary lines of the open directions
            for u, v, kind in zip(port.boundary_faces(), ref.boundary_faces(), bc):
                if kind.endswith("Transmissive"):
                    np.testing.assert_array_equal(u, v, err_msg=f"{magfield} {kind} boundary faces")


def test_port_rejects_unsupported_configurations():
    prob = vortex(8)
    for bad in (dict(U_update=5), dict(formula=7)):
        with pytest.raises(RuntimeError):
            make_solver("port", prob, 2, bad)


RK_RANDOM = dict(recon="Minmod", magfield="StaggerCT", eos_type="REDLICH_KWONG", m_alfa=0.4275, m_b=0.0866)


def test_strong_field_redlich_kwong_is_not_finite_in_the_reference():
    """The reference scheme (its C restatement, bit-identical to it) turns the Redlich-Kwong
    random field non-finite within two steps at beta = 1e-4, and stays finite at beta = 0.1."""
    from imex_b200.problems import random_field
    bad = make_solver("port", random_field(32, beta=1e-4), 2, RK_RANDOM)
    finite = True
    for _ in range(2):
        bad.step()
        finite = finite and bool(np.isfinite(bad.cons()).all())
    assert not finite
    good = make_solver("port", random_field(32), 2, RK_RANDOM)
    for _ in range(4):
        good.step()
    assert np.isfinite(good.cons()).all()


def test_random_field_reference_is_sensitive_to_its_gmres_tolerance():
    """On the random field the magnetic systems are stiff (about a hundred GMRES steps per
    solve): the reference's own result moves by ~1e-10 when only GMREStol changes from
    1e-14 to 1e-16.  This is the noise floor of any comparison between two correct
    implementations that sum in different orders on this workload."""
    from imex_b200.problems import random_field
    p = random_field(48)
    runs = []
    for tol in (1e-14, 1e-16):
        o = make_solver("port", p, 2, dict(RK_RANDOM, GMREStol=tol))
        for _ in range(5):
            o.step()
        runs.append(o.cons())
    worst = max(rel(runs[0][k], runs[1][k]) for k in range(8))
    assert 1e-11 < worst < 5e-9


@pytest.mark.skipif(not RefSolver.available(), reason="oracle/_ref not built")
@pytest.mark.parametrize("kind", ["vortex", "open_blast", "sheet_primstate"])
def test_port_ct_emf_diagnostics_print_as_the_reference(kind):
    """Diagnose_CT_EMF (constrained_transport.cpp:166-222): the restatement's figures, printed
    the reference's way (%.3e), are the reference's own printed lines."""
    from imex_b200.problems import open_blast
    if kind == "vortex":
        prob, st = vortex(24, 20), dict(recon="VanLeer", magfield="StaggerCT")
    elif kind == "open_blast":
        prob, st = open_blast(24, 20), dict(recon="WENO5", magfield="StaggerCT", p_floor=1e-8)
    else:
        prob, st = vortex_sheet(32), dict(recon="WENO5", magfield="PotentialA", p_floor=1e-8, theta=0.5,
                                          reconstate="PrimState")
    ref, port = make_solver("ref", prob, 2, st), make_solver("port", prob, 2, st)
    for _ in range(2):
        ref.step()
        port.step()
    r, p = ref.ct_diag(), port.ct_diag()
    assert set(r) == set(p) == {"central", "rusanov", "tilde", "TOTAL"}
    for name in r:
        assert ["%.3e" % v for v in p[name]] == ["%.3e" % v for v in r[name]], name


@pytest.mark.skipif(not RefSolver.available(), reason="oracle/_ref not built")
@pytest.mark.parametrize("name", ["Orszag_Tang", "blastwave", "blastwave2", "Rotor", "FieldLoop", "KHInstability",
                                  "ShockCloud"])
def test_reference_test_problems_are_the_references_initial_data(name):
    """imex_b200.problems.reference_test restates the reference's own u_initialization and
    A_initial for its 2D catalogue: the same cell states, faces, boundary faces and A_z."""
    from imex_b200.problems import REFERENCE_TESTS, reference_test
    tid, _, _, xbc, ybc, _ = REFERENCE_TESTS[name]
    p = reference_test(name, 24, 20)
    ref = RefSolver(p.nx, p.ny, 2, dict(p.settings), (p.x0, p.x1, p.y0, p.y1))
    ref.set_bc(xbc, ybc)
    got = ref.init_test(tid)
    for k in ("prim", "bx", "by", "A"):
        np.testing.assert_array_equal(getattr(p, k), got[k], err_msg=k)
    if p.bx_x0 is not None:
        np.testing.assert_array_equal(p.bx_x0, got["bx_x0"])
        np.testing.assert_array_equal(p.by_y0, got["by_y0"])
