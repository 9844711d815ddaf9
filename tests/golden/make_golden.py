"""Generate the golden fixtures of tests/golden from the reference solver itself.

The reference has no tests or known-answer vectors of its own, so the fixtures
are outputs of the reference's own code (oracle/_ref/libimexref.so, built from
the reference sources by `make -C oracle ref`) on small analytic inputs:

  step_<case>.npz  - initial data + state after a few full time steps
                     (main.cpp:335-561) and the dt of each step; the open-blast
                     cases run x_Transmissive / y_Transmissive and also store the
                     boundary normal faces (Bx at x_0, By at y_0);
  fn_<case>.npz    - single reference functions on fixed inputs:
                     TVDReconstruction, ShockDetector and the four matrix-free
                     operators of implicit_operators.cpp (fn_local_*: the operators
                     with the local dissipation, on the same inputs);
  adjoint_ref_fd64.npz - central finite differences of the reference's J on the
                     adjoint workload at 64 x 64 (50 steps, all 32 amplitudes).

Run from the repository root:  python tests/golden/make_golden.py [case ...]
(no arguments: every case; otherwise only the named step cases and/or "fn", "fn_local",
"adjoint_fd").
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from imex_b200.problems import open_blast, vortex, vortex_sheet  # noqa: E402
from oracle.bindings import RefSolver, make_solver  # noqa: E402

CFG0 = dict(recon="VanLeer", magfield="StaggerCT", GMREStol=1e-12)
CFG1 = dict(recon="WENO5", magfield="PotentialA", p_floor=1e-8, theta=0.5, GMREStol=1e-12)
STEP_CASES = {
    # name: (problem factory, RK stages, settings, steps)
    "vortex16_cfg0": (lambda: vortex(16), 2, CFG0, 3),
    "sheet16_cfg1": (lambda: vortex_sheet(16), 3, CFG1, 2),
    "vortex12x10_minmod_unstag": (lambda: vortex(12, 10), 2, dict(recon="Minmod", magfield="UnStaggerCT"), 2),
    "vortex16_eno3_nodivfree_rk1": (lambda: vortex(16), 1, dict(recon="ENO3", magfield="NoDivFree"), 2),
    "vortex16_norecon_nofloor_rk3": (lambda: vortex(16), 3,
                                     dict(recon="NoRecon", magfield="StaggerCT", floor_on=0), 2),
    "vortex16_primstate": (lambda: vortex(16), 2,
                           dict(recon="VanLeer", magfield="StaggerCT", reconstate="PrimState"), 2),
    "vortex16_rkeos": (lambda: vortex(16), 2,
                       dict(recon="VanLeer", magfield="StaggerCT", eos_type="REDLICH_KWONG",
                            m_alfa=0.4275, m_b=0.0866), 1),
    "vortex16_energy_modify": (lambda: vortex(16), 2,
                               dict(recon="WENO5", magfield="StaggerCT", Energy_modify=1), 1),
    # the energy formula: Energy_flux_Update + PreSubsystem_Energy (main.cpp:469-485)
    "vortex16_energyformula": (lambda: vortex(16), 2, dict(CFG0, formula="EnergyFormula"), 2),
    "sheet16_energyformula_rk3": (lambda: vortex_sheet(16), 3, dict(CFG1, formula="EnergyFormula"), 1),
    "vortex14x12_energyformula_unstag_rk1": (lambda: vortex(14, 12), 1,
                                             dict(recon="Minmod", magfield="UnStaggerCT",
                                                  formula="EnergyFormula"), 2),
    # transmissive boundaries (open_blast sets x_Transmissive / y_Transmissive)
    "blast16x14_minmod_open": (lambda: open_blast(16, 14), 2, dict(recon="Minmod", magfield="StaggerCT"), 3),
    "blast16_weno5_open_rk3": (lambda: open_blast(16), 3,
                               dict(recon="WENO5", magfield="StaggerCT", p_floor=1e-8), 2),
    "blast14x12_eno3_nodivfree_open": (lambda: open_blast(14, 12), 2, dict(recon="ENO3", magfield="NoDivFree"), 2),
    "blast16_primstate_rkeos_open": (lambda: open_blast(16), 2,
                                     dict(recon="VanLeer", reconstate="PrimState", magfield="StaggerCT",
                                          eos_type="REDLICH_KWONG", m_alfa=0.05, m_b=0.1), 2),
    "blast16_energyformula_open": (lambda: open_blast(16), 2,
                                   dict(recon="Minmod", magfield="StaggerCT", formula="EnergyFormula",
                                        GMREStol=1e-12), 2),
    "blast16_potentialA_weno5_open_rk3": (lambda: open_blast(16), 3,
                                          dict(recon="WENO5", magfield="PotentialA", p_floor=1e-8, theta=0.5), 2),
    "blast14x12_unstag_minmod_open": (lambda: open_blast(14, 12), 2, dict(recon="Minmod", magfield="UnStaggerCT"), 2),
    "blast16x12_xperiodic_open_y": (lambda: open_blast(16, 12), 2,
                                    dict(recon="VanLeer", magfield="StaggerCT", x_bc="x_Periodic",
                                         floor_on=0, PressureSolver="once_correction"), 2),
    # ConservationofU: E advanced by the enthalpy flux of the corrected momentum (imex_subsystems.cpp:303-392)
    "vortex16_conservationofU": (lambda: vortex(16), 2, dict(CFG0, U_update="ConservationofU"), 2),
    "blast16_conservationofU_open": (lambda: open_blast(16), 2,
                                     dict(recon="Minmod", magfield="StaggerCT", U_update="ConservationofU"), 2),
    "vortex16_conservationofU_rkeos": (lambda: vortex(16), 2,
                                       dict(recon="VanLeer", magfield="StaggerCT", U_update="ConservationofU",
                                            eos_type="REDLICH_KWONG", m_alfa=0.4275, m_b=0.0866), 1),
    # local Lax-Friedrichs dissipation (GLF = false): face speeds from the neighbouring cells in the
    # explicit fluxes (flux.cpp:108-389), the magnetic and pressure viscosities
    # (implicit_operators.cpp:311-353, 472-490, 584-607) and CollectMagFluxes (ct_flux.cpp:79-124)
    "vortex16_local_lf": (lambda: vortex(16), 2, dict(CFG0, GLF=0), 2),
    "sheet16_potentialA_local_lf_rk3": (lambda: vortex_sheet(16), 3, dict(CFG1, GLF=0, add_bvisc=1), 2),
    "blast16_local_lf_alfven_open": (lambda: open_blast(16), 2,
                                     dict(recon="Minmod", magfield="StaggerCT", GLF=0, add_pvisc="AlfvenSpeedp"), 2),
    "blast16x14_potentialA_local_lf_open": (lambda: open_blast(16, 14), 2,
                                            dict(recon="VanLeer", magfield="PotentialA", GLF=0, p_floor=1e-8,
                                                 theta=0.5), 2),
    "vortex14x12_unstag_energyformula_local_lf": (lambda: vortex(14, 12), 2,
                                                  dict(recon="Minmod", magfield="UnStaggerCT", GLF=0,
                                                       formula="EnergyFormula"), 2),
    "vortex16_local_lf_rkeos_conservationofU": (lambda: vortex(16), 2,
                                                dict(recon="VanLeer", magfield="StaggerCT", GLF=0,
                                                     U_update="ConservationofU", eos_type="REDLICH_KWONG",
                                                     m_alfa=0.4275, m_b=0.0866), 1),
}


def step_case(name: str, factory, rks: int, settings: dict, steps: int) -> None:
    prob = factory()
    ref = make_solver("ref", prob, rks, settings)
    dts, cons, faces_x, faces_y, As, lines_x, lines_y = [], [], [], [], [], [], []
    for _ in range(steps):
        dts.append(ref.step())
        cons.append(ref.cons())
        bx, by = ref.faces()
        faces_x.append(bx)
        faces_y.append(by)
        As.append(ref.vector_potential())
        bxb, byb = ref.boundary_faces()
        lines_x.append(bxb)
        lines_y.append(byb)
    extra = {}
    if prob.bx_x0 is not None:
        extra = dict(bx_x00=prob.bx_x0, by_y00=prob.by_y0, bx_x0=np.array(lines_x), by_y0=np.array(lines_y))
    np.savez_compressed(
        os.path.join(HERE, f"step_{name}.npz"),
        prim0=prob.prim, bx0=prob.bx, by0=prob.by, A0=prob.A, rks=rks,
        domain=np.array([prob.x0, prob.x1, prob.y0, prob.y1]),
        settings=np.array(repr(dict(prob.settings, **settings))),
        dt=np.array(dts), cons=np.array(cons), bx=np.array(faces_x), by=np.array(faces_y),
        A=np.array(As), div=np.array(ref.div_error()), **extra)


def fn_case() -> None:
    """Single functions on a perturbed vortex state (16 x 12 grid)."""
    prob = vortex(16, 12)
    rng = np.random.default_rng(20261203)
    base = make_solver("ref", prob, 2, CFG0)
    Q = base.cons()
    Qp = Q * (1.0 + 1e-3 * rng.standard_normal(Q.shape))
    ucon = Q * (1.0 + 1e-3 * rng.standard_normal(Q.shape))
    h = 0.013
    out = dict(Q=Qp, ucon=ucon, Qs=Q, h=h)
    for scheme in ("NoRecon", "Minmod", "VanLeer", "ENO3", "WENO5"):
        s = make_solver("ref", prob, 2, dict(recon=scheme, magfield="StaggerCT"))
        out[f"recon_{scheme}"] = s.reconstruct(Qp)
    s = make_solver("ref", prob, 2, dict(recon="Minmod", reconstate="PrimState", magfield="StaggerCT"))
    out["recon_Minmod_prim"] = s.reconstruct(Qp)
    s = make_solver("ref", prob, 2, CFG0)
    out["shock"] = s.shock(Qp)
    N = prob.nx * prob.ny
    x1 = rng.standard_normal(N)
    x3 = rng.standard_normal(3 * N)
    pf = np.abs(rng.standard_normal(N)) * 2e-7
    s.set_scalars(0.02, h, 1.3, 1.1, 0.9, 0.8, 1.5)
    out.update(x1=x1, x3=x3, pfreeze=pf, mbig=1.5e6,
               scalars=np.array([0.02, h, 1.3, 1.1, 0.9, 0.8, 1.5]))
    out["op_pressure_L"] = s.operator(0, ucon, Qp, Q, h, x1)
    out["op_pressure_J"] = s.operator(1, ucon, Qp, Q, h, x1, pfreeze=pf, mbig=1.5e6)
    out["op_magnetic_B"] = s.operator(2, ucon, Qp, Q, h, x3)
    out["op_energy"] = s.operator(4, ucon, Qp, Q, h, x1)
    sa = make_solver("ref", prob, 2, dict(CFG1))
    sa.set_scalars(0.02, h, 1.3, 1.1, 0.9, 0.8, 1.5)
    out["op_magnetic_A"] = sa.operator(3, ucon, Qp, Q, h, x3)
    np.savez_compressed(os.path.join(HERE, "fn_vortex16x12.npz"), **out)


ADJ_SETTINGS = dict(recon="VanLeer", magfield="StaggerCT", GMREStol=1e-14, fixed_dt=0.02)
ADJ_N, ADJ_STEPS, ADJ_H = 64, 50, 1e-6


def fn_local_case() -> None:
    """The matrix-free operators with the local dissipation (GLF = false) on the inputs of
    fn_vortex16x12.npz (implicit_operators.cpp:311-353, 472-490, 584-607)."""
    g = dict(np.load(os.path.join(HERE, "fn_vortex16x12.npz")))
    prob = vortex(16, 12)
    args = (g["ucon"], g["Q"], g["Qs"], float(g["h"]))
    out = {}
    for name, settings in (("", {}), ("_alfven", dict(add_pvisc="AlfvenSpeedp"))):
        s = make_solver("ref", prob, 2, dict(CFG0, GLF=0, **settings))
        s.set_scalars(*(float(v) for v in g["scalars"]))
        out[f"op_pressure_L{name}"] = s.operator(0, *args, g["x1"])
        out[f"op_pressure_J{name}"] = s.operator(1, *args, g["x1"], pfreeze=g["pfreeze"], mbig=float(g["mbig"]))
    out["op_magnetic_B"] = s.operator(2, *args, g["x3"])
    sa = make_solver("ref", prob, 2, dict(CFG1, GLF=0))
    sa.set_scalars(*(float(v) for v in g["scalars"]))
    out["op_magnetic_A"] = sa.operator(3, *args, g["x3"])
    np.savez_compressed(os.path.join(HERE, "fn_local_vortex16x12.npz"), **out)


def _adj_J(args):
    """J of the reference solver on the perturbed vortex with amplitudes a (one process each)."""
    a, rho_t, B_t = args
    from imex_b200.problems import perturbed_vortex
    pv = perturbed_vortex(ADJ_N)
    r = make_solver("ref", pv.problem(a), 2, ADJ_SETTINGS)
    for _ in range(ADJ_STEPS):
        r.step()
    c = r.cons()
    return 0.5 * np.sum((c[0] - rho_t) ** 2) + 0.5 * np.sum((c[5:8] - B_t) ** 2)


def adjoint_fd_case() -> None:
    """The adjoint workload's check at 64 x 64: central differences (h = 1e-6) of the reference's
    own FP64 J over 50 fixed-dt steps, for all 32 amplitudes, with the targets from the
    reference's unperturbed run."""
    import multiprocessing as mp
    from imex_b200.problems import perturbed_vortex
    pv = perturbed_vortex(ADJ_N)
    base = make_solver("ref", pv.base, 2, ADJ_SETTINGS)
    for _ in range(ADJ_STEPS):
        base.step()
    c = base.cons()
    rho_t, B_t = c[0], c[5:8]
    a0 = np.array(pv.amplitudes)
    jobs = [(a0, rho_t, B_t)]
    for m in range(len(a0)):
        for sgn in (1.0, -1.0):
            a = a0.copy()
            a[m] += sgn * ADJ_H
            jobs.append((a, rho_t, B_t))
    with mp.get_context("spawn").Pool(min(8, os.cpu_count() or 1)) as pool:
        Js = pool.map(_adj_J, jobs)
    fd = np.array([(Js[1 + 2 * m] - Js[2 + 2 * m]) / (2 * ADJ_H) for m in range(len(a0))])
    np.savez_compressed(os.path.join(HERE, "adjoint_ref_fd64.npz"), amplitudes=a0, J=np.array(Js[0]),
                        fd=fd, rho_t=rho_t, B_t=B_t, nsteps=ADJ_STEPS, h=ADJ_H,
                        settings=np.array(repr(ADJ_SETTINGS)))


def main() -> None:
    if not RefSolver.available():
        raise SystemExit("oracle/_ref/libimexref.so missing: run `make -C oracle ref` first")
    only = set(sys.argv[1:])
    for name, (factory, rks, settings, steps) in STEP_CASES.items():
        if only and name not in only:
            continue
        step_case(name, factory, rks, settings, steps)
        print("wrote", name)
    if not only or "fn" in only:
        fn_case()
        print("wrote fn_vortex16x12")
    if not only or "fn" in only or "fn_local" in only:
        fn_local_case()
        print("wrote fn_local_vortex16x12")
    if not only or "adjoint_fd" in only:
        adjoint_fd_case()
        print("wrote adjoint_ref_fd64")


if __name__ == "__main__":
    main()
