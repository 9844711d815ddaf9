"""The mixed-precision form: FP32 operator applications and Krylov vectors inside
FP64 iterative refinement (GMRES) or inside the FP64 nested Newton.  Every result
is compared with the FP64 oracle on the same inputs: relative L2 per field per
step <= 1e-8, the face divergence of B at round-off (<= 1e-12, the CT update
stays FP64) and p > 0."""
from __future__ import annotations

import numpy as np
import pytest

import imex_b200 as ix
from conftest import rel
from imex_b200.problems import random_field, vortex, vortex_sheet
from oracle.bindings import make_solver

pytestmark = pytest.mark.gpu

TOL = 1e-8  # relative L2 per field per step against the FP64 oracle
PRESSURE, MAGNETIC = 1, 2  # IMEX_MIXED_PRESSURE, IMEX_MIXED_MAGNETIC
CASES = [
    # name, problem, RK stages, settings, steps
    ("vortex_cfg0", lambda: vortex(48), 2, dict(recon="VanLeer", magfield="StaggerCT", GMREStol=1e-12), 6),
    ("sheet_cfg1", lambda: vortex_sheet(48), 3,
     dict(recon="WENO5", magfield="PotentialA", p_floor=1e-8, theta=0.5, GMREStol=1e-12), 4),
    ("vortex_nofloor", lambda: vortex(40, 36), 2, dict(recon="Minmod", magfield="UnStaggerCT", floor_on=0), 4),
    ("vortex_rkeos", lambda: vortex(32), 2,
     dict(recon="VanLeer", magfield="StaggerCT", eos_type="REDLICH_KWONG", m_alfa=0.4275, m_b=0.0866), 3),
    ("random_field", lambda: random_field(48), 2,
     dict(recon="Minmod", magfield="StaggerCT", eos_type="REDLICH_KWONG", m_alfa=0.4275, m_b=0.0866), 4),
    ("vortex_energy", lambda: vortex(48), 2,
     dict(recon="VanLeer", magfield="StaggerCT", formula="EnergyFormula", GMREStol=1e-12), 5),
    ("vortex_local_lf", lambda: vortex(48), 2,
     dict(recon="VanLeer", magfield="StaggerCT", GLF=0, add_pvisc="AlfvenSpeedp", GMREStol=1e-12), 4),
    ("sheet_local_lf", lambda: vortex_sheet(48), 3,
     dict(recon="WENO5", magfield="PotentialA", p_floor=1e-8, theta=0.5, GLF=0, GMREStol=1e-12), 3),
]


@pytest.mark.parametrize("scope", [PRESSURE, PRESSURE | MAGNETIC], ids=["pressure", "all"])
@pytest.mark.parametrize("name,factory,rks,settings,steps", CASES, ids=[c[0] for c in CASES])
def test_mixed_steps_match_fp64_oracle(name, factory, rks, settings, steps, scope):
    prob = factory()
    gpu = ix.Solver.for_problem(prob, rks, dict(settings, precision="mixed", mixed_solves=scope))
    cpu = make_solver("port", prob, rks, settings)
    worst = 0.0
    for _ in range(steps):
        dg, dc = gpu.step(), cpu.step()
        assert dg == pytest.approx(dc, rel=1e-8)
        a, b = gpu.cons(), cpu.cons()
        for k in range(8):
            e = rel(a[k], b[k])
            worst = max(worst, e)
            assert e <= TOL, (k, e)
        if settings["magfield"] == "StaggerCT":
            assert gpu.divergence()["face_l2"] <= 1e-12
        else:
            assert gpu.divergence()["cell_wrapped_l2"] <= 1e-12
        assert gpu.min_pressure() > 0.0
    if scope & MAGNETIC:
        assert gpu.stats()["refine_sweeps"] > 0  # the magnetic solves refine around FP32 cycles
    print(f"{name} scope={scope}: worst relative L2 vs FP64 oracle over {steps} steps = {worst:.2e}")
    gpu.close()


@pytest.mark.parametrize("op,settings", [
    ("magnetic_B", dict(recon="VanLeer", magfield="StaggerCT")),
    ("magnetic_A", dict(recon="WENO5", magfield="PotentialA", p_floor=1e-8, theta=0.5)),
    ("pressure_L", dict(recon="VanLeer", magfield="StaggerCT")),
])
def test_mixed_gmres_matches_fp64_solve(op, settings):
    """imex_gmres in the mixed form converges to the FP64 solve's tolerance."""
    prob = vortex(64) if op != "magnetic_A" else vortex_sheet(64)
    rks = 2 if op != "magnetic_A" else 3
    sols = []
    for prec in ("fp64", "mixed"):
        sv = ix.Solver.for_problem(prob, rks, dict(settings, precision=prec, GMREStol=1e-13,
                                                   mixed_solves=PRESSURE | MAGNETIC))
        sv.step()
        sv.prepare_operator(op, sv.scalars()["dt"] * 0.5)
        n = sv.nx * sv.ny * (3 if op.startswith("magnetic") else 1)
        b = sv.apply_operator(op, np.random.default_rng(3).standard_normal(n))
        x, st = sv.gmres(op, np.zeros(n), b)
        if prec == "mixed":
            assert st["refine_sweeps"] >= 1
        sols.append(x)
        sv.close()
    assert rel(sols[1], sols[0]) <= 1e-10
