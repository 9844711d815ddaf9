"""The energy formula (formula = EnergyFormula): Energy_flux_Update followed by
PreSubsystem_Energy, one preconditioned GMRES on the total energy E per stage with
the momentum corrected by -h (g-1) grad E (main.cpp:469-485).  Multi-step runs
against the FP64 oracle at the per-field 1e-10 target, with div B at round-off
and p > 0; the batched form against single runs."""
from __future__ import annotations

import numpy as np
import pytest

import imex_b200 as ix
from conftest import rel
from imex_b200.problems import vortex, vortex_sheet
from oracle.bindings import make_solver

pytestmark = pytest.mark.gpu

ECFG0 = dict(recon="VanLeer", magfield="StaggerCT", GMREStol=1e-12, formula="EnergyFormula")
ECFG1 = dict(recon="WENO5", magfield="PotentialA", p_floor=1e-8, theta=0.5, GMREStol=1e-12,
             formula="EnergyFormula")

RUNS = [
    ("vortex_stagger", lambda: vortex(64), 2, ECFG0, 10),
    ("sheet_potential", lambda: vortex_sheet(64), 3, ECFG1, 6),
    ("vortex_unstagger_rk1", lambda: vortex(48, 40), 1,
     dict(recon="Minmod", magfield="UnStaggerCT", formula="EnergyFormula"), 6),
]


@pytest.mark.parametrize("name,factory,rks,settings,steps", RUNS, ids=[r[0] for r in RUNS])
def test_energy_formula_runs_match_oracle(name, factory, rks, settings, steps):
    prob = factory()
    gpu = ix.Solver.for_problem(prob, rks, settings)
    cpu = make_solver("port", prob, rks, settings)
    for s in range(steps):
        assert gpu.step() == pytest.approx(cpu.step(), rel=1e-12)
        a, b = gpu.cons(), cpu.cons()
        for k in range(8):
            assert rel(a[k], b[k]) <= 1e-10, (s, k, rel(a[k], b[k]))
        d = gpu.divergence()
        assert min(d["face_l2"], d["cell_wrapped_l2"]) <= 1e-12
        assert gpu.min_pressure() > 0.0
    st = gpu.stats()
    assert st["gmres_solves"] > 0
    gpu.close()


def test_energy_solve_reports_its_profile_family():
    prob = vortex(64)
    gpu = ix.Solver.for_problem(prob, 2, ECFG0)
    gpu.profile_enable(True)
    gpu.step()
    fams = {f["name"]: f for f in gpu.profile()}
    assert fams["gmres_energy"]["launches"] == 2  # one energy solve per stage
    assert "nested_newton" not in fams or fams["nested_newton"]["launches"] == 0
    gpu.close()


def test_energy_formula_batch_matches_single_runs():
    probs = [vortex(24, kappa=0.7, mu=1.2), vortex(40, kappa=1.3, mu=0.6), vortex(48, 36, kappa=1.1, mu=0.8)]
    batch = ix.Batch(probs, 2, ECFG0)
    batch.step(3)
    for m, p in enumerate(probs):
        single = ix.Solver.for_problem(p, 2, ECFG0)
        cpu = make_solver("port", p, 2, ECFG0)
        for _ in range(3):
            single.step()
            cpu.step()
        a, b, c = batch.members[m].cons(), single.cons(), cpu.cons()
        for k in range(8):
            assert rel(a[k], b[k]) <= 1e-11, (m, k)
            assert rel(a[k], c[k]) <= 1e-10, (m, k)
        single.close()
    batch.close()
