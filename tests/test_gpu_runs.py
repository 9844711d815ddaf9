"""Multi-step runs on the GPU: parity with the oracle at the per-field 1e-10 target,
and size-independent properties at the benchmark sizes (div B at round-off,
p > 0, mass conservation on the periodic domain, determinism)."""
from __future__ import annotations

import numpy as np
import pytest

import imex_b200 as ix
from conftest import rel
from imex_b200.problems import vortex, vortex_sheet
from oracle.bindings import make_solver

pytestmark = pytest.mark.gpu

CFG0 = dict(recon="VanLeer", magfield="StaggerCT", GMREStol=1e-12)
CFG1 = dict(recon="WENO5", magfield="PotentialA", p_floor=1e-8, theta=0.5, GMREStol=1e-12)


def test_config0_full_run_to_t1_matches_oracle():
    """Smooth MHD vortex 64^2 on [-5,5]^2, RK2, VanLeer, staggered CT, to t = 1."""
    prob = vortex(64)
    settings = dict(CFG0, time_stop=1.0)
    gpu = ix.Solver.for_problem(prob, 2, settings)
    cpu = make_solver("port", prob, 2, settings)
    steps = 0
    while True:
        dg, dc = gpu.step(), cpu.step()
        steps += 1
        assert dg == pytest.approx(dc, rel=1e-12)
        assert gpu.divergence()["face_l2"] <= 1e-12
        assert gpu.min_pressure() > 0.0
        if gpu.scalars()["t"] >= 1.0 - 1e-12:
            break
        assert steps < 100
    assert cpu.scalars()["t"] == pytest.approx(1.0, abs=1e-12)
    a, b = gpu.cons(), cpu.cons()
    for k in range(8):
        assert rel(a[k], b[k]) <= 1e-10, k
    bxg, byg = gpu.faces()
    bxc, byc = cpu.faces()
    assert rel(bxg, bxc) <= 1e-10 and rel(byg, byc) <= 1e-10
    gpu.close()


def test_config1_physics_multistep_matches_oracle():
    """Vortex sheet (config-1 physics) at 64^2 for 12 RK3 steps."""
    prob = vortex_sheet(64)
    gpu = ix.Solver.for_problem(prob, 3, CFG1)
    cpu = make_solver("port", prob, 3, CFG1)
    for _ in range(12):
        gpu.step()
        cpu.step()
        d = gpu.divergence()
        assert d["cell_wrapped_l2"] <= 1e-12
        assert gpu.min_pressure() > 0.0
    a, b = gpu.cons(), cpu.cons()
    for k in range(8):
        assert rel(a[k], b[k]) <= 1e-10, k
    assert rel(gpu.vector_potential(), cpu.vector_potential()) <= 1e-10
    gpu.close()


def test_odd_rectangular_grid_matches_oracle():
    prob = vortex(17, 23)
    settings = dict(recon="WENO5", magfield="StaggerCT")
    gpu = ix.Solver.for_problem(prob, 2, settings)
    cpu = make_solver("port", prob, 2, settings)
    for _ in range(3):
        gpu.step()
        cpu.step()
    a, b = gpu.cons(), cpu.cons()
    for k in range(8):
        assert rel(a[k], b[k]) <= 1e-12, k
    gpu.close()


def test_benchmark_size_properties():
    """Config-1 workload at its full 1024^2: div B, positivity, mass, determinism."""
    prob = vortex_sheet(1024)
    settings = dict(CFG1, GMREStol=1e-14)
    runs = []
    for _ in range(2):
        gpu = ix.Solver.for_problem(prob, 3, settings)
        mass0 = gpu.cons()[0].sum()
        for _ in range(2):
            gpu.step()
            assert gpu.divergence()["cell_wrapped_l2"] <= 1e-12
            assert gpu.min_pressure() > 0.0
        cons = gpu.cons()
        assert abs(cons[0].sum() - mass0) / mass0 <= 1e-13
        runs.append(cons)
        gpu.close()
    np.testing.assert_array_equal(runs[0], runs[1])


def test_staggered_ct_keeps_face_divergence_at_roundoff_large():
    prob = vortex(512)
    gpu = ix.Solver.for_problem(prob, 2, CFG0)
    for _ in range(3):
        gpu.step()
        assert gpu.divergence()["face_l2"] <= 1e-12
        assert gpu.min_pressure() > 0.0
    gpu.close()


def test_random_field_redlich_kwong_matches_oracle():
    """Seeded low-Mach random field (Redlich-Kwong gas, beta 0.1) at 48^2, RK2.

    Before each step the GPU gets the oracle's state (the primitive state a reference step
    starts from, main.cpp:356-358), so the comparison after the step is the error of that
    one step.  On this field the reference's own result moves by ~5e-10 over 5 steps when
    only its GMRES tolerance changes (1e-14 -> 1e-16, see test_oracle.py), so two correct
    implementations that sum in different orders differ at that level: each step is held
    to 1e-9 and the free-running comparison after 6 steps to 5e-9."""
    from imex_b200.problems import random_field
    prob = random_field(48)
    settings = dict(recon="Minmod", magfield="StaggerCT", eos_type="REDLICH_KWONG", m_alfa=0.4275, m_b=0.0866)
    gpu = ix.Solver.for_problem(prob, 2, settings)
    free = ix.Solver.for_problem(prob, 2, settings)
    cpu = make_solver("port", prob, 2, settings)
    for _ in range(6):
        bx, by = cpu.faces()
        gpu.upload_state(cpu.prim(), bx, by, cpu.vector_potential())
        dt_c = cpu.step()
        assert gpu.step() == pytest.approx(dt_c, rel=1e-12)
        free.step()
        a, b = gpu.cons(), cpu.cons()
        for k in range(8):
            assert rel(a[k], b[k]) <= 1e-9, k
        assert gpu.divergence()["face_l2"] <= 1e-12
        assert gpu.min_pressure() > 0.0
    a, b = free.cons(), cpu.cons()
    for k in range(8):
        assert rel(a[k], b[k]) <= 5e-9, k
    gpu.close()
    free.close()
