"""The reference's 2D test catalogue (Orszag-Tang, the two blast waves, the rotor, the field
loop, Kelvin-Helmholtz; imex_b200.problems.reference_test, pinned to the reference's own
initial data in test_oracle.py) run on the GPU for a few steps against the oracle, with the
reference's default solver settings and with EMF-consistent staggered CT."""
from __future__ import annotations

import numpy as np
import pytest

import imex_b200 as ix
from conftest import rel
from imex_b200.problems import reference_test
from oracle.bindings import make_solver

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", ["Orszag_Tang", "blastwave", "blastwave2", "Rotor", "FieldLoop", "KHInstability",
                                  "ShockCloud"])
@pytest.mark.parametrize("settings", [dict(), dict(magfield="StaggerCT", recon="VanLeer")], ids=["defaults", "ct"])
def test_reference_test_problem_steps_match_oracle(name, settings):
    prob = reference_test(name, 40, 36)
    cpu = make_solver("port", prob, 2, settings)
    gpu = ix.Solver.for_problem(prob, 2, settings)
    for _ in range(3):
        assert gpu.step() == pytest.approx(cpu.step(), rel=1e-12)
    a, b = gpu.cons(), cpu.cons()
    assert np.isfinite(a).all()
    for k in range(8):
        assert rel(a[k], b[k]) <= 1e-10, (k, rel(a[k], b[k]))
    if settings.get("magfield") == "StaggerCT":
        # CT keeps the initial face divergence: round-off of the field's size for every problem
        # but the field loop, whose faces are averages of a cell field that is not div-free
        scale = max(1.0, float(np.abs(b[5:7]).max()))
        g_div, c_div = gpu.divergence()["face_l2"], cpu.div_error()
        if c_div > 1e-9 * scale:
            assert g_div == pytest.approx(c_div, rel=1e-6)
        else:
            assert g_div <= 1e-11 * scale
    gpu.close()
