"""Initial data: analytic fields with the properties the reference's set-up guarantees."""
from __future__ import annotations

import numpy as np
import pytest

from imex_b200.problems import vortex, vortex_sheet


def face_div(p):
    return (p.bx - np.roll(p.bx, 1, axis=1)) / p.dx + (p.by - np.roll(p.by, 1, axis=0)) / p.dy


def test_vortex_faces_are_divergence_free_and_cell_b_is_face_average():
    p = vortex(64)
    assert np.max(np.abs(face_div(p))) < 1e-13
    np.testing.assert_allclose(p.prim[5], 0.5 * (np.roll(p.bx, 1, axis=1) + p.bx), rtol=0, atol=0)
    assert p.prim[4].min() > 0.9 and np.allclose(p.prim[0], 1.0)
    # background flow (1, 1) plus the vortex
    assert abs(p.prim[1].mean() - 1.0) < 1e-3 and abs(p.prim[2].mean() - 1.0) < 1e-3


def test_vortex_kappa_mu_scale_the_perturbation():
    a, b = vortex(32, kappa=1.0, mu=1.0), vortex(32, kappa=0.5, mu=1.5)
    np.testing.assert_allclose(b.prim[1] - 1.0, 0.5 * (a.prim[1] - 1.0), rtol=1e-12, atol=1e-15)
    np.testing.assert_allclose(b.bx, 1.5 * a.bx, rtol=1e-12, atol=1e-15)


def test_vortex_sheet_fields():
    p = vortex_sheet(64)
    g = 5.0 / 3.0
    assert np.allclose(p.prim[0], g * g) and np.allclose(p.prim[4], g)
    assert abs(p.prim[1].mean()) < 1e-12 and abs(p.prim[5].mean()) < 1e-12
    # A_z = cos y + cos(2x)/2 reproduces B = (dAz/dy, -dAz/dx) = (-sin y, sin 2x) to O(dx^2)
    Az = p.A[2]
    bxc = (np.roll(Az, -1, axis=0) - np.roll(Az, 1, axis=0)) / (2 * p.dy)
    assert np.max(np.abs(bxc - p.prim[5])) < 1e-2


def test_rectangular_grids():
    p = vortex(17, 23)
    assert p.prim.shape == (8, 23, 17) and p.bx.shape == (23, 17)
    assert np.max(np.abs(face_div(p))) < 1e-12


def test_random_field_is_seeded_divergence_free_and_scaled():
    from imex_b200.problems import random_field
    a = random_field(64, seed=5)
    b = random_field(64, seed=5)
    c = random_field(64, seed=6)
    np.testing.assert_array_equal(a.prim, b.prim)
    assert not np.array_equal(a.prim, c.prim)
    h = 1.0 / 64
    div = (a.bx - np.roll(a.bx, 1, axis=1)) / h + (a.by - np.roll(a.by, 1, axis=0)) / h
    assert np.abs(div).max() <= 1e-12 * np.abs(a.bx).max() / h
    rho, p = a.prim[0], a.prim[4]
    assert abs(np.abs(rho - 1.0).max() - 0.1) < 1e-12
    assert abs(np.abs(p - 1.0).max() - 0.05) < 1e-12
    vmax = np.sqrt(a.prim[1] ** 2 + a.prim[2] ** 2).max()
    assert vmax == pytest.approx(1e-3 * np.sqrt(5.0 / 3.0), rel=1e-12)
    bmax2 = (a.prim[5] ** 2 + a.prim[6] ** 2).max()
    assert 2.0 / bmax2 == pytest.approx(0.1, rel=1e-12)
    assert a.settings["eos_type"] == "REDLICH_KWONG"
