"""The discrete adjoint (imex_adjoint_run / imex_adjoint_vjp) against central finite
differences of the same GPU forward map.

J = 1/2 |rho(T) - rho_t|^2 + 1/2 |B(T) - B_t|^2 after a few fixed-dt steps; the gradient
with respect to the initial primitive planes and face fields, contracted with a smooth
random direction, must match (J(x + eps d) - J(x - eps d)) / (2 eps) to 1e-6 relative.

The reconstruction limiters are not differentiable where a variable's slopes vanish
(uniform planes), so the directions leave the planes that are uniform in the vortex
(v_z, B_z) untouched and the base density is made non-uniform first.
"""
from __future__ import annotations

import types

import numpy as np
import pytest

import imex_b200 as ix
from imex_b200.problems import vortex

pytestmark = pytest.mark.gpu

CFG = dict(recon="VanLeer", magfield="StaggerCT", GMREStol=1e-14, fixed_dt=0.05)


def _smooth(rng, ny, nx, modes=3):
    y, x = np.mgrid[0:ny, 0:nx]
    f = np.zeros((ny, nx))
    for _ in range(modes):
        kx, ky = rng.integers(1, 3, size=2)
        f += rng.standard_normal() * np.cos(2 * np.pi * (kx * x / nx + ky * y / ny) + rng.uniform(0, 2 * np.pi))
    return f / np.abs(f).max()


def _base(n=24, seed=3):
    p = vortex(n)
    rng = np.random.default_rng(seed)
    prim = p.prim.copy()
    prim[0] *= 1.0 + 0.05 * _smooth(rng, p.ny, p.nx)
    return types.SimpleNamespace(**{**vars(p), "prim": prim})


def _direction(prob, seed=7, planes=(0, 1, 2, 4, 5, 6), faces=True):
    rng = np.random.default_rng(seed)
    dprim = np.zeros_like(prob.prim)
    for k in planes:
        dprim[k] = _smooth(rng, prob.ny, prob.nx) * (0.05 * np.abs(prob.prim[k]).max() + 0.01)
    dbx = _smooth(rng, prob.ny, prob.nx) * 0.01 if faces else np.zeros_like(prob.bx)
    dby = _smooth(rng, prob.ny, prob.nx) * 0.01 if faces else np.zeros_like(prob.by)
    return dprim, dbx, dby


def _targets(prob, rks, settings, steps):
    sv = ix.Solver.for_problem(prob, rks, settings)
    for _ in range(steps):
        sv.step()
    c = sv.cons()
    sv.close()
    rng = np.random.default_rng(11)
    rho_t = c[0] * (1.0 + 1e-2 * _smooth(rng, prob.ny, prob.nx))
    B_t = c[5:8] + 1e-2 * np.stack([_smooth(rng, prob.ny, prob.nx) for _ in range(3)])
    return rho_t, B_t


def _J(prob, rks, settings, steps, rho_t, B_t, prim, bx, by):
    p = types.SimpleNamespace(**{**vars(prob), "prim": prim, "bx": bx, "by": by})
    sv = ix.Solver.for_problem(p, rks, settings)
    for _ in range(steps):
        sv.step()
    c = sv.cons()
    sv.close()
    return 0.5 * np.sum((c[0] - rho_t) ** 2) + 0.5 * np.sum((c[5:8] - B_t) ** 2)


def _fd_check(prob, rks, settings, steps, ckpt, eps=1e-6, tol=1e-6, **dkw):
    # targets from a nearby run so that the cotangent is not small
    shifted = types.SimpleNamespace(**{**vars(prob), "prim": prob.prim * (1 + 1e-3)})
    rho_t, B_t = _targets(shifted, rks, settings, steps)
    sv = ix.Solver.for_problem(prob, rks, settings)
    J, gp, gx, gy = sv.adjoint_run(steps, rho_t, B_t, checkpoint_every=ckpt)
    sv.close()
    J0 = _J(prob, rks, settings, steps, rho_t, B_t, prob.prim, prob.bx, prob.by)
    assert J == pytest.approx(J0, rel=1e-12)
    dprim, dbx, dby = _direction(prob, **dkw)
    pred = float(np.sum(gp * dprim) + np.sum(gx * dbx) + np.sum(gy * dby))
    Jp = _J(prob, rks, settings, steps, rho_t, B_t, prob.prim + eps * dprim, prob.bx + eps * dbx, prob.by + eps * dby)
    Jm = _J(prob, rks, settings, steps, rho_t, B_t, prob.prim - eps * dprim, prob.bx - eps * dbx, prob.by - eps * dby)
    fd = (Jp - Jm) / (2 * eps)
    print(f"J={J:.6e} adjoint={pred:.12e} fd={fd:.12e} rel={abs(pred - fd) / abs(fd):.2e}")
    assert abs(pred - fd) <= tol * abs(fd)
    return gp, gx, gy


def test_adjoint_matches_finite_differences_rk2():
    _fd_check(_base(24), 2, CFG, steps=3, ckpt=2)


@pytest.mark.parametrize("planes,faces", [((0,), False), ((1, 2), False), ((4,), False), ((5, 6), False), ((), True)],
                         ids=["rho", "velocity", "pressure", "cellB", "faces"])
def test_adjoint_each_field_matches_finite_differences(planes, faces):
    _fd_check(_base(20, seed=5), 2, CFG, steps=2, ckpt=1, planes=planes, faces=faces)


def test_adjoint_rk3_floor_off_minmod():
    cfg = dict(CFG, recon="Minmod", floor_on=0, PressureSolver="once_correction")
    _fd_check(_base(20, seed=9), 3, cfg, steps=2, ckpt=1)


def _generic(n=20, seed=19):
    """The vortex with each non-uniform primitive plane perturbed by a smooth random field.
    PrimState reconstructs v, p and B themselves, and their vortex profiles have exactly
    equal neighbours on the symmetry lines, where the limiters have a kink (zero slope)."""
    p = vortex(n)
    rng = np.random.default_rng(seed)
    prim = p.prim.copy()
    for k in (0, 1, 2, 4, 5, 6):
        prim[k] = prim[k] + 0.02 * np.abs(prim[k]).max() * _smooth(rng, p.ny, p.nx)
    return types.SimpleNamespace(**{**vars(p), "prim": prim})


@pytest.mark.parametrize("rks,extra", [(2, dict(recon="VanLeer")), (3, dict(recon="WENO5"))],
                         ids=["vanleer_rk2", "weno5_rk3"])
def test_adjoint_prim_state_reconstruction(rks, extra):
    """PrimState: each face state is pri2con of the reconstructed primitive variables
    (reconstruction.cpp:272-281), so the reconstruction's adjoint couples all 8 planes."""
    _fd_check(_generic(20), rks, dict(CFG, reconstate="PrimState", **extra), steps=2, ckpt=1)


def test_adjoint_conservation_of_u():
    """ConservationofU (imex_subsystems.cpp:303-392): the energy is advanced by the central
    flux of the enthalpy at the final pressure instead of being redefined from it."""
    _fd_check(_base(20, seed=23), 2, dict(CFG, U_update="ConservationofU"), steps=2, ckpt=1)


def test_adjoint_energy_modify():
    """Energy_Modify (main.cpp:528-534): E += (|B_CT|^2 - |B_saved|^2) / 2 before the stage
    derivative, with B_saved the cell B after the magnetic sub-system."""
    _fd_check(_base(20, seed=29), 2, dict(CFG, Energy_Modify=1), steps=2, ckpt=1)


def test_adjoint_alfven_speed_pressure_viscosity():
    """AlfvenSpeedp: the pressure operator's viscosity scales with the step's Alfven maxima
    max Bx / sqrt(rho) and max By / sqrt(rho), whose adjoints go to the cells attaining them."""
    _fd_check(_base(20, seed=31), 2, dict(CFG, add_pvisc="AlfvenSpeedp"), steps=2, ckpt=1)


def test_adjoint_checkpointing_does_not_change_the_gradient():
    prob = _base(20, seed=13)
    rho_t, B_t = _targets(prob, 2, CFG, 4)
    rho_t = rho_t * 1.001
    outs = []
    for ckpt in (1, 3, 4):
        sv = ix.Solver.for_problem(prob, 2, CFG)
        outs.append(sv.adjoint_run(4, rho_t, B_t, checkpoint_every=ckpt))
        if ckpt == 1:
            # the context is left at the final state of the forward run
            ref = ix.Solver.for_problem(prob, 2, CFG)
            for _ in range(4):
                ref.step()
            np.testing.assert_array_equal(sv.cons(), ref.cons())
            ref.close()
        sv.close()
    for o in outs[1:]:
        assert o[0] == pytest.approx(outs[0][0], rel=1e-13)  # J is summed with atomics
        for a, b in zip(o[1:], outs[0][1:]):
            np.testing.assert_allclose(a, b, rtol=1e-10, atol=1e-14 * np.abs(b).max())


def test_adjoint_vjp_is_linear_in_the_cotangent():
    prob = _base(16, seed=17)
    rng = np.random.default_rng(1)
    l1 = rng.standard_normal((8, 16, 16))
    l2 = rng.standard_normal((8, 16, 16))
    g = []
    for lam in (l1, l2, 2.0 * l1 - 3.0 * l2):
        sv = ix.Solver.for_problem(prob, 2, CFG)
        g.append(sv.adjoint_vjp(2, lam, checkpoint_every=1))
        sv.close()
    for k in range(3):
        np.testing.assert_allclose(g[2][k], 2.0 * g[0][k] - 3.0 * g[1][k], rtol=1e-9,
                                   atol=1e-12 * np.abs(g[2][k]).max())


def test_adjoint_rejects_unsupported_configurations():
    prob = vortex(16)
    for extra in (dict(fixed_dt=0.0), dict(magfield="PotentialA"), dict(magfield="UnStaggerCT"),
                  dict(eos_type="REDLICH_KWONG"), dict(GLF=0), dict(precision="mixed")):
        sv = ix.Solver.for_problem(prob, 2, dict(CFG, **extra))
        with pytest.raises(ix.ImexError) as err:
            sv.adjoint_run(1, prob.prim[0], prob.prim[5:8])
        assert err.value.status == 2
        sv.close()
