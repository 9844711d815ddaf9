"""Ensembles (imex_batch): independent runs on uneven grids advanced together, with the
implicit solves of all members in one cooperative launch per solve and the step captured
in a CUDA graph.  Every member must match the same run done alone (its own context) and
the FP64 oracle; the batched solves only change how many CTAs each member's reductions
use, so members agree with their single runs to round-off."""
from __future__ import annotations

import numpy as np
import pytest

import imex_b200 as ix
from conftest import rel
from imex_b200.problems import vortex, vortex_ensemble, vortex_sheet
from oracle.bindings import make_solver

pytestmark = pytest.mark.gpu

CFG0 = dict(recon="VanLeer", magfield="StaggerCT", GMREStol=1e-12)


def _members():
    return [vortex(24, kappa=0.7, mu=1.2), vortex(40, kappa=1.3, mu=0.6), vortex(32, kappa=1.0, mu=1.0),
            vortex(64, kappa=0.9, mu=1.4), vortex(48, 36, kappa=1.1, mu=0.8)]


def _check_members(batch, probs, rks, settings, steps, tol_single, tol_oracle):
    for m, p in enumerate(probs):
        single = ix.Solver.for_problem(p, rks, settings)
        cpu = make_solver("port", p, rks, settings)
        for _ in range(steps):
            single.step()
            cpu.step()
        a, b, c = batch.members[m].cons(), single.cons(), cpu.cons()
        for k in range(8):
            assert rel(a[k], b[k]) <= tol_single, (m, k, rel(a[k], b[k]))
            assert rel(a[k], c[k]) <= tol_oracle, (m, k, rel(a[k], c[k]))
        single.close()


def test_batch_members_match_single_runs_and_oracle():
    probs = _members()
    batch = ix.Batch(probs, 2, CFG0)
    ms = batch.step(3)
    assert ms > 0.0
    info = batch.info()
    print("batch info:", info)
    assert info["solve_launches_per_step"] >= 2
    # one launch per explicit sub-step for all five members: far fewer than the members'
    # own launches (each member alone launches about 17 explicit kernels per RK2 step)
    assert info["streams"] == 0 and 0 < info["explicit_launches_per_step"] < 40
    for sv in batch.members:
        assert sv.divergence()["face_l2"] <= 1e-12
        assert sv.min_pressure() > 0.0
        assert sv.scalars()["timestep"] == 3
    _check_members(batch, probs, 2, CFG0, 3, 1e-11, 1e-10)
    batch.close()


def test_batch_local_dissipation_members_match_single_runs_and_oracle():
    """GLF = false: every member builds its own face viscosities before the batched solves."""
    probs = _members()[:3]
    settings = dict(CFG0, GLF=0, add_pvisc="AlfvenSpeedp")
    batch = ix.Batch(probs, 2, settings)
    batch.step(2)
    _check_members(batch, probs, 2, settings, 2, 1e-11, 1e-10)
    batch.close()


def test_batch_modes_agree():
    """Batched explicit launches (with and without the graph) and per-member launches on a
    pool of streams run the same kernel bodies on the same data: bit-identical members."""
    probs = _members()[:3]
    runs = [ix.Batch(probs, 2, CFG0, streams=0, graph=True), ix.Batch(probs, 2, CFG0, streams=0, graph=False),
            ix.Batch(probs, 2, CFG0, streams=3, graph=True), ix.Batch(probs, 2, CFG0, streams=2, graph=False)]
    for r in runs:
        r.step(2)
    assert not runs[1].info()["graph"] and not runs[3].info()["graph"]
    assert runs[2].info()["explicit_launches_per_step"] == -1
    for m in range(len(probs)):
        ref = runs[0].members[m].cons()
        for r in runs[1:]:
            c = r.members[m].cons()
            for k in range(8):
                assert np.array_equal(ref[k], c[k]), (m, k)
    for r in runs:
        r.close()


def test_batch_mixed_a_form_matches_fp64():
    """Vortex-sheet members (A form, floor on, RK3) in the mixed form against FP64 single runs."""
    probs = [vortex_sheet(32), vortex_sheet(48, 40), vortex_sheet(64)]
    cfg = dict(recon="WENO5", magfield="PotentialA", p_floor=1e-8, theta=0.5, GMREStol=1e-12)
    batch = ix.Batch(probs, 3, dict(cfg, precision="mixed"))
    batch.step(2)
    for m, p in enumerate(probs):
        single = ix.Solver.for_problem(p, 3, cfg)
        single.step()
        single.step()
        a, b = batch.members[m].cons(), single.cons()
        for k in range(8):
            assert rel(a[k], b[k]) <= 1e-8, (m, k)
        assert batch.members[m].divergence()["cell_wrapped_l2"] <= 1e-12
        single.close()
    batch.close()


def test_batch_autotune_restores_member_state():
    probs = vortex_ensemble(6, seed=11, smin=24, smax=64)
    settings = dict(CFG0, floor_on=0)  # the linear pressure solve (one GMRES per member)
    batch = ix.Batch(probs, 2, settings)
    tuned = batch.autotune(trial_steps=1)
    print("autotune:", tuned, batch.info())
    assert tuned["streams"] in (0, 4, 8, 16) and tuned["ms_per_step"] > 0
    assert tuned["solve_tile"] in ((32, 16), (64, 8), (32, 8))
    for sv in batch.members:
        assert sv.scalars()["timestep"] == 0  # every trial step was undone
    batch.step(2)
    _check_members(batch, probs, 2, settings, 2, 1e-10, 1e-10)
    batch.close()


@pytest.mark.parametrize("tile", [1, 2])
def test_batch_solve_tile_shapes_match_single_runs(tile):
    """The batched B-form solve on 64x8 or 32x8 tiles: the same operator on other
    tiles, so the members still match their single runs (32x16 tiles) and the oracle."""
    probs = _members()[:3]
    batch = ix.Batch(probs, 2, CFG0)
    batch.set_solve_tile(tile)
    batch.step(2)
    _check_members(batch, probs, 2, CFG0, 2, 1e-11, 1e-10)
    batch.close()
