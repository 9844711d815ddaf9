"""Failure paths on the GPU: every failure is reported as a status, the GPU is never
trapped, and the context stays usable.  Failures are provoked from the host
(tolerance 0, a restart cap of 1, NaN in the initial data, misuse of the API)."""
from __future__ import annotations

import numpy as np
import pytest

import imex_b200 as ix
from imex_b200.problems import vortex

pytestmark = pytest.mark.gpu


def test_gmres_restart_cap_is_reported_and_context_survives():
    prob = vortex(32)
    sv = ix.Solver.for_problem(prob, 2, dict(recon="VanLeer", magfield="StaggerCT", GMREStol=0.0,
                                             gmres_max_restarts=1, gmres_restart=5))
    with pytest.raises(ix.ImexError) as err:
        sv.step()
    assert err.value.status in (ix.ImexError(4, "").status, 5)
    # the context is still usable after the error
    d = sv.divergence()
    assert np.isfinite(d["face_l2"])
    sv.close()


def test_nonfinite_input_is_reported():
    prob = vortex(32)
    prob.prim[0, 5, 7] = np.nan
    sv = ix.Solver.for_problem(prob, 2, dict(recon="VanLeer", magfield="StaggerCT"))
    with pytest.raises(ix.ImexError) as err:
        sv.step()
    assert err.value.status == 6
    sv.close()


def test_ct_variant_must_match_magfield():
    prob = vortex(16)
    sv = ix.Solver.for_problem(prob, 2, dict(recon="VanLeer", magfield="PotentialA"))
    with pytest.raises(ix.ImexError) as err:
        sv.Staggered_CT_Consistent(0.01, 0)
    assert err.value.status == 1
    sv.close()


def test_bad_buffer_and_stage_indices():
    sv = ix.Solver.for_problem(vortex(16), 2, dict(recon="VanLeer", magfield="StaggerCT"))
    with pytest.raises(ix.ImexError):
        sv.get_buffer("Hs", index=2)
    with pytest.raises(ix.ImexError):
        sv.stage(5)
    sv.close()


def test_barrier_wait_times_out_and_reports_sync_error():
    """A device-wide barrier that waits for CTAs that never launch must give up after its
    bound (0.2 s here), return IMEX_ERR_SYNC, and leave the context usable."""
    sv = ix.Solver.for_problem(vortex(64), 2, dict(recon="VanLeer", magfield="StaggerCT"))
    us = sv.selftest_barrier(200)           # healthy barriers complete
    assert 0.0 < us < 1000.0
    with pytest.raises(ix.ImexError) as err:
        sv.selftest_barrier(5, phantom_blocks=1, timeout_s=0.2)
    assert err.value.status == 8
    dt = sv.step()                          # the solver still works afterwards
    assert dt > 0 and sv.divergence()["face_l2"] < 1e-12
    sv.close()


def test_strong_field_redlich_kwong_is_reported_like_the_reference_fails():
    """At beta = 1e-4 the reference scheme itself goes non-finite within two steps on the
    Redlich-Kwong random field; the GPU path must report that as a status, not carry on."""
    from imex_b200.problems import random_field
    prob = random_field(32, beta=1e-4)
    settings = dict(recon="Minmod", magfield="StaggerCT", eos_type="REDLICH_KWONG", m_alfa=0.4275, m_b=0.0866)
    sv = ix.Solver.for_problem(prob, 2, settings)
    with pytest.raises(ix.ImexError) as err:
        for _ in range(2):
            sv.step()
    assert err.value.status in (5, 6, 7, 9)  # Newton cap, non-finite, positivity or EOS iteration cap
    sv.scalars()  # the context still answers after the error
    sv.close()
