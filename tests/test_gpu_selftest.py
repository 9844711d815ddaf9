"""The library's own FP64 throughput measurement (the denominator of "FP64 bound")."""
from __future__ import annotations

import pytest

import imex_b200 as ix
from imex_b200.problems import vortex


@pytest.mark.gpu
def test_fp64_rates_are_measured_and_plausible():
    sv = ix.Solver.for_problem(vortex(16), 2, dict(recon="VanLeer", magfield="StaggerCT"))
    r = sv.selftest_fp64()
    # a B200 runs tens of FP64 TFLOP/s; a division costs several fused multiply-adds
    assert 5.0 < r["dfma_tflops"] < 200.0
    assert 0.0 < r["ddiv_per_s"] < r["dfma_per_s"]
    dt = sv.step()  # the context is still usable
    assert dt > 0
    sv.close()
