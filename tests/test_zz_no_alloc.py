"""imex_gmres_noalloc: the same GMRES solve as imex_gmres on the library's fixed
device scratch instead of allocated temporaries.  Compared through the C ABI
with imex_gmres on two calls in a row (host and device vectors), and the
oversize case is rejected with a clear error.  Collected last on purpose, so it
also runs after every other GPU test has used the device."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

import imex_b200 as ix
from imex_b200.problems import vortex, vortex_sheet

pytestmark = pytest.mark.gpu

CFG0 = dict(recon="VanLeer", magfield="StaggerCT", GMREStol=1e-12)
CFG1 = dict(recon="WENO5", magfield="PotentialA", p_floor=1e-8, theta=0.5, GMREStol=1e-12)
CASES = [
    ("pressure_L", lambda: vortex(64), 2, CFG0),
    ("magnetic_B", lambda: vortex(64), 2, CFG0),
    ("magnetic_A", lambda: vortex_sheet(64), 3, CFG1),
]


def _prepared(op, factory, rks, settings):
    sv = ix.Solver.for_problem(factory(), rks, settings)
    sv.step()  # leaves a real stage state in the context's buffers
    h = sv.scalars()["dt"] * 0.5
    sv.prepare_operator(op, h)
    n = sv.nx * sv.ny * (3 if op.startswith("magnetic") else 1)
    rng = np.random.default_rng(11)
    b = sv.apply_operator(op, rng.standard_normal(n))
    return sv, np.zeros(n), b


@pytest.mark.parametrize("op,factory,rks,settings", CASES)
def test_noalloc_matches_imex_gmres_on_two_calls(op, factory, rks, settings):
    sv, x0, b = _prepared(op, factory, rks, settings)
    ref, st_ref = sv.gmres(op, x0, b)
    assert st_ref["gmres_iters"] > 0
    for _ in range(2):
        got, st = sv.gmres_noalloc(op, x0, b)
        np.testing.assert_array_equal(got, ref)
        assert st["status"] == 0
    sv.close()


def test_noalloc_with_device_vectors():
    torch = pytest.importorskip("torch")
    op, factory, rks, settings = CASES[1]
    sv, x0, b = _prepared(op, factory, rks, settings)
    ref, _ = sv.gmres(op, x0, b)
    dp = C.POINTER(C.c_double)
    bd = torch.from_numpy(b).to("cuda")
    for _ in range(2):
        xd = torch.zeros(x0.size, dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        st = ix.SolveStats()
        rc = sv.lib.imex_gmres_noalloc(sv.ctx, ix.OP[op], C.cast(xd.data_ptr(), dp), C.cast(bd.data_ptr(), dp),
                                       C.byref(st))
        assert rc == 0, sv.lib.imex_last_error(sv.ctx)
        np.testing.assert_array_equal(xd.cpu().numpy(), ref)
    sv.close()


def test_noalloc_rejects_oversize_solve_and_context_survives():
    sv, x0, b = _prepared("magnetic_B", lambda: vortex(256), 2, CFG0)
    with pytest.raises(ix.ImexError) as err:
        sv.gmres_noalloc("magnetic_B", x0, b)
    assert err.value.status == 1
    assert "scratch" in str(err.value)
    x, st = sv.gmres("magnetic_B", x0, b)
    assert st["status"] == 0 and np.isfinite(x).all()
    sv.close()
