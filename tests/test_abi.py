"""The C-ABI library loads, exports every entry point of include/imex_b200.h, and its
host-side logic (defaults, validation) behaves as documented - no GPU needed."""
from __future__ import annotations

import ctypes as C
import os
import re
import subprocess

import pytest

from conftest import ROOT
import imex_b200 as ix
from oracle.bindings import DEFAULTS

HEADER = os.path.join(ROOT, "include", "imex_b200.h")


def header_functions() -> list[str]:
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(imex_[A-Za-z_0-9]+)\s*\(", text)))


def test_library_exports_every_declared_entry_point():
    lib = ix.load_library()
    names = header_functions()
    assert len(names) >= 45
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    out = subprocess.run(["nm", "-D", "--defined-only", ix.LIB_PATH], capture_output=True, text=True).stdout
    exported = set(re.findall(r" T (imex_[A-Za-z_0-9]+)", out))
    assert set(names) <= exported


def test_python_mirror_covers_the_header():
    assert set(header_functions()) == set(ix.exported_symbols())


def test_struct_layouts_match_the_header(tmp_path):
    src = tmp_path / "sizes.c"
    src.write_text(
        '#include <stdio.h>\n#include <stddef.h>\n#include "imex_b200.h"\n'
        'int main(void){printf("%zu %zu %zu %zu %zu %zu %zu %zu %zu %zu %zu\\n", sizeof(imex_config), sizeof(imex_step_scalars),'
        ' sizeof(imex_solve_stats), sizeof(imex_kernel_profile), offsetof(imex_config, mixed_max_refine),'
        ' offsetof(imex_config, gmres_restart), sizeof(imex_diagnostics_t), offsetof(imex_diagnostics_t, magE_max),'
        ' sizeof(imex_adjoint_opts), sizeof(imex_batch_tuning), offsetof(imex_batch_tuning, mixed_solves));'
        ' return 0;}\n')
    exe = tmp_path / "sizes"
    subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    vals = [int(v) for v in subprocess.run([str(exe)], capture_output=True, text=True).stdout.split()]
    assert vals == [C.sizeof(ix.Config), C.sizeof(ix.StepScalars), C.sizeof(ix.SolveStats),
                    C.sizeof(ix.KernelProfile), ix.Config.mixed_max_refine.offset,
                    ix.Config.gmres_restart.offset, C.sizeof(ix.Diagnostics), ix.Diagnostics.magE_max.offset,
                    C.sizeof(ix.AdjointOpts), C.sizeof(ix.BatchTuning), ix.BatchTuning.mixed_solves.offset]


def test_defaults_are_the_reference_defaults():
    cfg = ix.default_config()
    ref = dict(DEFAULTS)
    for key, table in ix.ENUMS.items():
        if key in ref:
            assert getattr(cfg, key) == table[ref[key]], key
    assert cfg.gamma_plasma == ref["gamma"]
    for key in ("GLF", "add_bvisc", "floor_on", "Pnewton_max", "vortex_test"):
        assert getattr(cfg, key) == ref[key], key
    for key in ("CFL", "GMREStol", "p_floor", "Mbig_fac", "theta", "Pnewton_tol", "shock_kappa1",
                "m_alfa", "m_b", "m_R", "m_cv"):
        assert getattr(cfg, key) == ref[key], key
    assert cfg.gmres_restart == 25  # implicit_operators.cpp:801
    assert cfg.RKs == 2 and cfg.x_bc == 2 and cfg.y_bc == 2


@pytest.mark.parametrize("override,status", [
    (dict(x_bc=1), 2), (dict(x_bc=3), 2), (dict(y_bc=4), 2), (dict(y_bc=1), 2),
    (dict(formula=2), 1),
    (dict(U_update=5), 1), (dict(arith=2), 1), (dict(RKs=4), 1), (dict(gmres_restart=31), 1),
    (dict(gmres_restart=0), 1), (dict(recon=7), 1), (dict(x_0=1.0, x_1=0.0), 1),
])
def test_create_rejects_invalid_or_unsupported_configs_before_touching_the_gpu(override, status):
    lib = ix.load_library()
    cfg = ix.make_config(override)
    h = C.c_void_p()
    assert lib.imex_create(C.byref(cfg), 16, 16, C.byref(h)) == status
    assert not h.value


def test_create_rejects_tiny_grids():
    lib = ix.load_library()
    cfg = ix.make_config({})
    h = C.c_void_p()
    assert lib.imex_create(C.byref(cfg), 3, 16, C.byref(h)) == 1


def test_status_strings():
    lib = ix.load_library()
    for code, text in ix.STATUS.items():
        assert lib.imex_status_string(code).decode() == text


def test_null_arguments_are_rejected():
    lib = ix.load_library()
    assert lib.imex_step(None, None) == 1
    assert lib.imex_destroy(None) == 0
    assert lib.imex_create(None, 8, 8, None) == 1
