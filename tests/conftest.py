"""Shared fixtures.  GPU tests carry @pytest.mark.gpu; the rest run on CPU."""
from __future__ import annotations

import glob
import os
import subprocess
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200)")


def _cuda_available() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def pytest_collection_modifyitems(config, items):
    if _cuda_available():
        return
    skip = pytest.mark.skip(reason="no CUDA device")
    for item in items:
        if "gpu" in item.keywords:
            item.add_marker(skip)


@pytest.fixture(scope="session", autouse=True)
def _oracle_port_built():
    """The C restatement is cheap to build; make sure it is current."""
    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "port"], check=True)


def golden_step_cases():
    return sorted(os.path.basename(p)[5:-4] for p in glob.glob(os.path.join(GOLDEN, "step_*.npz")))


def load_golden(name: str):
    return np.load(os.path.join(GOLDEN, name), allow_pickle=False)


def golden_problem(g):
    """Problem object from the inputs stored in a golden step fixture."""
    from imex_b200.problems import Problem
    prim = g["prim0"]
    ny, nx = prim.shape[1:]
    x0, x1, y0, y1 = g["domain"]
    settings = eval(str(g["settings"]))  # the repr of a plain dict of literals written by make_golden.py
    p = Problem("golden", nx, ny, x0, x1, y0, y1, prim, g["bx0"], g["by0"], g["A0"], settings=settings)
    if "bx_x00" in g.files:
        p.bx_x0, p.by_y0 = g["bx_x00"], g["by_y00"]
    return p, int(g["rks"]), settings


def rel(a, b) -> float:
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    n = np.linalg.norm(b.ravel())
    d = np.linalg.norm((a - b).ravel())
    return d / n if n > 0 else d
