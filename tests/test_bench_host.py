"""Host logic of bench.py that needs no GPU: replica aggregation over 2 gloo ranks,
clock-record parsing, workload table."""
from __future__ import annotations

import os
import socket

import pytest
import torch.multiprocessing as mp

import bench


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank: int, world: int, port: int, values, out):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    bench.barrier(world)
    out[rank] = bench.reduce_max(values[rank], world, device="cpu")
    dist.destroy_process_group()


def test_replica_time_is_the_max_over_ranks():
    world = 2
    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    values = [12.5, 17.25]
    mp.start_processes(_rank_main, args=(world, _free_port(), values, out), nprocs=world,
                       start_method="spawn", join=True)
    assert out[0] == out[1] == 17.25


def test_clock_summary_flags_throttle_reasons():
    c = bench.ClockSampler(0)
    c.lines = ["0, 1965, 1965, 700.0, 0x0, Not Active, Not Active, Not Active, Not Active",
               "0, 1800, 1965, 990.0, 0x4, Not Active, Not Active, Not Active, Active",
               "0, 1850, 1965, 995.0, 0x4, Not Active, Not Active, Not Active, Active"]
    s = c.summary()
    assert s["sm_mhz"] == 1850 and s["sm_max_mhz"] == 1965 and s["reasons"] == ["sw_power_cap"]


def test_workloads_and_peaks():
    assert bench.WORKLOADS["vortex_sheet_1024"]["rks"] == 3
    peak, kind = bench.measured_peaks()
    assert peak > 1000 and kind in ("measured", "fallback")


def test_reference_arm_config_matches_the_imex_arm():
    """Both arms print the same `config` object for the same workload and grid."""
    import argparse
    args = argparse.Namespace(workload="vortex_sheet_1024", precision="fp64")
    wl = bench.WORKLOADS["vortex_sheet_1024"]
    a = bench.arm_config(args, wl, 1024, 1024, 1)
    assert a["grid"] == "1024x1024" and a["workload"] == "vortex_sheet_1024"
    assert a == bench.arm_config(args, wl, 1024, 1024, 1)
    info = bench.host_info()
    assert info["nproc"] >= 1 and info["usable_cores"] >= 1


def test_reference_stage_stepping_matches_whole_steps():
    """The reference arm advances the reference one IMEX stage at a time (ref_stage); RKs
    stages in a row leave exactly the state of one whole reference time step."""
    import numpy as np
    from oracle.bindings import RefSolver, make_solver
    if not RefSolver.available():
        pytest.skip("oracle/_ref not built")
    wl = bench.WORKLOADS["vortex_sheet_1024"]
    prob = bench.make_problem(wl["problem"], 16)
    whole = make_solver("ref", prob, wl["rks"], wl["settings"])
    staged = bench._RefStages(prob, wl)
    assert staged.kind == "reference" and staged.unit_stages == 1
    for _ in range(2):
        whole.step()
        for _ in range(wl["rks"]):
            staged.advance()
    assert np.array_equal(whole.cons(), staged.solver.cons())
    assert np.array_equal(whole.vector_potential(), staged.solver.vector_potential())
    assert whole.scalars() == staged.solver.scalars()
