#!/usr/bin/env python
"""Throughput of the IMEX-RK stage on B200: cell-updates/s per IMEX stage.

Workload (default): the periodic vortex-sheet MHD problem on [0, 2*pi]^2 at
1024 x 1024 cells, gamma = 5/3, WENO5 reconstruction, vector-potential (A-form)
magnetic solve, nested-Newton pressure floor (p_floor = 1e-8, theta = 0.5),
IMEX-RK3, CFL 0.8, GMRES tolerance 1e-14 (the reference default).  One
benchmark step = one full time step = 3 IMEX stages.  Inputs are analytic
(no dataset).  The working set (~2 GB of state and Krylov vectors) is far
larger than the 126 MB L2, so no L2 flush is needed between steps.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl imex|reference]
                    [--workload vortex_sheet_1024|vortex_sheet_2048|vortex_64|random_field_2048|
                                open_blast_1024|vortex_ensemble_256] [--precision fp64|mixed]

vortex_ensemble_256 is the batched form: 256 independent vortex runs (seeded kappa, mu and
grid sides 64..512) advanced together through imex_batch (batched solves, CUDA graph,
autotuned streams and restart length).

Multi-GPU: the path does not shard (one 2D domain per GPU, "replicas only"):
N ranks each run an independent copy of the workload; value = total
cell-stage updates of all ranks / max over ranks of the timed span.

--impl reference times the reference solver's own CPU code (oracle/_ref,
built from the reference sources; else the C restatement) on the host with
the threads it can use (it is single-threaded), on the same workload and
grid as the GPU arm.  One of its benchmark steps is one IMEX stage of that
run (the metric is per stage, and one stage of the 1024^2 vortex sheet takes
the reference about 13 s on one core), so `--steps K --warmup W` runs W + K
consecutive stages.

The default line also carries a `mixed` object: the same workload in the
mixed-precision form (FP32 operator applications and Krylov updates inside
FP64 refinement), its speed against the FP64 line, and its relative L2 error
per field against the FP64 oracle on a small grid of the same physics.
The FP64 headline is timed with the live per-kernel profile off; the
per-kernel list and the roofline come from a second, profiled pass of the
same steps.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "cell-updates/s per IMEX stage"
CFG1 = dict(recon="WENO5", magfield="PotentialA", floor_on=1, p_floor=1e-8, theta=0.5,
            GMREStol=1e-14, CFL=0.8)
CFG0 = dict(recon="VanLeer", magfield="StaggerCT", GMREStol=1e-12, CFL=0.8)
CFG2 = dict(recon="Minmod", magfield="StaggerCT", floor_on=1, eos_type="REDLICH_KWONG", m_alfa=0.4275,
            m_b=0.0866, CFL=0.8)
WORKLOADS = {
    "vortex_sheet_1024": dict(problem="vortex_sheet", n=1024, rks=3, settings=CFG1,
                              desc="vortex-sheet MHD 1024^2, WENO5, A-form CT, floor on, RK3"),
    "vortex_sheet_2048": dict(problem="vortex_sheet", n=2048, rks=3, settings=CFG1,
                              desc="vortex-sheet MHD 2048^2, WENO5, A-form CT, floor on, RK3"),
    "vortex_64": dict(problem="vortex", n=64, rks=2, settings=CFG0,
                      desc="smooth MHD vortex 64^2, VanLeer, staggered CT, RK2"),
    "vortex_ensemble_256": dict(problem="vortex_ensemble", n=0, rks=2, settings=CFG0, members=256, precision="mixed",
                                desc="256 independent vortex runs (seed 2026: kappa, mu ~ U[0.5,1.5], square "
                                     "sides log-uniform 64..512), VanLeer, staggered CT, RK2, one ensemble"),
    "random_field_2048": dict(problem="random_field", n=2048, rks=2, settings=CFG2,
                              desc="seeded low-Mach random field 2048^2 (seed 2026, beta 0.1), Redlich-Kwong, "
                                   "Minmod, EMF-consistent staggered CT, floor on, RK2"),
}
CFG3 = dict(recon="WENO5", magfield="StaggerCT", floor_on=1, p_floor=1e-8, theta=0.5, GMREStol=1e-14, CFL=0.8)
WORKLOADS["open_blast_1024"] = dict(problem="open_blast", n=1024, rks=3, settings=CFG3,
                                    desc="smooth blast in an oblique field on the open unit square 1024^2 "
                                         "(transmissive x and y), WENO5, EMF-consistent staggered CT, floor on, RK3")


def make_problem(kind: str, n: int):
    from imex_b200.problems import open_blast, random_field, vortex, vortex_sheet
    if kind == "random_field":
        return random_field(n)
    if kind == "open_blast":
        return open_blast(n)
    return vortex(n) if kind == "vortex" else vortex_sheet(n)


def measured_peaks() -> tuple[float, str]:
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def ncu_traffic(family: str, workload: str, n: int) -> float | None:
    """Per-launch DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) of `family`
    from the committed ncu summary, when it was captured on this workload and grid."""
    path = os.path.join(ROOT, "profiles", "ncu_traffic.json")
    try:
        with open(path) as f:
            d = json.load(f)
        if d["workload"] != workload or int(d["n"]) != n:
            return None
        return float(d["families"][family]["dram_bytes_per_launch"])
    except Exception:
        return None


class ClockSampler:
    """SM clocks and throttle reasons during the timed region: NVML read every 10 ms from a
    thread (the timed region of the default workload lasts about 0.1 s), plus nvidia-smi every
    200 ms.  Both only read the GPU's state."""
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    # NVML clock-event reason bits (nvml.h): sw power cap, hw slowdown, sw / hw thermal
    NVML_BITS = {"sw_power_cap": 0x4, "hw_slowdown": 0x8, "sw_thermal_slowdown": 0x20,
                 "hw_thermal_slowdown": 0x40}

    def __init__(self, gpu: int):
        self.gpu = gpu
        self.proc = None
        self.nvml = []
        self._stop = None
        self._thread = None

    def _nvml_loop(self):
        try:
            import pynvml
            pynvml.nvmlInit()
            h = pynvml.nvmlDeviceGetHandleByIndex(self.gpu)
            self.nvml_max = pynvml.nvmlDeviceGetMaxClockInfo(h, pynvml.NVML_CLOCK_SM)
            while not self._stop.is_set():
                mhz = pynvml.nvmlDeviceGetClockInfo(h, pynvml.NVML_CLOCK_SM)
                try:
                    bits = pynvml.nvmlDeviceGetCurrentClocksEventReasons(h)
                except Exception:
                    bits = pynvml.nvmlDeviceGetCurrentClocksThrottleReasons(h)
                self.nvml.append((float(mhz), int(bits)))
                self._stop.wait(0.01)
            pynvml.nvmlShutdown()
        except Exception:
            pass

    def __enter__(self):
        import threading
        self._stop = threading.Event()
        self._thread = threading.Thread(target=self._nvml_loop, daemon=True)
        self._thread.start()
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.QUERY}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *exc):
        self.lines = []
        if self._thread is not None:
            self._stop.set()
            self._thread.join(timeout=5)
        if self.proc is not None:
            self.proc.terminate()
            try:
                out, _ = self.proc.communicate(timeout=5)
            except Exception:
                self.proc.kill()
                out, _ = self.proc.communicate()
            self.lines = [l for l in out.splitlines() if l.strip()]

    def summary(self) -> dict:
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in getattr(self, "lines", []):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for name, flag in zip(names, parts[5:9]):
                if flag.lower().startswith("active"):
                    reasons.add(name)
        for mhz, bits in self.nvml:
            sm.append(mhz)
            for name, bit in self.NVML_BITS.items():
                if bits & bit:
                    reasons.add(name)
        if smax is None and getattr(self, "nvml_max", None):
            smax = float(self.nvml_max)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm), "nvml_samples": len(self.nvml)}


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    return world, rank, local


def reduce_max(value: float, world: int, device: str = "cuda") -> float:
    """Max of a per-rank value over all ranks (the timed span of the slowest replica)."""
    if world == 1:
        return value
    import torch
    import torch.distributed as dist
    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(world: int) -> None:
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def host_info() -> dict:
    """CPU model and core counts of the host the CPU legs run on."""
    model = None
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    model = line.split(":", 1)[1].strip()
                    break
    except OSError:
        pass
    try:
        usable = len(os.sched_getaffinity(0))
    except Exception:
        usable = os.cpu_count()
    return {"cpu_model": model, "nproc": os.cpu_count(), "usable_cores": usable}


def arm_config(args, wl: dict, nx: int, ny: int, world: int) -> dict:
    """The `config` object both arms print for the same workload (so the lines compare)."""
    return {"workload": args.workload, "description": wl["desc"], "grid": f"{nx}x{ny}",
            "stages_per_step": wl["rks"], "precision": args.precision,
            "parallelism": f"replicas x{world}",
            "l2": "inputs larger than L2 (working set >> 126 MB); no flush"}


class _RefStages:
    """The reference CPU solver advanced one IMEX stage at a time (oracle/_ref's
    ref_stage), or one whole time step at a time when only the C restatement exists."""

    def __init__(self, prob, wl: dict):
        import ctypes as C
        from oracle.bindings import RefSolver, make_solver
        self.kind = "reference" if RefSolver.available() else "port"
        self.solver = make_solver("ref" if self.kind == "reference" else "port", prob, wl["rks"],
                                  wl["settings"])
        self.cells = prob.nx * prob.ny
        self.rks = wl["rks"]
        self._stage = None
        if self.kind == "reference":
            self._stage = self.solver.lib.ref_stage
            self._stage.restype, self._stage.argtypes = C.c_int, []

    @property
    def unit_stages(self) -> int:
        """IMEX stages one advance() runs."""
        return 1 if self._stage is not None else self.rks

    def advance(self) -> None:
        if self._stage is not None:
            if self._stage() < 0:
                raise RuntimeError("ref_stage failed")
        else:
            self.solver.step()


def cpu_reference_rate(prob, wl: dict, max_seconds: float, max_units: int = 4) -> dict:
    """The reference CPU solver on the workload's own grid, from t = 0: cell-stage updates
    per second over the first stages, stopping once `max_seconds` are spent (at least one)."""
    ref = _RefStages(prob, wl)
    done, t_total = 0, 0.0
    while done < max_units:
        t0 = time.perf_counter()
        ref.advance()
        t_total += time.perf_counter() - t0
        done += 1
        if t_total > max_seconds:
            break
    stages = done * ref.unit_stages
    info = host_info()
    return dict(value=ref.cells * stages / t_total, unit="cell-updates/s", cores=1, kind=ref.kind,
                sample=(f"the first {stages} IMEX stage(s) of the same run ({prob.nx}x{prob.ny}, from t=0) "
                        f"on one core of a {info['nproc']}-core host ({info['cpu_model']})"),
                host=info, seconds=t_total)


def run_reference(args, world: int, rank: int) -> None:
    """The reference's own CPU solver on the same workload and grid as the GPU arm: W warm-up
    and K timed benchmark steps of one IMEX stage each (rank 0 only)."""
    if rank != 0:
        return
    try:
        import oracle.bindings  # noqa: F401
    except Exception as exc:  # pragma: no cover
        print(json.dumps({"impl": "reference", "unavailable": f"oracle import failed: {exc}"}))
        return
    wl = WORKLOADS[args.workload]
    info = host_info()
    if wl["problem"] == "vortex_ensemble":
        # the reference has no batching: its members run one after another, one time step of
        # the next member (in ensemble order, smallest first) per benchmark step
        from imex_b200.problems import vortex_ensemble
        probs = sorted(vortex_ensemble(wl["members"], seed=2026), key=lambda q: q.nx * q.ny)
        runs = [_RefStages(p, wl) for p in probs[:args.warmup + args.steps]]
        for r in runs[:args.warmup]:
            for _ in range(r.rks // r.unit_stages):
                r.advance()
        t0 = time.perf_counter()
        cells = 0
        for r in runs[args.warmup:]:
            for _ in range(r.rks // r.unit_stages):
                r.advance()
            cells += r.cells * r.rks
        t = time.perf_counter() - t0
        value = cells / t
        ref = runs[0]
        nx = ny = 0
        config = arm_config(args, wl, nx, ny, world)
        config.pop("grid")
        unit_desc = "one time step of one member"
        sample = (f"{args.steps} members (the smallest, after {args.warmup} warm-up members), one time step "
                  f"each; single-threaded reference on one core of a {info['nproc']}-core host "
                  f"({info['cpu_model']})")
    else:
        prob = make_problem(wl["problem"], args.n or wl["n"])
        ref = _RefStages(prob, wl)
        for _ in range(args.warmup):
            ref.advance()
        t0 = time.perf_counter()
        for _ in range(args.steps):
            ref.advance()
        t = time.perf_counter() - t0
        stages = args.steps * ref.unit_stages
        value = ref.cells * stages / t
        config = arm_config(args, wl, prob.nx, prob.ny, world)
        unit_desc = "one IMEX stage" if ref.unit_stages == 1 else f"one time step ({ref.unit_stages} stages)"
        sample = (f"{args.steps} consecutive benchmark steps of {unit_desc} each, after {args.warmup} warm-up, "
                  f"of the {prob.nx}x{prob.ny} run; single-threaded reference on one core of a "
                  f"{info['nproc']}-core host ({info['cpu_model']})")
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "cell-updates/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": t / args.steps * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (analytic initial data, no dataset)",
        "config": config,
        "step_unit": unit_desc,
        "cpu_baseline": {"value": value, "unit": "cell-updates/s", "cores": 1, "kind": ref.kind,
                         "sample": sample, "host": info},
        "e2e": {"value": value, "unit": "cell-updates/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))
    if args.json_out:
        with open(args.json_out, "w") as f:
            json.dump(line, f, indent=1)


def run_ensemble(args, world: int, rank: int, local: int) -> None:
    """The batched form: all members of the ensemble advance together through imex_batch.
    value = cell-stage updates of all members (all ranks) / the timed span (max over ranks)."""
    import torch
    import imex_b200 as ix
    from imex_b200.problems import vortex_ensemble

    torch.cuda.set_device(local)
    wl = WORKLOADS[args.workload]
    probs = vortex_ensemble(wl["members"], seed=2026)
    settings = dict(wl["settings"])
    settings["precision"] = args.precision
    if args.mixed_solves is not None:
        settings["mixed_solves"] = args.mixed_solves
    batch = ix.Batch(probs, wl["rks"], settings)
    tuned = None if args.no_autotune else batch.autotune(trial_steps=1)
    launches0 = sum(m.kernel_launches() for m in batch.members)
    batch.step(1)  # captures the step (launch count of one step) and runs it
    info = batch.info()
    if info["explicit_launches_per_step"] >= 0:  # batched explicit sub-steps: the planned step's launches
        launches_per_step = info["explicit_launches_per_step"] + info["planned_solve_launches_per_step"]
    else:
        launches_per_step = (sum(m.kernel_launches() for m in batch.members) - launches0
                             + 2 * info["solve_launches_per_step"])
    for _ in range(max(args.warmup - 1, 2)):
        batch.step(1)
    cells_per_step = sum(p.nx * p.ny for p in probs) * wl["rks"]
    barrier(world)
    torch.cuda.synchronize()
    with ClockSampler(local) as clocks:
        ms = batch.step(args.steps)
    barrier(world)
    t_max = reduce_max(ms, world)
    value = world * cells_per_step * args.steps / (t_max / 1e3)

    # end to end: every member's state from pinned host memory in, the ensemble step, out
    e2e = None
    if not args.no_e2e:
        bufs = []
        for p in probs:
            n = p.nx * p.ny
            bufs.append([torch.empty(k * n, dtype=torch.float64, pin_memory=True) for k in (8, 1, 1, 3)])
        for m, sv in enumerate(batch.members):
            sv.download_state_ptr(*(t.data_ptr() for t in bufs[m]))
        e2e_steps = min(args.steps, 3)
        barrier(world)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(e2e_steps):
            for m, sv in enumerate(batch.members):
                sv.upload_state_ptr(*(t.data_ptr() for t in bufs[m]))
            batch.step(1)
            for m, sv in enumerate(batch.members):
                sv.download_state_ptr(*(t.data_ptr() for t in bufs[m]))
        torch.cuda.synchronize()
        wall = reduce_max((time.perf_counter() - t0) * 1e3, world)
        nbytes = sum(13 * p.nx * p.ny * 8 for p in probs)
        e2e = {"value": world * cells_per_step * e2e_steps / (wall / 1e3), "unit": "cell-updates/s",
               "h2d_bytes_per_step": nbytes, "d2h_bytes_per_step": nbytes, "steps": e2e_steps,
               "path": "imex_upload_state + imex_batch_step + imex_download_state per member, pinned host buffers"}
    stats = [m.stats() for m in batch.members]
    batch.close()

    # roofline: the largest member alone, with the live kernel profile
    big = max(probs, key=lambda p: p.nx * p.ny)
    sv = ix.Solver.for_problem(big, wl["rks"], settings)
    for _ in range(2):
        sv.step()
    sv.profile_enable(True)
    for _ in range(2):
        sv.step()
    prof = sv.profile()
    sv.close()
    peak, peak_kind = measured_peaks()
    dom = max(prof, key=lambda r: r["total_ms"])
    achieved = dom["alg_bytes"] / (dom["total_ms"] / 1e3) / 1e9
    roofline = {"kernel": dom["name"], "bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "traffic": None,
                "alg_bytes_per_launch": dom["alg_bytes"] / dom["launches"],
                "launches": dom["launches"], "ms_per_launch": dom["total_ms"] / dom["launches"],
                "measured_on": f"the largest member ({big.nx}x{big.ny}) run alone with the live profile",
                "peak_source": f"{peak_kind} hbm_gbs (MEASURED_PEAKS.json)"}
    if rank == 0:
        cpu = None
        if not args.no_cpu_baseline:
            cpu = ensemble_cpu_rate(probs, wl, max_seconds=12.0)
        line = {
            "metric": METRIC, "value": value, "unit": "cell-updates/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": t_max / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64" if args.precision == "fp64" else "f32+f64",
            "data": "synthetic (seeded vortex ensemble, no dataset)",
            "config": {"workload": args.workload, "description": wl["desc"], "members": len(probs),
                       "cells": sum(p.nx * p.ny for p in probs),
                       "sides": [min(p.nx for p in probs), max(p.nx for p in probs)],
                       "stages_per_step": wl["rks"], "precision": args.precision,
                       "parallelism": f"replicas x{world}", "autotuned": tuned, "batch": info,
                       "l2": "working set ~40 GB >> 126 MB L2; no flush"},
            "roofline": roofline,
            "cpu_baseline": cpu,
            "e2e": e2e,
            "gpu_launches": launches_per_step * args.steps,
            "clocks": clocks.summary(),
            "solver": {"gmres_iters": sum(s["gmres_iters"] for s in stats),
                       "newton_iters": sum(s["newton_iters"] for s in stats),
                       "status": max(s["status"] for s in stats)},
        }
        print(json.dumps(line))
        if args.json_out:
            with open(args.json_out, "w") as f:
                json.dump(line, f, indent=1)


def ensemble_cpu_rate(probs, wl, max_seconds: float) -> dict:
    """The reference CPU solver on the ensemble's members, smallest first, one step each,
    until about max_seconds of CPU time: cell-stage updates per second on one core."""
    from oracle.bindings import RefSolver, make_solver
    kind = "reference" if RefSolver.available() else "port"
    cells, t_total, done = 0, 0.0, 0
    for p in sorted(probs, key=lambda q: q.nx * q.ny):
        solver = make_solver("ref" if kind == "reference" else "port", p, wl["rks"], wl["settings"])
        t0 = time.perf_counter()
        solver.step()
        t_total += time.perf_counter() - t0
        cells += p.nx * p.ny * wl["rks"]
        done += 1
        if t_total > max_seconds:
            break
    info = host_info()
    return dict(value=cells / t_total, unit="cell-updates/s", cores=1, kind=kind,
                sample=(f"one time step of each of the {done} smallest members, one core of a "
                        f"{info['nproc']}-core host ({info['cpu_model']})"), host=info)


def adjoint_measure(n: int = 512, steps: int = 50, checkpoint_every: int = 10) -> dict:
    """The differentiation form on its own workload: the 32-mode perturbed vortex, J = misfit
    of rho and B against the unperturbed run, gradient w.r.t. the initial fields by the
    checkpointed discrete adjoint; the forward run is timed beside it, the adjoint by wall
    clock (it includes its recomputations, workspace and host synchronisations)."""
    import numpy as np
    import torch
    import imex_b200 as ix
    from imex_b200.problems import perturbed_vortex

    pv = perturbed_vortex(n)
    settings = dict(recon="VanLeer", magfield="StaggerCT", GMREStol=1e-12, fixed_dt=0.0025)
    sv = ix.Solver.for_problem(pv.base, 2, settings)
    for _ in range(steps):
        sv.step()
    c = sv.cons()
    sv.close()
    sv = ix.Solver.for_problem(pv.problem(), 2, settings)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(steps):
        sv.step()
    torch.cuda.synchronize()
    fwd = time.perf_counter() - t0
    sv.close()
    # a first adjoint run with the live profile gives the kernel shares; a second one, on a
    # fresh context with the profile off (its events around every launch family would be
    # timed too), gives the time
    sv = ix.Solver.for_problem(pv.problem(), 2, settings)
    sv.profile_enable(True)
    sv.adjoint_run(steps, c[0], c[5:8], checkpoint_every=checkpoint_every)
    prof = sv.profile()
    sv.close()
    sv = ix.Solver.for_problem(pv.problem(), 2, settings)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    J, gp, gx, gy = sv.adjoint_run(steps, c[0], c[5:8], checkpoint_every=checkpoint_every)
    adj = time.perf_counter() - t0
    sv.close()
    g = np.array([np.sum(gp[list(pv.PLANES)] * pv.dprim[m]) + np.sum(gx * pv.dbx[m]) + np.sum(gy * pv.dby[m])
                  for m in range(len(pv.amplitudes))])
    tot = sum(r["total_ms"] for r in prof) or 1.0
    return {"workload": f"perturbed_vortex_{n} (32 modes of v and A_z, amplitude 1e-2)", "steps": steps,
            "checkpoint_every": checkpoint_every, "forward_s": fwd, "adjoint_s": adj,
            "adjoint_over_forward": adj / fwd, "J": J, "grad_amplitudes_norm": float(np.linalg.norm(g)),
            "kernels": sorted(({"name": r["name"], "share": r["total_ms"] / tot} for r in prof),
                              key=lambda r: -r["share"])[:8]}


def main() -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="imex", choices=["imex", "reference"])
    ap.add_argument("--workload", default="vortex_sheet_1024", choices=sorted(WORKLOADS))
    ap.add_argument("--precision", default=None, choices=["fp64", "mixed"],
                    help="default: the workload's own (mixed for the ensemble, as its configuration asks; "
                         "fp64 otherwise, with the mixed pair measured beside it)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-adjoint", action="store_true", help="skip the adjoint-form measurement")
    ap.add_argument("--no-mixed", action="store_true", help="skip the mixed-precision pair")
    ap.add_argument("--no-autotune", action="store_true",
                    help="ensemble: keep the configured streams, restart length and mixed solves")
    ap.add_argument("--mixed-solves", type=int, default=None,
                    help="ensemble: the mixed solves (imex_mixed_solves bits) to start from, e.g. the set "
                         "an earlier autotune chose, with --no-autotune")
    ap.add_argument("--n", type=int, default=None, help="override the grid side (profiling cases)")
    ap.add_argument("--json-out", default=None)
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.precision is None:
        args.precision = WORKLOADS[args.workload].get("precision", "fp64")

    world, rank, local = dist_setup()
    if args.impl == "imex" and WORKLOADS[args.workload]["problem"] == "vortex_ensemble":
        run_ensemble(args, world, rank, local)
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
        return 0
    if args.impl == "reference":
        run_reference(args, world, rank)
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
        return 0

    import torch
    import imex_b200 as ix

    torch.cuda.set_device(local)
    wl = WORKLOADS[args.workload]
    prob = make_problem(wl["problem"], args.n or wl["n"])
    cells_per_step = prob.nx * prob.ny * wl["rks"]
    stream = torch.cuda.Stream()
    peak, peak_kind = measured_peaks()

    # ---- headline: K timed steps, live profile off
    run = timed_run(ix, prob, wl, args.precision, stream, args.steps, args.warmup, world, local,
                    clocks=True)
    solver = run.pop("solver")
    t_max = run["t_max_ms"]
    value = world * cells_per_step * args.steps / (t_max / 1e3)

    # ---- the same W + K steps once more, on a second context, with the per-kernel profile on
    # over the K steps (CUDA events per launch family): the kernel list describes the steps the
    # headline timed (later steps of this flow need more solver iterations)
    psv = ix.Solver.for_problem(prob, wl["rks"], dict(wl["settings"], precision=args.precision))
    psv.set_stream(stream.cuda_stream)
    for _ in range(args.warmup):
        psv.step()
    psv.reset_stats()
    psv.profile_enable(True)
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    start.record(stream)
    for _ in range(args.steps):
        psv.step()
    stop.record(stream)
    torch.cuda.synchronize()
    prof_ms = start.elapsed_time(stop)
    prof = psv.profile()
    psv.profile_enable(False)
    stats = psv.stats()
    psv.close()
    dom = max(prof, key=lambda r: r["total_ms"])
    achieved = dom["alg_bytes"] / (dom["total_ms"] / 1e3) / 1e9
    traffic = ncu_traffic(dom["name"], args.workload, prob.nx)
    total_prof_ms = sum(r["total_ms"] for r in prof)
    roofline = {"kernel": dom["name"], "bound": "hbm", "achieved": achieved, "peak": peak,
                "unit": "GB/s", "frac": achieved / peak, "traffic": traffic,
                "alg_bytes_per_launch": dom["alg_bytes"] / dom["launches"],
                "launches": dom["launches"], "ms_per_launch": dom["total_ms"] / dom["launches"],
                "share_of_step": dom["total_ms"] / total_prof_ms if total_prof_ms else None,
                "timing": "CUDA events around each launch family, in a profiled repeat of the headline's steps",
                "peak_source": "measured hbm_gbs (MEASURED_PEAKS.json)" if peak_kind == "measured"
                else "fallback 6650 GB/s"}
    step_bytes = sum(r["alg_bytes"] for r in prof)

    # ---- the device's FP64 rates (denominators of the FP64-bound stencil kernels)
    fp64 = solver.selftest_fp64()

    # ---- end to end through the C ABI: pinned host state in, step, state out, every step
    e2e = None
    if not args.no_e2e:
        e2e = e2e_run(solver, prob, stream, args.steps, world, cells_per_step)

    # ---- the mixed-precision form on the same workload, and its error against the FP64 oracle
    mixed = None
    if args.precision == "fp64" and not args.no_mixed:
        solver.close()
        solver = None
        mrun = timed_run(ix, prob, wl, "mixed", stream, args.steps, args.warmup, world, local, clocks=False)
        msv = mrun.pop("solver")
        mstats = msv.stats()
        m_ms = mrun["t_max_ms"]
        mixed = {"value": world * cells_per_step * args.steps / (m_ms / 1e3),
                 "ms_per_step": m_ms / args.steps, "speedup_vs_fp64": t_max / m_ms,
                 "solver": {"gmres_iters": mstats["gmres_iters"], "newton_iters": mstats["newton_iters"],
                            "refine_sweeps": mstats["refine_sweeps"], "status": mstats["status"]}}
        msv.close()
        if rank == 0:
            mixed["accuracy"] = mixed_accuracy(ix, wl, args.workload)
    elif args.precision == "mixed" and rank == 0:
        mixed = {"accuracy": mixed_accuracy(ix, wl, args.workload)}

    adjoint = None
    if rank == 0 and not args.no_adjoint:
        try:
            adjoint = adjoint_measure()
        except Exception as exc:
            adjoint = {"error": str(exc)}
    if rank == 0:
        cpu = None
        if not args.no_cpu_baseline:
            try:
                cpu = cpu_reference_rate(prob, wl, max_seconds=20.0)
                cpu.pop("seconds", None)
            except Exception as exc:
                cpu = {"value": None, "error": str(exc)}
        line = {
            "metric": METRIC, "value": value, "unit": "cell-updates/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": t_max / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64" if args.precision == "fp64" else "f32+f64",
            "data": "synthetic (analytic initial data, no dataset)",
            "config": arm_config(args, wl, prob.nx, prob.ny, world),
            "roofline": roofline,
            "cpu_baseline": cpu,
            "e2e": e2e,
            "gpu_launches": run["launches"],
            "clocks": run["clocks"],
            "mixed": mixed,
            "fp64_peak": {"dfma_tflops": fp64["dfma_tflops"], "ddiv_per_s": fp64["ddiv_per_s"],
                          "source": "imex_selftest_fp64 on this GPU, in this run"},
            "adjoint": adjoint,
            "solver": {"gmres_iters": stats["gmres_iters"], "gmres_solves": stats["gmres_solves"],
                       "newton_iters": stats["newton_iters"], "refine_sweeps": stats["refine_sweeps"],
                       "status": stats["status"],
                       "alg_bytes_per_step": step_bytes / args.steps,
                       "stage_hbm_frac": step_bytes / (prof_ms / 1e3) / 1e9 / peak,
                       "profiled_pass_ms_per_step": prof_ms / args.steps},
            "kernels": sorted(({"name": r["name"], "share": r["total_ms"] / total_prof_ms,
                                "launches": r["launches"],
                                "GBps": r["alg_bytes"] / (r["total_ms"] / 1e3) / 1e9 if r["total_ms"] else 0}
                               for r in prof), key=lambda r: -r["share"]),
        }
        print(json.dumps(line))
        if args.json_out:
            with open(args.json_out, "w") as f:
                json.dump(line, f, indent=1)
    if solver is not None:
        solver.close()
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    return 0


def timed_run(ix, prob, wl: dict, precision: str, stream, steps: int, warmup: int, world: int, local: int,
              clocks: bool) -> dict:
    """W warm-up steps, then K steps timed with CUDA events on the solver's stream between
    barriers and synchronisations; returns the solver and the max over ranks of the span."""
    import torch
    settings = dict(wl["settings"])
    settings["precision"] = precision
    solver = ix.Solver.for_problem(prob, wl["rks"], settings)
    solver.set_stream(stream.cuda_stream)
    for _ in range(warmup):
        solver.step()
    solver.reset_stats()
    k0 = solver.kernel_launches()
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier(world)
    torch.cuda.synchronize()
    sampler = ClockSampler(local) if clocks else None
    if sampler:
        sampler.__enter__()
    start.record(stream)
    for _ in range(steps):
        solver.step()
    stop.record(stream)
    torch.cuda.synchronize()
    if sampler:
        sampler.__exit__(None, None, None)
    barrier(world)
    t_ms = start.elapsed_time(stop)
    return {"solver": solver, "t_ms": t_ms, "t_max_ms": reduce_max(t_ms, world),
            "launches": solver.kernel_launches() - k0, "clocks": sampler.summary() if sampler else None}


def e2e_run(solver, prob, stream, steps: int, world: int, cells_per_step: int) -> dict:
    """The metric through the public API with host buffers: every step uploads the state from
    pinned host memory, steps, and downloads it (copies inside the timed region)."""
    import torch
    N = prob.nx * prob.ny
    h_prim = torch.empty(8 * N, dtype=torch.float64, pin_memory=True)
    h_bx = torch.empty(N, dtype=torch.float64, pin_memory=True)
    h_by = torch.empty(N, dtype=torch.float64, pin_memory=True)
    h_A = torch.empty(3 * N, dtype=torch.float64, pin_memory=True)
    ptrs = (h_prim.data_ptr(), h_bx.data_ptr(), h_by.data_ptr(), h_A.data_ptr())
    solver.download_state_ptr(*ptrs)
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier(world)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    start.record(stream)
    for _ in range(steps):
        solver.upload_state_ptr(*ptrs)
        solver.step()
        solver.download_state_ptr(*ptrs)
    stop.record(stream)
    torch.cuda.synchronize()
    wall = time.perf_counter() - t0
    e2e_ms = reduce_max(max(start.elapsed_time(stop), wall * 1e3), world)
    nbytes = (8 + 1 + 1 + 3) * N * 8
    return {"value": world * cells_per_step * steps / (e2e_ms / 1e3), "unit": "cell-updates/s",
            "h2d_bytes_per_step": nbytes, "d2h_bytes_per_step": nbytes,
            "path": "imex_upload_state + imex_step + imex_download_state, pinned host buffers"}


ACCURACY_N = 64
ACCURACY_STEPS = 20


def mixed_accuracy(ix, wl: dict, workload: str, n: int = ACCURACY_N, steps: int = ACCURACY_STEPS) -> dict:
    """Relative L2 error per field of the mixed form, and of the FP64 GPU path, against the FP64
    oracle (the reference's own solver when built, else its C restatement) after `steps` time
    steps of the same physics on an n x n grid."""
    import numpy as np
    from oracle.bindings import RefSolver, make_solver
    prob = make_problem(wl["problem"], n)
    kind = "reference" if RefSolver.available() else "port"
    ora = make_solver("ref" if kind == "reference" else "port", prob, wl["rks"], wl["settings"])
    for _ in range(steps):
        ora.step()
    want = ora.cons()
    out = {"oracle": f"FP64 {kind} solver on the CPU", "grid": f"{n}x{n}", "steps": steps}
    for prec in ("mixed", "fp64"):
        sv = ix.Solver.for_problem(prob, wl["rks"], dict(wl["settings"], precision=prec))
        for _ in range(steps):
            sv.step()
        got = sv.cons()
        sv.close()
        errs = [float(np.linalg.norm(got[k] - want[k]) / max(np.linalg.norm(want[k]), 1e-300))
                for k in range(8)]
        out[f"{prec}_max_rel_l2_per_field"] = max(errs)
        out[f"{prec}_rel_l2_per_field"] = errs
    return out


if __name__ == "__main__":
    sys.exit(main())
