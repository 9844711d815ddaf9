"""Test binding: the library's forward run and discrete adjoint as a torch.autograd.Function.

    cons_T = ImexRun.apply(prim0, bx0, by0, spec)

runs spec.nsteps steps through the C ABI from the initial primitive planes and face fields
and returns the final conserved planes; backward pulls the incoming cotangent back through
imex_adjoint_vjp (which recomputes the run from checkpoints).  Everything upstream (the
initial data as a function of parameters) and downstream (the misfit) is plain torch."""
from __future__ import annotations

import dataclasses
from dataclasses import dataclass

import numpy as np
import torch

import imex_b200 as ix
from imex_b200.problems import PerturbedVortex, Problem


@dataclass(frozen=True)
class RunSpec:
    base: Problem
    rks: int
    settings: dict
    nsteps: int
    checkpoint_every: int = 10


def _solver(spec: RunSpec, prim, bx, by) -> ix.Solver:
    p = dataclasses.replace(spec.base, prim=np.ascontiguousarray(prim), bx=np.ascontiguousarray(bx),
                            by=np.ascontiguousarray(by))
    return ix.Solver.for_problem(p, spec.rks, spec.settings)


class ImexRun(torch.autograd.Function):
    @staticmethod
    def forward(ctx, prim, bx, by, spec: RunSpec):
        sv = _solver(spec, prim.detach().numpy(), bx.detach().numpy(), by.detach().numpy())
        for _ in range(spec.nsteps):
            sv.step()
        cons = sv.cons()
        sv.close()
        ctx.spec = spec
        ctx.save_for_backward(prim, bx, by)
        return torch.from_numpy(cons)

    @staticmethod
    def backward(ctx, g):
        prim, bx, by = ctx.saved_tensors
        spec = ctx.spec
        sv = _solver(spec, prim.detach().numpy(), bx.detach().numpy(), by.detach().numpy())
        gp, gx, gy = sv.adjoint_vjp(spec.nsteps, g.detach().contiguous().numpy(),
                                    checkpoint_every=spec.checkpoint_every)
        sv.close()
        return torch.from_numpy(gp), torch.from_numpy(gx), torch.from_numpy(gy), None


def initial_fields(pv: PerturbedVortex, a: torch.Tensor):
    """prim, bx, by of the perturbed vortex as torch functions of the mode amplitudes a."""
    b = pv.base
    planes = torch.tensor(pv.PLANES)
    delta = torch.zeros((8, b.ny, b.nx), dtype=torch.float64)
    delta = delta.index_add(0, planes, torch.tensordot(a, torch.from_numpy(pv.dprim), dims=1))
    prim = torch.from_numpy(b.prim) + delta
    bx = torch.from_numpy(b.bx) + torch.tensordot(a, torch.from_numpy(pv.dbx), dims=1)
    by = torch.from_numpy(b.by) + torch.tensordot(a, torch.from_numpy(pv.dby), dims=1)
    return prim, bx, by


def misfit(cons: torch.Tensor, rho_t, B_t) -> torch.Tensor:
    """J = 1/2 |rho - rho_t|^2 + 1/2 |B - B_t|^2 over the cells."""
    rho_t = torch.as_tensor(rho_t)
    B_t = torch.as_tensor(B_t)
    return 0.5 * ((cons[0] - rho_t) ** 2).sum() + 0.5 * ((cons[5:8] - B_t) ** 2).sum()
