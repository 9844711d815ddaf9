"""Initial data for the benchmark and test workloads (analytic or seeded).

Every field is returned as interior-only SoA planes of shape (ny, nx), index
[j, i] with x fastest in memory, which is the layout the C ABI takes:

    prim  (8, ny, nx): rho, vx, vy, vz, p, Bx, By, Bz   (cell averages)
    bx    (ny, nx)   : Bx on the x-face (i+1/2, j)
    by    (ny, nx)   : By on the y-face (i, j+1/2)
    A     (3, ny, nx): vector potential at cell centres

Formulas follow the reference's initial conditions:
  * vortex:  initial_conditions.cpp:641-669 (cell state) and :698-717 (faces
    from corner A_z, cell B = face average), A_initial
    constrained_transport.cpp:389-394, generalised by the background flow
    (1,1) and the kappa/mu amplitudes of the vortex workload;
  * vortex sheet: the Orszag-Tang field of initial_conditions.cpp:426-435 in
    [0, 2*pi]^2 form, faces = average of neighbouring cell B as in
    initial_conditions.cpp:720-726, A_z = cos y + cos(2x)/2.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np


@dataclass
class Problem:
    name: str
    nx: int
    ny: int
    x0: float
    x1: float
    y0: float
    y1: float
    prim: np.ndarray
    bx: np.ndarray
    by: np.ndarray
    A: np.ndarray
    settings: dict = field(default_factory=dict)

    @property
    def dx(self) -> float:
        return (self.x1 - self.x0) / self.nx

    @property
    def dy(self) -> float:
        return (self.y1 - self.y0) / self.ny


def vortex(n: int = 64, ny: int | None = None, kappa: float = 1.0, mu: float = 1.0,
           background: tuple[float, float] = (1.0, 1.0), half_width: float = 5.0) -> Problem:
    """Smooth MHD vortex on the periodic square [-L, L]^2 (gamma = 5/3)."""
    nx = n
    ny = n if ny is None else ny
    x0, x1, y0, y1 = -half_width, half_width, -half_width, half_width
    dx = (x1 - x0) / nx
    dy = (y1 - y0) / ny
    i = np.arange(nx, dtype=np.float64)
    j = np.arange(ny, dtype=np.float64)
    xc = x0 + (i + 0.5) * dx
    yc = y0 + (j + 0.5) * dy
    X, Y = np.meshgrid(xc, yc)
    r2 = X * X + Y * Y
    exp_half = np.exp(0.5 * (1.0 - r2))
    exp_full = np.exp(1.0 - r2)
    two_pi = 2.0 * math.pi
    prim = np.zeros((8, ny, nx))
    prim[0] = 1.0
    prim[1] = background[0] - kappa / two_pi * exp_half * Y
    prim[2] = background[1] + kappa / two_pi * exp_half * X
    prim[4] = 1.0 + (mu * mu * (1.0 - r2) - kappa * kappa) * exp_full / (8.0 * math.pi * math.pi)

    # corner potential A_z at (i+1/2, j+1/2); faces are its exact differences
    xf = x0 + (i + 1.0) * dx
    yf = y0 + (j + 1.0) * dy
    XF, YF = np.meshgrid(xf, yf)
    az_corner = mu / two_pi * np.exp(0.5 * (1.0 - (XF * XF + YF * YF)))
    # Bx(i+1/2, j) = (Az(i+1/2, j+1/2) - Az(i+1/2, j-1/2)) / dy, periodic
    bx = (az_corner - np.roll(az_corner, 1, axis=0)) / dy
    # By(i, j+1/2) = -(Az(i+1/2, j+1/2) - Az(i-1/2, j+1/2)) / dx
    by = -(az_corner - np.roll(az_corner, 1, axis=1)) / dx
    prim[5] = 0.5 * (np.roll(bx, 1, axis=1) + bx)
    prim[6] = 0.5 * (np.roll(by, 1, axis=0) + by)
    A = np.zeros((3, ny, nx))
    A[2] = mu / two_pi * exp_half
    return Problem("vortex", nx, ny, x0, x1, y0, y1, prim, np.ascontiguousarray(bx),
                   np.ascontiguousarray(by), A,
                   settings=dict(gamma=5.0 / 3.0, vortex_test=1))


def vortex_sheet(n: int = 1024, ny: int | None = None, gamma: float = 5.0 / 3.0) -> Problem:
    """Periodic vortex-sheet (Orszag-Tang type) field on [0, 2*pi]^2."""
    nx = n
    ny = n if ny is None else ny
    x0, x1, y0, y1 = 0.0, 2.0 * math.pi, 0.0, 2.0 * math.pi
    dx = (x1 - x0) / nx
    dy = (y1 - y0) / ny
    xc = x0 + (np.arange(nx) + 0.5) * dx
    yc = y0 + (np.arange(ny) + 0.5) * dy
    X, Y = np.meshgrid(xc, yc)
    prim = np.zeros((8, ny, nx))
    prim[0] = gamma * gamma
    prim[1] = -np.sin(Y)
    prim[2] = np.sin(X)
    prim[4] = gamma
    prim[5] = -np.sin(Y)
    prim[6] = np.sin(2.0 * X)
    bx = 0.5 * (prim[5] + np.roll(prim[5], -1, axis=1))
    by = 0.5 * (prim[6] + np.roll(prim[6], -1, axis=0))
    A = np.zeros((3, ny, nx))
    A[2] = np.cos(Y) + 0.5 * np.cos(2.0 * X)
    return Problem("vortex_sheet", nx, ny, x0, x1, y0, y1, prim, bx, by, A,
                   settings=dict(gamma=gamma, vortex_test=0))
