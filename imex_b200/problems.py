"""Initial data for the benchmark and test workloads (analytic or seeded).

Every field is returned as interior-only SoA planes of shape (ny, nx), index
[j, i] with x fastest in memory, which is the layout the C ABI takes:

    prim  (8, ny, nx): rho, vx, vy, vz, p, Bx, By, Bz   (cell averages)
    bx    (ny, nx)   : Bx on the x-face (i+1/2, j)
    by    (ny, nx)   : By on the y-face (i, j+1/2)
    A     (3, ny, nx): vector potential at cell centres
    bx_x0 (ny,), by_y0 (nx,): only for a transmissive direction, the boundary normal
                       faces Bx(x_0, j) and By(i, y_0), which a periodic direction
                       identifies with the faces at x_1 / y_1

Formulas follow the reference's initial conditions:
  * vortex:  initial_conditions.cpp:641-669 (cell state) and :698-717 (faces
    from corner A_z, cell B = face average), A_initial
    constrained_transport.cpp:389-394, generalised by the background flow
    (1,1) and the kappa/mu amplitudes of the vortex workload;
  * vortex sheet: the Orszag-Tang field of initial_conditions.cpp:426-435 in
    [0, 2*pi]^2 form, faces = average of neighbouring cell B as in
    initial_conditions.cpp:720-726, A_z = cos y + cos(2x)/2;
  * random field: seeded low-Mach, magnetic-pressure-dominated Redlich-Kwong gas on
    the unit square (random Fourier sums; faces from a corner A_z as for the vortex);
  * open blast: a smooth pressure pulse in an oblique field with a shearing flow on the
    open unit square (x_Transmissive, y_Transmissive as the reference's blast and
    shock-tube tests, main.cpp:9-60), with every field varying across the boundaries.
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
    bx_x0: np.ndarray | None = None
    by_y0: np.ndarray | None = None

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


class _FourierModes:
    """Random Fourier sum f(x, y) = sum_{0<|k|<=kmax} a_k |k|^-2 cos(2 pi k.x + phi_k)
    on the unit square, a_k ~ N(0, 1), phi_k ~ U[0, 2 pi).  Evaluated separably as
    Re(Ey^T C Ex) with C[ky, kx] = a_k |k|^-2 e^{i phi_k}; derivatives scale C by 2 pi i k."""

    def __init__(self, rng: np.random.Generator, kmax: int):
        n = 2 * kmax + 1
        self.kmax = kmax
        self.C = np.zeros((n, n), dtype=np.complex128)
        for ky in range(-kmax, kmax + 1):
            for kx in range(-kmax, kmax + 1):
                k2 = kx * kx + ky * ky
                if k2 == 0 or k2 > kmax * kmax:
                    continue
                a = rng.standard_normal()
                phi = rng.uniform(0.0, 2.0 * math.pi)
                self.C[ky + kmax, kx + kmax] = a / k2 * np.exp(1j * phi)

    def eval(self, x: np.ndarray, y: np.ndarray, dx: int = 0, dy: int = 0) -> np.ndarray:
        """f (or its derivative d^dx/dx^dx d^dy/dy^dy) on the grid y[:, None], x[None, :]."""
        k = np.arange(-self.kmax, self.kmax + 1)
        C = self.C * (2j * math.pi * k[None, :]) ** dx * (2j * math.pi * k[:, None]) ** dy
        Ex = np.exp(2j * math.pi * k[:, None] * x[None, :])
        Ey = np.exp(2j * math.pi * k[:, None] * y[None, :])
        return np.real(Ey.T @ C @ Ex)


def random_field(n: int = 2048, seed: int = 2026, p0: float = 1.0, mach: float = 1e-3, beta: float = 0.1,
                 kmax: int = 8, gamma: float = 5.0 / 3.0, m_alfa: float = 0.4275, m_b: float = 0.0866) -> Problem:
    """Low-Mach, magnetic-pressure-dominated random field on the periodic unit square,
    Redlich-Kwong gas.  From the seed: rho = 1 + 0.1 f1 and p = p0 (1 + 0.05 f2), with
    f1, f2 random Fourier sums normalised to max |f| = 1; v = curl(psi) of a random
    streamfunction scaled to max |v| = mach * sqrt(gamma p0 / rho0) (the ideal-gas sound
    speed at the mean state is the Mach reference); B from a random vector potential A_z
    on cell corners (faces = its exact differences, so div B = 0 to round-off; cell B =
    face average), scaled to beta = 2 p0 / max|B|^2.  The modes are drawn in a fixed order
    (f1, f2, psi, A_z) from numpy's default generator with this seed.

    The default beta is 0.1 (magnetic pressure ten times the gas pressure): with the
    Redlich-Kwong gas the reference scheme itself turns the state non-finite within two
    steps at beta <= 0.03 on this field, so stronger fields have no reference result to
    match."""
    rng = np.random.default_rng(seed)
    f1, f2, psi, az = (_FourierModes(rng, kmax) for _ in range(4))
    nx = ny = n
    h = 1.0 / n
    xc = (np.arange(n) + 0.5) * h
    xf = (np.arange(n) + 1.0) * h  # corners (i+1/2, j+1/2)
    prim = np.zeros((8, ny, nx))
    g1 = f1.eval(xc, xc)
    g2 = f2.eval(xc, xc)
    prim[0] = 1.0 + 0.1 * g1 / np.abs(g1).max()
    prim[4] = p0 * (1.0 + 0.05 * g2 / np.abs(g2).max())
    vx = psi.eval(xc, xc, dy=1)
    vy = -psi.eval(xc, xc, dx=1)
    vmax = np.sqrt(vx * vx + vy * vy).max()
    vscale = mach * math.sqrt(gamma * p0 / 1.0) / vmax
    prim[1] = vx * vscale
    prim[2] = vy * vscale
    a_corner = az.eval(xf, xf)
    bx = (a_corner - np.roll(a_corner, 1, axis=0)) / h
    by = -(a_corner - np.roll(a_corner, 1, axis=1)) / h
    cbx = 0.5 * (np.roll(bx, 1, axis=1) + bx)
    cby = 0.5 * (np.roll(by, 1, axis=0) + by)
    bscale = math.sqrt(2.0 * p0 / beta) / np.sqrt(cbx * cbx + cby * cby).max()
    bx *= bscale
    by *= bscale
    prim[5] = cbx * bscale
    prim[6] = cby * bscale
    A = np.zeros((3, ny, nx))
    A[2] = az.eval(xc, xc) * bscale
    return Problem("random_field", nx, ny, 0.0, 1.0, 0.0, 1.0, prim, np.ascontiguousarray(bx),
                   np.ascontiguousarray(by), A,
                   settings=dict(gamma=gamma, vortex_test=0, eos_type="REDLICH_KWONG", m_alfa=m_alfa, m_b=m_b))


def open_blast(n: int = 64, ny: int | None = None, b0: float = 0.5, angle: float = 0.3) -> Problem:
    """Smooth blast in an oblique field on the open square [-1/2, 1/2]^2 (transmissive in x
    and y, gamma = 5/3).  rho = 1 + 0.3 g(r, 0.15) + 0.1 x, p = 0.5 + 2 g(r, 0.1) with
    g(r, s) = exp(-r^2 / s^2); v = (0.3 + 0.2 y, -0.2 + 0.1 sin(2 pi x), 0.05 x); A_z on the
    (nx + 1) x (ny + 1) corners = b0 (y cos a - x sin a) + 0.05 g(r, 0.2), so the faces
    (boundary faces included) are its exact differences and div B = 0 to round-off; cell B
    = face average; B_z = 0.1 (1 + y)."""
    nx = n
    ny = n if ny is None else ny
    x0, x1, y0, y1 = -0.5, 0.5, -0.5, 0.5
    dx, dy = (x1 - x0) / nx, (y1 - y0) / ny
    xc = x0 + (np.arange(nx) + 0.5) * dx
    yc = y0 + (np.arange(ny) + 0.5) * dy
    X, Y = np.meshgrid(xc, yc)
    g = lambda x, y, s: np.exp(-(x * x + y * y) / (s * s))
    prim = np.zeros((8, ny, nx))
    prim[0] = 1.0 + 0.3 * g(X, Y, 0.15) + 0.1 * X
    prim[1] = 0.3 + 0.2 * Y
    prim[2] = -0.2 + 0.1 * np.sin(2.0 * math.pi * X)
    prim[3] = 0.05 * X
    prim[4] = 0.5 + 2.0 * g(X, Y, 0.1)
    ca, sa = math.cos(angle), math.sin(angle)
    az = lambda x, y: b0 * (y * ca - x * sa) + 0.05 * g(x, y, 0.2)
    xf = x0 + np.arange(nx + 1) * dx  # corners (i - 1/2) for i = 0..nx
    yf = y0 + np.arange(ny + 1) * dy
    XF, YF = np.meshgrid(xf, yf)  # (ny + 1, nx + 1)
    ac = az(XF, YF)
    bx_all = (ac[1:, :] - ac[:-1, :]) / dy  # (ny, nx + 1): Bx at x-faces i - 1/2, i = 0..nx
    by_all = -(ac[:, 1:] - ac[:, :-1]) / dx  # (ny + 1, nx): By at y-faces j - 1/2
    bx, bx_x0 = bx_all[:, 1:], bx_all[:, 0]
    by, by_y0 = by_all[1:, :], by_all[0, :]
    prim[5] = 0.5 * (bx_all[:, :-1] + bx_all[:, 1:])
    prim[6] = 0.5 * (by_all[:-1, :] + by_all[1:, :])
    prim[7] = 0.1 * (1.0 + Y)
    A = np.zeros((3, ny, nx))
    A[2] = az(X, Y)
    return Problem("open_blast", nx, ny, x0, x1, y0, y1, prim, np.ascontiguousarray(bx), np.ascontiguousarray(by),
                   A, settings=dict(gamma=5.0 / 3.0, vortex_test=0, x_bc="x_Transmissive", y_bc="y_Transmissive"),
                   bx_x0=np.ascontiguousarray(bx_x0), by_y0=np.ascontiguousarray(by_y0))


# The 2D problems of the reference's test catalogue: the settings main.cpp:124-178 gives each
# (domain, gamma, boundaries, end time), the cell states of u_initialization
# (initial_conditions.cpp:426-594, the shock-cloud at :464-484), the faces it averages from neighbouring cells under those
# boundaries (initial_conditions.cpp:716-722) and the A_z of A_initial
# (constrained_transport.cpp:233-260).  A0 is the reference's amplitude constant (config.hpp:59).
_A0 = 1e-3
_S4P = math.sqrt(4.0 * math.pi)
REFERENCE_TESTS = {
    # name: (enum ordinal in config.hpp:29, domain, gamma, x_bc, y_bc, time_stop)
    "Orszag_Tang": (15, (0.0, 1.0, 0.0, 1.0), 1.4, "x_Periodic", "y_Periodic", 1.0),
    "blastwave": (16, (-0.5, 0.5, -0.5, 0.5), 1.4, "x_Transmissive", "y_Transmissive", 0.01),
    "Rotor": (18, (-0.5, 0.5, -0.5, 0.5), 1.4, "x_Transmissive", "y_Transmissive", 0.25),
    "FieldLoop": (19, (-1.0, 1.0, -0.5, 0.5), 5.0 / 3.0, "x_Periodic", "y_Periodic", 1.0),
    "KHInstability": (20, (0.0, 2.0, -0.5, 0.5), 1.4, "x_Periodic", "y_Periodic", (4.8 / _A0) / 6.0),
    "blastwave2": (26, (-0.5, 0.5, -0.5, 0.5), 1.4, "x_Transmissive", "y_Transmissive", 0.001),
    "ShockCloud": (27, (0.0, 1.0, 0.0, 1.0), 5.0 / 3.0, "x_Transmissive", "y_Transmissive", 0.06),
}


def reference_test(name: str, n: int = 128, ny: int | None = None) -> Problem:
    """One of the reference's 2D test problems (REFERENCE_TESTS) on an n x ny grid."""
    _, (x0, x1, y0, y1), gamma, xbc, ybc, t_end = REFERENCE_TESTS[name]
    nx = n
    ny = n if ny is None else ny
    dx, dy = (x1 - x0) / nx, (y1 - y0) / ny
    X, Y = np.meshgrid(x0 + (np.arange(nx) + 0.5) * dx, y0 + (np.arange(ny) + 0.5) * dy)
    prim = np.zeros((8, ny, nx))
    az = np.zeros((ny, nx))
    pi = math.pi
    if name == "Orszag_Tang":
        prim[0] = gamma * gamma
        prim[1] = -np.sin(2 * pi * Y)
        prim[2] = np.sin(2 * pi * X)
        prim[4] = gamma
        prim[5] = -np.sin(2 * pi * Y)
        prim[6] = np.sin(4 * pi * X)
        az = np.cos(2.0 * pi * Y) / (2.0 * pi) + np.cos(4.0 * pi * X) / (4.0 * pi)
    elif name in ("blastwave", "blastwave2"):
        p_in, b0 = (1000.0, 70.0) if name == "blastwave" else (10000.0, 1000.0)
        rad = np.sqrt(X * X + Y * Y)
        eps = 1 * math.sqrt(dx * dx + dy * dy)
        erf = np.vectorize(math.erf)
        prim[0] = 1.0
        prim[4] = 0.5 * (0.1 + p_in) + 0.5 * (0.1 - p_in) * erf((rad - 0.1) / eps)
        prim[5] = b0 / math.sqrt(4.0 * pi)
        az = (1.0 / math.sqrt(4.0 * pi) * b0) * Y
    elif name == "Rotor":
        disc = np.sqrt(X * X + Y * Y) <= 0.1
        prim[0] = np.where(disc, 10.0, 1.0)
        prim[1] = np.where(disc, -10 * Y, 0.0)
        prim[2] = np.where(disc, 10 * X, 0.0)
        prim[4] = 1.0
        prim[5] = 2.5 / math.sqrt(4 * pi)
        az = (2.5 / math.sqrt(4.0 * pi)) * Y
    elif name == "FieldLoop":
        r = np.sqrt(X * X + Y * Y)
        loop = r < 0.3
        prim[0] = 1.0
        prim[1] = 2.0
        prim[2] = 1.0
        prim[4] = 1e5
        with np.errstate(divide="ignore", invalid="ignore"):
            prim[5] = np.where(loop, (-_A0 * Y / r) / math.sqrt(4 * pi), 0.0)
            prim[6] = np.where(loop, (_A0 * X / r) / math.sqrt(4 * pi), 0.0)
        az = np.where(r < 0.3, (_A0 / math.sqrt(4.0 * pi)) * (0.3 - r), 0.0)
    elif name == "KHInstability":
        Mx = _A0
        eta = np.where((Y >= -9.0 / 32.0) & (Y < -7.0 / 32.0), 0.5 * (1.0 + np.sin(16.0 * pi * (Y + 0.25))),
              np.where((Y >= -7.0 / 32.0) & (Y < 7.0 / 32.0), 1.0,
              np.where((Y >= 7.0 / 32.0) & (Y < 9.0 / 32.0), 0.5 * (1.0 - np.sin(16.0 * pi * (Y - 0.25))), 0.0)))
        prim[0] = 1.4
        prim[1] = Mx * (1.0 - 2.0 * eta)
        prim[2] = 0.1 * Mx * np.sin(2.0 * pi * X)
        prim[4] = 1.0
        prim[5] = 0.1 * Mx
        az = 0.1 * _A0 * Y
    elif name == "ShockCloud":
        post = X < 0.6  # the shocked gas left of x = 0.6; the cloud of radius 0.15 at (0.8, 0.5)
        cloud = np.sqrt((X - 0.8) * (X - 0.8) + (Y - 0.5) * (Y - 0.5)) < 0.15
        prim[0] = np.where(post, 3.86859, np.where(cloud, 10.0, 1.0))
        prim[1] = np.where(post, 0.0, -11.2536)
        prim[4] = np.where(post, 167.345, 1.0)
        prim[6] = np.where(post, 2.1826182, 0.56418958)
        prim[7] = np.where(post, -2.1826182, 0.56418958)
        az = np.where(post, -2.1826182 * X, -1.30957092 - 0.56418958 * (X - 0.6))
        ay = np.where(post, -2.1826182 * X, -1.30957092 + 0.56418958 * (X - 0.6))
    else:
        raise KeyError(name)
    # faces: the average of the two cells beside each face, the outer cell by the boundary rule
    def beside(a, axis, periodic):
        nxt = np.roll(a, -1, axis=axis)
        if not periodic:  # transmissive: the cell past the last one is the last one
            idx = [slice(None)] * 2
            idx[axis] = -1
            nxt[tuple(idx)] = a[tuple(idx)]
        return 0.5 * (a + nxt)
    bx = beside(prim[5], 1, xbc == "x_Periodic")
    by = beside(prim[6], 0, ybc == "y_Periodic")
    A = np.zeros((3, ny, nx))
    A[2] = az
    if name == "ShockCloud":
        A[1] = ay
    settings = dict(gamma=gamma, vortex_test=0, x_bc=xbc, y_bc=ybc, time_stop=t_end)
    lines = {}
    if xbc == "x_Transmissive" or ybc == "y_Transmissive":  # the boundary face averages its cell twice
        lines = dict(bx_x0=np.ascontiguousarray(0.5 * (prim[5][:, 0] + prim[5][:, 0])),
                     by_y0=np.ascontiguousarray(0.5 * (prim[6][0, :] + prim[6][0, :])))
    return Problem(name, nx, ny, x0, x1, y0, y1, prim, np.ascontiguousarray(bx), np.ascontiguousarray(by), A,
                   settings=settings, **lines)


def vortex_ensemble(members: int = 256, seed: int = 2026, smin: int = 64, smax: int = 512) -> list[Problem]:
    """Independent vortex runs (the vortex formulas above): per member kappa, mu ~ U[0.5, 1.5]
    and a square grid whose side is drawn log-uniformly from [smin, smax] and made even."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(members):
        kappa = rng.uniform(0.5, 1.5)
        mu = rng.uniform(0.5, 1.5)
        side = int(round(math.exp(rng.uniform(math.log(smin), math.log(smax)))))
        side += side % 2
        out.append(vortex(side, kappa=kappa, mu=mu))
    return out


@dataclass
class PerturbedVortex:
    """The vortex with a seeded smooth perturbation of v and A_z: 32 Fourier modes, the first
    16 a streamfunction of the velocity (divergence-free), the last 16 the corner potential A_z
    (faces from its exact differences, cell B = face average).  The initial fields are linear
    in the mode amplitudes a: prim = base.prim + sum_m a_m dprim[m], likewise bx, by."""
    base: Problem
    dprim: np.ndarray  # (32, 4, ny, nx): the perturbed primitive planes PLANES = vx, vy, Bx, By
    dbx: np.ndarray    # (32, ny, nx)
    dby: np.ndarray
    amplitudes: np.ndarray  # (32,) the nominal amplitudes
    PLANES = (1, 2, 5, 6)

    def problem(self, a: np.ndarray | None = None) -> Problem:
        a = self.amplitudes if a is None else np.asarray(a, dtype=np.float64)
        b = self.base
        prim = b.prim.copy()
        prim[list(self.PLANES)] += np.tensordot(a, self.dprim, axes=1)
        bx = b.bx + np.tensordot(a, self.dbx, axes=1)
        by = b.by + np.tensordot(a, self.dby, axes=1)
        return Problem("perturbed_vortex", b.nx, b.ny, b.x0, b.x1, b.y0, b.y1, prim, np.ascontiguousarray(bx),
                       np.ascontiguousarray(by), b.A.copy(), settings=dict(b.settings))


def perturbed_vortex(n: int = 512, seed: int = 2026, amplitude: float = 1e-2, modes: int = 32,
                     kmax: int = 3) -> PerturbedVortex:
    """Adjoint workload: vortex(n) plus `modes` seeded Fourier modes (integer wavenumbers
    |k_x|, |k_y| <= kmax on the periodic square, uniform phases) of the velocity streamfunction
    (first half) and of A_z (second half), nominal amplitudes `amplitude` times N(0, 1)."""
    base = vortex(n)
    nx = ny = n
    L = base.x1 - base.x0
    dx, dy = base.dx, base.dy
    rng = np.random.default_rng(seed)
    xc = base.x0 + (np.arange(nx) + 0.5) * dx
    yc = base.y0 + (np.arange(ny) + 0.5) * dy
    X, Y = np.meshgrid(xc, yc)
    XF, YF = np.meshgrid(base.x0 + (np.arange(nx) + 1.0) * dx, base.y0 + (np.arange(ny) + 1.0) * dy)
    dprim = np.zeros((modes, 4, ny, nx))
    dbx = np.zeros((modes, ny, nx))
    dby = np.zeros((modes, ny, nx))
    for m in range(modes):
        while True:
            kx, ky = rng.integers(-kmax, kmax + 1, size=2)
            if kx or ky:
                break
        phase = rng.uniform(0.0, 2.0 * math.pi)
        wx, wy = 2.0 * math.pi * kx / L, 2.0 * math.pi * ky / L
        knorm = math.hypot(wx, wy)
        if m < modes // 2:
            # psi = cos(w.x + phase) / |w|: v = (d psi / dy, -d psi / dx)
            s = -np.sin(wx * X + wy * Y + phase) / knorm
            dprim[m, 0] = wy * s
            dprim[m, 1] = -wx * s
        else:
            az = np.cos(wx * XF + wy * YF + phase) / (knorm * knorm)
            bxm = (az - np.roll(az, 1, axis=0)) / dy
            bym = -(az - np.roll(az, 1, axis=1)) / dx
            dbx[m] = bxm
            dby[m] = bym
            dprim[m, 2] = 0.5 * (np.roll(bxm, 1, axis=1) + bxm)
            dprim[m, 3] = 0.5 * (np.roll(bym, 1, axis=0) + bym)
    amps = amplitude * rng.standard_normal(modes)
    return PerturbedVortex(base, dprim, dbx, dby, amps)


# ---- state files (the layout of imex_save_state_file / imex_load_state_file)
# header: 8-byte magic, int32 version, nx, ny, timestep, then float64 t, prev_dt, dt, x0, x1,
# y0, y1; then float64 planes prim (8), bx, by, A (3), each ny x nx with x fastest.
STATE_MAGIC = b"IMEXSTAT"
_STATE_HEADER = np.dtype([("magic", "S8"), ("version", "<i4"), ("nx", "<i4"), ("ny", "<i4"),
                          ("timestep", "<i4"), ("t", "<f8"), ("prev_dt", "<f8"), ("dt", "<f8"),
                          ("x0", "<f8"), ("x1", "<f8"), ("y0", "<f8"), ("y1", "<f8")])


def write_state_file(prob: Problem, path: str, t: float = 0.0, timestep: int = 0, prev_dt: float = 0.0) -> None:
    """The initial state of a problem as a state file (the input of the imex_run driver).  A
    problem with boundary normal faces (transmissive) writes version 2, which appends them."""
    lines = prob.bx_x0 is not None
    h = np.zeros((), dtype=_STATE_HEADER)
    h["magic"], h["version"], h["nx"], h["ny"], h["timestep"] = STATE_MAGIC, 2 if lines else 1, prob.nx, prob.ny, timestep
    h["t"], h["prev_dt"], h["dt"] = t, prev_dt, 0.0
    h["x0"], h["x1"], h["y0"], h["y1"] = prob.x0, prob.x1, prob.y0, prob.y1
    with open(path, "wb") as f:
        f.write(h.tobytes())
        for a in (prob.prim, prob.bx, prob.by, prob.A) + ((prob.bx_x0, prob.by_y0) if lines else ()):
            f.write(np.ascontiguousarray(a, dtype="<f8").tobytes())


def read_state_file(path: str) -> tuple[dict, np.ndarray, np.ndarray, np.ndarray, np.ndarray]:
    """(header, prim, bx, by, A) of a state file; a version-2 file's boundary normal faces are
    in header["bx_x0"] / header["by_y0"]."""
    with open(path, "rb") as f:
        raw = f.read()
    h = np.frombuffer(raw[:_STATE_HEADER.itemsize], dtype=_STATE_HEADER)[0]
    if bytes(h["magic"]) != STATE_MAGIC:
        raise ValueError(f"{path} is not a state file")
    nx, ny = int(h["nx"]), int(h["ny"])
    d = np.frombuffer(raw[_STATE_HEADER.itemsize:], dtype="<f8")
    N = nx * ny
    extra = nx + ny if int(h["version"]) == 2 else 0
    if d.size != 13 * N + extra:
        raise ValueError(f"{path}: expected {13 * N + extra} values, found {d.size}")
    prim = d[:8 * N].reshape(8, ny, nx)
    bx, by = d[8 * N:9 * N].reshape(ny, nx), d[9 * N:10 * N].reshape(ny, nx)
    A = d[10 * N:13 * N].reshape(3, ny, nx)
    header = {n: (h[n].item() if n != "magic" else bytes(h[n])) for n in _STATE_HEADER.names}
    if extra:
        header["bx_x0"], header["by_y0"] = d[13 * N:13 * N + ny].copy(), d[13 * N + ny:].copy()
    return header, prim.copy(), bx.copy(), by.copy(), A.copy()
