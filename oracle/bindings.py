"""ctypes bindings for the two CPU oracles (test infrastructure only).

* ``RefSolver``  - the reference solver's own code built by ``make -C oracle ref``
  into ``oracle/_ref/libimexref.so`` (see oracle/ref/ref_harness.cpp);
* ``PortSolver`` - the plain-C restatement ``oracle/imex_oracle.c`` built into
  ``oracle/liboracle.so``.

Both expose the same interface, so a test can run either one as the checker.
Only tests/, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg use
this module; the product never imports it.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_LIB = os.path.join(HERE, "_ref", "libimexref.so")
PORT_LIB = os.path.join(HERE, "liboracle.so")

# enum ordinals of include/config.hpp:27-41,118
FORMULA = {"EnergyFormula": 0, "PressureFormula": 1}
MAGFIELD = {"StaggerCT": 0, "UnStaggerCT": 1, "PotentialA": 2, "NoDivFree": 3}
RECON = {"NoRecon": 0, "Minmod": 1, "VanLeer": 2, "ENO3": 3, "WENO5": 4}
RECONSTATE = {"PrimState": 0, "ConsState": 1}
DTCALC = {"Fullydt": 0, "Alfvendt": 1, "IMEXdt": 2}
PVISC = {"MaterialSpeedp": 0, "AlfvenSpeedp": 1, "Noaddvisp": 2}
UUPDATE = {"ConservationofU": 0, "DefinitionofU": 1}
PSOLVER = {"no_correction": 0, "once_correction": 1, "all_correction": 2}
EOS = {"IDEAL_GAS": 0, "REDLICH_KWONG": 1}
XBC = {"x_Transmissive": 0, "x_Reflective": 1, "x_Periodic": 2, "x_Dirichlet": 3}
YBC = {"y_Transmissive": 0, "y_Reflective": 1, "y_Periodic": 2, "y_Dirichlet": 3, "y_JetInflow": 4}

# reference defaults, include/config.hpp:43-125
DEFAULTS = dict(
    formula="PressureFormula", magfield="NoDivFree", recon="Minmod", reconstate="ConsState",
    caltimestep="IMEXdt", add_pvisc="MaterialSpeedp", U_update="DefinitionofU",
    PressureSolver="all_correction", eos_type="IDEAL_GAS", GLF=1, add_bvisc=1, floor_on=1,
    Energy_modify=0, vortex_test=1, Pnewton_max=20, CFL=0.8, GMREStol=1e-14,
    gamma=5.0 / 3.0, p_floor=1e-7, Mbig_fac=1e6, theta=0.9, Pnewton_tol=1e-8,
    shock_kappa1=0.001, m_alfa=0.05, m_b=0.1, m_R=0.4, m_cv=1.0, time_stop=1e30, fixed_dt=0.0,
)

_ENUMS = dict(formula=FORMULA, magfield=MAGFIELD, recon=RECON, reconstate=RECONSTATE,
              caltimestep=DTCALC, add_pvisc=PVISC, U_update=UUPDATE, PressureSolver=PSOLVER,
              eos_type=EOS)


class Params(C.Structure):
    """Layout of ``ref_params`` (ref_harness.cpp) and ``ora_params`` (imex_oracle.h)."""
    _fields_ = [(n, C.c_int) for n in (
        "formula", "magfield", "recon", "reconstate", "caltimestep", "add_pvisc", "U_update",
        "PressureSolver", "eos_type", "GLF", "add_bvisc", "floor_on", "Energy_modify",
        "vortex_test", "Pnewton_max")] + [(n, C.c_double) for n in (
        "CFL", "GMREStol", "gamma_plasma", "p_floor", "Mbig_fac", "theta", "Pnewton_tol",
        "shock_kappa1", "m_alfa", "m_b", "m_R", "m_cv", "x0", "x1", "y0", "y1", "time_stop",
        "fixed_dt")]


def make_params(settings: dict, domain: tuple[float, float, float, float]) -> Params:
    s = dict(DEFAULTS)
    s.update(settings)
    p = Params()
    for name, table in _ENUMS.items():
        v = s[name]
        setattr(p, name, table[v] if isinstance(v, str) else int(v))
    for name in ("GLF", "add_bvisc", "floor_on", "Energy_modify", "vortex_test", "Pnewton_max"):
        setattr(p, name, int(s[name]))
    p.gamma_plasma = float(s["gamma"])
    for name in ("CFL", "GMREStol", "p_floor", "Mbig_fac", "theta", "Pnewton_tol", "shock_kappa1",
                 "m_alfa", "m_b", "m_R", "m_cv", "time_stop", "fixed_dt"):
        setattr(p, name, float(s[name]))
    p.x0, p.x1, p.y0, p.y1 = (float(v) for v in domain)
    return p


def _dp(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _c(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float64)


SUB = dict(combine=0, convective=1, magnetic=2, pflux=3, pressure=4, ct=5)
SNAP = dict(u_con=0, Qe=1, Qs=2, bx=3, by=4, bxQs=5, byQs=6, A=7, A_s=8, Fx=9, Fy=10)


class _Solver:
    prefix = ""
    libpath = ""
    _lib_cache: dict = {}

    def __init__(self, nx: int, ny: int, rks: int, settings: dict,
                 domain: tuple[float, float, float, float]):
        self.lib = self._load()
        self.nx, self.ny, self.rks = nx, ny, rks
        self.N = nx * ny
        self.params = make_params(settings, domain)
        rc = self._f("setup")(nx, ny, rks, C.byref(self.params))
        if rc != 0:
            raise RuntimeError(f"{self.prefix}setup failed ({rc})")

    @classmethod
    def available(cls) -> bool:
        return os.path.exists(cls.libpath)

    @classmethod
    def _load(cls):
        if cls.libpath not in _Solver._lib_cache:
            if not os.path.exists(cls.libpath):
                raise FileNotFoundError(f"{cls.libpath} missing; run `make -C oracle`")
            lib = C.CDLL(cls.libpath)
            p = cls.prefix
            D = C.POINTER(C.c_double)
            sig = {
                "setup": (C.c_int, [C.c_int, C.c_int, C.c_int, C.POINTER(Params)]),
                "load_prim": (C.c_int, [D, D, D, D]),
                "step": (C.c_double, [C.c_int]),
                "get_cons": (None, [D]), "get_prim": (None, [D]), "get_faces": (None, [D, D]),
                "get_A": (None, [D]), "get_Hs": (None, [C.c_int, D, D, D]),
                "get_scalars": (None, [D]), "set_scalars": (None, [D]),
                "get_tableau": (None, [D, D]),
                "get_snapshot": (C.c_int, [C.c_int, C.c_int, C.c_int, D]),
                "fn_reconstruct": (None, [D, D]), "fn_shock": (None, [D, D]),
                "fn_operator": (None, [C.c_int, D, D, D, C.c_double, D, C.c_double, D, D]),
                "fn_nested_newton": (None, [D, D, D, C.c_double, D, D]),
                "fn_substep": (None, [C.c_int, C.c_double, C.c_int, D, D, D, D, D, D, D, D, D,
                                      D, D]),
                "div_error": (C.c_double, []),
                "set_bc": (C.c_int, [C.c_int, C.c_int]),
                "set_boundary_faces": (None, [D, D]), "get_boundary_faces": (None, [D, D]),
                "get_snapshot_boundary": (C.c_int, [C.c_int, C.c_int, C.c_int, D]),
            }
            for name, (res, args) in sig.items():
                fn = getattr(lib, p + name)
                fn.restype = res
                fn.argtypes = args
            _Solver._lib_cache[cls.libpath] = lib
        return _Solver._lib_cache[cls.libpath]

    def _f(self, name):
        return getattr(self.lib, self.prefix + name)

    # ---- boundaries ----------------------------------------------------
    def set_bc(self, x_bc, y_bc) -> None:
        """x_bc / y_bc as names or ordinals (config.hpp:36-37); call before load()."""
        xb = XBC[x_bc] if isinstance(x_bc, str) else int(x_bc)
        yb = YBC[y_bc] if isinstance(y_bc, str) else int(y_bc)
        if self._f("set_bc")(xb, yb) != 0:
            raise RuntimeError(f"{self.prefix}set_bc({x_bc}, {y_bc}) refused")

    def set_boundary_faces(self, bx_x0, by_y0) -> None:
        """Bx on x = x_0 (ny values) and By on y = y_0 (nx values)."""
        bx0, by0 = _c(bx_x0), _c(by_y0)
        assert bx0.size == self.ny and by0.size == self.nx
        self._f("set_boundary_faces")(_dp(bx0), _dp(by0))

    def boundary_faces(self) -> tuple[np.ndarray, np.ndarray]:
        bx0, by0 = np.empty(self.ny), np.empty(self.nx)
        self._f("get_boundary_faces")(_dp(bx0), _dp(by0))
        return bx0, by0

    def snapshot_boundary(self, rks: int, sub: str, which: str) -> np.ndarray | None:
        w = SNAP[which]
        out = np.zeros(self.ny if w in (3, 5) else self.nx)
        rc = self._f("get_snapshot_boundary")(rks, SUB[sub], w, _dp(out))
        return None if rc != 0 else out

    # ---- whole steps -------------------------------------------------
    def load(self, prob) -> None:
        prim, bx, by, A = _c(prob.prim), _c(prob.bx), _c(prob.by), _c(prob.A)
        rc = self._f("load_prim")(_dp(prim), _dp(bx), _dp(by), _dp(A))
        if rc != 0:
            raise RuntimeError("load_prim failed")

    def step(self, snapshots: bool = False) -> float:
        return self._f("step")(1 if snapshots else 0)

    def cons(self) -> np.ndarray:
        out = np.empty((8, self.ny, self.nx))
        self._f("get_cons")(_dp(out))
        return out

    def prim(self) -> np.ndarray:
        out = np.empty((8, self.ny, self.nx))
        self._f("get_prim")(_dp(out))
        return out

    def faces(self) -> tuple[np.ndarray, np.ndarray]:
        bx = np.empty((self.ny, self.nx))
        by = np.empty((self.ny, self.nx))
        self._f("get_faces")(_dp(bx), _dp(by))
        return bx, by

    def vector_potential(self) -> np.ndarray:
        out = np.empty((3, self.ny, self.nx))
        self._f("get_A")(_dp(out))
        return out

    def stage_derivative(self, r: int):
        hs = np.empty((8, self.ny, self.nx))
        hsa = np.empty((3, self.ny, self.nx))
        hsb = np.empty((2, self.ny, self.nx))
        self._f("get_Hs")(r, _dp(hs), _dp(hsa), _dp(hsb))
        return hs, hsa, hsb

    SCALARS = ("dt", "adt", "B_max_x", "B_max_y", "vx_max", "vy_max", "a_max", "t", "ch",
               "v_max", "timestep", "Mbig", "max_floored", "min_p_ever")

    def scalars(self) -> dict:
        out = np.zeros(14)
        self._f("get_scalars")(_dp(out))
        return dict(zip(self.SCALARS, out.tolist()))

    def set_scalars(self, dt, adt, bmx, bmy, vxm, vym, amax) -> None:
        a = np.array([dt, adt, bmx, bmy, vxm, vym, amax], dtype=np.float64)
        self._f("set_scalars")(_dp(a))

    def tableau(self):
        ae = np.zeros(self.rks * self.rks)
        ai = np.zeros(self.rks * self.rks)
        self._f("get_tableau")(_dp(ae), _dp(ai))
        return ae.reshape(self.rks, self.rks), ai.reshape(self.rks, self.rks)

    def snapshot(self, rks: int, sub: str, which: str) -> np.ndarray | None:
        w = SNAP[which]
        shape = {0: (8,), 1: (8,), 2: (8,), 7: (3,), 8: (3,)}.get(w, ())
        out = np.zeros(shape + (self.ny, self.nx))
        rc = self._f("get_snapshot")(rks, SUB[sub], w, _dp(out))
        return None if rc != 0 else out

    def div_error(self) -> float:
        return self._f("div_error")()

    def init_test(self, test_id: int) -> dict:
        """The reference's own initial data of catalogue test `test_id` (reference library only)."""
        fn = self.lib.ref_init_test
        D = C.POINTER(C.c_double)
        fn.restype, fn.argtypes = C.c_int, [C.c_int, D, D, D, D, D, D]
        nx, ny = self.nx, self.ny
        out = dict(prim=np.empty((8, ny, nx)), bx=np.empty((ny, nx)), by=np.empty((ny, nx)), bx_x0=np.empty(ny),
                   by_y0=np.empty(nx), A=np.empty((3, ny, nx)))
        rc = fn(test_id, *(_dp(out[k]) for k in ("prim", "bx", "by", "bx_x0", "by_y0", "A")))
        if rc != 0:
            raise RuntimeError("ref_init_test failed")
        return out

    CT_DIAG_PARTS = ("central", "rusanov", "tilde", "TOTAL")

    def ct_diag(self) -> dict:
        """Diagnose_CT_EMF's figures on the current state: {part: (L2 Ez, max|Ez|, L2 dB/dt,
        max|dB/dt|)}.  The C restatement returns them at full precision; the reference's own
        function prints them (%.3e), and those printed lines are parsed."""
        if self.prefix == "ora_":
            out = np.zeros(16)
            fn = self.lib.ora_ct_diag
            fn.restype, fn.argtypes = None, [C.POINTER(C.c_double)]
            fn(_dp(out))
            return {name: tuple(out[4 * c:4 * c + 4].tolist()) for c, name in enumerate(self.CT_DIAG_PARTS)}
        import re
        import tempfile
        fn = self.lib.ref_ct_diag_print
        fn.restype, fn.argtypes = C.c_int, [C.c_char_p]
        with tempfile.NamedTemporaryFile("r", suffix=".txt") as f:
            if fn(f.name.encode()) != 0:
                raise RuntimeError("ref_ct_diag_print failed")
            text = open(f.name).read()
        out = {}
        for line in text.splitlines():
            m = re.match(r"\[CT-DIAG\]\s+(\S+)\s+Ez: L2=(\S+) max=(\S+) \| dB/dt: L2=(\S+) max=(\S+)", line)
            if m:
                out[m.group(1)] = tuple(float(v) for v in m.groups()[1:])
        return out

    # ---- single functions on caller-supplied state -------------------
    def reconstruct(self, Q: np.ndarray) -> np.ndarray:
        Q = _c(Q)
        out = np.zeros((4, 8, self.ny, self.nx))
        self._f("fn_reconstruct")(_dp(Q), _dp(out))
        return out

    def shock(self, Q: np.ndarray) -> np.ndarray:
        Q = _c(Q)
        out = np.zeros((self.ny, self.nx))
        self._f("fn_shock")(_dp(Q), _dp(out))
        return out

    def operator(self, op: int, ucon, Qe, Qs, h, x, pfreeze=None, mbig=0.0) -> np.ndarray:
        ucon, Qe, Qs, x = _c(ucon), _c(Qe), _c(Qs), _c(x)
        pf = _c(pfreeze) if pfreeze is not None else np.zeros(self.N)
        out = np.zeros_like(x)
        self._f("fn_operator")(op, _dp(ucon), _dp(Qe), _dp(Qs), h, _dp(pf), mbig, _dp(x),
                               _dp(out))
        return out

    def nested_newton(self, ucon, Qe, Qs, h, b, p0) -> np.ndarray:
        ucon, Qe, Qs, b = _c(ucon), _c(Qe), _c(Qs), _c(b)
        p = np.array(p0, dtype=np.float64, copy=True)
        self._f("fn_nested_newton")(_dp(ucon), _dp(Qe), _dp(Qs), h, _dp(b), _dp(p))
        return p

    def substep(self, sub: int, h: float, rks: int, ucon, Qe, Qs, bx, by, bxQs, byQs, A, A_s,
                Fx=None, Fy=None):
        ucon = np.array(ucon, dtype=np.float64, copy=True)
        bx = np.array(bx, dtype=np.float64, copy=True)
        by = np.array(by, dtype=np.float64, copy=True)
        A = np.array(A, dtype=np.float64, copy=True)
        Qe, Qs, bxQs, byQs, A_s = _c(Qe), _c(Qs), _c(bxQs), _c(byQs), _c(A_s)
        Fx = np.zeros((self.ny, self.nx)) if Fx is None else np.array(Fx, dtype=np.float64)
        Fy = np.zeros((self.ny, self.nx)) if Fy is None else np.array(Fy, dtype=np.float64)
        self._f("fn_substep")(sub, h, rks, _dp(ucon), _dp(Qe), _dp(Qs), _dp(bx), _dp(by),
                              _dp(bxQs), _dp(byQs), _dp(A), _dp(A_s), _dp(Fx), _dp(Fy))
        return dict(u_con=ucon, bx=bx, by=by, A=A, Fx=Fx, Fy=Fy)


class RefSolver(_Solver):
    """The reference's own solver (oracle/_ref/libimexref.so)."""
    prefix = "ref_"
    libpath = REF_LIB


class PortSolver(_Solver):
    """The C restatement (oracle/liboracle.so)."""
    prefix = "ora_"
    libpath = PORT_LIB


def make_solver(kind: str, prob, rks: int, settings: dict):
    cls = {"ref": RefSolver, "port": PortSolver}[kind]
    s = dict(prob.settings)
    s.update(settings)
    solver = cls(prob.nx, prob.ny, rks, s, (prob.x0, prob.x1, prob.y0, prob.y1))
    if "x_bc" in s or "y_bc" in s:
        solver.set_bc(s.get("x_bc", "x_Periodic"), s.get("y_bc", "y_Periodic"))
    solver.load(prob)
    if getattr(prob, "bx_x0", None) is not None:
        solver.set_boundary_faces(prob.bx_x0, prob.by_y0)
    return solver
