"""imex_b200: one IMEX-RK stage of the reference 2D ideal-MHD scheme on B200.

The product is ``libimex_b200.so`` (CUDA for sm_100a behind the C ABI of
``include/imex_b200.h``).  This module is a thin ctypes mirror of that ABI for
Python callers (tests, the benchmark).  It never computes anything itself:
if the shared library is missing it raises.

Names mirror the reference's interface: ``Solver.step()`` is one pass of
main.cpp:335-561, and the sub-step methods (``RusanovC_Update``,
``MagSubsystem_UpdateB``, ``PreSubsystem_Pressure`` ...) call the entry points
that replace the reference functions of the same names.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libimex_b200.so")

# enum ordinals of include/imex_b200.h (= reference include/config.hpp:27-41,118)
FORMULA = {"EnergyFormula": 0, "PressureFormula": 1}
MAGFIELD = {"StaggerCT": 0, "UnStaggerCT": 1, "PotentialA": 2, "NoDivFree": 3}
RECON = {"NoRecon": 0, "Minmod": 1, "VanLeer": 2, "ENO3": 3, "WENO5": 4}
RECONSTATE = {"PrimState": 0, "ConsState": 1}
DTCALC = {"Fullydt": 0, "Alfvendt": 1, "IMEXdt": 2}
PVISC = {"MaterialSpeedp": 0, "AlfvenSpeedp": 1, "Noaddvisp": 2}
UUPDATE = {"ConservationofU": 0, "DefinitionofU": 1}
PSOLVER = {"no_correction": 0, "once_correction": 1, "all_correction": 2}
EOS = {"IDEAL_GAS": 0, "REDLICH_KWONG": 1}
PRECISION = {"fp64": 0, "mixed": 1}
ARITH = {"exact": 0, "fast": 1}
XBC = {"x_Transmissive": 0, "x_Reflective": 1, "x_Periodic": 2, "x_Dirichlet": 3}
YBC = {"y_Transmissive": 0, "y_Reflective": 1, "y_Periodic": 2, "y_Dirichlet": 3, "y_JetInflow": 4}
ENUMS = dict(formula=FORMULA, magfield=MAGFIELD, recon=RECON, reconstate=RECONSTATE,
             caltimestep=DTCALC, add_pvisc=PVISC, U_update=UUPDATE, PressureSolver=PSOLVER,
             eos_type=EOS, precision=PRECISION, x_bc=XBC, y_bc=YBC, arith=ARITH)

OP = {"pressure_L": 0, "pressure_J": 1, "magnetic_B": 2, "magnetic_A": 3, "energy": 4}
BUF = {"cons": 0, "prim": 1, "cons_n": 2, "Qe": 3, "Qs": 4, "bx": 5, "by": 6, "bxQs": 7,
       "byQs": 8, "A": 9, "A_s": 10, "Fx": 11, "Fy": 12, "w": 13, "Hs": 14, "HsA": 15,
       "HsB": 16, "eta": 17, "bx_x0": 18, "by_y0": 19, "bxQs_x0": 20, "byQs_y0": 21}
BUF_PLANES = {"cons": 8, "prim": 8, "cons_n": 8, "Qe": 8, "Qs": 8, "bx": 1, "by": 1, "bxQs": 1,
              "byQs": 1, "A": 3, "A_s": 3, "Fx": 1, "Fy": 1, "w": 32, "Hs": 8, "HsA": 3,
              "HsB": 2, "eta": 1}
STATUS = {0: "ok", 1: "invalid argument", 2: "unsupported configuration", 3: "CUDA error",
          4: "GMRES reached its restart cap", 5: "nested Newton reached Pnewton_max",
          6: "non-finite value in a solve", 7: "pressure below theta*p_floor",
          8: "device barrier timed out", 9: "EOS Newton iteration hit its cap"}


class ImexError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"imex status {status} ({STATUS.get(status, '?')}): {msg}")
        self.status = status


class Config(C.Structure):
    """imex_config (include/imex_b200.h)."""
    _fields_ = [
        ("caltimestep", C.c_int), ("formula", C.c_int), ("magfield", C.c_int),
        ("add_pvisc", C.c_int), ("flux_diss", C.c_int), ("GLF", C.c_int), ("add_bvisc", C.c_int),
        ("U_update", C.c_int), ("vortex_test", C.c_int), ("RKs", C.c_int), ("CFL", C.c_double),
        ("recon", C.c_int), ("reconstate", C.c_int), ("x_bc", C.c_int), ("y_bc", C.c_int),
        ("PressureSolver", C.c_int), ("Energy_Modify", C.c_int), ("GMREStol", C.c_double),
        ("shock_kappa1", C.c_double), ("floor_on", C.c_int), ("p_floor", C.c_double),
        ("Mbig_fac", C.c_double), ("theta", C.c_double), ("Pnewton_max", C.c_int),
        ("Pnewton_tol", C.c_double), ("eos_type", C.c_int), ("gamma_plasma", C.c_double),
        ("m_alfa", C.c_double), ("m_b", C.c_double), ("m_R", C.c_double), ("m_cv", C.c_double),
        ("x_0", C.c_double), ("x_1", C.c_double), ("y_0", C.c_double), ("y_1", C.c_double),
        ("time_stop", C.c_double), ("fixed_dt", C.c_double), ("gmres_restart", C.c_int),
        ("gmres_max_restarts", C.c_int), ("precision", C.c_int), ("mixed_inner_tol", C.c_double),
        ("mixed_max_refine", C.c_int), ("mixed_solves", C.c_int), ("mixed_outer_tol", C.c_double),
        ("arith", C.c_int),
    ]


class StepScalars(C.Structure):
    _fields_ = [(n, C.c_double) for n in ("dt", "adt", "B_max_x", "B_max_y", "vx_max", "vy_max",
                                          "v_max", "a_max", "ch", "cA_x", "cA_y", "t")] + [
        ("timestep", C.c_int)]


class SolveStats(C.Structure):
    _fields_ = [(n, C.c_int) for n in ("gmres_solves", "gmres_iters", "gmres_restarts",
                                       "newton_iters", "max_floored", "refine_sweeps")] + [
        ("last_residual", C.c_double), ("min_p", C.c_double), ("status", C.c_int)]

    def as_dict(self) -> dict:
        return {n: getattr(self, n) for n, _ in self._fields_}


class BatchTuning(C.Structure):
    _fields_ = [("streams", C.c_int), ("gmres_restart", C.c_int), ("ms_per_step", C.c_double),
                ("mixed_solves", C.c_int), ("solve_tile_x", C.c_int), ("solve_tile_y", C.c_int)]


class Diagnostics(C.Structure):
    _fields_ = [("timestep", C.c_int), ("t", C.c_double), ("dt", C.c_double), ("div_error", C.c_double),
                ("B_inf", C.c_double), ("dt_comp", C.c_double), ("emin", C.c_double), ("emin_x", C.c_double),
                ("emin_y", C.c_double), ("mass", C.c_double), ("intE", C.c_double), ("magE_max", C.c_double)]

    def as_dict(self) -> dict:
        return {n: getattr(self, n) for n, _ in self._fields_}


class AdjointOpts(C.Structure):
    _fields_ = [("nsteps", C.c_int), ("checkpoint_every", C.c_int), ("gmres_tol", C.c_double)]


class KernelProfile(C.Structure):
    _fields_ = [("name", C.c_char * 32), ("launches", C.c_longlong), ("total_ms", C.c_double),
                ("alg_bytes", C.c_double)]


_D = C.POINTER(C.c_double)
_SIGS = {
    "imex_config_default": (None, [C.POINTER(Config)]),
    "imex_create": (C.c_int, [C.POINTER(Config), C.c_int, C.c_int, C.POINTER(C.c_void_p)]),
    "imex_destroy": (C.c_int, [C.c_void_p]),
    "imex_set_stream": (C.c_int, [C.c_void_p, C.c_void_p]),
    "imex_synchronize": (C.c_int, [C.c_void_p]),
    "imex_status_string": (C.c_char_p, [C.c_int]),
    "imex_last_error": (C.c_char_p, [C.c_void_p]),
    "imex_get_config": (C.c_int, [C.c_void_p, C.POINTER(Config)]),
    "imex_upload_prim": (C.c_int, [C.c_void_p, _D, _D, _D, _D]),
    "imex_upload_state": (C.c_int, [C.c_void_p, _D, _D, _D, _D]),
    "imex_download_state": (C.c_int, [C.c_void_p, _D, _D, _D, _D, _D]),
    "imex_set_boundary_faces": (C.c_int, [C.c_void_p, _D, _D]),
    "imex_ct_emf_diagnostics": (C.c_int, [C.c_void_p, _D]),
    "imex_get_boundary_faces": (C.c_int, [C.c_void_p, _D, _D]),
    "imex_step": (C.c_int, [C.c_void_p, _D]),
    "imex_begin_step": (C.c_int, [C.c_void_p]),
    "imex_stage": (C.c_int, [C.c_void_p, C.c_int]),
    "imex_end_step": (C.c_int, [C.c_void_p]),
    "imex_set_step_scalars": (C.c_int, [C.c_void_p, C.POINTER(StepScalars)]),
    "imex_get_step_scalars": (C.c_int, [C.c_void_p, C.POINTER(StepScalars)]),
    "imex_stage_combine": (C.c_int, [C.c_void_p, C.c_int]),
    "imex_TVDReconstruction": (C.c_int, [C.c_void_p]),
    "imex_RusanovC_Update": (C.c_int, [C.c_void_p, C.c_double, C.c_int]),
    "imex_MagSubsystem_UpdateB": (C.c_int, [C.c_void_p, C.c_double, C.c_int]),
    "imex_MagSubsystem_UpdateA": (C.c_int, [C.c_void_p, C.c_double, C.c_int]),
    "imex_Pressure_flux_Update": (C.c_int, [C.c_void_p, C.c_double, C.c_int]),
    "imex_PreSubsystem_Pressure": (C.c_int, [C.c_void_p, C.c_double, C.c_int]),
    "imex_PreSubsystem_Energy": (C.c_int, [C.c_void_p, C.c_double, C.c_int]),
    "imex_Energy_flux_Update": (C.c_int, [C.c_void_p, C.c_double, C.c_int]),
    "imex_Staggered_CT_Consistent": (C.c_int, [C.c_void_p, C.c_double, C.c_int]),
    "imex_Unstaggered_CT_Consistent": (C.c_int, [C.c_void_p, C.c_double, C.c_int]),
    "imex_Staggered_CT": (C.c_int, [C.c_void_p, C.c_double, C.c_int]),
    "imex_Unstaggered_CT": (C.c_int, [C.c_void_p, C.c_double, C.c_int]),
    "imex_stage_derivative": (C.c_int, [C.c_void_p, C.c_int]),
    "imex_buffer_count": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(C.c_size_t)]),
    "imex_set_buffer": (C.c_int, [C.c_void_p, C.c_int, C.c_int, _D]),
    "imex_get_buffer": (C.c_int, [C.c_void_p, C.c_int, C.c_int, _D]),
    "imex_prepare_operator": (C.c_int, [C.c_void_p, C.c_int, C.c_double]),
    "imex_set_newton_state": (C.c_int, [C.c_void_p, _D, C.c_double]),
    "imex_apply_operator": (C.c_int, [C.c_void_p, C.c_int, _D, _D]),
    "imex_gmres": (C.c_int, [C.c_void_p, C.c_int, _D, _D, C.POINTER(SolveStats)]),
    "imex_diagnostics": (C.c_int, [C.c_void_p, C.POINTER(Diagnostics)]),
    "imex_write_vtk": (C.c_int, [C.c_void_p, C.c_char_p, C.c_int]),
    "imex_write_fields_dat": (C.c_int, [C.c_void_p, C.c_char_p]),
    "imex_save_state_file": (C.c_int, [C.c_void_p, C.c_char_p]),
    "imex_load_state_file": (C.c_int, [C.c_void_p, C.c_char_p]),
    "imex_vtk_write_host": (C.c_int, [C.c_char_p, C.c_int, C.c_int, C.c_double, C.c_double, C.c_double,
                                      C.c_double, C.c_double, C.c_int, _D, _D]),
    "imex_dat_write_host": (C.c_int, [C.c_char_p, C.c_int, C.c_int, C.c_double, C.c_double, C.c_double,
                                      C.c_double, _D]),
    "imex_history_write_host": (C.c_int, [C.c_char_p, C.c_int, C.POINTER(C.c_int), _D]),
    "imex_adjoint_run": (C.c_int, [C.c_void_p, C.POINTER(AdjointOpts), _D, _D, _D, _D, _D, _D]),
    "imex_adjoint_vjp": (C.c_int, [C.c_void_p, C.POINTER(AdjointOpts), _D, _D, _D, _D, _D, _D]),
    "imex_gmres_noalloc": (C.c_int, [C.c_void_p, C.c_int, _D, _D, C.POINTER(SolveStats)]),
    "imex_batch_create": (C.c_int, [C.POINTER(Config), C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int),
                                    C.POINTER(C.c_void_p)]),
    "imex_batch_destroy": (C.c_int, [C.c_void_p]),
    "imex_batch_member": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(C.c_void_p)]),
    "imex_batch_configure": (C.c_int, [C.c_void_p, C.c_int, C.c_int]),
    "imex_batch_step": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(C.c_double)]),
    "imex_batch_autotune": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(BatchTuning)]),
    "imex_batch_info": (C.c_int, [C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int)]),
    "imex_batch_set_solve_tile": (C.c_int, [C.c_void_p, C.c_int]),
    "imex_batch_explicit_launches": (C.c_int, [C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_int)]),
    "imex_batch_last_error": (C.c_char_p, [C.c_void_p]),
    "imex_pressure_nested_newton": (C.c_int, [C.c_void_p, _D, _D, C.POINTER(SolveStats)]),
    "imex_shock_detector": (C.c_int, [C.c_void_p, _D, _D]),
    "imex_get_stats": (C.c_int, [C.c_void_p, C.POINTER(SolveStats)]),
    "imex_reset_stats": (C.c_int, [C.c_void_p]),
    "imex_divergence": (C.c_int, [C.c_void_p, _D, _D, _D, _D]),
    "imex_min_pressure": (C.c_int, [C.c_void_p, _D]),
    "imex_profile_enable": (C.c_int, [C.c_void_p, C.c_int]),
    "imex_profile_read": (C.c_int, [C.c_void_p, C.POINTER(KernelProfile), C.c_int,
                                    C.POINTER(C.c_int)]),
    "imex_kernel_launch_count": (C.c_int, [C.c_void_p, C.POINTER(C.c_longlong)]),
    "imex_set_barrier_timeout": (C.c_int, [C.c_void_p, C.c_double]),
    "imex_selftest_barrier": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_double, _D]),
    "imex_selftest_fp64": (C.c_int, [C.c_void_p, _D, _D]),
}

_lib = None


def load_library(path: str = LIB_PATH):
    """Load libimex_b200.so and declare every exported signature (raises if absent)."""
    global _lib
    if _lib is None:
        if not os.path.exists(path):
            raise ImportError(f"{path} is missing; build it with `python -m imex_b200.build` "
                              "(there is no CPU fallback)")
        lib = C.CDLL(path)
        for name, (res, args) in _SIGS.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
    return _lib


def exported_symbols() -> list[str]:
    return sorted(_SIGS)


def default_config() -> Config:
    cfg = Config()
    load_library().imex_config_default(C.byref(cfg))
    return cfg


def make_config(settings: dict | None = None, domain=None, rks: int | None = None) -> Config:
    """imex_config from reference-style settings (string enums or ordinals)."""
    cfg = default_config()
    s = dict(settings or {})
    if "gamma" in s:
        s["gamma_plasma"] = s.pop("gamma")
    if "Energy_modify" in s:
        s["Energy_Modify"] = s.pop("Energy_modify")
    for key, val in s.items():
        if key in ENUMS and isinstance(val, str):
            val = ENUMS[key][val]
        if not hasattr(cfg, key):
            raise KeyError(f"unknown setting {key}")
        ftype = dict(Config._fields_)[key]
        setattr(cfg, key, int(val) if ftype is C.c_int else float(val))
    if domain is not None:
        cfg.x_0, cfg.x_1, cfg.y_0, cfg.y_1 = (float(v) for v in domain)
    if rks is not None:
        cfg.RKs = int(rks)
    return cfg


def _dp(a: np.ndarray):
    return a.ctypes.data_as(_D)


def _c(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float64)


class Solver:
    """One imex_ctx: the state of one 2D MHD run (periodic or transmissive per direction) on the
    current GPU."""

    def __init__(self, nx: int, ny: int, settings: dict | None = None, domain=None,
                 rks: int | None = None, config: Config | None = None):
        self.lib = load_library()
        self.cfg = config if config is not None else make_config(settings, domain, rks)
        self.nx, self.ny = nx, ny
        self.N = nx * ny
        h = C.c_void_p()
        rc = self.lib.imex_create(C.byref(self.cfg), nx, ny, C.byref(h))
        if rc != 0:
            raise ImexError(rc, "imex_create failed")
        self.ctx = h

    @classmethod
    def for_problem(cls, prob, rks: int, settings: dict | None = None, **kw) -> "Solver":
        s = dict(prob.settings)
        s.update(settings or {})
        sv = cls(prob.nx, prob.ny, s, (prob.x0, prob.x1, prob.y0, prob.y1), rks, **kw)
        sv.load(prob)
        return sv

    @classmethod
    def _view(cls, lib, ctx, nx: int, ny: int) -> "Solver":
        """A Solver on a context owned elsewhere (an ensemble member); close() leaves it alive."""
        sv = cls.__new__(cls)
        sv.lib, sv.ctx, sv.nx, sv.ny, sv.N, sv._owns = lib, ctx, nx, ny, nx * ny, False
        return sv

    def close(self) -> None:
        if getattr(self, "ctx", None):
            if getattr(self, "_owns", True):
                self.lib.imex_destroy(self.ctx)
            self.ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc: int) -> None:
        if rc != 0:
            msg = self.lib.imex_last_error(self.ctx)
            raise ImexError(rc, msg.decode() if msg else "")

    # ---- state
    def load(self, prob) -> None:
        prim, bx, by, A = _c(prob.prim), _c(prob.bx), _c(prob.by), _c(prob.A)
        self._check(self.lib.imex_upload_prim(self.ctx, _dp(prim), _dp(bx), _dp(by), _dp(A)))
        if getattr(prob, "bx_x0", None) is not None:
            self.set_boundary_faces(prob.bx_x0, prob.by_y0)

    def set_boundary_faces(self, bx_x0, by_y0) -> None:
        """Bx on x = x_0 (ny values) and By on y = y_0 (nx values) of the transmissive
        directions (imex_set_boundary_faces); a periodic direction ignores its line."""
        bx0, by0 = _c(bx_x0).reshape(self.ny), _c(by_y0).reshape(self.nx)
        self._check(self.lib.imex_set_boundary_faces(self.ctx, _dp(bx0), _dp(by0)))

    def boundary_faces(self) -> tuple[np.ndarray, np.ndarray]:
        """(Bx on x = x_0, By on y = y_0); a periodic direction gives the faces at x_1 / y_1."""
        bx0, by0 = np.empty(self.ny), np.empty(self.nx)
        self._check(self.lib.imex_get_boundary_faces(self.ctx, _dp(bx0), _dp(by0)))
        return bx0, by0

    def _planes(self, k):
        return np.empty((k, self.ny, self.nx)) if k > 1 else np.empty((self.ny, self.nx))

    def cons(self) -> np.ndarray:
        out = self._planes(8)
        self._check(self.lib.imex_download_state(self.ctx, _dp(out), None, None, None, None))
        return out

    def prim(self) -> np.ndarray:
        out = self._planes(8)
        self._check(self.lib.imex_download_state(self.ctx, None, _dp(out), None, None, None))
        return out

    def faces(self):
        bx, by = self._planes(1), self._planes(1)
        self._check(self.lib.imex_download_state(self.ctx, None, None, _dp(bx), _dp(by), None))
        return bx, by

    def vector_potential(self) -> np.ndarray:
        out = self._planes(3)
        self._check(self.lib.imex_download_state(self.ctx, None, None, None, None, _dp(out)))
        return out

    def upload_state(self, prim, bx, by, A) -> None:
        """Hand the solver a state mid-run (keeps t, the step counter and dt history)."""
        prim, bx, by, A = _c(prim), _c(bx), _c(by), _c(A)
        self._check(self.lib.imex_upload_state(self.ctx, _dp(prim), _dp(bx), _dp(by), _dp(A)))

    def upload_state_ptr(self, prim: int, bx: int, by: int, A: int) -> None:
        """Same with raw host or device addresses (e.g. pinned buffers)."""
        self._check(self.lib.imex_upload_state(self.ctx, C.cast(prim, _D), C.cast(bx, _D),
                                               C.cast(by, _D), C.cast(A, _D)))

    def download_state_ptr(self, prim: int, bx: int, by: int, A: int) -> None:
        self._check(self.lib.imex_download_state(self.ctx, None, C.cast(prim, _D), C.cast(bx, _D),
                                                 C.cast(by, _D), C.cast(A, _D)))

    def set_stream(self, stream_ptr: int | None) -> None:
        self._check(self.lib.imex_set_stream(self.ctx, C.c_void_p(stream_ptr or 0)))

    def profile_enable(self, on: bool = True) -> None:
        self._check(self.lib.imex_profile_enable(self.ctx, 1 if on else 0))

    def profile(self) -> list[dict]:
        buf = (KernelProfile * 64)()
        n = C.c_int()
        self._check(self.lib.imex_profile_read(self.ctx, buf, 64, C.byref(n)))
        return [dict(name=buf[k].name.decode(), launches=buf[k].launches,
                     total_ms=buf[k].total_ms, alg_bytes=buf[k].alg_bytes) for k in range(n.value)]

    def set_barrier_timeout(self, seconds: float) -> None:
        self._check(self.lib.imex_set_barrier_timeout(self.ctx, seconds))

    def selftest_fp64(self) -> dict:
        """Measured FP64 rates of this device: fused multiply-adds and divisions per second."""
        fma, div = C.c_double(), C.c_double()
        self._check(self.lib.imex_selftest_fp64(self.ctx, C.byref(fma), C.byref(div)))
        return {"dfma_per_s": fma.value, "dfma_tflops": 2e-12 * fma.value, "ddiv_per_s": div.value}

    def selftest_barrier(self, iterations: int, phantom_blocks: int = 0, timeout_s: float = 1.0) -> float:
        """Mean microseconds per device-wide barrier (raises ImexError on a timeout)."""
        us = C.c_double()
        self._check(self.lib.imex_selftest_barrier(self.ctx, iterations, phantom_blocks, timeout_s,
                                                   C.byref(us)))
        return us.value

    def kernel_launches(self) -> int:
        n = C.c_longlong()
        self._check(self.lib.imex_kernel_launch_count(self.ctx, C.byref(n)))
        return n.value

    # ---- stepping
    def step(self) -> float:
        dt = C.c_double()
        self._check(self.lib.imex_step(self.ctx, C.byref(dt)))
        return dt.value

    def begin_step(self) -> None:
        self._check(self.lib.imex_begin_step(self.ctx))

    def stage(self, rks: int) -> None:
        self._check(self.lib.imex_stage(self.ctx, rks))

    def end_step(self) -> None:
        self._check(self.lib.imex_end_step(self.ctx))

    def synchronize(self) -> None:
        self._check(self.lib.imex_synchronize(self.ctx))

    def scalars(self) -> dict:
        s = StepScalars()
        self._check(self.lib.imex_get_step_scalars(self.ctx, C.byref(s)))
        return {n: getattr(s, n) for n, _ in StepScalars._fields_}

    def set_scalars(self, **kw) -> None:
        s = StepScalars()
        self._check(self.lib.imex_get_step_scalars(self.ctx, C.byref(s)))
        for k, v in kw.items():
            setattr(s, k, v)
        self._check(self.lib.imex_set_step_scalars(self.ctx, C.byref(s)))

    def stats(self) -> dict:
        s = SolveStats()
        self._check(self.lib.imex_get_stats(self.ctx, C.byref(s)))
        return s.as_dict()

    def reset_stats(self) -> None:
        self._check(self.lib.imex_reset_stats(self.ctx))

    # ---- buffers
    def _line(self, name: str) -> int | None:
        """Length of a boundary-face line buffer (ny for an x_0 line, nx for a y_0 line)."""
        return {"bx_x0": self.ny, "bxQs_x0": self.ny, "by_y0": self.nx, "byQs_y0": self.nx}.get(name)

    def get_buffer(self, name: str, index: int = 0) -> np.ndarray:
        n = self._line(name)
        out = np.empty(n) if n else self._planes(BUF_PLANES[name])
        self._check(self.lib.imex_get_buffer(self.ctx, BUF[name], index, _dp(out)))
        return out

    def set_buffer(self, name: str, data, index: int = 0) -> None:
        a = _c(data)
        want = self._line(name) or BUF_PLANES[name] * self.N
        if a.size != want:
            raise ValueError(f"{name}: expected {want} values, got {a.size}")
        self._check(self.lib.imex_set_buffer(self.ctx, BUF[name], index, _dp(a)))

    # ---- sub-steps (reference function names)
    def stage_combine(self, rks: int) -> None:
        self._check(self.lib.imex_stage_combine(self.ctx, rks))

    def TVDReconstruction(self) -> None:
        self._check(self.lib.imex_TVDReconstruction(self.ctx))

    def RusanovC_Update(self, h: float, rks: int = 0) -> None:
        self._check(self.lib.imex_RusanovC_Update(self.ctx, h, rks))

    def MagSubsystem_UpdateB(self, h: float, rks: int = 0) -> None:
        self._check(self.lib.imex_MagSubsystem_UpdateB(self.ctx, h, rks))

    def MagSubsystem_UpdateA(self, h: float, rks: int = 0) -> None:
        self._check(self.lib.imex_MagSubsystem_UpdateA(self.ctx, h, rks))

    def Pressure_flux_Update(self, h: float, rks: int = 0) -> None:
        self._check(self.lib.imex_Pressure_flux_Update(self.ctx, h, rks))

    def PreSubsystem_Pressure(self, h: float, rks: int = 0) -> None:
        self._check(self.lib.imex_PreSubsystem_Pressure(self.ctx, h, rks))

    def Energy_flux_Update(self, h: float, rks: int = 0) -> None:
        self._check(self.lib.imex_Energy_flux_Update(self.ctx, h, rks))

    def PreSubsystem_Energy(self, h: float, rks: int = 0) -> None:
        self._check(self.lib.imex_PreSubsystem_Energy(self.ctx, h, rks))

    def Staggered_CT_Consistent(self, h: float, rks: int = 0) -> None:
        self._check(self.lib.imex_Staggered_CT_Consistent(self.ctx, h, rks))

    def Unstaggered_CT_Consistent(self, h: float, rks: int = 0) -> None:
        self._check(self.lib.imex_Unstaggered_CT_Consistent(self.ctx, h, rks))

    def Staggered_CT(self, h: float, rks: int = 0) -> None:
        self._check(self.lib.imex_Staggered_CT(self.ctx, h, rks))

    def Unstaggered_CT(self, h: float, rks: int = 0) -> None:
        self._check(self.lib.imex_Unstaggered_CT(self.ctx, h, rks))

    def stage_derivative(self, rks: int) -> None:
        self._check(self.lib.imex_stage_derivative(self.ctx, rks))

    # ---- operators and solves
    def prepare_operator(self, op: str, h: float) -> None:
        self._check(self.lib.imex_prepare_operator(self.ctx, OP[op], h))

    def set_newton_state(self, p_freeze, mbig: float) -> None:
        pf = _c(p_freeze)
        self._check(self.lib.imex_set_newton_state(self.ctx, _dp(pf), mbig))

    def apply_operator(self, op: str, x) -> np.ndarray:
        x = _c(x)
        out = np.empty_like(x)
        self._check(self.lib.imex_apply_operator(self.ctx, OP[op], _dp(x), _dp(out)))
        return out

    def gmres(self, op: str, x0, b) -> tuple[np.ndarray, dict]:
        x = np.array(x0, dtype=np.float64, copy=True)
        b = _c(b)
        st = SolveStats()
        self._check(self.lib.imex_gmres(self.ctx, OP[op], _dp(x), _dp(b), C.byref(st)))
        return x, st.as_dict()

    def gmres_noalloc(self, op: str, x0, b) -> tuple[np.ndarray, dict]:
        """imex_gmres on the library's fixed device scratch: no device allocation."""
        x = np.array(x0, dtype=np.float64, copy=True)
        b = _c(b)
        st = SolveStats()
        self._check(self.lib.imex_gmres_noalloc(self.ctx, OP[op], _dp(x), _dp(b), C.byref(st)))
        return x, st.as_dict()

    # ---- output formats and diagnostics
    def diagnostics(self) -> dict:
        """The per-step quantities of the reference's console and history files."""
        d = Diagnostics()
        self._check(self.lib.imex_diagnostics(self.ctx, C.byref(d)))
        return d.as_dict()

    CT_DIAG_PARTS = ("central", "rusanov", "tilde", "TOTAL")

    def ct_emf_diagnostics(self) -> dict:
        """The reference's per-step [CT-DIAG] figures (Diagnose_CT_EMF): for each part of the
        corner EMF, (L2 of Ez, max |Ez|, L2 of |dB/dt|, max |dB/dt|)."""
        out = np.zeros(16)
        self._check(self.lib.imex_ct_emf_diagnostics(self.ctx, _dp(out)))
        return {name: tuple(out[4 * c:4 * c + 4].tolist()) for c, name in enumerate(self.CT_DIAG_PARTS)}

    def write_vtk(self, path: str, cycle: int = 0) -> None:
        self._check(self.lib.imex_write_vtk(self.ctx, str(path).encode(), cycle))

    def write_fields_dat(self, directory: str) -> None:
        self._check(self.lib.imex_write_fields_dat(self.ctx, str(directory).encode()))

    def save_state_file(self, path: str) -> None:
        self._check(self.lib.imex_save_state_file(self.ctx, str(path).encode()))

    def load_state_file(self, path: str) -> None:
        self._check(self.lib.imex_load_state_file(self.ctx, str(path).encode()))

    # ---- discrete adjoint
    def adjoint_run(self, nsteps: int, rho_target, B_target, checkpoint_every: int = 10,
                    gmres_tol: float = 0.0) -> tuple[float, np.ndarray, np.ndarray, np.ndarray]:
        """Run nsteps from the current state and return J = 1/2|rho - rho_t|^2 + 1/2|B - B_t|^2
        at the end with its gradient w.r.t. the initial primitive planes and face fields."""
        o = AdjointOpts(nsteps, checkpoint_every, gmres_tol)
        rt, Bt = _c(rho_target), _c(B_target)
        J = C.c_double()
        gp, gx, gy = self._planes(8), self._planes(1), self._planes(1)
        self._check(self.lib.imex_adjoint_run(self.ctx, C.byref(o), _dp(rt), _dp(Bt), C.byref(J), _dp(gp),
                                              _dp(gx), _dp(gy)))
        return J.value, gp, gx, gy

    def adjoint_vjp(self, nsteps: int, lam_cons, lam_bx=None, lam_by=None, checkpoint_every: int = 10,
                    gmres_tol: float = 0.0) -> tuple[np.ndarray, np.ndarray, np.ndarray]:
        """Run nsteps and pull the cotangent (lam_cons, lam_bx, lam_by) of the final state back
        to the initial primitive planes and face fields."""
        o = AdjointOpts(nsteps, checkpoint_every, gmres_tol)
        lc = _c(lam_cons)
        lx = _c(lam_bx) if lam_bx is not None else None
        ly = _c(lam_by) if lam_by is not None else None
        gp, gx, gy = self._planes(8), self._planes(1), self._planes(1)
        self._check(self.lib.imex_adjoint_vjp(self.ctx, C.byref(o), _dp(lc), _dp(lx) if lx is not None else None,
                                              _dp(ly) if ly is not None else None, _dp(gp), _dp(gx), _dp(gy)))
        return gp, gx, gy

    def nested_newton(self, p0, b) -> tuple[np.ndarray, dict]:
        p = np.array(p0, dtype=np.float64, copy=True)
        b = _c(b)
        st = SolveStats()
        self._check(self.lib.imex_pressure_nested_newton(self.ctx, _dp(p), _dp(b), C.byref(st)))
        return p, st.as_dict()

    def shock_detector(self, Q) -> np.ndarray:
        Q = _c(Q)
        out = self._planes(1)
        self._check(self.lib.imex_shock_detector(self.ctx, _dp(Q), _dp(out)))
        return out

    def divergence(self) -> dict:
        v = [C.c_double() for _ in range(4)]
        self._check(self.lib.imex_divergence(self.ctx, *[C.byref(x) for x in v]))
        return dict(face_l2=v[0].value, cell_wrapped_l2=v[1].value, cell_ref_l2=v[2].value,
                    cell_inf=v[3].value)

    def min_pressure(self) -> float:
        v = C.c_double()
        self._check(self.lib.imex_min_pressure(self.ctx, C.byref(v)))
        return v.value


class Batch:
    """An ensemble (imex_batch): independent runs of one configuration on uneven grids,
    advanced together.  ``members[m]`` is a Solver view on member m's context (state I/O
    and diagnostics); the batch owns the members."""

    def __init__(self, problems, rks: int, settings: dict | None = None, streams: int = 0, graph: bool = True):
        """streams = 0: each explicit sub-step is one launch for all members; streams > 0:
        each member launches its own kernels, the members spread over that many streams."""
        self.lib = load_library()
        p0 = problems[0]
        s = dict(p0.settings)
        s.update(settings or {})
        self.cfg = make_config(s, (p0.x0, p0.x1, p0.y0, p0.y1), rks)
        n = len(problems)
        nx = (C.c_int * n)(*[p.nx for p in problems])
        ny = (C.c_int * n)(*[p.ny for p in problems])
        h = C.c_void_p()
        rc = self.lib.imex_batch_create(C.byref(self.cfg), n, nx, ny, C.byref(h))
        if rc != 0:
            raise ImexError(rc, "imex_batch_create failed")
        self.b = h
        self.members = []
        for m, p in enumerate(problems):
            c = C.c_void_p()
            self._check(self.lib.imex_batch_member(self.b, m, C.byref(c)))
            sv = Solver._view(self.lib, c, p.nx, p.ny)
            sv.load(p)
            self.members.append(sv)
        if streams != 0 or not graph:
            self._check(self.lib.imex_batch_configure(self.b, streams, 1 if graph else 0))

    def _check(self, rc: int) -> None:
        if rc != 0:
            msg = self.lib.imex_batch_last_error(self.b)
            raise ImexError(rc, msg.decode() if msg else "")

    def step(self, steps: int = 1) -> float:
        """Advance every member `steps` steps; returns the device time in ms."""
        ms = C.c_double()
        self._check(self.lib.imex_batch_step(self.b, steps, C.byref(ms)))
        return ms.value

    def autotune(self, trial_steps: int = 2) -> dict:
        t = BatchTuning()
        self._check(self.lib.imex_batch_autotune(self.b, trial_steps, C.byref(t)))
        return dict(streams=t.streams, gmres_restart=t.gmres_restart, ms_per_step=t.ms_per_step,
                    mixed_solves=t.mixed_solves, solve_tile=(t.solve_tile_x, t.solve_tile_y))

    def set_solve_tile(self, tile: int) -> None:
        """Tile shape of the batched B-form solve (fast arithmetic): 0 = 32x16, 1 = 64x8,
        2 = 32x8 cells."""
        self._check(self.lib.imex_batch_set_solve_tile(self.b, tile))

    def info(self) -> dict:
        a, g, n = C.c_int(), C.c_int(), C.c_int()
        self._check(self.lib.imex_batch_info(self.b, C.byref(a), C.byref(g), C.byref(n)))
        msg = self.lib.imex_batch_last_error(self.b)
        e, sl = C.c_int(), C.c_int()
        self._check(self.lib.imex_batch_explicit_launches(self.b, C.byref(e), C.byref(sl)))
        return dict(streams=a.value, graph=bool(g.value), solve_launches_per_step=n.value,
                    explicit_launches_per_step=e.value, planned_solve_launches_per_step=sl.value,
                    note=msg.decode() if msg else "")

    def close(self) -> None:
        if getattr(self, "b", None):
            for sv in self.members:
                sv.ctx = None
            self.lib.imex_batch_destroy(self.b)
            self.b = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
