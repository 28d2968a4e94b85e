"""Host-side mirror of CRUNA's module interfaces over the C ABI of libcruna_b200.so.

``Cruna`` exposes the reference's procedure names with their argument meaning:

================================  =========================================================
reference procedure               here
================================  =========================================================
rhs_direct(rhs, q, t)             ``Cruna.rhs_direct(q, t) -> rhs``
rhs_adjoint(rhs, qs, q, g, t)     ``Cruna.rhs_adjoint(qs, q, g, t) -> rhs``
Dx1/Dx2/Dx3(q_x, q, h)            ``Cruna.Dx1(q, h=None) -> q_x`` (h absent -> dx = 1)
filter_i1/2/3(q)                  ``Cruna.filter_i1(q) -> q`` (new array)
time_stepper_direct(q1, q0, t)    ``Cruna.time_stepper_direct(q0, t) -> q1``
time_stepper_adjoint(...)         ``Cruna.time_stepper_adjoint(qs0, q0, g, t) -> qs1``
set_boundary_condition_q/qs/...   ``Cruna.set_boundary_condition_q(q, outside_rhs)`` etc.
calc_direct(Q, q0)                ``Cruna.calc_direct(q0, steps, store) -> q or (q, Q)``
calc_adjoint(Qs, qs0, Q)          ``Cruna.calc_adjoint(qs0, Q, g=None) -> qs``
================================  =========================================================

Arrays are numpy float64 in Fortran order: fields (n1, n2, n3), states (n1, n2, n3, 5).  A failing
call raises ``CrunaError`` carrying the library's status and message, where the reference prints
and calls ``stop_cruna``.  The library must be built (``public_b200.build``); there is no CPU
fallback.
"""
from __future__ import annotations

import ctypes as C
import dataclasses
import math
from pathlib import Path
from typing import Optional, Sequence, Tuple

import numpy as np

LIB_PATH = Path(__file__).resolve().parent / "libcruna_b200.so"

DIFF = {"empty": 0, "o2_e_c_o": 1, "o4_e_c_p": 2, "o4_e_c_o": 3, "o4_i_c_p_pade": 4, "o4_i_c_o_pade": 5,
        "o6_i_c_p": 6, "o6_i_c_o": 7, "o8_e_c_p": 8}
FILTER = {"empty": 0, "o2_i_c_p": 1, "o6_i_c_p": 2, "o2_i_c_o": 3, "o4_i_c_o": 4, "o6_i_c_o": 5,
          "o8_i_c_o": 6, "o10_i_c_o": 7, "o10_e_c_p": 8}
PRECISION = {"fp64": 0, "fp32": 1}
ABI_VERSION = 2

CRUNA_STOPPED = 1
ERRORS = {-1: "CRUNA_ERR_ARG", -2: "CRUNA_ERR_CUDA", -3: "CRUNA_ERR_NOMEM", -4: "CRUNA_ERR_STATE",
          -5: "CRUNA_ERR_UNSUPPORTED", -6: "CRUNA_ERR_NODEVICE", -7: "CRUNA_ERR_IO"}


class CrunaError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{ERRORS.get(code, code)}: {msg}")
        self.code = code


class _Config(C.Structure):
    _fields_ = [
        ("abi_version", C.c_int32), ("n", C.c_int32 * 3), ("x0", C.c_double * 3), ("x1", C.c_double * 3),
        ("diff", C.c_int32 * 3), ("filter", C.c_int32 * 3), ("filter_alpha", C.c_double),
        ("filter_strength", C.c_double), ("di_freq", C.c_int32 * 3), ("ai_freq", C.c_int32 * 3),
        ("gamma", C.c_double), ("R", C.c_double), ("W", C.c_double), ("mu0", C.c_double),
        ("T0", C.c_double), ("Pr", C.c_double), ("dt", C.c_double), ("heat_flux_dx", C.c_int32),
        ("precision", C.c_int32), ("sponge_length", C.c_double * 3), ("sponge_amplitude", C.c_double),
        ("sponge_shape", C.c_int32), ("device", C.c_int32), ("check_every", C.c_int32), ("kvector", C.c_int32),
    ]


class Objective(C.Structure):
    """struct cruna_objective: kind 1 = plane (p - p_inf)^2 integral, kind 2 = final kinetic energy."""
    _fields_ = [("kind", C.c_int32), ("normal", C.c_int32), ("index", C.c_int32), ("reserved", C.c_int32),
                ("p_inf", C.c_double)]


_P = C.c_void_p
_D = C.c_double
_I = C.c_int

class HpcOpts(C.Structure):
    """cruna_hpc_opts: the keys of cruna_hpc's main loop (src/main/cruna_hpc.f90:99-299)."""
    _fields_ = [("workdir", C.c_char_p), ("steps", C.c_int32), ("subsets", C.c_int32), ("dsfreq", C.c_int32),
                ("restart", C.c_int32), ("walltime", C.c_double), ("max_steps", C.c_int32),
                ("reserved", C.c_int32)]


_SIGNATURES = {
    "cruna_config_defaults": (None, [C.POINTER(_Config)]),
    "cruna_init": (_I, [C.POINTER(_Config), _P, _I, C.POINTER(_P)]),
    "cruna_free": (None, [_P]),
    "cruna_last_error": (C.c_char_p, [_P]),
    "cruna_sync": (_I, [_P]),
    "cruna_get_dx": (_I, [_P, _P]),
    "cruna_stream": (_P, [_P]),
    "cruna_set_reference": (_I, [_P, _P]),
    "cruna_set_reference_dev": (_I, [_P, _P]),
    "cruna_set_forcing": (_I, [_P, _P]),
    "cruna_set_forcing_dev": (_I, [_P, _P]),
    "cruna_diff": (_I, [_P, _I, _P, _P, _I, _D]),
    "cruna_diff_dev": (_I, [_P, _I, _P, _P, _I, _D]),
    "cruna_filter": (_I, [_P, _I, _P, _I]),
    "cruna_filter_dev": (_I, [_P, _I, _P, _I]),
    "cruna_rhs_direct": (_I, [_P, _P, _P, _D]),
    "cruna_rhs_direct_dev": (_I, [_P, _P, _P, _D]),
    "cruna_rhs_adjoint": (_I, [_P, _P, _P, _P, _P, _D]),
    "cruna_rhs_adjoint_dev": (_I, [_P, _P, _P, _P, _P, _D]),
    "cruna_step_direct": (_I, [_P, _P, _P, _D]),
    "cruna_step_direct_dev": (_I, [_P, _P, _P, _D]),
    "cruna_step_adjoint": (_I, [_P, _P, _P, _P, _P, _D]),
    "cruna_step_adjoint_dev": (_I, [_P, _P, _P, _P, _P, _D]),
    "cruna_bc_q": (_I, [_P, _P, _I]),
    "cruna_bc_qs": (_I, [_P, _P, _P, _I]),
    "cruna_bc_rhs": (_I, [_P, _P, _P]),
    "cruna_bc_rhss": (_I, [_P, _P, _P, _P]),
    "cruna_bc_q_dev": (_I, [_P, _P, _I]),
    "cruna_bc_qs_dev": (_I, [_P, _P, _P, _I]),
    "cruna_bc_rhs_dev": (_I, [_P, _P, _P]),
    "cruna_bc_rhss_dev": (_I, [_P, _P, _P, _P]),
    "cruna_run_direct": (_I, [_P, _P, _I, _I, _P]),
    "cruna_run_direct_dev": (_I, [_P, _P, _I, _I, _P]),
    "cruna_run_adjoint": (_I, [_P, _P, _P, _P, _I, _I]),
    "cruna_run_adjoint_dev": (_I, [_P, _P, _P, _P, _I, _I]),
    "cruna_check_state_dev": (_I, [_P, _P]),
    "cruna_rhs_path": (_I, [_P]),
    "cruna_set_force_generic": (_I, [_P, _I]),
    "cruna_set_tma_passes": (_I, [_P, _I]),
    "cruna_kernel_launches": (C.c_int64, [_P]),
    "cruna_profile_enable": (_I, [_P, _I]),
    "cruna_profile_report": (_I, [_P, C.c_char_p, _I]),
    "cruna_set_graphs": (_I, [_P, _I]),
    "cruna_set_snapshot_memory": (_I, [_P, _I]),
    "cruna_set_closure_normalisation": (_I, [_P, _I]),
    "cruna_diagnostics": (_I, [_P, _P, C.POINTER(C.c_double), C.POINTER(C.c_double)]),
    "cruna_diagnostics_dev": (_I, [_P, _P, C.POINTER(C.c_double), C.POINTER(C.c_double)]),
    "cruna_graph_stats": (_I, [_P, C.POINTER(C.c_int64), C.POINTER(C.c_int64)]),
    "cruna_rhs_direct_noalloc": (_I, [C.POINTER(_Config), _P, _P, _P, C.c_char_p, _I]),
    "cruna_mlp_create": (_I, [_I, C.c_uint64, C.POINTER(_P)]),
    "cruna_mlp_free": (None, [_P]),
    "cruna_mlp_last_error": (C.c_char_p, [_P]),
    "cruna_mlp_set_params": (_I, [_P, _P]),
    "cruna_mlp_get_params": (_I, [_P, _P]),
    "cruna_mlp_set_scaling": (_I, [_P, _P, _P, _P]),
    "cruna_mlp_forward_dev": (_I, [_P, _P, _P, C.c_longlong]),
    "cruna_mlp_grad_dev": (_I, [_P, _P, _P, _I, _P, C.POINTER(C.c_float)]),
    "cruna_mlp_train_dev": (_I, [_P, _P, _P, C.c_longlong, _I, _I, C.c_float, C.c_uint64, _P]),
    "cruna_box_filter_dev": (_I, [_P, _I, _P, _P, _P]),
    "cruna_closure_features_dev": (_I, [_P, _P, C.c_double, _P]),
    "cruna_set_closure": (_I, [_P, _P, C.c_double]),
    "cruna_set_closure_fused": (_I, [_P, _I]),
    "cruna_set_halo_exchange": (_I, [_P, _P, _P]),
    "cruna_objective_value": (_I, [_P, _P, _I, C.POINTER(Objective), C.POINTER(C.c_double)]),
    "cruna_objective_value_dev": (_I, [_P, _P, _I, C.POINTER(Objective), C.POINTER(C.c_double)]),
    "cruna_optimize": (_I, [_P, _P, C.POINTER(Objective), _I, _I, _I, _I, C.c_double, _P, _P, _P]),
    "cruna_optimize_dev": (_I, [_P, _P, C.POINTER(Objective), _I, _I, _I, _I, C.c_double, _P, _P, _P]),
    "cruna_set_adjoint_mode": (_I, [_P, _I]),
    "cruna_rhs_direct_vjp": (_I, [_P, _P, _P, _P, _P]),
    "cruna_rhs_direct_vjp_dev": (_I, [_P, _P, _P, _P, _P]),
    "cruna_step_direct_vjp": (_I, [_P, _P, _P, _P, _P, _I]),
    "cruna_step_direct_vjp_dev": (_I, [_P, _P, _P, _P, _P, _I]),
    "cruna_gradient": (_I, [_P, _P, _I, _I, C.POINTER(Objective), C.POINTER(C.c_double), _P, _P,
                            C.POINTER(C.c_int64)]),
    "cruna_gradient_dev": (_I, [_P, _P, _I, _I, C.POINTER(Objective), C.POINTER(C.c_double), _P, _P,
                                C.POINTER(C.c_int64)]),
    "cruna_lapack_dgttrf": (_I, [_I, _P, _P, _P, _P, _P]),
    "cruna_lapack_dgttrs": (None, [_I, _P, _P, _P, _P, _P, _P]),
    "cruna_io_fname": (_I, [C.c_char_p, _I, C.c_char_p, C.c_char_p, _I, _I, _I, _I]),
    "cruna_write_snapshot": (_I, [C.c_char_p, C.POINTER(C.c_int64), _P, C.c_char_p]),
    "cruna_read_snapshot": (_I, [C.c_char_p, C.POINTER(C.c_int64), _P, C.c_char_p, _I]),
    "cruna_write_restart": (_I, [C.c_char_p, _I, _I]),
    "cruna_read_restart": (_I, [C.c_char_p, C.POINTER(C.c_int), C.POINTER(C.c_int)]),
    "cruna_restart_start": (_I, [_I, _I, _I, C.POINTER(C.c_int), C.POINTER(C.c_int)]),
    "cruna_store_snapshot": (_I, [_P, C.c_char_p, C.c_char_p, _P, _I, _I]),
    "cruna_load_snapshot": (_I, [_P, C.c_char_p, C.c_char_p, _P, _I, _I]),
    "cruna_run_hpc": (_I, [_P, _P, C.POINTER(HpcOpts), C.POINTER(C.c_int), C.POINTER(C.c_int)]),
}

_lib = None


def load_library(path: Optional[Path] = None) -> C.CDLL:
    """Load libcruna_b200.so (raises if it is missing: there is no CPU fallback)."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = Path(path) if path else LIB_PATH
    if not p.exists():
        raise FileNotFoundError(f"{p} is not built; run `python -m public_b200.build`")
    lib = C.CDLL(str(p))
    for name, (res, args) in _SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if path is None:
        _lib = lib
    return lib


@dataclasses.dataclass
class Settings:
    """Solver settings; the keys mirror parameter.dat (geom.*, filter.*, material.*, time.dt, sponge.*)."""
    n: Tuple[int, int, int]
    x0: Tuple[float, float, float] = (0.0, 0.0, 0.0)
    x1: Tuple[float, float, float] = (1.0, 1.0, 1.0)
    diff: Tuple[str, str, str] = ("o4_e_c_p", "o4_e_c_p", "o4_e_c_p")
    filt: Tuple[str, str, str] = ("empty", "empty", "empty")
    alpha: float = 0.35
    strength: float = 0.2
    di_freq: Tuple[int, int, int] = (0, 0, 0)
    ai_freq: Tuple[int, int, int] = (0, 0, 0)
    gamma: float = 1.4
    R: float = 8.3144598
    W: float = 0.0289647
    mu0: float = 0.0
    T0: float = 273.0
    Pr: float = 0.71
    dt: float = 1e-3
    heat_flux_dx: bool = False
    precision: str = "fp64"
    sponge_length: Tuple[float, float, float] = (0.3, 0.3, 0.3)
    sponge_amplitude: float = 1.0
    sponge_shape: str = "quadratic"
    bc: Optional[np.ndarray] = None
    device: int = 0
    check_every: int = 0
    kvector: str = "diagonal"

    @classmethod
    def from_dict(cls, d: dict) -> "Settings":
        names = {f.name for f in dataclasses.fields(cls)}
        kw = {k: v for k, v in d.items() if k in names}
        for key in ("di_freq", "ai_freq"):
            if key in kw:
                kw[key] = tuple(0 if v >= 2**31 - 1 else int(v) for v in kw[key])
        return cls(**kw)

    def to_struct(self, lib: C.CDLL) -> _Config:
        c = _Config()
        lib.cruna_config_defaults(C.byref(c))
        c.abi_version = ABI_VERSION
        for d in range(3):
            c.n[d] = int(self.n[d])
            c.x0[d] = float(self.x0[d])
            c.x1[d] = float(self.x1[d])
            c.diff[d] = DIFF[self.diff[d]]
            c.filter[d] = FILTER[self.filt[d]]
            c.di_freq[d] = int(self.di_freq[d])
            c.ai_freq[d] = int(self.ai_freq[d])
            c.sponge_length[d] = float(self.sponge_length[d])
        c.filter_alpha = float(self.alpha)
        c.filter_strength = float(self.strength)
        c.gamma, c.R, c.W = float(self.gamma), float(self.R), float(self.W)
        c.mu0, c.T0, c.Pr = float(self.mu0), float(self.T0), float(self.Pr)
        c.dt = float(self.dt)
        c.heat_flux_dx = 1 if self.heat_flux_dx else 0
        c.precision = PRECISION[self.precision]
        c.sponge_amplitude = float(self.sponge_amplitude)
        c.sponge_shape = 0 if self.sponge_shape == "quadratic" else 1
        c.device = int(self.device)
        c.check_every = int(self.check_every)
        c.kvector = {"diagonal": 0, "orthogonal": 1, "hedgehog": 2}[self.kvector]
        return c


def _ptr(a: Optional[np.ndarray]):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


class Cruna:
    """One solver context on one GPU (the reference's per-rank module state)."""

    def __init__(self, settings: Settings, qref: Optional[np.ndarray] = None,
                 force: Optional[np.ndarray] = None, lib_path: Optional[Path] = None):
        self.lib = load_library(lib_path)
        self.s = settings
        self.n = tuple(int(v) for v in settings.n)
        cfg = settings.to_struct(self.lib)
        self._bc = None
        nbc = 0
        if settings.bc is not None and len(settings.bc):
            self._bc = np.ascontiguousarray(np.asarray(settings.bc, dtype=np.float64).reshape(-1, 10))
            nbc = self._bc.shape[0]
        h = C.c_void_p()
        rc = self.lib.cruna_init(C.byref(cfg), _ptr(self._bc), nbc, C.byref(h))
        if rc != 0:
            raise CrunaError(rc, self.lib.cruna_last_error(None).decode())
        self.h = h
        if qref is not None:
            self.set_reference(qref)
        if force is not None:
            self.set_forcing(force)

    # --------------------------------------------------------------------------------------------
    def close(self):
        if getattr(self, "h", None):
            self.lib.cruna_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def _check(self, rc: int):
        if rc != 0:
            raise CrunaError(rc, self.lib.cruna_last_error(self.h).decode())

    def _state(self, a: np.ndarray, nf: int = 5) -> np.ndarray:
        a = np.asarray(a, dtype=np.float64)
        shape = self.n + (nf,) if nf > 1 or a.ndim == 4 else self.n
        if a.size != int(np.prod(self.n)) * nf:
            raise CrunaError(-1, f"array of shape {a.shape} does not match grid {self.n} x {nf}")
        return np.asfortranarray(a.reshape(shape, order="F"))

    @property
    def dx(self) -> Tuple[float, float, float]:
        out = (C.c_double * 3)()
        self._check(self.lib.cruna_get_dx(self.h, out))
        return tuple(out)

    @property
    def rhs_path(self) -> str:
        return "fused" if self.lib.cruna_rhs_path(self.h) == 1 else "generic"

    def force_generic(self, on: bool = True):
        self._check(self.lib.cruna_set_force_generic(self.h, 1 if on else 0))

    def tma_passes(self, on: bool = True):
        """FP64 fused adjoint pass fed by TMA, or by per-thread loads (the default, faster on B200)."""
        self._check(self.lib.cruna_set_tma_passes(self.h, 1 if on else 0))

    @property
    def launches(self) -> int:
        return int(self.lib.cruna_kernel_launches(self.h))

    # --------------------------------------------------------------------------------------------
    def set_reference(self, qref: np.ndarray):
        q = self._state(qref)
        self._check(self.lib.cruna_set_reference(self.h, _ptr(q)))

    def set_forcing(self, f: Optional[np.ndarray]):
        if f is None:
            self._check(self.lib.cruna_set_forcing(self.h, None))
        else:
            ff = self._state(f)
            self._check(self.lib.cruna_set_forcing(self.h, _ptr(ff)))

    def _dx(self, d: int, q: np.ndarray, h: Optional[float]) -> np.ndarray:
        q = np.asarray(q, dtype=np.float64)
        nf = q.size // int(np.prod(self.n))
        a = self._state(q, nf)
        out = np.empty_like(a, order="F")
        self._check(self.lib.cruna_diff(self.h, d, _ptr(a), _ptr(out), nf, math.nan if h is None else float(h)))
        return out

    def Dx1(self, q, h=None):
        return self._dx(1, q, h)

    def Dx2(self, q, h=None):
        return self._dx(2, q, h)

    def Dx3(self, q, h=None):
        return self._dx(3, q, h)

    def _filter(self, d: int, q: np.ndarray) -> np.ndarray:
        q = np.asarray(q, dtype=np.float64)
        nf = q.size // int(np.prod(self.n))
        a = np.array(self._state(q, nf), order="F", copy=True)
        self._check(self.lib.cruna_filter(self.h, d, _ptr(a), nf))
        return a

    def filter_i1(self, q):
        return self._filter(1, q)

    def filter_i2(self, q):
        return self._filter(2, q)

    def filter_i3(self, q):
        return self._filter(3, q)

    def rhs_direct(self, q: np.ndarray, t: float = 0.0) -> np.ndarray:
        a = self._state(q)
        out = np.empty_like(a, order="F")
        self._check(self.lib.cruna_rhs_direct(self.h, _ptr(a), _ptr(out), float(t)))
        return out

    def rhs_adjoint(self, qs, q, g=None, t: float = 0.0) -> np.ndarray:
        a, b = self._state(qs), self._state(q)
        gg = None if g is None else self._state(g)
        out = np.empty_like(a, order="F")
        self._check(self.lib.cruna_rhs_adjoint(self.h, _ptr(a), _ptr(b), _ptr(gg), _ptr(out), float(t)))
        return out

    def time_stepper_direct(self, q0, t: float = 0.0) -> np.ndarray:
        a = self._state(q0)
        out = np.empty_like(a, order="F")
        self._check(self.lib.cruna_step_direct(self.h, _ptr(a), _ptr(out), float(t)))
        return out

    def time_stepper_adjoint(self, qs0, q0, g=None, t: float = 0.0) -> np.ndarray:
        a, b = self._state(qs0), self._state(q0)
        gg = None if g is None else self._state(g)
        out = np.empty_like(a, order="F")
        self._check(self.lib.cruna_step_adjoint(self.h, _ptr(a), _ptr(b), _ptr(gg), _ptr(out), float(t)))
        return out

    def set_boundary_condition_q(self, q, outside_rhs: bool = False) -> np.ndarray:
        a = np.array(self._state(q), order="F", copy=True)
        self._check(self.lib.cruna_bc_q(self.h, _ptr(a), 1 if outside_rhs else 0))
        return a

    def set_boundary_condition_qs(self, qs, q, outside_rhs: bool = False) -> np.ndarray:
        a = np.array(self._state(qs), order="F", copy=True)
        b = self._state(q)
        self._check(self.lib.cruna_bc_qs(self.h, _ptr(a), _ptr(b), 1 if outside_rhs else 0))
        return a

    def set_boundary_condition_rhs(self, rhs, q) -> np.ndarray:
        a = np.array(self._state(rhs), order="F", copy=True)
        b = self._state(q)
        self._check(self.lib.cruna_bc_rhs(self.h, _ptr(a), _ptr(b)))
        return a

    def set_boundary_condition_rhss(self, rhss, qs, q=None) -> np.ndarray:
        a = np.array(self._state(rhss), order="F", copy=True)
        b = self._state(qs)
        cq = None if q is None else self._state(q)
        self._check(self.lib.cruna_bc_rhss(self.h, _ptr(a), _ptr(b), _ptr(cq)))
        return a

    def calc_direct(self, q0, steps: int, store: bool = False, nt0: int = 0):
        """Loop of calc_direct (computation_direct.f90:64-107); store=True also returns [q0, q1, ...]."""
        a = np.array(self._state(q0), order="F", copy=True)
        traj = None
        if store:
            traj = np.empty((steps,) + a.shape[::-1], dtype=np.float64)   # C-order slabs of one state
        self._check(self.lib.cruna_run_direct(self.h, _ptr(a), int(nt0), int(steps), _ptr(traj)))
        if not store:
            return a
        Q = [np.array(self._state(q0), copy=True)]
        for s in range(steps):
            Q.append(np.asfortranarray(traj[s].reshape(-1).reshape(a.shape, order="F")))
        return a, Q

    def calc_adjoint(self, qs0, Q: Sequence[np.ndarray], g: Optional[Sequence[np.ndarray]] = None):
        """Loop of calc_adjoint (computation_adjoint.f90:60-108) over nt = len(Q)-1 .. 1, using Q[nt]."""
        steps = len(Q) - 1
        a = np.array(self._state(qs0), order="F", copy=True)
        Qt = np.stack([np.asarray(self._state(Q[nt])).reshape(-1, order="F") for nt in range(1, steps + 1)])
        Gt = None
        if g is not None:
            Gt = np.stack([np.asarray(self._state(g[nt])).reshape(-1, order="F") for nt in range(1, steps + 1)])
        self._check(self.lib.cruna_run_adjoint(self.h, _ptr(a), _ptr(np.ascontiguousarray(Qt)),
                                               _ptr(None if Gt is None else np.ascontiguousarray(Gt)),
                                               steps, steps))
        return a

    @staticmethod
    def objective(kind: str, normal: int = 2, index: int = 1, p_inf: float = 0.0) -> Objective:
        """kind 'plane_p2' (normal, 1-based index, p_inf), 'kinetic_energy' or 'enstrophy' (final time)."""
        o = Objective()
        o.kind = {"plane_p2": 1, "kinetic_energy": 2, "enstrophy": 3}[kind]
        o.normal, o.index, o.p_inf = int(normal), int(index), float(p_inf)
        return o

    # ---- learned closure (device pointers) ----
    def box_filter_dev(self, factor: int, q_ptr: int, qc_ptr: int, tau_ptr: int):
        """Box filter of the device state q into the coarse state and the subgrid stresses (floats)."""
        self._check(self.lib.cruna_box_filter_dev(self.h, int(factor), C.c_void_p(q_ptr), C.c_void_p(qc_ptr),
                                                  C.c_void_p(tau_ptr)))

    def closure_features_dev(self, q_ptr: int, delta: float, x_ptr: int):
        self._check(self.lib.cruna_closure_features_dev(self.h, C.c_void_p(q_ptr), float(delta), C.c_void_p(x_ptr)))

    def set_closure_normalisation(self, on: bool = True):
        """Scale-free closure features and outputs (grad u / |grad u|, |grad u| delta; tau / (rho (|grad u| delta)^2))."""
        self._check(self.lib.cruna_set_closure_normalisation(self.h, 1 if on else 0))

    def set_closure_fused(self, on: bool = True):
        """Closure evaluated inside the flux pass (default) or by separate launches."""
        self._check(self.lib.cruna_set_closure_fused(self.h, 1 if on else 0))

    def set_closure(self, mlp, delta: float = 0.0):
        """Attach a public_b200.closure.ClosureMLP (None detaches)."""
        self._check(self.lib.cruna_set_closure(self.h, None if mlp is None else mlp.h, float(delta)))
        self._closure = mlp  # keep the MLP alive while attached

    def set_halo_exchange(self, fn):
        """Install a z-slab halo callback (a ctypes function of public_b200.slabs.HALO_FN; None detaches)."""
        self._check(self.lib.cruna_set_halo_exchange(self.h, None if fn is None else C.cast(fn, C.c_void_p), None))
        self._halo_fn = fn

    def objective_value(self, q0, nsteps: int, objective: Objective) -> float:
        J = C.c_double()
        self._check(self.lib.cruna_objective_value(self.h, _ptr(self._state(q0)), int(nsteps), C.byref(objective),
                                                   C.byref(J)))
        return J.value

    def objective_value_dev(self, q0_ptr: int, nsteps: int, objective: Objective) -> float:
        J = C.c_double()
        self._check(self.lib.cruna_objective_value_dev(self.h, C.c_void_p(q0_ptr), int(nsteps), C.byref(objective),
                                                       C.byref(J)))
        return J.value

    def optimize(self, q0, objective: Objective, nsteps: int, nsnap: int, maxloop: int, ls_start: int,
                 alpha0: float, f0):
        """Optimisation loop of cruna.f90 on the forcing: returns (J per loop, alpha per loop, final f)."""
        a = self._state(q0)
        f = np.array(self._state(f0), order="F", copy=True)
        Jh = np.zeros(maxloop)
        ah = np.zeros(max(maxloop - 1, 1))
        self._check(self.lib.cruna_optimize(self.h, _ptr(a), C.byref(objective), int(nsteps), int(nsnap),
                                            int(maxloop), int(ls_start), float(alpha0), _ptr(f), _ptr(Jh),
                                            _ptr(ah)))
        return Jh, ah[:maxloop - 1], f

    def set_adjoint_mode(self, mode: int):
        """0: the reference's continuous adjoint (default); 1: the exact discrete adjoint."""
        self._check(self.lib.cruna_set_adjoint_mode(self.h, int(mode)))

    def rhs_direct_vjp(self, q, lam, grad_f=None):
        """(d rhs_direct/d q)^T lam; grad_f (a state array, updated in place) accumulates (d rhs/d f)^T lam."""
        a, l = self._state(q), self._state(lam)
        mu = np.empty_like(a, order="F")
        gf = None if grad_f is None else self._state(grad_f)
        self._check(self.lib.cruna_rhs_direct_vjp(self.h, _ptr(a), _ptr(l), _ptr(mu), _ptr(gf)))
        if grad_f is not None and gf is not grad_f:
            grad_f[...] = gf
        return mu

    def step_direct_vjp(self, q0, lam1, nt: int, grad_f=None):
        """Transpose of direct loop step nt at q0 applied to lam1 (grad_f accumulated in place)."""
        a, l = self._state(q0), self._state(lam1)
        out = np.empty_like(a, order="F")
        gf = None if grad_f is None else self._state(grad_f)
        self._check(self.lib.cruna_step_direct_vjp(self.h, _ptr(a), _ptr(l), _ptr(out), _ptr(gf), int(nt)))
        if grad_f is not None and gf is not grad_f:
            grad_f[...] = gf
        return out

    def gradient(self, q0, nsteps: int, nsnap: int, objective: Objective):
        """J, dJ/df, dJ/dq0 and the number of direct steps executed (binomial checkpointing)."""
        a = self._state(q0)
        gf = np.empty_like(a, order="F")
        gq = np.empty_like(a, order="F")
        J = C.c_double()
        steps = C.c_int64()
        self._check(self.lib.cruna_gradient(self.h, _ptr(a), int(nsteps), int(nsnap), C.byref(objective),
                                            C.byref(J), _ptr(gf), _ptr(gq), C.byref(steps)))
        return J.value, gf, gq, steps.value

    def gradient_dev(self, q0_ptr: int, nsteps: int, nsnap: int, objective: Objective,
                     grad_f_ptr: Optional[int], grad_q0_ptr: Optional[int]):
        J = C.c_double()
        steps = C.c_int64()
        self._check(self.lib.cruna_gradient_dev(self.h, C.c_void_p(q0_ptr), int(nsteps), int(nsnap),
                                                C.byref(objective), C.byref(J),
                                                None if grad_f_ptr is None else C.c_void_p(grad_f_ptr),
                                                None if grad_q0_ptr is None else C.c_void_p(grad_q0_ptr),
                                                C.byref(steps)))
        return J.value, steps.value

    def set_forcing_dev(self, f_ptr: Optional[int]):
        self._check(self.lib.cruna_set_forcing_dev(self.h, None if f_ptr is None else C.c_void_p(f_ptr)))

    # device-pointer variants (pointers from torch tensors or any CUDA allocation on the context's device)
    def rhs_direct_dev(self, q_ptr: int, rhs_ptr: int, t: float = 0.0):
        self._check(self.lib.cruna_rhs_direct_dev(self.h, C.c_void_p(q_ptr), C.c_void_p(rhs_ptr), float(t)))

    def step_direct_dev(self, q0_ptr: int, q1_ptr: int, t: float = 0.0):
        self._check(self.lib.cruna_step_direct_dev(self.h, C.c_void_p(q0_ptr), C.c_void_p(q1_ptr), float(t)))

    def step_adjoint_dev(self, qs0_ptr: int, q0_ptr: int, g_ptr: Optional[int], qs1_ptr: int, t: float = 0.0):
        self._check(self.lib.cruna_step_adjoint_dev(self.h, C.c_void_p(qs0_ptr), C.c_void_p(q0_ptr),
                                                    None if g_ptr is None else C.c_void_p(g_ptr),
                                                    C.c_void_p(qs1_ptr), float(t)))

    def run_direct_dev(self, q_ptr: int, nt0: int, nsteps: int, traj_ptr: Optional[int] = None):
        self._check(self.lib.cruna_run_direct_dev(self.h, C.c_void_p(q_ptr), int(nt0), int(nsteps),
                                                  None if traj_ptr is None else C.c_void_p(traj_ptr)))

    def run_adjoint_dev(self, qs_ptr: int, Q_ptr: int, g_ptr: Optional[int], nt_end: int, nsteps: int):
        self._check(self.lib.cruna_run_adjoint_dev(self.h, C.c_void_p(qs_ptr), C.c_void_p(Q_ptr),
                                                   None if g_ptr is None else C.c_void_p(g_ptr),
                                                   int(nt_end), int(nsteps)))

    def diagnostics(self, q) -> Tuple[float, float]:
        """(kinetic energy, enstrophy) volume integrals of a host state."""
        a = self._state(q)
        ke, en = C.c_double(), C.c_double()
        self._check(self.lib.cruna_diagnostics(self.h, _ptr(a), C.byref(ke), C.byref(en)))
        return ke.value, en.value

    def diagnostics_dev(self, q_ptr: int) -> Tuple[float, float]:
        ke, en = C.c_double(), C.c_double()
        self._check(self.lib.cruna_diagnostics_dev(self.h, C.c_void_p(q_ptr), C.byref(ke), C.byref(en)))
        return ke.value, en.value

    def set_snapshot_memory(self, host: bool):
        """Keep cruna_gradient's snapshots in pinned host memory (True) or in HBM (False, default).
        The pinned slots are kept for later gradient calls until False is set or the context closes."""
        self._check(self.lib.cruna_set_snapshot_memory(self.h, 1 if host else 0))

    def set_graphs(self, on: bool = True):
        """Record repeating loop steps as CUDA graphs inside run / gradient calls (default on)."""
        self._check(self.lib.cruna_set_graphs(self.h, 1 if on else 0))

    def graph_stats(self) -> Tuple[int, int]:
        """(graphs captured, graph replays) since the context was created."""
        cap, rep = C.c_int64(0), C.c_int64(0)
        self._check(self.lib.cruna_graph_stats(self.h, C.byref(cap), C.byref(rep)))
        return int(cap.value), int(rep.value)

    def profile(self, on: bool = True):
        self._check(self.lib.cruna_profile_enable(self.h, 1 if on else 0))

    def profile_report(self) -> dict:
        """{kernel family: (launches, total ms)} since profiling was enabled."""
        n = self.lib.cruna_profile_report(self.h, None, 0)
        if n < 0:
            self._check(n)
        buf = C.create_string_buffer(n + 1)
        self.lib.cruna_profile_report(self.h, buf, n + 1)
        out = {}
        for line in buf.value.decode().splitlines():
            name, cnt, ms = line.split()
            out[name] = (int(cnt), float(ms))
        return out

    def sync(self):
        self._check(self.lib.cruna_sync(self.h))

    def stream_handle(self) -> int:
        return int(self.lib.cruna_stream(self.h) or 0)

    # ---- snapshots and restart (src/main/cruna_hpc.f90:99-299, src/helper/io_helper.f90) -------
    def store_snapshot(self, q, workdir: str, ns: int, nt: int, kind: str = "data_direct_snapshot"):
        a = self._state(q)
        self._check(self.lib.cruna_store_snapshot(self.h, workdir.encode(), kind.encode(), _ptr(a), ns, nt))

    def load_snapshot(self, workdir: str, ns: int, nt: int, kind: str = "data_direct_snapshot") -> np.ndarray:
        a = np.zeros(self.n + (5,), order="F")
        self._check(self.lib.cruna_load_snapshot(self.h, workdir.encode(), kind.encode(), _ptr(a), ns, nt))
        return a

    def run_hpc(self, q0, workdir: str, steps: int, subsets: int = 1, dsfreq: int = 0, restart: bool = False,
                walltime: float = 0.0, max_steps: int = 0):
        """cruna_hpc's direct main loop with snapshots and restart; returns (q, stopped, (ns, nt)):
        stopped is True when the wall-time or step budget ended the call after storing a restart point."""
        a = np.array(self._state(q0), order="F", copy=True)
        o = HpcOpts(workdir.encode(), int(steps), int(subsets), int(dsfreq), 1 if restart else 0, float(walltime),
                    int(max_steps), 0)
        ns, nt = C.c_int(), C.c_int()
        rc = self.lib.cruna_run_hpc(self.h, _ptr(a), C.byref(o), C.byref(ns), C.byref(nt))
        if rc not in (0, CRUNA_STOPPED):
            self._check(rc)
        return a, rc == CRUNA_STOPPED, (ns.value, nt.value)


def _io_check(lib, rc: int) -> int:
    if rc < 0:
        raise CrunaError(rc, lib.cruna_last_error(None).decode())
    return rc


def io_fname(workdir: str, kind: str, ns: int = 1, nt: int = 0, world_block: int = 1, block_image: int = 1) -> str:
    """The reference's file name of a snapshot / restart file (src/helper/io_helper.f90:11-432), '.bin'."""
    lib = load_library()
    n = _io_check(lib, lib.cruna_io_fname(None, 0, workdir.encode(), kind.encode(), world_block, block_image, ns,
                                          nt))
    buf = C.create_string_buffer(n + 1)
    lib.cruna_io_fname(buf, n + 1, workdir.encode(), kind.encode(), world_block, block_image, ns, nt)
    return buf.value.decode()


def write_snapshot(path: str, data: np.ndarray, params: str = ""):
    """store_4d_rk (src/io/hdf5_single.f90:659-774) in the library's binary container."""
    lib = load_library()
    a = np.asfortranarray(np.asarray(data, dtype=np.float64))
    shape = tuple(a.shape) + (1,) * (4 - a.ndim)
    dims = (C.c_int64 * 4)(*shape)
    _io_check(lib, lib.cruna_write_snapshot(path.encode(), dims, _ptr(a), params.encode()))


def read_snapshot(path: str) -> Tuple[np.ndarray, str]:
    """The data (Fortran order, 4-D) and the params text of a snapshot file."""
    lib = load_library()
    dims = (C.c_int64 * 4)(0, 0, 0, 0)
    _io_check(lib, lib.cruna_read_snapshot(path.encode(), dims, None, None, 0))
    a = np.zeros(tuple(dims), order="F")
    txt = C.create_string_buffer(1 << 16)
    _io_check(lib, lib.cruna_read_snapshot(path.encode(), dims, _ptr(a), txt, 1 << 16))
    return a, txt.value.decode()


def write_restart(workdir: str, ns: int, nt: int):
    lib = load_library()
    _io_check(lib, lib.cruna_write_restart(workdir.encode(), int(ns), int(nt)))


def read_restart(workdir: str) -> Optional[Tuple[int, int]]:
    """(ns, nt) of restartfile.bin, or None when there is none (the reference then starts from 0)."""
    lib = load_library()
    ns, nt = C.c_int(), C.c_int()
    found = _io_check(lib, lib.cruna_read_restart(workdir.encode(), C.byref(ns), C.byref(nt)))
    return (ns.value, nt.value) if found == 1 else None


def restart_start(ns: int, nt: int, steps: int) -> Tuple[int, int]:
    """(s0, nt0) after restart point (ns, nt): src/main/cruna_hpc.f90:143-145."""
    lib = load_library()
    s0, nt0 = C.c_int(), C.c_int()
    _io_check(lib, lib.cruna_restart_start(int(ns), int(nt), int(steps), C.byref(s0), C.byref(nt0)))
    return s0.value, nt0.value
