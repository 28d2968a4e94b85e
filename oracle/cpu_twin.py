"""ctypes front end of oracle/cruna_cpu.c, the C + OpenMP restatement of the oracle used as the timed
CPU baseline (TEST INFRASTRUCTURE: only tests/ and bench.py's CPU legs use it).

build() compiles oracle/cruna_cpu.c into oracle/_build/libcruna_cpu.so (gcc -O3 -fopenmp, x86-64-v3);
run() advances (direct step + filters, adjoint step + filters) pairs on Fortran-ordered states.
"""
from __future__ import annotations

import ctypes as C
import shutil
import subprocess
from pathlib import Path
from typing import Optional

import numpy as np

HERE = Path(__file__).resolve().parent
SRC = HERE / "cruna_cpu.c"
LIB = HERE / "_build" / "libcruna_cpu.so"

# explicit periodic derivative cores the twin supports: half-width, coefficients, divisor
_DIFF = {
    "o4_e_c_p": (2, [0.0, 8.0, -1.0, 0.0, 0.0], 12.0),
    "o8_e_c_p": (4, [0.0, 4.0 / 5.0, -1.0 / 5.0, 4.0 / 105.0, -1.0 / 280.0], 1.0),
    "empty": (0, [0.0] * 5, 1.0),
}


class _Cfg(C.Structure):
    _fields_ = [("n", C.c_int * 3), ("dx", C.c_double * 3), ("r", C.c_int * 3), ("c", (C.c_double * 5) * 3),
                ("div", C.c_double * 3), ("fon", C.c_int * 3), ("fa", C.c_double * 6), ("blend", C.c_double),
                ("gamma", C.c_double), ("R", C.c_double), ("W", C.c_double), ("mu0", C.c_double),
                ("T0", C.c_double), ("Pr", C.c_double), ("dt", C.c_double), ("heat_flux_dx", C.c_int)]


def build(force: bool = False) -> Path:
    LIB.parent.mkdir(exist_ok=True)
    if LIB.exists() and not force and LIB.stat().st_mtime >= SRC.stat().st_mtime:
        return LIB
    cc = shutil.which("gcc") or "cc"
    cmd = [cc, "-O3", "-march=x86-64-v3", "-fopenmp", "-fPIC", "-shared", str(SRC), "-o", str(LIB), "-lm"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"building the CPU twin failed:\n{r.stderr}")
    return LIB


_lib = None


def load():
    global _lib
    if _lib is None:
        if not LIB.exists():
            build()
        _lib = C.CDLL(str(LIB))
        _lib.ccpu_run.restype = C.c_int
        _lib.ccpu_run.argtypes = [C.POINTER(_Cfg), C.c_void_p, C.c_void_p, C.c_int, C.c_int]
        _lib.ccpu_threads.restype = C.c_int
    return _lib


def supports(settings: dict) -> bool:
    return (all(s in _DIFF for s in settings["diff"]) and not settings.get("bc") is not None
            and all(f in ("empty", "o10_e_c_p") for f in settings.get("filt", ("empty",) * 3)))


def make_cfg(settings: dict) -> _Cfg:
    from oracle import cruna_oracle as O
    fields = {f.name for f in O.dataclasses.fields(O.Config)}
    oc = O.Config(**{k: v for k, v in settings.items() if k in fields})
    c = _Cfg()
    dx = oc.dx()
    for d in range(3):
        r, coef, div = _DIFF[oc.diff[d]]
        c.n[d] = oc.n[d]
        c.dx[d] = dx[d] if np.isfinite(dx[d]) else 1.0
        c.r[d] = r
        for m in range(5):
            c.c[d][m] = coef[m]
        c.div[d] = div
        c.fon[d] = 1 if (oc.filt[d] == "o10_e_c_p" and oc.di_freq[d] == 1) else 0
    fa = O.filter_interior_coeffs("o10_e_c_p", 0.0)
    for m in range(6):
        c.fa[m] = fa[m]
    c.blend = oc.strength
    c.gamma, c.R, c.W, c.mu0, c.T0, c.Pr, c.dt = oc.gamma, oc.R, oc.W, oc.mu0, oc.T0, oc.Pr, oc.dt
    c.heat_flux_dx = 1 if oc.heat_flux_dx else 0
    return c


def run(settings: dict, q: np.ndarray, qs: Optional[np.ndarray], nsteps: int, threads: int = 0):
    """Advances q (and qs, when given) in place by nsteps direct(+adjoint) step pairs."""
    lib = load()
    cfg = make_cfg(settings)
    assert q.flags.f_contiguous and (qs is None or qs.flags.f_contiguous)
    rc = lib.ccpu_run(C.byref(cfg), q.ctypes.data, None if qs is None else qs.ctypes.data, int(nsteps),
                      int(threads))
    if rc != 0:
        raise MemoryError("CPU twin could not allocate its temporaries")


def threads() -> int:
    return int(load().ccpu_threads())
