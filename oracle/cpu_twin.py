"""ctypes front end of oracle/cruna_cpu.c, the C + OpenMP restatement of the oracle used as the timed
CPU baseline (TEST INFRASTRUCTURE: only tests/ and the CPU legs of bench.py and oracle/cpu_legs.py use
it).

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
                ("T0", C.c_double), ("Pr", C.c_double), ("dt", C.c_double), ("heat_flux_dx", C.c_int),
                ("dkind", C.c_int * 3), ("dfac", (C.c_void_p * 4) * 3), ("dpiv", C.c_void_p * 3),
                ("fkind", C.c_int * 3), ("fo", C.c_double * 6), ("fbrow", (C.c_double * 11) * 4),
                ("ffac", (C.c_void_p * 4) * 3), ("fpiv", C.c_void_p * 3), ("nbc", C.c_int), ("bc", C.c_void_p),
                ("qref", C.c_void_p), ("shape", C.c_void_p)]

_COMPACT_DIFF = {"o6_i_c_o"}
_FILTERS = ("empty", "o10_e_c_p", "o10_i_c_o")
_BC_TYPES = (201, 400)


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
    """Periodic explicit cores with the periodic o10 filter (no boundary rows), or the mixing-layer set:
    o6 compact open derivatives, the o10 compact open filter, type-201 rows and the type-400 sponge."""
    bc = settings.get("bc")
    rows_ok = bc is None or all(int(round(r[0])) in _BC_TYPES for r in np.asarray(bc).reshape(-1, 10))
    filt = settings.get("filt", ("empty",) * 3)
    freq = settings.get("di_freq", (1, 1, 1))
    filters_ok = all(f in _FILTERS and (f == "empty" or fr == 1) for f, fr in zip(filt, freq))
    return all(s in _DIFF or s in _COMPACT_DIFF for s in settings["diff"]) and rows_ok and filters_ok


def _factors(f, keep: list):
    """dgttrf factors of the oracle (scipy's LAPACK) as pointers for the C restatement of dgttrs."""
    arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in (f.dl, f.d, f.du, f.du2)]
    piv = np.ascontiguousarray(f.ipiv, dtype=np.int32)
    keep.extend(arrs + [piv])
    return [a.ctypes.data for a in arrs], piv.ctypes.data


def make_cfg(settings: dict, qref: Optional[np.ndarray] = None) -> _Cfg:
    from oracle import cruna_oracle as O
    fields = {f.name for f in O.dataclasses.fields(O.Config)}
    oc = O.Config(**{k: v for k, v in settings.items() if k in fields})
    c = _Cfg()
    keep: list = []                      # arrays the C side reads through pointers during the run
    dx = oc.dx()
    for d in range(3):
        c.n[d] = oc.n[d]
        c.dx[d] = dx[d] if np.isfinite(dx[d]) else 1.0
        if oc.diff[d] in _COMPACT_DIFF:
            c.dkind[d] = 1
            ptrs, piv = _factors(O.diff_factors(oc.diff[d], oc.n[d]), keep)
            for m in range(4):
                c.dfac[d][m] = ptrs[m]
            c.dpiv[d] = piv
            c.div[d] = 1.0
        else:
            r, coef, div = _DIFF[oc.diff[d]]
            c.r[d] = r
            for m in range(5):
                c.c[d][m] = coef[m]
            c.div[d] = div
        on = oc.filt[d] != "empty" and oc.di_freq[d] == 1
        c.fon[d] = 1 if on else 0
        if on and oc.filt[d] == "o10_i_c_o":
            c.fkind[d] = 1
            ptrs, piv = _factors(O.filter_factors("o10_i_c_o", oc.n[d], oc.alpha), keep)
            for m in range(4):
                c.ffac[d][m] = ptrs[m]
            c.fpiv[d] = piv
    fa = O.filter_interior_coeffs("o10_e_c_p", 0.0)
    for m in range(6):
        c.fa[m] = fa[m]
    fo = O.filter_interior_coeffs("o10_i_c_o", oc.alpha)
    for m in range(6):
        c.fo[m] = fo[m]
    fb = O.filter_boundary_coeffs("o10_i_c_o", oc.alpha)
    for row in range(4):
        for m in range(11):
            c.fbrow[row][m] = fb[row, m]
    c.blend = oc.strength
    c.gamma, c.R, c.W, c.mu0, c.T0, c.Pr, c.dt = oc.gamma, oc.R, oc.W, oc.mu0, oc.T0, oc.Pr, oc.dt
    c.heat_flux_dx = 1 if oc.heat_flux_dx else 0
    if oc.bc is not None and len(oc.bc):
        bc = np.ascontiguousarray(np.asarray(oc.bc, dtype=np.float64).reshape(-1, 10))
        keep.append(bc)
        c.nbc, c.bc = bc.shape[0], bc.ctypes.data
        if qref is None:
            raise ValueError("boundary rows of types 201 / 400 need the reference state qref")
        qr = np.asfortranarray(qref, dtype=np.float64)
        keep.append(qr)
        c.qref = qr.ctypes.data
        if any(int(round(r[0])) == 400 for r in bc):
            sh = np.asfortranarray(O.sponge_shape(oc))
            keep.append(sh)
            c.shape = sh.ctypes.data
    c._keep = keep
    return c


def run(settings: dict, q: np.ndarray, qs: Optional[np.ndarray], nsteps: int, threads: int = 0,
        qref: Optional[np.ndarray] = None):
    """Advances q (and qs, when given) in place by nsteps direct(+adjoint) step pairs; qref is the
    reference state of boundary rows of types 201 and 400."""
    lib = load()
    cfg = make_cfg(settings, qref)
    assert q.flags.f_contiguous and (qs is None or qs.flags.f_contiguous)
    rc = lib.ccpu_run(C.byref(cfg), q.ctypes.data, None if qs is None else qs.ctypes.data, int(nsteps),
                      int(threads))
    if rc != 0:
        raise MemoryError("CPU twin could not allocate its temporaries")


def threads() -> int:
    return int(load().ccpu_threads())
