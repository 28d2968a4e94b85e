"""CPU tests of the C ABI: the library loads, exports every symbol the header declares, its LAPACK
restatement equals LAPACK, and the configuration defaults are the reference's."""
import ctypes as C
import os
import re

import numpy as np
import pytest
from scipy.linalg import lapack

from public_b200 import cruna
from tests.conftest import gpu_available

HEADER = os.path.join(os.path.dirname(os.path.dirname(__file__)), "include", "cruna_b200.h")


def declared_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(cruna_[a-z0-9_]+)\s*\(", src)))


def test_header_symbols_exported(lib):
    names = declared_functions()
    assert len(names) >= 40
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    # and the python binding knows every one of them
    assert set(names) <= set(cruna._SIGNATURES), set(names) - set(cruna._SIGNATURES)


@pytest.mark.parametrize("n", [3, 4, 7, 16, 65])
def test_dgttrf_dgttrs_equal_lapack(lib, n):
    rng = np.random.default_rng(n)
    for trial in range(4):
        dl, d, du = rng.standard_normal(n - 1), rng.standard_normal(n), rng.standard_normal(n - 1)
        if trial == 0:
            d *= 1e-3     # force row interchanges
        ref = lapack.dgttrf(dl, d, du)
        a, b, c = dl.copy(), d.copy(), du.copy()
        du2 = np.zeros(max(n - 2, 1))
        ipiv = np.zeros(n, dtype=np.int32)
        info = lib.cruna_lapack_dgttrf(n, a.ctypes.data, b.ctypes.data, c.ctypes.data, du2.ctypes.data,
                                       ipiv.ctypes.data)
        assert info == ref[5]
        assert np.array_equal(a, ref[0]) and np.array_equal(b, ref[1]) and np.array_equal(c, ref[2])
        assert np.array_equal(du2[:max(n - 2, 0)], ref[3][:max(n - 2, 0)]) and np.array_equal(ipiv, ref[4])
        x = rng.standard_normal(n)
        xr = lapack.dgttrs(*ref[:5], x.copy())[0]
        lib.cruna_lapack_dgttrs(n, a.ctypes.data, b.ctypes.data, c.ctypes.data, du2.ctypes.data,
                                ipiv.ctypes.data, x.ctypes.data)
        assert np.array_equal(x, xr)


def test_config_defaults_are_reference_defaults(lib):
    c = cruna._Config()
    lib.cruna_config_defaults(C.byref(c))
    assert c.abi_version == cruna.ABI_VERSION
    assert c.R == 8.3144598 and c.W == 0.0289647 and c.T0 == 273.0 and c.Pr == 0.71
    assert c.filter_alpha == 0.35 and c.sponge_amplitude == 1.0 and list(c.sponge_length) == [0.3] * 3


def test_settings_struct_roundtrip(lib):
    s = cruna.Settings(n=(8, 9, 10), diff=("o6_i_c_p", "o4_e_c_o", "empty"), filt=("o10_i_c_o",) * 3,
                       di_freq=(1, 2, 3), mu0=1e-3, precision="fp32")
    c = s.to_struct(lib)
    assert list(c.n) == [8, 9, 10] and list(c.diff) == [6, 3, 0] and list(c.filter) == [7, 7, 7]
    assert list(c.di_freq) == [1, 2, 3] and c.precision == 1 and c.mu0 == 1e-3


@pytest.mark.skipif(gpu_available(), reason="checks the no-device error path")
def test_init_without_device_fails_cleanly(lib):
    s = cruna.Settings(n=(8, 8, 8))
    with pytest.raises(cruna.CrunaError) as e:
        cruna.Cruna(s)
    assert e.value.code == -6


def test_missing_library_fails_loudly(tmp_path):
    with pytest.raises(FileNotFoundError):
        cruna.load_library(tmp_path / "nope.so")


def header_arity():
    """Number of parameters of every prototype in the header (function-pointer parameters count once)."""
    src = re.sub(r"/\*.*?\*/", "", open(HEADER).read(), flags=re.S)
    out = {}
    for m in re.finditer(r"\b(cruna_[a-z0-9_]+)\s*\(", src):
        depth, i = 1, m.end()
        while depth:
            depth += {"(": 1, ")": -1}.get(src[i], 0)
            i += 1
        params, depth, n = src[m.end():i - 1], 0, 1
        if src[i:].lstrip()[:1] != ";":
            continue                      # a function-pointer parameter or a macro, not a prototype
        for ch in params:
            depth += {"(": 1, ")": -1}.get(ch, 0)
            n += ch == "," and depth == 0
        out[m.group(1)] = 0 if params.strip() in ("", "void") else n
    return out


def test_python_binding_arity_matches_header():
    arity = header_arity()
    assert len(arity) >= 40
    bad = {k: (arity[k], len(cruna._SIGNATURES[k][1])) for k in arity
           if k in cruna._SIGNATURES and len(cruna._SIGNATURES[k][1]) != arity[k]}
    assert not bad, bad


def test_fortran_interfaces_match_header():
    """The iso_c_binding interfaces printed for Fortran cases bind existing entry points with the
    header's number of arguments."""
    doc = open(os.path.join(os.path.dirname(HEADER), os.pardir, "INTEGRATION.md")).read()
    arity = header_arity()
    found = re.findall(r"(?:function|subroutine)\s+(cruna_[a-z0-9_]+)\s*\(([^)]*)\)", doc)
    assert len(found) >= 30
    for name, args in found:
        assert name in arity, name
        n = len([a for a in args.replace("&", "").split(",") if a.strip()])
        assert n == arity[name], (name, n, arity[name])
