"""Generates the golden fixtures in this directory from the CPU oracle (oracle/cruna_oracle.py).

Run from the repository root:  python tests/golden/make_golden.py
The fixtures are small (<1 MB total) seeded / analytic cases; the tests compare both the oracle
(so that a change of the oracle is noticed) and the CUDA library against them.
"""
from __future__ import annotations

import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle import cruna_oracle as O  # noqa: E402
from public_b200 import cases  # noqa: E402

HERE = os.path.dirname(os.path.abspath(__file__))


def oracle_cfg(settings: dict) -> O.Config:
    names = {f.name for f in O.dataclasses.fields(O.Config)}
    return O.Config(**{k: v for k, v in settings.items() if k in names})


def operators():
    """Every derivative and filter core along every direction on one smooth random field."""
    n = (13, 12, 11)
    q = cases.smooth_random_state(n, seed=11)
    out = {"q": q}
    for s in O.DIFF_SCHEMES:
        cfg = O.Config(n=n, diff=(s, s, s))
        dx = cfg.dx()
        for d in range(3):
            out[f"diff_{s}_{d + 1}"] = O.Dx(cfg, d, q[..., 4], dx[d])
    for s in O.FILTER_SCHEMES:
        cfg = O.Config(n=n, filt=(s, s, s), alpha=0.3)
        for d in range(3):
            out[f"filter_{s}_{d + 1}"] = O.filter_dir(cfg, d, q[..., 4:5])[..., 0]
    np.savez_compressed(os.path.join(HERE, "operators.npz"), **out)


def tgv():
    s, q0 = cases.taylor_green(n=12, seed=0)
    s["mu0"] = 0.05                      # visible viscous terms on the coarse grid
    cfg = oracle_cfg(s)
    S = O.Solver(cfg)
    rhs = S.rhs_direct(q0)
    q5 = S.calc_direct(q0, 5)
    np.savez_compressed(os.path.join(HERE, "tgv12.npz"), q0=q0, rhs=rhs, q5=q5, mu0=s["mu0"], dt=s["dt"])


def pulse():
    s, q0 = cases.gaussian_pulse(n=(14, 15, 16))
    cfg = oracle_cfg(s)
    S = O.Solver(cfg, qref=q0.copy())
    rhs = S.rhs_direct(q0)
    q5 = S.calc_direct(q0, 5)
    qs0 = cases.smooth_random_state((14, 15, 16), seed=5, p0=0.0, rho0=0.0, amp=1.0)
    rhs_adj = S.rhs_adjoint(qs0, q5, np.zeros_like(q0))
    np.savez_compressed(os.path.join(HERE, "pulse14.npz"), q0=q0, rhs=rhs, q5=q5, qs0=qs0, rhs_adj=rhs_adj)


def vortex():
    s, q0 = cases.isentropic_vortex(n=32)
    cfg = oracle_cfg(s)
    S = O.Solver(cfg)
    q10 = S.calc_direct(q0, 10)
    np.savez_compressed(os.path.join(HERE, "vortex32.npz"), q0=q0, q10=q10, dt=s["dt"])


if __name__ == "__main__":
    operators()
    tgv()
    pulse()
    vortex()
    for f in sorted(os.listdir(HERE)):
        if f.endswith(".npz"):
            print(f, os.path.getsize(os.path.join(HERE, f)))
