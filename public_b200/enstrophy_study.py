"""Enstrophy-gradient study: Taylor-Green at Re 3200, Mach 0.2 with FP32 stencils and FP64 RK4 state.

    python -m public_b200.enstrophy_study [--n 576] [--steps 100] [--nsnap 3] [--ndir 2]
        [--eps 1e-3] [--precision fp32] [--host-snapshots] [--json out.json]

J is the enstrophy sum dV |curl u|^2 / 2 after --steps direct steps (``CRUNA_OBJ_ENSTROPHY``); its
gradient with respect to the initial state comes from ``cruna_gradient`` (the reference's continuous
adjoint, binomial checkpointing in --nsnap HBM snapshots).  The derivative along --ndir seeded random
perturbations of the initial velocity, q0 + eps (0, rho du, rho dv, rho dw, 0) with du, dv, dw ~ N(0, 1)
scaled by the velocity magnitude, is compared with central differences of J.  Time per direct step,
gradient time and direct steps executed are reported.

Device memory is kept to the context and four states: the gradient overwrites the device copy of q0
(grad_q0 aliases q0), --host-snapshots keeps the snapshots in pinned host memory, and the perturbed
states are formed in place -- which lets the 768^3 grid (18.1 GB per state) run on one GPU.
"""
from __future__ import annotations

import argparse
import json
import sys
import time

import numpy as np


def run(args) -> dict:
    import torch

    from . import cases
    from .cruna import Cruna, Settings

    dev = torch.device("cuda", 0)
    s, q0 = cases.taylor_green(n=args.n, mach=0.2, reynolds=3200.0, seed=0)
    s = dict(s, precision=args.precision)
    N = int(np.prod(q0.shape[:3]))
    u0 = float(np.max(np.abs(q0[..., 1] / q0[..., 0])))
    q = torch.from_numpy(np.ascontiguousarray(q0.ravel(order="F"))).to(dev)
    out = {"workload": f"Taylor-Green Re 3200 Mach 0.2, {args.n}^3, {args.steps} steps, {args.precision} stencils, "
                       f"{args.nsnap} snapshots", "t_end": args.steps * s["dt"]}
    torch.cuda.synchronize()
    with Cruna(Settings.from_dict(s)) as c:
        c.set_snapshot_memory(args.host_snapshots)
        obj = c.objective("enstrophy")
        torch.cuda.synchronize()
        t0 = time.time()
        J, adv = c.gradient_dev(q.data_ptr(), args.steps, args.nsnap, obj, None, q.data_ptr())  # q <- dJ/dq0
        c.sync()
        out.update(J=J, gradient_seconds=time.time() - t0, direct_steps=adv)
        print(json.dumps(out), file=sys.stderr, flush=True)
        gq = q
        q = torch.from_numpy(np.ascontiguousarray(q0.ravel(order="F"))).to(dev)
        torch.cuda.synchronize()
        st = torch.cuda.ExternalStream(c.stream_handle())
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        J0 = c.objective_value_dev(q.data_ptr(), args.steps, obj)
        e1.record(st)
        c.sync()
        out["J_objective_value"] = J0
        out["ms_per_direct_step_with_objective"] = e0.elapsed_time(e1) / args.steps
        print(json.dumps(out), file=sys.stderr, flush=True)
        gen = torch.Generator(device=dev)
        gen.manual_seed(5)
        dirs = []
        for k in range(args.ndir):
            d = torch.zeros_like(q)
            for v in range(3):
                d[(1 + v) * N:(2 + v) * N] = torch.randn(N, generator=gen, device=dev, dtype=torch.float64) * q[:N] * u0
            dot = sum(float(torch.dot(a, b).item()) for a, b in zip(gq.split(1 << 28), d.split(1 << 28)))
            dirs.append((d, dot))  # cuBLAS dot takes at most 2^31 - 1 elements: sum it in chunks
            if k == 0 and args.ndir == 1:
                break
        del gq
        torch.cuda.empty_cache()
        rows = []
        for d, ad in dirs:
            q.add_(d, alpha=args.eps)
            torch.cuda.current_stream().synchronize()
            Jp = c.objective_value_dev(q.data_ptr(), args.steps, obj)
            q.sub_(d, alpha=2 * args.eps)
            torch.cuda.current_stream().synchronize()
            Jm = c.objective_value_dev(q.data_ptr(), args.steps, obj)
            q.add_(d, alpha=args.eps)
            fd = (Jp - Jm) / (2 * args.eps)
            rows.append({"adjoint": ad, "fd": fd, "rel_err": abs(ad - fd) / abs(fd)})
        out["directions"] = rows
    return out


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--n", type=int, default=576)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--nsnap", type=int, default=3)
    ap.add_argument("--ndir", type=int, default=2)
    ap.add_argument("--eps", type=float, default=1e-3)
    ap.add_argument("--precision", default="fp32", choices=["fp64", "fp32"])
    ap.add_argument("--host-snapshots", action="store_true")
    ap.add_argument("--json", default=None)
    args = ap.parse_args(argv)
    res = run(args)
    line = json.dumps(res)
    print(line)
    if args.json:
        with open(args.json, "w") as fh:
            fh.write(line + "\n")


if __name__ == "__main__":
    main()
