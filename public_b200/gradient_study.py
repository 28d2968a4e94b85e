"""Adjoint-gradient study on the temporal mixing layer (the mixing-layer configuration with adjoint).

Objective: J = sum over the direct steps of dt * integral over the plane y = y_plane of (p - p_inf)^2 dA
(y_plane measured from the lower boundary of the 60-high box, 5 below the layer's centre by default)
(computed on the device, ``cruna_objective_value``); control: a time-constant forcing of the pressure
equation (the fifth RHS component).  For both adjoints the library offers -- the reference's
continuous inviscid adjoint (mode 0) and the exact discrete adjoint (mode 1) -- the gradient comes from
``cruna_gradient`` with binomial checkpointing in ``nsnap`` HBM snapshots, and is checked against
central finite differences of J on ``ndir`` random directions (seed 2).

The mixing layer has type-201 characteristic boundaries, which switch waves on the sign of v at the
y boundaries: J is only piecewise smooth, so a difference step must be small enough that no boundary
point changes branch; the study reports the comparison at two steps (``--eps``, default 1e-6 and
1e-7).

    python -m public_b200.gradient_study [--n 128 96 64] [--steps 200] [--nsnap 64] [--ndir 16]
        [--eps 1e-6 1e-7] [--fd-dirs K] [--modes 0 1] [--fd-from earlier.json] [--host-snapshots]
        [--json out.json]

A long horizon can be split over several processes: a run with ``--modes`` (none) computes and stores the
difference quotients, a later one with ``--fd-from`` reuses them and runs the adjoints.
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np


def run(args) -> dict:
    import torch

    from . import cases
    from .cruna import Cruna, Settings

    dev = torch.device("cuda", 0)
    n = tuple(args.n)
    s, q0 = cases.mixing_layer(n=n)
    L_y = s["x1"][1] - s["x0"][1]
    dy = L_y / (n[1] - 1)
    j_plane = int(round(args.y_plane / dy)) + 1       # 1-based index, distance from the lower y boundary
    p_inf = float(np.mean(q0[..., 4]))
    N = int(np.prod(n))
    q = torch.from_numpy(np.ascontiguousarray(q0.ravel(order="F"))).to(dev)
    f = torch.zeros(5 * N, dtype=torch.float64, device=dev)
    gf = torch.empty_like(f)
    out = {"workload": f"mixing layer {n[0]}x{n[1]}x{n[2]}, {args.steps} steps, plane y={args.y_plane} "
                       f"from the lower boundary (index {j_plane}), pressure-equation forcing, {args.nsnap} snapshots",
           "ndir": args.ndir}
    rng = np.random.Generator(np.random.PCG64(2))
    dirs = []
    for _ in range(args.ndir):
        d = np.zeros((N, 5))
        d[:, 4] = rng.standard_normal(N)
        dirs.append(torch.from_numpy(np.ascontiguousarray(d.T.ravel())).to(dev))
    # the library's _dev calls run on its own stream: every torch result they read must be complete
    torch.cuda.synchronize()
    with Cruna(Settings.from_dict(s), qref=q0, force=np.zeros_like(q0)) as c:
        obj = c.objective("plane_p2", normal=2, index=j_plane, p_inf=p_inf)
        c.set_forcing_dev(f.data_ptr())
        J0 = c.objective_value_dev(q.data_ptr(), args.steps, obj)
        out["J"] = J0
        fd = {}
        t0 = time.time()
        prior = {}
        if args.fd_from:
            # difference quotients of an earlier run of the same workload (same seeded directions)
            with open(args.fd_from) as fh:
                old = json.loads(fh.readline())
            if old.get("workload") != out["workload"]:
                raise ValueError("--fd-from holds another workload")
            prior = {float(k): np.array(v) for k, v in old["fd"].items()}
        for eps in args.eps:
            if eps in prior:
                fd[eps] = prior[eps]
                continue
            vals = []
            for d in dirs[args.fd_start:args.fd_start + args.fd_dirs]:
                fp = f + eps * d
                torch.cuda.current_stream().synchronize()
                c.set_forcing_dev(fp.data_ptr())
                Jp = c.objective_value_dev(q.data_ptr(), args.steps, obj)
                fm = f - eps * d
                torch.cuda.current_stream().synchronize()
                c.set_forcing_dev(fm.data_ptr())
                Jm = c.objective_value_dev(q.data_ptr(), args.steps, obj)
                vals.append((Jp - Jm) / (2 * eps))
            fd[eps] = np.array(vals)
        out["fd_seconds"] = time.time() - t0
        out["fd"] = {f"{eps:g}": v.tolist() for eps, v in fd.items()}
        out["fd_start"] = args.fd_start
        c.set_forcing_dev(f.data_ptr())
        if getattr(args, "host_snapshots", False):
            c.set_snapshot_memory(True)               # snapshots in pinned host memory, HBM cache of one
        for mode in args.modes:
            c.set_adjoint_mode(mode)
            torch.cuda.synchronize()
            t0 = time.time()
            J, adv = c.gradient_dev(q.data_ptr(), args.steps, args.nsnap, obj, gf.data_ptr(), None)
            c.sync()
            secs = time.time() - t0
            g5 = gf.view(5, N)[4]
            ad_all = np.array([float((g5 * d.view(5, N)[4]).sum().item()) for d in dirs])
            key = "continuous" if mode == 0 else "discrete"
            res = {"J": J, "direct_steps": adv, "seconds": secs}
            res["directional_derivatives"] = ad_all.tolist()
            for eps, v in fd.items():
                ad = ad_all[args.fd_start:args.fd_start + len(v)]
                rel = np.abs(ad - v) / np.maximum(np.abs(v), 1e-300)
                res[f"fd_rel_err_eps{eps:g}"] = {"median": float(np.median(rel)), "max": float(np.max(rel))}
                res[f"cosine_eps{eps:g}"] = float(np.dot(ad, v) / (np.linalg.norm(ad) * np.linalg.norm(v)))
            out[key] = res
        c.set_adjoint_mode(0)
    return out


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--n", type=int, nargs=3, default=[128, 96, 64])
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--nsnap", type=int, default=64)
    ap.add_argument("--ndir", type=int, default=16)
    ap.add_argument("--y-plane", type=float, default=25.0)
    ap.add_argument("--eps", type=float, nargs="+", default=[1e-6, 1e-7])
    ap.add_argument("--fd-dirs", type=int, default=None,
                    help="finite differences on the first K of the ndir directions only (default: all)")
    ap.add_argument("--fd-start", type=int, default=0,
                    help="first of the directions taken by the finite differences (with --fd-dirs: a later slice)")
    ap.add_argument("--fd-from", type=str, default=None,
                    help="reuse the difference quotients of an earlier run's JSON (same workload)")
    ap.add_argument("--modes", type=int, nargs="*", default=[0, 1],
                    help="adjoint modes to run: 0 continuous (reference), 1 exact discrete; none = FD only")
    ap.add_argument("--host-snapshots", action="store_true",
                    help="keep the binomial snapshots in pinned host memory (states too large for nsnap HBM copies)")
    ap.add_argument("--json", type=str, default=None)
    args = ap.parse_args(argv)
    if args.fd_dirs is None:
        args.fd_dirs = args.ndir
    res = run(args)
    line = json.dumps(res)
    print(line)
    if args.json:
        with open(args.json, "w") as fh:
            fh.write(line + "\n")


if __name__ == "__main__":
    main()
