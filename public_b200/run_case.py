"""Run one of the library's cases on the GPU and time its direct (and adjoint) loop steps.

    python -m public_b200.run_case --case mixing_layer --n 256 192 128 [--steps 10] [--warmup 3]
        [--adjoint] [--profile] [--no-graphs] [--json out.json]

Cases: taylor_green, mixing_layer, isentropic_vortex (n = one size), isotropic_turbulence.  The state
stays on the device; each timed call runs --steps loop steps through cruna_run_direct_dev (and, with
--adjoint, as many cruna_run_adjoint_dev steps on the final direct state), timed with CUDA events on
the context's stream.  --profile adds the library's per-family kernel times (events around each
launch; graphs are off while it is on).
"""
from __future__ import annotations

import argparse
import json

import numpy as np


def make_case(name: str, n):
    from . import cases
    if name == "taylor_green":
        return cases.taylor_green(n=n[0], seed=0)
    if name == "mixing_layer":
        return cases.mixing_layer(n=tuple(n))
    if name == "isentropic_vortex":
        return cases.isentropic_vortex(n=n[0])
    if name == "isotropic_turbulence":
        return cases.isotropic_turbulence(n=n[0])
    raise ValueError(f"unknown case {name}")


def run(args) -> dict:
    import torch

    from .cruna import Cruna, Settings

    dev = torch.device("cuda", 0)
    s, q = make_case(args.case, args.n)
    npts = int(np.prod(q.shape[:3]))
    qt = torch.from_numpy(np.ascontiguousarray(q.ravel(order="F"))).to(dev)
    out = {"case": args.case, "n": list(q.shape[:3]), "steps": args.steps}
    with Cruna(Settings.from_dict(s), qref=q) as c:
        c.set_graphs(not args.no_graphs)
        out["rhs_path"] = c.rhs_path
        st = torch.cuda.ExternalStream(c.stream_handle())
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        c.run_direct_dev(qt.data_ptr(), 0, args.warmup)
        c.sync()
        if args.profile:
            c.profile(True)
        e0.record(st)
        c.run_direct_dev(qt.data_ptr(), args.warmup, args.steps)
        e1.record(st)
        c.sync()
        out["direct_ms_per_step"] = e0.elapsed_time(e1) / args.steps
        out["direct_point_steps_per_s"] = npts / (out["direct_ms_per_step"] * 1e-3)
        if args.adjoint:
            qs = torch.zeros_like(qt)
            qs[: npts] = 1.0
            torch.cuda.current_stream().synchronize()   # the library reads qs on its own stream
            c.run_adjoint_dev(qs.data_ptr(), qt.data_ptr(), None, args.warmup, 1)
            c.sync()
            e0.record(st)
            for k in range(args.steps):     # the frozen direct state is the final one at every step
                c.run_adjoint_dev(qs.data_ptr(), qt.data_ptr(), None, args.steps - k, 1)
            e1.record(st)
            c.sync()
            out["adjoint_ms_per_step"] = e0.elapsed_time(e1) / args.steps
            out["adjoint_point_steps_per_s"] = npts / (out["adjoint_ms_per_step"] * 1e-3)
        if args.profile:
            rep = c.profile_report()
            c.profile(False)
            tot = sum(v[1] for v in rep.values()) or 1.0
            out["kernels"] = {k: {"launches": v[0], "total_ms": round(v[1], 4), "share": round(v[1] / tot, 4)}
                              for k, v in sorted(rep.items(), key=lambda kv: -kv[1][1])}
        out["graphs_captured_replayed"] = list(c.graph_stats())
    return out


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--case", default="mixing_layer")
    ap.add_argument("--n", type=int, nargs="+", default=[256, 192, 128])
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--adjoint", action="store_true")
    ap.add_argument("--profile", action="store_true")
    ap.add_argument("--no-graphs", action="store_true")
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
