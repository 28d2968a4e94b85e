"""Taylor-Green study: the plain FP64 path against the FP32-stencil path on the same seeded start.

    python -m public_b200.tgv_study [--n 256] [--steps 2000] [--every 50] [--json out.json]

The Taylor-Green configuration (Mach 0.1, Re 1600, o8 differences, o10 filter every step, RK4 at CFL
0.5; density perturbation 1e-4, seed 0) runs --steps steps in each precision; every --every steps the
kinetic energy and the enstrophy (cruna_diagnostics_dev, FP64 reductions) are recorded.  Reported:
both histories, their largest relative difference, the final per-variable relative L2 difference of
the FP32-stencil state from the FP64 state, and the time per step of each path (CUDA events).
"""
from __future__ import annotations

import argparse
import json

import numpy as np


def run(args) -> dict:
    import torch

    from . import cases
    from .cruna import Cruna, Settings

    dev = torch.device("cuda", 0)
    s, q0 = cases.taylor_green(n=args.n, seed=0)
    N = int(np.prod(q0.shape[:3]))
    out = {"workload": f"Taylor-Green {args.n}^3, {args.steps} steps, diagnostics every {args.every}",
           "t_end": args.steps * s["dt"]}
    finals = {}
    for prec in ("fp64", "fp32"):
        qt = torch.from_numpy(np.ascontiguousarray(q0.ravel(order="F"))).to(dev)
        hist = {"step": [], "kinetic_energy": [], "enstrophy": []}
        ms = 0.0
        with Cruna(Settings.from_dict(dict(s, precision=prec))) as c:
            st = torch.cuda.ExternalStream(c.stream_handle())
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            nt = 0
            while True:
                ke, z = c.diagnostics_dev(qt.data_ptr())
                hist["step"].append(nt)
                hist["kinetic_energy"].append(ke)
                hist["enstrophy"].append(z)
                if nt >= args.steps:
                    break
                k = min(args.every, args.steps - nt)
                e0.record(st)
                c.run_direct_dev(qt.data_ptr(), nt, k)
                e1.record(st)
                c.sync()
                ms += e0.elapsed_time(e1)
                nt += k
        out[prec] = {"history": hist, "ms_per_step": ms / args.steps,
                     "point_steps_per_s": N * args.steps / (ms * 1e-3)}
        finals[prec] = qt.view(5, N).double()
    a, b = finals["fp32"], finals["fp64"]
    out["fp32_vs_fp64_rel_l2"] = [float(torch.linalg.norm(a[v] - b[v]) / torch.linalg.norm(b[v]))
                                  if float(torch.linalg.norm(b[v])) > 0 else float(torch.linalg.norm(a[v]))
                                  for v in range(5)]
    for key in ("kinetic_energy", "enstrophy"):
        h64 = np.array(out["fp64"]["history"][key])
        h32 = np.array(out["fp32"]["history"][key])
        out[f"{key}_max_rel_diff"] = float(np.max(np.abs(h32 - h64) / np.abs(h64)))
    out["speedup_fp32"] = out["fp64"]["ms_per_step"] / out["fp32"]["ms_per_step"]
    return out


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--n", type=int, default=256)
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--every", type=int, default=50)
    ap.add_argument("--json", default=None)
    args = ap.parse_args(argv)
    res = run(args)
    line = json.dumps(res)
    print(json.dumps({k: v for k, v in res.items() if k not in ("fp64", "fp32")}))
    if args.json:
        with open(args.json, "w") as fh:
            fh.write(line + "\n")


if __name__ == "__main__":
    main()
