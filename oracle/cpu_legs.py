"""CPU baseline legs beside the headline: the C + OpenMP restatement of the oracle (cruna_cpu.c) timed on
the host cores, all of them and one, on the configurations of the benchmark suite.  TEST
INFRASTRUCTURE: it measures the reported CPU baselines and is never part of the product.

  python -m oracle.cpu_legs [--legs vortex tgv mixing] [--json out.json]

Legs (grid point-steps per second; the state generated once, one untimed warm-up step first):
  vortex   2-D isentropic vortex 256 x 256, 1000 direct steps on all threads, 200 on one thread
  tgv      Taylor-Green 256^3, 2 direct + 2 adjoint steps on all threads; 128^3, 1 + 1 on one thread
  mixing   mixing layer 512 x 384 x 256 (o6 compact y, o10 open filter, type-201 rows, sponge),
           3 direct + 3 adjoint steps on all threads
  closure  the closure configuration's coarse grid: isotropic turbulence 64^3, 100 direct steps of the
           plain filter-stabilised solve on all threads and 20 on one; the closure network
           (12 -> 64 -> 64 -> 6, GELU) in FP32 on the host cores through torch, forward and
           forward + backward of a mean-squared loss on 10^5 samples (best of 3 after a warm-up)
Direct and adjoint rates are separated by timing direct-only steps, then direct + adjoint pairs.
"""
from __future__ import annotations

import argparse
import json
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def _leg(settings, q0, qref, steps: int, threads: int, adjoint: bool) -> dict:
    from oracle import cpu_twin

    npts = int(np.prod(settings["n"]))
    q = np.array(q0, order="F", copy=True)
    cpu_twin.run(settings, q, None, 1, threads, qref=qref)              # warm-up (page faults, pool)
    t0 = time.perf_counter()
    cpu_twin.run(settings, q, None, steps, threads, qref=qref)
    t_dir = time.perf_counter() - t0
    out = {"points": npts, "steps": steps, "threads": threads if threads > 0 else cpu_twin.threads(),
           "direct_seconds": t_dir, "direct_point_steps_per_s": npts * steps / t_dir}
    if adjoint:
        q = np.array(q0, order="F", copy=True)
        qs = np.asfortranarray(1e-3 * np.ones_like(q0))
        cpu_twin.run(settings, q, qs, 1, threads, qref=qref)
        t0 = time.perf_counter()
        cpu_twin.run(settings, q, qs, steps, threads, qref=qref)
        t_pair = time.perf_counter() - t0
        t_adj = max(t_pair - t_dir, 1e-9)
        out.update({"pair_seconds": t_pair, "adjoint_point_steps_per_s": npts * steps / t_adj,
                    "pair_point_steps_per_s": npts * steps / t_pair})
    return out


def run(legs) -> dict:
    from oracle import cpu_twin
    from public_b200 import cases

    cpu_twin.build()
    res = {"host_threads": cpu_twin.threads(), "kind": "port (C + OpenMP restatement of the oracle)"}
    if "vortex" in legs:
        s, q0 = cases.isentropic_vortex(n=256)
        res["vortex_256x256"] = {"all": _leg(s, q0, None, 1000, 0, False), "one": _leg(s, q0, None, 200, 1, False)}
    if "tgv" in legs:
        s, q0 = cases.taylor_green(n=256, seed=0)
        s["ai_freq"] = (1, 1, 1)
        s1, q1 = cases.taylor_green(n=128, seed=0)
        s1["ai_freq"] = (1, 1, 1)
        res["taylor_green_256"] = {"all": _leg(s, q0, None, 2, 0, True)}
        res["taylor_green_128_one_thread"] = {"one": _leg(s1, q1, None, 1, 1, True)}
    if "mixing" in legs:
        s, q0 = cases.mixing_layer(n=(512, 384, 256))
        assert cpu_twin.supports(s)
        res["mixing_layer_512x384x256"] = {"all": _leg(s, q0, q0, 3, 0, True)}
    if "closure" in legs:
        s, q0 = cases.isotropic_turbulence(n=64)
        assert cpu_twin.supports(s)
        res["isotropic_coarse_64"] = {"all": _leg(s, q0, None, 100, 0, False), "one": _leg(s, q0, None, 20, 1, False)}
        res["closure_mlp_1e5_samples"] = _mlp_leg(100_000)
    return res


def _mlp_leg(n: int) -> dict:
    """The closure network on the host cores: torch FP32 (its CPU kernels, all its threads), samples/s of
    the forward pass and of forward + backward of a mean-squared loss."""
    import torch
    from oracle import cpu_twin

    torch.set_num_threads(cpu_twin.threads())        # a one-thread leg before may have left the pool at 1
    torch.manual_seed(0)
    net = torch.nn.Sequential(torch.nn.Linear(12, 64), torch.nn.GELU(), torch.nn.Linear(64, 64), torch.nn.GELU(),
                              torch.nn.Linear(64, 6))
    X = torch.randn(n, 12)
    Y = torch.randn(n, 6)

    def fwd():
        with torch.no_grad():
            net(X)

    def grad():
        net.zero_grad(set_to_none=True)
        torch.mean((net(X) - Y) ** 2).backward()

    out = {"samples": n, "threads": torch.get_num_threads(), "dtype": "f32"}
    for name, fn in (("forward", fwd), ("gradient", grad)):
        fn()
        best = float("inf")
        for _ in range(3):
            t0 = time.perf_counter()
            fn()
            best = min(best, time.perf_counter() - t0)
        out[f"{name}_seconds"] = best
        out[f"{name}_samples_per_s"] = n / best
    return out


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--legs", nargs="+", default=["vortex", "tgv", "mixing"],
                    choices=["vortex", "tgv", "mixing", "closure"])
    ap.add_argument("--json", type=str, default=None)
    args = ap.parse_args(argv)
    out = run(args.legs)
    line = json.dumps(out)
    print(line)
    if args.json:
        with open(args.json, "w") as fh:
            fh.write(line + "\n")


if __name__ == "__main__":
    main()
