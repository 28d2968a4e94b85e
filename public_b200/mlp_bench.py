"""Time the closure MLP's tensor-core kernels against their rooflines.

    python -m public_b200.mlp_bench [--n 16777216] [--train-n 2097152] [--batch 4096] [--steps 200]

Forward: n samples (12 float features in, 6 float stresses out; 72 bytes of HBM traffic and 10,496
algorithmic FLOPs per sample: 2 (12*64 + 64*64 + 64*6)), timed with CUDA events on the MLP's stream
after warm-up.  Gradient: the exact loss gradient over train-n samples (forward + backward,
3 x the forward FLOPs).  Training: Adam steps of `batch` samples.  Reports achieved GB/s and TFLOP/s
with the measured peaks (`MEASURED_PEAKS.json` when present).
"""
from __future__ import annotations

import argparse
import json
import os

import numpy as np

FLOP_FWD = 2 * (12 * 64 + 64 * 64 + 64 * 6)
BYTES_FWD = 4 * (12 + 6)


def run(args) -> dict:
    import torch

    from .closure import ClosureMLP

    dev = torch.device("cuda", 0)
    g = torch.Generator(device=dev)
    g.manual_seed(1)
    X = torch.randn((args.n, 12), generator=g, device=dev, dtype=torch.float32)
    Y = torch.empty((args.n, 6), device=dev, dtype=torch.float32)
    Xt = X[: args.train_n].contiguous()
    Yt = torch.randn((args.train_n, 6), generator=g, device=dev, dtype=torch.float32)
    peaks = {}
    path = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as fh:
            peaks = json.load(fh)
    hbm = float(peaks.get("hbm_gbs", 6650.0))
    tc = float(peaks.get("bf16_tflops", 1590.0))
    out = {"n": args.n, "train_n": args.train_n, "peaks": {"hbm_gbs": hbm, "bf16_tflops": tc,
                                                           "source": "measured" if peaks else "fallback"}}
    with ClosureMLP(0, seed=3) as mlp:
        mlp.set_scaling(np.zeros(12), np.ones(12), np.ones(6))
        torch.cuda.synchronize()
        for _ in range(3):
            mlp.forward(X, out=Y)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        reps = 10
        e0.record()
        for _ in range(reps):
            mlp.forward(X, out=Y)
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / reps
        out["forward"] = {"ms": ms, "GB/s": BYTES_FWD * args.n / (ms * 1e-3) / 1e9,
                          "TFLOP/s": FLOP_FWD * args.n / (ms * 1e-3) / 1e12}
        out["forward"]["hbm_frac"] = out["forward"]["GB/s"] / hbm
        out["forward"]["tensor_frac"] = out["forward"]["TFLOP/s"] / tc
        mlp.grad(Xt, Yt)
        torch.cuda.synchronize()
        e0.record()
        for _ in range(3):
            mlp.grad(Xt, Yt)
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / 3
        out["gradient"] = {"ms": ms, "TFLOP/s": 3 * FLOP_FWD * args.train_n / (ms * 1e-3) / 1e12}
        out["gradient"]["tensor_frac"] = out["gradient"]["TFLOP/s"] / tc
        mlp.train(Xt, Yt, batch=args.batch, steps=10, lr=1e-4, seed=1)
        torch.cuda.synchronize()
        e0.record()
        mlp.train(Xt, Yt, batch=args.batch, steps=args.steps, lr=1e-4, seed=2)
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / args.steps
        out["train_step"] = {"ms": ms, "batch": args.batch,
                             "TFLOP/s": 3 * FLOP_FWD * args.batch / (ms * 1e-3) / 1e12}
    return out


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--n", type=int, default=16777216)
    ap.add_argument("--train-n", type=int, default=2097152)
    ap.add_argument("--batch", type=int, default=4096)
    ap.add_argument("--steps", type=int, default=200)
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
