"""Learned subgrid closure study (the coarse-grid closure workload): decaying isotropic turbulence.

1. Fine DNS on n^3 (8th-order differences, o10 filter every step, RK4) from
   ``cases.isotropic_turbulence``; every ``every`` steps the solver box-filters the state by ``factor``
   (``cruna_box_filter_dev``: filtered state and exact Favre subgrid stresses) and computes the
   closure features on the coarse grid (``cruna_closure_features_dev``); a seeded random subset of the
   coarse points of each snapshot becomes training pairs, and the filtered kinetic energy is recorded.
2. The MLP (12 -> 64 -> 64 -> 6, BF16 tensor-core kernels) is trained with Adam on those pairs.
3. Two coarse runs start from the filtered initial state with dt_c = (every / 2) dt_f: the plain
   filter-stabilised coarse solve and the same solve with the closure attached (``cruna_set_closure``).
   Their kinetic energy is compared with the filtered DNS at every snapshot time, and the GPU time of
   each run (CUDA events, excluding set-up) with the fine DNS's.

    python -m public_b200.closure_study [--n 256] [--factor 4] [--steps 3000] [--every 10]
        [--samples 2000000] [--train-steps 3000] [--batch 4096] [--lr 1e-3] [--normalised] [--json out.json]
        [--calibrate 0.8 1.0 1.2] [--separate-closure]

--normalised trains and runs the scale-free closure (``cruna_set_closure_normalisation``): features
grad u / |grad u| and |grad u| delta, targets tau / (rho (|grad u| delta)^2).

4. For each --gradient-steps H (a multiple of --every): the gradient of the kinetic energy after H
   fine steps with respect to the initial fine state (continuous adjoint, binomial checkpointing),
   summed over each filter block -- the gradient with respect to the coarse initial state of a
   perturbation constant over the block -- against the coarse gradients over the same time
   (H / every * 2 coarse steps) of the plain and the closure-augmented coarse solve: cosine
   similarity over the momentum components (the initial velocity) and over the whole state.

--case tgv runs the same pipeline on the Taylor-Green vortex (--mach, --reynolds; the 768^3 -> 192^3
configuration with --n 768 --precision fp32 for the fine DNS).

5. --calibrate a1 a2 ...: a posteriori, the multiplier of the network's stresses among a1, a2, ... whose
   coarse run tracks the filtered DNS kinetic energy best over the first half of the snapshots; the
   whole horizon then scores it.  The closure runs inside the flux pass unless --separate-closure.

Prints one JSON object.  Data are synthetic (seeded spectrum, no dataset).
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np


def kinetic_energy(q, dV: float) -> float:
    """sum dV |rho u|^2 / (2 rho) of a Fortran-flattened device state (torch float64)."""
    N = q.numel() // 5
    rho, m = q[:N], q[N:4 * N].view(3, N)
    return float(((m * m).sum(0) / (2.0 * rho)).sum().item()) * dV


def run(args) -> dict:
    import torch

    from . import cases
    from .closure import ClosureMLP
    from .cruna import Cruna, Settings

    dev = torch.device("cuda", 0)
    if getattr(args, "case", "isotropic") == "tgv":
        s, q0 = cases.taylor_green(n=args.n, mach=args.mach, reynolds=args.reynolds, seed=args.seed)
    else:
        s, q0 = cases.isotropic_turbulence(n=args.n, seed=args.seed, mach_t=args.mach_t, re_lambda=args.re_lambda)
    nf, r = args.n, args.factor
    nc = nf // r
    dt_f = s["dt"]
    if args.every % 2:
        raise ValueError("--every must be even (coarse step = every/2 fine steps)")
    dt_c = (args.every // 2) * dt_f
    sc = dict(s, n=(nc, nc, nc), dt=dt_c)
    L = s["x1"][0] - s["x0"][0]
    dVf, dVc = (L / nf) ** 3, (L / nc) ** 3
    delta = r * L / nf
    Nc = nc ** 3
    snaps = args.steps // args.every
    per_snap = max(1, min(Nc, args.samples // max(snaps, 1)))
    rng = torch.Generator(device=dev)
    rng.manual_seed(args.seed + 17)

    q = torch.from_numpy(np.ascontiguousarray(q0.ravel(order="F"))).to(dev)
    qc = torch.empty(5 * Nc, dtype=torch.float64, device=dev)
    tau = torch.empty((Nc, 6), dtype=torch.float32, device=dev)
    feat = torch.empty((Nc, 12), dtype=torch.float32, device=dev)
    Xs, Ys = [], []
    ke_dns, t_dns = [], []
    st_fine = Settings.from_dict(s)
    st_fine.precision = getattr(args, "precision", "fp64")
    with Cruna(st_fine) as fine, Cruna(Settings.from_dict(sc)) as coarse:
        coarse.set_closure_normalisation(args.normalised)
        coarse.set_closure_fused(bool(args.fused_closure))
        # initial filtered state (start of both coarse runs)
        fine.box_filter_dev(r, q.data_ptr(), qc.data_ptr(), tau.data_ptr())
        fine.sync()
        qc0 = qc.clone()
        ke_dns.append(kinetic_energy(qc, dVc))
        t_dns.append(0.0)
        dns_ms = 0.0
        stream = torch.cuda.ExternalStream(fine.stream_handle(), device=dev)
        for k in range(snaps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            fine.run_direct_dev(q.data_ptr(), k * args.every, args.every)
            e1.record(stream)
            fine.box_filter_dev(r, q.data_ptr(), qc.data_ptr(), tau.data_ptr())
            fine.sync()
            dns_ms += e0.elapsed_time(e1)
            coarse.closure_features_dev(qc.data_ptr(), delta, feat.data_ptr())
            coarse.sync()
            pick = torch.randperm(Nc, generator=rng, device=dev)[:per_snap]
            Xs.append(feat[pick].clone())
            Ys.append(tau[pick].clone())
            ke_dns.append(kinetic_energy(qc, dVc))
            t_dns.append((k + 1) * args.every * dt_f)
        X = torch.cat(Xs).contiguous()
        Y = torch.cat(Ys).contiguous()
        # normalised closure: targets tau / (rho (g delta)^2), rho and g delta being features 9 and 11
        scale = (X[:, 9] * X[:, 11] * X[:, 11]).unsqueeze(1) if args.normalised else torch.ones_like(Y[:, :1])
        scale = torch.where(scale > 0, scale, torch.ones_like(scale))
        Yt = (Y / scale).contiguous()
        in_mean = X.mean(0).cpu().numpy()
        in_scale = X.std(0).cpu().numpy()
        in_scale[in_scale <= 1e-12] = 1.0     # constant features (the filter width)
        out_scale = Yt.std(0).cpu().numpy()
        out_scale[out_scale <= 1e-30] = 1.0
        nb = (X.shape[0] // args.batch) * args.batch
        X, Y, Yt, scale = X[:nb].contiguous(), Y[:nb].contiguous(), Yt[:nb].contiguous(), scale[:nb]

        mlp = ClosureMLP(0, seed=args.seed)
        mlp.set_scaling(in_mean, in_scale, out_scale)
        t0 = time.time()
        hist = mlp.train(X, Yt, batch=args.batch, steps=args.train_steps, lr=args.lr, seed=args.seed)
        train_s = time.time() - t0
        # explained variance of the stresses on the training pairs
        pred = mlp.forward(X) * scale
        ev = 1.0 - float(((pred - Y) ** 2).sum().item()) / float(((Y - Y.mean(0)) ** 2).sum().item())

        def coarse_run(with_closure: bool):
            coarse.set_closure(mlp if with_closure else None, delta)
            qq = qc0.clone()
            ke, ms = [kinetic_energy(qq, dVc)], 0.0
            cstream = torch.cuda.ExternalStream(coarse.stream_handle(), device=dev)
            for k in range(snaps):
                a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                a.record(cstream)
                coarse.run_direct_dev(qq.data_ptr(), k * 2, 2)
                b.record(cstream)
                coarse.sync()
                ms += a.elapsed_time(b)
                ke.append(kinetic_energy(qq, dVc))
            coarse.set_closure(None)
            return np.array(ke), ms

        ke_plain, ms_plain = coarse_run(False)
        ke_model, ms_model = coarse_run(True)
        calib = None
        if args.calibrate:
            # a posteriori: one multiplier of the network's stresses, fitted by coarse runs to the filtered
            # DNS kinetic energy over the first half of the snapshots only; the whole horizon then scores it
            half = max(1, snaps // 2)

            def window_err(ke):
                return float(np.max(np.abs(ke[:half + 1] - np.array(ke_dns[:half + 1])) / np.array(ke_dns[:half + 1])))

            trials = []
            for alpha in args.calibrate:
                mlp.set_scaling(in_mean, in_scale, out_scale * alpha)
                ke_a, _ = coarse_run(True)
                trials.append((window_err(ke_a), alpha, ke_a))
            best = min(trials, key=lambda t: t[0])
            mlp.set_scaling(in_mean, in_scale, out_scale * best[1])
            ke_cal, ms_cal = coarse_run(True)
            calib = {"alphas": [t[1] for t in trials], "window_errors": [t[0] for t in trials], "alpha": best[1],
                     "window_snapshots": half, "ke_closure": ke_cal.tolist(), "gpu_ms": ms_cal}
            mlp.set_scaling(in_mean, in_scale, out_scale)
        grad = [gradient_comparison(args, H, fine, coarse, mlp, q0, qc0, delta) for H in args.gradient_steps]
        mlp.close()
    ke_dns = np.array(ke_dns)

    def err(ke):
        return float(np.max(np.abs(ke - ke_dns) / ke_dns))

    def err0(ke):      # the same difference measured on the initial energy (error of the decay curve)
        return float(np.max(np.abs(ke - ke_dns)) / ke_dns[0])

    if calib is not None:
        calib["ke_max_rel_err"] = err(np.array(calib["ke_closure"]))
        calib["ke_max_err_of_initial"] = err0(np.array(calib["ke_closure"]))

    if getattr(args, "case", "isotropic") == "tgv":
        workload = (f"Taylor-Green {nf}^3 -> {nc}^3 (box filter x{r}), Mach {args.mach}, Re {args.reynolds}, "
                    f"{args.steps} fine steps, fine DNS in {getattr(args, 'precision', 'fp64')}")
    else:
        workload = (f"isotropic turbulence {nf}^3 -> {nc}^3 (box filter x{r}), Mach_t {args.mach_t}, "
                    f"Re_lambda {args.re_lambda}, {args.steps} fine steps")
    return {
        "workload": workload,
        "samples": int(X.shape[0]), "train_steps": args.train_steps, "batch": args.batch,
        "normalised": bool(args.normalised),
        "train_loss_first": float(hist[0]) if len(hist) else None,
        "train_loss_last": float(np.mean(hist[-20:])) if len(hist) else None,
        "explained_variance": ev, "train_seconds": train_s,
        "ke_decay_dns": float(ke_dns[-1] / ke_dns[0]),
        "ke_max_rel_err_plain": err(ke_plain), "ke_max_rel_err_closure": err(ke_model),
        "ke_max_err_of_initial_plain": err0(ke_plain), "ke_max_err_of_initial_closure": err0(ke_model),
        "calibration": calib, "closure_in_flux_pass": bool(args.fused_closure),
        "ke_final_rel_err_plain": float(abs(ke_plain[-1] - ke_dns[-1]) / ke_dns[-1]),
        "ke_final_rel_err_closure": float(abs(ke_model[-1] - ke_dns[-1]) / ke_dns[-1]),
        "gpu_ms_dns": dns_ms, "gpu_ms_coarse_plain": ms_plain, "gpu_ms_coarse_closure": ms_model,
        "speedup_closure_vs_dns": dns_ms / ms_model if ms_model > 0 else None,
        "times": [float(t) for t in t_dns], "ke_dns": ke_dns.tolist(), "ke_plain": ke_plain.tolist(),
        "ke_closure": ke_model.tolist(), "gradient": grad,
    }


def block_sum(g, n: int, r: int):
    """Sums of a Fortran-flattened n^3 state (torch, 5 fields) over r^3 blocks, as the Fortran-flattened
    (n/r)^3 state: flat index i + n (j + n k) + v n^3, so the view is (v, k, j, i)."""
    nc = n // r
    return g.view(5, nc, r, nc, r, nc, r).sum((2, 4, 6)).reshape(-1)


def gradient_comparison(args, H: int, fine, coarse, mlp, q0, qc0, delta) -> dict:
    """Cosine similarity of the block-summed fine gradient of the kinetic energy after H fine steps with
    the plain and closure-augmented coarse gradients (momentum components and whole state)."""
    import torch

    if H % args.every:
        raise ValueError("--gradient-steps must be a multiple of --every")
    Hc = H // args.every * 2
    nf, r = args.n, args.factor
    nc = nf // r
    dev = qc0.device
    qf = torch.from_numpy(np.ascontiguousarray(q0.ravel(order="F"))).to(dev)
    gf = torch.empty_like(qf)
    torch.cuda.synchronize()
    Jf, _ = fine.gradient_dev(qf.data_ptr(), H, args.gradient_snapshots, fine.objective("kinetic_energy"),
                              None, gf.data_ptr())
    fine.sync()
    g_block = block_sum(gf, nf, r)
    del qf, gf
    out = {"fine_steps": H, "coarse_steps": Hc, "J_fine": Jf}
    Nc = nc ** 3
    for name, model in (("plain", None), ("closure", mlp)):
        coarse.set_closure(model, delta)
        qq = qc0.clone()
        gc = torch.empty_like(qq)
        torch.cuda.synchronize()
        Jc, _ = coarse.gradient_dev(qq.data_ptr(), Hc, args.gradient_snapshots, coarse.objective("kinetic_energy"),
                                    None, gc.data_ptr())
        coarse.sync()
        coarse.set_closure(None)

        def cos(a, b):
            return float(torch.dot(a, b).item() / (torch.linalg.vector_norm(a) * torch.linalg.vector_norm(b)).item())

        out[name] = {"J": Jc, "cos_momentum": cos(g_block[Nc:4 * Nc], gc[Nc:4 * Nc]), "cos_state": cos(g_block, gc)}
    return out


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--n", type=int, default=256)
    ap.add_argument("--factor", type=int, default=4)
    ap.add_argument("--steps", type=int, default=3000)
    ap.add_argument("--every", type=int, default=10)
    ap.add_argument("--samples", type=int, default=2_000_000)
    ap.add_argument("--train-steps", type=int, default=3000)
    ap.add_argument("--batch", type=int, default=4096)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--seed", type=int, default=3)
    ap.add_argument("--mach-t", type=float, default=0.3)
    ap.add_argument("--re-lambda", type=float, default=100.0)
    ap.add_argument("--normalised", action="store_true",
                    help="scale-free closure: features grad u / |grad u|, |grad u| delta; targets tau / (rho (|grad u| delta)^2)")
    ap.add_argument("--gradient-steps", type=int, nargs="*", default=[],
                    help="horizons (fine steps) of the fine / coarse gradient comparison")
    ap.add_argument("--gradient-snapshots", type=int, default=64)
    ap.add_argument("--case", default="isotropic", choices=["isotropic", "tgv"],
                    help="decaying isotropic turbulence (default) or the Taylor-Green vortex")
    ap.add_argument("--mach", type=float, default=0.2, help="Taylor-Green Mach number")
    ap.add_argument("--reynolds", type=float, default=3200.0, help="Taylor-Green Reynolds number")
    ap.add_argument("--precision", default="fp64", choices=["fp64", "fp32"], help="precision of the fine DNS")
    ap.add_argument("--calibrate", type=float, nargs="*", default=[],
                    help="multipliers of the network's stresses tried a posteriori (first half of the horizon)")
    ap.add_argument("--separate-closure", dest="fused_closure", action="store_false",
                    help="closure as separate launches instead of inside the flux pass")
    ap.add_argument("--json", type=str, default=None)
    args = ap.parse_args(argv)
    out = run(args)
    line = json.dumps(out)
    print(line)
    if args.json:
        with open(args.json, "w") as f:
            f.write(line + "\n")


if __name__ == "__main__":
    main()
