"""Benchmark of the CRUNA direct + adjoint time step on B200.

Workload (the Taylor-Green configuration of the headline metric): 3-D Taylor-Green vortex, Mach 0.1,
Re 1600, periodic [0, 2pi]^3 on 256^3 points, 8th-order explicit differences, 10th-order explicit
filter (strength 0.2) in all three directions every step, classical RK4 at CFL 0.5, FP64.
One "step" = one direct RK4 step (+ filters) followed by one adjoint RK4 step (+ filters) of the
continuous adjoint on the direct state it produced; the unit is grid point-steps per second, i.e.
points x (direct+adjoint step pairs) / s.  Inputs (q: 671 MB, qs: 671 MB) are larger than the 126 MB
L2, so no explicit flush is needed between iterations.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--n 256]

--impl reference times the C + OpenMP restatement of the reference's algorithm (oracle/cruna_cpu.c,
checked against the numpy oracle; the Fortran reference itself cannot be built on this image) on all
host cores on the same 256^3 configuration, one direct+adjoint step pair per timed step, the state
generated once before the warm-up.  --gpus N without a launcher re-executes the script through
torch.distributed.run with N ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import tempfile
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "point-steps/s direct+adjoint"
UNIT = "point-steps/s"

# algorithmic HBM bytes per grid point and launch of each kernel family (FP64 state): the compulsory
# reads and writes of one launch
ALG_BYTES_FP64 = {
    "pass_g": 40 + 15 * 8,          # read q, write 15 fields
    "pass_d": 9 * 8 + 6 * 8 + 140,  # read 9 stencil fields + 6 centre fields, RK stage I/O (average)
    "adj_pass": 40 + 40 + 140,      # read qs, read frozen q, RK stage I/O (average)
    "line_filter": 5 * 8 * 2,       # read + write 5 fields
    "filter_xy": 5 * 8 * 2,         # read + write 5 fields (x and y filters of each plane)
    "filter_z": 5 * 8 * 2,          # read + write 5 fields
}


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


# ------------------------------------------------------------------------------------------------
# CPU legs (oracle): bounded samples of the same physics
# ------------------------------------------------------------------------------------------------
class CpuTwin:
    """The C + OpenMP restatement of the oracle (oracle/cruna_cpu.c) on an n^3 Taylor-Green state of the
    benchmark's configuration, generated once; pair() advances one direct+adjoint step pair in place."""

    def __init__(self, n: int, threads: int = 0):
        import numpy as np

        from oracle import cpu_twin
        from public_b200 import cases

        self.twin = cpu_twin
        self.n, self.threads = n, threads
        s, q0 = cases.taylor_green(n=n, seed=0)
        s["ai_freq"] = (1, 1, 1)
        self.s = s
        self.q = np.array(q0, order="F", copy=True)
        self.qs = np.asfortranarray(1e-3 * np.ones_like(q0))
        self.cores = threads if threads > 0 else cpu_twin.threads()

    def pairs(self, k: int) -> float:
        """Runs k step pairs; returns the wall time in seconds."""
        t0 = time.perf_counter()
        self.twin.run(self.s, self.q, self.qs, k, self.threads)
        return time.perf_counter() - t0


def cpu_sample(n: int, pairs: int, threads: int = 0):
    """Times `pairs` direct+adjoint step pairs of the CPU twin on an n^3 Taylor-Green state after one
    untimed warm-up pair (page faults, thread pool); returns (point-steps/s, seconds, threads used)."""
    tw = CpuTwin(n, threads)
    tw.pairs(1)
    dt = tw.pairs(pairs)
    return n ** 3 * pairs / dt, dt, tw.cores


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    n = args.ref_n or args.n
    tw = CpuTwin(n)
    for _ in range(args.warmup):                         # untimed warm-up pairs
        tw.pairs(1)
    steps = max(1, args.steps)
    times = [tw.pairs(1) for _ in range(steps)]        # one step pair of the workload per timed step
    total = sum(times)
    value = n ** 3 * steps / total
    sample = (f"{n}^3 Taylor-Green (the benchmark's configuration), one direct+adjoint step pair per timed "
              f"step, C+OpenMP restatement on all host threads")
    out = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": steps, "warmup": args.warmup, "ms_per_step": 1e3 * total / steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded Taylor-Green state, 1e-4 density noise)",
        "config": {"workload": f"taylor-green {n}^3 Mach 0.1 Re 1600: o8 FD, o10 explicit filter every step, "
                               f"RK4 direct step + continuous-adjoint RK4 step",
                   "points": n ** 3, "sample": sample, "same_config": n == args.n},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": tw.cores, "kind": "port", "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "note": "C + OpenMP restatement of the reference algorithm in the reference's call structure "
                "(the Fortran/MPI/HDF5 reference cannot be built on this image)",
    }
    print(json.dumps(out))
    return 0


# ------------------------------------------------------------------------------------------------
class ClockSampler:
    """nvidia-smi clocks / throttle reasons during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.dev = device_index
        self.proc = None
        # raw samples (the JSON line carries their summary); CRUNA_CLOCKS_DIR keeps them elsewhere
        self.path = os.path.join(os.environ.get("CRUNA_CLOCKS_DIR", tempfile.gettempdir()),
                                 f"clocks_bench_{os.getpid()}.csv")

    def start(self):
        try:
            os.makedirs(os.path.dirname(self.path), exist_ok=True)
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.dev}", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "50"], stdout=self.f, stderr=subprocess.DEVNULL)
            # nvidia-smi needs a moment before its first sample; start timing once it is reporting
            t0 = time.time()
            while time.time() - t0 < 3.0 and os.path.getsize(self.path) == 0:
                time.sleep(0.02)
        except Exception:
            self.proc = None

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.f.close()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        with open(self.path) as f:
            for line in f:
                parts = [p.strip() for p in line.split(",")]
                if len(parts) < 9:
                    continue
                try:
                    sm.append(float(parts[1]))
                    smax = float(parts[2])
                except ValueError:
                    continue
                for nm, v in zip(names, parts[5:9]):
                    if v.lower().startswith("active"):
                        reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


def run_ours(args):
    import numpy as np
    import torch

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    torch.cuda.set_device(local)

    # CPU baseline first (spawned processes, before heavy GPU work), rank 0 at N=1 only
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        n_cpu = args.ref_n or args.n
        v, wall, cores = cpu_sample(n_cpu, args.cpu_pairs)
        cpu = {"value": v, "unit": UNIT, "cores": cores, "kind": "port",
               "sample": f"{n_cpu}^3 Taylor-Green, {args.cpu_pairs} direct+adjoint step pairs after one warm-up "
                         f"pair, C+OpenMP restatement of the oracle on all host threads",
               "seconds": round(wall, 2)}

    from public_b200 import cases
    from public_b200.cruna import Cruna, Settings

    s, q0 = cases.taylor_green(n=args.n, seed=rank)
    s["ai_freq"] = (1, 1, 1)
    slabs = None
    if world > 1 or args.slabs:
        # z slabs: the global grid is n x n x (n * world) (the Taylor-Green field repeated along z, each
        # slab with its own density noise); each rank holds n^3 interior points plus H = 2R = 8 halo
        # planes per side, refreshed through NCCL point-to-point before every z-reading pass (--slabs on
        # one GPU: the same path, the single slab exchanging with itself)
        from public_b200.slabs import ZSlabs
        L = s["x1"][2] - s["x0"][2]
        slabs = ZSlabs((args.n, args.n, args.n * world), halo=8, rank=rank, world=world)
        s = slabs.local_settings(dict(s, n=(args.n, args.n, args.n * world), x1=(s["x1"][0], s["x1"][1], L * world)))
        q0 = ZSlabs((args.n, args.n, args.n), halo=8).local_state(q0)
    st = Settings.from_dict(s)
    st.device = local
    st.precision = args.precision
    ctx = Cruna(st)
    if args.tma:
        ctx.tma_passes(True)
    if slabs is not None:
        slabs.attach(ctx)
    N = args.n ** 3                                   # interior points of this rank
    NL = int(np.prod(s["n"]))                         # points held (with halo planes)
    dev = torch.device("cuda", local)
    q = torch.from_numpy(np.ascontiguousarray(q0.ravel(order="F"))).to(dev)
    qs = torch.full_like(q, 1e-3)
    qp, qsp = q.data_ptr(), qs.data_ptr()
    stream = torch.cuda.ExternalStream(ctx.stream_handle(), device=dev)
    torch.cuda.synchronize()

    def step(nt):
        ctx.run_direct_dev(qp, nt, 1)
        ctx.run_adjoint_dev(qsp, qp, None, nt + 1, 1)

    for w in range(args.warmup):
        step(w)
    ctx.sync()

    # ---- device-resident timing -----------------------------------------------------------------
    ev = [[torch.cuda.Event(enable_timing=True) for _ in range(3)] for _ in range(args.steps)]
    ctx.profile(True)
    launches0 = ctx.launches
    clocks = ClockSampler(local)
    clocks.start()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    for k in range(args.steps):
        nt = args.warmup + k
        ev[k][0].record(stream)
        ctx.run_direct_dev(qp, nt, 1)
        ev[k][1].record(stream)
        ctx.run_adjoint_dev(qsp, qp, None, nt + 1, 1)
        ev[k][2].record(stream)
    ctx.sync()
    torch.cuda.synchronize()
    clk = clocks.stop()
    launches = ctx.launches - launches0
    prof = ctx.profile_report()
    ctx.profile(False)
    t_dir = sum(e[0].elapsed_time(e[1]) for e in ev)
    t_adj = sum(e[1].elapsed_time(e[2]) for e in ev)
    t_tot = sum(e[0].elapsed_time(e[2]) for e in ev)
    if dist:
        t = torch.tensor([t_tot, t_dir, t_adj], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        t_tot, t_dir, t_adj = [float(x) for x in t.tolist()]
    ms = t_tot / args.steps
    value = world * N * args.steps / (t_tot / 1e3)

    # ---- end-to-end through the host-pointer C ABI (pinned host buffers) ------------------------
    bytes_state = 5 * NL * 8
    e2e_value, e2e_steps = None, 0
    if not args.no_e2e:
        hq = torch.empty(5 * NL, dtype=torch.float64, pin_memory=True)
        hqs = torch.empty(5 * NL, dtype=torch.float64, pin_memory=True)
        hq.copy_(q.cpu())
        hqs.copy_(qs.cpu())
        import ctypes as C
        lib = ctx.lib
        e2e_steps = max(1, min(args.steps, 3))
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for k in range(e2e_steps):
            nt = args.warmup + args.steps + k
            ctx._check(lib.cruna_run_direct(ctx.h, C.c_void_p(hq.data_ptr()), nt, 1, None))
            ctx._check(lib.cruna_run_adjoint(ctx.h, C.c_void_p(hqs.data_ptr()), C.c_void_p(hq.data_ptr()), None,
                                             nt + 1, 1))
        t_e2e = time.perf_counter() - t0
        if dist:
            t = torch.tensor([t_e2e], device=dev)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            t_e2e = float(t.item())
        e2e_value = world * N * e2e_steps / t_e2e

    # ---- roofline of the dominant kernel --------------------------------------------------------
    peak, peak_kind = load_peaks()
    dom = max(prof.items(), key=lambda kv: kv[1][1]) if prof else None
    roof = None
    if dom:
        name, (cnt, tot_ms) = dom
        per_pt = ALG_BYTES_FP64.get(name)
        if per_pt is not None and args.precision == "fp32" and name == "pass_g":
            per_pt = 40 + 15 * 4
        if per_pt is not None and args.precision == "fp32" and name == "pass_d":
            per_pt = 15 * 4 + 140
        avg_s = tot_ms / cnt / 1e3
        achieved = (per_pt * NL / avg_s / 1e9) if per_pt else None
        roof = {"bound": "hbm", "kernel": name, "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": (achieved / peak) if achieved else None, "peak_source": peak_kind,
                "traffic": traffic_from_profiles(name, args.n, args.precision),
                "alg_bytes_per_point": per_pt, "avg_launch_ms": avg_s * 1e3, "launches": cnt}
    kernels = {k: {"launches": v[0], "total_ms": round(v[1], 3), "share": round(v[1] / max(t_tot, 1e-9), 4)}
               for k, v in sorted(prof.items(), key=lambda kv: -kv[1][1])}
    B_alg = 760 + 920
    out = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64" if args.precision == "fp64" else "f32-stencil/f64-state",
        "data": "synthetic (seeded Taylor-Green state, 1e-4 density noise)",
        "config": {"workload": f"taylor-green {args.n}^3 Mach 0.1 Re 1600: o8 FD, o10 explicit filter every "
                               f"step, RK4 direct step + continuous-adjoint RK4 step",
                   "points": N, "parallelism": (f"z slabs x{world}: n x n x {args.n * world} global grid, "
                                                 f"8 halo planes per side, "
                                                 + ("NCCL point-to-point exchange" if world > 1
                                                    else "exchange of the single slab with itself"))
                   if slabs is not None else "single GPU",
                   "l2": f"inputs ({bytes_state / 1e6:.0f} MB per state) larger than L2; no flush",
                   "precision": args.precision, "rhs_path": ctx.rhs_path},
        "direct": {"value": N * args.steps / (t_dir / 1e3), "unit": UNIT, "ms_per_step": t_dir / args.steps},
        "adjoint": {"value": N * args.steps / (t_adj / 1e3), "unit": UNIT, "ms_per_step": t_adj / args.steps},
        "hbm_alg": {"bytes_per_point_step": B_alg, "achieved_gbs": value / world * B_alg / 1e9,
                    "frac": value / world * B_alg / 1e9 / peak},
        "roofline": roof,
        "kernels": kernels,
        "gpu_launches": int(launches),
        "clocks": clk,
        "e2e": ({"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": 3 * bytes_state,
                 "d2h_bytes_per_step": 2 * bytes_state, "steps": e2e_steps,
                 "api": "cruna_run_direct + cruna_run_adjoint on pinned host buffers"}
                if e2e_value is not None else None),
        "cpu_baseline": cpu,
    }
    ctx.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(out))
    return 0


def traffic_from_profiles(kernel: str, n: int, precision: str):
    """DRAM bytes per launch of `kernel` from a committed ncu summary, scaled to n^3 points."""
    path = os.path.join(ROOT, "profiles", f"{kernel}_tgv_{precision}.txt")
    try:
        with open(path) as f:
            for line in f:
                if line.startswith("dram_bytes_per_point:"):
                    return float(line.split(":")[1]) * n ** 3
    except OSError:
        pass
    return None


def relaunch(n: int) -> int:
    """--gpus N without a launcher: start N ranks of this script through torch.distributed.run (one
    process per GPU, rendezvous on 127.0.0.1) and return its status; rank 0 prints the JSON line."""
    import socket

    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", f"--nproc-per-node={n}",
           "--master-addr=127.0.0.1", f"--master-port={port}", os.path.abspath(__file__), "--", *sys.argv[1:]]
    return subprocess.call(cmd)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", type=int, default=256)
    ap.add_argument("--ref-n", type=int, default=0,
                    help="grid of the CPU legs (default: --n, the benchmark's own configuration)")
    ap.add_argument("--cpu-pairs", type=int, default=2, help="timed step pairs of the cpu_baseline leg")
    ap.add_argument("--precision", default="fp64", choices=["fp64", "fp32"])
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--slabs", action="store_true",
                    help="z-slab decomposition with halo exchange also on one GPU (the path --gpus N runs)")
    ap.add_argument("--tma", action="store_true",
                    help="FP64 adjoint pass fed by TMA instead of the per-thread-load kernel (the default)")
    ap.add_argument("--no-e2e", action="store_true",
                    help="skip the host-buffer run (grids whose staging would not fit beside the device working set)")
    args = ap.parse_args()
    if args.gpus > 1 and "WORLD_SIZE" not in os.environ:
        return relaunch(args.gpus)
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
