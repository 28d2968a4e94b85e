"""The measurement scripts behind the profile summaries run end to end on small sizes: run_case
(direct and adjoint timing, kernel-family profile), tgv_study (FP64 against FP32 stencils with
kinetic-energy and enstrophy histories), enstrophy_study (enstrophy gradient against central
differences) and mlp_bench (closure MLP kernels)."""
import argparse

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_run_case_times_and_profiles():
    from public_b200 import run_case
    base = dict(case="mixing_layer", n=[32, 48, 16], steps=3, warmup=1, adjoint=True, no_graphs=False, json=None)
    out = run_case.run(argparse.Namespace(**base, profile=False))
    assert out["rhs_path"] == "generic" and out["direct_ms_per_step"] > 0 and out["adjoint_ms_per_step"] > 0
    out = run_case.run(argparse.Namespace(**dict(base, adjoint=False), profile=True))
    assert abs(sum(v["share"] for v in out["kernels"].values()) - 1.0) < 1e-3
    out = run_case.run(argparse.Namespace(**dict(base, case="taylor_green", n=[24], adjoint=False), profile=False))
    assert out["rhs_path"] == "fused"


def test_tgv_study_small():
    from public_b200 import tgv_study
    out = tgv_study.run(argparse.Namespace(n=24, steps=20, every=10))
    assert len(out["fp64"]["history"]["step"]) == 3
    assert max(out["fp32_vs_fp64_rel_l2"]) < 1e-5
    assert out["kinetic_energy_max_rel_diff"] < 1e-6 and out["enstrophy_max_rel_diff"] < 1e-5


def test_enstrophy_study_small():
    from public_b200 import enstrophy_study
    base = dict(n=24, steps=6, nsnap=2, ndir=1, eps=1e-4, precision="fp64")
    out = enstrophy_study.run(argparse.Namespace(**base, host_snapshots=False))
    assert out["J"] == pytest.approx(out["J_objective_value"], rel=1e-12)
    assert out["directions"][0]["rel_err"] < 1e-2
    host = enstrophy_study.run(argparse.Namespace(**base, host_snapshots=True))
    assert host["J"] == out["J"] and host["directions"][0]["adjoint"] == out["directions"][0]["adjoint"]


def test_mlp_bench_small():
    from public_b200 import mlp_bench
    out = mlp_bench.run(argparse.Namespace(n=131072, train_n=16384, batch=1024, steps=5))
    for key in ("forward", "gradient", "train_step"):
        assert np.isfinite(out[key]["ms"]) and out[key]["ms"] > 0


def test_gradient_study_split_over_two_runs(tmp_path):
    """The mixing-layer gradient study split as a long horizon would be: difference quotients first
    (no adjoint), then both adjoints against the stored quotients; the discrete adjoint matches them."""
    import json

    from public_b200 import gradient_study
    base = dict(n=[16, 14, 12], steps=6, nsnap=3, ndir=3, y_plane=25.0, eps=[1e-7], fd_dirs=2, fd_start=0)
    first = gradient_study.run(argparse.Namespace(**base, fd_from=None, modes=[], json=None))
    assert "continuous" not in first and len(first["fd"]["1e-07"]) == 2
    path = tmp_path / "fd.json"
    path.write_text(json.dumps(first) + "\n")
    second = gradient_study.run(argparse.Namespace(**base, fd_from=str(path), modes=[0, 1], json=None))
    assert second["fd"] == first["fd"]
    assert len(second["discrete"]["directional_derivatives"]) == 3
    assert second["discrete"]["fd_rel_err_eps1e-07"]["max"] < 1e-4
