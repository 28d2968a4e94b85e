"""bench.py's reference arm on the host cores (no GPU): one JSON line with the contract's keys, and
only rank 0 reports under a multi-rank launch."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def run_bench(extra_env, *args):
    env = dict(os.environ, **extra_env)
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), *args], cwd=ROOT, env=env,
                       capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    return [ln for ln in r.stdout.splitlines() if ln.strip()]


def test_reference_arm_prints_one_contract_line():
    lines = run_bench({}, "--impl", "reference", "--steps", "1", "--warmup", "0", "--ref-n", "24")
    out = json.loads(lines[-1])
    for key in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
                "scaling", "dtype", "config", "cpu_baseline", "e2e"):
        assert key in out, key
    assert out["impl"] == "reference" and out["value"] > 0 and out["higher_is_better"] is True
    assert out["cpu_baseline"]["kind"] in ("port", "reference") and out["cpu_baseline"]["cores"] >= 1
    assert out["e2e"]["value"] == out["value"] and out["e2e"]["h2d_bytes_per_step"] == 0


def test_reference_arm_other_ranks_are_silent():
    lines = run_bench({"RANK": "1", "WORLD_SIZE": "2", "LOCAL_RANK": "1"},
                      "--impl", "reference", "--gpus", "2", "--steps", "1", "--warmup", "0", "--ref-n", "24")
    assert lines == []


def test_gpus_flag_launches_the_ranks_itself():
    """`bench.py --gpus 2` without a launcher starts two ranks through torch.distributed.run; the
    reference arm's rank 0 alone prints, so the run yields exactly one JSON line with n_gpus 2."""
    env = {k: v for k, v in os.environ.items() if k not in ("RANK", "WORLD_SIZE", "LOCAL_RANK")}
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2",
                        "--steps", "1", "--warmup", "0", "--n", "16"], cwd=ROOT, env=env, capture_output=True,
                       text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.strip()]
    assert len(lines) == 1, lines
    out = json.loads(lines[0])
    assert out["impl"] == "reference" and out["n_gpus"] == 2 and out["config"]["same_config"] is True
    assert abs(out["ms_per_step"] / 1e3 - 16 ** 3 / out["value"]) < 1e-9 * out["ms_per_step"]
