"""bench.py's reference arm on the CPU: one JSON line with the contract's keys,
on a small catchment (the GPU arm is exercised on a B200)."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_reference_arm_prints_one_contract_line():
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
                          "--cells", "96", "--steps", "2", "--warmup", "3"],
                         capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [ln for ln in out.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step",
              "higher_is_better", "scaling", "vs_baseline", "dtype", "data", "config",
              "cpu_baseline", "e2e"):
        assert k in d, k
    assert d["impl"] == "reference" and d["value"] > 0
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["e2e"]["value"] == d["value"]
    assert d["cpu_baseline"]["kind"] in ("reference", "port") and d["cpu_baseline"]["cores"] >= 1


def test_reference_arm_other_ranks_exit_quietly():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2")
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
                          "--cells", "96", "--steps", "1", "--warmup", "3"],
                         capture_output=True, text=True, timeout=300, cwd=ROOT, env=env)
    assert out.returncode == 0
    assert not [ln for ln in out.stdout.splitlines() if ln.startswith("{")]


def test_launch_count_claim_follows_the_launch_form():
    """The GPU arm's `gpu_launches` claim: one launch per step for 64-wide tiles
    at the default register cap (pairs_mixed_kernel), the two builds for a
    3-CTA cap and for 32-wide tiles."""
    import argparse

    sys.path.insert(0, ROOT)
    import bench

    def args(tile, minb):
        return argparse.Namespace(tile=list(tile), minb=minb)

    assert bench.one_launch_step(args((32, 64), 0)) and bench.one_launch_step(args((32, 64), 4))
    assert not bench.one_launch_step(args((32, 64), 3))
    assert not bench.one_launch_step(args((32, 32), 0))
    assert bench.step_kernel_name(args((32, 64), 0)).startswith("pairs_mixed_kernel")
    assert bench.step_kernel_name(args((32, 64), 3)).startswith("pairs_step_kernel")
    assert bench.step_kernel_name(args((32, 32), 5)).startswith("rows_step_kernel")
