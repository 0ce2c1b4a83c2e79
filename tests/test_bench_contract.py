"""The benchmark's reference arm (CPU oracle) prints the one-line JSON contract.

The GPU arm needs a B200; its line is checked by running bench.py there.  The
reference arm runs here: one particle of each ensemble size through the CPU
oracle, on all host cores.
"""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_reference_arm_json_line():
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                          "--warmup", "3"], cwd=ROOT, capture_output=True, text=True, timeout=600, check=True)
    line = json.loads(out.stdout.strip().splitlines()[-1])
    for key in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
                "scaling", "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert key in line, key
    assert line["impl"] == "reference"
    assert line["unit"] == "pt-steps/s" and line["value"] > 0
    assert line["steps"] == 1 and line["warmup"] == 3 and line["n_gpus"] == 1
    assert line["cpu_baseline"]["kind"] == "port" and line["cpu_baseline"]["cores"] >= 1
    assert line["cpu_baseline"]["value"] == line["value"]
    assert line["e2e"]["value"] == line["value"]
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["e2e"]["d2h_bytes_per_step"] == 0
    # the GPU arm's own config (same workload, same point count), the sample named in cpu_baseline
    sys.path.insert(0, ROOT)
    import bench
    ns = bench.ensemble()[0]
    assert line["config"] == bench.ensemble_config(bench.COUNT, bench.SIZES, sum(n * n for n in ns), 1)
    assert "one of each size" in line["cpu_baseline"]["sample"]


def test_reference_arm_other_ranks_exit_quietly():
    """Under torchrun with N > 1 only rank 0 times the oracle and prints the line."""
    env = dict(os.environ, WORLD_SIZE="2", RANK="1", LOCAL_RANK="1")
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                          "--warmup", "3"], cwd=ROOT, capture_output=True, text=True, timeout=300, env=env)
    assert out.returncode == 0, out.stderr
    assert out.stdout.strip() == ""
