"""The bench's reference arm (bench.py --impl reference) on the CPU: it converges the warm-up
steps and the sampled timed steps with the oracle, prints one JSON line in the product line's
metric and unit, and never loads this package's CUDA library (its cases come from the oracle's
own mesh and noise generators).  Run in a fresh process on the small plain workload."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

SNIPPET = r"""
import argparse, json, sys
sys.argv = ["bench.py", "--impl", "reference", "--workload", "plain-51", "--steps", "3", "--warmup", "0",
            "--sample-steps", "1"]
import bench
bench.main()
pkg = sys.modules.get("solver_cfd_b200")
maps = open("/proc/self/maps").read()
print(json.dumps({"lib_object": pkg is not None and pkg._lib is not None, "so_mapped": "libacs_b200.so" in maps}))
"""


def test_reference_arm_runs_the_oracle_without_the_library(orc):
    out = subprocess.run([sys.executable, "-c", SNIPPET], cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [l for l in out.stdout.splitlines() if l.startswith("{")]
    line, probe = json.loads(lines[-2]), json.loads(lines[-1])
    assert line["impl"] == "reference"
    assert line["unit"] == "steps/s" and line["higher_is_better"] is True and line["value"] > 0
    assert line["metric"] == "converged physical steps/s at pseudo-time residual 1e-6"
    iters = line["config"]["pseudo_iterations_per_step"]
    assert list(iters) == ["0"] and len(iters["0"]) == 1 and iters["0"][0] > 1
    assert line["cpu_baseline"]["kind"] == "port" and line["e2e"]["h2d_bytes_per_step"] == 0
    assert probe == {"lib_object": False, "so_mapped": False}, probe
