"""AddressSanitizer + UndefinedBehaviorSanitizer over the host code: the product's mesh and noise
generators (solver-cfd_b200/csrc/mesh.cpp, part of the C ABI) and the CPU oracle, driven by
tests/sanitize/host_checks.cpp on small and odd geometries (reference domain down to imax = 6,
channels with odd sizes and zero, one or two porous blocks).  compute-sanitizer is not available
for the device code; the device kernels are covered by the bit-exact comparisons against the
oracle on the same kinds of geometry."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.skipif(shutil.which("g++") is None, reason="needs g++")
def test_host_code_under_asan_and_ubsan(tmp_path):
    exe = str(tmp_path / "host_checks")
    cmd = ["g++", "-std=c++17", "-O1", "-g", "-fno-omit-frame-pointer", "-fopenmp", "-ffp-contract=off",
           "-fsanitize=address,undefined", "-fno-sanitize-recover=all",
           os.path.join(ROOT, "tests", "sanitize", "host_checks.cpp"),
           os.path.join(ROOT, "oracle", "acs_oracle.cpp"),
           os.path.join(ROOT, "solver-cfd_b200", "csrc", "mesh.cpp"), "-o", exe]
    subprocess.run(cmd, check=True, capture_output=True, text=True)
    env = dict(os.environ, OMP_NUM_THREADS="2",
               ASAN_OPTIONS="detect_leaks=0:abort_on_error=0:halt_on_error=1",
               UBSAN_OPTIONS="print_stacktrace=1:halt_on_error=1")
    r = subprocess.run([exe], capture_output=True, text=True, env=env, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "host checks passed" in r.stdout
    assert "runtime error" not in r.stderr and "AddressSanitizer" not in r.stderr, r.stderr
