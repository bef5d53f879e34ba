"""Host check of the FP32 su(3) exponential of the fused force epilogues
(su3.cuh exp_su3) against the general FP64 Cayley-Hamilton exponential, on
random su(3) matrices of norm 1e-5 .. 3.4 (tests/cpp/exp_su3_check.cpp)."""

import os
import subprocess

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_exp_su3_matches_fp64(tmp_path):
    exe = os.path.join(str(tmp_path), "exp_su3_check")
    cmd = ["g++", "-std=c++17", "-O2", "-ffp-contract=off", "-I", os.path.join(ROOT, "qlat_b200", "csrc"),
           "-I", "/usr/local/cuda/include", os.path.join(ROOT, "tests", "cpp", "exp_su3_check.cpp"), "-o", exe]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    # FP32 resolution (6e-8) times the size of exp's entries and the rounding of ~20 recursion steps
    r = subprocess.run([exe, "1e-6"], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
