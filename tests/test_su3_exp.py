"""Host check of the su(3) exponential of the fused force epilogues (su3.cuh
exp_su3), FP32 and FP64, against the general FP64 Cayley-Hamilton exponential
(all 20 terms), on random su(3) matrices of norm 1e-5 .. 3.4
(tests/cpp/exp_su3_check.cpp)."""

import os
import subprocess

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_exp_su3_matches_fp64(tmp_path):
    exe = os.path.join(str(tmp_path), "exp_su3_check")
    cmd = ["g++", "-std=c++17", "-O2", "-ffp-contract=off", "-I", os.path.join(ROOT, "qlat_b200", "csrc"),
           "-I", "/usr/local/cuda/include", os.path.join(ROOT, "tests", "cpp", "exp_su3_check.cpp"), "-o", exe]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    # FP32: its resolution (6e-8) times the size of exp's entries and the rounding of ~20 recursion steps;
    # FP64: the same polynomial to rounding (the omitted terms are below 2^-56)
    r = subprocess.run([exe, "1e-6", "1e-14"], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
