"""The C++ layer include/qlat_b200.hpp: the reference's C++ HMC driver
(examples-cpp/hmc/main.cpp) rewritten on it (tests/cpp/hmc_main.cpp) compiles
against the library (CPU) and, on the GPU, prints the reference's CHECK lines
(examples-cpp/hmc/log) to 12 digits."""

import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB_DIR = os.path.join(ROOT, "qlat_b200")


def build_driver(out_dir):
    exe = os.path.join(out_dir, "hmc_main")
    cmd = ["g++", "-std=c++17", "-O2", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"),
           os.path.join(ROOT, "tests", "cpp", "hmc_main.cpp"), "-L", LIB_DIR, "-lqlat_b200",
           f"-Wl,-rpath,{LIB_DIR}", "-o", exe]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-3000:]
    return exe


def test_cpp_driver_compiles_and_links(tmp_path):
    if not os.path.exists(os.path.join(LIB_DIR, "libqlat_b200.so")):
        pytest.skip("library not built")
    assert os.path.exists(build_driver(str(tmp_path)))


@pytest.mark.gpu
def test_cpp_driver_reproduces_reference_log(tmp_path, goldens):
    exe = build_driver(str(tmp_path))
    r = subprocess.run([exe], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-3000:]
    got = [(int(m.group(1)), float(m.group(2)))
           for m in re.finditer(r"CHECK: test_hmc: traj=(\d+) ; plaq_avg=\s*(\S+) ;", r.stdout)]
    rows = goldens["cpp_hmc"]["rows"]
    assert len(got) == len(rows) == 8
    for (t, p), (tr, pr, _) in zip(got, rows):
        assert t == tr
        assert abs(p - pr) <= 1e-12 * abs(pr), (t, p, pr)
    assert "CHECK: finished successfully." in r.stdout
    # reversibility lines of traj 1 and 2 (hmc.pyx:211 bound)
    for m in re.finditer(r"reversed gf_diff:\s*(\S+) /\s*(\S+)", r.stdout):
        assert float(m.group(1)) <= 1e-12 * float(m.group(2))
