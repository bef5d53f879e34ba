"""The C++ layer include/qlat_b200.hpp: the reference's C++ HMC and flowed-HMC
drivers (examples-cpp/hmc/main.cpp, examples-cpp/flowed-hmc/main.cpp)
rewritten on it (tests/cpp/hmc_main.cpp, tests/cpp/flowed_hmc_main.cpp)
compile against the library (CPU) and, on the GPU, print the reference's CHECK
lines (examples-cpp/hmc/log, examples-cpp/flowed-hmc/log) to 12 digits.  A
time-slab caller written on the bare C ABI (tests/cpp/slab_hook_main.cpp: a C
halo hook, owned-site sums) reproduces the plain trajectory on the GPU."""

import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB_DIR = os.path.join(ROOT, "qlat_b200")


CUDA = os.environ.get("CUDA_HOME", "/usr/local/cuda")
# drivers that allocate their own device buffers (the halo hook's) use the CUDA runtime too
CUDART = {"slab_hook_main": ["-I", os.path.join(CUDA, "include"), "-L", os.path.join(CUDA, "lib64"), "-lcudart"]}


def build_driver(out_dir, name="hmc_main"):
    exe = os.path.join(out_dir, name)
    cmd = ["g++", "-std=c++17", "-O2", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"),
           os.path.join(ROOT, "tests", "cpp", name + ".cpp"), "-L", LIB_DIR, "-lqlat_b200",
           f"-Wl,-rpath,{LIB_DIR}", *CUDART.get(name, []), "-o", exe]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-3000:]
    return exe


@pytest.mark.parametrize("name", ["hmc_main", "flowed_hmc_main", "api_surface", "slab_hook_main"])
def test_cpp_driver_compiles_and_links(tmp_path, name):
    if not os.path.exists(os.path.join(LIB_DIR, "libqlat_b200.so")):
        pytest.skip("library not built")
    assert os.path.exists(build_driver(str(tmp_path), name))


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


@pytest.mark.gpu
def test_cpp_flowed_driver_reproduces_reference_log(tmp_path, goldens):
    exe = build_driver(str(tmp_path), "flowed_hmc_main")
    r = subprocess.run([exe], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-3000:]
    got = [(int(m.group(1)), float(m.group(2)))
           for m in re.finditer(r"CHECK: test_hmc: traj=(\d+) ; plaq_avg=\s*(\S+) ;", r.stdout)]
    rows = goldens["cpp_flowed_hmc"]["rows"]
    assert len(got) == len(rows) == 3
    for (t, p), (tr, pr, _) in zip(got, rows):
        assert t == tr
        assert abs(p - pr) <= 1e-11 * abs(pr), (t, p, pr)
    assert "CHECK: finished successfully." in r.stdout
    # the inverse flow undoes the flow, and the trajectory reverses
    for m in re.finditer(r"gf_flow_inv gf_diff:\s*(\S+) /\s*(\S+)", r.stdout):
        assert float(m.group(1)) <= 1e-20 * float(m.group(2))
    for m in re.finditer(r"reversed gf_diff:\s*(\S+) /\s*(\S+)", r.stdout):
        assert float(m.group(1)) <= 1e-12 * float(m.group(2))


@pytest.mark.gpu
def test_cpp_api_surface_matches_python(q, tmp_path):
    """The C++ wrappers return what the Python API returns on the same seeds."""
    import numpy as np
    exe = build_driver(str(tmp_path), "api_surface")
    r = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-3000:]
    got = {ln.split()[0]: float(ln.split()[1]) for ln in r.stdout.splitlines() if ln.strip()}
    geo = q.Geometry((4, 4, 4, 8))
    rs = q.RngState("api-surface")
    gf = q.GaugeField(geo)
    gf.set_rand(rs.split("gf"), 0.3, 2)
    mf, mfd = q.FieldRealD(geo, 4), q.FieldRealD(geo, 4)
    mf.set_rand(rs.split("mf"), 4.0, 1.0)
    mfd.set_rand(rs.split("mfd"), 4.0, 1.0)
    gm, gmd = q.GaugeMomentum(geo), q.GaugeMomentum(geo)
    gm.set_rand_fa(mf, rs.split("gm"))
    gmd.set_rand_fa(mfd, rs.split("gmd"))
    want = {"gm_hamilton_fa": q.gm_hamilton_node_fa(gm, mf), "project": q.project_gauge_transform(gm, gmd, mf, mfd)}
    g1 = gf.copy()
    q.gf_evolve_fa(g1, gm, mf, 0.1)
    q.gf_evolve_fa_dual(g1, gmd, mfd, 0.1)
    q.gf_evolve_dual(g1, gmd, 0.05)
    want["plaq_fa"] = g1.plaq()
    F, Fd = q.GaugeMomentum(geo), q.GaugeMomentum(geo)
    q.set_gm_force(F, gf, q.GaugeAction(2.13, -0.331))
    q.set_gm_force_dual(Fd, gf, F)
    want["qnorm_force_dual"] = Fd.qnorm()
    want["dot"] = float(q.dot_gauge_momentum(gm, gmd).to_numpy().sum())
    gr = q.FieldRealD(geo, 3)
    gr.set_rand_g(rs.split("g"), 0.5, 2.0)
    want["g_rand"] = float(gr.to_numpy().sum())
    fp = q.gf_plaq_field(gf)
    want.update(plaq_field=float(fp.to_numpy().sum()), energy=float(q.gf_energy_density_field(gf).to_numpy().sum()),
                energy_dir=float(q.gf_energy_density_dir_field(gf).to_numpy().sum()),
                paf=float(q.gf_plaq_action_density_field(gf).to_numpy().sum()),
                spaf=float(q.gf_spatial_plaq_action_density_field(gf).to_numpy().sum()),
                topo_clf=float(q.gf_topology_field_clf(gf).to_numpy().sum()),
                topo_5=float(q.gf_topology_field(gf).to_numpy().sum()), topology_charge_5=q.topology_charge_5(gf),
                z=q.gf_wilson_flow_force(gf, -0.331).qnorm(), zp=q.gf_plaq_flow_force(gf, fp).qnorm())
    g2 = gf.copy()
    q.gf_wilson_flow_step(g2, 0.05, c1=-0.331, wilson_flow_integrator_type="euler")
    want["plaq_euler"] = g2.plaq()
    fi = q.mk_flow_info_step(rs.split("fi"), 0.1)
    want["flow_steps"] = len(fi.v)
    act, ld = q.gf_hamilton_flowed(gf, q.GaugeAction(2.31, -0.331), fi)
    want["flowed_action"] = act - ld
    g3 = gf.copy()
    m3 = q.GaugeMomentum(geo)
    m3.set_rand(rs.split("mom"), 1.0)
    want["delta_h_mixed"] = q.run_hmc_evolve_pure_gauge(m3, g3, q.GaugeAction(2.13, -0.331), None, 6,
                                                        precision="mixed", reunit_interval=4)
    want["plaq_mixed"] = g3.plaq()
    for k, v in want.items():
        assert abs(got[k] - v) <= 1e-12 * max(abs(v), 1.0), (k, got[k], v)
    assert got["flow_round_trip"] < 1e-24 * gf.qnorm()


@pytest.mark.gpu
def test_cpp_slab_hook_driver(tmp_path):
    exe = build_driver(str(tmp_path), "slab_hook_main")
    r = subprocess.run([exe], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    assert "CHECK: slab hook ok" in r.stdout
