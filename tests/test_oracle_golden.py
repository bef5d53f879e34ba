"""The CPU oracle against the golden values in the reference's own test logs
(examples-cpp/hmc/log and examples-py/*.log.json).  This pins the oracle
before it is used to check the CUDA library."""

import numpy as np
import pytest

TS = (4, 4, 4, 8)


def rel(a, b):
    return abs(a - b) / max(abs(b), 1e-300)


def test_sha256_fips_vectors(oracle):
    # FIPS 180-4 example messages
    assert oracle.sha256_hex(b"abc") == "ba7816bf8f01cfea414140de5dae2223b00361a396177a9cb410ff61f20015ad"
    assert oracle.sha256_hex(b"") == "e3b0c44298fc1c149afbf4c8996fb92427ae41e4649b934ca495991b7852b855"
    assert oracle.sha256_hex(b"abcdbcdecdefdefgefghfghighijhijkijkljklmklmnlmnomnopnopq") == \
        "248d6a61d20638b8e5c026930c3e6039a33ce45964ff2167f6ecedd419db06c1"


def test_cpp_hmc_log(oracle, goldens):
    """examples-cpp/hmc/main.cpp: 4 FG trajectories each of Iwasaki b=2.13 and Wilson b=5.5."""
    rows = goldens["cpp_hmc"]["rows"]
    k = 0
    for beta, c1 in [(2.13, -0.331), (5.5, 0.0)]:
        rs = oracle.RngState("test_hmc-4x4x4x8")
        gf = oracle.new_field(TS)
        oracle.set_unit(gf, TS)
        for traj in range(1, 5):
            r = rs.split(f"hmc-{traj}")
            gf0 = gf.copy()
            gm = oracle.new_field(TS)
            oracle.set_rand_gauge_momentum(gm, TS, r.split("set_rand_gauge_momentum"), 1.0)
            oracle.run_hmc_evolve(gm, gf0, TS, beta, c1, 6, 1.0)
            gf[...] = gf0  # traj <= 20: always updated
            p = oracle.gf_avg_plaq(gf, TS)
            assert rows[k][0] == traj
            assert rel(p, rows[k][1]) < 1e-12
            assert rel(512 * 6 * (1 - p), rows[k][2]) < 1e-11
            k += 1


def test_py_hmc_log(oracle, goldens):
    """examples-py/hmc-pure-gauge.py job test-4nt8: hot start, 8 trajectories with Metropolis."""
    g = goldens["py_hmc"]
    rs = oracle.RngState("run_hmc-test-4nt8")
    gf = oracle.new_field(TS)
    oracle.gf_set_rand(gf, TS, rs.split("init"), 0.1, 2)
    for traj in range(1, 9):
        flag, dh = oracle.run_hmc_pure_gauge(gf, TS, 2.13, -0.331, traj, rs.split("run_hmc_pure_gauge"),
                                             n_step=6, md_time=1.0, is_always_accept=traj < 4)
        p = oracle.gf_avg_plaq(gf, TS)
        assert rel(p, g["plaq"][traj - 1]) < 1e-12
        assert abs(dh - g["delta_h"][traj - 1]) < 1e-8
        assert rel(dh, g["delta_h"][traj - 1]) < g["eps_delta_h"]


def test_py_hmc_test_log(oracle, goldens):
    g = goldens["py_hmc_test"]
    for (beta, c1), key in [((2.13, -0.331), "iwasaki_plaq"), ((5.5, 0.0), "wilson_plaq")]:
        rs = oracle.RngState("test_hmc-[4, 4, 4, 8]")
        gf = oracle.new_field(TS)
        oracle.set_unit(gf, TS)
        for traj in range(1, 5):
            oracle.run_hmc_pure_gauge(gf, TS, beta, c1, traj, rs.split("run_hmc_pure_gauge"), is_always_accept=True)
            assert rel(oracle.gf_avg_plaq(gf, TS), g[key][traj - 1]) < 1e-12


def test_flow_log(oracle, goldens):
    g = goldens["flow"]
    rs = oracle.RngState("seed")
    gf = oracle.new_field(TS)
    oracle.gf_set_rand(gf, TS, rs.split("gf-init"), 0.5, 10)
    t = gf.copy()
    oracle.gf_wilson_flow_step(t, TS, 0.1, 0.0, "runge-kutta")
    assert rel(oracle.gf_avg_plaq(t, TS), g["rk3_plaq"]) < 1e-12
    t = gf.copy()
    oracle.gf_wilson_flow_step(t, TS, 0.1, 0.0, "euler")
    assert rel(oracle.gf_avg_plaq(t, TS), g["euler_plaq"]) < 1e-12
    for c1, v in g["c1_plaq"].items():
        t = gf.copy()
        oracle.gf_wilson_flow_step(t, TS, 0.1, float(c1))
        assert rel(oracle.gf_avg_plaq(t, TS), v) < 1e-12
    t = gf.copy()
    el = oracle.gf_wilson_flow(t, TS, 0.3, 3, 0.0)
    assert np.allclose(el, g["flow3_energy"], rtol=1e-12, atol=0)
    assert rel(oracle.gf_avg_plaq(t, TS), g["flow3_plaq"]) < 1e-12


def test_gf_utils_topology_log(oracle, goldens):
    """examples-py/gf-utils.py: clover charge at t = 0..5 of Iwasaki (c1=-0.331) flow, 50 steps per unit."""
    g = goldens["gf_utils"]
    rs = oracle.RngState("seed")
    gf = oracle.new_field(TS)
    oracle.gf_set_rand(gf, TS, rs.split("gf-init"), 0.5, 10)
    assert rel(oracle.gf_avg_plaq(gf, TS), g["hot_plaq"]) < 1e-10
    assert abs(oracle.gf_topology_clf(gf, TS) - g["topo_clf"]["0"]) < 1e-12
    for t in ("1.0", "2.0", "3.0"):
        oracle.gf_wilson_flow(gf, TS, 1.0, 50, -0.331)
        assert rel(oracle.gf_topology_clf(gf, TS), g["topo_clf"][t]) < g["eps_topo"]


def test_gf_utils_topology_5li_log(oracle, goldens):
    """examples-py/gf-utils.py: the 5-loop improved charge (gf_topology) and the
    sum of its five terms at t = 0, 1, 2 of the c1 = -0.331 flow."""
    g = goldens["gf_utils"]
    rs = oracle.RngState("seed")
    gf = oracle.new_field(TS)
    oracle.gf_set_rand(gf, TS, rs.split("gf-init"), 0.5, 10)
    for t in ("0", "1.0", "2.0"):
        if t != "0":
            oracle.gf_wilson_flow(gf, TS, 1.0, 50, -0.331)
        q = oracle.gf_topology(gf, TS)
        assert abs(q - g["topo_5li"][t]) < g["eps_topo"] * max(1.0, abs(q)), (t, q)
        terms = oracle.clf_topology_field_5_terms(gf, TS).sum(axis=0)
        assert abs(terms.sum() - g["topo_5li_terms_sum"][t]) < g["eps_topo"] * max(1.0, abs(q))


def test_metropolis_draw_conventions(oracle):
    """The C++ metropolis_accept draws u_rand_gen(rs, 0.0, 1.0) = 1 - u
    (hmc.cpp:91); the Python one draws u_rand_gen(1.0, 0.0) = u (hmc.pyx:149)."""
    rs = oracle.RngState("m")
    u = rs.copy().u_rand_gen(1.0, 0.0)
    v = rs.copy().u_rand_gen(0.0, 1.0)
    assert abs((1.0 - u) - v) < 1e-15
