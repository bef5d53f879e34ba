"""HMC and gradient flow on the GPU against the reference's golden logs and
the oracle: the same driver scripts as examples-cpp/hmc/main.cpp,
examples-py/hmc-pure-gauge*.py, flow-and-smear.py and gf-utils.py, run
through the qlat-compatible API of the CUDA library."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TS = (4, 4, 4, 8)


def rel(a, b):
    return abs(a - b) / max(abs(b), 1e-300)


def test_cpp_hmc_log(q, goldens):
    """examples-cpp/hmc/main.cpp (C++ metropolis semantics, always updated for traj <= 20)."""
    rows = goldens["cpp_hmc"]["rows"]
    k = 0
    for beta, c1 in [(2.13, -0.331), (5.5, 0.0)]:
        ga = q.GaugeAction(beta, c1)
        geo = q.Geometry(TS)
        rs = q.RngState("test_hmc-4x4x4x8")
        gf = q.GaugeField(geo)
        gf.set_unit()
        for traj in range(1, 5):
            r = rs.split(f"hmc-{traj}")
            gf0 = gf.copy()
            gm = q.GaugeMomentum(geo)
            q.set_rand_gauge_momentum(gm, 1.0, r.split("set_rand_gauge_momentum"))
            dh = q.run_hmc_evolve_pure_gauge(gm, gf0, ga, r, 6, 1.0)
            q.metropolis_accept_cpp(dh, traj, r.split("metropolis_accept"))
            gf @= gf0
            p = q.gf_avg_plaq(gf)
            assert rows[k][0] == traj
            assert rel(p, rows[k][1]) < 1e-12, (traj, p, rows[k][1])
            k += 1


def test_py_hmc_log(q, oracle, goldens):
    """examples-py/hmc-pure-gauge.py test-4nt8: plaq and delta_h per trajectory
    and the accept/reject sequence of the oracle."""
    g = goldens["py_hmc"]
    ga = q.GaugeAction(2.13, -0.331)
    rs = q.RngState("run_hmc-test-4nt8")
    gf = q.GaugeField(q.Geometry(TS))
    gf.set_rand(rs.split("init"), 0.1, 2)
    # oracle replay for the accept sequence
    ors = oracle.RngState("run_hmc-test-4nt8")
    ogf = oracle.new_field(TS)
    oracle.gf_set_rand(ogf, TS, ors.split("init"), 0.1, 2)
    for traj in range(1, 9):
        flag, dh = q.run_hmc_pure_gauge(gf, ga, traj, rs.split("run_hmc_pure_gauge"), n_step=6, md_time=1.0,
                                        is_always_accept=traj < 4, is_reverse_test=traj < 2)
        oflag, odh = oracle.run_hmc_pure_gauge(ogf, TS, 2.13, -0.331, traj, ors.split("run_hmc_pure_gauge"),
                                               n_step=6, md_time=1.0, is_always_accept=traj < 4)
        p = q.gf_avg_plaq(gf)
        assert flag == oflag
        assert rel(p, g["plaq"][traj - 1]) < g["eps_plaq"]
        assert rel(p, oracle.gf_avg_plaq(ogf, TS)) < 1e-12
        assert rel(dh, g["delta_h"][traj - 1]) < g["eps_delta_h"]
        assert abs(dh - odh) < 1e-9


def test_py_hmc_test_log(q, goldens):
    g = goldens["py_hmc_test"]
    for (beta, c1), key in [((2.13, -0.331), "iwasaki_plaq"), ((5.5, 0.0), "wilson_plaq")]:
        ga = q.GaugeAction(beta, c1)
        rs = q.RngState("test_hmc-[4, 4, 4, 8]")
        gf = q.GaugeField(q.Geometry(TS))
        q.set_unit(gf)
        for traj in range(1, 5):
            q.run_hmc_pure_gauge(gf, ga, traj, rs.split("run_hmc_pure_gauge"), is_always_accept=True)
            assert rel(q.gf_avg_plaq(gf), g[key][traj - 1]) < g["eps"]


def test_reversibility(q):
    """hmc.pyx:200-211: forward then backward returns to the start within 1e-12."""
    ga = q.GaugeAction(2.13, -0.331)
    gf = q.GaugeField(q.Geometry((4, 4, 4, 4)))
    gf.set_rand(q.RngState("rev"), 0.3, 1)
    q.run_hmc_pure_gauge(gf, ga, 1, q.RngState("rev-hmc"), is_reverse_test=True)
    dsum, dnorm, norm = q.run_hmc_pure_gauge.last_reverse
    assert dnorm <= 1e-12 * norm
    assert abs(dsum) < 1e-9


def test_leapfrog_chain_8x4(q, oracle):
    """8^4 Wilson beta=5.5 leapfrog, 6 steps, 10 trajectories from a scale-1.0
    hot start: plaquette and delta_h against the oracle and an identical
    accept/reject sequence."""
    ts = (8, 8, 8, 8)
    ga = q.GaugeAction(5.5, 0.0)
    rs = q.RngState("b200-c1-8x4-wilson")
    gf = q.GaugeField(q.Geometry(ts))
    gf.set_rand(rs.split("gf-init"), 1.0, 1)
    oracle.set_log_mode(1)
    try:
        ors = oracle.RngState("b200-c1-8x4-wilson")
        ogf = oracle.new_field(ts)
        oracle.gf_set_rand(ogf, ts, ors.split("gf-init"), 1.0, 1)
        assert np.array_equal(np.asarray(gf), ogf)
        for traj in range(1, 11):
            flag, dh = q.run_hmc_pure_gauge(gf, ga, traj, rs.split("hmc"), n_step=6, integrator="leapfrog")
            oflag, odh = oracle.run_hmc_pure_gauge(ogf, ts, 5.5, 0.0, traj, ors.split("hmc"), n_step=6,
                                                   integrator="leapfrog")
            assert flag == oflag
            assert abs(dh - odh) <= 1e-12 * 4096 * 6 * 3 * 5.5
            assert rel(q.gf_avg_plaq(gf), oracle.gf_avg_plaq(ogf, ts)) < 1e-12
    finally:
        oracle.set_log_mode(0)


def test_mixed_precision_trajectory(q):
    """FP32 molecular dynamics with FP64 Hamiltonians: delta_h and the new
    plaquette agree with the FP64 form to FP32 accuracy."""
    ts = (6, 6, 6, 12)
    ga = q.GaugeAction(2.13, -0.331)
    gf = q.GaugeField(q.Geometry(ts))
    gf.set_rand(q.RngState("mixed").split("gf-init"), 0.3, 1)
    gm = q.GaugeMomentum(gf.geo)
    gm.set_rand(q.RngState("mixed").split("mom"), 1.0)
    g64, m64 = gf.copy(), gm.copy()
    dh64 = q.run_hmc_evolve_pure_gauge(m64, g64, ga, None, 8, 1.0, precision="fp64")
    for reunit in (4, 0):
        g32, m32 = gf.copy(), gm.copy()
        dh32 = q.run_hmc_evolve_pure_gauge(m32, g32, ga, None, 8, 1.0, precision="mixed", reunit_interval=reunit)
        assert abs(dh32 - dh64) < 2e-3 * max(1.0, abs(dh64)) + 5e-4
        assert abs(q.gf_avg_plaq(g32) - q.gf_avg_plaq(g64)) < 1e-6


def test_flow_log(q, goldens):
    g = goldens["flow"]
    rs = q.RngState("seed")
    gf = q.GaugeField(q.Geometry(TS))
    gf.set_rand(rs.split("gf-init"), 0.5, 10)
    t = gf.copy()
    q.gf_wilson_flow_step(t, 0.1, c1=0.0, wilson_flow_integrator_type="runge-kutta")
    assert rel(t.plaq(), g["rk3_plaq"]) < g["eps"]
    t = gf.copy()
    q.gf_wilson_flow_step(t, 0.1, c1=0.0, wilson_flow_integrator_type="euler")
    assert rel(t.plaq(), g["euler_plaq"]) < g["eps"]
    for c1, v in g["c1_plaq"].items():
        t = gf.copy()
        q.gf_wilson_flow_step(t, 0.1, c1=float(c1))
        assert rel(t.plaq(), v) < g["eps"]
    t = gf.copy()
    el = q.gf_wilson_flow(t, 0.3, 3, c1=0.0)
    assert np.allclose(el, g["flow3_energy"], rtol=g["eps"], atol=0)
    assert rel(t.plaq(), g["flow3_plaq"]) < g["eps"]


def test_gf_utils_topology_log(q, goldens):
    g = goldens["gf_utils"]
    rs = q.RngState("seed")
    gf = q.GaugeField(q.Geometry(TS))
    gf.set_rand(rs.split("gf-init"), 0.5, 10)
    assert rel(gf.plaq(), g["hot_plaq"]) < 1e-10
    assert abs(q.gf_topology_clf(gf) - g["topo_clf"]["0"]) < 1e-12
    for t in ("0", "1.0", "2.0", "3.0", "4.0", "5.0"):
        if t != "0":
            q.gf_wilson_flow(gf, 1.0, 50, c1=-0.331)
            assert rel(q.gf_topology_clf(gf), g["topo_clf"][t]) < g["eps_topo"]
        # 5-loop improved charge (topo_5li) and the sum of its terms
        q5 = q.gf_topology(gf)
        assert abs(q5 - g["topo_5li"][t]) < g["eps_topo"] * max(1.0, abs(q5)), (t, q5)
        assert abs(q.gf_topology_terms(gf).sum() - g["topo_5li_terms_sum"][t]) < g["eps_topo"] * max(1.0, abs(q5))


@pytest.mark.parametrize("ts", [(6, 6, 6, 12), (3, 5, 7, 4)])
def test_mixed_trajectory_equals_its_steps(q, ts):
    """The mixed trajectory, whose H0 / H1 kernels also convert the fields,
    equals the same steps run one by one (FP64 Hamiltonians, FP32 copies,
    FP32 molecular dynamics with re-unitarisation every 4 steps, copies back,
    unitarize, FP64 Hamiltonians) bit for bit: delta_h, links and momenta.
    3 x 5 x 7 x 4 has a partly filled last block of 32 sites."""
    import ctypes
    from qlat_b200._lib import HALO_HOOK, call
    ga = q.GaugeAction(2.13, -0.331)
    gf = q.GaugeField(q.Geometry(ts))
    gf.set_rand(q.RngState("mixed-steps").split("gf-init"), 0.3, 1)
    gm = q.GaugeMomentum(gf.geo)
    gm.set_rand(q.RngState("mixed-steps").split("mom"), 1.0)
    g1, m1 = gf.copy(), gm.copy()
    dh = q.run_hmc_evolve_pure_gauge(m1, g1, ga, None, 8, 1.0, precision="mixed", reunit_interval=4)
    g2, m2 = gf.copy(), gm.copy()
    h0 = q.gm_hamilton_node(m2) + q.gf_hamilton_node(g2, ga)
    g32, m32 = g2.copy(precision=q.F32), m2.copy(precision=q.F32)
    call("qgb_run_md_hooked", m32.handle, g32.handle, ga.beta(), ga.c1(), 8, 1.0, 0, 4, 0,
         ctypes.cast(None, HALO_HOOK), None)
    g2 @= g32
    m2 @= m32
    q.unitarize(g2)
    h1 = q.gm_hamilton_node(m2) + q.gf_hamilton_node(g2, ga)
    assert dh == h1 - h0
    assert np.array_equal(np.asarray(g1), np.asarray(g2))
    assert np.array_equal(np.asarray(m1), np.asarray(m2))


@pytest.mark.parametrize("n_step", [5, 6])
def test_mixed_leapfrog_close_to_fp64(q, n_step):
    """The mixed form's leapfrog, each step one launch that writes the next
    links into the other of two buffers (odd and even step counts end in
    either), against the FP64 leapfrog of the reference's composition."""
    ts = (6, 6, 6, 12)
    ga = q.GaugeAction(5.5, 0.0)
    gf = q.GaugeField(q.Geometry(ts))
    gf.set_rand(q.RngState("mixed-lf").split("gf-init"), 0.3, 1)
    gm = q.GaugeMomentum(gf.geo)
    gm.set_rand(q.RngState("mixed-lf").split("mom"), 1.0)
    g64, m64 = gf.copy(), gm.copy()
    dh64 = q.run_hmc_evolve_pure_gauge(m64, g64, ga, None, n_step, 1.0, integrator="leapfrog", precision="fp64")
    for reunit in (4, 0):
        g32, m32 = gf.copy(), gm.copy()
        dh32 = q.run_hmc_evolve_pure_gauge(m32, g32, ga, None, n_step, 1.0, integrator="leapfrog",
                                           precision="mixed", reunit_interval=reunit)
        assert abs(dh32 - dh64) < 2e-3 * max(1.0, abs(dh64)) + 5e-4, (reunit, dh32, dh64)
        assert abs(q.gf_avg_plaq(g32) - q.gf_avg_plaq(g64)) < 1e-6


@pytest.mark.parametrize("precision,integrator", [("fp64", "force-gradient"), ("mixed", "force-gradient"),
                                                  ("mixed", "leapfrog")])
def test_trajectory_graph_replay_matches_direct(q, precision, integrator):
    """A trajectory replayed from its CUDA graph (second call records, later
    calls replay) is bit for bit the trajectory of direct launches, with the
    same kernel count."""
    geo = q.Geometry((4, 4, 6, 8))
    ga = q.GaugeAction(2.13, -0.331)
    rs = q.RngState("test_graph_replay")
    start = q.GaugeField(geo)
    start.set_rand(rs.split("init"), 0.3, 2)
    gm0 = q.GaugeMomentum(geo)
    gm0.set_rand(rs.split("gm"), 1.0)
    kw = dict(integrator=integrator, precision=precision, reunit_interval=2)
    gf, gm = q.GaugeField(geo), q.GaugeMomentum(geo)
    q.set_trajectory_graphs(False)
    try:
        gf @= start
        gm @= gm0
        l0 = q.launch_count()
        dh_direct = q.run_hmc_evolve_pure_gauge(gm, gf, ga, None, 5, 1.0, **kw)
        n_direct = q.launch_count() - l0
        gf_direct, gm_direct = np.asarray(gf).copy(), np.asarray(gm).copy()
    finally:
        q.set_trajectory_graphs(True)
    assert q.trajectory_graph_count() == 0
    for call in range(4):
        gf @= start
        gm @= gm0
        l0 = q.launch_count()
        dh = q.run_hmc_evolve_pure_gauge(gm, gf, ga, None, 5, 1.0, **kw)
        assert q.launch_count() - l0 == n_direct
        assert dh == dh_direct, (call, dh, dh_direct)
        assert np.array_equal(np.asarray(gf), gf_direct), call
        assert np.array_equal(np.asarray(gm), gm_direct), call
        assert q.trajectory_graph_count() == (0 if call == 0 else 1)
    # another parameter is another graph
    gf @= start
    gm @= gm0
    q.run_hmc_evolve_pure_gauge(gm, gf, ga, None, 6, 1.0, **kw)
    q.run_hmc_evolve_pure_gauge(gm, gf, ga, None, 6, 1.0, **kw)
    assert q.trajectory_graph_count() == 2
