"""Two more of the reference's HMC examples, replayed from their drivers'
logic against their golden logs:

- examples-py/hmc-pure-gauge-symmetric.py: every link moved by a momentum from
  the left and a dual momentum from the right (gf_evolve + gf_evolve_dual,
  set_gm_force_dual), Omelyan force gradient, 8 trajectories.  On the CPU
  oracle and on the GPU.
- examples-py/hmc-pure-gauge-flowed.py: flowed HMC with the flow of
  FlowInfo.add_rand_order_flow(rng, 0.1), the output-argument forms
  gf_flow(gf, gf0, fi) / gf_flow_inv(gf, gf1, fi) of qlat.fthmc, 8
  trajectories (the fifth is rejected).  On the GPU.
"""

import math

import pytest

EPS = 1e-10


# ---- hmc-pure-gauge-symmetric.py (lines 34-209) ----------------------------------------------


def symmetric_oracle(o, g):
    h, ts = g["hmc"], tuple(g["total_site"])
    beta, c1 = h["beta"], h["c1"]

    def evolve(gf, gm, gmd, dt):
        o.gf_evolve(gf, gm, ts, dt)
        o.gf_evolve_dual(gf, gmd, ts, dt)

    def gm_evolve_fg(gm, gmd, gf_init, fg_dt, dt):
        gf = gf_init.copy()
        F, Fd = o.new_field(ts), o.new_field(ts)
        o.set_gm_force(F, gf, ts, beta, c1)
        o.set_gm_force_dual(Fd, gf, F, ts)
        evolve(gf, F, Fd, fg_dt)
        o.set_gm_force(F, gf, ts, beta, c1)
        o.set_gm_force_dual(Fd, gf, F, ts)
        gm += F * dt
        gmd += Fd * dt

    def ham(gm, gmd, gf):
        return o.gm_hamilton_node(gm, ts) + o.gm_hamilton_node(gmd, ts) + o.gf_hamilton_node(gf, ts, beta, c1)

    def run_hmc_evolve(gm, gmd, gf, n_step, md_time):
        energy = ham(gm, gmd, gf)
        dt = md_time / n_step
        lam = 0.5 * (1.0 - 1.0 / math.sqrt(3.0))
        ttheta = (2.0 - math.sqrt(3.0)) / 48.0 * dt * dt * dt
        evolve(gf, gm, gmd, lam * dt)
        for i in range(n_step):
            gm_evolve_fg(gm, gmd, gf, 4.0 * ttheta / dt, 0.5 * dt)
            evolve(gf, gm, gmd, (1.0 - 2.0 * lam) * dt)
            gm_evolve_fg(gm, gmd, gf, 4.0 * ttheta / dt, 0.5 * dt)
            evolve(gf, gm, gmd, (2.0 if i < n_step - 1 else 1.0) * lam * dt)
        o.unitarize(gf, ts)
        return ham(gm, gmd, gf) - energy

    rs = o.RngState(f"run_hmc-{g['job_tag']}")
    gf = o.new_field(ts)
    o.gf_set_rand(gf, ts, rs.split("init"), 0.1, 2)
    plaqs = []
    for traj in range(1, h["max_traj"] + 1):
        r = rs.split("run_hmc_traj").split(f"{traj}")
        gf0 = gf.copy()
        gm, gmd = o.new_field(ts), o.new_field(ts)
        o.set_rand_gauge_momentum(gm, ts, r.split("set_rand_gauge_momentum"), 1.0)
        o.set_rand_gauge_momentum(gmd, ts, r.split("set_rand_gauge_momentum_dual"), 1.0)
        dh = run_hmc_evolve(gm, gmd, gf0, h["n_step"], h["md_time"])
        flag, _ = o.metropolis_accept_py(dh, r.split("metropolis_accept"))
        if flag or traj < h["max_traj_always_accept"]:
            gf = gf0
        plaqs.append(o.gf_avg_plaq(gf, ts))
    return plaqs


def symmetric_gpu(q, g):
    h = g["hmc"]
    ga = q.GaugeAction(h["beta"], h["c1"])
    geo = q.Geometry(tuple(g["total_site"]))

    def evolve(gf, gm, gmd, dt):
        q.gf_evolve(gf, gm, dt)
        q.gf_evolve_dual(gf, gmd, dt)

    def gm_evolve_fg(gm, gmd, gf_init, fg_dt, dt):
        gf = gf_init.copy()
        F, Fd = q.GaugeMomentum(geo), q.GaugeMomentum(geo)
        q.set_gm_force(F, gf, ga)
        q.set_gm_force_dual(Fd, gf, F)
        evolve(gf, F, Fd, fg_dt)
        q.set_gm_force(F, gf, ga)
        q.set_gm_force_dual(Fd, gf, F)
        F *= dt
        Fd *= dt
        gm += F
        gmd += Fd

    def ham(gm, gmd, gf):
        return q.gm_hamilton_node(gm) + q.gm_hamilton_node(gmd) + q.gf_hamilton_node(gf, ga)

    def run_hmc_evolve(gm, gmd, gf, n_step, md_time):
        energy = ham(gm, gmd, gf)
        dt = md_time / n_step
        lam = 0.5 * (1.0 - 1.0 / math.sqrt(3.0))
        ttheta = (2.0 - math.sqrt(3.0)) / 48.0 * dt * dt * dt
        evolve(gf, gm, gmd, lam * dt)
        for i in range(n_step):
            gm_evolve_fg(gm, gmd, gf, 4.0 * ttheta / dt, 0.5 * dt)
            evolve(gf, gm, gmd, (1.0 - 2.0 * lam) * dt)
            gm_evolve_fg(gm, gmd, gf, 4.0 * ttheta / dt, 0.5 * dt)
            evolve(gf, gm, gmd, (2.0 if i < n_step - 1 else 1.0) * lam * dt)
        gf.unitarize()
        return ham(gm, gmd, gf) - energy

    rs = q.RngState(f"run_hmc-{g['job_tag']}")
    gf = q.GaugeField(geo)
    gf.set_rand(rs.split("init"), 0.1, 2)
    plaqs = []
    for traj in range(1, h["max_traj"] + 1):
        r = rs.split("run_hmc_traj").split(f"{traj}")
        gf0 = gf.copy()
        gm, gmd = q.GaugeMomentum(geo), q.GaugeMomentum(geo)
        gm.set_rand(r.split("set_rand_gauge_momentum"), 1.0)
        gmd.set_rand(r.split("set_rand_gauge_momentum_dual"), 1.0)
        dh = run_hmc_evolve(gm, gmd, gf0, h["n_step"], h["md_time"])
        if traj < h["max_traj_reverse_test"]:
            gm_r, gmd_r, gf0_r = gm.copy(), gmd.copy(), gf0.copy()
            run_hmc_evolve(gm_r, gmd_r, gf0_r, h["n_step"], -h["md_time"])
            gf0_r -= gf
            assert gf0_r.qnorm() <= 1e-12 * gf0.qnorm()
        flag, _ = q.metropolis_accept(dh, traj, r.split("metropolis_accept"))
        if flag or traj < h["max_traj_always_accept"]:
            gf @= gf0
        plaqs.append(gf.plaq())
    return plaqs


def test_symmetric_example_on_the_oracle(oracle, goldens):
    g = goldens["py_hmc_symmetric"]
    oracle.set_log_mode(1)
    try:
        got = symmetric_oracle(oracle, g)
    finally:
        oracle.set_log_mode(0)
    for t, (a, b) in enumerate(zip(got, g["plaq"])):
        assert abs(a - b) <= EPS * abs(b), (t + 1, a, b)


@pytest.mark.gpu
def test_symmetric_example_on_the_gpu(q, goldens):
    g = goldens["py_hmc_symmetric"]
    for t, (a, b) in enumerate(zip(symmetric_gpu(q, g), g["plaq"])):
        assert abs(a - b) <= EPS * abs(b), (t + 1, a, b)


# ---- hmc-pure-gauge-flowed.py (lines 27-249) -------------------------------------------------


def flowed_gpu(q, g):
    h = g["hmc"]
    ga = q.GaugeAction(h["beta"], h["c1"])
    geo = q.Geometry(tuple(g["total_site"]))

    def gm_evolve_fg(gm, gf_init, fi, fg_dt, dt):
        gf = q.GaugeField(geo)
        gf @= gf_init
        gm_force = q.GaugeMomentum(geo)
        q.set_gm_force_flowed(gm_force, gf, ga, fi)
        q.gf_evolve(gf, gm_force, fg_dt)
        q.set_gm_force_flowed(gm_force, gf, ga, fi)
        gm_force *= dt
        gm += gm_force

    def run_hmc_evolve_flowed(gm, gf, fi, steps, md_time):
        energy = q.gm_hamilton_node(gm) + q.gf_hamilton_flowed_node(gf, ga, fi)
        dt = md_time / steps
        lam = 0.5 * (1.0 - 1.0 / math.sqrt(3.0))
        ttheta = (2.0 - math.sqrt(3.0)) / 48.0 * dt * dt * dt
        q.gf_evolve(gf, gm, lam * dt)
        for i in range(steps):
            gm_evolve_fg(gm, gf, fi, 4.0 * ttheta / dt, 0.5 * dt)
            q.gf_evolve(gf, gm, (1.0 - 2.0 * lam) * dt)
            gm_evolve_fg(gm, gf, fi, 4.0 * ttheta / dt, 0.5 * dt)
            q.gf_evolve(gf, gm, (2.0 if i < steps - 1 else 1.0) * lam * dt)
        q.unitarize(gf)
        return q.gm_hamilton_node(gm) + q.gf_hamilton_flowed_node(gf, ga, fi) - energy

    rs = q.RngState(f"run_hmc-{g['job_tag']}")
    gf = q.GaugeField(geo)
    gf.set_rand(rs.split("init"), 0.1, 2)
    plaqs = []
    for traj in range(1, h["max_traj"] + 1):
        r = rs.split("run_hmc_traj").split(f"{traj}")
        fi = q.FlowInfo()
        fi.add_rand_order_flow(r.split("mk_flow_info"), h["fp"]["time"])
        gf0 = q.GaugeField(geo)
        q.gf_flow_inv(gf0, gf, fi)
        if traj < h["max_traj_reverse_test"]:
            gf_r = q.GaugeField(geo)
            q.gf_flow(gf_r, gf0, fi)
            gf_r -= gf
            assert gf_r.qnorm() <= 1e-12 * gf.qnorm()
        gm = q.GaugeMomentum(geo)
        gm.set_rand(r.split("set_rand_gauge_momentum"), 1.0)
        dh = run_hmc_evolve_flowed(gm, gf0, fi, h["n_step"], h["md_time"])
        if traj < h["max_traj_reverse_test"]:
            gm_r, gf0_r = gm.copy(), gf0.copy()
            run_hmc_evolve_flowed(gm_r, gf0_r, fi, h["n_step"], -h["md_time"])
            q.gf_flow(gf0_r, gf0_r, fi)
            gf0_r -= gf
            assert gf0_r.qnorm() <= 1e-12 * gf0.qnorm()
        flag, _ = q.metropolis_accept(dh, traj, r.split("metropolis_accept"))
        if flag or traj < h["max_traj_always_accept"]:
            q.gf_flow(gf, gf0, fi)
        plaqs.append(gf.plaq())
    return plaqs


@pytest.mark.gpu
def test_flowed_example_on_the_gpu(q, goldens):
    g = goldens["py_hmc_flowed"]
    for t, (a, b) in enumerate(zip(flowed_gpu(q, g), g["plaq"])):
        assert abs(a - b) <= EPS * abs(b), (t + 1, a, b)


@pytest.mark.gpu
def test_flowed_force_no_det_of_the_action_force(q):
    """set_gm_force_flowed_no_det(F, F_pre, gf0, fi) with F_pre the action's
    force on the flowed field equals set_gm_force_flowed(..., with_det=False)."""
    import numpy as np
    geo = q.Geometry((4, 4, 4, 8))
    gf0 = q.GaugeField(geo)
    gf0.set_rand(q.RngState("no-det").split("gf"), 0.3, 1)
    fi = q.FlowInfo()
    fi.add_rand_order_flow(q.RngState("no-det-fi"), 0.1, -0.01)
    fi.add_flow(1, 2, 0.05)
    ga = q.GaugeAction(2.31, -0.331)
    gfl = q.GaugeField(geo)
    q.gf_flow(gfl, gf0, fi)
    pre = q.GaugeMomentum(geo)
    q.set_gm_force(pre, gfl, ga)
    a, b = q.GaugeMomentum(geo), q.GaugeMomentum(geo)
    q.set_gm_force_flowed_no_det(a, pre, gf0, fi)
    q.set_gm_force_flowed(b, gf0, ga, fi, with_det=False)
    assert np.abs(np.asarray(a) - np.asarray(b)).max() < 1e-15
    assert len(fi.v) == 17 and "mask=1, mu=2" in fi.show()
