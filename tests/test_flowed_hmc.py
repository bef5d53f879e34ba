"""Flowed HMC with masked invertible flows (flowed-hmc.cpp) against the
reference library itself (oracle/_ref/ref_flowed, built from the reference's
sources: the flow, its inverse, the flowed action and log-determinant, the
force with and without the determinant term on a seeded configuration) and
against the reference driver's golden log (examples-cpp/flowed-hmc/log)."""

import json
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_FLOWED = os.path.join(ROOT, "oracle", "_ref", "ref_flowed")
needs_ref = pytest.mark.skipif(not os.path.exists(REF_FLOWED), reason="oracle/_ref/ref_flowed not built")
TS = (4, 4, 4, 8)


def run_ref(out_dir, sigma=0.3, fi_seed="fi-seed", eps=0.1, eps2=-0.01, beta=2.31, c1=-0.331):
    env = dict(os.environ, q_verbose="-1", OMP_NUM_THREADS="4")
    r = subprocess.run([REF_FLOWED, str(out_dir), *map(str, TS), str(sigma), fi_seed, str(eps), str(eps2), str(beta),
                        str(c1)], capture_output=True, text=True, env=env, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    info = json.loads([ln for ln in r.stdout.splitlines() if ln.startswith("{\"steps\"")][-1])
    load = lambda name: np.fromfile(os.path.join(out_dir, name), dtype=np.complex128).reshape(-1, 4, 3, 3)  # noqa
    return info, load


def nrel(a, b):
    return float(np.linalg.norm((a - b).ravel()) / np.linalg.norm(b.ravel()))


@needs_ref
def test_flow_info_matches_reference(tmp_path):
    import qlat_b200 as q
    info, _ = run_ref(tmp_path)
    fi = q.mk_flow_info_step(q.RngState("fi-seed"), 0.1, -0.01)
    got = [[s.mask, s.mu, s.epsilon, s.flow_size] for s in fi.v]
    assert got == info["steps"]
    one = q.mk_flow_info_step(q.RngState("fi-seed"), 0.1)
    assert sorted((s.mask, s.mu) for s in one.v) == sorted((m, mu) for m in (1, 2) for mu in range(4))


@pytest.mark.gpu
@needs_ref
def test_flow_stages_match_reference(q, tmp_path):
    info, load = run_ref(tmp_path)
    fi = q.FlowInfo(q.FlowStepInfo(*s) for s in info["steps"])
    gf0 = q.GaugeField(q.Geometry(TS))
    gf0.from_numpy(load("gf0.bin"))
    # the flow and its inverse
    assert nrel(np.asarray(q.gf_flow(gf0, fi)), load("flow.bin")) < 1e-13
    assert nrel(np.asarray(q.gf_flow_inv(gf0, fi)), load("flow_inv.bin")) < 1e-13
    # inverse then flow returns the field (the reverse test of main.cpp:run_hmc)
    back = q.gf_flow(q.gf_flow_inv(gf0, fi), fi)
    assert nrel(np.asarray(back), np.asarray(gf0)) < 1e-13
    # flowed action and the Jacobian's log-determinant
    ga = q.GaugeAction(2.31, -0.331)
    act, ld = q.gf_hamilton_flowed(gf0, ga, fi)
    assert abs(act - info["flowed_action"]) < 1e-12 * abs(info["flowed_action"])
    assert abs(ld - info["ln_det"]) < 1e-12 * abs(info["ln_det"])
    # force: propagated back without and with the determinant term
    F = q.GaugeMomentum(gf0.geo)
    q.set_gm_force_flowed(F, gf0, ga, fi, with_det=False)
    assert nrel(np.asarray(F), load("force_no_det.bin")) < 1e-12
    q.set_gm_force_flowed(F, gf0, ga, fi)
    assert nrel(np.asarray(F), load("force.bin")) < 1e-12


@pytest.mark.gpu
def test_flowed_force_is_minus_half_gradient_of_action(q):
    """dS/dw along a random su(3) direction X (U -> exp(w X) U) equals
    -2 <F, X> for the flowed action S = S(flow(U)) - ln det (4-point finite
    differences, h = 1e-4)."""
    gf0 = q.GaugeField(q.Geometry(TS))
    gf0.set_rand(q.RngState("flowed-fd").split("gf-init"), 0.3, 1)
    fi = q.mk_flow_info_step(q.RngState("flowed-fd-fi"), 0.1, -0.01)
    ga = q.GaugeAction(2.31, -0.331)
    F = q.GaugeMomentum(gf0.geo)
    q.set_gm_force_flowed(F, gf0, ga, fi)
    Fn = np.asarray(F)
    for k in range(3):
        X = q.GaugeMomentum(gf0.geo)
        X.set_rand(q.RngState(f"flowed-fd-dir-{k}"), 1.0)

        def S(h):
            u = gf0.copy()
            q.gf_evolve(u, X, h)
            return q.gf_hamilton_flowed_node(u, ga, fi)

        h = 1e-4
        fd = (8 * (S(h) - S(-h)) - (S(2 * h) - S(-2 * h))) / (12 * h)
        an = -2.0 * float(-0.5 * np.einsum("smij,smji->", Fn, np.asarray(X)).real)
        assert abs(fd - an) < 1e-6 * abs(fd), (k, fd, an)


@pytest.mark.gpu
def test_flowed_hmc_reference_log(q, goldens):
    """examples-cpp/flowed-hmc/main.cpp: 4^3 x 8, Iwasaki beta = 2.31, hot start
    set_g_rand_color_matrix_field(RngState(), 1.0), three trajectories of 6
    force-gradient steps with the flow mk_flow_info_step(rs, 0.1, -0.01); the
    plaquette after each."""
    g = goldens["cpp_flowed_hmc"]
    ga = q.GaugeAction(g["beta"], g["c1"])
    gf = q.GaugeField(q.Geometry(tuple(g["total_site"])))
    gf.set_unit()
    gf.set_rand(q.RngState(), 1.0, 1)
    rs = q.RngState("test_hmc-4x4x4x8")
    wl = {t: w for t, _, w in goldens["py_hmc_flowed_test"]["rows"]}
    for traj, plaq_ref, _ in g["rows"]:
        q.run_flowed_hmc(gf, ga, traj, rs.split(f"hmc-{traj}"))
        p = q.gf_avg_plaq(gf)
        assert abs(p - plaq_ref) <= 1e-11 * abs(plaq_ref), (traj, p, plaq_ref)
        # examples-py/hmc-pure-gauge-flowed-test.py: the same chain, with the 1 x 1 Wilson loop
        w = q.gf_avg_wilson_loop_normalized_tr(gf, 1, 1)
        assert abs(w - wl[traj]) <= 1e-10 * abs(wl[traj]), (traj, w, wl[traj])
