"""Batches of independent chains (qlat_b200.ChainBatch): every chain matches
the oracle's run_hmc_pure_gauge for its own lattice, beta, c1 and RngState,
and the CUDA-graph replay gives the same numbers as direct launches."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SITES = [(4, 4, 4, 4), (3, 4, 5, 6), (4, 4, 4, 6), (6, 6, 6, 6)]
BETAS = [5.6, 6.0, 2.13, 5.8]
C1S = [0.0, 0.0, -0.331, 0.0]


def make(q, precision_seed="batch"):
    b = q.ChainBatch(SITES, BETAS, C1S)
    rs = [q.RngState(f"{precision_seed}-{c}") for c in range(len(SITES))]
    b.set_rand([r.split("gf-init") for r in rs], 1.0, 1)
    return b, rs


def test_batch_hot_start_matches_oracle(q, oracle):
    b, rs = make(q)
    oracle.set_log_mode(1)
    try:
        for c, ts in enumerate(SITES):
            ref = oracle.new_field(ts)
            oracle.gf_set_rand(ref, ts, oracle.RngState(f"batch-{c}").split("gf-init"), 1.0, 1)
            assert np.array_equal(b.chain_to_numpy(c), ref)
    finally:
        oracle.set_log_mode(0)


@pytest.mark.parametrize("integrator", ["leapfrog", "force-gradient"])
def test_batch_chains_match_oracle(q, oracle, integrator):
    b, rs = make(q)
    oracle.set_log_mode(1)
    try:
        refs = []
        for c, ts in enumerate(SITES):
            ref = oracle.new_field(ts)
            oracle.gf_set_rand(ref, ts, oracle.RngState(f"batch-{c}").split("gf-init"), 1.0, 1)
            refs.append(ref)
        for traj in (1, 2):
            flags, dh = b.run_hmc(traj, rs, 6, integrator=integrator)
            plaq = b.plaq()
            for c, ts in enumerate(SITES):
                oflag, odh = oracle.run_hmc_pure_gauge(refs[c], ts, BETAS[c], C1S[c], traj,
                                                       oracle.RngState(f"batch-{c}"), n_step=6,
                                                       integrator=integrator)
                assert flags[c] == oflag, (traj, c)
                assert abs(dh[c] - odh) < 1e-9 * max(1.0, np.prod(ts) / 100), (traj, c, dh[c], odh)
                assert abs(plaq[c] - oracle.gf_avg_plaq(refs[c], ts)) < 1e-12, (traj, c)
    finally:
        oracle.set_log_mode(0)


def test_graph_replay_equals_direct_launches(q):
    b1, rs = make(q)
    b2, _ = make(q)
    for traj in (1, 2, 3):
        m = [r.split(f"{traj}").split("set_rand_gauge_momentum") for r in rs]
        d1 = b1.trajectory(m, 5, use_graph=True)
        d2 = b2.trajectory(m, 5, use_graph=False)
        assert np.array_equal(d1, d2)
        b1.accept([True] * len(SITES))
        b2.accept([True] * len(SITES))
    assert np.array_equal(b1.plaq(), b2.plaq())


def test_mixed_batch_close_to_fp64(q):
    b64, rs = make(q)
    b32, _ = make(q)
    m = [r.split("1").split("set_rand_gauge_momentum") for r in rs]
    d64 = b64.trajectory(m, 10, integrator="leapfrog")
    d32 = b32.trajectory(m, 10, integrator="leapfrog", precision="mixed")
    assert np.all(np.abs(d32 - d64) < 5e-3 * np.maximum(1.0, np.abs(d64)))


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_batch_force_shapes_agree(q, precision):
    """Every launch shape of the batched force (qgb_batch_autotune's table)
    gives the same trajectory; the autotuner keeps one of them.  The mixed
    form's leapfrog runs each step as one launch (odd and even step counts:
    the links end in either buffer)."""
    res = {}
    for v in range(4):
        for n_step in (5, 6):
            b, rs = make(q)
            b.set_force_variant(precision, v)
            m = [r.split("1").split("set_rand_gauge_momentum") for r in rs]
            dh = b.trajectory(m, n_step, integrator="leapfrog", precision=precision)
            b.accept([True] * len(SITES))
            res[(v, n_step)] = (dh, b.plaq())
    tol = 0.0 if precision == "fp64" else 1e-6
    for (v, n_step), (dh, plaq) in res.items():
        d0, p0 = res[(0, n_step)]
        assert np.all(np.abs(dh - d0) <= tol * np.maximum(1.0, np.abs(d0))), (v, n_step)
        assert np.all(np.abs(plaq - p0) <= tol), (v, n_step)
    b, _ = make(q)
    best, ms = b.autotune(precision, reps=2)
    assert 0 <= best < 4 and ms > 0


def test_batch_at_c5_size(q):
    """The 256-chain batch of the batched-chains workload (64 each of 4^4,
    6^4, 8^4, 12^4, Wilson, betas 5.6 .. 6.2, hot starts at scale 1, leapfrog
    of 10 steps): one chain of each size against the same chain run alone
    through run_hmc_pure_gauge (same decisions, delta_h, plaquette), and the
    mixed form's per-chain plaquettes against the FP64 form's."""
    sizes = [(L, L, L, L) for L in (4, 6, 8, 12) for _ in range(64)]
    betas = list(np.linspace(5.6, 6.2, len(sizes)))
    rs = [q.RngState("c5-size").split(f"chain-{c}") for c in range(len(sizes))]
    plaqs = {}
    for prec in ("fp64", "mixed"):
        b = q.ChainBatch(sizes, betas)
        b.set_rand([r.split("gf-init") for r in rs], 1.0, 1)
        rows = []
        for traj in (1, 2):
            flags, dh = b.run_hmc(traj, rs, 10, precision=prec, is_always_accept=traj < 2)
            rows.append((list(flags), np.array(dh), b.plaq()))
        plaqs[prec] = rows[-1][2]
        if prec != "fp64":
            continue
        for c in (0, 64, 128, 255):
            gf = q.GaugeField(q.Geometry(sizes[c]))
            gf.set_rand(rs[c].split("gf-init"), 1.0, 1)
            ga = q.GaugeAction(betas[c], 0.0)
            for traj in (1, 2):
                flag, dh = q.run_hmc_pure_gauge(gf, ga, traj, rs[c], n_step=10, integrator="leapfrog",
                                                is_always_accept=traj < 2)
                bflags, bdh, bplaq = rows[traj - 1]
                assert bool(bflags[c]) == bool(flag), (c, traj)
                assert abs(bdh[c] - dh) < 1e-9 * max(1.0, np.prod(sizes[c]) / 100), (c, traj, bdh[c], dh)
                assert abs(bplaq[c] - q.gf_avg_plaq(gf)) < 1e-12, (c, traj)
    assert np.abs(plaqs["mixed"] - plaqs["fp64"]).max() < 2e-5
