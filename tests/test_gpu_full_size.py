"""Checks at the benchmark's own size, 24^3 x 64 (884,736 sites, site indices
up to six digits in the per-site random streams), and at the gradient-flow
configuration's 32^4.

- The hot start and the momenta are bit-exact against the oracle (run with a
  correctly rounded log) on every site.
- The gauge action and the kinetic energy agree with the oracle to 1e-12.
- The FP64 trajectory is reversible: run backwards from its end it returns to
  its start (squared difference within 1e-12 of the field's squared norm, the
  bound of hmc.pyx:211), and delta_h changes sign.
- The mixed trajectory from the same state matches the FP64 one: plaquette
  within 1e-6, delta_h within 5% (plus 0.05) of the FP64 value.
- 32^4: one RK3 flow step matches the oracle (links 1e-13, energy density
  1e-12, clover charge 1e-9; with FP32 links 1e-6 and 1e-4).
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TS = (24, 24, 24, 64)
SEED = "b200-c2-24x64-iwasaki"
BETA, C1 = 2.13, -0.331


@pytest.fixture(scope="module")
def fields(q, oracle):
    rs = q.RngState(SEED)
    gf = q.GaugeField(q.Geometry(TS))
    gf.set_rand(rs.split("gf-init"), 0.3, 1)
    gm = q.GaugeMomentum(gf.geo)
    gm.set_rand(rs.split("1").split("set_rand_gauge_momentum"), 1.0)
    ors = oracle.RngState(SEED)
    ogf, ogm = oracle.new_field(TS), oracle.new_field(TS)
    oracle.set_log_mode(1)
    try:
        oracle.gf_set_rand(ogf, TS, ors.split("gf-init"), 0.3, 1)
        oracle.set_rand_gauge_momentum(ogm, TS, ors.split("1").split("set_rand_gauge_momentum"), 1.0)
    finally:
        oracle.set_log_mode(0)
    return gf, gm, ogf, ogm


def test_random_fields_bit_exact_at_full_size(q, fields):
    gf, gm, ogf, ogm = fields
    assert np.array_equal(np.asarray(gf).view(np.uint64), ogf.view(np.uint64))
    assert np.array_equal(np.asarray(gm).view(np.uint64), ogm.view(np.uint64))
    assert q.rng_ambiguous_count() == 0


def test_hamiltonians_at_full_size(q, oracle, fields):
    gf, gm, ogf, ogm = fields
    ga = q.GaugeAction(BETA, C1)
    hg, og = q.gf_hamilton_node(gf, ga), oracle.gf_hamilton_node(ogf, TS, BETA, C1)
    hm, om = q.gm_hamilton_node(gm), oracle.gm_hamilton_node(ogm, TS)
    assert abs(hg - og) <= 1e-12 * abs(og)
    assert abs(hm - om) <= 1e-12 * abs(om)


def test_trajectory_properties_at_full_size(q, fields):
    gf, gm, _, _ = fields
    ga = q.GaugeAction(BETA, C1)
    # FP64: forward, then backward from the end with the same momenta
    g64, m64 = gf.copy(), gm.copy()
    dh = q.run_hmc_evolve_pure_gauge(m64, g64, ga, None, 8, 1.0)
    g_r, m_r = g64.copy(), m64.copy()
    dh_rev = q.run_hmc_evolve_pure_gauge(m_r, g_r, ga, None, 8, -1.0)
    g_r -= gf
    assert g_r.qnorm() <= 1e-12 * gf.qnorm()  # the bound of hmc.pyx:211 (squared norms)
    assert abs(dh + dh_rev) <= 1e-6 * max(1.0, abs(dh))
    # mixed from the same state
    g32, m32 = gf.copy(), gm.copy()
    dh32 = q.run_hmc_evolve_pure_gauge(m32, g32, ga, None, 8, 1.0, precision="mixed", reunit_interval=4)
    assert abs(q.gf_avg_plaq(g32) - q.gf_avg_plaq(g64)) < 1e-6
    assert abs(dh32 - dh) <= 0.05 * abs(dh) + 0.05


def test_flow_at_full_size(q, oracle):
    """The gradient-flow configuration's lattice, 32^4: after one RK3 step
    (eps = 0.05, Wilson flow) from the seeded hot start, the links, the
    energy density and the clover charge agree with the oracle, in FP64 and
    (to FP32 accuracy) with FP32 links."""
    ts = (32, 32, 32, 32)
    rs = "b200-c3-32x32-flow"
    gf = q.GaugeField(q.Geometry(ts))
    gf.set_rand(q.RngState(rs).split("gf-init"), 0.5, 1)
    g32 = gf.copy(precision=q.F32)
    ogf = oracle.new_field(ts)
    oracle.set_log_mode(1)
    try:
        oracle.gf_set_rand(ogf, ts, oracle.RngState(rs).split("gf-init"), 0.5, 1)
    finally:
        oracle.set_log_mode(0)
    q.gf_wilson_flow_step(gf, 0.05, c1=0.0)
    q.gf_wilson_flow_step(g32, 0.05, c1=0.0)
    oracle.gf_wilson_flow_step(ogf, ts, 0.05, 0.0)
    got = np.asarray(gf)
    assert float(np.linalg.norm((got - ogf).ravel()) / np.linalg.norm(ogf.ravel())) < 1e-13
    e, oe = q.gf_energy_density(gf), oracle.gf_energy_density(ogf, ts)
    assert abs(e - oe) <= 1e-12 * abs(oe)
    qc, oq = q.gf_topology_clf(gf), oracle.gf_topology_clf(ogf, ts)
    assert abs(qc - oq) <= 1e-9
    assert abs(q.gf_energy_density(g32) - oe) <= 1e-6 * abs(oe)
    assert abs(q.gf_topology_clf(g32) - oq) <= 1e-4
