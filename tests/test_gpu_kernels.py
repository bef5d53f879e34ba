"""Parity of each CUDA kernel with the CPU oracle, through the C ABI.

FP64 bar: bit-exact for the random fields (hot start, momenta) against the
oracle run with a correctly rounded log; 1e-13 normwise for force, evolve and
flow fields; 1e-12 relative for the reductions.  FP32 storage: 2e-6 normwise.
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GEOS = [(4, 4, 4, 8), (3, 4, 5, 6)]
ACTIONS = [(5.5, 0.0), (2.13, -0.331), (0.9, -1.4008)]


def nrel(a, b):
    return float(np.linalg.norm((a - b).ravel()) / np.linalg.norm(b.ravel()))


def hot_start(q, oracle, ts, seed="gpu-kernels", sigma=0.5, n_step=3):
    rs = q.RngState(seed).split("gf-init")
    gf = q.GaugeField(q.Geometry(ts))
    gf.set_rand(rs, sigma, n_step)
    ref = oracle.new_field(ts)
    oracle.set_log_mode(1)
    oracle.gf_set_rand(ref, ts, oracle.RngState(seed).split("gf-init"), sigma, n_step)
    oracle.set_log_mode(0)
    return gf, ref


@pytest.mark.parametrize("ts", GEOS)
def test_hot_start_bit_exact(q, oracle, ts):
    gf, ref = hot_start(q, oracle, ts)
    got = np.asarray(gf)
    assert got.shape == ref.shape
    assert np.array_equal(got.view(np.uint64), ref.view(np.uint64))
    # against the C library's log: identical except where glibc's log is not
    # correctly rounded, and then only in the last bits
    ref_libm = oracle.new_field(ts)
    oracle.gf_set_rand(ref_libm, ts, oracle.RngState("gpu-kernels").split("gf-init"), 0.5, 3)
    assert nrel(got, ref_libm) < 1e-14
    assert q.rng_ambiguous_count() == 0


@pytest.mark.parametrize("ts", GEOS)
def test_momentum_bit_exact(q, oracle, ts):
    rs = q.RngState("traj-7").split("set_rand_gauge_momentum")
    gm = q.GaugeMomentum(q.Geometry(ts))
    gm.set_rand(rs, 1.0)
    ref = oracle.new_field(ts)
    oracle.set_log_mode(1)
    oracle.set_rand_gauge_momentum(ref, ts, oracle.RngState("traj-7").split("set_rand_gauge_momentum"), 1.0)
    oracle.set_log_mode(0)
    got = np.asarray(gm)
    assert np.array_equal(got.view(np.uint64), ref.view(np.uint64))
    ref_libm = oracle.new_field(ts)
    oracle.set_rand_gauge_momentum(ref_libm, ts, oracle.RngState("traj-7").split("set_rand_gauge_momentum"), 1.0)
    diff = got != ref_libm
    assert diff.mean() < 0.01
    assert nrel(got, ref_libm) < 1e-15
    # gm_hamilton_node on the same momenta
    h = q.gm_hamilton_node(gm)
    assert abs(h - oracle.gm_hamilton_node(ref, ts)) <= 1e-12 * abs(h)


@pytest.mark.parametrize("ts", GEOS)
@pytest.mark.parametrize("beta,c1", ACTIONS)
def test_set_gm_force(q, oracle, ts, beta, c1):
    gf, ref = hot_start(q, oracle, ts)
    F = q.GaugeMomentum(gf.geo)
    q.set_gm_force(F, gf, q.GaugeAction(beta, c1))
    Fr = oracle.new_field(ts)
    oracle.set_gm_force(Fr, ref, ts, beta, c1)
    assert nrel(np.asarray(F), Fr) < 1e-13


@pytest.mark.parametrize("ts", GEOS)
@pytest.mark.parametrize("beta,c1", ACTIONS)
def test_hamiltonians_and_plaquette(q, oracle, ts, beta, c1):
    gf, ref = hot_start(q, oracle, ts)
    ga = q.GaugeAction(beta, c1)
    h = q.gf_hamilton_node(gf, ga)
    hr = oracle.gf_hamilton_node(ref, ts, beta, c1)
    assert abs(h - hr) <= 1e-12 * abs(hr)
    sp = q.gf_sum_re_tr_plaq_node_no_comm(gf)
    assert abs(sp - oracle.gf_sum_re_tr_plaq(ref, ts)) <= 1e-12 * abs(sp)
    sr = q.gf_sum_re_tr_rect_node_no_comm(gf)
    assert abs(sr - oracle.gf_sum_re_tr_rect(ref, ts)) <= 1e-12 * abs(sr)
    p = q.gf_avg_plaq(gf)
    assert abs(p - oracle.gf_avg_plaq(ref, ts)) <= 1e-13


@pytest.mark.parametrize("ts", GEOS)
@pytest.mark.parametrize("step", [0.1, -0.37, 0.9])
def test_gf_evolve(q, oracle, ts, step):
    gf, ref = hot_start(q, oracle, ts)
    gm = q.GaugeMomentum(gf.geo)
    gm.set_rand(q.RngState("mom"), 1.0)
    gmr = np.asarray(gm)
    q.gf_evolve(gf, gm, step)
    oracle.gf_evolve(ref, np.ascontiguousarray(gmr), ts, step)
    assert nrel(np.asarray(gf), ref) < 1e-13


def test_unitarize(q, oracle):
    ts = (4, 4, 4, 4)
    gf, ref = hot_start(q, oracle, ts)
    rng = np.random.default_rng(3)
    noisy = ref + 1e-3 * (rng.standard_normal(ref.shape) + 1j * rng.standard_normal(ref.shape))
    gf.from_numpy(noisy)
    gf.unitarize()
    r = np.ascontiguousarray(noisy)
    oracle.unitarize(r, ts)
    assert nrel(np.asarray(gf), r) < 1e-14


@pytest.mark.parametrize("ts", GEOS)
@pytest.mark.parametrize("c1", [0.0, -0.331])
@pytest.mark.parametrize("integ", ["runge-kutta", "euler"])
def test_flow_step(q, oracle, ts, c1, integ):
    gf, ref = hot_start(q, oracle, ts)
    q.gf_wilson_flow_step(gf, 0.05, c1=c1, wilson_flow_integrator_type=integ)
    oracle.gf_wilson_flow_step(ref, ts, 0.05, c1, integ)
    assert nrel(np.asarray(gf), ref) < 1e-13


@pytest.mark.parametrize("ts", GEOS)
def test_energy_density_and_topology(q, oracle, ts):
    gf, ref = hot_start(q, oracle, ts)
    e = q.gf_energy_density(gf)
    assert abs(e - oracle.gf_energy_density(ref, ts)) <= 1e-12 * abs(e)
    ef = q.gf_energy_density_field(gf)
    assert nrel(np.asarray(ef)[:, 0], oracle.gf_energy_density_field(ref, ts)) < 1e-13
    qt = q.gf_topology_clf(gf)
    assert abs(qt - oracle.gf_topology_clf(ref, ts)) <= 1e-12 * max(1.0, abs(qt))
    tf = q.gf_topology_field_clf(gf)
    assert nrel(np.asarray(tf)[:, 0], oracle.clf_topology_field(ref, ts)) < 1e-12


@pytest.mark.parametrize("ts", GEOS)
def test_topology_5li(q, oracle, ts):
    """The five terms of the 5-loop improved charge per site, their per-site sum
    and the lattice sums (qcd.cpp:425-509) against the oracle."""
    gf, ref = hot_start(q, oracle, ts)
    terms_ref = oracle.clf_topology_field_5_terms(ref, ts)
    terms = np.asarray(q.gf_topology_terms_field(gf))
    assert terms.shape == terms_ref.shape
    assert np.abs(terms - terms_ref).max() <= 1e-12 * max(1.0, np.abs(terms_ref).max())
    tot = np.asarray(q.gf_topology_field(gf))[:, 0]
    assert np.abs(tot - terms_ref.sum(axis=1)).max() <= 1e-12 * max(1.0, np.abs(terms_ref).max())
    assert np.allclose(q.gf_topology_terms(gf), terms_ref.sum(axis=0), rtol=0, atol=1e-11)
    assert abs(q.gf_topology(gf) - oracle.gf_topology(ref, ts)) <= 1e-11


def test_fp32_storage(q, oracle):
    ts = (4, 4, 4, 8)
    gf, ref = hot_start(q, oracle, ts)
    g32 = gf.copy(precision=q.F32)
    F = q.GaugeMomentum(gf.geo, precision=q.F32)
    q.set_gm_force(F, g32, q.GaugeAction(2.13, -0.331))
    Fr = oracle.new_field(ts)
    oracle.set_gm_force(Fr, ref, ts, 2.13, -0.331)
    assert nrel(np.asarray(F), Fr) < 2e-6
    assert abs(q.gf_avg_plaq(g32) - oracle.gf_avg_plaq(ref, ts)) < 1e-6


def test_field_algebra(q):
    ts = (4, 4, 4, 4)
    geo = q.Geometry(ts)
    a = q.GaugeMomentum(geo)
    a.set_rand(q.RngState("a"), 1.0)
    b = q.GaugeMomentum(geo)
    b.set_rand(q.RngState("b"), 1.0)
    A, B = np.asarray(a), np.asarray(b)
    c = a.copy()
    c *= 0.25
    c += b
    c -= a
    assert np.allclose(np.asarray(c), 0.25 * A + B - A, rtol=0, atol=1e-14)
    assert abs(a.qnorm() - float(np.sum(np.abs(A) ** 2))) < 1e-10 * a.qnorm()


def test_errors_are_reported(q):
    geo = q.Geometry((4, 4, 4, 4))
    gf = q.GaugeField(geo)
    gm = q.GaugeMomentum(q.Geometry((4, 4, 4, 8)))
    with pytest.raises(q.QlatB200Error) as e:
        q.gf_evolve(gf, gm, 0.1)
    assert e.value.code == 7
    with pytest.raises(q.QlatB200Error):
        q.set_gm_force(gf, gf, q.GaugeAction(1.0, 0.0))


@pytest.mark.parametrize("prec", ["f64", "f32"])
@pytest.mark.parametrize("ts", [(3, 4, 5, 6), (4, 4, 4, 8), (8, 4, 2, 6)])
def test_every_force_variant(q, oracle, prec, ts):
    """All launch shapes of the autotuner compute the same force, on lattices
    whose site count is a multiple of 32 and not (3 x 4 x 5 x 6: a partly
    filled last block of 32 sites)."""
    gf, ref = hot_start(q, oracle, ts)
    g = gf if prec == "f64" else gf.copy(precision=q.F32)
    tol = 1e-13 if prec == "f64" else 2e-6
    Fr = {}
    for c1 in (0.0, -0.331):
        Fr[c1] = oracle.new_field(ts)
        oracle.set_gm_force(Fr[c1], ref, ts, 2.0, c1)
    P = q.F64 if prec == "f64" else q.F32
    saved = {rect: q.force_get_variant(P, rect) for rect in (False, True)}
    try:
        for v in range(len(q.force_variants())):
            for c1 in (0.0, -0.331):
                q.force_set_variant(P, c1 != 0.0, v)
                F = q.GaugeMomentum(gf.geo, precision=P)
                q.set_gm_force(F, g, q.GaugeAction(2.0, c1))
                assert nrel(np.asarray(F), Fr[c1]) < tol, (v, c1)
    finally:
        for rect, v in saved.items():
            q.force_set_variant(P, rect, v)


@pytest.mark.gpu
@pytest.mark.parametrize("c1", [-0.331, 0.0])
def test_force_shapes_agree_in_every_mode(q, c1):
    """The FP32 force shapes used by the mixed trajectory -- two-row chains
    (variant 10) and the corner field with its separate pass (14) -- give the
    same mixed trajectory (force + exponential, force + momentum update + link
    update) and the same FP32 flow stage, to FP32 rounding."""
    ts = (8, 4, 4, 8)
    ga = q.GaugeAction(2.13, c1)
    gf = q.GaugeField(q.Geometry(ts))
    gf.set_rand(q.RngState("shapes").split("gf-init"), 0.3, 1)
    gm = q.GaugeMomentum(gf.geo)
    gm.set_rand(q.RngState("shapes").split("mom"), 1.0)
    saved = q.force_get_variant(q.F32, c1 != 0.0)
    res = {}
    try:
        for v in (10, 14):
            q.force_set_variant(q.F32, c1 != 0.0, v)
            g, m = gf.copy(), gm.copy()
            dh = q.run_hmc_evolve_pure_gauge(m, g, ga, None, 4, 1.0, precision="mixed", reunit_interval=4)
            w = gf.copy(precision=q.F32)
            q.gf_wilson_flow_step(w, 0.05, c1=c1)
            res[v] = (dh, np.asarray(g), np.asarray(w))
    finally:
        q.force_set_variant(q.F32, c1 != 0.0, saved)
    for v in (14,):
        assert abs(res[v][0] - res[10][0]) < 1e-4 * max(1.0, abs(res[10][0])), (v, res[v][0], res[10][0])
        assert nrel(res[v][1], res[10][1]) < 1e-6, v
        assert nrel(res[v][2], res[10][2]) < 1e-6, v


@pytest.mark.gpu
def test_upload_pipelined(q):
    """qgb_field_upload_pipelined: each call leaves the field equal to host_now,
    whether it was prefetched by the call before or not (pinned and pageable
    buffers, changing buffers, FP64 and FP32 fields)."""
    import torch
    geo = q.Geometry((4, 4, 4, 8))
    V = geo.total_volume
    rng = np.random.default_rng(11)
    bufs = []
    for pinned in (True, True, False):
        t = torch.empty((V, 4, 3, 3), dtype=torch.complex128, pin_memory=pinned)
        t.numpy()[...] = rng.standard_normal((V, 4, 3, 3)) + 1j * rng.standard_normal((V, 4, 3, 3))
        bufs.append(t)
    for prec in (q.F64, q.F32):
        gf = q.GaugeField(geo, precision=prec)
        tol = 0 if prec == q.F64 else 1e-6
        order = [0, 1, 0, 2, 2, 1]
        for k, i in enumerate(order):
            nxt = bufs[order[k + 1]].data_ptr() if k + 1 < len(order) else None
            gf.upload_host_pipelined(bufs[i].data_ptr(), nxt)
            assert np.abs(np.asarray(gf) - bufs[i].numpy()).max() <= tol * 10, (prec, k)
        # a prefetch that is not committed next is dropped, not applied
        gf.upload_host_pipelined(bufs[0].data_ptr(), bufs[1].data_ptr())
        gf.upload_host_pipelined(bufs[2].data_ptr(), None)
        assert np.abs(np.asarray(gf) - bufs[2].numpy()).max() <= tol * 10


@pytest.mark.gpu
def test_download_async(q):
    """qgb_field_download_async: three queued downloads in a row (the third
    reuses the first's staging slot), FP64 and FP32 fields, into pinned host
    buffers, equal the synchronous download once qgb_synchronize returns, also
    when the field changes after a download was queued."""
    import torch
    geo = q.Geometry((4, 4, 4, 8))
    V = geo.total_volume
    fields = []
    for k, prec in enumerate((q.F64, q.F32, q.F64)):
        f = q.GaugeField(geo, precision=prec)
        f.set_rand(q.RngState(f"dl-{k}"), 0.5, 1)
        fields.append(f)
    expect = [np.asarray(f).copy() for f in fields]
    hosts = [torch.zeros((V, 4, 3, 3), dtype=torch.complex128, pin_memory=True) for _ in fields]
    for f, h in zip(fields, hosts):
        f.download_host_async(h.data_ptr())
    fields[0].set_rand(q.RngState("dl-changed"), 0.5, 1)  # queued after the first download
    q.synchronize()
    for e, h in zip(expect, hosts):
        assert np.array_equal(h.numpy(), e)


@pytest.mark.gpu
def test_field_storage_pool(q):
    """A destroyed field's storage is pooled and reused by the next field of
    its size, which still starts at zero; release_field_pool frees it."""
    geo = q.Geometry((4, 4, 4, 8))
    nbytes = 4 * 4 * 4 * 8 * 4 * 18 * 8  # 512 sites (a multiple of 32), 4 links, 18 doubles
    q.release_field_pool()
    f = q.GaugeField(geo)
    f.set_rand(q.RngState("pool"), 0.5, 1)
    del f
    g = q.GaugeField(geo)  # takes the pooled block
    assert not np.asarray(g).any()
    assert q.release_field_pool() == 0
    del g
    assert q.release_field_pool() == nbytes
    assert q.release_field_pool() == 0
