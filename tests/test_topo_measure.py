"""Topology measurement along flows: the plaquette field, the clover
plaquette-action densities, the plaquette-weighted flows of gf_flow_topo
(instanton_map.py:91-191), field min / max / per-timeslice sums, and the
smear_measure_topo driver (instanton_map.py:1327-1569).

CPU: the oracle against the reference's golden logs (examples-py/gf-flow-topo
and the gf_flow_topo entries of examples-py/flow-and-smear), including the
random-projection signatures of the fields (get_data_sig_arr,
qlat_utils/utils.py:436-451, rng_state.pyx:161-183, field_base.pyx:111-150).
GPU: the library against the oracle and the same goldens, and
smear_measure_topo against a replica of the driver on the oracle.
"""

import math

import numpy as np
import pytest

TS = (4, 4, 4, 8)
FLOW_KINDS = ["Wilson", "Iwasaki", "DBW2", "Freeze", "Shrink", "Localize", "Preserve"]


def data_sig_arr(o, arr, n_per_site, rs, k=3, ts=TS):
    """get_data_sig_arr of a field: per i, sum of the data times a uniform
    [-1, 1) field drawn from rs.split(str(i)) (one draw per number of a site)."""
    V = o.volume(ts)
    out = []
    for i in range(k):
        fu = np.zeros((V, n_per_site))
        o.field_set_u_rand(fu, ts, rs.split(f"{i}"), 1.0, -1.0)
        out.append((np.asarray(arr).reshape(V, n_per_site) * fu).sum())
    return out


def close(a, b, eps):
    if isinstance(b, list):
        return all(close(x, y, eps) for x, y in zip(a, b))
    return abs(complex(a) - complex(b)) <= eps * max(abs(complex(b)), 1e-300)


def _golden_value(v):
    if isinstance(v, list):
        return [complex(x[0], x[1]) if isinstance(x, list) else x for x in v]
    return v


def flow_topo_records(o, flow_step, plaq_field_of, gf, as_numpy):
    """The measurement sequence of gf-flow-topo.py on a gauge field, with the
    given flow step and plaquette field (oracle or library)."""
    rs_sig = o.RngState()
    out = []

    def rec():
        fp = np.asarray(plaq_field_of(gf))
        out.append(("gf plaq", fp.sum() / o.volume(TS) / 6))
        out.append(("gf plaq_min", fp.min()))
        out.append(("gf_sig", data_sig_arr(o, as_numpy(gf).reshape(-1, 36), 36, rs_sig)))
        out.append(("plaq_sig", data_sig_arr(o, fp, 6, rs_sig)))

    rec()
    ft = 0.0
    for kind in [None, "Freeze", "Shrink", "Localize", "Preserve"]:
        for _ in range(5):
            ft += flow_step(gf, kind)
        out.append(("flow_time", ft))
        rec()
    return out


def check_records(got, rows, eps):
    assert len(got) == len(rows)
    for (name, v), (gname, gv) in zip(got, rows):
        assert name == gname
        assert close(v, _golden_value(gv), eps), (name, v, gv)


def test_oracle_gf_flow_topo_log(oracle, goldens):
    o = oracle
    g = goldens["gf_flow_topo"]
    gf = o.new_field(TS)
    o.gf_set_rand(gf, TS, o.RngState("seed").split("gf-init"), 0.5, 10)
    got = flow_topo_records(o, lambda u, k: o.gf_flow_topo(u, TS, 0.1, k), lambda u: o.gf_plaq_field(u, TS), gf,
                            lambda u: u)
    check_records(got, g["rows"], 1e-13)


def test_oracle_flow_and_smear_flow_topo(oracle, goldens):
    o = oracle
    gold = goldens["flow"]["flow_topo"]
    gf0 = o.new_field(TS)
    o.gf_set_rand(gf0, TS, o.RngState("seed").split("gf-init"), 0.5, 10)
    cases = [(k, k, "euler") for k in FLOW_KINDS] + [(f"c1={c1}", c1, "euler") for c1 in (0.0, -0.331, -1.4008)]
    cases += [("Wilson euler", "Wilson", "euler"), ("Wilson runge-kutta", "Wilson", "runge-kutta")]
    for name, kind, integ in cases:
        gf = gf0.copy()
        for _ in range(3):
            o.gf_flow_topo(gf, TS, 0.1, kind, integ)
        assert abs(o.gf_avg_plaq(gf, TS) - gold[name]) < 1e-13 * abs(gold[name]) + 1e-15, name


def test_oracle_plaq_action_density_sum_rule(oracle):
    """Summed over the lattice, the clover plaquette-action density is
    6 V (1 - average plaquette): every plaquette enters four clovers with
    weight 1/4."""
    o = oracle
    gf = o.new_field(TS)
    o.gf_set_rand(gf, TS, o.RngState("paf").split("gf-init"), 0.4, 2)
    V = o.volume(TS)
    paf = o.clf_plaq_action_density_field(gf, TS)
    assert abs(paf.sum() - 6 * V * (1 - o.gf_avg_plaq(gf, TS))) < 1e-11 * paf.sum()
    fp = o.gf_plaq_field(gf, TS)
    assert abs(fp.mean() - o.gf_avg_plaq(gf, TS)) < 1e-14


# ---- GPU --------------------------------------------------------------------------------


def _gf(q, o, seed="seed", sigma=0.5, n_step=10):
    gf = q.GaugeField(q.Geometry(TS))
    gf.set_rand(q.RngState(seed).split("gf-init"), sigma, n_step)
    ref = o.new_field(TS)
    o.gf_set_rand(ref, TS, o.RngState(seed).split("gf-init"), sigma, n_step)
    return gf, ref


@pytest.mark.gpu
def test_gpu_site_fields_and_reductions(q, oracle):
    o = oracle
    gf, ref = _gf(q, o, "sites", 0.4, 2)
    fp = q.gf_plaq_field(gf)
    ref_fp = o.gf_plaq_field(ref, TS)
    assert np.abs(fp.to_numpy() - ref_fp).max() < 1e-14
    for spatial, fn in ((False, q.gf_plaq_action_density_field), (True, q.gf_spatial_plaq_action_density_field)):
        assert np.abs(fn(gf).to_numpy()[:, 0] - o.clf_plaq_action_density_field(ref, TS, spatial)).max() < 1e-13
    assert abs(q.gf_plaq_action_density(gf) - o.clf_plaq_action_density_field(ref, TS).mean()) < 1e-13
    # reductions of a real field with several components
    a = fp.to_numpy()
    assert np.array_equal(fp.glb_min(), a.min(axis=0, keepdims=True))
    assert np.array_equal(fp.glb_max(), a.max(axis=0, keepdims=True))
    for t_dir in range(4):
        ts = fp.glb_sum_tslice(t_dir=t_dir)
        xg = q.Geometry(TS).xg_arr()
        want = np.stack([a[xg[:, t_dir] == t].sum(axis=0) for t in range(TS[t_dir])])
        assert np.abs(ts - want).max() < 1e-12
    assert np.abs(fp.glb_sum() - a.sum(axis=0, keepdims=True)).max() < 1e-11
    from qlat_b200.topo_measure import field_abs
    neg = q.FieldRealD(q.Geometry(TS), 6)
    neg.from_numpy(a - 0.5)
    assert np.array_equal(field_abs(neg).to_numpy(), np.abs(a - 0.5))


@pytest.mark.gpu
def test_gpu_plaq_flow_force_matches_oracle(q, oracle):
    o = oracle
    gf, ref = _gf(q, o, "pff", 0.4, 2)
    rng = np.random.default_rng(3)
    factor = rng.random((o.volume(TS), 6)) + 0.5
    pf = q.FieldRealD(q.Geometry(TS), 6)
    pf.from_numpy(factor)
    z = q.gf_plaq_flow_force(gf, pf)
    zr = o.set_plaq_flow_z(ref, factor, TS)
    assert np.abs(np.asarray(z) - zr).max() < 1e-13
    # unit factors: the Wilson-flow force
    pf.from_numpy(np.ones_like(factor))
    z1 = q.gf_plaq_flow_force(gf, pf)
    assert np.abs(np.asarray(z1) - np.asarray(q.gf_wilson_flow_force(gf, 0.0))).max() < 1e-13


@pytest.mark.gpu
def test_gpu_gf_flow_topo_kinds(q, oracle, goldens):
    """Each flow kind, three steps of 0.1, against the oracle and the
    flow-and-smear golden."""
    o = oracle
    gold = goldens["flow"]["flow_topo"]
    gf0, ref0 = _gf(q, o)
    for kind in FLOW_KINDS:
        gf, ref = gf0.copy(), ref0.copy()
        adv = [q.gf_flow_topo(gf, 0.1, kind) for _ in range(3)]
        adv_ref = [o.gf_flow_topo(ref, TS, 0.1, kind) for _ in range(3)]
        assert np.allclose(adv, adv_ref, rtol=1e-13, atol=0), kind
        assert np.abs(np.asarray(gf) - ref).max() < 1e-12, kind
        assert abs(gf.plaq() - gold[kind]) < 1e-12 * abs(gold[kind]) + 1e-15, kind
    gf = gf0.copy()
    for _ in range(3):
        q.gf_flow_topo(gf, 0.1, "Wilson", "runge-kutta")
    assert abs(gf.plaq() - gold["Wilson runge-kutta"]) < 1e-12


@pytest.mark.gpu
def test_gpu_gf_flow_topo_log(q, oracle, goldens):
    """gf-flow-topo.py on the GPU: plaquette, its minimum, the flow time and the
    signatures of the gauge and plaquette fields after each stage."""
    o = oracle
    gf, _ = _gf(q, o)
    got = flow_topo_records(o, lambda u, k: q.gf_flow_topo(u, 0.1, k), q.gf_plaq_field, gf,
                            lambda u: np.asarray(u))
    check_records(got, goldens["gf_flow_topo"]["rows"], 1e-10)


def oracle_smear_measure_topo(o, gf, smear_info_list, energy_derivative_info):
    """smear_measure_topo (instanton_map.py:1327-1569) on the oracle."""
    V = o.volume(TS)
    T = TS[3]
    sv = V / T
    t_of = np.arange(V) // (TS[0] * TS[1] * TS[2])
    ts_sum = lambda f: np.array([f[t_of == t].sum() for t in range(T)])  # noqa: E731
    state = {"t": 0.0}
    topo_list, energy_list = [], []

    def flow(u, eps, kind, integ):
        return o.gf_flow_topo(u, TS, eps, kind, integ)

    def measure():
        fp = o.gf_plaq_field(gf, TS)
        ed = o.gf_energy_density_field(gf, TS)
        topo = o.clf_topology_field_5_terms(gf, TS).sum(axis=1)
        tclf = o.clf_topology_field(gf, TS)
        eps, kind, integ = energy_derivative_info
        g1 = gf.copy()
        flow(g1, eps, kind, integ)
        e1 = o.gf_energy_density_field(g1, TS)
        g1 = gf.copy()
        flow(g1, -eps, kind, integ)
        edd = (e1 - o.gf_energy_density_field(g1, TS)) * (1 / (2 * eps))
        paf = o.clf_plaq_action_density_field(gf, TS)
        topo_list.append({
            "flow_time": state["t"], "plaq": o.gf_avg_plaq(gf, TS), "plaq_min": fp.min(), "plaq_max": fp.max(),
            "energy_density": ed.sum() / V, "energy_density_tslice": ts_sum(ed) / sv,
            "energy_deriv": edd.sum() / V, "energy_deriv_tslice": ts_sum(edd) / sv,
            "topo": topo.sum(), "topo_tslice": ts_sum(topo), "topo_clf": tclf.sum(), "topo_clf_tslice": ts_sum(tclf),
            "abs_topo": np.abs(topo).sum(), "abs_topo_tslice": ts_sum(np.abs(topo)),
            "plaq_action_density": paf.sum() / V, "plaq_action_density_tslice": ts_sum(paf) / sv,
        })

    measure()
    for step, n, kind, integ in smear_info_list:
        target = state["t"] + n * step
        while state["t"] < target - step / 3:
            state["t"] += flow(gf, step, kind, integ)
            fp = o.gf_plaq_field(gf, TS)
            ed = o.gf_energy_density_field(gf, TS)
            energy_list.append({"flow_time": state["t"], "plaq": o.gf_avg_plaq(gf, TS), "plaq_min": fp.min(),
                                "plaq_max": fp.max(), "energy_density": ed.sum() / V,
                                "energy_density_tslice": ts_sum(ed) / sv})
        measure()
    return topo_list, energy_list


@pytest.mark.gpu
def test_gpu_smear_measure_topo_matches_oracle(q, oracle, tmp_path):
    o = oracle
    gf, ref = _gf(q, o, "smt", 0.3, 4)
    info = [[0.05, 4, "Wilson", "euler"], [0.1, 3, "Localize", "euler"], [0.05, 2, "Iwasaki", "runge-kutta"],
            [0.1, 2, "Freeze", "euler"]]
    edi = [0.0125, 0.0, "euler"]
    topo, energy = q.smear_measure_topo(gf, info, energy_derivative_info=edi, info_path=str(tmp_path / "info"),
                                        density_field_path=str(tmp_path / "df"))
    topo_r, energy_r = oracle_smear_measure_topo(o, ref, info, edi)
    assert len(topo) == len(topo_r) == len(info) + 1 and len(energy) == len(energy_r)
    for a, b in list(zip(topo, topo_r)) + list(zip(energy, energy_r)):
        assert set(a) == set(b)
        for k in a:
            va, vb = np.asarray(a[k], dtype=float), np.asarray(b[k], dtype=float)
            scale = max(float(np.abs(vb).max()), 1e-3)
            assert np.abs(va - vb).max() <= 1e-10 * scale, (k, va, vb)
    assert (tmp_path / "info" / "info.pickle").exists()
    assert (tmp_path / "df" / "smear-step-0" / "topo.npy").exists()
    assert math.isclose(topo[-1]["flow_time"], topo_r[-1]["flow_time"], rel_tol=1e-13)


@pytest.mark.gpu
def test_gpu_odd_lattice(q, oracle):
    """3x4x5x6 (V = 360, padded 32-site blocks, odd extents): plaquette field,
    action densities, weighted flow step and per-timeslice sums."""
    o = oracle
    ts = (3, 4, 5, 6)
    gf = q.GaugeField(q.Geometry(ts))
    gf.set_rand(q.RngState("odd").split("gf-init"), 0.4, 2)
    ref = o.new_field(ts)
    o.gf_set_rand(ref, ts, o.RngState("odd").split("gf-init"), 0.4, 2)
    fp = q.gf_plaq_field(gf)
    assert np.abs(fp.to_numpy() - o.gf_plaq_field(ref, ts)).max() < 1e-14
    for spatial in (False, True):
        f = q.gf_spatial_plaq_action_density_field(gf) if spatial else q.gf_plaq_action_density_field(gf)
        assert np.abs(f.to_numpy()[:, 0] - o.clf_plaq_action_density_field(ref, ts, spatial)).max() < 1e-13
    a = fp.to_numpy()
    xg = q.Geometry(ts).xg_arr()
    for t_dir in range(4):
        want = np.stack([a[xg[:, t_dir] == t].sum(axis=0) for t in range(ts[t_dir])])
        assert np.abs(fp.glb_sum_tslice(t_dir=t_dir) - want).max() < 1e-12
    assert np.array_equal(fp.glb_min(), a.min(axis=0, keepdims=True))
    for kind in ("Localize", "Shrink"):
        g, r = gf.copy(), ref.copy()
        adv = q.gf_flow_topo(g, 0.1, kind)
        assert abs(adv - o.gf_flow_topo(r, ts, 0.1, kind)) < 1e-13 * adv
        assert np.abs(np.asarray(g) - r).max() < 1e-12, kind


def test_oracle_energy_density_dir_sums_to_density(oracle):
    o = oracle
    gf = o.new_field(TS)
    o.gf_set_rand(gf, TS, o.RngState("edir").split("gf-init"), 0.4, 2)
    d = o.gf_energy_density_dir_field(gf, TS)
    assert np.abs(d.sum(axis=1) - o.gf_energy_density_field(gf, TS)).max() < 1e-13


@pytest.mark.gpu
def test_gpu_energy_density_dir_and_charge_5(q, oracle):
    o = oracle
    for ts in (TS, (3, 4, 5, 6)):
        gf = q.GaugeField(q.Geometry(ts))
        gf.set_rand(q.RngState("edir").split("gf-init"), 0.4, 2)
        ref = o.new_field(ts)
        o.gf_set_rand(ref, ts, o.RngState("edir").split("gf-init"), 0.4, 2)
        d = q.gf_energy_density_dir_field(gf).to_numpy()
        assert np.abs(d - o.gf_energy_density_dir_field(ref, ts)).max() < 1e-13
        assert np.abs(d.sum(axis=1) - q.gf_energy_density_field(gf).to_numpy()[:, 0]).max() < 1e-13
        assert q.topology_charge_5(gf) == q.gf_topology(gf)


def test_oracle_wilson_loop_1x1_is_the_timelike_plaquette(oracle):
    """gf_avg_wilson_loop(gf, 1, 1) averages the plaquettes of the planes (i, 3)."""
    o = oracle
    gf = o.new_field(TS)
    o.gf_set_rand(gf, TS, o.RngState("wl").split("gf-init"), 0.4, 2)
    fp = o.gf_plaq_field(gf, TS)
    assert abs(o.gf_avg_wilson_loop_normalized_tr(gf, TS, 1, 1) - fp[:, [2, 4, 5]].mean()) < 1e-14


@pytest.mark.gpu
def test_gpu_wilson_loops(q, oracle):
    o = oracle
    for ts in (TS, (3, 4, 5, 6)):
        gf = q.GaugeField(q.Geometry(ts))
        gf.set_rand(q.RngState("wl").split("gf-init"), 0.3, 2)
        ref = o.new_field(ts)
        o.gf_set_rand(ref, ts, o.RngState("wl").split("gf-init"), 0.3, 2)
        for l, t in ((1, 1), (1, 2), (2, 1), (2, 3)):
            a = q.gf_avg_wilson_loop_normalized_tr(gf, l, t)
            b = o.gf_avg_wilson_loop_normalized_tr(ref, ts, l, t)
            assert abs(a - b) < 1e-13, (ts, l, t, a, b)
