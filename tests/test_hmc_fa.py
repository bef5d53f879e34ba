"""Field-accelerated HMC (per-link masses, dual momenta, projection of the
gauge-transformation motion; hmc.cpp:121-201, 330-396, 492-645).

CPU: the oracle's restatement against the reference library itself
(oracle/_ref/ref_fa, built from the reference's sources), bit for bit; and an
oracle-driven replica of the reference's field-accelerated example
(examples-py/hmc-pure-gauge-fa-sym.py) against that example's golden log.
GPU: every library entry point against the oracle on seeded inputs, the
gauge-invariance property of set_gauge_transform_momentum, and the library's
trajectory driver (qlat_b200.run_hmc_fa) against the golden log.
"""

import json
import math
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_FA = os.path.join(ROOT, "oracle", "_ref", "ref_fa")
needs_ref = pytest.mark.skipif(not os.path.exists(REF_FA), reason="oracle/_ref/ref_fa not built")
TS = (4, 4, 4, 8)
SEED, DT, BETA, C1 = "fa-test", 0.1, 2.31, -0.331
# the golden log prints 16 digits; over 8 trajectories the trajectory-level
# rounding differences (FMA contraction, reduction order) grow to ~1e-13
GOLDEN_EPS = 1e-10


def seeded_inputs(o, ts=TS, seed=SEED):
    """The inputs ref_fa builds: a hot start, masses in [1, 4) with +inf on the
    links (site + 2 mu) % 7 == 3 (mf) / 5 (mf_dual), momenta drawn with them."""
    V = o.volume(ts)
    rs = o.RngState(seed)
    gf0 = o.new_field(ts)
    o.gf_set_rand(gf0, ts, rs.split("gf"), 0.3, 2)
    mf = np.zeros((V, 4))
    mfd = np.zeros((V, 4))
    o.field_set_u_rand(mf, ts, rs.split("mf"), 4.0, 1.0)
    o.field_set_u_rand(mfd, ts, rs.split("mfd"), 4.0, 1.0)
    i = np.arange(V)[:, None] + 2 * np.arange(4)[None, :]
    mf[i % 7 == 3] = np.inf
    mfd[i % 7 == 5] = np.inf
    gm = o.new_field(ts)
    gmd = o.new_field(ts)
    o.set_rand_gauge_momentum_fa(gm, mf, ts, rs.split("gm"))
    o.set_rand_gauge_momentum_fa(gmd, mfd, ts, rs.split("gmd"))
    return rs, gf0, mf, mfd, gm, gmd


@needs_ref
def test_oracle_matches_reference_library(oracle, tmp_path):
    o = oracle
    env = dict(os.environ, q_verbose="-1", OMP_NUM_THREADS="4")
    r = subprocess.run([REF_FA, str(tmp_path), *map(str, TS), SEED, str(DT), str(BETA), str(C1)],
                       capture_output=True, text=True, env=env, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    info = json.loads([ln for ln in r.stdout.splitlines() if ln.startswith('{"h_gm"')][-1])
    V = o.volume(TS)
    C = lambda n: np.fromfile(tmp_path / f"{n}.bin", dtype=np.complex128).reshape(V, -1, 3, 3)  # noqa: E731
    Rl = lambda n, m: np.fromfile(tmp_path / f"{n}.bin", dtype=np.float64).reshape(V, m)  # noqa: E731
    rs, gf0, mf, mfd, gm, gmd = seeded_inputs(o)
    assert np.array_equal(gf0, C("gf0"))
    assert np.array_equal(mf, Rl("mf", 4)) and np.array_equal(mfd, Rl("mfd", 4))
    assert np.array_equal(gm, C("gm")) and np.array_equal(gmd, C("gmd"))
    assert o.gm_hamilton_node_fa(gm, mf, TS) == info["h_gm"]
    assert o.gm_hamilton_node_fa(gmd, mfd, TS) == info["h_gmd"]
    gmp, gmdp = gm.copy(), gmd.copy()
    assert o.project_gauge_transform(gmp, gmdp, mf, mfd, TS) == info["change_qnorm"]
    assert np.array_equal(gmp, C("gm_proj")) and np.array_equal(gmdp, C("gmd_proj"))
    for name, fn in (("evolve_fa", lambda g: o.gf_evolve_fa(g, gm, mf, TS, DT)),
                     ("evolve_fa_dual", lambda g: o.gf_evolve_fa_dual(g, gmd, mfd, TS, DT)),
                     ("evolve_dual", lambda g: o.gf_evolve_dual(g, gmd, TS, DT))):
        g = gf0.copy()
        fn(g)
        assert np.array_equal(g, C(name)), name
    F = o.new_field(TS)
    o.set_gm_force(F, gf0, TS, BETA, C1)
    Fd = o.new_field(TS)
    o.set_gm_force_dual(Fd, gf0, F, TS)
    assert np.array_equal(Fd, C("force_dual"))
    gtm = np.ascontiguousarray(C("gtm")[:, :1])
    a, b = o.new_field(TS), o.new_field(TS)
    o.set_gauge_transform_momentum(a, b, gtm, TS)
    assert np.array_equal(a, C("gt_gm")) and np.array_equal(b, C("gt_gmd"))
    assert np.array_equal(o.dot_gauge_momentum(gm, gmd, TS), Rl("dot", 4))
    gr = np.zeros((V, 3))
    o.field_set_g_rand(gr, TS, rs.split("g"), 0.5, 2.0)
    assert np.array_equal(gr, Rl("grand", 3))


# ---- the example's driver on the oracle (hmc-pure-gauge-fa-sym.py:112-680) ----------


class OracleFa:
    """The reference example's trajectory logic over the oracle's arrays."""

    def __init__(self, o, params, job_seed):
        self.o = o
        self.p = params
        self.ts = tuple(params["total_site"])
        self.V = o.volume(self.ts)
        self.seed = job_seed

    def evolve(self, gf, gm, gmd, mf, mfd, dt):
        self.o.gf_evolve_fa(gf, gm, mf, self.ts, dt)
        self.o.gf_evolve_fa_dual(gf, gmd, mfd, self.ts, dt)

    def gm_evolve_fg(self, gm, gmd, gf_init, mf, mfd, fg_dt, dt, proj):
        o, ts, h = self.o, self.ts, self.p["hmc"]
        gf = gf_init.copy()
        F, Fd = o.new_field(ts), o.new_field(ts)
        o.set_gm_force(F, gf, ts, h["beta"], h["c1"])
        o.set_gm_force_dual(Fd, gf, F, ts)
        if proj:
            o.project_gauge_transform(F, Fd, mf, mfd, ts)
        self.evolve(gf, F, Fd, mf, mfd, fg_dt)
        o.set_gm_force(F, gf, ts, h["beta"], h["c1"])
        o.set_gm_force_dual(Fd, gf, F, ts)
        gm += F * dt
        gmd += Fd * dt
        if proj:
            o.project_gauge_transform(gm, gmd, mf, mfd, ts)

    def hamiltonian(self, gm, gmd, gf, mf, mfd):
        o, ts, h = self.o, self.ts, self.p["hmc"]
        return (o.gm_hamilton_node_fa(gm, mf, ts) + o.gm_hamilton_node_fa(gmd, mfd, ts)
                + o.gf_hamilton_node(gf, ts, h["beta"], h["c1"]))

    def run_hmc_evolve(self, gm, gmd, gf, mf, mfd, n_step, md_time, proj):
        energy = self.hamiltonian(gm, gmd, gf, mf, mfd)
        dt = md_time / n_step
        lam = 0.5 * (1.0 - 1.0 / math.sqrt(3.0))
        ttheta = (2.0 - math.sqrt(3.0)) / 48.0 * dt * dt * dt
        self.evolve(gf, gm, gmd, mf, mfd, lam * dt)
        for i in range(n_step):
            self.gm_evolve_fg(gm, gmd, gf, mf, mfd, 4.0 * ttheta / dt, 0.5 * dt, proj)
            self.evolve(gf, gm, gmd, mf, mfd, (1.0 - 2.0 * lam) * dt)
            self.gm_evolve_fg(gm, gmd, gf, mf, mfd, 4.0 * ttheta / dt, 0.5 * dt, proj)
            self.evolve(gf, gm, gmd, mf, mfd, (2.0 if i < n_step - 1 else 1.0) * lam * dt)
        self.o.unitarize(gf, self.ts)
        return self.hamiltonian(gm, gmd, gf, mf, mfd) - energy

    def refresh(self, traj, force, rs, st):
        o, ts, V = self.o, self.ts, self.V
        fa = self.p["hmc"]["fa"]
        proj = fa["is_project_gauge_transform"]
        cri = fa.get("complete_refresh_interval", 1)
        mass_type, mass_list, interval_list = fa.get("mass_type"), fa.get("mass_list"), fa.get("interval_list")
        rs = rs.split(f"{traj}")
        if traj % cri == 0 or force:
            if mass_type is None:
                st["mf"][:] = 1.0
                st["mfd"][:] = 1.0
                st["sel"] = [np.ones((V, 4), bool)]
                st["seld"] = st["sel"]
            elif mass_type == "random":
                o.field_set_u_rand(st["mf"], ts, rs.split("fa_mass"), 4.0, 1.0)
                o.field_set_u_rand(st["mfd"], ts, rs.split("fa_mass_dual"), 4.0, 1.0)
                s, sd = st["mf"] < 2.0, st["mfd"] < 2.0
                st["sel"], st["seld"] = [s, ~s], [sd, ~sd]
            else:
                ri = rs.rand_gen() % V
                off = []
                for n in ts:
                    off.append(ri % n)
                    ri //= n
                i = np.arange(V)
                xg = np.stack([i % ts[0], (i // ts[0]) % ts[1], (i // (ts[0] * ts[1])) % ts[2],
                               i // (ts[0] * ts[1] * ts[2])], axis=1) - np.array(off)
                count = np.zeros((V, 4), np.int32)
                for m in range(4):
                    for n in range(4):
                        if n != m:
                            count[xg[:, n] % 2 == 0, m] += 1
                if mass_type == "grid-2":
                    st["sel"] = [count == k for k in range(4)]
                    st["seld"] = st["sel"]
                else:
                    ev = (xg.sum(-1) % 2 == 0)[:, None]
                    st["sel"] = [(count == k) & ev for k in range(4)] + [(count == k) & ~ev for k in range(4)]
                    st["seld"] = [(count == k) & ~ev for k in range(4)] + [(count == k) & ev for k in range(4)]
                for idx, mass in enumerate(mass_list):
                    st["mf"][st["sel"][idx]] = mass
                    st["mfd"][st["seld"][idx]] = mass
            o.set_rand_gauge_momentum_fa(st["gm"], st["mf"], ts, rs.split("set_rand_gauge_momentum"))
            o.set_rand_gauge_momentum_fa(st["gmd"], st["mfd"], ts, rs.split("set_rand_gauge_momentum_dual"))
            if proj:
                o.project_gauge_transform(st["gm"], st["gmd"], st["mf"], st["mfd"], ts)
        else:
            gm1, gmd1 = o.new_field(ts), o.new_field(ts)
            if proj:
                o.set_rand_gauge_momentum_fa(gm1, st["mf"], ts, rs.split("set_rand_gauge_momentum_g"))
                o.set_rand_gauge_momentum_fa(gmd1, st["mfd"], ts, rs.split("set_rand_gauge_momentum_dual_g"))
                gm2, gmd2 = gm1.copy(), gmd1.copy()
                o.project_gauge_transform(gm2, gmd2, st["mf"], st["mfd"], ts)
                st["gm"] -= gm2 - gm1
                st["gmd"] -= gmd2 - gmd1
            o.set_rand_gauge_momentum_fa(gm1, st["mf"], ts, rs.split("set_rand_gauge_momentum"))
            o.set_rand_gauge_momentum_fa(gmd1, st["mfd"], ts, rs.split("set_rand_gauge_momentum_dual"))
            for sel, interval in zip(st["sel"], interval_list):
                if traj % interval == 0:
                    st["gm"][sel] = gm1[sel]
            for sel, interval in zip(st["seld"], interval_list):
                if traj % interval == 0:
                    st["gmd"][sel] = gmd1[sel]
            if proj:
                o.project_gauge_transform(st["gm"], st["gmd"], st["mf"], st["mfd"], ts)

    def run(self, n_traj):
        o, ts, h = self.o, self.ts, self.p["hmc"]
        proj = h["fa"]["is_project_gauge_transform"]
        rs = o.RngState(f"run_hmc-{self.seed}")
        gf = o.new_field(ts)
        o.gf_set_rand(gf, ts, rs.split("init"), 0.1, 2)
        st = {"mf": np.zeros((self.V, 4)), "mfd": np.zeros((self.V, 4)), "gm": o.new_field(ts),
              "gmd": o.new_field(ts)}
        plaqs = []
        for traj in range(n_traj):
            self.refresh(traj, traj == 0, rs.split("run_hmc_mass_mom_refresh"), st)
            traj += 1
            rt = rs.split("run_hmc_traj").split(f"{traj}")
            gf0, gm0, gmd0 = gf.copy(), st["gm"].copy(), st["gmd"].copy()
            if proj:
                o.project_gauge_transform(gm0, gmd0, st["mf"], st["mfd"], ts)
            dh = self.run_hmc_evolve(gm0, gmd0, gf0, st["mf"], st["mfd"], h["n_step"], h["md_time"], proj)
            flag, _ = o.metropolis_accept_py(dh, rt.split("metropolis_accept"))
            if flag or traj < h["max_traj_always_accept"]:
                gf, st["gm"], st["gmd"] = gf0, gm0, gmd0
            else:
                st["gm"] *= -1
                st["gmd"] *= -1
            plaqs.append(o.gf_avg_plaq(gf, ts))
        return plaqs


def test_oracle_driver_reproduces_reference_log(oracle, goldens):
    """All five jobs of the example, eight trajectories each (the oracle's
    primitives and the example's refresh / selection / Metropolis logic)."""
    for job in goldens["py_hmc_fa_sym"]["jobs"]:
        got = OracleFa(oracle, job["params"], job["job_tag"]).run(len(job["plaq"]))
        for t, (a, b) in enumerate(zip(got, job["plaq"])):
            assert abs(a - b) <= GOLDEN_EPS * abs(b), (job["job_tag"], t + 1, a, b)


# ---- GPU: the library against the oracle ---------------------------------------------


def _upload(q, arr, cls, mult=4, precision=64):
    f = cls(q.Geometry(TS), mult, precision=precision) if cls is q.FieldRealD or cls is q.FieldColorMatrix else \
        cls(q.Geometry(TS), precision=precision)
    f.from_numpy(arr)
    return f


def _nrel(a, b):
    return float(np.linalg.norm((np.asarray(a) - b).ravel()) / max(np.linalg.norm(np.asarray(b).ravel()), 1e-300))


@pytest.mark.gpu
def test_gpu_primitives_match_oracle(q, oracle):
    o = oracle
    rs_o, gf0, mf, mfd, gm, gmd = seeded_inputs(o)
    rs = q.RngState(SEED)
    geo = q.Geometry(TS)
    # per-site uniform masses and momenta drawn with them, from the same states
    qmf = q.FieldRealD(geo, 4)
    qmf.set_rand(rs.split("mf"), 4.0, 1.0)
    ref_mf = np.zeros_like(mf)
    o.field_set_u_rand(ref_mf, TS, rs_o.split("mf"), 4.0, 1.0)
    assert np.array_equal(qmf.to_numpy(), ref_mf)
    qmf.from_numpy(mf)
    qmfd = _upload(q, mfd, q.FieldRealD)
    qgm = q.GaugeMomentum(geo)
    qgm.set_rand_fa(qmf, rs.split("gm"))
    assert _nrel(qgm, gm) < 1e-15
    assert not np.asarray(qgm)[np.isinf(mf)].any()
    qgm.from_numpy(gm)
    qgmd = _upload(q, gmd, q.GaugeMomentum)
    assert abs(q.gm_hamilton_node_fa(qgm, qmf) - o.gm_hamilton_node_fa(gm, mf, TS)) < 1e-12 * abs(
        o.gm_hamilton_node_fa(gm, mf, TS))
    # the three evolutions
    qgf0 = _upload(q, gf0, q.GaugeField)
    for name, qf, of in (("fa", lambda g: q.gf_evolve_fa(g, qgm, qmf, DT), lambda g: o.gf_evolve_fa(g, gm, mf, TS, DT)),
                         ("fa_dual", lambda g: q.gf_evolve_fa_dual(g, qgmd, qmfd, DT),
                          lambda g: o.gf_evolve_fa_dual(g, gmd, mfd, TS, DT)),
                         ("dual", lambda g: q.gf_evolve_dual(g, qgmd, DT), lambda g: o.gf_evolve_dual(g, gmd, TS, DT))):
        g = qgf0.copy()
        qf(g)
        r = gf0.copy()
        of(r)
        assert np.abs(np.asarray(g) - r).max() < 1e-14, name
    # dual force
    F = q.GaugeMomentum(geo)
    q.set_gm_force(F, qgf0, q.GaugeAction(BETA, C1))
    Fd = q.GaugeMomentum(geo)
    q.set_gm_force_dual(Fd, qgf0, F)
    ref_fd = o.new_field(TS)
    o.set_gm_force_dual(ref_fd, gf0, np.asarray(F), TS)
    assert _nrel(Fd, ref_fd) < 1e-14
    # projection of the gauge-transformation motion (masses with +inf)
    a, b = qgm.copy(), qgmd.copy()
    ch = q.project_gauge_transform(a, b, qmf, qmfd)
    ra, rb = gm.copy(), gmd.copy()
    ch_ref = o.project_gauge_transform(ra, rb, mf, mfd, TS)
    assert abs(ch - ch_ref) < 1e-13 * ch_ref
    assert _nrel(a, ra) < 1e-14 and _nrel(b, rb) < 1e-14
    # gauge-transformation momenta and dot products
    gtm = q.FieldColorMatrix(geo, 1)
    gtm.from_numpy(gm[:, :1])
    a, b = q.GaugeMomentum(geo), q.GaugeMomentum(geo)
    q.set_gauge_transform_momentum(a, b, gtm)
    ra, rb = o.new_field(TS), o.new_field(TS)
    o.set_gauge_transform_momentum(ra, rb, np.ascontiguousarray(gm[:, :1]), TS)
    assert np.array_equal(np.asarray(a), ra) and np.array_equal(np.asarray(b), rb)
    assert np.abs(q.dot_gauge_momentum(qgm, qgmd).to_numpy() - o.dot_gauge_momentum(gm, gmd, TS)).max() < 1e-13
    # Gaussian real field
    g3 = q.FieldRealD(geo, 3)
    g3.set_rand_g(rs.split("g"), 0.5, 2.0)
    r3 = np.zeros((o.volume(TS), 3))
    o.field_set_g_rand(r3, TS, rs_o.split("g"), 0.5, 2.0)
    assert np.array_equal(g3.to_numpy(), r3)


@pytest.mark.gpu
def test_gpu_selection_assignment(q):
    geo = q.Geometry(TS)
    V = geo.total_volume
    rng = np.random.default_rng(5)
    sel = rng.random((V, 4)) < 0.3
    a, b = q.GaugeMomentum(geo), q.GaugeMomentum(geo)
    a.set_rand(q.RngState("sel-a"))
    b.set_rand(q.RngState("sel-b"))
    na, nb = np.asarray(a), np.asarray(b)
    a[sel] = b.selected(sel)
    want = na.copy()
    want[sel] = nb[sel]
    assert np.array_equal(np.asarray(a), want)
    mf = q.FieldRealD(geo, 4)
    q.set_unit(mf)
    mf[sel] = 2.5
    assert np.array_equal(mf.to_numpy(), np.where(sel, 2.5, 1.0))
    mf[sel] = np.inf
    assert np.isinf(mf.to_numpy()[sel]).all()


@pytest.mark.gpu
def test_gauge_transform_momentum_is_a_gauge_transformation(q):
    """gf_evolve(gm) then gf_evolve_dual(gm_dual) with the momenta of
    set_gauge_transform_momentum is U_mu(x) -> e^{dt g(x)} U_mu(x) e^{-dt g(x+mu)}:
    the plaquette and the action do not change, the links do; and the
    projection removes (nearly all of) such a motion."""
    geo = q.Geometry(TS)
    gf = q.GaugeField(geo)
    gf.set_rand(q.RngState("gt-gf"), 0.3, 2)
    gtm = q.FieldColorMatrix(geo, 1)
    m = q.GaugeMomentum(geo)
    m.set_rand(q.RngState("gt-m"))
    gtm.from_numpy(np.asarray(m)[:, :1])
    gm, gmd = q.GaugeMomentum(geo), q.GaugeMomentum(geo)
    q.set_gauge_transform_momentum(gm, gmd, gtm)
    g2 = gf.copy()
    q.gf_evolve(g2, gm, 0.3)
    q.gf_evolve_dual(g2, gmd, 0.3)
    ga = q.GaugeAction(2.13, -0.331)
    assert abs(q.gf_hamilton_node(g2, ga) - q.gf_hamilton_node(gf, ga)) < 1e-10 * abs(q.gf_hamilton_node(gf, ga))
    assert np.abs(np.asarray(g2) - np.asarray(gf)).max() > 1e-2
    mf = q.FieldRealD(geo, 4)
    q.set_unit(mf)
    mfd = q.FieldRealD(geo, 4)
    q.set_unit(mfd)
    q.project_gauge_transform(gm, gmd, mf, mfd)
    # a single projection pass removes 1/8 of ... the average exactly: what is
    # left is orthogonal to the motion of the same average
    ch2 = q.project_gauge_transform(gm.copy(), gmd.copy(), mf, mfd)
    assert ch2 < 1e-24


@pytest.mark.gpu
def test_fp32_fields(q, oracle):
    o = oracle
    _, gf0, mf, mfd, gm, gmd = seeded_inputs(o)
    geo = q.Geometry(TS)
    qmf, qmfd = _upload(q, mf, q.FieldRealD), _upload(q, mfd, q.FieldRealD)
    g = _upload(q, gf0, q.GaugeField, precision=32)
    p = _upload(q, gm, q.GaugeMomentum, precision=32)
    pd = _upload(q, gmd, q.GaugeMomentum, precision=32)
    q.gf_evolve_fa(g, p, qmf, DT)
    q.gf_evolve_fa_dual(g, pd, qmfd, DT)
    r = gf0.copy()
    o.gf_evolve_fa(r, gm, mf, TS, DT)
    o.gf_evolve_fa_dual(r, gmd, mfd, TS, DT)
    assert np.abs(np.asarray(g) - r).max() < 2e-6
    ch = q.project_gauge_transform(p, pd, qmf, qmfd)
    ch_ref = o.project_gauge_transform(gm.copy(), gmd.copy(), mf, mfd, TS)
    assert abs(ch - ch_ref) < 1e-5 * ch_ref
    assert geo.total_volume == o.volume(TS)


@pytest.mark.gpu
def test_run_hmc_fa_reference_log(q, goldens):
    """The library's driver, all five jobs of the example's golden log."""
    for job in goldens["py_hmc_fa_sym"]["jobs"]:
        recs = q.run_hmc_fa(job["params"], job["job_tag"])
        for rec, b in zip(recs, job["plaq"]):
            assert abs(rec["plaq"] - b) <= GOLDEN_EPS * abs(b), (job["job_tag"], rec["traj"], rec["plaq"], b)


@pytest.mark.gpu
def test_gpu_fa_odd_lattice(q, oracle):
    """3x4x5x6 (V = 360, not a multiple of the 32-site blocks): projection,
    dual force and both evolutions against the oracle, masses with +inf."""
    o = oracle
    ts = (3, 4, 5, 6)
    _, gf0, mf, mfd, gm, gmd = seeded_inputs(o, ts, "fa-odd")
    geo = q.Geometry(ts)
    up = lambda a, f: (f.from_numpy(a), f)[1]  # noqa: E731
    qmf, qmfd = up(mf, q.FieldRealD(geo, 4)), up(mfd, q.FieldRealD(geo, 4))
    qgm, qgmd = up(gm, q.GaugeMomentum(geo)), up(gmd, q.GaugeMomentum(geo))
    qgf = up(gf0, q.GaugeField(geo))
    a, b = qgm.copy(), qgmd.copy()
    ch = q.project_gauge_transform(a, b, qmf, qmfd)
    ra, rb = gm.copy(), gmd.copy()
    assert abs(ch - o.project_gauge_transform(ra, rb, mf, mfd, ts)) < 1e-13 * ch
    assert np.abs(np.asarray(a) - ra).max() < 1e-14 and np.abs(np.asarray(b) - rb).max() < 1e-14
    g = qgf.copy()
    q.gf_evolve_fa(g, qgm, qmf, DT)
    q.gf_evolve_fa_dual(g, qgmd, qmfd, DT)
    r = gf0.copy()
    o.gf_evolve_fa(r, gm, mf, ts, DT)
    o.gf_evolve_fa_dual(r, gmd, mfd, ts, DT)
    assert np.abs(np.asarray(g) - r).max() < 1e-14
    F, Fd = q.GaugeMomentum(geo), q.GaugeMomentum(geo)
    q.set_gm_force(F, qgf, q.GaugeAction(BETA, C1))
    q.set_gm_force_dual(Fd, qgf, F)
    rfd = o.new_field(ts)
    o.set_gm_force_dual(rfd, gf0, np.asarray(F), ts)
    assert np.abs(np.asarray(Fd) - rfd).max() < 1e-13
    assert abs(q.gm_hamilton_node_fa(qgm, qmf) - o.gm_hamilton_node_fa(gm, mf, ts)) < 1e-12 * o.gm_hamilton_node_fa(
        gm, mf, ts)
