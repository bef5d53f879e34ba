"""Field-accelerated HMC: per-link masses and dual momenta on the GPU.

Library functions (qlat/hmc.pyx:51-110, hmc.cpp:121-201, 330-396, 492-645):
``set_rand_gauge_momentum_fa``, ``gm_hamilton_node_fa``, ``gf_evolve_fa``,
``gf_evolve_fa_dual``, ``gf_evolve_dual``, ``set_gm_force_dual``,
``project_gauge_transform``, ``set_gauge_transform_momentum``,
``dot_gauge_momentum``.

The trajectory driver below follows the reference's field-accelerated example
(examples-py/hmc-pure-gauge-fa-sym.py:112-680): masses refreshed completely
every ``complete_refresh_interval`` trajectories (unit, random in [1, 4), or
by the number of even directions of a shifted 2^4 grid, optionally split by
parity), partial momentum refreshes of the selections in between, an Omelyan
force-gradient integrator moving each link by both momenta, the
gauge-transformation motion projected out of momenta and forces, and the
Python-API Metropolis step.  Its parameters are a plain dict with the keys of
the example's ``set_param(job_tag, ...)`` table.
"""

from __future__ import annotations

import ctypes
import math

import numpy as np

from ._lib import call
from .field import FieldColorMatrix, FieldRealD, GaugeAction, GaugeField, GaugeMomentum, Geometry, RngState
from .field import set_unit
from .hmc import gf_hamilton_node, metropolis_accept, set_gm_force

# ---- library functions ---------------------------------------------------------


def set_rand_gauge_momentum_fa(gm: GaugeMomentum, mf: FieldRealD, rng: RngState):
    """hmc.pyx:59-60 -> set_rand_gauge_momentum(gm, mf, rs) (hmc.cpp:121-149):
    unit-sigma momenta scaled by sqrt(mass); zero where the mass is +inf."""
    call("qgb_set_rand_gauge_momentum_fa", gm.handle, mf.handle, rng.c)


def gm_hamilton_node_fa(gm: GaugeMomentum, mf: FieldRealD) -> float:
    """hmc.pyx:65-66 -> gm_hamilton_node(gm, mf) (hmc.cpp:175-201)."""
    o = ctypes.c_double()
    call("qgb_gm_hamilton_node_fa", gm.handle, mf.handle, ctypes.byref(o))
    return o.value


def gf_evolve_fa(gf: GaugeField, gm: GaugeMomentum, mf: FieldRealD, step_size: float):
    """hmc.pyx:77-78 -> gf_evolve(gf, gm, mf, dt) (hmc.cpp:350-372): U = exp(dt/m P) U."""
    call("qgb_gf_evolve_fa", gf.handle, gm.handle, mf.handle, float(step_size))


def gf_evolve_fa_dual(gf: GaugeField, gm_dual: GaugeMomentum, mf_dual: FieldRealD, step_size: float):
    """hmc.pyx:80-81 -> gf_evolve_dual(gf, gm_dual, mf_dual, dt) (hmc.cpp:374-396):
    U = U exp(-dt/m P)."""
    call("qgb_gf_evolve_fa_dual", gf.handle, gm_dual.handle, mf_dual.handle, float(step_size))


def gf_evolve_dual(gf: GaugeField, gm_dual: GaugeMomentum, step_size: float):
    """hmc.pyx:74-75 -> gf_evolve_dual(gf, gm_dual, dt) (hmc.cpp:330-348): U = U exp(-dt P)."""
    call("qgb_gf_evolve_dual", gf.handle, gm_dual.handle, float(step_size))


def set_gm_force_dual(gm_force_dual: GaugeMomentum, gf: GaugeField, gm_force: GaugeMomentum):
    """hmc.pyx:97-98 -> set_gm_force_dual (hmc.cpp:492-513): -U^+ F U."""
    call("qgb_set_gm_force_dual", gm_force_dual.handle, gf.handle, gm_force.handle)


def project_gauge_transform(gm: GaugeMomentum, gm_dual: GaugeMomentum, mf: FieldRealD, mf_dual: FieldRealD,
                            *, want_change: bool = True) -> float | None:
    """hmc.pyx:100-104 -> project_gauge_transform (hmc.cpp:515-589): remove the
    gauge-transformation motion; returns qnorm of the removed per-site average
    / volume (with ``want_change=False`` nothing is read back and the call
    stays asynchronous)."""
    if not want_change:
        call("qgb_project_gauge_transform", gm.handle, gm_dual.handle, mf.handle, mf_dual.handle, None)
        return None
    o = ctypes.c_double()
    call("qgb_project_gauge_transform", gm.handle, gm_dual.handle, mf.handle, mf_dual.handle, ctypes.byref(o))
    return o.value


def set_gauge_transform_momentum(gm: GaugeMomentum, gm_dual: GaugeMomentum, gtm: FieldColorMatrix):
    """hmc.pyx:106-112 -> set_gauge_transform_momentum (hmc.cpp:591-626)."""
    call("qgb_set_gauge_transform_momentum", gm.handle, gm_dual.handle, gtm.handle)


def dot_gauge_momentum(gm1: GaugeMomentum, gm2: GaugeMomentum) -> FieldRealD:
    """dot_gauge_momentum (hmc.cpp:628-645): f_mu(x) = Re tr(gm1^+ gm2)."""
    f = FieldRealD(gm1.geo, 4)
    call("qgb_dot_gauge_momentum", f.handle, gm1.handle, gm2.handle)
    return f


# ---- trajectory driver (examples-py/hmc-pure-gauge-fa-sym.py) ----------------------


class MomentumAutoCorr:
    """Autocorrelation of the momenta within the selections
    (hmc-pure-gauge-fa-sym.py:36-109): ``auto_corr_list[k]`` holds
    [MD time, sum over selection k of dot_gauge_momentum(gm, gm_at_refresh)]."""

    def refresh_mac(self, gm, gm_dual, sel_list, sel_dual_list, info_list):
        assert len(sel_list) == len(sel_dual_list)
        self.info_list = info_list
        self.auto_corr_list = [[] for _ in range(2 * len(sel_list))]
        self.time = 0.0
        self.gm = gm.copy()
        self.gm_dual = gm_dual.copy()
        self.sel_list = sel_list
        self.sel_dual_list = sel_dual_list
        self.add_mac(gm, gm_dual, 0.0)

    def add_mac(self, gm, gm_dual, dt):
        self.time += dt
        f1 = dot_gauge_momentum(gm, self.gm).to_numpy()
        f2 = dot_gauge_momentum(gm_dual, self.gm_dual).to_numpy()
        idx = 0
        for sel in self.sel_list:
            self.auto_corr_list[idx].append([self.time, float(f1[sel].sum())])
            idx += 1
        for sel in self.sel_dual_list:
            self.auto_corr_list[idx].append([self.time, float(f2[sel].sum())])
            idx += 1

    def data(self):
        return list(zip(self.info_list, [np.array(v, dtype=np.float64) for v in self.auto_corr_list]))


class _Scratch:
    """Fields reused by every force-gradient step of a trajectory."""

    def __init__(self, geo: Geometry, precision: int):
        self.gf = GaugeField(geo, precision=precision)
        self.force = GaugeMomentum(geo, precision=precision)
        self.force_dual = GaugeMomentum(geo, precision=precision)


def fa_gf_evolve(gf, gm, gm_dual, mf, mf_dual, dt):
    """hmc-pure-gauge-fa-sym.py:112-115: both momenta move the links."""
    gf_evolve_fa(gf, gm, mf, dt)
    gf_evolve_fa_dual(gf, gm_dual, mf_dual, dt)


def fa_gm_evolve_fg(gm, gm_dual, gf_init, mf, mf_dual, ga, fg_dt, dt, *, is_project_gauge_transform,
                    scratch: _Scratch | None = None):
    """hmc-pure-gauge-fa-sym.py:117-148: the force-gradient momentum update of
    both momenta."""
    s = scratch if scratch is not None else _Scratch(gf_init.geo, gf_init.precision)
    gf, gm_force, gm_force_dual = s.gf, s.force, s.force_dual
    gf @= gf_init
    set_gm_force(gm_force, gf, ga)
    set_gm_force_dual(gm_force_dual, gf, gm_force)
    if is_project_gauge_transform:
        project_gauge_transform(gm_force, gm_force_dual, mf, mf_dual, want_change=False)
    fa_gf_evolve(gf, gm_force, gm_force_dual, mf, mf_dual, fg_dt)
    set_gm_force(gm_force, gf, ga)
    set_gm_force_dual(gm_force_dual, gf, gm_force)
    gm_force *= dt
    gm_force_dual *= dt
    gm += gm_force
    gm_dual += gm_force_dual
    if is_project_gauge_transform:
        project_gauge_transform(gm, gm_dual, mf, mf_dual, want_change=False)


def fa_run_hmc_evolve(gm, gm_dual, gf, mf, mf_dual, ga, rs, n_step, md_time, *, is_project_gauge_transform,
                      mom_auto_corr=None) -> float:
    """hmc-pure-gauge-fa-sym.py:150-213 (Omelyan force gradient); returns delta_h."""
    energy = gm_hamilton_node_fa(gm, mf) + gm_hamilton_node_fa(gm_dual, mf_dual) + gf_hamilton_node(gf, ga)
    dt = md_time / n_step
    lam = 0.5 * (1.0 - 1.0 / math.sqrt(3.0))
    theta = (2.0 - math.sqrt(3.0)) / 48.0
    ttheta = theta * dt * dt * dt
    scratch = _Scratch(gf.geo, gf.precision)
    fa_gf_evolve(gf, gm, gm_dual, mf, mf_dual, lam * dt)
    for i in range(n_step):
        fa_gm_evolve_fg(gm, gm_dual, gf, mf, mf_dual, ga, 4.0 * ttheta / dt, 0.5 * dt,
                        is_project_gauge_transform=is_project_gauge_transform, scratch=scratch)
        fa_gf_evolve(gf, gm, gm_dual, mf, mf_dual, (1.0 - 2.0 * lam) * dt)
        fa_gm_evolve_fg(gm, gm_dual, gf, mf, mf_dual, ga, 4.0 * ttheta / dt, 0.5 * dt,
                        is_project_gauge_transform=is_project_gauge_transform, scratch=scratch)
        if i < n_step - 1:
            fa_gf_evolve(gf, gm, gm_dual, mf, mf_dual, 2.0 * lam * dt)
        else:
            fa_gf_evolve(gf, gm, gm_dual, mf, mf_dual, lam * dt)
        if mom_auto_corr is not None:
            mom_auto_corr.add_mac(gm, gm_dual, dt)
    gf.unitarize()
    return (gm_hamilton_node_fa(gm, mf) + gm_hamilton_node_fa(gm_dual, mf_dual) + gf_hamilton_node(gf, ga)
            - energy)


def fa_run_hmc_traj(gf, gm, gm_dual, mf, mf_dual, ga, traj, rs, *, is_reverse_test=False, n_step=6, md_time=1.0,
                    is_always_accept=False, is_project_gauge_transform=True, mom_auto_corr=None, log=None):
    """hmc-pure-gauge-fa-sym.py:215-313: one trajectory with the optional
    reversibility test and the Metropolis step; returns (flag, delta_h)."""
    rs = rs.split(f"{traj}")
    gf0 = gf.copy()
    gm0 = gm.copy()
    gm_dual0 = gm_dual.copy()
    if is_project_gauge_transform:
        change_qnorm = project_gauge_transform(gm0, gm_dual0, mf, mf_dual)
        if change_qnorm > 1e-8 and log is not None:
            log(f"fa_run_hmc_traj: project_gauge_transform: change_qnorm={change_qnorm}")
    delta_h = fa_run_hmc_evolve(gm0, gm_dual0, gf0, mf, mf_dual, ga, rs, n_step, md_time,
                                is_project_gauge_transform=is_project_gauge_transform, mom_auto_corr=mom_auto_corr)
    if is_reverse_test:
        gm_r = gm0.copy()
        gm_dual_r = gm_dual0.copy()
        gf0_r = gf0.copy()
        delta_h_rev = fa_run_hmc_evolve(gm_r, gm_dual_r, gf0_r, mf, mf_dual, ga, rs, n_step, -md_time,
                                        is_project_gauge_transform=is_project_gauge_transform)
        gf0_r -= gf
        gm_r -= gm
        gm_dual_r -= gm_dual
        if log is not None:
            log(f"fa_run_hmc_traj: reversed delta_diff: {delta_h + delta_h_rev} / {delta_h}")
        assert gf0_r.qnorm() <= 1e-12 * gf.qnorm()
        assert gm_r.qnorm() <= 1e-12 * gm.qnorm()
        assert gm_dual_r.qnorm() <= 1e-12 * gm_dual.qnorm()
    flag, accept_prob = metropolis_accept(delta_h, traj, rs.split("metropolis_accept"))
    if flag or is_always_accept:
        gf @= gf0
        gm @= gm0
        gm_dual @= gm_dual0
    else:
        gm *= -1.0
        gm_dual *= -1.0
    return flag, delta_h


def _grid2_count(geo: Geometry, rs: RngState) -> tuple[np.ndarray, np.ndarray]:
    """Per link, the number of the other three directions in which the site's
    coordinate relative to a random offset is even; and the parity of that
    relative coordinate (hmc-pure-gauge-fa-sym.py:411-423, 462-475)."""
    xg_rel = geo.xg_arr().astype(np.int64) - np.array(rs.c_rand_gen(geo.total_site), dtype=np.int64)
    count = np.zeros(xg_rel.shape, np.int32)
    for m in range(4):
        for n in range(4):
            if n != m:
                count[xg_rel[:, n] % 2 == 0, m] += 1
    is_even = (xg_rel.sum(-1) % 2 == 0)[:, None]
    return count, is_even


def fa_run_hmc_mass_mom_refresh(params, traj, is_force_refresh, rs, mf, mf_dual, gm, gm_dual, sel_list,
                                sel_dual_list, mom_auto_corr):
    """hmc-pure-gauge-fa-sym.py:315-551: complete refresh of masses, selections
    and momenta every ``complete_refresh_interval`` trajectories (or when
    forced), otherwise a refresh of the selections whose interval divides traj."""
    rs = rs.split(f"{traj}")
    geo = mf.geo
    fa = params["hmc"]["fa"]
    is_project_gauge_transform = fa["is_project_gauge_transform"]
    complete_refresh_interval = fa.get("complete_refresh_interval", 1)
    mass_type = fa.get("mass_type")
    mass_list = fa.get("mass_list")
    interval_list = fa.get("interval_list")
    if isinstance(interval_list, list):
        for interval in interval_list:
            assert complete_refresh_interval % interval == 0
    is_refresh = traj % complete_refresh_interval == 0 or is_force_refresh
    if is_refresh:
        if mass_type is None:
            set_unit(mf)
            set_unit(mf_dual)
            sel = np.ones((geo.total_volume, 4), dtype=bool)
            sel_list[:] = [sel]
            sel_dual_list[:] = [sel]
            info_list = [[True, 1.0, complete_refresh_interval], [False, 1.0, complete_refresh_interval]]
        elif mass_type == "random":
            mf.set_rand(rs.split("fa_mass"), 4.0, 1.0)
            mf_dual.set_rand(rs.split("fa_mass_dual"), 4.0, 1.0)
            sel = mf.to_numpy() < 2.0
            sel_dual = mf_dual.to_numpy() < 2.0
            sel_list[:] = [sel, ~sel]
            sel_dual_list[:] = [sel_dual, ~sel_dual]
            info_list = [[True, 1.5, interval_list[0]], [True, 3.0, interval_list[1]],
                         [False, 1.5, interval_list[0]], [False, 3.0, interval_list[1]]]
            assert len(sel_list) == len(interval_list)
        elif mass_type in ("grid-2", "grid-2-eo"):
            count, is_even = _grid2_count(geo, rs)
            if mass_type == "grid-2":
                sel_list[:] = [count == k for k in range(4)]
                sel_dual_list[:] = sel_list
            else:
                is_odd = ~is_even
                sel_list[:] = ([(count == k) & is_even for k in range(4)] + [(count == k) & is_odd for k in range(4)])
                sel_dual_list[:] = ([(count == k) & is_odd for k in range(4)]
                                    + [(count == k) & is_even for k in range(4)])
            assert len(sel_list) == len(interval_list) == len(mass_list)
            for idx, mass in enumerate(mass_list):
                mf[sel_list[idx]] = float(mass)
                mf_dual[sel_dual_list[idx]] = float(mass)
            info_list = ([[True, m, i] for m, i in zip(mass_list, interval_list)]
                         + [[False, m, i] for m, i in zip(mass_list, interval_list)])
        else:
            raise ValueError(f"fa_run_hmc_mass_mom_refresh: mass_type={mass_type}")
        gm.set_rand_fa(mf, rs.split("set_rand_gauge_momentum"))
        gm_dual.set_rand_fa(mf_dual, rs.split("set_rand_gauge_momentum_dual"))
        if is_project_gauge_transform:
            project_gauge_transform(gm, gm_dual, mf, mf_dual, want_change=False)
        mom_auto_corr.refresh_mac(gm, gm_dual, sel_list, sel_dual_list, info_list)
    else:
        gm1 = GaugeMomentum(geo, precision=gm.precision)
        gm_dual1 = GaugeMomentum(geo, precision=gm.precision)
        if is_project_gauge_transform:
            # first add the gauge-transformation component back
            gm1.set_rand_fa(mf, rs.split("set_rand_gauge_momentum_g"))
            gm_dual1.set_rand_fa(mf_dual, rs.split("set_rand_gauge_momentum_dual_g"))
            gm2 = gm1.copy()
            gm_dual2 = gm_dual1.copy()
            project_gauge_transform(gm2, gm_dual2, mf, mf_dual, want_change=False)
            gm2 -= gm1
            gm_dual2 -= gm_dual1
            gm -= gm2
            gm_dual -= gm_dual2
        gm1.set_rand_fa(mf, rs.split("set_rand_gauge_momentum"))
        gm_dual1.set_rand_fa(mf_dual, rs.split("set_rand_gauge_momentum_dual"))
        assert len(sel_list) == len(interval_list) == len(sel_dual_list)
        for sel, interval in zip(sel_list, interval_list):
            if traj % interval == 0:
                gm[sel] = gm1.selected(sel)
        for sel_dual, interval in zip(sel_dual_list, interval_list):
            if traj % interval == 0:
                gm_dual[sel_dual] = gm_dual1.selected(sel_dual)
        if is_project_gauge_transform:
            project_gauge_transform(gm, gm_dual, mf, mf_dual, want_change=False)


def run_hmc_fa(params: dict, job_seed: str, *, precision: int = 64, log=None, on_traj=None) -> list[dict]:
    """hmc-pure-gauge-fa-sym.py:582-680 from a fresh start: per trajectory a
    mass / momentum refresh, then a trajectory; returns one record per
    trajectory (traj, plaq, flag, delta_h).  ``job_seed`` is the example's
    get_job_seed(job_tag) (the job tag unless a seed is set).  Saving
    configurations and the topology measurements of the example are left to
    ``on_traj(traj, gf)``."""
    h = params["hmc"]
    total_site = tuple(params["total_site"])
    complete_refresh_interval = h["fa"].get("complete_refresh_interval", 1)
    ga = GaugeAction(h["beta"], h["c1"])
    geo = Geometry(total_site)
    rs = RngState(f"run_hmc-{job_seed}")
    gf = GaugeField(geo, precision=precision)
    mf = FieldRealD(geo, 4)
    mf_dual = FieldRealD(geo, 4)
    gm = GaugeMomentum(geo, precision=precision)
    gm_dual = GaugeMomentum(geo, precision=precision)
    mom_auto_corr = MomentumAutoCorr()
    gf.set_rand(rs.split("init"), 0.1, 2)
    is_force_refresh = True
    sel_list, sel_dual_list = [], []
    records = []
    for traj in range(0, h["max_traj"]):
        fa_run_hmc_mass_mom_refresh(params, traj, is_force_refresh, rs.split("run_hmc_mass_mom_refresh"), mf,
                                    mf_dual, gm, gm_dual, sel_list, sel_dual_list, mom_auto_corr)
        is_force_refresh = False
        traj += 1
        flag, delta_h = fa_run_hmc_traj(
            gf, gm, gm_dual, mf, mf_dual, ga, traj, rs.split("run_hmc_traj"), n_step=h["n_step"],
            md_time=h["md_time"], is_always_accept=traj < h["max_traj_always_accept"],
            is_reverse_test=traj < h["max_traj_reverse_test"],
            is_project_gauge_transform=h["fa"]["is_project_gauge_transform"], mom_auto_corr=mom_auto_corr, log=log)
        rec = {"traj": traj, "plaq": gf.plaq(), "flag": bool(flag), "delta_h": delta_h}
        records.append(rec)
        if log is not None:
            log(f"run_hmc_fa: {rec}")
        if traj % complete_refresh_interval == 0:
            rec["mom_auto_corr"] = mom_auto_corr.data()
        if on_traj is not None:
            on_traj(traj, gf)
    return records
