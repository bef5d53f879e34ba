"""Pure-gauge HMC on the GPU with qlat's Python API (qlat/qlat/hmc.pyx).

Every function keeps the reference's name, arguments and return value.  The
integrators run as one stream of fused CUDA kernels inside the library
(qgb_run_hmc_evolve); ``run_hmc_evolve_pure_gauge`` accepts ``precision``
("fp64" for the plain form, "mixed" for FP32 molecular dynamics with FP64
Hamiltonians) and ``integrator`` ("force-gradient" as in the reference, or
"leapfrog").
"""

from __future__ import annotations

import ctypes
import math

from . import _lib
from ._lib import call
from .field import GaugeAction, GaugeField, GaugeMomentum, RngState

INTEGRATORS = {"force-gradient": 0, "leapfrog": 1}


def _d():
    return ctypes.c_double()


def glb_sum_double(x: float) -> float:
    """Single node: the global sum is the local value (mpi.h:273-308)."""
    return float(x)


def set_rand_gauge_momentum(gm: GaugeMomentum, sigma: float, rng: RngState):
    """hmc.cpp:107-119"""
    call("qgb_set_rand_gauge_momentum", gm.handle, float(sigma), rng.c)


def gm_hamilton_node(gm: GaugeMomentum) -> float:
    """hmc.cpp:151-173"""
    o = _d()
    call("qgb_gm_hamilton_node", gm.handle, ctypes.byref(o))
    return o.value


def gf_hamilton_node(gf: GaugeField, ga: GaugeAction) -> float:
    """hmc.cpp:279-298"""
    o = _d()
    call("qgb_gf_hamilton_node", gf.handle, ga.beta(), ga.c1(), ctypes.byref(o))
    return o.value


def gf_hamilton(gf: GaugeField, ga: GaugeAction) -> float:
    """hmc.cpp:300-309"""
    return glb_sum_double(gf_hamilton_node(gf, ga))


def gf_sum_re_tr_plaq_node_no_comm(gf: GaugeField) -> float:
    o = _d()
    call("qgb_gf_sum_re_tr_plaq_node", gf.handle, ctypes.byref(o))
    return o.value


def gf_sum_re_tr_rect_node_no_comm(gf: GaugeField) -> float:
    o = _d()
    call("qgb_gf_sum_re_tr_rect_node", gf.handle, ctypes.byref(o))
    return o.value


def gf_avg_plaq(gf: GaugeField) -> float:
    """qcd.cpp:94-142"""
    o = _d()
    call("qgb_gf_avg_plaq", gf.handle, ctypes.byref(o))
    return o.value


def gf_avg_wilson_loop_normalized_tr(gf: GaugeField, l: int, t: int) -> float:
    """qcd.pyx:250-254 -> gf_avg_wilson_loop (qcd-utils.cpp:359-400): Re tr / 3 of
    the l x t Wilson loop (spatial side l, time side t), averaged over sites and
    the three spatial directions."""
    o = _d()
    call("qgb_gf_avg_wilson_loop_normalized_tr", gf.handle, int(l), int(t), ctypes.byref(o))
    return o.value


def gf_evolve(gf: GaugeField, gm: GaugeMomentum, step_size: float):
    """hmc.cpp:311-328: U <- unitarize(exp(step_size P) U)"""
    call("qgb_gf_evolve", gf.handle, gm.handle, float(step_size))


def set_gm_force(gm_force: GaugeMomentum, gf: GaugeField, ga: GaugeAction):
    """hmc.cpp:466-490"""
    if gm_force._h is None:
        gm_force.init(gf.geo)
    call("qgb_set_gm_force", gm_force.handle, gf.handle, ga.beta(), ga.c1())


def unitarize(gf: GaugeField):
    """qcd.cpp:346-359"""
    call("qgb_unitarize", gf.handle)


def metropolis_accept(delta_h: float, traj: int, rs: RngState):
    """hmc.pyx:139-155 (Python API semantics: accept if delta_h <= 0 or
    u_rand_gen(1, 0) <= exp(-delta_h)); returns (flag, accept_prob)."""
    flag_d = 0.0
    accept_prob = 0.0
    if delta_h <= 0.0:
        accept_prob = 1.0
        flag_d = 1.0
    else:
        accept_prob = math.exp(-delta_h)
        rand_num = rs.u_rand_gen(1.0, 0.0)
        if rand_num <= accept_prob:
            flag_d = 1.0
    flag_d = glb_sum_double(flag_d)
    accept_prob = glb_sum_double(accept_prob)
    return flag_d > 0.5, accept_prob


def metropolis_accept_cpp(delta_h: float, traj: int, rs: RngState):
    """hmc.cpp:77-105 (C++ API semantics); returns (flag, accept_prob)."""
    p = ctypes.c_double()
    f = ctypes.c_int32()
    call("qgb_metropolis_accept", float(delta_h), int(traj), rs.c, ctypes.byref(p), ctypes.byref(f))
    return bool(f.value), p.value


def gm_evolve_fg_pure_gauge(gm: GaugeMomentum, gf_init: GaugeField, ga: GaugeAction, fg_dt: float, dt: float):
    """hmc.pyx:157-167: gm += dt F(exp(fg_dt F(gf)) gf), fused on the GPU."""
    call("qgb_gm_evolve_fg", gm.handle, gf_init.handle, ga.beta(), ga.c1(), float(fg_dt), float(dt))


def run_hmc_evolve_pure_gauge(gm: GaugeMomentum, gf: GaugeField, ga: GaugeAction, rs: RngState | None,
                              n_step: int, md_time: float = 1.0, *, integrator: str = "force-gradient",
                              precision: str = "fp64", reunit_interval: int = 4) -> float:
    """hmc.pyx:169-188.  Returns delta_h."""
    o = _d()
    if precision == "fp64":
        call("qgb_run_hmc_evolve", gm.handle, gf.handle, ga.beta(), ga.c1(), int(n_step), float(md_time),
             INTEGRATORS[integrator], ctypes.byref(o))
    elif precision == "mixed":
        call("qgb_run_hmc_evolve_mixed", gm.handle, gf.handle, ga.beta(), ga.c1(), int(n_step), float(md_time),
             INTEGRATORS[integrator], int(reunit_interval), ctypes.byref(o))
    else:
        raise ValueError(f"precision must be 'fp64' or 'mixed', not {precision!r}")
    return glb_sum_double(o.value)


def run_hmc_pure_gauge(gf: GaugeField, ga: GaugeAction, traj: int, rs: RngState, *, is_reverse_test=False,
                       n_step=6, md_time=1.0, is_always_accept=False, integrator="force-gradient",
                       precision="fp64", reunit_interval=4):
    """hmc.pyx:190-216.  Returns (flag, delta_h)."""
    rs = rs.split(f"{traj}")
    geo = gf.geo
    gf0 = GaugeField(geo)
    gf0 @= gf
    gm = GaugeMomentum(geo)
    gm.set_rand(rs.split("set_rand_gauge_momentum"), 1.0)
    kw = dict(integrator=integrator, precision=precision, reunit_interval=reunit_interval)
    delta_h = run_hmc_evolve_pure_gauge(gm, gf0, ga, rs, n_step, md_time, **kw)
    if is_reverse_test:
        gm_r = GaugeMomentum(geo)
        gm_r @= gm
        gf0_r = GaugeField(geo)
        gf0_r @= gf0
        delta_h_rev = run_hmc_evolve_pure_gauge(gm_r, gf0_r, ga, rs, n_step, -md_time, **kw)
        gf0_r -= gf
        gf_diff_norm = gf0_r.qnorm()
        gf_norm = gf0.qnorm()
        run_hmc_pure_gauge.last_reverse = (delta_h + delta_h_rev, gf_diff_norm, gf_norm)
        assert gf_diff_norm <= 1e-12 * gf_norm or precision != "fp64"
    flag, accept_prob = metropolis_accept(delta_h, traj, rs.split("metropolis_accept"))
    if flag or is_always_accept:
        gf @= gf0
    return flag, delta_h


run_hmc_pure_gauge.last_reverse = None
