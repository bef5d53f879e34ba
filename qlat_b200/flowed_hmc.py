"""Flowed HMC with masked invertible flows (flowed-hmc.h / flowed-hmc.cpp;
driver examples-cpp/flowed-hmc/main.cpp), on the GPU in FP64.

HMC evolves U0; the physical field is U = flow(U0), a product of masked,
invertible smearing steps.  The action of U0 is S(flow(U0)) - ln det of the
flow's Jacobian, and the force propagates S's force back through the steps
with the log-determinants' force added at each step.
"""

from __future__ import annotations

import ctypes
import math
from dataclasses import dataclass

from . import _lib
from ._lib import call
from .field import F64, GaugeAction, GaugeField, GaugeMomentum, RngState


class _Step(ctypes.Structure):
    _fields_ = [("mask", ctypes.c_int32), ("mu", ctypes.c_int32), ("epsilon", ctypes.c_double),
                ("flow_size", ctypes.c_int32)]


@dataclass
class FlowStepInfo:
    """FlowStepInfo (flowed-hmc.h:26-41)."""
    mask: int
    mu: int
    epsilon: float
    flow_size: int = 1


class FlowInfo:
    """FlowInfo (flowed-hmc.h:43-45; qlat.fthmc.FlowInfo, fthmc.py:14-36): the
    flow steps in order."""

    def __init__(self, v=None):
        self.v = list(v or [])

    def add_flow(self, eo: int, mu: int, epsilon: float, flow_size: int = 1) -> None:
        """Append one step (fthmc.py:21-22): mask eo (1 or 2) of direction mu."""
        self.v.append(FlowStepInfo(int(eo), int(mu), float(epsilon), int(flow_size)))

    def add_rand_order_flow(self, rng: RngState, epsilon: float, *args) -> None:
        """Append mk_flow_info_step(rng, epsilon[, epsilon2]) (fthmc.py:24-31)."""
        if len(args) > 1:
            raise ValueError("add_rand_order_flow: at most one second epsilon")
        self.v.extend(mk_flow_info_step(rng, epsilon, *args).v)

    def show(self) -> str:
        return repr(self)

    def _c(self):
        arr = (_Step * max(1, len(self.v)))()
        for i, s in enumerate(self.v):
            arr[i] = _Step(int(s.mask), int(s.mu), float(s.epsilon), int(s.flow_size))
        return arr, len(self.v)

    def __repr__(self):
        return "\n".join(f"fi.v[{i}]: mask={s.mask}, mu={s.mu}, epsilon={s.epsilon:.4f}, flow_size={s.flow_size}."
                         for i, s in enumerate(self.v))


def mk_flow_info_step(rs: RngState, epsilon: float, epsilon2: float | None = None) -> FlowInfo:
    """mk_flow_info_step(rs, epsilon[, epsilon2]) (flowed-hmc.cpp:21-69)."""
    out = (_Step * 16)()
    n = ctypes.c_int32()
    call("qgb_flow_info_step", rs.c, float(epsilon), float(epsilon2 or 0.0), int(epsilon2 is not None), out,
         ctypes.byref(n))
    return FlowInfo(FlowStepInfo(out[i].mask, out[i].mu, out[i].epsilon, out[i].flow_size) for i in range(n.value))


def _flow(name, args):
    if len(args) == 3:  # (gf, gf0, fi): into gf, which may be gf0 itself
        gf, gf0, fi = args
        if gf._h is None:
            gf.init(gf0.geo)
        out = gf if gf is not gf0 else GaugeField(gf0.geo)
    elif len(args) == 2:  # (gf0, fi): a new field
        gf0, fi = args
        gf = out = GaugeField(gf0.geo)
    else:
        raise TypeError(f"{name}: (gf, gf0, fi) or (gf0, fi)")
    arr, n = fi._c()
    call("qgb_" + name, out.handle, gf0.handle, arr, n)
    if out is not gf:
        gf @= out
    return None if len(args) == 3 else gf


def gf_flow(*args):
    """gf_flow(gf, gf0, fi) (flowed-hmc.cpp:540-566; fthmc.py:38-42): gf = the
    flow of gf0.  gf_flow(gf0, fi) returns a new field."""
    return _flow("gf_flow", args)


def gf_flow_inv(*args):
    """gf_flow_inv(gf, gf1, fi) (flowed-hmc.cpp:568-594; fthmc.py:44-48): gf =
    the inverse flow of gf1.  gf_flow_inv(gf1, fi) returns a new field."""
    return _flow("gf_flow_inv", args)


def gf_flow_and_ln_det_node(gf0: GaugeField, fi: FlowInfo):
    """(flowed field, ln det of the flow's Jacobian) (flowed-hmc.cpp:1257-1299)."""
    gf = GaugeField(gf0.geo)
    arr, n = fi._c()
    ld = ctypes.c_double()
    call("qgb_gf_flow_and_ln_det_node", gf.handle, gf0.handle, arr, n, ctypes.byref(ld))
    return gf, ld.value


def gf_hamilton_flowed(gf0: GaugeField, ga: GaugeAction, fi: FlowInfo):
    """(flowed_action, ln_det) (flowed-hmc.cpp:1310-1321); the action of gf0 is
    flowed_action - ln_det."""
    arr, n = fi._c()
    a, ld = ctypes.c_double(), ctypes.c_double()
    call("qgb_gf_hamilton_flowed_node", gf0.handle, ga.beta(), ga.c1(), arr, n, ctypes.byref(a), ctypes.byref(ld))
    return a.value, ld.value


def gf_hamilton_flowed_node(gf0: GaugeField, ga: GaugeAction, fi: FlowInfo) -> float:
    """flowed-hmc.cpp:1301-1308"""
    a, ld = gf_hamilton_flowed(gf0, ga, fi)
    return a - ld


def set_gm_force_flowed(gm_force: GaugeMomentum, gf0: GaugeField, ga: GaugeAction, fi: FlowInfo,
                        *, with_det: bool = True) -> None:
    """set_gm_force_flowed (flowed-hmc.cpp:1500-1509); with_det=False gives the
    force of the flowed field propagated back without the determinant term."""
    arr, n = fi._c()
    call("qgb_set_gm_force_flowed", gm_force.handle, gf0.handle, ga.beta(), ga.c1(), arr, n, int(bool(with_det)))


def set_gm_force_flowed_no_det(gm_force: GaugeMomentum, gm_force_pre: GaugeMomentum, gf0: GaugeField,
                               fi: FlowInfo) -> None:
    """set_gm_force_flowed_no_det (flowed-hmc.cpp:1511-1520; fthmc.py:62-67):
    gm_force_pre, a force on the flowed field, propagated back to gf0 without
    the determinant term."""
    arr, n = fi._c()
    call("qgb_set_gm_force_flowed_no_det", gm_force.handle, gm_force_pre.handle, gf0.handle, arr, n)


def gm_evolve_fg_flowed(gm: GaugeMomentum, gf_init: GaugeField, ga: GaugeAction, fi: FlowInfo, fg_dt: float,
                        dt: float) -> None:
    """examples-cpp/flowed-hmc/main.cpp:gm_evolve_fg"""
    from .hmc import gf_evolve
    gf = gf_init.copy()
    gm_force = GaugeMomentum(gf.geo)
    set_gm_force_flowed(gm_force, gf, ga, fi)
    gf_evolve(gf, gm_force, fg_dt)
    set_gm_force_flowed(gm_force, gf, ga, fi)
    gm_force *= dt
    gm += gm_force


def run_hmc_evolve_flowed(gm: GaugeMomentum, gf: GaugeField, ga: GaugeAction, fi: FlowInfo, steps: int,
                          md_time: float = 1.0) -> float:
    """examples-cpp/flowed-hmc/main.cpp:run_hmc_evolve_flowed: force-gradient
    molecular dynamics of gf (the unflowed field) with the flowed action;
    returns delta_h."""
    from .hmc import gf_evolve, gm_hamilton_node, unitarize
    energy = gm_hamilton_node(gm) + gf_hamilton_flowed_node(gf, ga, fi)
    dt = md_time / steps
    lam = 0.5 * (1.0 - 1.0 / math.sqrt(3.0))
    theta = (2.0 - math.sqrt(3.0)) / 48.0
    ttheta = theta * dt * dt * dt
    gf_evolve(gf, gm, lam * dt)
    for i in range(steps):
        gm_evolve_fg_flowed(gm, gf, ga, fi, 4.0 * ttheta / dt, 0.5 * dt)
        gf_evolve(gf, gm, (1.0 - 2.0 * lam) * dt)
        gm_evolve_fg_flowed(gm, gf, ga, fi, 4.0 * ttheta / dt, 0.5 * dt)
        gf_evolve(gf, gm, (2.0 * lam if i < steps - 1 else lam) * dt)
    unitarize(gf)
    return gm_hamilton_node(gm) + gf_hamilton_flowed_node(gf, ga, fi) - energy


def run_flowed_hmc(gf: GaugeField, ga: GaugeAction, traj: int, rs: RngState, *, epsilon: float = 0.1,
                   epsilon2: float = -0.01, steps: int = 6, md_time: float = 1.0, always_accept_until: int = 20):
    """examples-cpp/flowed-hmc/main.cpp:run_hmc: flow steps from
    rs.split("mk_flow_info"), U0 = flow^-1(gf), momenta, molecular dynamics,
    the C++ Metropolis step, gf = flow(U0) if accepted (or traj <=
    always_accept_until).  Returns (flag, delta_h)."""
    from .hmc import metropolis_accept_cpp
    fi = mk_flow_info_step(rs.split("mk_flow_info"), epsilon, epsilon2)
    gf0 = gf_flow_inv(gf, fi)
    gm = GaugeMomentum(gf.geo)
    gm.set_rand(rs.split("set_rand_gauge_momentum"), 1.0)
    delta_h = run_hmc_evolve_flowed(gm, gf0, ga, fi, steps, md_time)
    flag, _ = metropolis_accept_cpp(delta_h, traj, rs.split("metropolis_accept"))
    if flag or traj <= always_accept_until:
        gf @= gf_flow(gf0, fi)
    return flag, delta_h
